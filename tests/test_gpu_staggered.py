"""Parity of the staggered-field step on the GPU (pamhd_gpu_staggered_*, through the C ABI) with
the CPU oracle (oracle/mode_s.hpp) and with the reference program's own outputs, periodic grids
(bounded ones: test_gpu_staggered_bounded.py).

Tolerance: the GPU solves faces with FMA contraction and Newton reciprocals, the oracle in the
reference's operation order; the cell and face updates are written in the oracle's order without
contraction.  Per step every cell variable and face value agrees within 1e-12 of that field's
largest magnitude (vectors as a whole), the bar of the cell-centred parity tests.
"""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states
from test_oracle_pin import STAGGERED_CASES, _load, _mhd_diff_ok

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12
GROUPS = ([0], [1, 2, 3], [4], [5, 6, 7])


def state_err(a, b):
    a = a.reshape(8, -1)
    b = b.reshape(8, -1)
    worst = 0.0
    for rows in GROUPS:
        scale = max(np.abs(b[rows]).max(), 1e-300)
        worst = max(worst, float(np.abs(a[rows] - b[rows]).max() / scale))
    return worst


def face_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(port, n, solver, L, gamma=states.GAMMA_53, mu0=1.0, cfl=0.4):
    cfg = pg.Config(n=n, solver=solver, cell_length=L, adiabatic_index=gamma, vacuum_permeability=mu0,
                    time_step_factor=cfl)
    return pg.StaggeredContext(cfg), port.staggered_grid(po.make_cfg(n, solver, L, gamma, mu0, cfl))


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("shape", [(6, 5, 7), (1, 9, 12), (1, 1, 16)])
def test_steps_match_oracle(port, solver, shape):
    """3-D, 2-D and 1-D periodic grids (one-cell dimensions are their own neighbours), every solver:
    the priming step and 12 steps, state, faces and dt compared after every step."""
    L = (0.1, 0.12, 0.09)
    U, faces, _ = states.staggered_random(shape, L, np.random.default_rng(3))
    n = (shape[2], shape[1], shape[0])
    gpu, ora = pair(port, n, po.SOLVERS[solver], L)
    gpu.set_state(U, faces)
    ora.set_state(U, faces)
    for s in range(13):
        cap = 0.0 if s == 0 else 1.0
        dg = gpu.step(cap)
        do, flag, _, _ = ora.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300)
        Ug, Fg = gpu.get_state()
        Uo, Fo = ora.get_state()
        assert state_err(Ug, Uo) <= STEP_TOL, s
        assert face_err(Fg, Fo) <= STEP_TOL, s


@pytest.mark.parametrize("solver", ["rusanov", "hlld_athena"])
def test_tiled_grid_matches_oracle(port, solver):
    """A grid of 100 x 254 x 48 cells: the face solves run as 32 x 4 tiles marching several z planes
    each (five per block on a 148-SM GPU, the last chunk three), with partial tiles at the +x and +y
    edges; the priming step and two steps against the oracle.  The state is a random 24 x 127 x 50
    pattern repeated twice along each axis, whose periods fall across the tile edges."""
    L = (0.1, 0.12, 0.09)
    U, faces, _ = states.staggered_random((24, 127, 50), L, np.random.default_rng(11))
    U, faces = np.tile(U, (1, 2, 2, 2)), np.tile(faces, (1, 2, 2, 2))
    shape = U.shape[1:]
    n = (shape[2], shape[1], shape[0])
    gpu, ora = pair(port, n, po.SOLVERS[solver], L)
    gpu.set_state(U, faces)
    ora.set_state(U, faces)
    for s in range(3):
        cap = 0.0 if s == 0 else 1.0
        dg = gpu.step(cap)
        do, flag, _, _ = ora.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300)
        Ug, Fg = gpu.get_state()
        Uo, Fo = ora.get_state()
        assert state_err(Ug, Uo) <= STEP_TOL, s
        assert face_err(Fg, Fo) <= STEP_TOL, s


@pytest.mark.parametrize("case", list(STAGGERED_CASES))
def test_reproduces_reference_program_output(case, tmp_path):
    """The reference program's Alfven waves (Rusanov, CFL 0.5, t = 0 .. 1; with and without a
    background field), run through the C ABI as the program runs them: same step count and time,
    every cell within the reference's own comparison (tests/mhd/mhd_diff.py, 1e-15 defaults)."""
    g = _load("dc_goldens.npz")
    U0, faces, _, *bg = STAGGERED_CASES[case]()
    n = (U0.shape[3], U0.shape[2], U0.shape[1])
    cfg = pg.Config(n=n, solver=pg.RUSANOV, cell_length=tuple(g[case + "_cell_length"]),
                    adiabatic_index=float(g[case + "_gamma"]), vacuum_permeability=float(g[case + "_mu0"]),
                    time_step_factor=0.5)
    with pg.StaggeredContext(cfg) as ctx:
        ctx.set_state(U0, faces)
        if bg:
            ctx.set_background(bg[0])
        ctx.step(0.0)
        t, steps, t_end = 0.0, 0, float(g[case + "_time"])
        while t < t_end:
            t += ctx.step(t_end - t)
            steps += 1
        U, _ = ctx.get_state()
        # the result as the program saves it: a .dc file, read back
        path = str(tmp_path / f"mhd_{steps:09d}.dc")
        ctx.save_dc(path, steps, t)
        head, back = pg.read_dc(path)
        assert head["step"] == steps and head["time"] == t
        np.testing.assert_array_equal(back, U)
    assert steps == int(g[case + "_step"]) and t == t_end
    out = U.reshape(8, -1)
    ref = g[case + "_state"]
    assert _mhd_diff_ok(out, ref)
    assert np.abs(out - ref).max() <= 2e-15


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_background_field_matches_oracle(port, solver):
    """A background field that varies over the faces (a uniform field plus a random one), every
    solver (Rusanov and HLL use it, HLLD and Roe ignore it, as the reference's): per step against
    the oracle."""
    L = (0.1, 0.12, 0.09)
    shape = (5, 6, 7)
    rng = np.random.default_rng(8)
    U, faces, _ = states.staggered_random(shape, L, rng)
    bg = rng.normal(0, 0.05, (3, 3) + shape) + np.array([0.2, 0.4, -0.3])[None, :, None, None, None]
    gpu, ora = pair(port, (7, 6, 5), po.SOLVERS[solver], L)
    gpu.set_state(U, faces)
    ora.set_state(U, faces)
    gpu.set_background(bg)
    ora.set_background(bg)
    for s in range(8):
        cap = 0.0 if s == 0 else 1.0
        dg = gpu.step(cap)
        do, flag, _, _ = ora.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300)
        Ug, Fg = gpu.get_state()
        Uo, Fo = ora.get_state()
        assert state_err(Ug, Uo) <= STEP_TOL, s
        assert face_err(Fg, Fo) <= STEP_TOL, s


def test_batched_steps_equal_single_steps(port):
    """steps(n, t_end) (launches only, the cap t_end - t read on the device) computes the same
    bits as step-by-step calls, stops at t_end and leaves the state unchanged afterwards."""
    U, faces, L = states.staggered_random((4, 6, 8), (0.1, 0.1, 0.1), np.random.default_rng(5))
    cfg = pg.Config(n=(8, 6, 4), solver=pg.HLLD, cell_length=L, time_step_factor=0.4)
    a, b = pg.StaggeredContext(cfg), pg.StaggeredContext(cfg)
    a.set_state(U, faces)
    b.set_state(U, faces)
    a.step(0.0)
    b.step(0.0)
    t_end = 0.05
    t = 0.0
    n = 0
    while t < t_end:
        t += a.step(t_end - t)
        n += 1
    b.steps(n + 5, t_end)
    b.sync()
    tb, nb, _ = b.time()
    assert tb == t and nb == n + 1   # the priming step counts
    Ua, Fa = a.get_state()
    Ub, Fb = np.zeros_like(Ua), np.zeros_like(Fa)
    assert b.get_state(out=(Ub, Fb))[0] is Ub   # the caller's arrays, filled in place
    assert np.array_equal(Ua, Ub) and np.array_equal(Fa, Fb)
    with pytest.raises(ValueError):
        b.get_state(out=(Ub[:, ::2], Fb))


def test_divergence_is_kept():
    U, faces, L = states.staggered_random((8, 8, 8), (0.1, 0.1, 0.1), np.random.default_rng(9))
    cfg = pg.Config(n=(8, 8, 8), solver=pg.HLLD, cell_length=L, time_step_factor=0.4)
    with pg.StaggeredContext(cfg) as ctx:
        ctx.set_state(U, faces)
        ctx.step(0.0)
        ctx.steps(40, 1e30)
        ctx.sync()
        _, F = ctx.get_state()
    div0 = states.face_divergence(faces, L)
    assert np.abs(states.face_divergence(F, L) - div0).max() <= 1e-12 * np.abs(F).max() / 0.1


def test_failure_reports_oracle_face_and_keeps_state(port):
    """A cell with negative pressure: the step fails with the oracle's flag at the oracle's first
    failing face, and the state is left as it was."""
    L = (0.1, 0.1, 0.1)
    U, faces, _ = states.staggered_random((4, 4, 4), L, np.random.default_rng(1))
    U[4, 2, 1, 3] = 0.01   # total energy below the magnetic energy
    gpu, ora = pair(port, (4, 4, 4), pg.HLL, L)
    gpu.set_state(U, faces)
    ora.set_state(U, faces)
    dt, flag, cell, d = ora.step(0.0)
    assert flag != 0
    with pytest.raises(pg.PhysicsError) as e:
        gpu.step(0.0)
    assert e.value.flags == flag and tuple(e.value.cell) == cell and e.value.direction == d
    Ug, Fg = gpu.get_state()
    assert np.array_equal(Ug, U) and np.array_equal(Fg, faces)


def test_rejects_invalid_sides():
    """Periodic on one side only, a bounded dimension of one cell, two VALUE sides, and a background
    field on a bounded grid are refused."""
    C, V = pg.BC_COPY, pg.BC_VALUE
    v = [1.0, 0, 0, 0, 2.0, 0, 0, 0]
    bad = [
        dict(n=(8, 8, 4), bc_lo=(C, 0, 0), bc_hi=(0, 0, 0)),
        dict(n=(8, 8, 1), bc_lo=(C, 0, C), bc_hi=(C, 0, C)),
        dict(n=(8, 8, 4), bc_lo=(V, V, 0), bc_hi=(C, C, 0), value_lo=[v, v, None]),
    ]
    for kw in bad:
        with pytest.raises(pg.PamhdError) as e:
            pg.StaggeredContext(pg.Config(solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1), **kw))
        assert e.value.code == pg.ERR_ARGUMENT
    cfg = pg.Config(n=(8, 8, 1), solver=pg.HLL, cell_length=(0.1, 0.1, 0.1), bc_lo=(C, 0, 0), bc_hi=(C, 0, 0))
    with pg.StaggeredContext(cfg) as ctx:
        with pytest.raises(pg.PamhdError) as e:
            ctx.set_background(np.zeros((3, 3, 1, 8, 8)))
        assert e.value.code == pg.ERR_ARGUMENT
