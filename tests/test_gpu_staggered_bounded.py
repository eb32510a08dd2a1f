"""The staggered-field step on bounded grids (pamhd_gpu_staggered_* with COPY and VALUE sides: a
layer of boundary cells as the reference's solar-wind box) against the CPU oracle
(oracle/mode_s.hpp), per step, every solver.

Tolerance as the periodic staggered tests: the GPU solves faces with FMA contraction and Newton
reciprocals, the oracle in the reference's operation order; the cell, face, copy-sync and layer
updates are written in the oracle's order without contraction.  Per step every cell variable and
face value agrees within 1e-12 of that field's largest magnitude (vectors as a whole).
"""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12
GROUPS = ([0], [1, 2, 3], [4], [5, 6, 7])
C, V, P = pg.BC_COPY, pg.BC_VALUE, pg.BC_PERIODIC


def state_err(a, b):
    a = a.reshape(8, -1)
    b = b.reshape(8, -1)
    worst = 0.0
    for rows in GROUPS:
        scale = max(np.abs(b[rows]).max(), 1e-300)
        worst = max(worst, float(np.abs(a[rows] - b[rows]).max() / scale))
    return worst


def faces_err(a, b):
    return max(float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)) for x, y in zip(a, b))


def bounded_faces(faces, cfg):
    """The periodic face field of states.staggered_random with the high wall of each bounded
    dimension appended (the face that wraps around to the first): divergence-free as before."""
    out = []
    for d, shape in enumerate(pg.staggered_face_shapes(cfg)):
        f = faces[d]
        if shape != f.shape:
            ax = 2 - d
            first = np.take(f, [0], axis=ax)
            f = np.concatenate([f, first], axis=ax)
        out.append(np.ascontiguousarray(f))
    return out


def make_pair(port, n, solver, L, bc_lo, bc_hi, value=None, cfl=0.4):
    vlo = [None] * 3
    vhi = [None] * 3
    for d in range(3):
        if bc_lo[d] == V:
            vlo[d] = value
        if bc_hi[d] == V:
            vhi[d] = value
    cfg = pg.Config(n=n, solver=solver, cell_length=L, time_step_factor=cfl, bc_lo=bc_lo, bc_hi=bc_hi,
                    value_lo=vlo, value_hi=vhi)
    ocfg = po.make_cfg(n, solver, L, states.GAMMA_53, 1.0, cfl, bc_lo, bc_hi,
                       value_lo=[v if v is not None else [0.0] * 8 for v in vlo],
                       value_hi=[v if v is not None else [0.0] * 8 for v in vhi])
    return cfg, pg.StaggeredContext(cfg), port.staggered_grid(ocfg)


def inflow_of(U):
    """A VALUE state near the grid's mean state: the first cell with its density raised."""
    v = U[:, 0, 0, 0].copy()
    v[0] *= 1.3
    v[1:4] *= 1.3
    return v


CASES = {
    # name: (n, bc_lo, bc_hi)
    "copy_every_side": ((6, 5, 7), (C, C, C), (C, C, C)),
    "inflow_x_copy_y_periodic_z": ((7, 6, 5), (V, C, P), (C, C, P)),
    "inflow_high_y_2d": ((12, 9, 1), (C, C, P), (C, V, P)),
}


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("case", list(CASES))
def test_bounded_steps_match_oracle(port, solver, case):
    """The priming step and 10 steps (an inflow table switching state at the third step's time
    where the grid has a VALUE side): dt, state and faces after every step."""
    n, bc_lo, bc_hi = CASES[case]
    L = (0.1, 0.12, 0.09)
    shape = (n[2], n[1], n[0])
    U, faces, _ = states.staggered_random(shape, L, np.random.default_rng(5))
    value = inflow_of(U)
    cfg, gpu, ora = make_pair(port, n, po.SOLVERS[solver], L, bc_lo, bc_hi, value)
    F = bounded_faces(faces, cfg)
    gpu.set_state(U, F)
    ora.set_state(U, F)
    if V in bc_lo or V in bc_hi:
        d = (list(bc_lo) + list(bc_hi)).index(V) % 3
        side = 0 if V in bc_lo else 1
        later = value.copy()
        later[0] *= 0.9
        later[1:4] *= 1.1
        for g in (gpu, ora):
            g.set_inflow(d, side, [0.02], [value, later])
    for s in range(11):
        cap = 0.0 if s == 0 else 1.0
        dg = gpu.step(cap)
        do, flag, _, _ = ora.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300), s
        Ug, Fg = gpu.get_state()
        Uo, Fo = ora.get_state()
        assert state_err(Ug, Uo) <= STEP_TOL, s
        assert faces_err(Fg, Fo) <= STEP_TOL, s
    gpu.close()


def test_uniform_state_is_kept():
    """A uniform state whose VALUE side holds the same state stays uniform (to round-off of the
    energy's recomputation from pressure)."""
    n = (6, 5, 4)
    U = np.zeros((8, n[2], n[1], n[0]))
    u = np.array([1.0, 0.3, -0.1, 0.05, 2.0, 0.5, 0.2, -0.3])
    U[:] = u[:, None, None, None]
    cfg = pg.Config(n=n, solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1), time_step_factor=0.4,
                    bc_lo=(V, C, C), bc_hi=(C, C, C), value_lo=[list(u), None, None])
    with pg.StaggeredContext(cfg) as ctx:
        F = [np.full(s, u[5 + d]) for d, s in enumerate(pg.staggered_face_shapes(cfg))]
        ctx.set_state(U, F)
        ctx.step(0.0)
        ctx.steps(20, 1e30)
        ctx.sync()
        Ug, Fg = ctx.get_state()
    assert np.abs(Ug - U).max() <= 1e-14 * 4
    assert max(np.abs(Fg[d] - F[d]).max() for d in range(3)) <= 1e-15


def test_steps_equal_single_steps(port):
    """steps(n) on the context's stream gives the bits of n single steps."""
    n, bc_lo, bc_hi = CASES["inflow_x_copy_y_periodic_z"]
    L = (0.1, 0.12, 0.09)
    U, faces, _ = states.staggered_random((n[2], n[1], n[0]), L, np.random.default_rng(8))
    value = inflow_of(U)
    cfg, a, _ = make_pair(port, n, pg.HLL, L, bc_lo, bc_hi, value)
    b = pg.StaggeredContext(cfg)
    F = bounded_faces(faces, cfg)
    for g in (a, b):
        g.set_state(U, F)
        g.step(0.0)
    for _ in range(7):
        a.step(1e30)
    b.steps(7, 1e30)
    b.sync()
    Ua, Fa = a.get_state()
    Ub, Fb = b.get_state()
    assert np.array_equal(Ua, Ub)
    assert all(np.array_equal(x, y) for x, y in zip(Fa, Fb))
    a.close()
    b.close()


def test_failure_in_the_layer_reports_the_oracle_face(port):
    """An inflow state of negative pressure: the first failing face lies in the boundary layer
    (layer coordinate -1), reported as the oracle reports it, and the state is kept."""
    n = (5, 4, 4)
    L = (0.1, 0.1, 0.1)
    U, faces, _ = states.staggered_random((n[2], n[1], n[0]), L, np.random.default_rng(2))
    bad = U[:, 0, 0, 0].copy()
    bad[4] = 0.01   # total energy below the magnetic energy
    cfg, gpu, ora = make_pair(port, n, pg.HLL, L, (V, C, C), (C, C, C), bad)
    F = bounded_faces(faces, cfg)
    gpu.set_state(U, F)
    ora.set_state(U, F)
    # set_state filled the layer: the inflow plane's inner cells took its normal field
    U0, F0 = gpu.get_state()
    dt, flag, cell, d = ora.step(0.0)
    assert flag != 0 and cell[0] == -1
    with pytest.raises(pg.PhysicsError) as e:
        gpu.step(0.0)
    assert e.value.flags == flag and tuple(e.value.cell) == cell and e.value.direction == d
    Ug, Fg = gpu.get_state()
    assert np.array_equal(Ug, U0) and all(np.array_equal(x, y) for x, y in zip(Fg, F0))
    gpu.close()


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena", "hlld_athena", "roe_athena"])
@pytest.mark.parametrize("name", ["periodic_3d", "copy_box", "wind_minus_x", "wind_plus_y_2d"])
def test_matches_reference_step(name, solver):
    """The GPU against the reference's own staggered step (the solar-wind box's loop, compiled
    unchanged; committed outputs, see test_staggered_ref_pin.py): the priming step and five steps,
    state and faces within 1e-12, dt within 1e-13."""
    import test_staggered_ref_pin as R
    U, F, dts, value = R.golden(name, solver)
    n, bc_lo, bc_hi = R.CASES[name]
    vlo = [list(value) if k == V else None for k in bc_lo]
    vhi = [list(value) if k == V else None for k in bc_hi]
    cfg = pg.Config(n=n, solver=R.SOLVERS[solver], cell_length=R.LENGTHS, time_step_factor=0.4, bc_lo=bc_lo,
                    bc_hi=bc_hi, value_lo=vlo, value_hi=vhi)
    U0, F0 = R.case_input(name)
    with pg.StaggeredContext(cfg) as ctx:
        ctx.set_state(U0, F0)
        got = [ctx.step(0.0 if s == 0 else 1e300) for s in range(R.STEPS)]
        Ug, Fg = ctx.get_state()
    assert np.abs(np.array(got) - dts).max() <= 1e-13 * dts.max()
    assert state_err(Ug, U) <= STEP_TOL
    assert faces_err(list(Fg), F) <= STEP_TOL


@pytest.mark.parametrize("solver", ["hll_athena", "hlld_athena"])
def test_many_blocks_match_oracle(port, solver):
    """A 44 x 38 x 30 box (about 55,000 cells with the layer: every kernel's grid-stride loop over
    many blocks, and a 40 x 32 inflow plane over several blocks) with inflow on +z and COPY
    elsewhere: the priming step and three steps against the oracle."""
    n, bc_lo, bc_hi = (44, 38, 30), (C, C, C), (C, C, V)
    L = (0.1, 0.12, 0.09)
    U, faces, _ = states.staggered_random((n[2], n[1], n[0]), L, np.random.default_rng(13))
    value = inflow_of(U)
    cfg, gpu, ora = make_pair(port, n, po.SOLVERS[solver], L, bc_lo, bc_hi, value)
    F = bounded_faces(faces, cfg)
    gpu.set_state(U, F)
    ora.set_state(U, F)
    for s in range(4):
        cap = 0.0 if s == 0 else 1.0
        dg = gpu.step(cap)
        do, flag, _, _ = ora.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300), s
        Ug, Fg = gpu.get_state()
        Uo, Fo = ora.get_state()
        assert state_err(Ug, Uo) <= STEP_TOL, s
        assert faces_err(Fg, Fo) <= STEP_TOL, s
    gpu.close()
