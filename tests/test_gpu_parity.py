"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerance: the GPU computes in FP64 with FMA contraction and reciprocals,
the oracle in the reference's exact operation order, so results agree to
round-off.  Per step the bar is a relative state error <= 1e-12: for every
variable, |gpu - oracle| <= 1e-12 * max(|oracle| over that variable's
field) per cell (a field-normwise relative error; momentum and field
components pass through zero, where a cellwise ratio is meaningless).
Face fluxes use the same bar per face: |gpu - oracle| <= 1e-12 * max over
the face's eight flux components.
"""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12


def field_err(a, b):
    """max over variables of max|a - b| / max|b| (b = oracle)."""
    a = a.reshape(8, -1)
    b = b.reshape(8, -1)
    scale = np.abs(b).max(axis=1)
    scale[scale == 0] = 1.0
    return float((np.abs(a - b).max(axis=1) / scale).max())


def pair(port, n, solver, lengths, gamma, mu0, cfl, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0),
         value_lo=None, value_hi=None):
    cfg = pg.Config(n=n, solver=solver, cell_length=lengths, adiabatic_index=gamma, vacuum_permeability=mu0,
                    time_step_factor=cfl, bc_lo=bc_lo, bc_hi=bc_hi,
                    value_lo=value_lo or [None] * 3, value_hi=value_hi or [None] * 3)
    ocfg = po.make_cfg(n, solver, lengths, gamma, mu0, cfl, bc_lo, bc_hi, value_lo, value_hi)
    return pg.Context(cfg), port.grid(ocfg, threads=8)


# ---------------------------------------------------------------- solver level

@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_face_flux_matches_oracle(port, solver):
    rng = np.random.default_rng(11)
    a, b = states.nearby_face_states(20000, rng)
    c = states.random_face_states(20000, rng)
    d = states.random_face_states(20000, rng)
    e, f = states.edge_case_face_states()
    neg = np.vstack([a, c, e])
    pos = np.vstack([b, d, f])
    sid = po.SOLVERS[solver]
    for mu0, bg in ((1.0, None), (1.0, rng.normal(0, 0.3, (neg.shape[0], 3))), (4e-7 * np.pi, None)):
        scale = np.ones(8)
        if mu0 != 1.0:
            scale[5:8] = np.sqrt(mu0)
        n_, p_ = neg * scale, pos * scale
        fo, so, go = port.face_flux(sid, n_, p_, bg, 5 / 3, mu0)
        fg, sg, gg = pg.face_flux(sid, n_, p_, bg, 5 / 3, mu0)
        # every face the reference rejects is rejected with the same class of error
        assert np.array_equal(gg != 0, go != 0)
        assert np.array_equal(gg[go != 0], go[go != 0])
        ok = go == 0
        row = np.abs(fo[ok]).max(axis=1, keepdims=True)
        row[row == 0] = 1.0
        assert (np.abs(fg[ok] - fo[ok]) / row).max() <= STEP_TOL
        assert (np.abs(sg[ok] - so[ok]) / np.maximum(so[ok], 1e-300)).max() <= STEP_TOL


# ---------------------------------------------------------------- one step from identical inputs

CASES = {
    "periodic3d": dict(n=(12, 10, 9), lengths=(1 / 12, 1 / 10, 1 / 9), gamma=5 / 3, mu0=1.0, cfl=0.4),
    "periodic3d_wide": dict(n=(70, 19, 11), lengths=(0.01, 0.02, 0.03), gamma=5 / 3, mu0=1.0, cfl=0.4),
    "orszag_tang64": dict(n=(64, 64, 1), lengths=(1 / 64, 1 / 64, 1.0), gamma=5 / 3, mu0=1.0, cfl=0.4),
    "briowu200": dict(n=(200, 1, 1), lengths=(1 / 200, 1.0, 1.0), gamma=2.0, mu0=1.0, cfl=0.5,
                      bc_lo=(1, 0, 0), bc_hi=(1, 0, 0)),
}


def initial_state(key, rng):
    c = CASES[key]
    nx, ny, nz = c["n"]
    if key.startswith("orszag"):
        return states.orszag_tang(nx)
    if key.startswith("briowu"):
        return states.brio_wu(nx)
    return states.smooth_3d((nz, ny, nx), rng, amp=0.15)


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("key", list(CASES))
def test_one_step_matches_oracle(port, key, solver):
    rng = np.random.default_rng(21)
    U0 = initial_state(key, rng)
    c = dict(CASES[key])
    gpu, ora = pair(port, c.pop("n"), po.SOLVERS[solver], c.pop("lengths"), c.pop("gamma"), c.pop("mu0"),
                    c.pop("cfl"), **c)
    gpu.set_state(U0)
    ora.set_state(U0)
    # priming step: dt = 0, state unchanged, speeds recorded (tests/mhd/test.cpp:462)
    assert gpu.step(1.0) == 0.0
    assert ora.step(1.0)[0] == 0.0
    np.testing.assert_array_equal(gpu.get_state(), U0)
    # one real step from identical inputs
    dg = gpu.step(1.0)
    do, flag, _, _ = ora.step(1.0)
    assert flag == 0
    assert abs(dg - do) <= STEP_TOL * do
    assert field_err(gpu.get_state(), ora.get_state()) <= STEP_TOL


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_bounded_grid_matches_oracle(port, solver):
    """COPY and VALUE sides plus a periodic one: ghost refresh and the boundary-layer speeds."""
    rng = np.random.default_rng(5)
    U0 = states.smooth_3d((7, 9, 11), rng, amp=0.1)
    inflow = np.array([1.2, 0.3 * 1.2, 0.2 * 1.2, 0.0,
                       states.energy(1.2, np.array([[0.3], [0.2], [0.0]]), 0.7,
                                     np.array([[0.4], [0.1], [-0.2]]), 5 / 3)[0], 0.4, 0.1, -0.2])
    gpu, ora = pair(port, (11, 9, 7), po.SOLVERS[solver], (0.09, 0.11, 0.13), 5 / 3, 1.0, 0.4,
                    bc_lo=(po.BC_VALUE, po.BC_COPY, po.BC_PERIODIC), bc_hi=(po.BC_COPY, po.BC_COPY, po.BC_PERIODIC),
                    value_lo=[inflow, None, None])
    gpu.set_state(U0)
    ora.set_state(U0)
    for step in range(6):
        dg = gpu.step(1.0)
        do, flag, _, _ = ora.step(1.0)
        assert flag == 0
        assert abs(dg - do) <= 1e-12 * max(do, 1e-300) or dg == do == 0.0
        assert field_err(gpu.get_state(), ora.get_state()) <= STEP_TOL * (1 + step)


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("layout", ["bounded3d", "yz_plane"])
def test_max_signal_matches_oracle(port, layout, solver):
    """pamhd_gpu_step's max_signal output: per dimension the largest face speed of the step (the
    maxima of the reference's Max_v, ghost-ghost faces of non-periodic sides included), equal to
    the oracle's to round-off, and the next step's dt follows from it by the CFL rule."""
    rng = np.random.default_rng(13)
    if layout == "bounded3d":
        n, lengths = (11, 9, 7), (0.09, 0.11, 0.13)
        U0 = states.smooth_3d((7, 9, 11), rng, amp=0.1)
        bc = dict(bc_lo=(po.BC_COPY, po.BC_COPY, po.BC_PERIODIC), bc_hi=(po.BC_COPY, po.BC_COPY, po.BC_PERIODIC))
    else:  # a y-z grid: the context relabels its axes, max_signal stays in the caller's axes
        n, lengths = (1, 16, 12), (1.0, 1 / 16, 1 / 12)
        U0 = states.smooth_3d((12, 16, 1), rng, amp=0.1)
        bc = {}
    gpu, ora = pair(port, n, po.SOLVERS[solver], lengths, 5 / 3, 1.0, 0.4, **bc)
    gpu.set_state(U0)
    ora.set_state(U0)
    prev = None
    for step in range(4):
        dg, sig = gpu.step_signal(1.0)
        do, flag, _, _ = ora.step(1.0)
        assert flag == 0
        so = ora.max_signal()
        assert np.all((sig == 0) == (so == 0))
        assert np.abs(sig - so).max() <= 1e-12 * so.max()
        if prev is not None:
            # the lagged rule: dt = min over dimensions of CFL * dx_d / max_signal_d of the last step
            expect = min(0.4 * lengths[d] / prev[d] for d in range(3) if prev[d] > 0)
            assert dg == min(expect, 1.0)
        prev = sig


# ---------------------------------------------------------------- trajectories

@pytest.mark.parametrize("solver", ["rusanov", "hll_athena", "hlld_athena"])
def test_orszag_tang_trajectory(port, solver):
    """50 steps of Orszag-Tang 64^2: dt history and state stay within round-off growth."""
    U0 = states.orszag_tang(64)
    c = dict(CASES["orszag_tang64"])
    gpu, ora = pair(port, c.pop("n"), po.SOLVERS[solver], c.pop("lengths"), c.pop("gamma"), c.pop("mu0"),
                    c.pop("cfl"))
    gpu.set_state(U0)
    ora.set_state(U0)
    t_o, dts_o = ora.run(0.0, 10.0, 50)
    gpu.steps(50, 10.0)
    gpu.sync()
    t_g, n_g, _ = gpu.time()
    dts_g = gpu.dt_history(50)
    assert n_g == 50
    np.testing.assert_allclose(dts_g, dts_o, rtol=1e-10, atol=0)
    assert abs(t_g - t_o) <= 1e-10 * t_o
    assert field_err(gpu.get_state(), ora.get_state()) <= 1e-9


def test_brio_wu_to_t_end(port):
    """Brio-Wu, 1000 cells, gamma 2, HLLD, CFL 0.5, copy boundaries, to t = 0.1."""
    U0 = states.brio_wu(1000)
    gpu, ora = pair(port, (1000, 1, 1), po.HLLD, (1e-3, 1.0, 1.0), 2.0, 1.0, 0.5,
                    bc_lo=(po.BC_COPY, 0, 0), bc_hi=(po.BC_COPY, 0, 0))
    gpu.set_state(U0)
    ora.set_state(U0)
    t_o, dts_o = ora.run(0.0, 0.1, 100000)
    gpu.steps(len(dts_o) + 5, 0.1)
    t_g, n_g, _ = gpu.time()
    assert t_o == pytest.approx(0.1, abs=0) or abs(t_o - 0.1) < 1e-15
    assert abs(t_g - t_o) <= 1e-13
    dts_g = gpu.dt_history(n_g)
    np.testing.assert_allclose(dts_g[: len(dts_o)], dts_o, rtol=1e-9)
    assert field_err(gpu.get_state(), ora.get_state()) <= 1e-8


# ---------------------------------------------------------------- properties at any size

def test_graph_steps_equal_single_steps():
    rng = np.random.default_rng(8)
    U0 = states.smooth_3d((20, 24, 40), rng)
    cfg = pg.Config(n=(40, 24, 20), solver=pg.HLLD, cell_length=(0.025, 0.04, 0.05), time_step_factor=0.4)
    a, b = pg.Context(cfg), pg.Context(cfg)
    a.set_state(U0)
    b.set_state(U0)
    for _ in range(14):
        a.step(1e9)
    b.steps(14, 1e9)
    b.sync()
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    np.testing.assert_array_equal(a.dt_history(14), b.dt_history(14))


def test_translation_invariance_bitwise():
    """Shifting a periodic initial state by whole cells shifts the solution bit for bit:
    every face is solved by the same arithmetic wherever it sits in the tiling."""
    rng = np.random.default_rng(9)
    U0 = states.smooth_3d((16, 20, 72), rng)
    cfg = pg.Config(n=(72, 20, 16), solver=pg.HLLD, cell_length=(0.02, 0.05, 0.06), time_step_factor=0.4)
    a, b = pg.Context(cfg), pg.Context(cfg)
    shift = (5, 7, 13)  # z, y, x
    a.set_state(U0)
    b.set_state(np.roll(U0, shift, axis=(1, 2, 3)))
    a.steps(7, 1e9)
    b.steps(7, 1e9)
    np.testing.assert_array_equal(np.roll(a.get_state(), shift, axis=(1, 2, 3)), b.get_state())


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_conservation_on_periodic_grid(solver):
    rng = np.random.default_rng(10)
    U0 = states.smooth_3d((24, 32, 40), rng)
    cfg = pg.Config(n=(40, 32, 24), solver=po.SOLVERS[solver], cell_length=(0.025, 0.03, 0.04),
                    time_step_factor=0.4)
    g = pg.Context(cfg)
    g.set_state(U0)
    t0 = g.totals()
    g.steps(20, 1e9)
    t1 = g.totals()
    absum = np.abs(U0).reshape(8, -1).sum(axis=1) * 0.025 * 0.03 * 0.04
    assert np.all(np.abs(t1 - t0) <= 1e-13 * absum)


def test_invalid_state_reported_like_oracle(port):
    rng = np.random.default_rng(5)
    U0 = states.smooth_3d((6, 5, 40), rng)
    U0[4, 3, 2, 17] = 0.0  # negative pressure in cell x=17, y=2, z=3
    gpu, ora = pair(port, (40, 5, 6), po.HLLD, (0.025, 0.2, 0.16), 5 / 3, 1.0, 0.4)
    gpu.set_state(U0)
    ora.set_state(U0)
    _, flag, cell, d = ora.step(0.0)
    with pytest.raises(pg.PhysicsError) as e:
        gpu.step(0.0)
    assert e.value.flags == flag == pg.FLAG_PRESSURE
    assert e.value.cell == cell and e.value.direction == d


def test_time_capped_at_t_end():
    U0 = states.orszag_tang(32)
    cfg = pg.Config(n=(32, 32, 1), solver=pg.HLL, cell_length=(1 / 32, 1 / 32, 1.0), time_step_factor=0.4)
    g = pg.Context(cfg)
    g.set_state(U0)
    g.steps(400, 0.05)
    t, n, _ = g.time()
    assert t == 0.05 and n == 400


def test_blast_positivity_failure_matches_oracle(port):
    """The 64^3 magnetised blast loses positivity in the reference scheme (first-order HLLD, cell-
    centred field): the GPU must stop at the same step, on the same face, with the same error."""
    n = 64
    U0 = states.blast_wave(n)
    gpu, ora = pair(port, (n, n, n), po.HLLD, (1 / n,) * 3, 5 / 3, 1.0, 0.4)
    gpu.set_state(U0)
    ora.set_state(U0)
    fail_o = fail_g = None
    for step in range(120):
        do, flag, cell, d = ora.step(1e30)
        if flag:
            fail_o = (step, flag, cell, d)
            break
        dg = gpu.step(1e30)
        assert abs(dg - do) <= 1e-10 * max(do, 1e-300) or dg == do == 0.0
    assert fail_o is not None
    try:
        gpu.step(1e30)
    except pg.PhysicsError as e:
        fail_g = (fail_o[0], e.flags, e.cell, e.direction)
    assert fail_g == fail_o


def test_steps_after_a_failure_hold_the_grid():
    """The reference aborts in the step whose face fails (mhd/solve.hpp:156-181): here that step
    completes and every later one leaves the grid as it left it.  The 64^3 blast loses positivity
    after some steps; then steps one at a time, in a CUDA graph and split in two parts keep the
    state, the time, the step count and the dt history, and report the error again; set_state
    starts over."""
    n = 64
    U0 = states.blast_wave(n)
    cfg = pg.Config(n=(n, n, n), solver=pg.HLLD, cell_length=(1 / n,) * 3, time_step_factor=0.4)
    g = pg.Context(cfg)
    g.set_state(U0)
    failed = None
    for step in range(120):
        try:
            g.step(1e30)
        except pg.PhysicsError as e:
            failed = (step, e.flags, e.cell, e.direction)
            break
    assert failed is not None and failed[0] > 5
    held = g.get_state()
    t, count, _ = g.time()
    assert count == failed[0] + 1
    history = g.dt_history(200)
    assert len(history) == count and history[-1] > 0.0
    for _ in range(2):
        with pytest.raises(pg.PhysicsError) as e:
            g.step(1e30)
        assert (e.value.flags, e.value.cell, e.value.direction) == failed[1:]
    g.steps(13, 1e30)
    with pytest.raises(pg.PhysicsError):
        g.sync()
    g.step_part(1, 1e30)
    g.step_part(2, 1e30)
    with pytest.raises(pg.PhysicsError):
        g.sync()
    np.testing.assert_array_equal(g.get_state(), held)
    assert g.time() == (t, count, 0.0)
    np.testing.assert_array_equal(g.dt_history(200), history)
    g.set_state(U0)
    assert g.step(1e30) == 0.0 and g.step(1e30) == history[1]
    assert g.status()[0] == 0


@pytest.mark.parametrize("count", [0, 1, 33, 257])
def test_face_flux_empty_and_ragged_batches(port, count):
    """Batches of no face, one face and counts that leave partial blocks: the same results as
    the oracle face by face (an empty batch is a valid call that does nothing)."""
    rng = np.random.default_rng(12)
    a, b = states.nearby_face_states(max(count, 1), rng)
    a, b = a[:count], b[:count]
    fo, so, go = port.face_flux(po.HLLD, a, b, None, 5 / 3, 1.0)
    fg, sg, gg = pg.face_flux(po.HLLD, a, b, None, 5 / 3, 1.0)
    assert fg.shape == (count, 8) and sg.shape == (count,) and gg.shape == (count,)
    assert np.array_equal(gg, go)
    if count:
        row = np.maximum(np.abs(fo).max(axis=1, keepdims=True), 1e-300)
        assert (np.abs(fg - fo) / row).max() <= STEP_TOL
        assert (np.abs(sg - so) / np.maximum(so, 1e-300)).max() <= STEP_TOL


# ---------------------------------------------------------------- the configured workloads

def test_blast_256_configured(port):
    """The headline workload at its size: the 256^3 magnetised blast, HLLD, CFL 0.4, periodic.
    The priming step and two steps against the oracle (on every host thread) at the per-step bar;
    then size-independent properties over 20 more steps: the conserved totals stay within
    round-off, and a copy of the state shifted by whole cells stays the shifted solution bit for
    bit."""
    import os
    n = 256
    U0 = states.blast_wave(n)
    gpu, _ = pair(port, (n, n, n), po.HLLD, (1 / n,) * 3, 5 / 3, 1.0, 0.4)
    ora = port.grid(po.make_cfg((n, n, n), po.HLLD, (1 / n,) * 3, 5 / 3, 1.0, 0.4),
                    threads=max(1, len(os.sched_getaffinity(0))))
    gpu.set_state(U0)
    ora.set_state(U0)
    for s in range(3):
        cap = 0.0 if s == 0 else 1.0
        do, flag, _, _ = ora.step(cap)
        dg = gpu.step(cap)
        assert flag == 0
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300)
        assert field_err(gpu.get_state(), ora.get_state()) <= STEP_TOL, s
    del ora
    shift = (17, 5, 200)   # z, y, x
    b = pg.Context(gpu.cfg)
    U3 = gpu.get_state()
    b.set_state(np.roll(U3, shift, axis=(1, 2, 3)))
    gpu.set_state(U3)
    t0 = gpu.totals()
    gpu.steps(20, 1e9)
    b.steps(20, 1e9)
    t1 = gpu.totals()
    Uf = gpu.get_state()
    # round-off of 16.7 M cell updates a step (random signs): about sqrt(N) eps of the sum of |U|
    absum = np.maximum(np.abs(U3).reshape(8, -1).sum(axis=1), np.abs(Uf).reshape(8, -1).sum(axis=1)) / n ** 3
    assert np.all(np.abs(t1 - t0) <= 1e-11 * absum)
    np.testing.assert_array_equal(np.roll(Uf, shift, axis=(1, 2, 3)), b.get_state())


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_brio_wu_configured_every_solver(port, solver):
    """The shock-tube workload with each solver: 1000 cells on [0, 1], gamma 2, CFL 0.5, copy
    boundaries, to t = 0.1; same step count, dt history within 1e-9, state within 1e-8."""
    U0 = states.brio_wu(1000)
    gpu, ora = pair(port, (1000, 1, 1), po.SOLVERS[solver], (1e-3, 1.0, 1.0), 2.0, 1.0, 0.5,
                    bc_lo=(po.BC_COPY, 0, 0), bc_hi=(po.BC_COPY, 0, 0))
    gpu.set_state(U0)
    ora.set_state(U0)
    t_o, dts_o = ora.run(0.0, 0.1, 100000)
    gpu.steps(len(dts_o) + 5, 0.1)
    gpu.sync()
    t_g, n_g, _ = gpu.time()
    assert abs(t_g - t_o) <= 1e-13
    dts_g = gpu.dt_history(n_g)
    np.testing.assert_allclose(dts_g[: len(dts_o)], dts_o, rtol=1e-9)
    assert np.all(dts_g[len(dts_o):] == 0.0)
    assert field_err(gpu.get_state(), ora.get_state()) <= 1e-8


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_orszag_tang_512_configured(port, solver):
    """The 2-D workload at its size: Orszag-Tang 512^2, periodic, gamma 5/3, CFL 0.4, up to 1000
    steps with each solver.  Every 50 steps both are restarted from the GPU's state (a priming
    step, then one step from identical inputs must agree to 1e-12, the per-step bar); in between
    they run independently (dt within 1e-9).  The reference scheme loses positivity on this
    problem near t = 0.104 for some solvers: the GPU must stop at the same step and face, with
    the same error class, as the oracle, or both run all the steps."""
    n = 512
    U0 = states.orszag_tang(n)
    gpu, ora = pair(port, (n, n, 1), po.SOLVERS[solver], (1 / n, 1 / n, 1.0), 5 / 3, 1.0, 0.4)
    gpu.set_state(U0)
    ora.set_state(U0)
    fail_g = fail_o = None
    for s in range(1001):
        if s % 50 == 0 and s > 0:
            U = gpu.get_state()
            gpu.set_state(U)
            ora.set_state(U)
            assert gpu.step(1.0) == 0.0 and ora.step(1.0)[0] == 0.0
            checked = True
        else:
            checked = False
        try:
            dg = gpu.step(1.0)
        except pg.PhysicsError as e:
            fail_g = (s, tuple(e.cell), e.direction, e.flags)
        do, flag, cell, d = ora.step(1.0)
        if flag:
            fail_o = (s, tuple(cell), d, flag)
        if fail_g or fail_o:
            break
        assert abs(dg - do) <= 1e-9 * max(do, 1e-300) or dg == do == 0.0
        if checked:
            assert abs(dg - do) <= STEP_TOL * do, s
            assert field_err(gpu.get_state(), ora.get_state()) <= STEP_TOL, s
    # the same step and first failing face; the GPU's flags (all failures of the step, OR-ed)
    # include the oracle's (the first face's)
    assert (fail_g is None) == (fail_o is None), (fail_g, fail_o)
    if fail_g is not None:
        assert fail_g[:3] == fail_o[:3], (fail_g, fail_o)
        assert fail_g[3] & fail_o[3], (fail_g, fail_o)


@pytest.mark.parametrize("case,vx", [("da_px", 1.0), ("da_mx", -1.0)])
def test_reproduces_reference_program_output(case, vx):
    """The reference program's own output (tests/mhd/reference/hydrodynamic/density_advection/1d/
    {+x,-x}/rusanov/mhd_000000917.dc, via tests/golden/dc_goldens.npz): density advection, 200
    periodic cells, Rusanov, CFL 0.5, t = 0 .. 1.  Same 917 steps and final time, state within
    1e-12 of the reference's."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "dc_goldens.npz"))
    gamma = float(g[case + "_gamma"])
    n = int(g[case + "_cells"][0])
    U0 = states.density_advection(n, gamma, vx, float(g[case + "_proton_mass"]))
    cfg = pg.Config(n=(n, 1, 1), solver=pg.RUSANOV, cell_length=tuple(g[case + "_cell_length"]),
                    adiabatic_index=gamma, vacuum_permeability=float(g[case + "_mu0"]), time_step_factor=0.5)
    ctx = pg.Context(cfg)
    ctx.set_state(U0)
    t_end = float(g[case + "_time"])
    ctx.steps(int(g[case + "_step"]) + 10, t_end)
    ctx.sync()
    t, steps, _ = ctx.time()
    dts = ctx.dt_history(steps)
    assert abs(t - t_end) <= 1e-14
    assert int((dts > 0).sum()) == int(g[case + "_step"])
    out = ctx.get_state().reshape(8, n)
    ref = g[case + "_state"]
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert (np.abs(out - ref).max(axis=1) / scale).max() <= STEP_TOL
    # the same state through the reference's file format, and back into a context
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "mhd_000000917.dc")
        ctx.save_dc(path, step=int(g[case + "_step"]), time=t, proton_mass=float(g[case + "_proton_mass"]))
        info, U = pg.read_dc(path)
        assert info["step"] == int(g[case + "_step"]) and info["periodic"] == (True, True, True)
        assert np.array_equal(U.reshape(8, n), out)
        ctx2 = pg.Context(cfg)
        ctx2.load_dc(path)
        assert np.array_equal(ctx2.get_state().reshape(8, n), out)


# ---------------------------------------------------------------- other active dimensions

RELABEL_CASES = {
    "yz_periodic": dict(n=(1, 12, 10), lengths=(1.0, 0.08, 0.1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "xz_copy": dict(n=(14, 1, 10), lengths=(0.07, 1.0, 0.1), bc_lo=(po.BC_COPY, 0, po.BC_COPY),
                    bc_hi=(po.BC_COPY, 0, po.BC_COPY)),
    "z_copy": dict(n=(1, 1, 40), lengths=(1.0, 1.0, 0.025), bc_lo=(0, 0, po.BC_COPY), bc_hi=(0, 0, po.BC_COPY)),
    "y_periodic": dict(n=(1, 36, 1), lengths=(1.0, 0.03, 1.0), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
}


@pytest.mark.parametrize("solver", ["hll_athena", "hlld_athena", "roe_athena"])
@pytest.mark.parametrize("key", list(RELABEL_CASES))
def test_other_active_dimensions_match_oracle(port, key, solver):
    """Grids that are not x, x-y or x-y-z run with relabelled axes on the GPU; the oracle steps
    them as they are.  Per step within 1e-12."""
    c = RELABEL_CASES[key]
    nx, ny, nz = c["n"]
    rng = np.random.default_rng(41)
    U0 = states.smooth_3d((nz, ny, nx), rng, amp=0.1)
    gpu, ora = pair(port, c["n"], po.SOLVERS[solver], c["lengths"], 5 / 3, 1.0, 0.4, bc_lo=c["bc_lo"],
                    bc_hi=c["bc_hi"])
    gpu.set_state(U0)
    ora.set_state(U0)
    for step in range(6):
        dg = gpu.step(1.0)
        do, flag, _, _ = ora.step(1.0)
        assert flag == 0
        assert abs(dg - do) <= STEP_TOL * max(do, 1e-300) or dg == do == 0.0
        assert field_err(gpu.get_state(), ora.get_state()) <= STEP_TOL * (1 + step), step


def test_yz_grid_equals_xy_grid_bitwise():
    """A y-z grid runs as the x-y grid with its axes rotated: the same bits."""
    rng = np.random.default_rng(43)
    ny, nz = 20, 16
    U_yz = states.smooth_3d((nz, ny, 1), rng, amp=0.1)            # (8, nz, ny, 1)
    # the rotated problem: x' = y, y' = z, z' = x; momentum and field components rotate with the axes
    U_xy = np.empty((8, 1, nz, ny))
    for v, u in enumerate((0, 2, 3, 1, 4, 6, 7, 5)):
        U_xy[v, 0] = U_yz[u, :, :, 0]
    a = pg.Context(pg.Config(n=(1, ny, nz), solver=pg.HLLD, cell_length=(1.0, 0.05, 0.0625), time_step_factor=0.4))
    b = pg.Context(pg.Config(n=(ny, nz, 1), solver=pg.HLLD, cell_length=(0.05, 0.0625, 1.0), time_step_factor=0.4))
    a.set_state(U_yz)
    b.set_state(U_xy)
    a.steps(12, 1e9)
    b.steps(12, 1e9)
    a.sync()
    b.sync()
    Ya, Xb = a.get_state(), b.get_state()
    for v, u in enumerate((0, 2, 3, 1, 4, 6, 7, 5)):
        np.testing.assert_array_equal(Xb[v, 0], Ya[u, :, :, 0])
    np.testing.assert_array_equal(a.dt_history(12), b.dt_history(12))
    np.testing.assert_array_equal(a.totals()[[0, 2, 3, 1, 4, 6, 7, 5]], b.totals())


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena", "hlld_athena", "roe_athena"])
@pytest.mark.parametrize("name", ["blast_3d", "smooth_3d", "orszag_tang_2d", "smooth_1d"])
def test_steps_match_reference_step_functions(name, solver):
    """The GPU step against the reference's own step functions (minimize_timestep, the substep
    plan, get_all_fluxes, update_mhd_state, compiled unchanged; committed outputs, see
    test_cell_centred_ref_pin.py): the priming step and nine steps, every dt within 1e-13 and the
    state within 1e-12 of each field's largest magnitude."""
    import test_cell_centred_ref_pin as R
    U, dts = R.golden(name, solver)
    n, lengths = R.CASES[name]
    cfg = pg.Config(n=n, solver=R.SOLVERS[solver], cell_length=lengths, adiabatic_index=states.GAMMA_53,
                    time_step_factor=0.4)
    ctx = pg.Context(cfg)
    try:
        ctx.set_state(R.case_input(name))
        got = [ctx.step(0.0 if s == 0 else 1e300) for s in range(R.STEPS)]
        Ug = ctx.get_state()
    finally:
        ctx.close()
    assert np.abs(np.array(got) - dts).max() <= 1e-13 * dts.max()
    for rows in ([0], [1, 2, 3], [4], [5, 6, 7]):
        assert np.abs(Ug[rows] - U[rows]).max() <= 1e-12 * np.abs(U[rows]).max(), rows
