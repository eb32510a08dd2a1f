"""Pins the CPU oracle to the reference (CPU only).

The oracle (oracle/mhd_oracle.hpp, oracle/mode_c.hpp) restates the
reference's solvers and step.  These tests hold it to:
  - the fixtures in tests/golden, made by tests/golden/make_golden.py from
    the reference's own solver headers and its tests/mhd/reference.cpp;
  - the live reference build (oracle/_ref) where the reference tree exists;
  - the reference's shipped goldens tests/mhd/mhd_{rusanov,hll_athena}.ref at
    the reference's own tolerance (tests/mhd/reference.cpp:637-640);
  - rotation symmetry, the property mhd_diff.py --rotate checks;
  - the reference program's own output files (tests/mhd/reference/**/*.dc, extracted into
    tests/golden/dc_goldens.npz by tests/golden/make_dc_golden.py with the reference's reader)
    for the cases whose field is zero, where its staggered-field step reduces to the
    cell-centred one: same step count, state within a few ulps after 917 steps;
  - the same program's Alfven-wave outputs, which pin the staggered-field step
    (oracle/mode_s.hpp), with and without a background field: same step count, every cell
    within the tolerances of the reference's own comparison (tests/mhd/mhd_diff.py:232-241).
Bit-for-bit equality is required wherever both sides run the same
arithmetic (the oracle is built with -ffp-contract=off, as the reference).
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
import states

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF_TESTS = os.path.join(po.REFERENCE, "tests", "mhd")


def _load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_face_flux_matches_reference_fixture(port, solver):
    g = _load("face_flux.npz")
    flux, speed, flags = port.face_flux(po.SOLVERS[solver], g["neg"], g["pos"], g["bg"])
    np.testing.assert_array_equal(flags, g[f"{solver}_flags"])
    np.testing.assert_array_equal(flux, g[f"{solver}_flux"])
    np.testing.assert_array_equal(speed, g[f"{solver}_speed"])


@pytest.mark.parametrize("solver", list(po.SOLVERS))
def test_face_flux_matches_live_reference(port, ref, solver):
    rng = np.random.default_rng(7)
    neg = states.random_face_states(4000, rng)
    pos = states.random_face_states(4000, rng)
    a, b = states.nearby_face_states(4000, rng)
    neg = np.vstack([neg, a])
    pos = np.vstack([pos, b])
    bg = rng.normal(0, 0.3, (neg.shape[0], 3))
    for mu0 in (1.0, 4e-7 * np.pi):
        scale = np.ones(8)
        if mu0 != 1.0:
            scale[5:8] = np.sqrt(mu0)  # same Alfven speeds in SI field units
        f1, s1, g1 = port.face_flux(po.SOLVERS[solver], neg * scale, pos * scale, bg * scale[5:8], 5 / 3, mu0)
        f2, s2, g2 = ref.face_flux(po.SOLVERS[solver], neg * scale, pos * scale, bg * scale[5:8], 5 / 3, mu0)
        np.testing.assert_array_equal(g1, g2)
        np.testing.assert_array_equal(f1, f2)
        np.testing.assert_array_equal(s1, s2)


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena"])
def test_reference_1d_matches_reference_program(port, solver):
    out, steps = port.reference_1d(po.SOLVERS[solver])
    assert steps == {"rusanov": 944, "hll_athena": 945}[solver]
    np.testing.assert_array_equal(out, _load("ref1d.npz")[solver])


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena"])
def test_reference_1d_matches_shipped_golden(port, solver):
    path = os.path.join(REF_TESTS, f"mhd_{solver}.ref")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    gold = np.loadtxt(path)
    out, _ = port.reference_1d(po.SOLVERS[solver])
    # verify_mhd: relative error <= 1e-6 where either value exceeds 1e-25 (reference.cpp:637-742)
    big = (out > 1e-25) | (gold > 1e-25)
    rel = np.abs(out - gold) / np.maximum(np.abs(out), np.abs(gold)).clip(1e-300)
    assert rel[big].max() <= 1e-6


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena"])
def test_reference_program_passes_its_own_golden(solver):
    if not (os.path.exists(po.REF_EXE) and os.path.isdir(REF_TESTS)):
        pytest.skip("reference build not present")
    r = subprocess.run([po.REF_EXE, "--solver", solver], cwd=REF_TESTS, capture_output=True, timeout=120)
    assert r.returncode == 0, r.stderr


def _run(o, key, solver):
    rng = np.random.default_rng(20261203 + 1)
    if key == "periodic":
        U0 = states.smooth_3d((4, 5, 6), rng)
        cfg = po.make_cfg((6, 5, 4), solver, (1 / 6, 1 / 5, 1 / 4), 5 / 3, 1.0, 0.4)
        steps, max_dt = 4, 1.0
    elif key == "bounded":
        U0 = states.smooth_3d((4, 5, 6), rng)
        inflow = np.array([1.2, 0.3 * 1.2, 0.2 * 1.2, 0.0,
                           states.energy(1.2, np.array([[0.3], [0.2], [0.0]]), 0.7,
                                         np.array([[0.4], [0.1], [-0.2]]), 5 / 3)[0], 0.4, 0.1, -0.2])
        cfg = po.make_cfg((6, 5, 4), solver, (0.2, 0.25, 0.3), 5 / 3, 1.0, 0.4,
                          bc_lo=(po.BC_COPY, po.BC_VALUE, po.BC_PERIODIC),
                          bc_hi=(po.BC_COPY, po.BC_COPY, po.BC_PERIODIC), value_lo=[None, inflow, None])
        steps, max_dt = 4, 1.0
    else:
        U0 = states.brio_wu(64)
        cfg = po.make_cfg((64, 1, 1), solver, (1 / 64, 1, 1), 2.0, 1.0, 0.5,
                          bc_lo=(po.BC_COPY, 0, 0), bc_hi=(po.BC_COPY, 0, 0))
        steps, max_dt = 12, 0.1
    g = o.grid(cfg)
    g.set_state(U0)
    traj, dts = [U0], []
    for _ in range(steps):
        dt, flag, _, _ = g.step(max_dt)
        if flag:
            break
        dts.append(dt)
        traj.append(g.get_state())
    return np.array(traj), np.array(dts)


@pytest.mark.parametrize("key,solver", [("periodic", s) for s in po.SOLVERS]
                         + [("bounded", "hll_athena"), ("bounded", "hlld_athena")]
                         + [("briowu", s) for s in po.SOLVERS])
def test_mode_c_matches_reference_fixture(port, key, solver):
    g = _load("mode_c.npz")
    traj, dts = _run(port, key, po.SOLVERS[solver])
    np.testing.assert_array_equal(dts, g[f"{key}_{solver}_dt"])
    np.testing.assert_array_equal(traj, g[f"{key}_{solver}_traj"])


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("axis", [1, 2])
def test_mode_c_rotation_symmetry(port, solver, axis):
    """A 1-D tube along y or z equals the tube along x with vector components rotated
    (get_rotated_vector, mhd/common.hpp:612), bit for bit."""
    n = 48
    Ux = states.brio_wu(n)
    ext = [1, 1, 1]
    ext[axis] = n
    lens = [1.0, 1.0, 1.0]
    lens[axis] = 1 / n
    perm = {1: [2, 0, 1], 2: [1, 2, 0]}[axis]  # component c of the rotated tube = component perm[c] of x
    U = np.zeros((8, ext[2], ext[1], ext[0]))
    line = Ux[:, 0, 0, :]
    for c in range(3):
        U[1 + c].reshape(-1)[:] = line[1 + perm[c]]
        U[5 + c].reshape(-1)[:] = line[5 + perm[c]]
    U[0].reshape(-1)[:] = line[0]
    U[4].reshape(-1)[:] = line[4]
    bc_lo = [0, 0, 0]
    bc_hi = [0, 0, 0]
    cfg_x = po.make_cfg((n, 1, 1), po.SOLVERS[solver], (1 / n, 1, 1), 2.0, 1.0, 0.5,
                        bc_lo=(po.BC_COPY, 0, 0), bc_hi=(po.BC_COPY, 0, 0))
    bc_lo[axis] = po.BC_COPY
    bc_hi[axis] = po.BC_COPY
    cfg_r = po.make_cfg(ext, po.SOLVERS[solver], lens, 2.0, 1.0, 0.5, bc_lo=bc_lo, bc_hi=bc_hi)
    gx, gr = port.grid(cfg_x), port.grid(cfg_r)
    gx.set_state(Ux)
    gr.set_state(U)
    for _ in range(8):
        dx = gx.step(0.1)
        dr = gr.step(0.1)
        assert dx[0] == dr[0] and dx[1] == dr[1]
        if dx[1]:
            break
        a = gx.get_state()[:, 0, 0, :]
        b = gr.get_state().reshape(8, -1)
        for c in range(3):
            np.testing.assert_array_equal(b[1 + c], a[1 + perm[c]])
            np.testing.assert_array_equal(b[5 + c], a[5 + perm[c]])
        np.testing.assert_array_equal(b[[0, 4]], a[[0, 4]])


def test_mode_c_threads_do_not_change_bits(port):
    rng = np.random.default_rng(3)
    U0 = states.smooth_3d((16, 12, 10), rng)
    cfg = po.make_cfg((10, 12, 16), po.HLLD, (0.1, 0.1, 0.1), 5 / 3, 1.0, 0.4)
    a, b = port.grid(cfg, threads=1), port.grid(cfg, threads=4)
    a.set_state(U0)
    b.set_state(U0)
    for _ in range(3):
        assert a.step(1.0)[0] == b.step(1.0)[0]
    np.testing.assert_array_equal(a.get_state(), b.get_state())


def test_mode_c_conserves_totals_on_periodic_grid(port):
    rng = np.random.default_rng(4)
    U0 = states.smooth_3d((8, 8, 8), rng)
    cfg = po.make_cfg((8, 8, 8), po.HLLD, (1 / 8, 1 / 8, 1 / 8), 5 / 3, 1.0, 0.4)
    g = port.grid(cfg)
    g.set_state(U0)
    for _ in range(5):
        g.step(1.0)
    U = g.get_state()
    t0 = U0.reshape(8, -1).sum(1)
    t1 = U.reshape(8, -1).sum(1)
    scale = np.abs(U0).reshape(8, -1).sum(1)
    assert np.all(np.abs(t1 - t0) <= 1e-13 * scale)


def test_invalid_state_reports_first_failing_face(port):
    rng = np.random.default_rng(5)
    U0 = states.smooth_3d((4, 4, 4), rng)
    U0[4, 2, 1, 3] = 0.0  # negative pressure in cell (x=3, y=1, z=2)
    cfg = po.make_cfg((4, 4, 4), po.HLLD, (0.25, 0.25, 0.25), 5 / 3, 1.0, 0.4)
    g = port.grid(cfg)
    g.set_state(U0)
    dt, flag, cell, d = g.step(0.0)
    assert flag == 2  # PAMHD_FLAG_PRESSURE
    # first face in x-fastest cell order touching the bad cell: the +z face of (3, 1, 1)
    assert cell == (3, 1, 1) and d == 3


@pytest.mark.parametrize("case,vx", [("da_px", 1.0), ("da_mx", -1.0)])
def test_mode_c_reproduces_reference_program_output(port, case, vx):
    """Density advection, 200 periodic cells, Rusanov, CFL 0.5, t = 0 .. 1: the reference
    program wrote its state after 917 steps; the oracle's step (priming step, lagged CFL dt,
    time cap, update) reproduces it."""
    g = _load("dc_goldens.npz")
    gamma = float(g[case + "_gamma"])
    n = int(g[case + "_cells"][0])
    U0 = states.density_advection(n, gamma, vx, float(g[case + "_proton_mass"]))
    grid = port.grid(po.make_cfg((n, 1, 1), po.RUSANOV, tuple(g[case + "_cell_length"]), gamma,
                                 float(g[case + "_mu0"]), 0.5))
    grid.set_state(U0)
    t, dts = grid.run(0.0, float(g[case + "_time"]), 100000)
    assert t == float(g[case + "_time"])
    assert int((dts > 0).sum()) == int(g[case + "_step"])   # plus the dt = 0 priming step
    out = grid.get_state().reshape(8, n)
    ref = g[case + "_state"]
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert (np.abs(out - ref).max(axis=1) / scale).max() <= 1e-14


def _mhd_diff_ok(out, ref, tol=1e-15, floor=1e-15):
    """The per-cell comparison of tests/mhd/mhd_diff.py:189-225 with its default tolerances:
    (|a - b| - floor) / max(|a|, |b|) <= tol for mass density, |v|, total energy and |B|."""
    def within(a, b):
        denom = np.maximum(np.abs(a), np.abs(b))
        diff = np.abs(a - b) - floor
        return bool(np.all((denom == 0) | (diff / np.where(denom == 0, 1, denom) <= tol)))

    v1 = np.linalg.norm(out[1:4] / out[0], axis=0)
    v2 = np.linalg.norm(ref[1:4] / ref[0], axis=0)
    return (within(out[0], ref[0]) and within(v1, v2) and within(out[4], ref[4])
            and within(np.linalg.norm(out[5:8], axis=0), np.linalg.norm(ref[5:8], axis=0)))


STAGGERED_CASES = {
    "alf_px": lambda: states.alfven_1d(100, 1),
    "alf_mx": lambda: states.alfven_1d(100, -1),
    "alf_r1": lambda: states.alfven_2d(False),
    "alf_r2": lambda: states.alfven_2d(True),
    "alf_b1": lambda: states.alfven_2d(False, background=True),
    "alf_b2": lambda: states.alfven_2d(True, background=True),
}


def run_staggered(grid_owner, case, solver=po.RUSANOV):
    """Runs a staggered-field golden case as the reference's program does (tests/mhd/test.cpp:
    422-537): initial state, the dt = 0 priming step, then steps capped by the time left until
    t = 1.  Returns (state (8, cells), faces (3, cells), steps, t)."""
    g = _load("dc_goldens.npz")
    U0, faces, _, *bg = STAGGERED_CASES[case]()
    n = (U0.shape[3], U0.shape[2], U0.shape[1])
    cfg = po.make_cfg(n, solver, tuple(g[case + "_cell_length"]), float(g[case + "_gamma"]),
                      float(g[case + "_mu0"]), 0.5)
    grid = grid_owner.staggered_grid(cfg)
    grid.set_state(U0, faces)
    if bg:
        grid.set_background(bg[0])
    grid.step(0.0)
    t, steps, t_end = 0.0, 0, float(g[case + "_time"])
    while t < t_end:
        dt, flag, _, _ = grid.step(t_end - t)
        assert flag == 0
        t += dt
        steps += 1
    U, F = grid.get_state()
    return U.reshape(8, -1), F.reshape(3, -1), steps, t


@pytest.mark.parametrize("case", list(STAGGERED_CASES))
def test_mode_s_reproduces_reference_program_output(port, case):
    """The reference program's staggered-field Alfven waves (Rusanov, CFL 0.5, t = 0 .. 1): the
    oracle takes the same number of steps to the same time and every cell passes the reference's
    own comparison against the program's output at its default 1e-15 tolerances."""
    g = _load("dc_goldens.npz")
    out, _, steps, t = run_staggered(port, case)
    assert steps == int(g[case + "_step"])
    assert t == float(g[case + "_time"])
    ref = g[case + "_state"]
    assert _mhd_diff_ok(out, ref)
    # every conservative value within 2e-15 absolute (all are of order 1 or less here)
    assert np.abs(out - ref).max() <= 2e-15


@pytest.mark.parametrize("case", ["alf_px", "alf_r1", "alf_b2"])
def test_mode_s_restated_solvers_equal_reference_headers(port, ref, case):
    """The staggered step driven by the reference's own solver headers computes the same bits."""
    a = run_staggered(port, case)
    b = run_staggered(ref, case)
    assert a[2] == b[2]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena", "hlld_athena"])
def test_mode_s_keeps_divergence(port, solver):
    """Constrained transport: the discrete divergence of the face field does not change."""
    U, faces, L = states.staggered_random((6, 5, 7), (0.1, 0.12, 0.09), np.random.default_rng(7))
    cfg = po.make_cfg((7, 5, 6), po.SOLVERS[solver], L, states.GAMMA_53, 1.0, 0.4)
    grid = port.staggered_grid(cfg)
    grid.set_state(U, faces)
    div0 = states.face_divergence(faces, L)
    grid.step(0.0)
    for _ in range(10):
        dt, flag, _, _ = grid.step(1.0)
        assert flag == 0 and dt > 0
    _, F = grid.get_state()
    assert np.abs(states.face_divergence(F, L) - div0).max() <= 1e-12 * np.abs(F).max() / min(L)


def test_mode_s_cyclic_rotation(port):
    """The staggered step commutes with the cyclic relabelling x -> y -> z of axes, vector
    components and faces (the property the reference's rotated golden checks use,
    mhd_diff.py --rotate).  The face fluxes and face-field changes are relabelled bit for bit;
    the pressure sums of update_vol_B add the components in grid order, so the states agree to
    rounding."""
    U0, faces, L = states.alfven_1d(20, 1)

    def run(U, faces, L):
        n = (U.shape[3], U.shape[2], U.shape[1])
        grid = port.staggered_grid(po.make_cfg(n, po.HLLD, L, 1.6666666666666667, 1.0, 0.5))
        grid.set_state(U, faces)
        grid.step(0.0)
        for _ in range(15):
            grid.step(1.0)
        return grid.get_state()

    def to_y(U, F):
        # data along x -> along y; components (x, y, z) -> (z, x, y)
        return np.moveaxis(U, 3, 2)[[0, 3, 1, 2, 4, 7, 5, 6]], np.moveaxis(F, 3, 2)[[2, 0, 1]]

    a_U, a_F = run(U0, faces, L)
    U1, F1 = to_y(U0, faces)
    b_U, b_F = run(U1, F1, (L[2], L[0], L[1]))
    e_U, e_F = to_y(a_U, a_F)
    np.testing.assert_allclose(b_U, e_U, rtol=0, atol=1e-14)
    np.testing.assert_allclose(b_F, e_F, rtol=0, atol=1e-14)
