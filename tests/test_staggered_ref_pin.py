"""The staggered-field step of the oracle (oracle/mode_s.hpp) pinned to the reference's own step:
timestep() of mhd/solve.hpp (get_fluxes with assign_face_dBs_f{x,y,z}, update_mhd_state,
update_vol_B, sync_magnetic_field) and, on a bounded box, the solar-wind box's
apply_boundaries_sw_box with the program's loop around them (tests/mhd/solar_wind_box.cpp:
446-553), compiled unchanged from the reference tree on a one-rank box stand-in for dccrg
(oracle/ref_stag_bridge.cpp, built by oracle/Makefile where the reference tree is present).

Cases: a 3-D periodic grid (the staggered step in 3-D, which the reference's own output files pin
in 1-D and 2-D only), a box bounded on every side (COPY), a box with the wind entering through -x,
and a 2-D box with the wind entering through +y; every solver; the priming step and five steps.
The reference's outputs are committed (tests/golden/staggered_ref.npz, made by
tests/golden/make_staggered_golden.py from the reference build); the oracle agrees within 1e-13
(the reference sums each face's twelve edge terms, and its two copies of a face, in its own
order); where the reference build is present it reproduces the fixture bit for bit.  The GPU is
held to the same fixture in test_gpu_staggered_bounded.py."""
import ctypes
import os

import numpy as np
import pytest

from oracle import pyoracle as po
import states

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "staggered_ref.npz")
REF_LIB = os.path.join(po.ORACLE_DIR, "_ref", "libstag_ref.so")
P32 = ctypes.POINTER(ctypes.c_int32)
PD = ctypes.POINTER(ctypes.c_double)
C, V, P = po.BC_COPY, po.BC_VALUE, po.BC_PERIODIC
LENGTHS = (0.1, 0.12, 0.09)
STEPS = 6
# the wind's number density (proton mass 1), velocity, pressure and field
WIND = (1.3, 0.2, -0.05, 0.03, 0.9, 0.3, -0.2, 0.1)
CASES = {
    "periodic_3d": ((5, 4, 6), (P, P, P), (P, P, P)),
    "copy_box": ((5, 4, 3), (C, C, C), (C, C, C)),
    "wind_minus_x": ((6, 5, 4), (V, C, C), (C, C, C)),
    "wind_plus_y_2d": ((10, 8, 1), (C, C, P), (C, V, P)),
}
SOLVERS = {"rusanov": po.RUSANOV, "hll_athena": po.HLL, "hlld_athena": po.HLLD, "roe_athena": po.ROE}


def case_input(name):
    """The seeded state of a case: cells (8, nz, ny, nx) and the three face arrays, a smooth random
    state with a divergence-free face field (the high wall of a bounded dimension the face that
    wraps around to the first)."""
    n, bc_lo, bc_hi = CASES[name]
    U, faces, _ = states.staggered_random((n[2], n[1], n[0]), LENGTHS, np.random.default_rng(5))
    out = []
    for d, shape in enumerate(po.staggered_face_shapes(n, bc_lo, bc_hi)):
        f = faces[d]
        if shape != f.shape:
            f = np.concatenate([f, np.take(f, [0], axis=2 - d)], axis=2 - d)
        out.append(np.ascontiguousarray(f))
    return U, out


def load_ref_run():
    """The reference's run function (None where its build is absent)."""
    if not os.path.exists(REF_LIB):
        return None
    L = ctypes.CDLL(REF_LIB)
    L.ref_stag_run.argtypes = [P32, PD, P32, P32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, PD, PD, PD, ctypes.c_int32, PD, PD, PD, PD]

    def run(name, solver):
        n, bc_lo, bc_hi = CASES[name]
        U, F = case_input(name)
        shapes = po.staggered_face_shapes(n, bc_lo, bc_hi)
        cells = np.ascontiguousarray(U).reshape(-1)
        faces = np.concatenate([f.reshape(-1) for f in F])
        co, fo = np.zeros_like(cells), np.zeros_like(faces)
        dts, value = np.zeros(STEPS), np.zeros(8)
        wind = np.asarray(WIND, dtype=np.float64)
        rc = L.ref_stag_run((ctypes.c_int32 * 3)(*n), (ctypes.c_double * 3)(*LENGTHS), (ctypes.c_int32 * 3)(*bc_lo),
                            (ctypes.c_int32 * 3)(*bc_hi), solver, states.GAMMA_53, 1.0, 0.4,
                            cells.ctypes.data_as(PD), faces.ctypes.data_as(PD), wind.ctypes.data_as(PD), STEPS,
                            co.ctypes.data_as(PD), fo.ctypes.data_as(PD), dts.ctypes.data_as(PD),
                            value.ctypes.data_as(PD))
        if rc != 0:
            raise RuntimeError("the reference's step stopped")
        out, at = [], 0
        for s in shapes:
            k = int(np.prod(s))
            out.append(fo[at:at + k].reshape(s))
            at += k
        return co.reshape(U.shape), out, dts, value
    return run


def golden(name, solver_name):
    g = np.load(GOLD)
    key = f"{name}_{solver_name}"
    return g[key + "_cells"], [g[key + f"_faces{d}"] for d in range(3)], g[key + "_dts"], g[name + "_" + solver_name + "_value"]


def oracle_run(port, name, solver, value):
    n, bc_lo, bc_hi = CASES[name]
    vlo = [value if k == V else None for k in bc_lo]
    vhi = [value if k == V else None for k in bc_hi]
    g = port.staggered_grid(po.make_cfg(n, solver, LENGTHS, states.GAMMA_53, 1.0, 0.4, bc_lo, bc_hi, vlo, vhi))
    U, F = case_input(name)
    g.set_state(U, F)
    dts = []
    for s in range(STEPS):
        dt, flag, _, _ = g.step(0.0 if s == 0 else 1e300)
        assert flag == 0
        dts.append(dt)
    Uo, Fo = g.get_state()
    return Uo, list(Fo), np.array(dts)


def rel(a, b, rows=None):
    if rows is None:
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    return max(float(np.abs(a[r] - b[r]).max() / max(np.abs(b[r]).max(), 1e-300)) for r in rows)


@pytest.mark.parametrize("solver", list(SOLVERS))
@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_step(port, name, solver):
    U, F, dts, value = golden(name, solver)
    Uo, Fo, do = oracle_run(port, name, SOLVERS[solver], value)
    assert np.abs(do - dts).max() <= 1e-13 * dts.max()
    assert rel(Uo, U, ([0], [1, 2, 3], [4], [5, 6, 7])) <= 1e-13
    assert max(rel(Fo[d], F[d]) for d in range(3)) <= 1e-13


@pytest.mark.parametrize("name", list(CASES))
def test_reference_build_reproduces_fixture(name):
    run = load_ref_run()
    if run is None:
        pytest.skip("reference build (oracle/_ref) not available")
    for solver, sid in SOLVERS.items():
        U, F, dts, value = golden(name, solver)
        Ur, Fr, dr, vr = run(name, sid)
        assert np.array_equal(Ur, U) and np.array_equal(dr, dts) and np.array_equal(vr, value)
        assert all(np.array_equal(a, b) for a, b in zip(Fr, F))
