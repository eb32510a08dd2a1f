"""The cell-centred step of the oracle (oracle/mode_c.hpp) pinned BIT FOR BIT to the reference's
own step functions: set_minmax_substepping_period, minimize_timestep, the substep plan,
get_all_fluxes and update_mhd_state of mhd/solve.hpp in timestep()'s order (its face-field parts
left out: no update_vol_B, no sync, the cell's volume field keeping the flux update), compiled
unchanged from the reference tree on a one-rank box stand-in for dccrg
(oracle/ref_stag_bridge.cpp: ref_cell_centred_run, built by oracle/Makefile where the reference
tree is present).

Cases: the 3-D blast wave (the configured workload's state, 8^3), a smooth 3-D state, the 2-D
Orszag-Tang vortex (a dimension of one cell without faces, as the reference's 2-D grids with
periodic {true, true, false}) and a smooth 1-D state; every solver; the priming step and nine
steps.  The reference's outputs are committed (tests/golden/cell_centred_ref.npz, made by
tests/golden/make_cell_centred_golden.py); the oracle reproduces them bit for bit, state and
every dt; where the reference build is present, it reproduces the fixture bit for bit too.  The
GPU is held to the same fixture in test_gpu_parity.py.

Local time stepping the same way (ref_cell_centred_substep_run: the options' per-cell
substep-min / substep-max evaluated at the cell centres, then the substep loop of timestep(),
mhd/solve.hpp:1865-1902): a 3-D grid with periods forced to 1 and 2 in two halves, and a 2-D grid
with a dense, slow half and free exponents up to 3 (periods reaching 4), every solver, eight
steps; the oracle's substepped step (oracle/substep.hpp) reproduces state, step lengths and
largest periods bit for bit, and the GPU's (test_gpu_substep.py) is within 1e-12."""
import ctypes
import os

import numpy as np
import pytest

from oracle import pyoracle as po
import states

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cell_centred_ref.npz")
REF_LIB = os.path.join(po.ORACLE_DIR, "_ref", "libstag_ref.so")
P32 = ctypes.POINTER(ctypes.c_int32)
PD = ctypes.POINTER(ctypes.c_double)
STEPS = 10
SOLVERS = {"rusanov": po.RUSANOV, "hll_athena": po.HLL, "hlld_athena": po.HLLD, "roe_athena": po.ROE}
CASES = {
    # name: (n, cell lengths)
    "blast_3d": ((8, 8, 8), (1 / 8, 1 / 8, 1 / 8)),
    "smooth_3d": ((6, 5, 7), (0.1, 0.12, 0.09)),
    "orszag_tang_2d": ((16, 16, 1), (1 / 16, 1 / 16, 1.0)),
    "smooth_1d": ((40, 1, 1), (0.025, 1.0, 1.0)),
}


def case_input(name):
    n, _ = CASES[name]
    if name == "blast_3d":
        return states.blast_wave(8)
    if name == "orszag_tang_2d":
        return states.orszag_tang(16)
    return states.smooth_3d((n[2], n[1], n[0]), np.random.default_rng(3), amp=0.1)


def load_ref_run():
    if not os.path.exists(REF_LIB):
        return None
    L = ctypes.CDLL(REF_LIB)
    L.ref_cell_centred_run.argtypes = [P32, PD, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       PD, ctypes.c_int32, PD, PD]

    def run(name, solver):
        n, lengths = CASES[name]
        U = np.ascontiguousarray(case_input(name), dtype=np.float64)
        cells = U.reshape(-1)
        out, dts = np.zeros_like(cells), np.zeros(STEPS)
        rc = L.ref_cell_centred_run((ctypes.c_int32 * 3)(*n), (ctypes.c_double * 3)(*lengths), solver,
                                    states.GAMMA_53, 1.0, 0.4, cells.ctypes.data_as(PD), STEPS,
                                    out.ctypes.data_as(PD), dts.ctypes.data_as(PD))
        if rc != 0:
            raise RuntimeError("the reference's step stopped")
        return out.reshape(U.shape), dts
    return run


def golden(name, solver):
    g = np.load(GOLD)
    return g[f"{name}_{solver}_cells"], g[f"{name}_{solver}_dts"]


@pytest.mark.parametrize("solver", list(SOLVERS))
@pytest.mark.parametrize("name", list(CASES))
def test_oracle_equals_reference_step(port, name, solver):
    U, dts = golden(name, solver)
    n, lengths = CASES[name]
    g = port.grid(po.make_cfg(n, SOLVERS[solver], lengths, states.GAMMA_53, 1.0, 0.4))
    g.set_state(case_input(name))
    got = []
    for s in range(STEPS):
        dt, flag, _, _ = g.step(0.0 if s == 0 else 1e300)
        assert flag == 0
        got.append(dt)
    assert np.array_equal(np.array(got), dts)
    assert np.array_equal(g.get_state(), U)


@pytest.mark.parametrize("name", list(CASES))
def test_reference_build_reproduces_fixture(name):
    run = load_ref_run()
    if run is None:
        pytest.skip("reference build (oracle/_ref) not available")
    for solver, sid in SOLVERS.items():
        U, dts = golden(name, solver)
        Ur, dr = run(name, sid)
        assert np.array_equal(Ur, U) and np.array_equal(dr, dts)


# ---------------------------------------------------------------- local time stepping

SUB_STEPS = 8
SUB_CASES = {
    "forced_periods_3d": ((8, 6, 7), (0.1, 0.12, 0.09)),
    "slow_half_2d": ((16, 12, 1), (0.1, 0.12, 1.0)),
}


def sub_case(name):
    """State and exponent bounds (smallest, largest) of a substepped case."""
    n, _ = SUB_CASES[name]
    shape = (n[2], n[1], n[0])
    U = states.smooth_3d(shape, np.random.default_rng(3), amp=0.1)
    half = np.broadcast_to((np.arange(n[0]) < n[0] // 2)[None, None, :], shape)
    if name == "forced_periods_3d":
        e = np.where(half, 0, 1).astype(np.int32)
        return U, e, e.copy()
    U = U.copy()
    U[0][half] *= 16.0
    U[1:4][:, half] *= 16.0
    return U, np.zeros(shape, np.int32), np.full(shape, 3, np.int32)


def load_ref_substep_run():
    if not os.path.exists(REF_LIB):
        return None
    L = ctypes.CDLL(REF_LIB)
    L.ref_cell_centred_substep_run.argtypes = [P32, PD, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, PD, P32, P32, ctypes.c_int32, PD, PD, P32]

    def run(name, solver):
        n, lengths = SUB_CASES[name]
        U, smin, smax = sub_case(name)
        cells = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
        out, dts = np.zeros_like(cells), np.zeros(SUB_STEPS)
        top = np.zeros(SUB_STEPS, dtype=np.int32)
        rc = L.ref_cell_centred_substep_run((ctypes.c_int32 * 3)(*n), (ctypes.c_double * 3)(*lengths), solver,
                                            states.GAMMA_53, 1.0, 0.4, cells.ctypes.data_as(PD),
                                            smin.ctypes.data_as(P32), smax.ctypes.data_as(P32), SUB_STEPS,
                                            out.ctypes.data_as(PD), dts.ctypes.data_as(PD), top.ctypes.data_as(P32))
        if rc != 0:
            raise RuntimeError("the reference's step stopped")
        return out.reshape(U.shape), dts, top
    return run


def sub_golden(name, solver):
    g = np.load(GOLD)
    k = f"sub_{name}_{solver}"
    return g[k + "_cells"], g[k + "_dts"], g[k + "_periods"]


@pytest.mark.parametrize("solver", list(SOLVERS))
@pytest.mark.parametrize("name", list(SUB_CASES))
def test_oracle_substeps_equal_reference(port, name, solver):
    U, dts, top = sub_golden(name, solver)
    n, lengths = SUB_CASES[name]
    U0, smin, smax = sub_case(name)
    g = port.substep_grid(po.make_cfg(n, SOLVERS[solver], lengths, states.GAMMA_53, 1.0, 0.4))
    g.set_state(U0)
    g.set_exponents(smin, smax)
    got, ks = [], []
    for s in range(SUB_STEPS):
        dt, k, _, flag = g.step(0.0 if s == 0 else 1e300)
        assert flag == 0
        got.append(dt)
        ks.append(k)
    assert np.array_equal(np.array(got), dts) and np.array_equal(np.array(ks), top)
    assert top.max() > 1   # the cases do substep
    assert np.array_equal(g.get_state(), U)


@pytest.mark.parametrize("name", list(SUB_CASES))
def test_reference_build_reproduces_substep_fixture(name):
    run = load_ref_substep_run()
    if run is None:
        pytest.skip("reference build (oracle/_ref) not available")
    for solver, sid in SOLVERS.items():
        U, dts, top = sub_golden(name, solver)
        Ur, dr, tr = run(name, sid)
        assert np.array_equal(Ur, U) and np.array_equal(dr, dts) and np.array_equal(tr, top)

