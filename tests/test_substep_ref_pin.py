"""The substep plan of the oracle (oracle/substep.hpp) pinned to the reference's own substepping
functions (substepping.hpp: set_minmax_substepping_period in both forms,
restrict_substepping_period, update_substeps), compiled unchanged from the reference tree on a
single-rank uniform-grid stand-in for dccrg (oracle/ref_substep_bridge.cpp, built by
oracle/Makefile where the reference tree is present): on the same per-cell CFL limits, exponent
bounds and cap, every cell's period, the substep length and the largest period agree bit for bit,
on 3-D and 2-D periodic grids, with the cap below, inside and above the limits, with cells whose
limit is 0, and where the reference aborts (a cell's smallest exponent above its largest after
the cap), both refuse.  The GPU is held to the oracle's plan per step in test_gpu_substep.py."""
import ctypes
import os

import numpy as np
import pytest

from oracle import pyoracle as po

P32 = ctypes.POINTER(ctypes.c_int32)
PD = ctypes.POINTER(ctypes.c_double)


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "substep_plan.npz")


def lengths_of(n):
    return (0.1, 0.12, 0.09 if n[2] > 1 else 1.0)


def load_ref_plan():
    """The reference's plan function (None where its build is absent)."""
    if not os.path.exists(po.REF_SUBSTEP_LIB):
        try:
            po.build()
        except Exception:
            pass
    if not os.path.exists(po.REF_SUBSTEP_LIB):
        return None
    L = ctypes.CDLL(po.REF_SUBSTEP_LIB)
    L.ref_substep_plan.argtypes = [P32, PD, PD, P32, P32, ctypes.c_double, P32, PD, P32]

    def plan(n, lengths, limits, smin, smax, max_dt):
        nn = (ctypes.c_int32 * 3)(*n)
        ll = (ctypes.c_double * 3)(*lengths)
        lim = np.ascontiguousarray(limits, dtype=np.float64).reshape(-1)
        a = np.ascontiguousarray(smin, dtype=np.int32).reshape(-1)
        b = np.ascontiguousarray(smax, dtype=np.int32).reshape(-1)
        periods = np.zeros(lim.size, dtype=np.int32)
        sub, top = ctypes.c_double(0), ctypes.c_int32(0)
        rc = L.ref_substep_plan(nn, ll, lim.ctypes.data_as(PD), a.ctypes.data_as(P32), b.ctypes.data_as(P32),
                                max_dt, periods.ctypes.data_as(P32), ctypes.byref(sub), ctypes.byref(top))
        if rc != 0:
            return None
        return periods.reshape(np.shape(limits)), sub.value, top.value
    return plan


@pytest.fixture(scope="module")
def ref_plan():
    plan = load_ref_plan()
    if plan is None:
        pytest.skip("reference build (oracle/_ref) not available")
    return plan


def oracle_plan(port, n, lengths, limits, smin, smax, max_dt):
    g = port.substep_grid(po.make_cfg(n, po.HLL, lengths, 5 / 3, 1.0, 0.4))
    g.set_exponents(smin, smax)
    return g.plan(limits, max_dt)


def cases():
    rng = np.random.default_rng(20261206)
    out = []
    for n in ((9, 7, 6), (12, 10, 1), (5, 5, 5)):
        shape = (n[2], n[1], n[0])
        for kind in ("spread", "regions", "zero_limit", "uniform"):
            if kind == "uniform":
                limits = np.full(shape, 0.37)
            else:
                limits = 0.01 * np.exp(rng.uniform(0.0, 3.0, shape))
            if kind == "zero_limit":
                limits.reshape(-1)[rng.choice(limits.size, 3, replace=False)] = 0.0
            lo = rng.integers(0, 3, shape)
            hi = lo + rng.integers(0, 3, shape)
            if kind == "regions":
                lo[:] = 0
                hi[:] = 0
                hi[..., n[0] // 2:] = 3
            for cap in (0.5 * limits[limits > 0].min(), 3.0 * limits.max(), float(np.median(limits))):
                out.append((n, shape, kind, limits, lo, hi, cap))
    return out


@pytest.mark.parametrize("case", range(36))
def test_plan_equals_reference_functions(port, ref_plan, case):
    n, shape, kind, limits, lo, hi, cap = cases()[case]
    lengths = lengths_of(n)
    r = ref_plan(n, lengths, limits, lo, hi, cap)
    o = oracle_plan(port, n, lengths, limits, lo, hi, cap)
    assert (r is None) == (o is None), (kind, r, o)
    if r is None:
        return
    np.testing.assert_array_equal(o[0], r[0])
    assert o[1] == r[1] and o[2] == r[2], (o[1:], r[1:])


def test_some_cases_take_every_branch(port, ref_plan):
    """The cases reach the cap branch (every period 1), plans with several periods, and the abort."""
    seen = set()
    for n, shape, kind, limits, lo, hi, cap in cases():
        r = ref_plan(n, lengths_of(n), limits, lo, hi, cap)
        if r is None:
            seen.add("abort")
        elif r[2] == 1:
            seen.add("one period")
        else:
            seen.add("several periods")
    assert seen == {"abort", "one period", "several periods"}, seen


def test_plan_equals_committed_reference_plans(port):
    """The same pin against the reference's plans stored in tests/golden/substep_plan.npz (made by
    tests/golden/make_substep_golden.py), so that it also runs where the reference tree is absent."""
    gold = np.load(GOLD)
    for i, (n, shape, kind, limits, lo, hi, cap) in enumerate(cases()):
        o = oracle_plan(port, n, lengths_of(n), limits, lo, hi, cap)
        if int(gold[f"c{i}_abort"]):
            assert o is None, i
            continue
        np.testing.assert_array_equal(o[0], gold[f"c{i}_periods"])
        assert o[1] == float(gold[f"c{i}_substep"]) and o[2] == int(gold[f"c{i}_max"]), i
