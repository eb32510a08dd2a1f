"""Local time stepping on the GPU (pamhd_gpu_substep_*, through the C ABI) against the CPU oracle
(oracle/substep.hpp): periods, substep counts and step lengths, and the state after every step
within 1e-12 of each field's largest magnitude (the cell-centred bar: the face solves round
differently, the updates follow the oracle's order)."""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states
from test_substep_oracle import regions

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12


def err(a, b):
    a, b = a.reshape(8, -1), b.reshape(8, -1)
    worst = 0.0
    for rows in ([0], [1, 2, 3], [4], [5, 6, 7]):
        worst = max(worst, float(np.abs(a[rows] - b[rows]).max() / max(np.abs(b[rows]).max(), 1e-300)))
    return worst


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("shape", [(1, 12, 12), (6, 8, 10), (1, 1, 40)])
def test_regional_periods_match_oracle(port, solver, shape):
    n = (shape[2], shape[1], shape[0])
    L = (0.1, 0.1, 0.1)
    U = states.smooth_3d(shape, np.random.default_rng(2))
    cfg = dict(n=n, solver=po.SOLVERS[solver], cell_length=L, adiabatic_index=states.GAMMA_53, time_step_factor=0.4)
    gpu = pg.SubstepContext(pg.Config(**cfg))
    ora = port.substep_grid(po.make_cfg(n, po.SOLVERS[solver], L, states.GAMMA_53, 1.0, 0.4))
    if shape[1] > 1:
        e = regions(shape)
    else:
        x = (np.arange(shape[2]) + 0.5) / shape[2] - 0.5
        e = np.broadcast_to(np.where(x < 0, 0, 2)[None, None, :], shape).astype(np.int32)
    gpu.set_state(U)
    ora.set_state(U)
    gpu.set_exponents(e, e)
    ora.set_exponents(e, e)
    for s in range(6):
        cap = 0.0 if s == 0 else 1.0
        dg, kg = gpu.step(cap)
        do, ko, po_, flag = ora.step(cap)
        assert flag == 0 and kg == ko
        assert abs(dg - do) <= 1e-13 * max(do, 1e-300)
        np.testing.assert_array_equal(gpu.periods(), po_)
        assert err(gpu.get_state(), ora.get_state()) <= STEP_TOL, s


def test_zero_exponents_are_the_plain_step():
    shape, n, L = (4, 6, 8), (8, 6, 4), (0.1, 0.12, 0.09)
    U = states.smooth_3d(shape, np.random.default_rng(3))
    cfg = pg.Config(n=n, solver=pg.HLLD, cell_length=L, time_step_factor=0.4)
    a, b = pg.SubstepContext(cfg), pg.Context(cfg)
    a.set_state(U)
    b.set_state(U)
    for s in range(5):
        cap = 0.0 if s == 0 else 1.0
        da, k = a.step(cap)
        db = b.step(cap)
        assert k == 1 and abs(da - db) <= 1e-13 * max(db, 1e-300)
        assert err(a.get_state(), b.get_state()) <= STEP_TOL
    out = np.zeros_like(U)
    assert a.get_state(out=out) is out   # the caller's array, filled in place
    assert np.array_equal(out, a.get_state())


def test_failure_is_reported():
    shape, n, L = (4, 4, 4), (4, 4, 4), (0.1, 0.1, 0.1)
    U = states.smooth_3d(shape, np.random.default_rng(4))
    U[4, 1, 2, 3] = 1e-3
    ctx = pg.SubstepContext(pg.Config(n=n, solver=pg.HLL, cell_length=L))
    ctx.set_state(U)
    with pytest.raises(pg.PhysicsError) as e:
        ctx.step(0.0)
    assert e.value.flags != 0


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena", "hlld_athena", "roe_athena"])
@pytest.mark.parametrize("name", ["forced_periods_3d", "slow_half_2d"])
def test_matches_reference_substep_loop(name, solver):
    """The GPU's substepped step against the reference's own substep loop (the options' exponent
    bounds per cell, the plan and the substeps of timestep(), compiled unchanged; committed
    outputs, see test_cell_centred_ref_pin.py): eight steps, step lengths within 1e-13, largest
    periods equal, state within 1e-12."""
    import test_cell_centred_ref_pin as R
    U, dts, top = R.sub_golden(name, solver)
    n, lengths = R.SUB_CASES[name]
    U0, smin, smax = R.sub_case(name)
    cfg = pg.Config(n=n, solver=R.SOLVERS[solver], cell_length=lengths, adiabatic_index=states.GAMMA_53,
                    time_step_factor=0.4)
    with pg.SubstepContext(cfg) as gpu:
        gpu.set_state(U0)
        gpu.set_exponents(smin, smax)
        got = [gpu.step(0.0 if s == 0 else 1e300) for s in range(R.SUB_STEPS)]
        Ug = gpu.get_state()
    assert np.abs(np.array([g[0] for g in got]) - dts).max() <= 1e-13 * dts.max()
    assert np.array_equal(np.array([g[1] for g in got]), top)
    assert err(Ug, U) <= STEP_TOL
