"""Time-stamped inflow of VALUE sides (pamhd_gpu_set_inflow, pamhd_gpu_batch_set_inflow): the
solar-wind boundary of the reference (mhd/solar_wind_box.hpp:227-268), whose ghost state is the
table entry selected by how many timestamps the simulation time has passed.  The GPU writes the
ghosts inside the step; the oracle (oracle/mode_c.hpp, Mode_C_Grid::set_inflow) sets them after
each step.  Both must agree step by step, across the switches of the table."""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu

GAMMA = 5 / 3


def inflow_state(rho, vx, p, B):
    v = np.array([[vx], [0.0], [0.0]])
    Bv = np.array(B, float).reshape(3, 1)
    E = states.energy(rho, v, p, Bv, GAMMA)[0]
    return np.array([rho, rho * vx, 0.0, 0.0, E, *B])


TABLE_STATES = np.array([inflow_state(1.0, 0.5, 0.6, (0.0, 0.3, 0.1)),
                         inflow_state(1.6, 0.9, 1.1, (0.0, 0.5, -0.2)),
                         inflow_state(0.8, 0.3, 0.4, (0.0, 0.1, 0.3))])


def field_err(a, b):
    a = a.reshape(8, -1)
    b = b.reshape(8, -1)
    scale = np.abs(b).max(axis=1)
    scale[scale == 0] = 1.0
    return float((np.abs(a - b).max(axis=1) / scale).max())


def make_case(solver):
    rng = np.random.default_rng(31)
    n = (16, 12, 10)
    U0 = states.smooth_3d((n[2], n[1], n[0]), rng, amp=0.1)
    bc_lo = (pg.BC_VALUE, pg.BC_COPY, pg.BC_PERIODIC)
    bc_hi = (pg.BC_COPY, pg.BC_COPY, pg.BC_PERIODIC)
    cfg = pg.Config(n=n, solver=solver, cell_length=(0.05, 0.06, 0.07), adiabatic_index=GAMMA,
                    time_step_factor=0.4, bc_lo=bc_lo, bc_hi=bc_hi, value_lo=[TABLE_STATES[0], None, None])
    ocfg = po.make_cfg(n, solver, (0.05, 0.06, 0.07), GAMMA, 1.0, 0.4, bc_lo, bc_hi,
                       [TABLE_STATES[0], None, None])
    return U0, cfg, ocfg


@pytest.mark.parametrize("solver", [pg.HLL, pg.HLLD])
def test_table_switches_match_oracle(port, solver):
    U0, cfg, ocfg = make_case(solver)
    gpu = pg.Context(cfg)
    ora = port.grid(ocfg, threads=4)
    gpu.set_state(U0)
    ora.set_state(U0)
    # learn the step size, then put the switches between steps 3-4 and 7-8
    gpu.step(1.0)
    dt = gpu.step(1.0)
    gpu.set_state(U0)
    times = np.array([3.5 * dt, 7.5 * dt])
    gpu.set_inflow(0, 0, times, TABLE_STATES)
    ora.set_inflow(0, 0, times, TABLE_STATES)
    t_g = t_o = 0.0
    for step in range(12):
        dg = gpu.step(1.0)
        do, flag, _, _ = ora.step(1.0)
        assert flag == 0
        assert abs(dg - do) <= 1e-12 * max(do, 1e-300) or dg == do == 0.0
        t_g += dg
        t_o += do
        assert field_err(gpu.get_state(), ora.get_state()) <= 1e-12 * (1 + step), step
    assert t_o > times[-1]   # both switches happened inside the run


def test_constant_table_equals_configured_value():
    """A table with no timestamps holds one state: the same bits as the configured VALUE side."""
    U0, cfg, _ = make_case(pg.HLL)
    a, b = pg.Context(cfg), pg.Context(cfg)
    a.set_state(U0)
    b.set_state(U0)
    b.set_inflow(0, 0, [], TABLE_STATES[:1])
    a.steps(10, 1e9)
    b.steps(10, 1e9)
    a.sync()
    b.sync()
    np.testing.assert_array_equal(a.get_state(), b.get_state())


def test_batch_tables_equal_single_contexts():
    """Two boxes with different tables, batched: the same bits as each box in its own context."""
    U0, cfg, _ = make_case(pg.HLL)
    boxes = [cfg, cfg]
    tables = [(np.array([0.004, 0.009]), TABLE_STATES), (np.array([0.006]), TABLE_STATES[1:])]
    batch = pg.Batch(boxes)
    for i in range(2):
        batch.set_state(i, U0)
        batch.set_inflow(i, 0, 0, *tables[i])
    batch.steps(14)
    batch.sync()
    for i in range(2):
        ctx = pg.Context(cfg)
        ctx.set_state(U0)
        ctx.set_inflow(0, 0, *tables[i])
        ctx.steps(14, 1e300)
        ctx.sync()
        np.testing.assert_array_equal(batch.get_state(i), ctx.get_state())
        np.testing.assert_array_equal(batch.dt_history(i, 14), ctx.dt_history(14))


def test_rejects_tables_on_other_sides():
    U0, cfg, _ = make_case(pg.HLL)
    ctx = pg.Context(cfg)
    with pytest.raises(pg.PamhdError):
        ctx.set_inflow(1, 0, [0.1], TABLE_STATES[:2])      # a COPY side
    with pytest.raises(pg.PamhdError):
        ctx.set_inflow(0, 0, [0.2, 0.1], TABLE_STATES)     # timestamps not increasing
