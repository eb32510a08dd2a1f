"""The batched ensemble (pamhd_gpu_batch_*) through the C ABI.

A batch runs the same tile code as a single-grid context, so every box of a
batch must match, bit for bit, the same box run alone; one box is also held
to the CPU oracle at the step tolerance of test_gpu_parity.py (1e-12,
field-normwise)."""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu


def wind_cfg(n, inflow, solver=pg.HLL, shape=None):
    shape = shape or (n, n, n)
    return pg.Config(n=shape, solver=solver, cell_length=(states.EARTH_RADIUS_CELL,) * 3,
                     adiabatic_index=5 / 3, vacuum_permeability=states.MU0_SI, time_step_factor=0.5,
                     bc_lo=(pg.BC_VALUE, pg.BC_COPY, pg.BC_COPY), bc_hi=(pg.BC_COPY,) * 3,
                     value_lo=[inflow, None, None])


def small_ensemble():
    boxes = states.solar_wind_ensemble(nboxes=5, sizes=(12, 17, 24, 33))
    cfgs, U0s = [], []
    for i, b in enumerate(boxes):
        n = b["n"]
        shape = (n, n + i, max(2, n - 2 * i))  # uneven boxes, not cubes
        cfgs.append(wind_cfg(n, b["inflow"], shape=shape))
        U = np.broadcast_to(b["interior"][:, None, None, None], (8, shape[2], shape[1], shape[0])).copy()
        rng = np.random.default_rng(i)
        U[0] *= 1 + 0.05 * rng.random(U[0].shape)  # some structure
        U0s.append(U)
    return cfgs, U0s


def test_batch_equals_single_contexts_bitwise():
    cfgs, U0s = small_ensemble()
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.steps(14)
    batch.sync()
    for i, (cfg, U) in enumerate(zip(cfgs, U0s)):
        ctx = pg.Context(cfg)
        ctx.set_state(U)
        ctx.steps(14, 1e300)
        ctx.sync()
        np.testing.assert_array_equal(batch.get_state(i), ctx.get_state())
        np.testing.assert_array_equal(batch.dt_history(i, 14), ctx.dt_history(14))
        assert batch.time(i) == ctx.time()


def test_boxes_take_their_own_timesteps():
    cfgs, U0s = small_ensemble()
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.steps(5)
    dts = [batch.time(i)[2] for i in range(len(cfgs))]
    assert len(set(dts)) == len(dts) and min(dts) > 0


def test_batch_box_matches_oracle(port):
    b = states.solar_wind_ensemble(nboxes=1, sizes=(20,))[0]
    n = b["n"]
    U = states.ensemble_state(b)
    U[0] *= 1 + 0.1 * np.random.default_rng(3).random(U[0].shape)
    cfg = wind_cfg(n, b["inflow"])
    batch = pg.Batch([cfg, wind_cfg(12, b["inflow"])])
    batch.set_state(0, U)
    batch.set_state(1, states.ensemble_state({"n": 12, "interior": b["interior"]}))
    ora = port.grid(po.make_cfg((n, n, n), po.HLL, (states.EARTH_RADIUS_CELL,) * 3, 5 / 3, states.MU0_SI, 0.5,
                                bc_lo=(po.BC_VALUE, po.BC_COPY, po.BC_COPY), bc_hi=(po.BC_COPY,) * 3,
                                value_lo=[b["inflow"], None, None]), threads=8)
    ora.set_state(U)
    for step in range(4):
        batch.steps(1)
        do, flag, _, _ = ora.step(1e300)
        assert flag == 0
        dg = batch.time(0)[2]
        assert abs(dg - do) <= 1e-12 * max(do, 1e-300) or dg == do == 0.0
        a = batch.get_state(0).reshape(8, -1)
        o = ora.get_state().reshape(8, -1)
        scale = np.abs(o).max(axis=1)
        scale[scale == 0] = 1.0
        assert (np.abs(a - o).max(axis=1) / scale).max() <= 1e-12 * (1 + step)


def test_configured_boxes_match_oracle_in_the_persistent_run(port):
    """Boxes of the configured ensemble (its seed, its 32^3, 64^3 and 96^3 sizes, their own winds),
    20 steps in one persistent launch, against the oracle at the per-step bar grown with the step
    count: the state and every step's dt of each box."""
    boxes = states.solar_wind_ensemble()
    picked = []
    for size in (32, 64, 96):
        picked.append(next(b for b in boxes if b["n"] == size))
    cfgs = [wind_cfg(b["n"], b["inflow"]) for b in picked]
    batch = pg.Batch(cfgs)
    for i, b in enumerate(picked):
        batch.set_state(i, states.ensemble_state(b))
    steps = 20
    batch.run(steps)
    batch.sync()
    for i, b in enumerate(picked):
        n = b["n"]
        ora = port.grid(po.make_cfg((n, n, n), po.HLL, (states.EARTH_RADIUS_CELL,) * 3, 5 / 3, states.MU0_SI, 0.5,
                                    bc_lo=(po.BC_VALUE, po.BC_COPY, po.BC_COPY), bc_hi=(po.BC_COPY,) * 3,
                                    value_lo=[b["inflow"], None, None]), threads=8)
        ora.set_state(states.ensemble_state(b))
        dts = []
        for _ in range(steps):
            do, flag, _, _ = ora.step(1e300)
            assert flag == 0
            dts.append(do)
        dg = batch.dt_history(i, steps)
        assert len(dg) == steps
        for a, o in zip(dg, dts):
            assert abs(a - o) <= 1e-12 * max(o, 1e-300) or a == o == 0.0
        a = batch.get_state(i).reshape(8, -1)
        o = ora.get_state().reshape(8, -1)
        scale = np.abs(o).max(axis=1)
        scale[scale == 0] = 1.0
        assert (np.abs(a - o).max(axis=1) / scale).max() <= 1e-12 * steps, n


@pytest.mark.parametrize("persistent", [False, True])
def test_one_dimensional_box_equals_its_context(persistent):
    """A 1-D grid (the Brio-Wu shock tube, 1000 cells, COPY ends) as a batch of one box, per-step
    launches or the persistent run, capped at t_end: the same bits, time and step count as the
    same grid in its own context."""
    U = states.brio_wu(1000)
    cfg = pg.Config(n=(1000, 1, 1), solver=pg.HLLD, cell_length=(1e-3, 1.0, 1.0), adiabatic_index=2.0,
                    time_step_factor=0.5, bc_lo=(pg.BC_COPY, 0, 0), bc_hi=(pg.BC_COPY, 0, 0))
    batch = pg.Batch([cfg])
    batch.set_state(0, U)
    ctx = pg.Context(cfg)
    ctx.set_state(U)
    for n in (7, 60, 300):
        if persistent:
            batch.run(n, 0.02)
        else:
            batch.steps(n, 0.02)
        batch.sync()
        ctx.steps(n, 0.02)
        ctx.sync()
        np.testing.assert_array_equal(batch.get_state(0), ctx.get_state())
        assert batch.time(0) == ctx.time()
    assert ctx.time()[0] == 0.02


def test_box_failing_late_in_a_persistent_run_holds_its_failing_step():
    """The 64^3 magnetised blast loses positivity after some tens of steps: run as a batch of one
    box for 80 steps in one persistent launch, it holds the state, time and step count its own
    context has right after the failing step (later steps of the launch hold the box)."""
    n = 64
    U = states.blast_wave(n)
    cfg = pg.Config(n=(n, n, n), solver=pg.HLLD, cell_length=(1 / n,) * 3, time_step_factor=0.4)
    ctx = pg.Context(cfg)
    ctx.set_state(U)
    failed = None
    for step in range(80):
        try:
            ctx.step(1e30)
        except pg.PhysicsError:
            failed = step
            break
    assert failed is not None and 5 < failed < 70
    batch = pg.Batch([cfg])
    batch.set_state(0, U)
    batch.run(80)
    with pytest.raises(pg.PhysicsError):
        batch.sync()
    np.testing.assert_array_equal(batch.get_state(0), ctx.get_state())
    t, count, _ = ctx.time()
    assert batch.time(0)[:2] == (t, count) and count == failed + 1
    np.testing.assert_array_equal(batch.dt_history(0, 100), ctx.dt_history(100))


@pytest.mark.parametrize("solver", [pg.RUSANOV, pg.HLL, pg.HLLD, 4])
def test_every_solver_gives_the_context_bits_in_every_batch_kernel(solver):
    """The 48^3 magnetised blast (periodic) with each solver: a batch of one box, tiles of 4 and of
    8 rows, per-step launches and the persistent run, against the same grid in its own context
    (32 x 8 tiles, 32 x 4 for Roe): the same bits after 6 steps."""
    n = 48
    U = states.blast_wave(n)
    cfg = pg.Config(n=(n, n, n), solver=solver, cell_length=(1 / n,) * 3, time_step_factor=0.4)
    ctx = pg.Context(cfg)
    ctx.set_state(U)
    ctx.steps(6, 1e300)
    ctx.sync()
    ref = ctx.get_state()
    for rows in (4, 8):
        for persistent in (False, True):
            batch = pg.Batch([cfg])
            batch.set_state(0, U)
            batch.set_tiling(rows, 16, 1 << 20)
            (batch.run if persistent else batch.steps)(6)
            batch.sync()
            np.testing.assert_array_equal(batch.get_state(0), ref)
            assert batch.time(0) == ctx.time()


def test_tuner_restores_state():
    cfgs, U0s = small_ensemble()
    tuned, plain = pg.Batch(cfgs), pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        tuned.set_state(i, U)
        plain.set_state(i, U)
    planes, grid = tuned.tune(2)
    assert planes in (8, 16, 32, 64) and grid >= 1
    for i, U in enumerate(U0s):
        np.testing.assert_array_equal(tuned.get_state(i), U)
    tuned.steps(9)
    plain.steps(9)
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(tuned.get_state(i), plain.get_state(i))


@pytest.mark.parametrize("tile_rows", [4, 8])
@pytest.mark.parametrize("planes", [8, 64])
def test_every_tiling_gives_the_same_bits(tile_rows, planes):
    """The tile shapes and work splits the autotuner chooses among compute every face with the
    same arithmetic: the same bits as each box in its own context."""
    cfgs, U0s = small_ensemble()
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.set_tiling(tile_rows, planes, 1 << 20)
    assert batch.tiling()[:2] == (tile_rows, planes)
    batch.steps(9)
    batch.sync()
    for i, (cfg, U) in enumerate(zip(cfgs, U0s)):
        ctx = pg.Context(cfg)
        ctx.set_state(U)
        ctx.steps(9, 1e300)
        ctx.sync()
        np.testing.assert_array_equal(batch.get_state(i), ctx.get_state())


def test_batch_reports_failing_box():
    cfgs, U0s = small_ensemble()
    U0s[2] = U0s[2].copy()
    U0s[2][4, 1, 2, 3] = 0.0  # negative pressure in box 2
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.steps(1)
    with pytest.raises(pg.PhysicsError) as e:
        batch.sync()
    assert "box 2" in str(e.value) and e.value.flags == pg.FLAG_PRESSURE
    for i in (0, 1, 3, 4):
        assert batch.status(i)[0] == 0


@pytest.mark.parametrize("persistent", [False, True])
def test_failed_box_stops_while_the_others_go_on(persistent):
    """A box whose face fails stops after that step (its state, time and step count stay, as a
    reference run aborts there) while the other boxes take every step, bit for bit as in their
    own contexts; in one launch per step and in the persistent run."""
    cfgs, U0s = small_ensemble()
    U0s[2] = U0s[2].copy()
    U0s[2][4, 1, 2, 3] = 0.0  # negative pressure in box 2: its first step fails
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.steps(1)
    with pytest.raises(pg.PhysicsError):
        batch.sync()
    held = batch.get_state(2)
    assert batch.time(2) == (0.0, 1, 0.0)
    if persistent:
        batch.run(12)
    else:
        batch.steps(12)
    with pytest.raises(pg.PhysicsError) as e:
        batch.sync()
    assert "box 2" in str(e.value)
    np.testing.assert_array_equal(batch.get_state(2), held)
    assert batch.time(2) == (0.0, 1, 0.0)
    np.testing.assert_array_equal(batch.dt_history(2, 20), [0.0])
    for i in (0, 1, 3, 4):
        assert batch.status(i)[0] == 0
        ctx = pg.Context(cfgs[i])
        ctx.set_state(U0s[i])
        ctx.steps(13, 1e300)
        ctx.sync()
        np.testing.assert_array_equal(batch.get_state(i), ctx.get_state())
        np.testing.assert_array_equal(batch.dt_history(i, 20), ctx.dt_history(20))
        assert batch.time(i) == ctx.time()


# ---------------------------------------------------------------- the persistent run


@pytest.mark.parametrize("tile_rows,planes", [(4, 8), (8, 32)])
def test_persistent_run_equals_per_step_launches_bitwise(tile_rows, planes):
    """pamhd_gpu_batch_run (every step in one launch, each box's step waiting for its previous
    one) against pamhd_gpu_batch_steps (one launch per step): the same bits, box by box, including
    the boundary-face speeds that set each box's timestep; run twice in a row (graph replay, and the
    parity and phase of the second run differ from the first's)."""
    cfgs, U0s = small_ensemble()
    a, b = pg.Batch(cfgs), pg.Batch(cfgs)
    for batch in (a, b):
        batch.set_tiling(tile_rows, planes, 1)
        for i, U in enumerate(U0s):
            batch.set_state(i, U)
    a.steps(11)
    a.steps(8)
    a.sync()
    b.run(11)
    b.run(8)
    b.sync()
    grid, items, graphed = b.run_info()
    assert grid > 1 and items > 0
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(b.get_state(i), a.get_state(i))
        np.testing.assert_array_equal(b.dt_history(i, 19), a.dt_history(i, 19))
        assert b.time(i) == a.time(i)


def test_persistent_run_tuner_restores_state():
    cfgs, U0s = small_ensemble()
    a, b = pg.Batch(cfgs), pg.Batch(cfgs)
    for batch in (a, b):
        for i, U in enumerate(U0s):
            batch.set_state(i, U)
    rows, planes = b.tune_run(2)
    assert rows in (4, 8) and planes in (8, 16, 32, 64)
    a.set_tiling(rows, planes, 1)
    a.steps(6)
    b.run(6)
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(b.get_state(i), a.get_state(i))


def test_persistent_run_wait_timeout_is_reported():
    """A wait that runs out (a limit of 0 polls: the first block to take an item of step 1 before
    its box's step 0 is done gives up at once) ends the launch with PAMHD_FLAG_TIMEOUT on every
    box and PAMHD_ERR_TIMEOUT from sync, without a fault; the batch is usable again after
    set_state."""
    cfgs, U0s = small_ensemble()
    batch = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
    batch.set_wait_limit(0)
    batch.run(5)
    with pytest.raises(pg.PamhdError) as e:
        batch.sync()
    assert e.value.code == pg.ERR_TIMEOUT
    for i in range(len(cfgs)):
        assert batch.status(i)[0] & pg.FLAG_TIMEOUT
    batch.set_wait_limit(10_000_000)
    ref = pg.Batch(cfgs)
    for i, U in enumerate(U0s):
        batch.set_state(i, U)
        ref.set_state(i, U)
    batch.run(4)
    batch.sync()
    ref.steps(4)
    ref.sync()
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(batch.get_state(i), ref.get_state(i))
