"""Slab decomposition on the device: a grid cut into z slabs (contexts with BC_EXTERNAL cut
sides) must step bit for bit like the whole grid, once the cut planes are exchanged and the speed
reductions merged after every step.  One GPU holds every slab here (each its own context and
stream); the halo copies and the merge are done with torch between the steps, in the order
pamhd_b200.slabs does them over torch.distributed with one slab per GPU: either after whole
steps, or (split) between the two parts of each step, the new cut planes first, the interior
after, as SlabGrid.steps overlaps the exchange with the interior."""
import numpy as np
import pytest
import torch

import pamhd_b200 as pg
from pamhd_b200 import slabs
import states

pytestmark = pytest.mark.gpu


def run_slabs(cfg, U, world, steps, split=False):
    parts = []
    for r in range(world):
        local, z0 = slabs.slab_config(cfg, world, r)
        lo, hi = slabs.neighbours(cfg, world, r)
        ctx = pg.Context(local)
        ctx.set_state(U[:, z0:z0 + local.n[2]])
        parts.append((ctx, lo, hi))
    dev = torch.device("cuda", 0)

    def planes(ctx, side, ghost):
        ptrs, count = ctx.halo(side, ghost)
        return [slabs.device_tensor(p, count, torch.float64, dev) for p in ptrs]

    def exchange():
        torch.cuda.synchronize()
        for ctx, lo, hi in parts:
            if lo is not None:
                for d, s in zip(planes(ctx, 0, 1), planes(parts[lo][0], 1, 0)):
                    d.copy_(s)
            if hi is not None:
                for d, s in zip(planes(ctx, 1, 1), planes(parts[hi][0], 0, 0)):
                    d.copy_(s)
        torch.cuda.synchronize()

    def merge():
        torch.cuda.synchronize()
        slots = [slabs.device_tensor(ctx.speed_slot(), 4, torch.int64, dev) for ctx, _, _ in parts]
        m = slots[0].clone()
        for s in slots[1:]:
            m = torch.maximum(m, s)
        for s in slots:
            s.copy_(m)
        torch.cuda.synchronize()

    exchange()
    for _ in range(steps + 1):  # the priming step, then `steps` steps
        if split:
            # the new first and last planes of every slab, their exchange (the halo addresses are
            # the new state's between the parts), then the planes between
            for ctx, _, _ in parts:
                ctx.step_part(1, 1e30)
            exchange()
            for ctx, _, _ in parts:
                ctx.step_part(2, 1e30)
        else:
            for ctx, _, _ in parts:
                ctx.steps(1, 1e30)
            exchange()
        merge()
    for ctx, _, _ in parts:
        ctx.sync()
    out = np.concatenate([ctx.get_state() for ctx, _, _ in parts], axis=1)
    dts = [ctx.dt_history(steps + 1) for ctx, _, _ in parts]
    for ctx, _, _ in parts:
        ctx.close()
    return out, dts


def run_whole(cfg, U, steps):
    ctx = pg.Context(cfg)
    ctx.set_state(U)
    ctx.steps(steps + 1, 1e30)
    ctx.sync()
    out, dts = ctx.get_state(), ctx.dt_history(steps + 1)
    ctx.close()
    return out, dts


CASES = {
    "periodic": dict(bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "copy_sides": dict(bc_lo=(pg.BC_COPY, pg.BC_COPY, pg.BC_COPY), bc_hi=(pg.BC_COPY, pg.BC_COPY, pg.BC_COPY)),
    "x_copy_z_periodic": dict(bc_lo=(pg.BC_COPY, 0, 0), bc_hi=(pg.BC_COPY, 0, 0)),
    "z_inflow": dict(bc_lo=(0, 0, pg.BC_VALUE), bc_hi=(0, 0, pg.BC_COPY)),
}


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("solver", [pg.HLLD, pg.HLL])
def test_slabs_match_the_whole_grid(case, world, solver):
    rng = np.random.default_rng(17)
    nz, ny, nx = 12, 10, 14
    U = states.smooth_3d((nz, ny, nx), rng, amp=0.1)
    kw = dict(CASES[case])
    if case == "z_inflow":
        kw["value_lo"] = [None, None, U[:, 0, 0, 0].copy()]
    cfg = pg.Config(n=(nx, ny, nz), solver=solver, cell_length=(0.1, 0.12, 0.09), time_step_factor=0.4, **kw)
    steps = 8
    whole, dts = run_whole(cfg, U, steps)
    cut, slab_dts = run_slabs(cfg, U, world, steps)
    for d in slab_dts:
        assert np.array_equal(d, dts)
    assert np.array_equal(cut, whole)


@pytest.mark.parametrize("world,case,nz", [(2, "periodic", 12), (3, "z_inflow", 12), (3, "copy_sides", 7)])
@pytest.mark.parametrize("solver", [pg.HLLD, pg.ROE])
def test_split_steps_match_the_whole_grid(case, world, nz, solver):
    """Steps in two parts with the exchange between them (slabs of 2 to 4 planes, so part 2 has
    nothing to do on some) step like the whole grid, bit for bit."""
    rng = np.random.default_rng(19)
    ny, nx = 9, 11
    U = states.smooth_3d((nz, ny, nx), rng, amp=0.1)
    kw = dict(CASES[case])
    if case == "z_inflow":
        kw["value_lo"] = [None, None, U[:, 0, 0, 0].copy()]
    cfg = pg.Config(n=(nx, ny, nz), solver=solver, cell_length=(0.1, 0.12, 0.09), time_step_factor=0.4, **kw)
    steps = 6
    whole, dts = run_whole(cfg, U, steps)
    cut, slab_dts = run_slabs(cfg, U, world, steps, split=True)
    for d in slab_dts:
        assert np.array_equal(d, dts)
    assert np.array_equal(cut, whole)


def test_split_step_of_one_context_equals_a_step():
    """On a single context (no exchange), part 1 then part 2 is one step; the parts alternate and a
    whole step is refused between them."""
    rng = np.random.default_rng(23)
    n = (10, 8, 9)
    U = states.smooth_3d(n[::-1], rng, amp=0.1)
    cfg = pg.Config(n=n, solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1), time_step_factor=0.4,
                    bc_lo=(pg.BC_COPY, 0, pg.BC_COPY), bc_hi=(pg.BC_COPY, 0, pg.BC_COPY))
    whole, dts = run_whole(cfg, U, 4)
    ctx = pg.Context(cfg)
    try:
        ctx.set_state(U)
        with pytest.raises(pg.PamhdError) as e:
            ctx.step_part(2, 1e30)
        assert e.value.code == pg.ERR_STATE
        for _ in range(5):
            ctx.step_part(1, 1e30)
            for refused in (lambda: ctx.step_part(1, 1e30), lambda: ctx.steps(1, 1e30)):
                with pytest.raises(pg.PamhdError) as e:
                    refused()
                assert e.value.code == pg.ERR_STATE
            ctx.step_part(2, 1e30)
        ctx.sync()
        assert np.array_equal(ctx.get_state(), whole)
        assert np.array_equal(ctx.dt_history(5), dts)
    finally:
        ctx.close()
    flat = pg.Context(pg.Config(n=(8, 8, 1), solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1)))
    try:
        flat.set_state(states.smooth_3d((1, 8, 8), rng, amp=0.1))
        with pytest.raises(pg.PamhdError) as e:
            flat.step_part(1, 1e30)
        assert e.value.code == pg.ERR_ARGUMENT
    finally:
        flat.close()
