"""Host logic of the z-slab decomposition (pamhd_b200/slabs.py) on CPU: slab bounds, neighbours,
slab configurations, and the halo exchange and speed merge over torch.distributed with the gloo
backend, world sizes 2 and 3.  The ranks step a seeded 3-D field with a stencil that reads the
z neighbours (the role the MHD step plays on the GPU) and must reproduce the whole-grid result
bit for bit; the merged speed slot must equal the maximum over the whole grid."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import pamhd_b200 as pg
from pamhd_b200 import slabs


def test_slab_bounds_cover_the_grid():
    for nz in (2, 7, 64, 257):
        for world in range(1, 5):
            if world > 1 and nz // world < 2:
                with pytest.raises(ValueError):
                    [slabs.slab_bounds(nz, world, r) for r in range(world)]
                continue
            parts = [slabs.slab_bounds(nz, world, r) for r in range(world)]
            assert parts[0][0] == 0
            for (a, n), (b, _) in zip(parts, parts[1:]):
                assert a + n == b
            assert parts[-1][0] + parts[-1][1] == nz
            assert max(p[1] for p in parts) - min(p[1] for p in parts) <= 1


def test_neighbours_and_configs():
    per = pg.Config(n=(8, 8, 12), solver=pg.HLLD, cell_length=(1, 1, 1))
    assert slabs.neighbours(per, 1, 0) == (None, None)
    assert slabs.neighbours(per, 2, 0) == (1, 1)
    assert slabs.neighbours(per, 3, 0) == (2, 1)
    assert slabs.neighbours(per, 3, 2) == (1, 0)
    c, z0 = slabs.slab_config(per, 3, 1)
    assert c.n == (8, 8, 4) and z0 == 4
    assert c.bc_lo[2] == pg.BC_EXTERNAL and c.bc_hi[2] == pg.BC_EXTERNAL
    assert c.bc_lo[:2] == per.bc_lo[:2]
    inflow = [1.0, 0, 0, 0, 2.0, 0, 0, 0]
    wall = pg.Config(n=(8, 8, 12), solver=pg.HLL, cell_length=(1, 1, 1),
                     bc_lo=(pg.BC_PERIODIC, pg.BC_PERIODIC, pg.BC_VALUE),
                     bc_hi=(pg.BC_PERIODIC, pg.BC_PERIODIC, pg.BC_COPY),
                     value_lo=[None, None, inflow])
    assert slabs.neighbours(wall, 3, 0) == (None, 1)
    assert slabs.neighbours(wall, 3, 2) == (1, None)
    c0, _ = slabs.slab_config(wall, 3, 0)
    c2, _ = slabs.slab_config(wall, 3, 2)
    assert c0.bc_lo[2] == pg.BC_VALUE and c0.value_lo[2] == inflow and c0.bc_hi[2] == pg.BC_EXTERNAL
    assert c2.bc_lo[2] == pg.BC_EXTERNAL and c2.bc_hi[2] == pg.BC_COPY
    same, z0 = slabs.slab_config(wall, 1, 0)
    assert same is wall and z0 == 0


def test_external_sides_validated_by_the_library():
    """EXTERNAL is a z-only kind and needs z faces; argument checks run before any CUDA call."""
    import ctypes
    from pamhd_b200 import build
    build.build()
    L = pg.lib()
    bad = [
        dict(n=(8, 8, 8), bc_lo=(pg.BC_EXTERNAL, 0, 0), bc_hi=(pg.BC_COPY, 0, 0)),   # x cut
        dict(n=(8, 8, 1), bc_lo=(0, 0, pg.BC_EXTERNAL), bc_hi=(0, 0, pg.BC_EXTERNAL)),  # no z faces
        dict(n=(8, 8, 8), bc_lo=(0, 0, pg.BC_EXTERNAL), bc_hi=(0, 0, pg.BC_PERIODIC)),  # half periodic
    ]
    for kw in bad:
        cfg = pg.Config(solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1), **kw).to_c()
        h = ctypes.c_void_p()
        assert L.pamhd_gpu_create(ctypes.byref(cfg), ctypes.byref(h)) == pg.ERR_ARGUMENT, kw


# ---------------------------------------------------------------- exchange over gloo

def field(nz, ny, nx, seed=5):
    return np.random.default_rng(seed).normal(size=(8, nz, ny, nx))


def stencil(G):
    """One update of a padded (8, nz + 2, ny, nx) field from its z ghosts and x / y periodic
    neighbours; returns the new interior and per-variable 'speeds' (a non-negative max)."""
    c = G[:, 1:-1]
    new = c + 0.1 * (G[:, :-2] - 2 * c + G[:, 2:]) + 0.05 * (np.roll(c, 1, 3) - np.roll(c, -1, 2))
    return new, np.abs(new).max(axis=(1, 2, 3))[:3]


def whole_grid(U, steps, periodic):
    G = np.zeros((8, U.shape[1] + 2) + U.shape[2:])
    G[:, 1:-1] = U
    speeds = []
    for _ in range(steps):
        if periodic:
            G[:, 0], G[:, -1] = G[:, -2], G[:, 1]
        else:
            G[:, 0], G[:, -1] = G[:, 1], G[:, -2]     # copy ends
        new, s = stencil(G)
        G[:, 1:-1] = new
        speeds.append(s)
    return G[:, 1:-1], speeds


def _rank_main(rank, world, port, periodic, steps, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nz, ny, nx = 12, 5, 6
        cfg = pg.Config(n=(nx, ny, nz), solver=pg.HLLD, cell_length=(1, 1, 1),
                        bc_lo=(0, 0, 0 if periodic else pg.BC_COPY), bc_hi=(0, 0, 0 if periodic else pg.BC_COPY))
        local, z0 = slabs.slab_config(cfg, world, rank)
        lo, hi = slabs.neighbours(cfg, world, rank)
        nzl = local.n[2]
        U = field(nz, ny, nx)
        G = np.zeros((8, nzl + 2, ny, nx))
        G[:, 1:-1] = U[:, z0:z0 + nzl]
        T = torch.from_numpy(G)   # shares memory with G
        send_lo = [T[v, 1] for v in range(8)]
        send_hi = [T[v, nzl] for v in range(8)]
        recv_lo = [T[v, 0] for v in range(8)]
        recv_hi = [T[v, nzl + 1] for v in range(8)]
        merged = []
        for _ in range(steps):
            slabs.exchange_halos(None, lo, hi, send_lo, send_hi, recv_lo, recv_hi)
            if lo is None:
                G[:, 0] = G[:, 1]
            if hi is None:
                G[:, -1] = G[:, -2]
            new, s = stencil(G)
            G[:, 1:-1] = new
            slot = torch.tensor(np.append(s, 0.0).view(np.int64).copy())
            slabs.merge_speeds(None, slot)
            merged.append(slot.numpy().view(np.float64)[:3].copy())
        np.save(os.path.join(out, f"slab{rank}.npy"), G[:, 1:-1])
        np.save(os.path.join(out, f"speeds{rank}.npy"), np.array(merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _rank_overlapped(rank, world, port, periodic, steps, out):
    """The split step of SlabGrid.steps (slabs.overlapped_steps) with the same stand-in stencil: the
    new first and last planes first, their exchange into the new ghost planes, then the planes
    between, into a second buffer (ping-pong, as the contexts' states)."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nz, ny, nx = 12, 5, 6
        cfg = pg.Config(n=(nx, ny, nz), solver=pg.HLLD, cell_length=(1, 1, 1),
                        bc_lo=(0, 0, 0 if periodic else pg.BC_COPY), bc_hi=(0, 0, 0 if periodic else pg.BC_COPY))
        local, z0 = slabs.slab_config(cfg, world, rank)
        lo, hi = slabs.neighbours(cfg, world, rank)
        nzl = local.n[2]
        U = field(nz, ny, nx)
        bufs = [np.zeros((8, nzl + 2, ny, nx)) for _ in range(2)]
        bufs[0][:, 1:-1] = U[:, z0:z0 + nzl]
        cur = [0]
        merged, speeds = [], []

        def planes(G):
            T = torch.from_numpy(G)
            return ([T[v, 1] for v in range(8)], [T[v, nzl] for v in range(8)],
                    [T[v, 0] for v in range(8)], [T[v, nzl + 1] for v in range(8)])

        def ends(G):
            if lo is None:
                G[:, 0] = G[:, 1]
            if hi is None:
                G[:, -1] = G[:, -2]

        # the current planes once, as after set_state
        slabs.exchange_halos(None, lo, hi, *planes(bufs[0]))
        ends(bufs[0])

        def boundary():
            G, N = bufs[cur[0]], bufs[cur[0] ^ 1]
            new, _ = stencil(G)
            N[:, 1], N[:, nzl] = new[:, 0], new[:, -1]

        def exchange_new():
            slabs.exchange_halos(None, lo, hi, *planes(bufs[cur[0] ^ 1]))

        def interior():
            G, N = bufs[cur[0]], bufs[cur[0] ^ 1]
            new, s = stencil(G)
            N[:, 2:nzl] = new[:, 1:-1]
            speeds.append(s)

        def finish(_):
            ends(bufs[cur[0] ^ 1])
            slot = torch.tensor(np.append(speeds[-1], 0.0).view(np.int64).copy())
            slabs.merge_speeds(None, slot)
            merged.append(slot.numpy().view(np.float64)[:3].copy())
            cur[0] ^= 1

        slabs.overlapped_steps(steps, boundary, exchange_new, interior, finish)
        np.save(os.path.join(out, f"slab{rank}.npy"), bufs[cur[0]][:, 1:-1])
        np.save(os.path.join(out, f"speeds{rank}.npy"), np.array(merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_gloo_slabs_reproduce_the_whole_grid(tmp_path, world, periodic):
    steps = 4
    mp.start_processes(_rank_main, args=(world, free_port(), periodic, steps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    U = field(12, 5, 6)
    ref, speeds = whole_grid(U, steps, periodic)
    parts = [np.load(tmp_path / f"slab{r}.npy") for r in range(world)]
    assert np.array_equal(np.concatenate(parts, axis=1), ref)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"speeds{r}.npy"), np.array(speeds))


@pytest.mark.parametrize("world,periodic", [(2, True), (3, False)])
def test_gloo_overlapped_schedule_reproduces_the_whole_grid(tmp_path, world, periodic):
    """The split step's order: exchanging the new cut planes before the interior is computed gives
    the whole grid's result, bit for bit."""
    steps = 4
    mp.start_processes(_rank_overlapped, args=(world, free_port(), periodic, steps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    U = field(12, 5, 6)
    ref, speeds = whole_grid(U, steps, periodic)
    parts = [np.load(tmp_path / f"slab{r}.npy") for r in range(world)]
    assert np.array_equal(np.concatenate(parts, axis=1), ref)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"speeds{r}.npy"), np.array(speeds))
