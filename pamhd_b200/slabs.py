"""One grid split into z slabs, one slab per GPU (one process per GPU).

The reference distributes a grid over MPI ranks with dccrg and updates the
remote neighbours of each rank's cells between flux computations
(mhd/solve.hpp:1767-1791); the timestep is the minimum over all ranks
(mhd/solve.hpp:1933-2014, reduced over ranks).  Here a uniform grid is cut
along z into contiguous slabs:

  * each slab is an ordinary context whose cut z sides are BC_EXTERNAL:
    the step kernel computes the faces between the ghost plane and the
    slab like any other face, but never writes the ghost plane;
  * every step is split in two launches (pamhd_gpu_step_part): first the
    new state of the slab's first and last planes, then the planes between;
    as soon as the first launch is done each slab sends its new first and
    last planes to the neighbouring slabs' new ghost planes (exchange_halos:
    one batch of point-to-point sends / receives over torch.distributed,
    NCCL on GPUs, on a stream of its own) while the second launch computes
    the interior, as the reference posts its remote-neighbour copies, solves
    the inner cells and then waits for the copies (mhd/solve.hpp:1767-1802);
    after set_state the current planes are exchanged once;
  * the speed reduction the next step takes its dt from is combined by an
    element-wise max over all slabs (merge_speeds: one all-reduce of four
    64-bit words), so every slab takes the grid's dt.  The dt rule is
    lagged (the speeds of step n give the dt of step n + 1), so nothing
    waits for the reduction until the next step begins.

All of it is ordered on the context's stream: no host synchronisation per
step.  A single-slab grid (world size 1) keeps its own boundaries and needs
no exchange.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from . import BC_EXTERNAL, BC_PERIODIC, Config, Context

# message tags: a plane travelling to the higher / lower neighbour
TAG_UP, TAG_DOWN = 1, 2


def slab_bounds(nz: int, world: int, rank: int) -> tuple[int, int]:
    """(first plane, planes) of `rank`'s slab: nz planes split as evenly as possible, the first
    nz % world slabs one plane thicker."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(nz, world)
    planes = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    if world > 1 and planes < 2:
        raise ValueError(f"{nz} z planes cannot be cut into {world} slabs of two planes or more")
    return first, planes


def neighbours(cfg: Config, world: int, rank: int) -> tuple[int | None, int | None]:
    """Ranks holding the slabs below and above `rank`'s (None at a non-periodic grid side)."""
    if world == 1:
        return None, None
    periodic = cfg.bc_lo[2] == BC_PERIODIC
    lo = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic else None)
    return lo, hi


def slab_config(cfg: Config, world: int, rank: int) -> tuple[Config, int]:
    """The configuration of `rank`'s slab and the global index of its first plane."""
    if cfg.n[2] < 2 and world > 1:
        raise ValueError("a grid without z faces cannot be cut along z")
    first, planes = slab_bounds(int(cfg.n[2]), world, rank)
    if world == 1:
        return cfg, 0
    lo, hi = neighbours(cfg, world, rank)
    bc_lo, bc_hi = list(cfg.bc_lo), list(cfg.bc_hi)
    value_lo, value_hi = list(cfg.value_lo), list(cfg.value_hi)
    if lo is not None:
        bc_lo[2] = BC_EXTERNAL
        value_lo[2] = None
    if hi is not None:
        bc_hi[2] = BC_EXTERNAL
        value_hi[2] = None
    local = replace(cfg, n=(cfg.n[0], cfg.n[1], planes), bc_lo=tuple(bc_lo), bc_hi=tuple(bc_hi),
                    value_lo=value_lo, value_hi=value_hi)
    return local, first


def exchange_halos(comm, lo: int | None, hi: int | None, send_lo, send_hi, recv_lo, recv_hi) -> None:
    """Point-to-point exchange of the cut planes: send_lo / send_hi (eight tensors each, the first
    and last interior planes) go to the lower / upper neighbour, whose planes arrive in recv_lo /
    recv_hi (the ghost planes).  Posting order and tags agree on both ends, so that with two
    slabs on a periodic grid (both neighbours the same rank) each message still lands in the
    right plane: every rank first sends up then down, and first receives from below then from
    above."""
    import torch.distributed as dist
    ops = []
    for v in range(8):
        if hi is not None:
            ops.append(dist.P2POp(dist.isend, send_hi[v], hi, comm, TAG_UP))
        if lo is not None:
            ops.append(dist.P2POp(dist.isend, send_lo[v], lo, comm, TAG_DOWN))
        if lo is not None:
            ops.append(dist.P2POp(dist.irecv, recv_lo[v], lo, comm, TAG_UP))
        if hi is not None:
            ops.append(dist.P2POp(dist.irecv, recv_hi[v], hi, comm, TAG_DOWN))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


def merge_speeds(comm, slot) -> None:
    """Element-wise max over all slabs of the four 64-bit words of a speed reduction (the maxima
    are non-negative doubles, whose bit patterns order like the doubles; the flag word is 0 or
    1), in place."""
    import torch.distributed as dist
    dist.all_reduce(slot, op=dist.ReduceOp.MAX, group=comm)


def device_tensor(ptr: int, count: int, dtype, device):
    """A torch tensor over `count` elements at device address `ptr` (no copy)."""
    import torch

    typestr = {torch.float64: "<f8", torch.int64: "<i8"}[dtype]

    class _View:
        __cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                    "version": 2, "strides": None}

    t = torch.as_tensor(_View(), device=device)
    assert t.data_ptr() == ptr and t.dtype == dtype
    return t


def overlapped_steps(n: int, boundary, exchange_new, interior, finish) -> None:
    """The order of n split steps: boundary() computes the new first and last planes,
    exchange_new() starts sending them and receiving the neighbours' into the new ghost planes
    (returning what finish needs to wait for), interior() computes the planes between while the
    exchange is in flight, finish(pending) waits for the exchange and merges the speed
    reductions.  Shared by SlabGrid and its CPU tests."""
    for _ in range(int(n)):
        boundary()
        pending = exchange_new()
        interior()
        finish(pending)


class SlabGrid:
    """This rank's slab of a grid cut along z, on this rank's GPU (cfg.device), exchanging with
    the other ranks of `comm` (a torch.distributed group; None = the default group)."""

    def __init__(self, cfg: Config, comm=None, world: int | None = None, rank: int | None = None):
        import torch
        import torch.distributed as dist
        if world is None:
            world = dist.get_world_size(comm) if dist.is_initialized() else 1
        if rank is None:
            rank = dist.get_rank(comm) if dist.is_initialized() else 0
        self.world, self.rank, self.comm = world, rank, comm
        self.global_cfg = cfg
        self.cfg, self.z0 = slab_config(cfg, world, rank)
        self.lo, self.hi = neighbours(cfg, world, rank)
        self.ctx = Context(self.cfg)
        self.device = torch.device("cuda", cfg.device)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream(), device=self.device)
        self.comm_stream = torch.cuda.Stream(device=self.device) if world > 1 else None
        self._halos = {}   # address of the current state's first plane -> the four plane lists
        self._slots = {}   # address of a reduction slot -> tensor

    # -- the exchange, on the context's stream
    def halo_tensors(self):
        """(send_lo, send_hi, recv_lo, recv_hi) of the current state, eight tensors each."""
        import torch
        key = self.ctx.halo(0, 0)[0][0]
        if key not in self._halos:
            views = []
            for side, ghost in ((0, 0), (1, 0), (0, 1), (1, 1)):
                ptrs, count = self.ctx.halo(side, ghost)
                views.append([device_tensor(p, count, torch.float64, self.device) for p in ptrs])
            self._halos[key] = tuple(views)
        return self._halos[key]

    def speed_tensor(self):
        import torch
        ptr = self.ctx.speed_slot()
        if ptr not in self._slots:
            self._slots[ptr] = device_tensor(ptr, 4, torch.int64, self.device)
        return self._slots[ptr]

    def exchange(self):
        if self.world == 1:
            return
        import torch
        send_lo, send_hi, recv_lo, recv_hi = self.halo_tensors()
        with torch.cuda.stream(self.stream):
            exchange_halos(self.comm, self.lo, self.hi, send_lo, send_hi, recv_lo, recv_hi)

    def exchange_async(self):
        """Between the two parts of a split step: sends the new first and last planes and receives
        the neighbours' into the new ghost planes, on the communication stream once the first part
        is done; returns the event that marks the exchange complete."""
        import torch
        ready = torch.cuda.Event()
        ready.record(self.stream)
        self.comm_stream.wait_event(ready)
        send_lo, send_hi, recv_lo, recv_hi = self.halo_tensors()
        with torch.cuda.stream(self.comm_stream):
            exchange_halos(self.comm, self.lo, self.hi, send_lo, send_hi, recv_lo, recv_hi)
        done = torch.cuda.Event()
        done.record(self.comm_stream)
        return done

    def finish_step(self, exchanged):
        """The step's end: the context's stream waits for the exchange, then the speed merge."""
        self.stream.wait_event(exchanged)
        self.merge()

    def merge(self):
        if self.world == 1:
            return
        import torch
        with torch.cuda.stream(self.stream):
            merge_speeds(self.comm, self.speed_tensor())

    # -- the Context interface, slab-wise
    def set_state(self, U_local: np.ndarray):
        """U_local: this slab's (8, planes, ny, nx) part of the grid's state."""
        self.ctx.set_state(U_local)
        self.exchange()

    def set_state_device(self, ptrs):
        self.ctx.set_state_device(ptrs)
        self.exchange()

    def get_state(self, out=None):
        return self.ctx.get_state(out)

    def get_state_device(self, ptrs):
        self.ctx.get_state_device(ptrs)

    def steps(self, n: int, t_end: float):
        """n steps (the first after set_state is the dt = 0 priming step), each split so that the
        halo exchange of its new cut planes overlaps the computation of its interior, then the
        speed merge; nothing here waits for the GPU."""
        if self.world == 1:
            self.ctx.steps(n, t_end)
            return
        overlapped_steps(n, lambda: self.ctx.step_part(1, t_end), self.exchange_async,
                         lambda: self.ctx.step_part(2, t_end), self.finish_step)

    def sync(self):
        self.ctx.sync()

    def time(self):
        return self.ctx.time()

    def close(self):
        self.ctx.close()
