#!/usr/bin/env python
"""Benchmark of the fused FP64 finite-volume MHD step on B200.

Workload (one line of JSON on rank 0): the 3-D magnetised blast wave,
256^3 periodic cells on [-0.5, 0.5]^3, gamma 5/3, mu0 1, HLLD, CFL 0.4:
rho 1, p 0.1 (10 inside r < 0.1), B0 = (1, 1, 0)/sqrt(2) plus a seeded
random-phase divergence-free perturbation of 1% over wavenumbers 1-8.
A step is one pass of the fused kernel over all 256^3 cells.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value    cell-updates/s, K steps with the state resident in HBM, timed by
         CUDA events on the context's stream (max over ranks; N ranks run
         N independent 256^3 boxes: weak scaling, no collective in the step)
e2e      the same metric through the C ABI with host buffers: set_state
         from pinned host arrays, K steps, get_state back, all timed
roofline achieved HBM GB/s at the algorithmic 128 B per cell-update (8 FP64
         values read, 8 written) over the mean kernel duration, against the
         measured copy bandwidth
cpu_baseline  the reference's own solver code (oracle/_ref, compiled from
         the reference headers) on the host cores, on a bounded sample
--impl reference  that CPU path alone on the full configured grid, same steps,
         warm-up and segments as the GPU arm, all host threads
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "HLLD FP64 cell-updates/s at 256³ (% HBM peak); batched vs plain; adjoint/fwd cost"
UNIT = "cell-updates/s"
T_END = 1e30
BYTES_PER_CELL_UPDATE = 128  # 8 FP64 read + 8 FP64 written
CFL = 0.4
SEGMENT = 20
WARM_SEGMENTS = 5  # untimed whole segments after the warm-up steps (graph capture, clock settling)


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--n", type=int, default=256, help="cells per dimension")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the other configured workloads")
    p.add_argument("--configs-solver", default=None,
                   help="with --only configs: the Orszag-Tang run of this solver alone (rusanov, hll_athena, hlld_athena, roe_athena)")
    p.add_argument("--only", choices=["batched", "adjoint", "configs", "staggered", "two_population", "substep"],
                   help="run one section alone and print it (for profiling)")
    p.add_argument("--boxes", type=int, default=64, help="boxes of the batched section")
    p.add_argument("--batched-steps", type=int, default=500)
    p.add_argument("--no-tune", action="store_true", help="batched section without the autotuner")
    p.add_argument("--adjoint-steps", type=int, default=200)
    p.add_argument("--no-fd-check", action="store_true")
    p.add_argument("--no-staggered", action="store_true", help="skip the staggered-field section")
    p.add_argument("--staggered-n", type=int, default=256)
    p.add_argument("--staggered-steps", type=int, default=20)
    p.add_argument("--no-two-population", action="store_true", help="skip the two-population section")
    p.add_argument("--two-population-n", type=int, default=256)
    p.add_argument("--no-substep", action="store_true", help="skip the local time stepping section")
    return p.parse_args()


def workload(n):
    return {
        "workload": f"3-D magnetised blast wave, {n}^3 periodic, gamma 5/3, HLLD, CFL {CFL}, FP64",
        "cells": n ** 3,
        "solver": "hlld_athena",
        "inputs": "synthetic seeded (seed 20261203): rho 1, p 0.1 / 10 in r<0.1, B0 (1,1,0)/sqrt2 + 1% dB",
        "l2": f"state {8 * 8 * n ** 3 / 1e9:.2f} GB per copy > 126 MB L2: no flush needed",
    }


def blast_state(n):
    import states
    return states.blast_wave(n)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_count(n, key="step_kernel_hlld"):
    """A per-launch count of the step kernel from the committed ncu summary (DRAM bytes, or FP64
    flops for key step_kernel_hlld_fp64), scaled from the captured grid to n^3 cells."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and parts[0] == key:
                cells, value = float(parts[1]), float(parts[2])
                return value * (n ** 3) / cells
    except OSError:
        pass
    return None


def ncu_traffic(n):
    return ncu_count(n, "step_kernel_hlld")


def ncu_source(key):
    """The commit whose kernel source the committed count of `key` was captured from."""
    try:
        for line in open(os.path.join(ROOT, "profiles", "traffic.txt")):
            parts = line.split()
            if len(parts) >= 4 and parts[0] == key:
                return parts[3]
    except OSError:
        pass
    return None


def fp64_roof(n, kernel_ms, clocks):
    """The second roof: FP64 flops of one step (ncu count per cell-update x cells) per second
    against the chip's FP64 rate, 148 SMs x 64 FMA lanes x 2 flops at the median SM clock sampled
    during the timed region (the max clock when no sample was taken)."""
    flops = ncu_count(n, "step_kernel_hlld_fp64")
    if flops is None:
        return None
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    peak = 148 * 64 * 2 * mhz * 1e6 / 1e12
    achieved = flops / (kernel_ms / 1e3) / 1e12
    return {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "flop_per_cell_update": flops / n ** 3,
            "peak_source": f"148 SMs x 64 FP64 FMA/cycle x 2 at {mhz:.0f} MHz (nominal rate, measured clock)"}


def pinned(shape, like=None):
    """A host array in pinned (page-locked) memory, as a numpy view of a torch tensor; returns the
    tensor (to keep the memory alive) and the view, filled from `like` when given."""
    import torch
    t = torch.empty(tuple(shape), dtype=torch.float64, pin_memory=True)
    v = t.numpy()
    if like is not None:
        v[...] = like
    return t, v


def section_roofline(n, key, alg_bytes, updates, ms, clk, scope):
    """Roofline of a step of several kernels, taken as a whole: the algorithmic bytes of one step
    (the state read and written once per cell-update) over the step's measured time against the
    measured copy bandwidth; the DRAM traffic and the FP64 flops of one step from the committed
    ncu counts (profiles/traffic.txt, scaled from the captured grid to n^3 cells); the FP64 roof at
    the SM clock sampled during the timed region."""
    peak, peak_kind = peaks()
    achieved = alg_bytes * updates / (ms / 1e3) / 1e9
    out = {"bound": "hbm", "scope": scope, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": ncu_count(n, key), "traffic_scope": "one step, all its kernels",
           "traffic_source_commit": ncu_source(key),
           "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
           "algorithmic_bytes_per_cell_update": alg_bytes, "step_ms": ms}
    flops = ncu_count(n, key + "_fp64")
    if flops is not None:
        mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
        fpeak = 148 * 64 * 2 * mhz * 1e6 / 1e12
        fa = flops / (ms / 1e3) / 1e12
        out["fp64"] = {"achieved": fa, "peak": fpeak, "unit": "TFLOP/s", "frac": fa / fpeak,
                       "flop_per_cell_update": flops / updates,
                       "peak_source": f"148 SMs x 64 FP64 FMA/cycle x 2 at {mhz:.0f} MHz (nominal rate, measured clock)"}
    return out


class ClockSampler:
    """Samples SM clock and throttle reasons with NVML while the timed region runs."""

    def __init__(self, device):
        self.samples, self.reasons = [], set()
        self.stop = threading.Event()
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
        self.t = threading.Thread(target=self.run, daemon=True)

    def run(self):
        if self.nv is None:
            return
        names = {
            0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
            0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown",
        }
        while not self.stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in names.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        self.t.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        self.t.join()

    def summary(self):
        return {
            "sm_mhz": float(np.median(self.samples)) if self.samples else None,
            "sm_max_mhz": self.max_mhz,
            "reasons": sorted(self.reasons),
            "samples": len(self.samples),
        }


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_grid(U_full, n, world, threads):
    """The reference's own solver code (oracle/_ref, compiled from the reference headers; the
    restated port where that build is absent) in the restated Mode C driver on the host cores, on
    the grid the GPU arm steps: n x n x (world n) cells, the blast cube repeated along z."""
    from oracle import pyoracle as po
    kind = "reference"
    try:
        o = po.Oracle("reference")
    except Exception:
        o = po.Oracle("port")
        kind = "port"
    U = np.ascontiguousarray(np.concatenate([U_full] * world, axis=1)) if world > 1 else U_full
    cfg = po.make_cfg((n, n, n * world), po.HLLD, (1 / n, 1 / n, 1 / n), 5 / 3, 1.0, CFL)
    g = o.grid(cfg, threads=threads)
    return g, U, kind


def cpu_timed_steps(g, U, steps, warmup):
    """The GPU arm's schedule on the CPU: priming step and warm-up steps, then `steps` timed steps
    in segments of at most SEGMENT, each restarted from the initial state with its dt = 0 priming
    step outside the clock.  Returns the seconds spent in the timed steps."""
    g.set_state(U)
    g.step(T_END)  # priming
    for _ in range(min(warmup, SEGMENT - 1)):
        g.step(T_END)
    el, left = 0.0, steps
    while left > 0:
        seg = min(SEGMENT, left)
        g.set_state(U)
        g.step(T_END)
        t0 = time.perf_counter()
        for _ in range(seg):
            dt, flag, _, _ = g.step(T_END)
            if flag:
                raise RuntimeError("reference step failed")
        el += time.perf_counter() - t0
        left -= seg
    return el


def cpu_baseline(U_full, n):
    """The CPU path on the full configured grid (all host threads), a bounded number of steps
    (about 10 s of wall time); one core on a thin slab beside it (the reference runs one MPI rank
    per core, so one core is its unit of scale)."""
    threads = cpu_threads()
    g, U, kind = cpu_grid(U_full, n, 1, threads)
    g.set_state(U)
    g.step(T_END)  # priming
    t0 = time.perf_counter()
    g.step(T_END)
    one = time.perf_counter() - t0
    steps = int(max(1, min(8, 10.0 / max(one, 1e-3))))
    el = cpu_timed_steps(g, U, steps, 0)
    rate = n ** 3 * steps / el
    del g
    # one core: a periodic slab of 4 z-planes from the middle of the blast
    from oracle import pyoracle as po
    o = po.Oracle(kind)
    z0 = (n - 4) // 2
    Us = np.ascontiguousarray(U_full[:, z0:z0 + 4])
    g1 = o.grid(po.make_cfg((n, n, 4), po.HLLD, (1 / n, 1 / n, 1 / n), 5 / 3, 1.0, CFL), threads=1)
    g1.set_state(Us)
    g1.step(1.0)
    t0 = time.perf_counter()
    for _ in range(2):
        g1.step(T_END)
    el1 = time.perf_counter() - t0
    return {
        "value": rate,
        "unit": UNIT,
        "cores": threads,
        "kind": kind,
        "sample": f"{steps} HLLD steps of the full {n}^3 periodic blast after its priming step "
                  f"({el:.1f} s wall on {threads} threads, std::thread over cells)",
        "one_core": {"value": n * n * 4 * 2 / el1, "unit": UNIT,
                     "sample": f"2 HLLD steps on a {n}x{n}x4 periodic slab of the blast, 1 thread "
                               f"({el1:.1f} s wall; a separate sample, not the configured grid)"},
        "cpu": cpu_model(),
    }


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def configs_section(local, cpu=True, solver=None):
    """The other configured workloads, GPU beside the reference's solver headers on the host cores
    (a bounded sample each): cell-updates/s of the shock tube run to its end time and of 100
    Orszag-Tang 512^2 steps with each solver (the reference scheme keeps positivity that long).
    solver: the Orszag-Tang run of that solver alone (no shock tube)."""
    import torch
    import pamhd_b200 as pg
    import states
    from oracle import pyoracle as po

    def gpu_rate(cfg, U, steps, t_end):
        ctx = pg.Context(cfg)
        st = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        # the steps that advance time (a run to t_end stops moving once there)
        ctx.set_state(U)
        ctx.steps(steps + 1, t_end)
        ctx.sync()
        steps = int((ctx.dt_history(steps + 1) > 0).sum())
        best = None
        for _ in range(3):
            ctx.set_state(U)
            ctx.steps(1, t_end)
            ctx.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            ctx.steps(steps, t_end)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        ctx.sync()
        ctx.close()
        return best, steps

    def cpu_rate(ocfg, U, steps, t_end, threads):
        try:
            o = po.Oracle("reference")
        except Exception:
            o = po.Oracle("port")
        g = o.grid(ocfg, threads=threads)
        g.set_state(U)
        g.step(t_end)
        t0 = time.perf_counter()
        done = 0
        for _ in range(steps):
            dt, flag, _, _ = g.step(t_end)
            if flag or dt == 0.0:
                break
            done += 1
        return (time.perf_counter() - t0) * 1e3, done

    out = {}
    if solver is not None and solver not in po.SOLVERS:
        raise ValueError(f"--configs-solver: one of {sorted(po.SOLVERS)}")
    # shock tube: 1000 cells, gamma 2, HLLD, CFL 0.5, copy boundaries, to t = 0.1
    if solver is None:
        U = states.brio_wu(1000)
        cfg = pg.Config(n=(1000, 1, 1), solver=pg.HLLD, cell_length=(1e-3, 1.0, 1.0), adiabatic_index=2.0,
                        time_step_factor=0.5, bc_lo=(pg.BC_COPY, 0, 0), bc_hi=(pg.BC_COPY, 0, 0), device=local)
        ms, steps = gpu_rate(cfg, U, 2000, 0.1)
        entry = {"workload": "Brio-Wu 1000 cells, HLLD, CFL 0.5, to t = 0.1", "steps": steps,
                 "gpu": 1000 * steps / (ms / 1e3), "gpu_ms": ms, "unit": UNIT}
        if cpu:
            ocfg = po.make_cfg((1000, 1, 1), po.HLLD, (1e-3, 1.0, 1.0), 2.0, 1.0, 0.5, (1, 0, 0), (1, 0, 0))
            cms, csteps = cpu_rate(ocfg, U, 2000, 0.1, 1)
            entry.update(cpu_one_core=1000 * csteps / (cms / 1e3), cpu_sample=f"{csteps} steps, 1 thread")
        out["brio_wu"] = entry
    # Orszag-Tang 512^2, each solver, 100 steps
    n = 512
    U = states.orszag_tang(n)
    for name, sid in po.SOLVERS.items():
        if solver is not None and name != solver:
            continue
        cfg = pg.Config(n=(n, n, 1), solver=sid, cell_length=(1 / n, 1 / n, 1.0), adiabatic_index=5 / 3,
                        time_step_factor=0.4, device=local)
        ms, steps = gpu_rate(cfg, U, 100, 10.0)
        entry = {"workload": f"Orszag-Tang {n}^2 periodic, {name}, CFL 0.4, 100 steps", "steps": steps,
                 "gpu": n * n * steps / (ms / 1e3), "gpu_ms": ms, "unit": UNIT}
        if cpu:
            threads = cpu_threads()
            ocfg = po.make_cfg((n, n, 1), sid, (1 / n, 1 / n, 1.0), 5 / 3, 1.0, 0.4)
            cms, csteps = cpu_rate(ocfg, U, 5, 10.0, threads)
            entry.update(cpu=n * n * csteps / (cms / 1e3), cpu_cores=threads, cpu_sample=f"{csteps} steps")
        out[f"orszag_tang_{name}"] = entry
    return out


def batched_section(local, steps=500, nboxes=64, tune=True, sequential=True):
    """Batched ensemble (64 uneven SI solar-wind boxes, HLL, 500 steps) in one batch against the same
    boxes run one after another, each in its own context (sequential per-box launches)."""
    import torch
    import pamhd_b200 as pg
    import states

    boxes = states.solar_wind_ensemble(nboxes=nboxes)
    cfgs = [pg.Config(n=(b["n"],) * 3, solver=pg.HLL, cell_length=(states.EARTH_RADIUS_CELL,) * 3,
                      adiabatic_index=5 / 3, vacuum_permeability=states.MU0_SI, time_step_factor=0.5,
                      bc_lo=(pg.BC_VALUE, pg.BC_COPY, pg.BC_COPY), bc_hi=(pg.BC_COPY,) * 3,
                      value_lo=[b["inflow"], None, None], device=local) for b in boxes]
    cells = sum(b["n"] ** 3 for b in boxes)
    dev = torch.device("cuda", local)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # the persistent run: all steps of every box in one cooperative launch, graph-replayed
    batch = pg.Batch(cfgs, device=local)
    for i, b in enumerate(boxes):
        batch.set_state(i, states.ensemble_state(b))
    run_tiling = batch.tune_run(3) if tune else None
    st = torch.cuda.ExternalStream(batch.stream(), device=dev)
    batched_ms = timed(lambda: batch.run(steps))
    run_grid, run_items, graphed = batch.run_info()
    # a box whose state the reference scheme rejects stops after its failing step (later steps only
    # copy it): it is counted, not hidden, and the value counts the cell updates the boxes made
    failed = [i for i in range(len(boxes)) if batch.status(i)[0] != 0]
    taken = [batch.time(i)[1] for i in range(len(boxes))]
    updates = sum(b["n"] ** 3 * t for b, t in zip(boxes, taken))
    failed_steps = {}
    batch.close()

    # the same ensemble with one launch per step (graph-replayed), for comparison
    batch = pg.Batch(cfgs, device=local)
    for i, b in enumerate(boxes):
        batch.set_state(i, states.ensemble_state(b))
    if tune:
        batch.tune(3)
    tiling = batch.tiling()
    st = torch.cuda.ExternalStream(batch.stream(), device=dev)
    per_step_ms = timed(lambda: batch.steps(steps))
    batch.close()
    plain_ms = 0.0
    for cfg, b in zip(cfgs, boxes if sequential else []):
        ctx = pg.Context(cfg)
        ctx.set_state(states.ensemble_state(b))
        cs = torch.cuda.ExternalStream(ctx.stream(), device=dev)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        p0.record(cs)
        ctx.steps(steps, 1e300)
        p1.record(cs)
        torch.cuda.synchronize()
        plain_ms += p0.elapsed_time(p1)
        if ctx.status()[0] != 0:
            failed_steps[len(failed_steps)] = True
        ctx.close()
    batched = updates / (batched_ms / 1e3)
    healthy_cells = sum(b["n"] ** 3 for i, b in enumerate(boxes) if i not in failed)
    plain = updates / (plain_ms / 1e3) if sequential else None
    return {
        "workload": f"{len(boxes)} independent SI solar-wind boxes, edges from {{32,48,64,96,128}} "
                    f"({cells} cells), HLL, inflow -x, copy elsewhere, per-box CFL 0.5 timestep, {steps} steps",
        "value": batched,
        "unit": UNIT,
        "ms": batched_ms,
        "launch": {"kernels": 1, "graph_replayed": graphed, "blocks": run_grid, "work_items_per_step": run_items,
                   "tuned": None if run_tiling is None else {"tile": f"32x{run_tiling[0]}",
                                                             "planes_per_item": run_tiling[1]}},
        "healthy_boxes_value": healthy_cells * steps / (batched_ms / 1e3),
        "healthy_boxes": len(boxes) - len(failed),
        "per_step_launches": {"value": updates / (per_step_ms / 1e3), "ms": per_step_ms,
                              "tuned": {"tile": f"32x{tiling[0]}", "planes_per_item": tiling[1],
                                        "grid": tiling[2], "by": "autotuner" if tune else "defaults"}},
        "plain_sequential": plain,
        "plain_ms": plain_ms,
        "batched_over_plain": batched / plain if sequential else None,
        "boxes_failed": failed,
        "boxes_failed_steps": {i: taken[i] for i in failed},
        "boxes_failed_note": "boxes whose state hit the positivity check of the reference scheme within the "
                             "run, with the steps each took (the failing one included); they stop there, and "
                             "value counts the cell updates made. The CPU oracle fails the same three boxes; the "
                             "step differs (box 24: 236 there) because these boxes amplify round-off about 30x "
                             "per 10 steps (the oracle against itself with a 1e-15 perturbation fails box 36 at "
                             f"step 111 instead of 146); same count in the sequential run: {len(failed_steps)}",
        "what": "batched: all steps of all boxes in one persistent cooperative launch (a box's step waits only for "
                "its own previous step; each box its own lagged CFL dt), replayed from a CUDA graph; "
                "per_step_launches: the same ensemble with one launch per step; plain: each box in its own context, "
                "one box after another (the same tile code); healthy_boxes_value counts only the boxes that keep "
                "positivity over the whole run, against the same time; device time by CUDA events",
    }


def adjoint_section(local, n=256, steps=200, every=20, fd=True):
    """Discrete adjoint cost: Orszag-Tang n^2, HLLD, `steps` steps, checkpoints every `every` steps,
    J = magnetic energy in [0.4, 0.6]^2 at the last step.  Forward: the steps alone.  Gradient: the
    adjoint call, i.e. its forward run with checkpoints, the recompute of every segment and the
    reverse sweep."""
    import torch
    import pamhd_b200 as pg
    import states

    U0 = states.orszag_tang(n)
    # CFL 0.25: the reference scheme loses positivity on this problem at t = 0.104 (step 158 at
    # CFL 0.4); 200 steps at 0.25 end at t = 0.084
    cfg = pg.Config(n=(n, n, 1), solver=pg.HLLD, cell_length=(1 / n, 1 / n, 1.0), adiabatic_index=5 / 3,
                    vacuum_permeability=1.0, time_step_factor=0.25, device=local)
    ctx = pg.Context(cfg)
    st = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="xy")
    mask = ((X >= 0.4) & (X <= 0.6) & (Y >= 0.4) & (Y <= 0.6)).astype(float)[None]

    def fwd_ms():
        ctx.set_state(U0)
        ctx.step(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        ctx.steps(steps, 1e300)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    fwd_ms()
    forward = min(fwd_ms() for _ in range(3))
    UN = ctx.get_state()
    dts = ctx.dt_history(steps)
    seed = np.zeros_like(UN)
    seed[5:8] = UN[5:8] * mask / n ** 2

    def adj_ms():
        ctx.set_state(U0)
        ctx.step(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        ctx.adjoint(steps, every, seed, dt_in=dts)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    adj_ms()
    gradient = min(adj_ms() for _ in range(3))

    if not fd:
        ctx.close()
        return {"forward_ms": forward, "gradient_ms": gradient, "adjoint_over_forward": gradient / forward}

    # gradient check: 16 seeded Gaussian directions in (rho, v) at fixed p and B, central
    # differences at h = 1e-6 of the field rms and h/2 on the frozen dt schedule, Richardson-combined
    ctx.set_state(U0)
    ctx.step(0.0)
    grad, _, _ = ctx.adjoint(steps, every, seed, dt_in=dts)
    rho0, v0 = U0[0], U0[1:4] / U0[0]
    p0 = (5 / 3 - 1) * (U0[4] - 0.5 * (U0[1:4] ** 2).sum(0) / U0[0] - 0.5 * (U0[5:8] ** 2).sum(0))
    g_rho = grad[0] + (grad[1:4] * v0).sum(0) + grad[4] * 0.5 * (v0 ** 2).sum(0)
    g_v = grad[1:4] * rho0 + grad[4] * rho0 * v0
    rms_rho, rms_v = np.sqrt((rho0 ** 2).mean()), np.sqrt((v0[:2] ** 2).mean())

    def J_of(rho, v):
        U = U0.copy()
        U[0] = rho
        U[1:4] = rho * v
        U[4] = p0 / (5 / 3 - 1) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (U0[5:8] ** 2).sum(0)
        ctx.set_state(U)
        ctx.step(0.0)
        ctx.steps_dt(dts)
        return float((0.5 * (ctx.get_state()[5:8] ** 2).sum(0) * mask).sum() / n ** 2)

    rng = np.random.default_rng(20261205)
    ads, fds = [], []
    for _ in range(16):
        d_rho = rng.normal(size=rho0.shape)
        d_v = rng.normal(size=v0.shape)
        d_v[2] = 0.0
        h_rho, h_v = 1e-6 * rms_rho, 1e-6 * rms_v
        D = [(J_of(rho0 + f * h_rho * d_rho, v0 + f * h_v * d_v) - J_of(rho0 - f * h_rho * d_rho, v0 - f * h_v * d_v))
             / (2 * f) for f in (1.0, 0.5)]
        fds.append((4 * D[1] - D[0]) / 3)
        ads.append(float((g_rho * d_rho).sum() * h_rho + (g_v * d_v).sum() * h_v))
    ads, fds = np.array(ads), np.array(fds)
    ctx.close()
    return {
        "workload": f"Orszag-Tang {n}^2 periodic, HLLD, CFL 0.25, {steps} steps, checkpoints every {every}, "
                    "J = magnetic energy in [0.4,0.6]^2, gradient w.r.t. the initial state",
        "forward_ms": forward,
        "gradient_ms": gradient,
        "adjoint_over_forward": gradient / forward,
        "reverse_step_over_forward_step": (gradient - forward) / forward,
        "fd_check": {"directions": 16, "h": "1e-6 of the field rms, Richardson with h/2",
                     "max_err_over_max_fd": float(np.abs(ads - fds).max() / np.abs(fds).max()),
                     "bar": 1e-6},
        "what": "gradient_ms: the pamhd_gpu_adjoint call (forward run with checkpoints, recompute of every "
                "segment, reverse sweep); forward_ms: the same steps alone; device time by CUDA events; "
                "adjoint_over_forward: the whole gradient against the forward run; "
                "reverse_step_over_forward_step: (gradient - forward) / forward, the cost of one adjoint step "
                "(recompute overlapped) against one forward step",
    }


def staggered_section(local, n=256, steps=20, solver="hlld_athena", cpu=True):
    """Staggered-field step (face field by constrained transport): n^3 periodic cells (n a multiple
    of 64 or below it), a smooth seeded 64^3 state with a divergence-free face field
    (states.staggered_random) repeated periodically, CFL 0.4.  Timed:
    `steps` steps launched back to back on the context's stream (three kernels per step), CUDA
    events.  CPU: the oracle's staggered step on one core on a 32^3 sample."""
    import torch
    import pamhd_b200 as pg
    import states

    sid = pg.SOLVERS[solver]
    L = (1.0 / n,) * 3
    # a 64^3 periodic pattern repeated to n^3 (periodic, divergence-free faces; fast to build)
    m = min(n, 64)
    reps = (1, n // m, n // m, n // m)
    U, faces, _ = states.staggered_random((m, m, m), L, np.random.default_rng(20261206), field_amp=0.001 / n)
    U, faces = np.tile(U, reps), np.tile(faces, reps)
    cfg = pg.Config(n=(n, n, n), solver=sid, cell_length=L, adiabatic_index=5 / 3, vacuum_permeability=1.0,
                    time_step_factor=0.4, device=local)
    with pg.StaggeredContext(cfg) as ctx:
        ctx.set_state(U, faces)
        ctx.step(0.0)
        ctx.steps(3, T_END)
        ctx.sync()
        st = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            e0.record(st)
            ctx.steps(steps, T_END)
            e1.record(st)
            ctx.sync()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # end to end through the Python API: pinned host arrays in, the priming step and `steps`
        # steps, pinned host arrays out, host clock
        keep = [pinned(U.shape, U), pinned(faces.shape, faces), pinned(U.shape), pinned(faces.shape)]
        hU, hF, hUo, hFo = (k[1] for k in keep)
        t0 = time.perf_counter()
        ctx.set_state(hU, hF)
        ctx.step(0.0)
        ctx.steps(steps, T_END)
        ctx.get_state(out=(hUo, hFo))
        e2e_sec = time.perf_counter() - t0
    moved = (U.nbytes + faces.nbytes) / (steps + 1)
    # the same state in a bounded box: inflow on -x (the state of the first cell, denser), COPY on
    # every other side; the box's layer of boundary cells and the plain (untiled) kernels
    bc_lo, bc_hi = (pg.BC_VALUE, pg.BC_COPY, pg.BC_COPY), (pg.BC_COPY,) * 3
    inflow = U[:, 0, 0, 0].copy()
    inflow[0:4] *= 1.3
    bcfg = pg.Config(n=(n, n, n), solver=sid, cell_length=L, adiabatic_index=5 / 3, vacuum_permeability=1.0,
                     time_step_factor=0.4, bc_lo=bc_lo, bc_hi=bc_hi, value_lo=[list(inflow), None, None],
                     device=local)
    bfaces = []
    for d, shape in enumerate(pg.staggered_face_shapes(bcfg)):
        f = faces[d]
        if shape != f.shape:
            f = np.concatenate([f, np.take(f, [0], axis=2 - d)], axis=2 - d)
        bfaces.append(np.ascontiguousarray(f))
    with pg.StaggeredContext(bcfg) as ctx:
        ctx.set_state(U, bfaces)
        ctx.step(0.0)
        ctx.steps(3, T_END)
        ctx.sync()
        st = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        ctx.steps(steps, T_END)
        e1.record(st)
        ctx.sync()
        torch.cuda.synchronize()
        bms = e0.elapsed_time(e1) / steps
    bounded = {"workload": f"{n}^3 bounded box: inflow on -x, COPY elsewhere, {solver}, the same state",
               "value": n ** 3 / (bms * 1e-3), "unit": UNIT, "ms_per_step": bms, "steps": steps,
               "gpu_launches": 5 * steps,
               "what": "one thread per cell: face solves, face field, cell update, layer fill, inflow plane"}
    out = {
        "workload": f"{n}^3 periodic, {solver}, smooth state with a divergence-free face field, CFL 0.4",
        "value": n ** 3 / (ms * 1e-3),
        "unit": UNIT,
        "ms_per_step": ms,
        "steps": steps,
        "gpu_launches": 3 * steps,
        "roofline": section_roofline(n, "staggered_step_hlld", 176, n ** 3, ms, clocks.summary(),
                                     "whole step: faces_kernel + field_kernel + cell_kernel"),
        "e2e": {"value": n ** 3 * (steps + 1) / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": moved,
                "d2h_bytes_per_step": moved,
                "what": f"StaggeredContext.set_state from pinned host arrays + the priming step + {steps} "
                        f"steps + get_state to pinned host arrays, host clock"},
        "clocks": clocks.summary(),
        "bounded": bounded,
    }
    if cpu:
        from oracle import pyoracle as po
        m = 32
        Uc, Fc, Lc = states.staggered_random((m, m, m), (1.0 / m,) * 3, np.random.default_rng(20261206),
                                             field_amp=0.001 / m)
        g = po.Oracle("port").staggered_grid(po.make_cfg((m, m, m), sid, Lc, 5 / 3, 1.0, 0.4))
        g.set_state(Uc, Fc)
        g.step(0.0)
        t0 = time.perf_counter()
        k = 3
        for _ in range(k):
            g.step(T_END)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": m ** 3 * k / sec, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"oracle staggered step, {m}^3, {k} steps"}
    return out


def two_population_section(local, n=256, steps=20, cpu=True):
    """Two-population step (N_solve + apply_fluxes_N, split Rusanov): n^3 periodic cells (n a
    multiple of 64 or below it), two smooth seeded populations sharing one field
    (states.two_population_random, a 64^3 pattern repeated), the loop dt = min(0.4 max_dt, t_end - t)
    on the device.  CPU: the oracle's step on one core on a 32^3 sample."""
    import torch
    import pamhd_b200 as pg
    import states

    m = min(n, 64)
    reps = (1, n // m, n // m, n // m)
    U = np.tile(states.two_population_random((m, m, m), np.random.default_rng(20261208)), reps)
    with pg.TwoPopulationContext((n, n, n), (1.0 / n,) * 3, pg.RUSANOV, 5 / 3, 1.0, 0.0, local) as ctx:
        ctx.set_state(U)
        ctx.run(4, 0.4, T_END)
        ctx.sync()
        st = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            e0.record(st)
            ctx.run(steps, 0.4, T_END)
            e1.record(st)
            ctx.sync()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # end to end through the Python API: a pinned host array in, `steps` steps of the device loop,
        # a pinned host array out, host clock
        keep = [pinned(U.shape, U), pinned(U.shape)]
        hU, hUo = (k[1] for k in keep)
        t0 = time.perf_counter()
        ctx.set_state(hU)
        ctx.run(steps, 0.4, T_END)
        ctx.get_state(out=hUo)
        e2e_sec = time.perf_counter() - t0
    out = {
        "workload": f"{n}^3 periodic, two populations sharing one field, split Rusanov, CFL 0.4",
        "value": n ** 3 / (ms * 1e-3),
        "unit": UNIT,
        "ms_per_step": ms,
        "steps": steps,
        "gpu_launches": 2 * steps,
        "roofline": section_roofline(n, "two_population_step_rusanov", 208, n ** 3, ms, clocks.summary(),
                                     "whole step: npop_fused_kernel + restore_kernel"),
        "e2e": {"value": n ** 3 * steps / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": U.nbytes / steps,
                "d2h_bytes_per_step": U.nbytes / steps,
                "what": f"TwoPopulationContext.set_state from a pinned host array + {steps} steps + "
                        f"get_state to a pinned host array, host clock"},
        "clocks": clocks.summary(),
    }
    if cpu:
        from oracle import pyoracle as po
        k = 32
        Uc = states.two_population_random((k, k, k), np.random.default_rng(20261208))
        g = po.Oracle("port").two_population_grid((k, k, k), (1.0 / k,) * 3, po.RUSANOV, 5 / 3, 1.0, 0.0)
        g.set_state(Uc)
        max_dt = g.step(0.0)[0]
        t0 = time.perf_counter()
        reps_cpu = 3
        for _ in range(reps_cpu):
            max_dt = g.step(0.4 * max_dt)[0]
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k ** 3 * reps_cpu / sec, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"oracle two-population step, {k}^3, {reps_cpu} steps"}
    return out


def substep_section(local, n=128, steps=10, solver="hlld_athena", cpu=True):
    """Local time stepping: n^3 periodic cells, a smooth seeded state, exponent 0 where y < 0 and 1
    elsewhere (the regions of tests/mhd/config_files/hydrodynamic/substep/100cells/x2.json), CFL 0.4.
    Timed: `steps` host-driven steps (each plans its periods on the device, then runs its
    substeps).  value: cells advanced per second over the step length (every cell once per step);
    updates_per_s counts each cell's updates (two per step in the period-1 region).  CPU: the
    oracle on one core on a 24^3 sample."""
    import torch
    import pamhd_b200 as pg
    import states

    m = min(n, 64)
    reps = (1, n // m, n // m, n // m)
    U = np.tile(states.smooth_3d((m, m, m), np.random.default_rng(20261209), amp=0.05), reps)
    y = (np.arange(n) + 0.5) / n - 0.5
    e = np.broadcast_to(np.where(y < 0, 0, 1)[None, :, None], (n, n, n)).astype(np.int32)
    cfg = pg.Config(n=(n, n, n), solver=pg.SOLVERS[solver], cell_length=(1.0 / n,) * 3, adiabatic_index=5 / 3,
                    vacuum_permeability=1.0, time_step_factor=0.4, device=local)
    with pg.SubstepContext(cfg) as ctx:
        ctx.set_state(U)
        ctx.set_exponents(e, e)
        ctx.step(0.0)
        ctx.step(T_END)
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            t0 = time.perf_counter()
            subs = 0
            for _ in range(steps):
                subs += ctx.step(T_END)[1]
            sec = time.perf_counter() - t0
        periods = ctx.periods()
        # end to end through the Python API: a pinned host array in, the priming step and `steps`
        # steps, a pinned host array out, host clock
        keep = [pinned(U.shape, U), pinned(U.shape)]
        hU, hUo = (k[1] for k in keep)
        t0 = time.perf_counter()
        ctx.set_state(hU)
        ctx.step(0.0)
        for _ in range(steps):
            ctx.step(T_END)
        ctx.get_state(out=hUo)
        e2e_sec = time.perf_counter() - t0
    updates = float((subs / steps) * (1.0 / periods).sum())
    ms = 1e3 * sec / steps
    out = {
        "workload": f"{n}^3 periodic, {solver}, exponent 0 for y < 0 and 1 elsewhere, CFL 0.4",
        "value": n ** 3 * steps / sec,
        "unit": "cell-steps/s",
        "updates_per_s": updates * steps / sec,
        "ms_per_step": ms,
        "substeps_per_step": subs / steps,
        "gpu_launches": steps * 5 + 2 * subs,
        "gpu_launches_what": "per step the plan's five kernels (one restriction pass: the exponents given satisfy "
                             "the neighbour rule) and faces_kernel + update_kernel per substep",
        "timing": "host clock around synchronous steps (each step plans on the device and reads the plan back)",
        "roofline": section_roofline(n, "substep_step_hlld", 128, updates, ms, clocks.summary(),
                                     "whole step: the plan's kernels and faces_kernel + update_kernel per substep"),
        "e2e": {"value": n ** 3 * (steps + 1) / e2e_sec, "unit": "cell-steps/s",
                "h2d_bytes_per_step": U.nbytes / (steps + 1), "d2h_bytes_per_step": U.nbytes / (steps + 1),
                "what": f"SubstepContext.set_state from a pinned host array + the priming step + {steps} "
                        f"steps + get_state to a pinned host array, host clock"},
        "clocks": clocks.summary(),
    }
    if cpu:
        from oracle import pyoracle as po
        k = 24
        Uc = states.smooth_3d((k, k, k), np.random.default_rng(20261209), amp=0.05)
        yc = (np.arange(k) + 0.5) / k - 0.5
        ec = np.broadcast_to(np.where(yc < 0, 0, 1)[None, :, None], (k, k, k)).astype(np.int32)
        g = po.Oracle("port").substep_grid(po.make_cfg((k, k, k), pg.SOLVERS[solver], (1.0 / k,) * 3, 5 / 3, 1.0, 0.4))
        g.set_state(Uc)
        g.set_exponents(ec, ec)
        g.step(0.0)
        t0 = time.perf_counter()
        for _ in range(2):
            g.step(T_END)
        out["cpu_baseline"] = {"value": k ** 3 * 2 / (time.perf_counter() - t0), "unit": "cell-steps/s",
                               "cores": 1, "kind": "port", "sample": f"oracle substepped step, {k}^3, 2 steps"}
    return out


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def bench_config(n, world, steps):
    """The `config` of the bench line, the same for the GPU arm and the reference arm."""
    return dict(workload(n),
                parallelism=(f"{world} z slabs of {n}^3 of one {n}x{n}x{n * world} grid "
                             f"(the blast cube repeated along z), one per GPU; cut planes "
                             f"and the speed reduction exchanged over NCCL every step"
                             if world > 1 else f"one {n}^3 grid on one GPU"),
                timing=f"{steps} steps in segments of <= {SEGMENT} from the initial state "
                       f"(the blast fails positivity later in the reference scheme)")


def run_reference(a):
    """The reference arm: the reference's own HLLD solver code (compiled from its headers) in the
    restated cell-centred driver, on every host thread, stepping the same grid as the GPU arm
    (n^3, or n x n x (N n) for N ranks) with the same warm-up and segment schedule."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    n = a.n
    threads = cpu_threads()
    g, U, kind = cpu_grid(blast_state(n), n, world, threads)
    el = cpu_timed_steps(g, U, a.steps, a.warmup)
    cells = n ** 3 * world
    value = cells * a.steps / el
    sample = (f"{a.steps} timed HLLD steps of the full {n}x{n}x{n * world} grid, {threads} host threads "
              f"(std::thread over cells), the reference's solver headers compiled from source")
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * el / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": bench_config(n, world, a.steps),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
                         "cpu": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200(a):
    import torch
    import pamhd_b200 as pg

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    n = a.n
    U = blast_state(n)
    cells = n ** 3
    # N GPUs: one n x n x (N n) grid (the blast cube repeated along z, periodic) cut into N z slabs of
    # n^3, one per GPU, halo planes and the speed reduction exchanged over NCCL after every step
    from pamhd_b200.slabs import SlabGrid
    cfg = pg.Config(n=(n, n, n * world), solver=pg.HLLD, cell_length=(1 / n,) * 3, adiabatic_index=5 / 3,
                    vacuum_permeability=1.0, time_step_factor=CFL, device=local)
    grid = SlabGrid(cfg)
    ctx = grid.ctx

    # pinned host buffers for the end-to-end measurement
    host_in = torch.from_numpy(U.reshape(8, -1)).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # The configured blast (pressure ratio 100, plasma beta 0.2 outside) loses positivity in the
    # reference's own first-order scheme after a few tens of steps (the oracle fails at step 38 at
    # 64^3 and step 43 at 128^3, whatever the CFL).  So the timed steps run in segments of at most
    # SEGMENT steps, each restarted from the initial state; the restart and its dt = 0 priming step
    # are outside the CUDA events.
    dev_init = torch.from_numpy(U.reshape(8, -1)).to(f"cuda:{local}")
    init_ptrs = [dev_init[k].data_ptr() for k in range(8)]

    def restart():
        grid.set_state_device(init_ptrs)
        grid.steps(1, T_END)  # priming step (dt = 0)

    def checked_sync():
        try:
            ctx.sync()
        except pg.PhysicsError as e:
            raise SystemExit(f"step failed: flags {e.flags} at cell {e.cell} direction {e.direction}")

    restart()
    grid.steps(min(a.warmup, SEGMENT - 1), T_END)
    # beyond the W warm-up steps, untimed: whole segments as the timed ones run them, so that the
    # context's CUDA graph of the step sequence is captured and instantiated here (host work that
    # would otherwise fall inside the first timed segment) and the SM clock has settled after the
    # host-side set-up
    for _ in range(WARM_SEGMENTS):
        restart()
        grid.steps(SEGMENT - 1, T_END)
    checked_sync()
    starts, ends = [], []
    barrier()
    torch.cuda.synchronize()
    left = a.steps
    with ClockSampler(local) as clocks:
        while left > 0:
            seg = min(SEGMENT, left)
            restart()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            grid.steps(seg, T_END)
            ev1.record(stream)
            starts.append(ev0)
            ends.append(ev1)
            left -= seg
        torch.cuda.synchronize()
    barrier()
    checked_sync()
    ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in zip(starts, ends)))
    value = world * cells * a.steps / (ms / 1e3)
    kernel_ms = ms / a.steps  # one fused kernel per step (periodic grid: no boundary kernel)

    # ---- end to end through the C ABI with host buffers: one segment as a user runs it
    ptr_in = [host_in[k].data_ptr() for k in range(8)]
    ptr_out = [host_out[k].data_ptr() for k in range(8)]
    L = pg.lib()
    e2e_steps = min(SEGMENT, a.steps)
    barrier()
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    rc = L.pamhd_gpu_set_state(ctx.h, pg._pointers(ptr_in))
    assert rc == 0, rc
    grid.exchange()
    grid.steps(e2e_steps, T_END)
    rc = L.pamhd_gpu_get_state(ctx.h, pg._pointers(ptr_out))
    assert rc == 0, rc
    e_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    checked_sync()
    e_ms = max_over_ranks(e_start.elapsed_time(e_end))
    e2e = world * cells * e2e_steps / (e_ms / 1e3)
    state_bytes = 8 * 8 * cells

    peak, peak_kind = peaks()
    achieved = BYTES_PER_CELL_UPDATE * cells / (kernel_ms / 1e3) / 1e9
    traffic = ncu_traffic(n)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms / a.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(n, world, a.steps),
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "traffic_source": f"ncu DRAM bytes of one launch at 160^3 scaled to {n}^3 by cell count, captured from "
                              f"the kernel source of commit {ncu_source('step_kernel_hlld')} "
                              f"(profiles/step_kernel_hlld_blast160.md)",
            "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_cell_update": BYTES_PER_CELL_UPDATE,
            "kernel_ms": kernel_ms,
            "fp64": fp64_roof(n, kernel_ms, clocks.summary()),
        },
        "e2e": {
            "value": e2e,
            "unit": UNIT,
            "h2d_bytes_per_step": state_bytes / e2e_steps,
            "d2h_bytes_per_step": state_bytes / e2e_steps,
            "what": f"set_state from pinned host arrays + {e2e_steps} steps (the first is the dt = 0 priming "
                    f"step) + get_state to pinned host arrays ({state_bytes / 1e9:.2f} GB each way per run, "
                    f"amortised per step)",
        },
        "gpu_launches": a.steps,
        "clocks": clocks.summary(),
        "warmup_detail": f"{min(a.warmup, SEGMENT - 1)} warm-up steps, then {WARM_SEGMENTS} untimed whole segments "
                         f"(CUDA graph capture and clock settling), then the timed segments",
    }
    if not a.no_batched:
        line["batched"] = batched_section(local, steps=a.batched_steps, nboxes=a.boxes, tune=not a.no_tune)
    if not a.no_adjoint:
        line["adjoint"] = adjoint_section(local, steps=a.adjoint_steps, fd=not a.no_fd_check)
    if not a.no_configs and world == 1:
        line["configs"] = configs_section(local, cpu=rank == 0 and not a.no_cpu_baseline)
    if not a.no_staggered and world == 1:
        line["staggered"] = staggered_section(local, n=a.staggered_n, steps=a.staggered_steps,
                                              cpu=rank == 0 and not a.no_cpu_baseline)
    if not a.no_two_population and world == 1:
        line["two_population"] = two_population_section(local, n=a.two_population_n,
                                                        cpu=rank == 0 and not a.no_cpu_baseline)
    if not a.no_substep and world == 1:
        line["substep"] = substep_section(local, cpu=rank == 0 and not a.no_cpu_baseline)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(U, n)
        except Exception as e:  # a missing oracle build must not hide the GPU number
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable",
                                    "sample": str(e)}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_only(a):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if a.only == "batched":
        out = batched_section(local, steps=a.batched_steps, nboxes=a.boxes, tune=not a.no_tune,
                              sequential=False)
    elif a.only == "adjoint":
        out = adjoint_section(local, steps=a.adjoint_steps, fd=not a.no_fd_check)
    elif a.only == "staggered":
        out = staggered_section(local, n=a.staggered_n, steps=a.staggered_steps, cpu=not a.no_cpu_baseline)
    elif a.only == "two_population":
        out = two_population_section(local, n=a.two_population_n, cpu=not a.no_cpu_baseline)
    elif a.only == "substep":
        out = substep_section(local, cpu=not a.no_cpu_baseline)
    else:
        out = configs_section(local, cpu=not a.no_cpu_baseline, solver=a.configs_solver)
    print(json.dumps({a.only: out}), flush=True)
    return 0


def main():
    a = args_()
    if a.impl == "reference":
        return run_reference(a)
    if a.only:
        return run_only(a)
    return run_b200(a)


if __name__ == "__main__":
    sys.exit(main())
