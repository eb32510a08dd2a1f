"""Generates the golden fixtures of tests/golden from the REFERENCE's own code.

Run in a container where the reference tree exists (oracle/Makefile builds
oracle/_ref from it):
    python tests/golden/make_golden.py

  face_flux.npz  face problems (random, near-smooth, edge and invalid cases) and
                 the flux, speed and failure flag of each of the four solvers,
                 computed by the reference headers (mhd/rusanov.hpp:67,
                 hll_athena.hpp:65, hlld_athena.hpp:62, roe_athena.hpp:575)
  ref1d.npz      the final state of tests/mhd/reference.cpp --save (the program
                 that wrote the shipped mhd_*.ref goldens) for rusanov and
                 hll_athena, full double precision
  mode_c.npz     short Mode C runs on small grids with the reference solvers
                 driven by the oracle's grid restatement (periodic 3-D, copy and
                 value boundaries, a 1-D Brio-Wu tube), state after every step
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import pyoracle as po  # noqa: E402
import states  # noqa: E402

SEED = 20261203


def face_flux_cases():
    rng = np.random.default_rng(SEED)
    a = states.random_face_states(96, rng)
    b = states.random_face_states(96, rng)
    c, d = states.nearby_face_states(96, rng)
    e, f = states.edge_case_face_states()
    neg = np.vstack([a, c, e])
    pos = np.vstack([b, d, f])
    bg = np.zeros((neg.shape[0], 3))
    bg[:48] = rng.normal(0, 0.5, (48, 3))  # background field on some random faces
    return neg, pos, bg


def small_grid_runs(ref):
    rng = np.random.default_rng(SEED + 1)
    runs = {}
    U0 = states.smooth_3d((4, 5, 6), rng)
    for name, sid in po.SOLVERS.items():
        cfg = po.make_cfg((6, 5, 4), sid, (1 / 6, 1 / 5, 1 / 4), 5 / 3, 1.0, 0.4)
        g = ref.grid(cfg)
        g.set_state(U0)
        traj, dts = [U0], []
        for _ in range(4):
            dt, flag, _, _ = g.step(1.0)
            assert flag == 0, name
            dts.append(dt)
            traj.append(g.get_state())
        runs[f"periodic_{name}"] = (U0, np.array(traj), np.array(dts))
    # copy on x, inflow value on -y, copy on +y, periodic z
    inflow = np.array([1.2, 0.3 * 1.2, 0.2 * 1.2, 0.0,
                       states.energy(1.2, np.array([[0.3], [0.2], [0.0]]), 0.7,
                                     np.array([[0.4], [0.1], [-0.2]]), 5 / 3)[0], 0.4, 0.1, -0.2])
    for name in ("hll_athena", "hlld_athena"):
        cfg = po.make_cfg((6, 5, 4), po.SOLVERS[name], (0.2, 0.25, 0.3), 5 / 3, 1.0, 0.4,
                          bc_lo=(po.BC_COPY, po.BC_VALUE, po.BC_PERIODIC),
                          bc_hi=(po.BC_COPY, po.BC_COPY, po.BC_PERIODIC),
                          value_lo=[None, inflow, None])
        g = ref.grid(cfg)
        g.set_state(U0)
        traj, dts = [U0], []
        for _ in range(4):
            dt, flag, _, _ = g.step(1.0)
            assert flag == 0, name
            dts.append(dt)
            traj.append(g.get_state())
        runs[f"bounded_{name}"] = (U0, np.array(traj), np.array(dts))
    # Brio-Wu, 64 cells, gamma 2, copy boundaries, 12 steps
    Ub = states.brio_wu(64)
    for name, sid in po.SOLVERS.items():
        cfg = po.make_cfg((64, 1, 1), sid, (1 / 64, 1, 1), 2.0, 1.0, 0.5,
                          bc_lo=(po.BC_COPY, po.BC_PERIODIC, po.BC_PERIODIC),
                          bc_hi=(po.BC_COPY, po.BC_PERIODIC, po.BC_PERIODIC))
        g = ref.grid(cfg)
        g.set_state(Ub)
        traj, dts = [Ub], []
        for _ in range(12):
            dt, flag, _, _ = g.step(0.1)
            if flag != 0:
                break
            dts.append(dt)
            traj.append(g.get_state())
        runs[f"briowu_{name}"] = (Ub, np.array(traj), np.array(dts))
    return runs


def main():
    po.build()
    if not os.path.exists(po.REF_LIB):
        raise SystemExit("the reference build oracle/_ref is missing")
    ref = po.Oracle("reference")

    neg, pos, bg = face_flux_cases()
    out = {"neg": neg, "pos": pos, "bg": bg}
    for name, sid in po.SOLVERS.items():
        f, s, g = ref.face_flux(sid, neg, pos, bg)
        out[f"{name}_flux"] = f
        out[f"{name}_speed"] = s
        out[f"{name}_flags"] = g
    np.savez_compressed(os.path.join(HERE, "face_flux.npz"), **out)

    ref1d = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name in ("rusanov", "hll_athena"):
            subprocess.run([po.REF_EXE, "--solver", name, "--save", "--no-verify"], cwd=tmp, check=True)
            ref1d[name] = np.loadtxt(os.path.join(tmp, f"mhd_{name}.dat"))
    np.savez_compressed(os.path.join(HERE, "ref1d.npz"), **ref1d)

    runs = small_grid_runs(ref)
    flat = {}
    for key, (U0, traj, dts) in runs.items():
        flat[f"{key}_traj"] = traj
        flat[f"{key}_dt"] = dts
    np.savez_compressed(os.path.join(HERE, "mode_c.npz"), **flat)
    for f in ("face_flux.npz", "ref1d.npz", "mode_c.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
