"""Generates tests/golden/two_population.npz from the REFERENCE's own two-population code.

Run in a container where the reference tree exists (oracle/Makefile builds oracle/_ref from it):
    python tests/golden/make_two_population_golden.py

  split_*       face problems on total states (random, near-smooth and edge cases) and the split
                fluxes (negative side, positive side, both times area and dt), signal speed and
                failure flag of the reference's get_flux_N_rusanov (mhd/N_rusanov.hpp:61) and
                get_flux_N_hll (mhd/N_hll_athena.hpp:47), compiled from its headers
  prog_rusanov  the final state of tests/mhd/two_reference.cpp --solver rusanov --save (1002 cells,
                totals rho, mom xyz, E, B xyz per cell as the program writes them, 16 digits)
  gold_rusanov  the reference's golden file tests/mhd/2mhd_rusanov.ref (the same layout)
  prog_hll_aborts  1 if the program with --solver hll_athena aborts (it does: a face meets a
                negative pressure, so 2mhd_hll_athena.ref is not reproducible by the current code)
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

REF = po.REFERENCE  # the PAMHD_REFERENCE environment variable
TWO_EXE = os.path.join(po.ORACLE_DIR, "_ref", "two_reference.exe")
SEED = 20261207
AREA, DT = 0.37, 0.013


def split_cases():
    rng = np.random.default_rng(SEED)
    a = states.random_face_states(96, rng)
    b = states.random_face_states(96, rng)
    c, d = states.nearby_face_states(96, rng)
    e, f = states.edge_case_face_states()
    return np.vstack([a, c, e]), np.vstack([b, d, f])


def main():
    po.build()
    if not os.path.exists(po.REF_LIB) or not os.path.exists(TWO_EXE):
        raise SystemExit("the reference build oracle/_ref is missing")
    ref = po.Oracle("reference")
    neg, pos = split_cases()
    out = {"split_neg": neg, "split_pos": pos, "split_area": AREA, "split_dt": DT}
    for name in ("rusanov", "hll_athena"):
        fn, fp, s, g = ref.face_flux_N(po.SOLVERS[name], neg, pos, AREA, DT)
        out[f"split_{name}_neg"] = fn
        out[f"split_{name}_pos"] = fp
        out[f"split_{name}_speed"] = s
        out[f"split_{name}_flags"] = g
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([TWO_EXE, "--solver", "rusanov", "--save", "--no-verify"], cwd=tmp, check=True)
        out["prog_rusanov"] = np.loadtxt(os.path.join(tmp, "mhd_rusanov.dat"))
        r = subprocess.run([TWO_EXE, "--solver", "hll_athena", "--no-verify"], cwd=tmp,
                           capture_output=True, text=True)
        out["prog_hll_aborts"] = int(r.returncode != 0)
    out["gold_rusanov"] = np.loadtxt(os.path.join(REF, "tests", "mhd", "2mhd_rusanov.ref"))
    np.savez_compressed(os.path.join(HERE, "two_population.npz"), **out)
    print({k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
