"""Generates tests/golden/substep_plan.npz from the REFERENCE's own substepping functions.

Run in a container where the reference tree exists (oracle/Makefile builds
oracle/_ref/libsubstep_ref.so from its substepping.hpp):
    python tests/golden/make_substep_golden.py

For every case of tests/test_substep_ref_pin.py (per-cell CFL limits, exponent bounds, cap; 3-D and
2-D periodic grids) it stores the reference's plan: every cell's period, the substep length and the
largest period, or abort = 1 where the reference stops on unexpected substeps.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import test_substep_ref_pin as T  # noqa: E402


def main():
    plan = T.load_ref_plan()
    if plan is None:
        raise SystemExit("the reference build oracle/_ref/libsubstep_ref.so is missing")
    out = {}
    for i, (n, shape, kind, limits, lo, hi, cap) in enumerate(T.cases()):
        r = plan(n, T.lengths_of(n), limits, lo, hi, cap)
        out[f"c{i}_abort"] = np.array(1 if r is None else 0)
        if r is not None:
            out[f"c{i}_periods"] = r[0]
            out[f"c{i}_substep"] = np.array(r[1])
            out[f"c{i}_max"] = np.array(r[2])
    np.savez_compressed(os.path.join(HERE, "substep_plan.npz"), **out)


if __name__ == "__main__":
    main()
