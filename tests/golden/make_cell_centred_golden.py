"""Generates tests/golden/cell_centred_ref.npz from the REFERENCE's own step functions.

Run in a container where the reference tree exists (oracle/Makefile builds
oracle/_ref/libstag_ref.so from its mhd/solve.hpp and substepping.hpp):
    python tests/golden/make_cell_centred_golden.py

For every case and solver of tests/test_cell_centred_ref_pin.py it stores the reference's cell
state after the priming step and nine steps, and every step's dt; for the substepped cases, the
state after eight steps, every step's length and largest period.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import test_cell_centred_ref_pin as T  # noqa: E402


def main():
    run = T.load_ref_run()
    if run is None:
        raise SystemExit("the reference build oracle/_ref/libstag_ref.so is missing")
    out = {}
    for name in T.CASES:
        for solver, sid in T.SOLVERS.items():
            U, dts = run(name, sid)
            out[f"{name}_{solver}_cells"] = U
            out[f"{name}_{solver}_dts"] = dts
    sub = T.load_ref_substep_run()
    for name in T.SUB_CASES:
        for solver, sid in T.SOLVERS.items():
            U, dts, top = sub(name, sid)
            out[f"sub_{name}_{solver}_cells"] = U
            out[f"sub_{name}_{solver}_dts"] = dts
            out[f"sub_{name}_{solver}_periods"] = top
    np.savez_compressed(os.path.join(HERE, "cell_centred_ref.npz"), **out)


if __name__ == "__main__":
    main()
