"""Generates tests/golden/staggered_ref.npz from the REFERENCE's own staggered-field step.

Run in a container where the reference tree exists (oracle/Makefile builds
oracle/_ref/libstag_ref.so from its mhd/solve.hpp, common_functions.hpp and
mhd/solar_wind_box.hpp):
    python tests/golden/make_staggered_golden.py

For every case and solver of tests/test_staggered_ref_pin.py it stores the reference's state after
the priming step and five steps (cells, the three face arrays), every step's dt, and the
conservative state its wind cells took.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import test_staggered_ref_pin as T  # noqa: E402


def main():
    run = T.load_ref_run()
    if run is None:
        raise SystemExit("the reference build oracle/_ref/libstag_ref.so is missing")
    out = {}
    for name in T.CASES:
        for solver, sid in T.SOLVERS.items():
            U, F, dts, value = run(name, sid)
            key = f"{name}_{solver}"
            out[key + "_cells"] = U
            for d in range(3):
                out[key + f"_faces{d}"] = F[d]
            out[key + "_dts"] = dts
            out[key + "_value"] = value
    np.savez_compressed(os.path.join(HERE, "staggered_ref.npz"), **out)


if __name__ == "__main__":
    main()
