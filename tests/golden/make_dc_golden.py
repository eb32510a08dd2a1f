"""Extracts golden states from the reference's own program outputs (.dc files shipped with the
reference's tests) into tests/golden/dc_goldens.npz, with the reference's own reader
(tests/common.py: get_metadata, get_cells, get_cell_data).

Run where the reference tree exists:
    python tests/golden/make_dc_golden.py

Zero-field cases, for which the reference's staggered-field ("Mode S") program reduces to the
cell-centred step of this library (the hydrodynamic part of the update is the same flux
difference, mhd/solve.hpp:1543-1576, and the field terms vanish):

  da_px, da_mx  tests/mhd/reference/hydrodynamic/density_advection/1d/{+x,-x}/rusanov/
                mhd_000000917.dc: 200 periodic cells on [0, 1], gamma 1.6666666667, mu0 1,
                proton mass 1, CFL 0.5, Rusanov, run from t = 0 to t = 1
                (tests/mhd/config_files/hydrodynamic/density_advection/1d/{+x,-x}/rusanov.json)

Alfven waves, which pin the staggered-field step itself (Rusanov, CFL 0.5, t = 0 .. 1,
uniform level-0 grids, periodic):

  alf_px, alf_mx  tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/1d/{+x,-x}/small_rusanov/
                  mhd_000000202.dc: 100 x 1 x 1 cells on [0, 1]^3
  alf_r1, alf_r2  tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/2d/x/small_rusanov{1,2}/
                  mhd_0000000{18,33}.dc: 1 x 10 x 10 cells, volume (1, 2/sqrt 3, 2), travelling
                  and standing wave
  alf_b1, alf_b2  .../2d/x/small_rusanov_bgB{1,2}/mhd_0000000{18,33}.dc: the same waves with the
                  field split into a constant background (0, 0.86603, 0.5) and the perturbation

Each case stores: step, time, gamma, mu0, proton mass, the state (8, cells) in the reference's
variable order (rho, mom xyz, E, B xyz) ordered by cell id, and the cell length.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.pyoracle import REFERENCE as REF  # noqa: E402 (the PAMHD_REFERENCE environment variable)
CASES = {
    "da_px": "tests/mhd/reference/hydrodynamic/density_advection/1d/+x/rusanov/mhd_000000917.dc",
    "da_mx": "tests/mhd/reference/hydrodynamic/density_advection/1d/-x/rusanov/mhd_000000917.dc",
    "alf_px": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/1d/+x/small_rusanov/mhd_000000202.dc",
    "alf_mx": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/1d/-x/small_rusanov/mhd_000000202.dc",
    "alf_r1": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/2d/x/small_rusanov1/mhd_000000018.dc",
    "alf_r2": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/2d/x/small_rusanov2/mhd_000000033.dc",
    "alf_b1": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/2d/x/small_rusanov_bgB1/mhd_000000018.dc",
    "alf_b2": "tests/mhd/reference/magnetohydrodynamic/Alfvén_wave/2d/x/small_rusanov_bgB2/mhd_000000033.dc",
}


def read_dc(path):
    sys.path.insert(0, os.path.join(REF, "tests"))
    import common  # the reference's reader
    with open(path, "rb") as f:
        meta = common.get_metadata(f)
        cells = common.get_cells(f, meta["total_cells"])
        data = common.get_cell_data(f, meta, range(len(cells)), ["mhd     "])
    order = np.argsort(cells)
    U = np.zeros((8, len(cells)))
    for j, i in enumerate(order):
        rho, mom, nrj, mag = data[i]["mhd     "]
        U[:, j] = [rho, mom[0], mom[1], mom[2], nrj, mag[0], mag[1], mag[2]]
    return meta, np.array(cells)[order], U


def main():
    out = {}
    for key, rel in CASES.items():
        meta, cells, U = read_dc(os.path.join(REF, rel))
        assert list(cells) == list(range(1, len(cells) + 1)), "level-0 cells 1..n expected"
        out[key + "_state"] = U
        out[key + "_step"] = meta["sim_step"]
        out[key + "_time"] = meta["sim_time"]
        out[key + "_gamma"] = meta["adiabatic_index"]
        out[key + "_mu0"] = meta["vacuum_permeability"]
        out[key + "_proton_mass"] = meta["proton_mass"]
        out[key + "_cell_length"] = np.array(meta["lvl_0_cell_length"])
        out[key + "_cells"] = np.array(meta["ref_lvl_0_cells"])
        print(key, meta["sim_step"], meta["sim_time"], meta["adiabatic_index"], meta["ref_lvl_0_cells"],
              float(np.abs(U[5:8]).max()))
    np.savez_compressed(os.path.join(HERE, "dc_goldens.npz"), **out)


if __name__ == "__main__":
    main()
