"""Reading and writing the reference's .dc output files (pamhd_dc_write / _read_info / _read),
host only, no GPU: round trips, the reference's own shipped output files (read here and by the
reference's reader), and files this library writes read back by the reference's reader."""
import os
import struct
import sys

import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po

REF = po.REFERENCE
GOLD = os.path.join(os.path.dirname(__file__), "golden")
SHIPPED = {
    "da_px": "tests/mhd/reference/hydrodynamic/density_advection/1d/+x/rusanov/mhd_000000917.dc",
    "da_mx": "tests/mhd/reference/hydrodynamic/density_advection/1d/-x/rusanov/mhd_000000917.dc",
}


@pytest.fixture(scope="module", autouse=True)
def built():
    from pamhd_b200 import build
    build.build()


def sample(shape=(3, 4, 5), seed=3):
    return np.random.default_rng(seed).normal(size=(8,) + shape)


def test_round_trip(tmp_path):
    U = sample()
    path = str(tmp_path / "a.dc")
    pg.write_dc(path, U, step=17, time=0.25, adiabatic_index=5 / 3, proton_mass=1.67e-27,
                vacuum_permeability=4e-7 * np.pi, cell_length=(0.1, 0.2, 0.3), periodic=(True, False, True),
                start=(-1.0, 0.5, 2.0))
    info, V = pg.read_dc(path)
    assert np.array_equal(U, V)
    assert info["step"] == 17 and info["time"] == 0.25 and info["n"] == (5, 4, 3) and info["cells"] == 60
    assert info["periodic"] == (True, False, True)
    assert info["start"] == (-1.0, 0.5, 2.0) and info["cell_length"] == (0.1, 0.2, 0.3)
    assert info["proton_mass"] == 1.67e-27 and info["vacuum_permeability"] == 4e-7 * np.pi


def test_layout_matches_the_reference_file_header(tmp_path):
    """Byte positions of the fixed header: the cell list starts at byte 168 with one variable,
    the variable's name follows the cell list."""
    U = sample((1, 1, 7))
    path = str(tmp_path / "b.dc")
    pg.write_dc(path, U, step=1, time=0.0, adiabatic_index=2.0, proton_mass=1.0, vacuum_permeability=1.0,
                cell_length=(1.0, 1.0, 1.0))
    raw = open(path, "rb").read()
    assert struct.unpack_from("<QQ", raw, 0) == (4, 1)
    assert raw[56] == 1                                    # one variable
    (offset,) = struct.unpack_from("<Q", raw, 57)
    assert offset == 168 + 7 * 8
    assert struct.unpack_from("<Q", raw, 65)[0] == 0x1234567890abcdef
    assert list(struct.unpack_from("<7Q", raw, 168)) == list(range(1, 8))
    assert raw[offset:offset + 8] == b"mhd     "
    assert len(raw) == offset + 8 + 7 * 64


def test_rejects_malformed_files(tmp_path):
    U = sample((1, 2, 2))
    path = str(tmp_path / "c.dc")
    pg.write_dc(path, U, step=0, time=0.0, adiabatic_index=2.0, proton_mass=1.0, vacuum_permeability=1.0,
                cell_length=(1.0, 1.0, 1.0))
    raw = bytearray(open(path, "rb").read())
    bad_version = bytearray(raw)
    struct.pack_into("<Q", bad_version, 0, 3)
    open(tmp_path / "v.dc", "wb").write(bad_version)
    with pytest.raises(pg.PamhdError) as e:
        pg.read_dc(str(tmp_path / "v.dc"))
    assert e.value.code == pg.ERR_ARGUMENT
    open(tmp_path / "t.dc", "wb").write(raw[: len(raw) - 9])
    with pytest.raises(pg.PamhdError) as e:
        pg.read_dc(str(tmp_path / "t.dc"))
    assert e.value.code == pg.ERR_IO
    with pytest.raises(pg.PamhdError) as e:
        pg.read_dc(str(tmp_path / "missing.dc"))
    assert e.value.code == pg.ERR_IO


@pytest.mark.skipif(not os.path.isdir(REF), reason="needs the reference tree")
@pytest.mark.parametrize("case", list(SHIPPED))
def test_reads_the_reference_output(case):
    """The reference program's own output files read by this library equal what the reference's
    reader extracted into the fixture."""
    g = np.load(os.path.join(GOLD, "dc_goldens.npz"))
    info, U = pg.read_dc(os.path.join(REF, SHIPPED[case]))
    assert info["step"] == int(g[case + "_step"]) and info["time"] == float(g[case + "_time"])
    assert info["adiabatic_index"] == float(g[case + "_gamma"])
    assert info["n"] == tuple(int(c) for c in g[case + "_cells"])
    assert np.array_equal(U.reshape(8, -1), g[case + "_state"])


@pytest.mark.skipif(not os.path.isdir(REF), reason="needs the reference tree")
def test_reference_reader_reads_our_files(tmp_path):
    sys.path.insert(0, os.path.join(REF, "tests"))
    import common
    U = sample((2, 3, 4), seed=9)
    path = str(tmp_path / "d.dc")
    pg.write_dc(path, U, step=5, time=1.5, adiabatic_index=5 / 3, proton_mass=2.0, vacuum_permeability=3.0,
                cell_length=(0.5, 0.25, 0.125), periodic=(True, True, False), start=(1.0, 2.0, 3.0))
    with open(path, "rb") as f:
        meta = common.get_metadata(f)
        cells = common.get_cells(f, meta["total_cells"])
        data = common.get_cell_data(f, meta, range(len(cells)), ["mhd     "])
    assert meta["sim_step"] == 5 and meta["sim_time"] == 1.5 and meta["proton_mass"] == 2.0
    assert meta["ref_lvl_0_cells"] == [4, 3, 2] and meta["periodicity"] == [1, 1, 0]
    assert meta["grid_start"] == [1.0, 2.0, 3.0] and meta["lvl_0_cell_length"] == [0.5, 0.25, 0.125]
    flat = U.reshape(8, -1)
    for i, cid in enumerate(cells):
        rho, mom, nrj, mag = data[i]["mhd     "]
        got = [rho, *mom, nrj, *mag]
        assert np.array_equal(got, flat[:, cid - 1])


@pytest.mark.skipif(not os.path.isdir(REF), reason="needs the reference tree")
@pytest.mark.parametrize("case,vx", [("da_px", 1.0), ("da_mx", -1.0)])
def test_reference_diff_tool_accepts_our_output(tmp_path, port, case, vx):
    """The oracle's density-advection run, written by this library, against the reference
    program's own output, checked by the reference's comparison tool (tests/mhd/mhd_diff.py,
    which also requires every header field to match) at 1e-14."""
    import subprocess
    import states
    from oracle import pyoracle as po
    g = np.load(os.path.join(GOLD, "dc_goldens.npz"))
    gamma = float(g[case + "_gamma"])
    n = int(g[case + "_cells"][0])
    grid = port.grid(po.make_cfg((n, 1, 1), po.RUSANOV, tuple(g[case + "_cell_length"]), gamma, 1.0, 0.5))
    grid.set_state(states.density_advection(n, gamma, vx))
    t, dts = grid.run(0.0, 1.0, 100000)
    ours = str(tmp_path / "mhd_000000917.dc")
    pg.write_dc(ours, grid.get_state(), step=int((dts > 0).sum()), time=t, adiabatic_index=gamma,
                proton_mass=1.0, vacuum_permeability=1.0, cell_length=tuple(g[case + "_cell_length"]))
    tool = os.path.join(REF, "tests", "mhd", "mhd_diff.py")
    r = subprocess.run([sys.executable, tool, "--mass", "1e-14", "--velocity", "1e-14", "--energy", "1e-14",
                        ours, os.path.join(REF, SHIPPED[case])], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
