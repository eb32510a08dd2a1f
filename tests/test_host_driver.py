"""A C++ program on the C ABI alone (tests/host/abi_driver.cpp): built here against
include/pamhd_gpu.h and libpamhd_gpu.so; on the GPU it runs the shock tube to t = 0.1 the way a
PAMHD program's time loop would and writes a .dc file, which must match the oracle's run."""
import os
import subprocess

import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "host", "abi_driver.cpp")
EXE = os.path.join(HERE, "host", "_build", "abi_driver")


def build_driver():
    from pamhd_b200 import build
    build.build()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    libdir = os.path.join(ROOT, "pamhd_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-o", EXE,
                    SRC, "-L", libdir, "-lpamhd_gpu", f"-Wl,-rpath,{libdir}"], check=True)
    return EXE


def test_driver_builds_on_the_c_abi():
    assert os.path.exists(build_driver())


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["hlld_athena", "roe_athena"])
def test_driver_matches_oracle(tmp_path, port, solver):
    exe = build_driver()
    out = str(tmp_path / "mhd.dc")
    r = subprocess.run([exe, str(po.SOLVERS[solver]), "1000", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    steps, t, _ = r.stdout.split()
    ora = port.grid(po.make_cfg((1000, 1, 1), po.SOLVERS[solver], (1e-3, 1.0, 1.0), 2.0, 1.0, 0.5,
                                (po.BC_COPY, 0, 0), (po.BC_COPY, 0, 0)))
    ora.set_state(states.brio_wu(1000))
    t_o, dts = ora.run(0.0, 0.1, 100000)
    assert int(steps) == int((dts > 0).sum())
    assert abs(float(t) - t_o) <= 1e-13
    info, U = pg.read_dc(out)
    assert info["step"] == int(steps) and info["n"] == (1000, 1, 1)
    ref = ora.get_state().reshape(8, -1)
    got = U.reshape(8, -1)
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert (np.abs(got - ref).max(axis=1) / scale).max() <= 1e-8
