"""The C-ABI library loads and exports what include/*.h declares (CPU only, no GPU calls
beyond argument validation, which happens before any CUDA call)."""
import ctypes
import glob
import os
import re

import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(pamhd_gpu_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from pamhd_b200 import build
    build.build()
    return pg.lib()


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "pamhd_gpu_step" in names and "pamhd_gpu_face_flux" in names
    assert len(names) >= 15


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports(lib, name):
    assert hasattr(lib, name), name


def test_abi_version_and_errstr(lib):
    assert lib.pamhd_gpu_abi_version() == 2
    assert lib.pamhd_gpu_errstr(pg.ERR_PHYSICS).decode().startswith("a face met")


def test_cfg_layout_matches_oracle():
    assert ctypes.sizeof(pg._Cfg) == ctypes.sizeof(po.Cfg)
    for (a, ta), (b, tb) in zip(pg._Cfg._fields_, po.Cfg._fields_):
        assert a == b and ctypes.sizeof(ta) == ctypes.sizeof(tb)
        assert getattr(pg._Cfg, a).offset == getattr(po.Cfg, b).offset


@pytest.mark.parametrize("change", [
    dict(solver=1),                       # rusanov_staggered aborts in the reference dispatcher
    dict(solver=9),
    dict(n=(1, 1, 1)),                    # no active dimension
    dict(cell_length=(0.0, 1.0, 1.0)),
    dict(adiabatic_index=1.0),
    dict(vacuum_permeability=0.0),
    dict(time_step_factor=0.0),
    dict(bc_lo=(0, 0, 0), bc_hi=(1, 0, 0)),  # periodic on one side only
    dict(n=(2, 8 * 65535 + 1, 1)),           # more rows of 32 x 8 tiles than a launch can have
    dict(n=(2, 4 * 65535 + 1, 1), solver=4),  # Roe's 32 x 4 tiles
])
def test_create_rejects_invalid_config(lib, change):
    kw = dict(n=(8, 8, 8), solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1))
    kw.update(change)
    cfg = pg.Config(**kw).to_c()
    h = ctypes.c_void_p()
    assert lib.pamhd_gpu_create(ctypes.byref(cfg), ctypes.byref(h)) == pg.ERR_ARGUMENT
    assert not h.value


def test_null_arguments_rejected(lib):
    assert lib.pamhd_gpu_create(None, None) == pg.ERR_ARGUMENT
    assert lib.pamhd_gpu_step(None, 0.0, None, None) == pg.ERR_ARGUMENT
    assert lib.pamhd_gpu_destroy(None) == pg.OK


@pytest.mark.parametrize("n", [(1, 8, 8), (8, 1, 8), (1, 8, 1), (1, 1, 8)])
def test_any_active_dimensions_pass_the_checks(lib, n):
    """Grids whose active dimensions are not x, x-y or x-y-z are relabelled, not rejected (without
    a GPU the call then fails at its first CUDA call, not at the argument checks)."""
    cfg = pg.Config(n=n, solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1)).to_c()
    h = ctypes.c_void_p()
    rc = lib.pamhd_gpu_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc != pg.ERR_ARGUMENT
    if h.value:
        lib.pamhd_gpu_destroy(h)


@pytest.mark.parametrize("change", [
    dict(bc_lo=(pg.BC_COPY, 0, 0)),                 # periodic on one side only
    dict(bc_lo=(0, 0, pg.BC_VALUE)),
    dict(bc_lo=(pg.BC_VALUE, pg.BC_VALUE, 0), bc_hi=(pg.BC_COPY, pg.BC_COPY, 0)),   # two inflow sides
    dict(n=(4, 4, 1), bc_lo=(0, 0, pg.BC_COPY), bc_hi=(0, 0, pg.BC_COPY)),         # one cell, bounded
    dict(bc_lo=(pg.BC_EXTERNAL, 0, 0), bc_hi=(pg.BC_EXTERNAL, 0, 0)),              # no slab cuts
    dict(solver=1),
    dict(n=(0, 4, 4)),
    dict(cell_length=(0.1, -0.1, 0.1)),
    dict(adiabatic_index=0.5),
    dict(n=(1, 8 * 65535 + 1, 1)),                 # more rows of face tiles (8 cells high) than a launch can have
])
def test_staggered_create_rejects_invalid_config(lib, change):
    lib.pamhd_gpu_staggered_create.argtypes = [ctypes.POINTER(pg._Cfg), ctypes.POINTER(ctypes.c_void_p)]
    kw = dict(n=(4, 4, 4), solver=pg.RUSANOV, cell_length=(0.1, 0.1, 0.1))
    kw.update(change)
    cfg = pg.Config(**kw).to_c()
    h = ctypes.c_void_p()
    assert lib.pamhd_gpu_staggered_create(ctypes.byref(cfg), ctypes.byref(h)) == pg.ERR_ARGUMENT
    assert not h.value
    assert lib.pamhd_gpu_staggered_create(None, None) == pg.ERR_ARGUMENT
    assert lib.pamhd_gpu_staggered_destroy(None) == pg.OK


@pytest.mark.parametrize("change", [
    dict(solver=3),                 # the two-population step has Rusanov and HLL only
    dict(n=(0, 4, 4)),
    dict(length=(0.1, 0.0, 0.1)),
    dict(gamma=1.0),
    dict(mu0=-1.0),
    dict(min_pressure=-1.0),
])
def test_two_population_create_rejects_invalid_arguments(lib, change):
    I3, D3 = ctypes.c_int32 * 3, ctypes.c_double * 3
    lib.pamhd_gpu_npop_create.argtypes = [I3, D3, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    kw = dict(n=(4, 4, 4), length=(0.1, 0.1, 0.1), solver=pg.RUSANOV, gamma=5 / 3, mu0=1.0, min_pressure=0.0)
    kw.update(change)
    h = ctypes.c_void_p()
    rc = lib.pamhd_gpu_npop_create(I3(*kw["n"]), D3(*kw["length"]), kw["solver"], kw["gamma"], kw["mu0"],
                                   kw["min_pressure"], 0, ctypes.byref(h))
    assert rc == pg.ERR_ARGUMENT and not h.value
    assert lib.pamhd_gpu_npop_destroy(None) == pg.OK


@pytest.mark.parametrize("change", [
    dict(bc_lo=(pg.BC_COPY, 0, 0), bc_hi=(pg.BC_COPY, 0, 0)),   # local time stepping is periodic only
    dict(solver=1),
    dict(n=(1, 1, 1)),
    dict(time_step_factor=0.0),
])
def test_substep_create_rejects_invalid_config(lib, change):
    lib.pamhd_gpu_substep_create.argtypes = [ctypes.POINTER(pg._Cfg), ctypes.POINTER(ctypes.c_void_p)]
    kw = dict(n=(4, 4, 4), solver=pg.HLLD, cell_length=(0.1, 0.1, 0.1))
    kw.update(change)
    cfg = pg.Config(**kw).to_c()
    h = ctypes.c_void_p()
    assert lib.pamhd_gpu_substep_create(ctypes.byref(cfg), ctypes.byref(h)) == pg.ERR_ARGUMENT
    assert not h.value
    assert lib.pamhd_gpu_substep_destroy(None) == pg.OK
