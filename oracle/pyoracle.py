"""ctypes access to the CPU oracle libraries.

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may import this module.  It is the checker, never the
thing measured or shipped.

Two libraries expose the same entry points (oracle/capi_body.hpp):
  port       oracle/_build/liboracle.so   restated solvers (mhd_oracle.hpp)
  reference  oracle/_ref/libpamhd_ref.so  the reference's own solver headers
Both drive the solvers with the same grid restatements: Mode C (mode_c.hpp)
and the staggered-field step (mode_s.hpp).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libpamhd_ref.so")
# the reference's substepping.hpp on a single-rank uniform-grid stand-in (ref_substep_bridge.cpp)
REF_SUBSTEP_LIB = os.path.join(ORACLE_DIR, "_ref", "libsubstep_ref.so")
REF_EXE = os.path.join(ORACLE_DIR, "_ref", "reference.exe")

RUSANOV, RUSANOV_STAGGERED, HLL, HLLD, ROE = 0, 1, 2, 3, 4
SOLVERS = {"rusanov": RUSANOV, "hll_athena": HLL, "hlld_athena": HLLD, "roe_athena": ROE}
BC_PERIODIC, BC_COPY, BC_VALUE = 0, 1, 2


class Cfg(ctypes.Structure):
    """Layout of pamhd_cfg (include/pamhd_gpu.h)."""

    _fields_ = [
        ("n", ctypes.c_int32 * 3),
        ("solver", ctypes.c_int32),
        ("cell_length", ctypes.c_double * 3),
        ("adiabatic_index", ctypes.c_double),
        ("vacuum_permeability", ctypes.c_double),
        ("time_step_factor", ctypes.c_double),
        ("bc_lo", ctypes.c_int32 * 3),
        ("bc_hi", ctypes.c_int32 * 3),
        ("value_lo", (ctypes.c_double * 8) * 3),
        ("value_hi", (ctypes.c_double * 8) * 3),
        ("device", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


# Where the reference's source tree is read from, by the oracle's build and by the tests that pin
# against its own files: the PAMHD_REFERENCE environment variable (the reference tree is absent
# on machines that only run the built oracle; the pins that need it are skipped there).
REFERENCE = os.environ.get("PAMHD_REFERENCE", "/root/reference")


def make_cfg(n, solver, cell_length, gamma, mu0, cfl, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0),
             value_lo=None, value_hi=None, device=0) -> Cfg:
    c = Cfg()
    for d in range(3):
        c.n[d] = int(n[d])
        c.cell_length[d] = float(cell_length[d])
        c.bc_lo[d] = int(bc_lo[d])
        c.bc_hi[d] = int(bc_hi[d])
        for k in range(8):
            c.value_lo[d][k] = 0.0 if value_lo is None or value_lo[d] is None else float(value_lo[d][k])
            c.value_hi[d][k] = 0.0 if value_hi is None or value_hi[d] is None else float(value_hi[d][k])
    c.solver = int(solver)
    c.adiabatic_index = float(gamma)
    c.vacuum_permeability = float(mu0)
    c.time_step_factor = float(cfl)
    c.device = int(device)
    c.reserved = 0
    return c


def build(quiet: bool = True) -> None:
    """Runs oracle/Makefile (the reference targets only where the reference tree exists)."""
    out = subprocess.run(["make", "-C", ORACLE_DIR], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_P = ctypes.POINTER
_D = ctypes.c_double
_DP = _P(ctypes.c_double)


def _soa_in(arrays):
    ptrs = (ctypes.c_void_p * 8)()
    keep = []
    for k in range(8):
        a = np.ascontiguousarray(arrays[k], dtype=np.float64)
        keep.append(a)
        ptrs[k] = a.ctypes.data
    return ptrs, keep


class Oracle:
    """One oracle library: 'port' (restated solvers) or 'reference' (reference headers)."""

    def __init__(self, kind: str = "port"):
        path = PORT_LIB if kind == "port" else REF_LIB
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (the reference build needs the reference tree)")
        self.kind = kind
        self.lib = ctypes.CDLL(path)
        p = "oracle_" if kind == "port" else "ref_"
        L = self.lib
        self._face_flux = getattr(L, p + "face_flux")
        self._face_flux.restype = ctypes.c_int64
        self._face_flux.argtypes = [ctypes.c_int32, ctypes.c_int64, _DP, _DP, _DP, _D, _D, _DP, _DP,
                                    _P(ctypes.c_uint32)]
        self._create = getattr(L, p + "grid_create")
        self._create.restype = ctypes.c_void_p
        self._create.argtypes = [_P(Cfg)]
        self._destroy = getattr(L, p + "grid_destroy")
        self._destroy.argtypes = [ctypes.c_void_p]
        self._threads = getattr(L, p + "grid_set_threads")
        self._threads.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        self._set = getattr(L, p + "grid_set_state")
        self._set.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._get = getattr(L, p + "grid_get_state")
        self._get.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._step = getattr(L, p + "grid_step")
        self._step.argtypes = [ctypes.c_void_p, _D, _DP, _P(ctypes.c_uint32), _P(ctypes.c_int32),
                               _P(ctypes.c_int32)]
        self._step_dt = getattr(L, p + "grid_step_dt")
        self._step_dt.argtypes = [ctypes.c_void_p, _D, _P(ctypes.c_uint32)]
        self._run = getattr(L, p + "grid_run")
        self._run.restype = ctypes.c_int64
        self._run.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int64, _DP, _DP]
        self._max_signal = getattr(L, p + "grid_max_signal")
        self._max_signal.argtypes = [ctypes.c_void_p, _DP]
        self._set_inflow = getattr(L, p + "grid_set_inflow")
        self._set_inflow.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]
        self._screate = getattr(L, p + "sgrid_create")
        self._screate.restype = ctypes.c_void_p
        self._screate.argtypes = [_P(Cfg)]
        self._sdestroy = getattr(L, p + "sgrid_destroy")
        self._sdestroy.argtypes = [ctypes.c_void_p]
        self._sset = getattr(L, p + "sgrid_set_state")
        self._sset.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self._sget = getattr(L, p + "sgrid_get_state")
        self._sget.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self._sbg = getattr(L, p + "sgrid_set_background")
        self._sbg.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._sinflow = getattr(L, p + "sgrid_set_inflow")
        self._sinflow.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]
        self._sstep = getattr(L, p + "sgrid_step")
        self._sstep.argtypes = [ctypes.c_void_p, _D, _DP, _P(ctypes.c_uint32), _P(ctypes.c_int32),
                                _P(ctypes.c_int32)]
        self._face_flux_N = getattr(L, p + "face_flux_N")
        self._face_flux_N.restype = ctypes.c_int64
        self._face_flux_N.argtypes = [ctypes.c_int32, ctypes.c_int64, _DP, _DP, _D, _D, _D, _D, _DP, _DP, _DP,
                                      _P(ctypes.c_uint32)]
        self._ref2 = getattr(L, p + "reference_2pop_1d")
        self._ref2.restype = ctypes.c_int32
        self._ref2.argtypes = [ctypes.c_int32, ctypes.c_int32, _D, _D, _DP]
        self._ncreate = getattr(L, p + "ngrid_create")
        self._ncreate.restype = ctypes.c_void_p
        self._ncreate.argtypes = [_P(ctypes.c_int32), _DP, ctypes.c_int32, _D, _D, _D]
        self._ndestroy = getattr(L, p + "ngrid_destroy")
        self._ndestroy.argtypes = [ctypes.c_void_p]
        self._nset = getattr(L, p + "ngrid_set_state")
        self._nset.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._nget = getattr(L, p + "ngrid_get_state")
        self._nget.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._nstep = getattr(L, p + "ngrid_step")
        self._nstep.argtypes = [ctypes.c_void_p, _D, _DP, _P(ctypes.c_uint32), _P(ctypes.c_int32),
                                _P(ctypes.c_int32)]
        self._lcreate = getattr(L, p + "lgrid_create")
        self._lcreate.restype = ctypes.c_void_p
        self._lcreate.argtypes = [_P(Cfg)]
        self._ldestroy = getattr(L, p + "lgrid_destroy")
        self._ldestroy.argtypes = [ctypes.c_void_p]
        self._lset = getattr(L, p + "lgrid_set_state")
        self._lset.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._lget = getattr(L, p + "lgrid_get_state")
        self._lget.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._lexp = getattr(L, p + "lgrid_set_exponents")
        self._lexp.argtypes = [ctypes.c_void_p, _P(ctypes.c_int32), _P(ctypes.c_int32)]
        self._lstep = getattr(L, p + "lgrid_step")
        self._lstep.argtypes = [ctypes.c_void_p, _D, _DP, _P(ctypes.c_int32), _P(ctypes.c_int32),
                                _P(ctypes.c_uint32)]
        self._lplan = getattr(L, p + "lgrid_plan")
        self._lplan.argtypes = [ctypes.c_void_p, _DP, _D, _P(ctypes.c_int32), _DP, _P(ctypes.c_int32)]
        self._last_error = getattr(L, p + "last_error")
        self._last_error.restype = ctypes.c_char_p
        if kind == "port":
            self._ref1d = L.oracle_reference_1d
            self._ref1d.restype = ctypes.c_int32
            self._ref1d.argtypes = [ctypes.c_int32, ctypes.c_int32, _D, _D, _DP]

    def last_error(self) -> str:
        return self._last_error().decode()

    def face_flux(self, solver, neg, pos, bg=None, gamma=5.0 / 3.0, mu0=1.0):
        """neg, pos: (n, 8); bg: (n, 3) or None.  Returns flux (n, 8), speed (n,), flags (n,)."""
        neg = np.ascontiguousarray(neg, dtype=np.float64)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        n = neg.shape[0]
        flux = np.zeros((n, 8))
        speed = np.zeros(n)
        flags = np.zeros(n, dtype=np.uint32)
        bgp = None
        if bg is not None:
            bg = np.ascontiguousarray(bg, dtype=np.float64)
            bgp = bg.ctypes.data_as(_DP)
        self._face_flux(solver, n, neg.ctypes.data_as(_DP), pos.ctypes.data_as(_DP), bgp, gamma, mu0,
                        flux.ctypes.data_as(_DP), speed.ctypes.data_as(_DP),
                        flags.ctypes.data_as(_P(ctypes.c_uint32)))
        return flux, speed, flags

    def reference_1d(self, solver, cells=1002, t_end=1.0, length=1e5):
        out = np.zeros((cells, 8))
        steps = self._ref1d(solver, cells, t_end, length, out.ctypes.data_as(_DP))
        if steps < 0:
            raise RuntimeError(self.last_error())
        return out, steps

    def face_flux_N(self, solver, neg, pos, area=1.0, dt=1.0, gamma=5.0 / 3.0, mu0=1.0):
        """Two-population split solver on total states (n, 8): returns flux_neg, flux_pos (n, 8),
        speed (n,), flags (n,)."""
        neg = np.ascontiguousarray(neg, dtype=np.float64)
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        n = neg.shape[0]
        fn, fp = np.zeros((n, 8)), np.zeros((n, 8))
        speed = np.zeros(n)
        flags = np.zeros(n, dtype=np.uint32)
        self._face_flux_N(solver, n, neg.ctypes.data_as(_DP), pos.ctypes.data_as(_DP), area, dt, gamma, mu0,
                          fn.ctypes.data_as(_DP), fp.ctypes.data_as(_DP), speed.ctypes.data_as(_DP),
                          flags.ctypes.data_as(_P(ctypes.c_uint32)))
        return fn, fp, speed, flags

    def reference_2pop_1d(self, solver, cells=1002, t_end=1.0, length=1e5):
        """The scheme of tests/mhd/two_reference.cpp: (cells, 13) state and the step count."""
        out = np.zeros((cells, 13))
        steps = self._ref2(solver, cells, t_end, length, out.ctypes.data_as(_DP))
        if steps < 0:
            raise RuntimeError(self.last_error())
        return out, steps

    def two_population_grid(self, n, length, solver, gamma, mu0, min_pressure) -> "OracleTwoPopulationGrid":
        return OracleTwoPopulationGrid(self, n, length, solver, gamma, mu0, min_pressure)

    def substep_grid(self, cfg: Cfg) -> "OracleSubstepGrid":
        return OracleSubstepGrid(self, cfg)

    def grid(self, cfg: Cfg, threads: int = 1) -> "OracleGrid":
        return OracleGrid(self, cfg, threads)

    def staggered_grid(self, cfg: Cfg) -> "OracleStaggeredGrid":
        return OracleStaggeredGrid(self, cfg)


class OracleGrid:
    """A Mode C grid in the oracle; state arrays are (8, nz, ny, nx)."""

    def __init__(self, oracle: Oracle, cfg: Cfg, threads: int = 1):
        self.o = oracle
        self.cfg = cfg
        self.shape = (cfg.n[2], cfg.n[1], cfg.n[0])
        self.h = oracle._create(ctypes.byref(cfg))
        if not self.h:
            raise ValueError(oracle.last_error())
        oracle._threads(self.h, threads)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.o._destroy(h)
            self.h = None

    def set_state(self, U):
        ptrs, keep = _soa_in([U[k].reshape(-1) for k in range(8)])
        rc = self.o._set(self.h, ptrs)
        if rc != 0:
            raise ValueError(self.o.last_error())

    def get_state(self):
        U = np.zeros((8,) + self.shape)
        ptrs = (ctypes.c_void_p * 8)()
        for k in range(8):
            ptrs[k] = U[k].ctypes.data
        self.o._get(self.h, ptrs)
        return U

    def set_inflow(self, dim, side, times, states):
        """Time-stamped states of a VALUE side: states[i] (8 conservative values) holds while i of
        the timestamps are <= the simulation time; len(states) == len(times) + 1."""
        times = np.ascontiguousarray(times, dtype=np.float64).reshape(-1)
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
        rc = self.o._set_inflow(self.h, dim, side, len(times), times.ctypes.data_as(_DP), states.ctypes.data_as(_DP))
        if rc != 0:
            raise ValueError(self.o.last_error())

    def step(self, max_dt):
        """Returns (dt, flag, cell, dir); flag != 0 when a face failed (state not updated)."""
        dt = ctypes.c_double(0)
        flag = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.o._step(self.h, max_dt, ctypes.byref(dt), ctypes.byref(flag), cell, ctypes.byref(d))
        if rc not in (0, 3):
            raise ValueError(self.o.last_error())
        return dt.value, flag.value, tuple(cell), d.value

    def max_signal(self):
        """Largest face signal speed of the last step along x, y, z (max of Max_v)."""
        out = np.zeros(3)
        self.o._max_signal(self.h, out.ctypes.data_as(_DP))
        return out

    def step_dt(self, dt):
        """One step with a prescribed dt; returns the failure flag (0 when fine)."""
        flag = ctypes.c_uint32(0)
        rc = self.o._step_dt(self.h, dt, ctypes.byref(flag))
        if rc not in (0, 3):
            raise ValueError(self.o.last_error())
        return flag.value

    def run(self, t_start, t_end, max_steps):
        hist = np.zeros(max_steps)
        t = ctypes.c_double(0)
        steps = self.o._run(self.h, t_start, t_end, max_steps, ctypes.byref(t), hist.ctypes.data_as(_DP))
        if steps < 0:
            raise RuntimeError(self.o.last_error())
        return t.value, hist[:steps]


def staggered_face_shapes(n, bc_lo, bc_hi):
    """Shapes (z, y, x) of the three face arrays of a staggered grid: the -d face of every cell, and
    along a bounded dimension (not periodic, two cells or more) the high wall too."""
    shapes = []
    for d in range(3):
        ext = [int(n[2]), int(n[1]), int(n[0])]
        if int(n[d]) > 1 and not (bc_lo[d] == BC_PERIODIC and bc_hi[d] == BC_PERIODIC):
            ext[2 - d] += 1
        shapes.append(tuple(ext))
    return shapes


class OracleStaggeredGrid:
    """A staggered-field grid in the oracle (periodic, COPY or VALUE sides).  Cell state arrays are
    (8, nz, ny, nx); face field arrays: the normal field of every cell's -x, -y and -z face, shapes
    from staggered_face_shapes (n + 1 along a bounded dimension); on a periodic grid the three
    come as one (3, nz, ny, nx) array."""

    def __init__(self, oracle: Oracle, cfg: Cfg):
        self.o = oracle
        self.cfg = cfg
        self.shape = (cfg.n[2], cfg.n[1], cfg.n[0])
        self.face_shapes = staggered_face_shapes(list(cfg.n), list(cfg.bc_lo), list(cfg.bc_hi))
        self.periodic = all(s == self.shape for s in self.face_shapes)
        self.h = oracle._screate(ctypes.byref(cfg))
        if not self.h:
            raise ValueError(oracle.last_error())

    def set_inflow(self, dim, side, times, states):
        """Time-stamped states of the VALUE side, as OracleGrid.set_inflow."""
        times = np.ascontiguousarray(times, dtype=np.float64).reshape(-1)
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
        rc = self.o._sinflow(self.h, dim, side, len(times), times.ctypes.data_as(_DP), states.ctypes.data_as(_DP))
        if rc != 0:
            raise ValueError(self.o.last_error())

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.o._sdestroy(h)
            self.h = None

    def set_state(self, U, faces):
        ptrs, keep = _soa_in([U[k].reshape(-1) for k in range(8)])
        fptrs = (ctypes.c_void_p * 3)()
        fkeep = []
        for d in range(3):
            a = np.ascontiguousarray(faces[d], dtype=np.float64)
            if a.size != int(np.prod(self.face_shapes[d])):
                raise ValueError(f"faces[{d}]: {self.face_shapes[d]} expected, {a.shape} given")
            fkeep.append(a.reshape(-1))
            fptrs[d] = fkeep[-1].ctypes.data
        rc = self.o._sset(self.h, ptrs, fptrs)
        if rc != 0:
            raise ValueError(self.o.last_error())

    def set_background(self, bg):
        """bg: (3, 3, nz, ny, nx): bg[d, c] = component c of the background field at every cell's
        -d face; None clears it."""
        if bg is None:
            self.o._sbg(self.h, None)
            return
        bg = np.ascontiguousarray(bg, dtype=np.float64).reshape((9,) + self.shape)
        ptrs = (ctypes.c_void_p * 9)(*[bg[k].ctypes.data for k in range(9)])
        self._bg_keep = bg
        self.o._sbg(self.h, ptrs)

    def get_state(self):
        U = np.zeros((8,) + self.shape)
        faces = np.zeros((3,) + self.shape) if self.periodic else [np.zeros(s) for s in self.face_shapes]
        ptrs = (ctypes.c_void_p * 8)()
        for k in range(8):
            ptrs[k] = U[k].ctypes.data
        fptrs = (ctypes.c_void_p * 3)()
        for d in range(3):
            fptrs[d] = faces[d].ctypes.data
        self.o._sget(self.h, ptrs, fptrs)
        return U, faces

    def step(self, max_dt):
        """Returns (dt, flag, cell, dir); flag != 0 when a face failed (state not updated)."""
        dt = ctypes.c_double(0)
        flag = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.o._sstep(self.h, max_dt, ctypes.byref(dt), ctypes.byref(flag), cell, ctypes.byref(d))
        if rc not in (0, 3):
            raise ValueError(self.o.last_error())
        return dt.value, flag.value, tuple(cell), d.value


class OracleTwoPopulationGrid:
    """A two-population grid in the oracle (N_solve + apply_fluxes_N, periodic).  State arrays are
    (13, nz, ny, nx): rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz."""

    def __init__(self, oracle: Oracle, n, length, solver, gamma, mu0, min_pressure):
        self.o = oracle
        self.shape = (int(n[2]), int(n[1]), int(n[0]))
        nn = (ctypes.c_int32 * 3)(*[int(v) for v in n])
        ll = (ctypes.c_double * 3)(*[float(v) for v in length])
        self.h = oracle._ncreate(nn, ll, solver, gamma, mu0, min_pressure)
        if not self.h:
            raise ValueError(oracle.last_error())

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.o._ndestroy(h)
            self.h = None

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((13,) + self.shape)
        ptrs = (ctypes.c_void_p * 13)(*[U[k].ctypes.data for k in range(13)])
        self._keep = U
        self.o._nset(self.h, ptrs)

    def get_state(self):
        U = np.zeros((13,) + self.shape)
        ptrs = (ctypes.c_void_p * 13)(*[U[k].ctypes.data for k in range(13)])
        self.o._nget(self.h, ptrs)
        return U

    def step(self, dt):
        """Returns (max_dt for the next step, flag, cell, dir)."""
        m = ctypes.c_double(0)
        flag = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.o._nstep(self.h, dt, ctypes.byref(m), ctypes.byref(flag), cell, ctypes.byref(d))
        if rc not in (0, 3):
            raise ValueError(self.o.last_error())
        return m.value, flag.value, tuple(cell), d.value


class OracleSubstepGrid:
    """A cell-centred grid with local time stepping in the oracle (periodic); state (8, nz, ny, nx),
    exponent bounds (nz, ny, nx) int32."""

    def __init__(self, oracle: Oracle, cfg: Cfg):
        self.o = oracle
        self.shape = (cfg.n[2], cfg.n[1], cfg.n[0])
        self.h = oracle._lcreate(ctypes.byref(cfg))
        if not self.h:
            raise ValueError(oracle.last_error())

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.o._ldestroy(h)
            self.h = None

    def set_state(self, U):
        ptrs, keep = _soa_in([U[k].reshape(-1) for k in range(8)])
        if self.o._lset(self.h, ptrs) != 0:
            raise ValueError(self.o.last_error())

    def get_state(self):
        U = np.zeros((8,) + self.shape)
        ptrs = (ctypes.c_void_p * 8)()
        for k in range(8):
            ptrs[k] = U[k].ctypes.data
        self.o._lget(self.h, ptrs)
        return U

    def set_exponents(self, mins, maxs):
        a = np.ascontiguousarray(mins, dtype=np.int32).reshape(-1)
        b = np.ascontiguousarray(maxs, dtype=np.int32).reshape(-1)
        if self.o._lexp(self.h, a.ctypes.data_as(_P(ctypes.c_int32)), b.ctypes.data_as(_P(ctypes.c_int32))) != 0:
            raise ValueError(self.o.last_error())

    def plan(self, limits, max_dt):
        """The substep plan from given CFL limits (nz, ny, nx) on the exponent bounds set before:
        (periods (nz, ny, nx), substep length, largest period), or None where the reference would
        abort on unexpected substeps."""
        lim = np.ascontiguousarray(limits, dtype=np.float64).reshape(-1)
        periods = np.zeros(self.shape, dtype=np.int32)
        sub = ctypes.c_double(0)
        top = ctypes.c_int32(0)
        rc = self.o._lplan(self.h, lim.ctypes.data_as(_DP), max_dt, periods.ctypes.data_as(_P(ctypes.c_int32)),
                           ctypes.byref(sub), ctypes.byref(top))
        if rc != 0:
            return None
        return periods, sub.value, top.value

    def step(self, max_dt):
        """Returns (dt, substeps, periods (nz, ny, nx), flag)."""
        dt = ctypes.c_double(0)
        k = ctypes.c_int32(0)
        periods = np.zeros(self.shape, dtype=np.int32)
        flag = ctypes.c_uint32(0)
        rc = self.o._lstep(self.h, max_dt, ctypes.byref(dt), ctypes.byref(k),
                           periods.ctypes.data_as(_P(ctypes.c_int32)), ctypes.byref(flag))
        if rc not in (0, 3):
            raise ValueError(self.o.last_error())
        return dt.value, k.value, periods, flag.value
