"""Python binding of the B200 finite-volume MHD step (libpamhd_gpu.so).

Every call goes through the C ABI of include/pamhd_gpu.h; there is no
Python or CPU implementation of the step here.  If the library is missing
the import of a context fails loudly (build it with `python -m
pamhd_b200.build`).

    from pamhd_b200 import Context, Config, HLLD
    ctx = Context(Config(n=(256, 256, 256), solver=HLLD, cell_length=(1/256,)*3,
                         adiabatic_index=5/3, vacuum_permeability=1.0, time_step_factor=0.4))
    ctx.set_state(U)            # (8, nz, ny, nx) float64: rho, mom xyz, E, B xyz
    ctx.step(0.0)               # dt = 0 priming step, as tests/mhd/test.cpp:462
    ctx.steps(200, t_end=1e9)   # 200 steps, no host synchronisation
    U = ctx.get_state()
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpamhd_gpu.so")

RUSANOV, RUSANOV_STAGGERED, HLL, HLLD, ROE = 0, 1, 2, 3, 4
SOLVERS = {"rusanov": RUSANOV, "hll_athena": HLL, "hlld_athena": HLLD, "roe_athena": ROE}
BC_PERIODIC, BC_COPY, BC_VALUE, BC_EXTERNAL = 0, 1, 2, 3

OK, ERR_ARGUMENT, ERR_CUDA, ERR_PHYSICS, ERR_STATE, ERR_TIMEOUT = 0, 1, 2, 3, 4, 5
ERR_TOO_LARGE = 6
ERR_IO = 7
NOALLOC_MAX_FACES = 16384
FLAG_DENSITY, FLAG_PRESSURE, FLAG_WAVE_SPEED, FLAG_FLUX = 1, 2, 4, 8
FLAG_ROE_DENSITY, FLAG_ROE_PRESSURE, FLAG_NEW_STATE, FLAG_TIMEOUT = 16, 32, 64, 128


class PamhdError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {errstr(code)} ({code})")
        self.code = code


class PhysicsError(PamhdError):
    """A face met a state the reference would throw std::domain_error on."""

    def __init__(self, code, what, flags=0, cell=(0, 0, 0), direction=0):
        super().__init__(code, what)
        self.flags = flags
        self.cell = cell
        self.direction = direction


class _Cfg(ctypes.Structure):
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


@dataclass
class Config:
    """pamhd_cfg of include/pamhd_gpu.h."""

    n: tuple
    solver: int
    cell_length: tuple
    adiabatic_index: float = 5.0 / 3.0
    vacuum_permeability: float = 1.0
    time_step_factor: float = 0.5
    bc_lo: tuple = (BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)
    bc_hi: tuple = (BC_PERIODIC, BC_PERIODIC, BC_PERIODIC)
    value_lo: list = field(default_factory=lambda: [None, None, None])
    value_hi: list = field(default_factory=lambda: [None, None, None])
    device: int = 0

    def to_c(self) -> _Cfg:
        c = _Cfg()
        for d in range(3):
            c.n[d] = int(self.n[d])
            c.cell_length[d] = float(self.cell_length[d])
            c.bc_lo[d] = int(self.bc_lo[d])
            c.bc_hi[d] = int(self.bc_hi[d])
            for k in range(8):
                c.value_lo[d][k] = 0.0 if self.value_lo[d] is None else float(self.value_lo[d][k])
                c.value_hi[d][k] = 0.0 if self.value_hi[d] is None else float(self.value_hi[d][k])
        c.solver = int(self.solver)
        c.adiabatic_index = float(self.adiabatic_index)
        c.vacuum_permeability = float(self.vacuum_permeability)
        c.time_step_factor = float(self.time_step_factor)
        c.device = int(self.device)
        c.reserved = 0
        return c


_lib = None
_P = ctypes.POINTER
_D = ctypes.c_double
_DP = _P(ctypes.c_double)


def lib() -> ctypes.CDLL:
    """Loads libpamhd_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pamhd_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.pamhd_gpu_abi_version.restype = ctypes.c_int
    L.pamhd_gpu_errstr.restype = ctypes.c_char_p
    L.pamhd_gpu_errstr.argtypes = [ctypes.c_int]
    L.pamhd_gpu_create.argtypes = [_P(_Cfg), _P(ctypes.c_void_p)]
    L.pamhd_gpu_destroy.argtypes = [ctypes.c_void_p]
    for name in ("pamhd_gpu_set_state", "pamhd_gpu_get_state", "pamhd_gpu_set_state_device",
                 "pamhd_gpu_get_state_device"):
        getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.pamhd_gpu_step.argtypes = [ctypes.c_void_p, _D, _DP, _DP]
    L.pamhd_gpu_steps.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
    L.pamhd_gpu_sync.argtypes = [ctypes.c_void_p]
    L.pamhd_gpu_get_stream.argtypes = [ctypes.c_void_p, _P(ctypes.c_void_p)]
    L.pamhd_gpu_time.argtypes = [ctypes.c_void_p, _DP, _P(ctypes.c_int64), _DP]
    L.pamhd_gpu_dt_history.argtypes = [ctypes.c_void_p, _DP, ctypes.c_int32, _P(ctypes.c_int32)]
    L.pamhd_gpu_status.argtypes = [ctypes.c_void_p, _P(ctypes.c_uint32), _P(ctypes.c_int32), _P(ctypes.c_int32)]
    L.pamhd_gpu_totals.argtypes = [ctypes.c_void_p, _DP]
    L.pamhd_gpu_face_flux.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, _DP, _DP, _DP, _D, _D,
                                      _DP, _DP, _P(ctypes.c_uint32)]
    V = ctypes.c_void_p
    L.pamhd_gpu_steps_dt.argtypes = [V, ctypes.c_int32, _DP]
    L.pamhd_gpu_adjoint.argtypes = [V, ctypes.c_int32, ctypes.c_int32, V, V, _DP, _DP, _DP]
    L.pamhd_gpu_batch_create.argtypes = [ctypes.c_int32, ctypes.c_int32, _P(_Cfg), _P(V)]
    L.pamhd_gpu_batch_destroy.argtypes = [V]
    L.pamhd_gpu_batch_set_state.argtypes = [V, ctypes.c_int32, V]
    L.pamhd_gpu_batch_get_state.argtypes = [V, ctypes.c_int32, V]
    L.pamhd_gpu_batch_steps.argtypes = [V, ctypes.c_int32, _D]
    L.pamhd_gpu_batch_tune.argtypes = [V, ctypes.c_int32, _P(ctypes.c_int32), _P(ctypes.c_int32)]
    L.pamhd_gpu_batch_sync.argtypes = [V]
    L.pamhd_gpu_batch_get_stream.argtypes = [V, _P(V)]
    L.pamhd_gpu_batch_time.argtypes = [V, ctypes.c_int32, _DP, _P(ctypes.c_int64), _DP]
    L.pamhd_gpu_batch_dt_history.argtypes = [V, ctypes.c_int32, _DP, ctypes.c_int32, _P(ctypes.c_int32)]
    L.pamhd_gpu_batch_status.argtypes = [V, ctypes.c_int32, _P(ctypes.c_uint32), _P(ctypes.c_int32),
                                         _P(ctypes.c_int32)]
    if L.pamhd_gpu_abi_version() != 2:
        raise ImportError("libpamhd_gpu.so ABI version mismatch")
    _lib = L
    return L


def errstr(code: int) -> str:
    try:
        return lib().pamhd_gpu_errstr(code).decode()
    except ImportError:
        return "unknown"


def _pointers(arrays):
    ptrs = (ctypes.c_void_p * 8)()
    for k in range(8):
        ptrs[k] = arrays[k]
    return ptrs


class Context:
    """A pamhd_ctx: one uniform grid on one GPU."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.L = lib()
        self.shape = (int(cfg.n[2]), int(cfg.n[1]), int(cfg.n[0]))
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        rc = self.L.pamhd_gpu_create(ctypes.byref(self._c), ctypes.byref(h))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pamhd_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc == ERR_PHYSICS:
            flags, cell, d = self.status()
            raise PhysicsError(rc, what, flags, cell, d)
        if rc != OK:
            raise PamhdError(rc, what)

    def set_state(self, U: np.ndarray):
        """U: (8, nz, ny, nx) float64 host array."""
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((8,) + self.shape)
        self._check(self.L.pamhd_gpu_set_state(self.h, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_set_state")

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        U = np.empty((8,) + self.shape) if out is None else out
        self._check(self.L.pamhd_gpu_get_state(self.h, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_get_state")
        return U

    def set_state_device(self, ptrs):
        """ptrs: eight device pointers (ints), e.g. torch tensor data_ptr()s."""
        self._check(self.L.pamhd_gpu_set_state_device(self.h, _pointers(ptrs)), "pamhd_gpu_set_state_device")

    def get_state_device(self, ptrs):
        self._check(self.L.pamhd_gpu_get_state_device(self.h, _pointers(ptrs)), "pamhd_gpu_get_state_device")

    def step(self, max_dt: float) -> float:
        dt = ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_step(self.h, max_dt, ctypes.byref(dt), None), "pamhd_gpu_step")
        return dt.value

    def step_signal(self, max_dt: float):
        """One step as step(); returns (dt, max_signal): the step length and the largest face
        signal speed of the step along x, y and z (the reference's Max_v, maximised per axis)."""
        dt = ctypes.c_double(0)
        sig = (ctypes.c_double * 3)()
        self._check(self.L.pamhd_gpu_step(self.h, max_dt, ctypes.byref(dt), sig), "pamhd_gpu_step")
        return dt.value, np.array(sig[:], dtype=np.float64)

    def steps(self, n: int, t_end: float):
        self._check(self.L.pamhd_gpu_steps(self.h, int(n), float(t_end)), "pamhd_gpu_steps")

    def step_part(self, part: int, t_end: float):
        """Half of a step (pamhd_gpu_step_part): part 1 the first and last z planes, part 2 the others
        and the step's end."""
        fn = self.L.pamhd_gpu_step_part
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        self._check(fn(self.h, int(part), float(t_end)), "pamhd_gpu_step_part")

    def set_inflow(self, dim: int, side: int, times, states):
        """Time-stamped inflow of a VALUE side (pamhd_gpu_set_inflow): states[i] (8 conservative
        values) holds while i of the increasing timestamps are <= the simulation time."""
        fn = self.L.pamhd_gpu_set_inflow
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]
        times = np.ascontiguousarray(times, dtype=np.float64).reshape(-1)
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
        if len(states) != len(times) + 1:
            raise ValueError("set_inflow: one state more than timestamps")
        self._check(fn(self.h, dim, side, len(times), times.ctypes.data_as(_DP), states.ctypes.data_as(_DP)),
                    "pamhd_gpu_set_inflow")

    def save_dc(self, path: str, step: int, time: float, proton_mass: float = 1.0, start=(0.0, 0.0, 0.0)):
        """Writes the current state as a reference .dc file (pamhd_dc_write)."""
        c = self.cfg
        write_dc(path, self.get_state(), step=step, time=time, adiabatic_index=c.adiabatic_index,
                 proton_mass=proton_mass, vacuum_permeability=c.vacuum_permeability, cell_length=c.cell_length,
                 periodic=tuple(c.bc_lo[d] == BC_PERIODIC for d in range(3)), start=start)

    def load_dc(self, path: str) -> dict:
        """Sets the state from a reference .dc file of this grid's size; returns its header."""
        info, U = read_dc(path)
        if info["n"] != tuple(int(v) for v in self.cfg.n):
            raise PamhdError(ERR_ARGUMENT, f"load_dc: {path} holds {info['n']} cells, the grid {tuple(self.cfg.n)}")
        self.set_state(U)
        return info

    def halo(self, side: int, ghost: int):
        """Device addresses of the eight variables' z plane (pamhd_gpu_halo) in the current state
        and the plane length in doubles."""
        fn = self.L.pamhd_gpu_halo
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_void_p), _P(ctypes.c_int64)]
        planes = (ctypes.c_void_p * 8)()
        count = ctypes.c_int64(0)
        self._check(fn(self.h, side, ghost, planes, ctypes.byref(count)), "pamhd_gpu_halo")
        return [int(p) for p in planes], int(count.value)

    def speed_slot(self) -> int:
        """Device address of the speed reduction the next step reads (pamhd_gpu_speed_slot)."""
        fn = self.L.pamhd_gpu_speed_slot
        fn.argtypes = [ctypes.c_void_p, _P(ctypes.c_void_p)]
        p = ctypes.c_void_p()
        self._check(fn(self.h, ctypes.byref(p)), "pamhd_gpu_speed_slot")
        return int(p.value)

    def stream(self) -> int:
        """The cudaStream_t of the context, as an integer handle."""
        s = ctypes.c_void_p()
        self._check(self.L.pamhd_gpu_get_stream(self.h, ctypes.byref(s)), "pamhd_gpu_get_stream")
        return int(s.value or 0)

    def sync(self):
        self._check(self.L.pamhd_gpu_sync(self.h), "pamhd_gpu_sync")

    def steps_dt(self, dts):
        """Steps with the given dt each (a frozen schedule) instead of the CFL rule."""
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        self._check(self.L.pamhd_gpu_steps_dt(self.h, len(dts), dts.ctypes.data_as(_DP)), "pamhd_gpu_steps_dt")

    def adjoint(self, nsteps: int, every: int, seed: np.ndarray, dt_in=None):
        """Runs nsteps steps (checkpoint every `every`) and returns (grad, grad_value, dts):
        grad = (dU_N/dU_0)^T seed, grad_value = gradient with respect to the VALUE side states
        (3, 2, 8), dts = the dt schedule used."""
        seed = np.ascontiguousarray(seed, dtype=np.float64).reshape((8,) + self.shape)
        grad = np.zeros((8,) + self.shape)
        gv = np.zeros(48)
        dts = np.zeros(nsteps)
        din = None
        if dt_in is not None:
            dt_in = np.ascontiguousarray(dt_in, dtype=np.float64)
            din = dt_in.ctypes.data_as(_DP)
        rc = self.L.pamhd_gpu_adjoint(self.h, int(nsteps), int(every),
                                      _pointers([seed[k].ctypes.data for k in range(8)]),
                                      _pointers([grad[k].ctypes.data for k in range(8)]),
                                      gv.ctypes.data_as(_DP), din, dts.ctypes.data_as(_DP))
        self._check(rc, "pamhd_gpu_adjoint")
        return grad, gv.reshape(3, 2, 8), dts

    def time(self):
        t, n, dt = ctypes.c_double(0), ctypes.c_int64(0), ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_time(self.h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(dt)),
                    "pamhd_gpu_time")
        return t.value, n.value, dt.value

    def dt_history(self, count: int) -> np.ndarray:
        out = np.zeros(count)
        w = ctypes.c_int32(0)
        self._check(self.L.pamhd_gpu_dt_history(self.h, out.ctypes.data_as(_DP), count, ctypes.byref(w)),
                    "pamhd_gpu_dt_history")
        return out[: w.value]

    def status(self):
        f = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.L.pamhd_gpu_status(self.h, ctypes.byref(f), cell, ctypes.byref(d))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_status")
        return f.value, tuple(cell), d.value

    def totals(self) -> np.ndarray:
        out = np.zeros(8)
        self._check(self.L.pamhd_gpu_totals(self.h, out.ctypes.data_as(_DP)), "pamhd_gpu_totals")
        return out


def staggered_face_shapes(cfg: Config):
    """Shapes (z, y, x) of the three face arrays of a staggered grid: the -d face of every cell,
    and along a bounded dimension (not periodic, two cells or more) the high wall as well."""
    shapes = []
    for d in range(3):
        ext = [int(cfg.n[2]), int(cfg.n[1]), int(cfg.n[0])]
        if int(cfg.n[d]) > 1 and not (cfg.bc_lo[d] == BC_PERIODIC and cfg.bc_hi[d] == BC_PERIODIC):
            ext[2 - d] += 1
        shapes.append(tuple(ext))
    return shapes


class StaggeredContext:
    """A pamhd_stag: the staggered-field step (face magnetic field by constrained transport) on
    one uniform grid, periodic or bounded (COPY / VALUE sides, a layer of boundary cells as the
    reference's solar-wind box).  Cell arrays are (8, nz, ny, nx) as Context; face arrays: the
    normal field of every cell's -x, -y and -z face, n + 1 along a bounded dimension
    (staggered_face_shapes); on a periodic grid the three come as one (3, nz, ny, nx) array."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.L = lib()
        L = self.L
        V = ctypes.c_void_p
        L.pamhd_gpu_staggered_create.argtypes = [_P(_Cfg), _P(V)]
        L.pamhd_gpu_staggered_destroy.argtypes = [V]
        L.pamhd_gpu_staggered_set_state.argtypes = [V, V, V]
        L.pamhd_gpu_staggered_get_state.argtypes = [V, V, V]
        L.pamhd_gpu_staggered_set_background.argtypes = [V, V]
        L.pamhd_gpu_staggered_step.argtypes = [V, _D, _DP]
        L.pamhd_gpu_staggered_steps.argtypes = [V, ctypes.c_int32, _D]
        L.pamhd_gpu_staggered_sync.argtypes = [V]
        L.pamhd_gpu_staggered_time.argtypes = [V, _DP, _P(ctypes.c_int64), _DP]
        L.pamhd_gpu_staggered_status.argtypes = [V, _P(ctypes.c_uint32), _P(ctypes.c_int32), _P(ctypes.c_int32)]
        L.pamhd_gpu_staggered_get_stream.argtypes = [V, _P(V)]
        L.pamhd_gpu_staggered_set_inflow.argtypes = [V, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]
        self.shape = (int(cfg.n[2]), int(cfg.n[1]), int(cfg.n[0]))
        self.face_shapes = staggered_face_shapes(cfg)
        self.periodic = all(f == self.shape for f in self.face_shapes)
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        rc = L.pamhd_gpu_staggered_create(ctypes.byref(self._c), ctypes.byref(h))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_staggered_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pamhd_gpu_staggered_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc == ERR_PHYSICS:
            flags, cell, d = self.status()
            raise PhysicsError(rc, what, flags, cell, d)
        if rc != OK:
            raise PamhdError(rc, what)

    def set_state(self, U: np.ndarray, faces):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((8,) + self.shape)
        arrays = []
        for d in range(3):
            a = np.ascontiguousarray(faces[d], dtype=np.float64)
            if a.shape != self.face_shapes[d]:
                raise ValueError(f"set_state: faces[{d}] of shape {self.face_shapes[d]} expected, {a.shape} given")
            arrays.append(a)
        fp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrays])
        self._check(self.L.pamhd_gpu_staggered_set_state(self.h, _pointers([U[k].ctypes.data for k in range(8)]), fp),
                    "pamhd_gpu_staggered_set_state")

    def set_inflow(self, dim: int, side: int, times, states):
        """Time-stamped states of the VALUE side (pamhd_gpu_staggered_set_inflow): states[i] (8
        conservative values) holds while i of the increasing timestamps are <= the time."""
        times = np.ascontiguousarray(times, dtype=np.float64).reshape(-1)
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
        if len(states) != len(times) + 1:
            raise ValueError("set_inflow: one more state than timestamps")
        self._check(self.L.pamhd_gpu_staggered_set_inflow(self.h, int(dim), int(side), len(times),
                                                          times.ctypes.data_as(_DP), states.ctypes.data_as(_DP)),
                    "pamhd_gpu_staggered_set_inflow")

    def set_background(self, bg):
        """bg: (3, 3, nz, ny, nx), bg[d, c] = component c of the background field at every cell's
        -d face; None removes it."""
        if bg is None:
            self._check(self.L.pamhd_gpu_staggered_set_background(self.h, None), "pamhd_gpu_staggered_set_background")
            return
        bg = np.ascontiguousarray(bg, dtype=np.float64).reshape((9,) + self.shape)
        ptrs = (ctypes.c_void_p * 9)(*[bg[k].ctypes.data for k in range(9)])
        self._check(self.L.pamhd_gpu_staggered_set_background(self.h, ptrs), "pamhd_gpu_staggered_set_background")

    def get_state(self, out=None):
        """Returns (U, faces); out: an optional pair of C-contiguous float64 arrays of those shapes to
        fill (pinned host memory makes the copy run at full speed).  faces is one (3, nz, ny, nx)
        array on a periodic grid, a list of the three face arrays on a bounded one."""
        if out is None:
            out = (np.empty((8,) + self.shape),
                   np.empty((3,) + self.shape) if self.periodic else [np.empty(f) for f in self.face_shapes])
        U, faces = out
        checks = [(U, (8,) + self.shape)] + [(faces[d], self.face_shapes[d]) for d in range(3)]
        for a, shape in checks:
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("get_state: out arrays must be C-contiguous float64 of the state's shapes")
        fp = (ctypes.c_void_p * 3)(*[faces[d].ctypes.data for d in range(3)])
        self._check(self.L.pamhd_gpu_staggered_get_state(self.h, _pointers([U[k].ctypes.data for k in range(8)]), fp),
                    "pamhd_gpu_staggered_get_state")
        return U, faces

    def step(self, max_dt: float) -> float:
        dt = ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_staggered_step(self.h, max_dt, ctypes.byref(dt)), "pamhd_gpu_staggered_step")
        return dt.value

    def save_dc(self, path: str, step: int, time: float, proton_mass: float = 1.0, start=(0.0, 0.0, 0.0)):
        """Writes the cell state (mass, momentum, energy, volume field) as a reference .dc file,
        the variable the reference's MHD program saves (mhd/save.hpp:75-375)."""
        c = self.cfg
        periodic = tuple(c.bc_lo[d] == BC_PERIODIC and c.bc_hi[d] == BC_PERIODIC for d in range(3))
        write_dc(path, self.get_state()[0], step=step, time=time, adiabatic_index=c.adiabatic_index,
                 proton_mass=proton_mass, vacuum_permeability=c.vacuum_permeability, cell_length=c.cell_length,
                 periodic=periodic, start=start)

    def steps(self, n: int, t_end: float):
        self._check(self.L.pamhd_gpu_staggered_steps(self.h, int(n), float(t_end)), "pamhd_gpu_staggered_steps")

    def sync(self):
        self._check(self.L.pamhd_gpu_staggered_sync(self.h), "pamhd_gpu_staggered_sync")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.pamhd_gpu_staggered_get_stream(self.h, ctypes.byref(s)), "pamhd_gpu_staggered_get_stream")
        return s.value or 0

    def time(self):
        t, n, dt = ctypes.c_double(0), ctypes.c_int64(0), ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_staggered_time(self.h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(dt)),
                    "pamhd_gpu_staggered_time")
        return t.value, n.value, dt.value

    def status(self):
        f = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.L.pamhd_gpu_staggered_status(self.h, ctypes.byref(f), cell, ctypes.byref(d))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_staggered_status")
        return f.value, tuple(cell), d.value


class TwoPopulationContext:
    """A pamhd_npop: the two-population step (N_solve + apply_fluxes_N) on one uniform periodic
    grid.  State arrays are (13, nz, ny, nx): rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz."""

    def __init__(self, n, cell_length, solver=RUSANOV, adiabatic_index=5.0 / 3.0, vacuum_permeability=1.0,
                 min_pressure=0.0, device=0):
        self.L = lib()
        L = self.L
        V = ctypes.c_void_p
        I3 = ctypes.c_int32 * 3
        D3 = ctypes.c_double * 3
        L.pamhd_gpu_npop_create.argtypes = [I3, D3, ctypes.c_int32, _D, _D, _D, ctypes.c_int32, _P(V)]
        L.pamhd_gpu_npop_destroy.argtypes = [V]
        L.pamhd_gpu_npop_set_state.argtypes = [V, V]
        L.pamhd_gpu_npop_get_state.argtypes = [V, V]
        L.pamhd_gpu_npop_step.argtypes = [V, _D, _DP]
        L.pamhd_gpu_npop_run.argtypes = [V, ctypes.c_int32, _D, _D]
        L.pamhd_gpu_npop_sync.argtypes = [V]
        L.pamhd_gpu_npop_time.argtypes = [V, _DP, _P(ctypes.c_int64), _DP]
        L.pamhd_gpu_npop_status.argtypes = [V, _P(ctypes.c_uint32), _P(ctypes.c_int32), _P(ctypes.c_int32)]
        L.pamhd_gpu_npop_get_stream.argtypes = [V, _P(V)]
        self.shape = (int(n[2]), int(n[1]), int(n[0]))
        h = ctypes.c_void_p()
        rc = L.pamhd_gpu_npop_create(I3(*[int(v) for v in n]), D3(*[float(v) for v in cell_length]), int(solver),
                                     float(adiabatic_index), float(vacuum_permeability), float(min_pressure),
                                     int(device), ctypes.byref(h))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_npop_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pamhd_gpu_npop_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc == ERR_PHYSICS:
            flags, cell, d = self.status()
            raise PhysicsError(rc, what, flags, cell, d)
        if rc != OK:
            raise PamhdError(rc, what)

    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((13,) + self.shape)
        ptrs = (ctypes.c_void_p * 13)(*[U[k].ctypes.data for k in range(13)])
        self._check(self.L.pamhd_gpu_npop_set_state(self.h, ptrs), "pamhd_gpu_npop_set_state")

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """Returns the state (13, nz, ny, nx); out: an optional C-contiguous float64 array to fill."""
        U = out if out is not None else np.empty((13,) + self.shape)
        if U.shape != (13,) + self.shape or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError("get_state: out must be C-contiguous float64 of shape (13, nz, ny, nx)")
        ptrs = (ctypes.c_void_p * 13)(*[U[k].ctypes.data for k in range(13)])
        self._check(self.L.pamhd_gpu_npop_get_state(self.h, ptrs), "pamhd_gpu_npop_get_state")
        return U

    def step(self, dt: float) -> float:
        """One step of length dt; returns the next step's limit (min over faces of d_len / speed)."""
        m = ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_npop_step(self.h, float(dt), ctypes.byref(m)), "pamhd_gpu_npop_step")
        return m.value

    def run(self, n: int, cfl: float, t_end: float):
        self._check(self.L.pamhd_gpu_npop_run(self.h, int(n), float(cfl), float(t_end)), "pamhd_gpu_npop_run")

    def sync(self):
        self._check(self.L.pamhd_gpu_npop_sync(self.h), "pamhd_gpu_npop_sync")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.pamhd_gpu_npop_get_stream(self.h, ctypes.byref(s)), "pamhd_gpu_npop_get_stream")
        return s.value or 0

    def time(self):
        t, n, dt = ctypes.c_double(0), ctypes.c_int64(0), ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_npop_time(self.h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(dt)),
                    "pamhd_gpu_npop_time")
        return t.value, n.value, dt.value

    def status(self):
        f = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.L.pamhd_gpu_npop_status(self.h, ctypes.byref(f), cell, ctypes.byref(d))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_npop_status")
        return f.value, tuple(cell), d.value


class SubstepContext:
    """A pamhd_sub: the cell-centred step with local time stepping on one uniform periodic grid.
    State arrays (8, nz, ny, nx) as Context; exponent bounds (nz, ny, nx) int32."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.L = lib()
        L = self.L
        V = ctypes.c_void_p
        I = _P(ctypes.c_int32)
        L.pamhd_gpu_substep_create.argtypes = [_P(_Cfg), _P(V)]
        L.pamhd_gpu_substep_destroy.argtypes = [V]
        L.pamhd_gpu_substep_set_state.argtypes = [V, V]
        L.pamhd_gpu_substep_get_state.argtypes = [V, V]
        L.pamhd_gpu_substep_set_exponents.argtypes = [V, I, I]
        L.pamhd_gpu_substep_step.argtypes = [V, _D, _DP, I]
        L.pamhd_gpu_substep_periods.argtypes = [V, I]
        L.pamhd_gpu_substep_status.argtypes = [V, _P(ctypes.c_uint32), I, I]
        self.shape = (int(cfg.n[2]), int(cfg.n[1]), int(cfg.n[0]))
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        rc = L.pamhd_gpu_substep_create(ctypes.byref(self._c), ctypes.byref(h))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_substep_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pamhd_gpu_substep_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc == ERR_PHYSICS:
            flags, cell, d = self.status()
            raise PhysicsError(rc, what, flags, cell, d)
        if rc != OK:
            raise PamhdError(rc, what)

    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((8,) + self.shape)
        self._check(self.L.pamhd_gpu_substep_set_state(self.h, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_substep_set_state")

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """Returns the state (8, nz, ny, nx); out: an optional C-contiguous float64 array to fill."""
        U = out if out is not None else np.empty((8,) + self.shape)
        if U.shape != (8,) + self.shape or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError("get_state: out must be C-contiguous float64 of shape (8, nz, ny, nx)")
        self._check(self.L.pamhd_gpu_substep_get_state(self.h, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_substep_get_state")
        return U

    def set_exponents(self, mins, maxs):
        a = np.ascontiguousarray(mins, dtype=np.int32).reshape(-1)
        b = np.ascontiguousarray(maxs, dtype=np.int32).reshape(-1)
        I = _P(ctypes.c_int32)
        self._check(self.L.pamhd_gpu_substep_set_exponents(self.h, a.ctypes.data_as(I), b.ctypes.data_as(I)),
                    "pamhd_gpu_substep_set_exponents")

    def step(self, max_dt: float):
        """Returns (dt, substeps)."""
        dt = ctypes.c_double(0)
        k = ctypes.c_int32(0)
        self._check(self.L.pamhd_gpu_substep_step(self.h, float(max_dt), ctypes.byref(dt), ctypes.byref(k)),
                    "pamhd_gpu_substep_step")
        return dt.value, k.value

    def periods(self) -> np.ndarray:
        p = np.empty(self.shape, dtype=np.int32)
        self._check(self.L.pamhd_gpu_substep_periods(self.h, p.ctypes.data_as(_P(ctypes.c_int32))),
                    "pamhd_gpu_substep_periods")
        return p

    def status(self):
        f = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.L.pamhd_gpu_substep_status(self.h, ctypes.byref(f), cell, ctypes.byref(d))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_substep_status")
        return f.value, tuple(cell), d.value


def _check_face_shapes(neg, pos, bg):
    """The C entry points read n rows of every array: refuse arrays of other shapes before the
    call (a shorter array would be read past its end)."""
    if neg.ndim != 2 or neg.shape[1] != 8 or pos.shape != neg.shape:
        raise ValueError(f"neg and pos must both be (n, 8); got {neg.shape} and {pos.shape}")
    if bg is not None and np.shape(bg) != (neg.shape[0], 3):
        raise ValueError(f"bg must be None or ({neg.shape[0]}, 3); got {np.shape(bg)}")


def face_flux(solver, neg, pos, bg=None, gamma=5.0 / 3.0, mu0=1.0, device=0):
    """Solver-level entry point (pamhd_gpu_face_flux).  neg, pos: (n, 8); bg: (n, 3) or None.
    Returns flux (n, 8), speed (n,), flags (n,); failed faces have flags != 0 (no exception)."""
    L = lib()
    neg = np.ascontiguousarray(neg, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    _check_face_shapes(neg, pos, bg)
    n = neg.shape[0]
    flux = np.zeros((n, 8))
    speed = np.zeros(n)
    flags = np.zeros(n, dtype=np.uint32)
    bgp = None
    if bg is not None:
        bg = np.ascontiguousarray(bg, dtype=np.float64)
        bgp = bg.ctypes.data_as(_DP)
    rc = L.pamhd_gpu_face_flux(device, solver, n, neg.ctypes.data_as(_DP), pos.ctypes.data_as(_DP), bgp,
                               gamma, mu0, flux.ctypes.data_as(_DP), speed.ctypes.data_as(_DP),
                               flags.ctypes.data_as(_P(ctypes.c_uint32)))
    if rc not in (OK, ERR_PHYSICS):
        raise PamhdError(rc, "pamhd_gpu_face_flux")
    return flux, speed, flags


def face_flux_noalloc(solver, neg, pos, bg=None, gamma=5.0 / 3.0, mu0=1.0, device=0):
    """face_flux through pamhd_gpu_face_flux_noalloc: no device allocation, at most
    NOALLOC_MAX_FACES faces per call (PamhdError with ERR_TOO_LARGE beyond that); calls on one
    device share one scratch area, so concurrent calls from several threads race."""
    L = lib()
    fn = L.pamhd_gpu_face_flux_noalloc
    fn.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, _DP, _DP, _DP, _D, _D, _DP, _DP,
                   _P(ctypes.c_uint32)]
    neg = np.ascontiguousarray(neg, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    _check_face_shapes(neg, pos, bg)
    n = neg.shape[0]
    flux = np.zeros((n, 8))
    speed = np.zeros(n)
    flags = np.zeros(n, dtype=np.uint32)
    bgp = None
    if bg is not None:
        bg = np.ascontiguousarray(bg, dtype=np.float64)
        bgp = bg.ctypes.data_as(_DP)
    rc = fn(device, solver, n, neg.ctypes.data_as(_DP), pos.ctypes.data_as(_DP), bgp, gamma, mu0,
            flux.ctypes.data_as(_DP), speed.ctypes.data_as(_DP), flags.ctypes.data_as(_P(ctypes.c_uint32)))
    if rc not in (OK, ERR_PHYSICS):
        raise PamhdError(rc, "pamhd_gpu_face_flux_noalloc")
    return flux, speed, flags


class DcInfo(ctypes.Structure):
    """pamhd_dc_info of include/pamhd_gpu.h: the header of a .dc file."""

    _fields_ = [
        ("step", ctypes.c_uint64),
        ("time", ctypes.c_double),
        ("adiabatic_index", ctypes.c_double),
        ("proton_mass", ctypes.c_double),
        ("vacuum_permeability", ctypes.c_double),
        ("n", ctypes.c_int32 * 3),
        ("periodic", ctypes.c_int32 * 3),
        ("start", ctypes.c_double * 3),
        ("cell_length", ctypes.c_double * 3),
        ("cells", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {"step": int(self.step), "time": self.time, "adiabatic_index": self.adiabatic_index,
                "proton_mass": self.proton_mass, "vacuum_permeability": self.vacuum_permeability,
                "n": tuple(self.n), "periodic": tuple(bool(p) for p in self.periodic),
                "start": tuple(self.start), "cell_length": tuple(self.cell_length), "cells": int(self.cells)}


def write_dc(path: str, U: np.ndarray, *, step: int, time: float, adiabatic_index: float, proton_mass: float,
             vacuum_permeability: float, cell_length, periodic=(True, True, True), start=(0.0, 0.0, 0.0)):
    """Writes the state U (8, nz, ny, nx) as a reference .dc file (pamhd_dc_write)."""
    L = lib()
    L.pamhd_dc_write.argtypes = [ctypes.c_char_p, _P(DcInfo), ctypes.c_void_p]
    U = np.ascontiguousarray(U, dtype=np.float64)
    info = DcInfo()
    info.step = int(step)
    info.time = float(time)
    info.adiabatic_index = float(adiabatic_index)
    info.proton_mass = float(proton_mass)
    info.vacuum_permeability = float(vacuum_permeability)
    for d in range(3):
        info.n[d] = int(U.shape[3 - d])
        info.periodic[d] = int(bool(periodic[d]))
        info.start[d] = float(start[d])
        info.cell_length[d] = float(cell_length[d])
    rc = L.pamhd_dc_write(os.fsencode(path), ctypes.byref(info), _pointers([U[k].ctypes.data for k in range(8)]))
    if rc != OK:
        raise PamhdError(rc, "pamhd_dc_write")


def read_dc(path: str):
    """Reads a reference .dc file of a uniform grid: (header dict, state (8, nz, ny, nx))."""
    L = lib()
    L.pamhd_dc_read_info.argtypes = [ctypes.c_char_p, _P(DcInfo)]
    L.pamhd_dc_read.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    info = DcInfo()
    rc = L.pamhd_dc_read_info(os.fsencode(path), ctypes.byref(info))
    if rc != OK:
        raise PamhdError(rc, "pamhd_dc_read_info")
    U = np.empty((8, info.n[2], info.n[1], info.n[0]))
    rc = L.pamhd_dc_read(os.fsencode(path), _pointers([U[k].ctypes.data for k in range(8)]))
    if rc != OK:
        raise PamhdError(rc, "pamhd_dc_read")
    return info.as_dict(), U


class Batch:
    """A pamhd_batch: independent boxes advanced together, each with its own timestep."""

    def __init__(self, cfgs, device: int = 0):
        self.L = lib()
        self.cfgs = list(cfgs)
        self.shapes = [(int(c.n[2]), int(c.n[1]), int(c.n[0])) for c in self.cfgs]
        arr = (_Cfg * len(self.cfgs))(*[c.to_c() for c in self.cfgs])
        self._arr = arr
        h = ctypes.c_void_p()
        rc = self.L.pamhd_gpu_batch_create(device, len(self.cfgs), arr, ctypes.byref(h))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pamhd_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what, box=None):
        if rc == ERR_PHYSICS:
            boxes = range(len(self.cfgs)) if box is None else [box]
            for b in boxes:
                flags, cell, d = self.status(b)
                if flags:
                    raise PhysicsError(rc, f"{what} (box {b})", flags, cell, d)
            raise PhysicsError(rc, what)
        if rc != OK:
            raise PamhdError(rc, what)

    def set_state(self, box: int, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape((8,) + self.shapes[box])
        self._check(self.L.pamhd_gpu_batch_set_state(self.h, box, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_batch_set_state")

    def tiling(self):
        """(tile rows, z planes per work item, grid) in use (pamhd_gpu_batch_tiling)."""
        fn = self.L.pamhd_gpu_batch_tiling
        fn.argtypes = [ctypes.c_void_p, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32)]
        t, p, g = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
        self._check(fn(self.h, ctypes.byref(t), ctypes.byref(p), ctypes.byref(g)), "pamhd_gpu_batch_tiling")
        return t.value, p.value, g.value

    def set_tiling(self, tile_rows: int, planes: int, grid: int):
        """Sets the work split (pamhd_gpu_batch_set_tiling)."""
        fn = self.L.pamhd_gpu_batch_set_tiling
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        self._check(fn(self.h, tile_rows, planes, grid), "pamhd_gpu_batch_set_tiling")

    def set_inflow(self, box: int, dim: int, side: int, times, states):
        """Time-stamped inflow of a VALUE side of one box (pamhd_gpu_batch_set_inflow)."""
        fn = self.L.pamhd_gpu_batch_set_inflow
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]
        times = np.ascontiguousarray(times, dtype=np.float64).reshape(-1)
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
        if len(states) != len(times) + 1:
            raise ValueError("set_inflow: one state more than timestamps")
        self._check(fn(self.h, box, dim, side, len(times), times.ctypes.data_as(_DP), states.ctypes.data_as(_DP)),
                    "pamhd_gpu_batch_set_inflow", box)

    def get_state(self, box: int) -> np.ndarray:
        U = np.empty((8,) + self.shapes[box])
        self._check(self.L.pamhd_gpu_batch_get_state(self.h, box, _pointers([U[k].ctypes.data for k in range(8)])),
                    "pamhd_gpu_batch_get_state")
        return U

    def steps(self, n: int, t_end: float = 1e300):
        self._check(self.L.pamhd_gpu_batch_steps(self.h, int(n), float(t_end)), "pamhd_gpu_batch_steps")

    def tune(self, trial_steps: int = 3):
        planes, grid = ctypes.c_int32(0), ctypes.c_int32(0)
        self._check(self.L.pamhd_gpu_batch_tune(self.h, trial_steps, ctypes.byref(planes), ctypes.byref(grid)),
                    "pamhd_gpu_batch_tune")
        return planes.value, grid.value

    def run(self, n: int, t_end: float = 1e300):
        """n steps of every box in one persistent launch, graph-replayed (pamhd_gpu_batch_run)."""
        fn = self.L.pamhd_gpu_batch_run
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, _D]
        self._check(fn(self.h, int(n), float(t_end)), "pamhd_gpu_batch_run")

    def set_wait_limit(self, polls: int):
        """Polls a wait of the persistent run makes before it gives up (pamhd_gpu_batch_set_wait_limit)."""
        fn = self.L.pamhd_gpu_batch_set_wait_limit
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        self._check(fn(self.h, int(polls)), "pamhd_gpu_batch_set_wait_limit")

    def run_info(self):
        """(blocks, work items per step, graph-replayed) of the persistent run (pamhd_gpu_batch_run_info)."""
        fn = self.L.pamhd_gpu_batch_run_info
        fn.argtypes = [ctypes.c_void_p, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32)]
        g, i, r = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
        self._check(fn(self.h, ctypes.byref(g), ctypes.byref(i), ctypes.byref(r)), "pamhd_gpu_batch_run_info")
        return g.value, i.value, bool(r.value)

    def tune_run(self, trial_steps: int = 3):
        """Autotuner of the persistent run (pamhd_gpu_batch_tune_run): (tile rows, z planes per item)."""
        fn = self.L.pamhd_gpu_batch_tune_run
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_int32), _P(ctypes.c_int32)]
        t, p = ctypes.c_int32(0), ctypes.c_int32(0)
        self._check(fn(self.h, trial_steps, ctypes.byref(t), ctypes.byref(p)), "pamhd_gpu_batch_tune_run")
        return t.value, p.value

    def sync(self):
        self._check(self.L.pamhd_gpu_batch_sync(self.h), "pamhd_gpu_batch_sync")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.pamhd_gpu_batch_get_stream(self.h, ctypes.byref(s)), "pamhd_gpu_batch_get_stream")
        return int(s.value or 0)

    def time(self, box: int):
        t, n, dt = ctypes.c_double(0), ctypes.c_int64(0), ctypes.c_double(0)
        self._check(self.L.pamhd_gpu_batch_time(self.h, box, ctypes.byref(t), ctypes.byref(n), ctypes.byref(dt)),
                    "pamhd_gpu_batch_time")
        return t.value, n.value, dt.value

    def dt_history(self, box: int, count: int) -> np.ndarray:
        out = np.zeros(count)
        w = ctypes.c_int32(0)
        self._check(self.L.pamhd_gpu_batch_dt_history(self.h, box, out.ctypes.data_as(_DP), count, ctypes.byref(w)),
                    "pamhd_gpu_batch_dt_history")
        return out[: w.value]

    def status(self, box: int):
        f = ctypes.c_uint32(0)
        cell = (ctypes.c_int32 * 3)()
        d = ctypes.c_int32(0)
        rc = self.L.pamhd_gpu_batch_status(self.h, box, ctypes.byref(f), cell, ctypes.byref(d))
        if rc != OK:
            raise PamhdError(rc, "pamhd_gpu_batch_status")
        return f.value, tuple(cell), d.value
