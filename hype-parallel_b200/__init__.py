"""hype_parallel_b200 -- Python view of the C ABI in include/hype_gpu.h.

The product is the shared library ``lib/libhype_b200.so`` (sm_100a kernels and
their C host runtime).  This module only binds it with ctypes so that tests,
benchmarks and Python callers reach the same entry points a C caller (or the
PETSc glue, csrc/petsc_glue.c) would.  It never computes on the CPU: if the
library is missing it raises, and every call goes through the CUDA path.

Mirrors HyPE-2D's interface for the hot path:

* ``Solver.rhs_function_prim(t, U, RHS)`` -- ``RHSFunctionPrim`` (rhs_function_prim.c:12,
  hype.h:306): fills RHS, returns the Ctx->dt it sets.
* ``Solver.solve(t0, t_final, max_steps)`` -- the TS loop of hype.c:337-384.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libhype_b200.so")

# include/hype_gpu.h
OK, ERR_INVALID, ERR_CUDA, ERR_INADMISSIBLE, ERR_TIMEOUT, ERR_NOMEM, ERR_NO_DEVICE, ERR_BUSY = range(8)
EULER, KAPILA_5EQN, BAER_NUNZIATO = 0, 1, 2
BC_WALL, BC_INLET, BC_PERIODIC, BC_REFLECTIVE, BC_TRANSMISSIVE = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1
FLAG_BN_FIX_P2 = 1
NVAR = {EULER: 4, KAPILA_5EQN: 6, BAER_NUNZIATO: 9}


class HypeError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class _Cfg(ctypes.Structure):
    _fields_ = [("system", ctypes.c_int), ("order", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double), ("y_min", ctypes.c_double),
                ("y_max", ctypes.c_double), ("cfl", ctypes.c_double),
                ("bc_left", ctypes.c_int), ("bc_right", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_top", ctypes.c_int),
                ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("pi1", ctypes.c_double), ("pi2", ctypes.c_double),
                ("precision", ctypes.c_int), ("flags", ctypes.c_uint), ("device", ctypes.c_int)]


@dataclasses.dataclass
class Config:
    """Run-time form of HyPE-2D's compile-time and AppCtx parameters (hype_config)."""
    system: int = KAPILA_5EQN
    order: int = 2
    nx: int = 256
    ny: int = 256
    x_min: float = 0.0
    x_max: float = 1.0
    y_min: float = 0.0
    y_max: float = 1.0
    cfl: float = 0.4
    bc_left: int = BC_TRANSMISSIVE
    bc_right: int = BC_TRANSMISSIVE
    bc_bottom: int = BC_TRANSMISSIVE
    bc_top: int = BC_TRANSMISSIVE
    gamma1: float = 4.4
    gamma2: float = 1.4
    pi1: float = 6.0e8
    pi2: float = 0.0
    precision: int = PREC_FP64
    flags: int = 0
    device: int = 0

    @property
    def nvar(self) -> int:
        return NVAR[self.system]

    def c_struct(self) -> _Cfg:
        return _Cfg(**dataclasses.asdict(self))


_DP = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> None:
    """Compile lib/libhype_b200.so (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    """The loaded C library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C hype-parallel_b200`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.hype_create.argtypes = [ctypes.POINTER(_Cfg), ctypes.POINTER(vp)]
        L.hype_destroy.argtypes = [vp]
        L.hype_last_error.argtypes = [vp]
        L.hype_last_error.restype = ctypes.c_char_p
        L.hype_status_string.restype = ctypes.c_char_p
        L.hype_rhs_prim.argtypes = [vp, ctypes.c_double, _DP, _DP, _DP]
        L.hype_rhs_prim_device.argtypes = [vp, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, _DP]
        L.hype_set_state.argtypes = [vp, _DP]
        L.hype_get_state.argtypes = [vp, _DP]
        L.hype_solve.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        L.hype_begin.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.hype_advance.argtypes = [vp, ctypes.c_int]
        L.hype_wait.argtypes = [vp, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        L.hype_totals.argtypes = [vp, ctypes.c_int, _DP, _DP, _DP]
        L.hype_launch_info.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 3 + [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        L.hype_last_elapsed_ms.argtypes = [vp, _DP]
        L.hype_time_stage.argtypes = [vp, ctypes.c_int, _DP]
        L.hype_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.hype_config_default.argtypes = [ctypes.POINTER(_Cfg)]
        for name in ("hype_ic_shock_bubble",):
            getattr(L, name).argtypes = [ctypes.POINTER(_Cfg), ctypes.c_uint64, ctypes.c_int, _DP]
        for name in ("hype_ic_bn_discs", "hype_ic_euler_quadrants"):
            getattr(L, name).argtypes = [ctypes.POINTER(_Cfg), ctypes.c_uint64, _DP]
        L.hype_ic_smooth_vortex.argtypes = [ctypes.POINTER(_Cfg), _DP]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def default_config() -> Config:
    c = _Cfg()
    lib().hype_config_default(ctypes.byref(c))
    return Config(**{f: getattr(c, f) for f, _ in _Cfg._fields_})


# ---------------------------------------------------------------------------
# seeded initial data (host code in the library)
# ---------------------------------------------------------------------------
def initial_state(cfg: Config, kind: str, seed: int = 0, nbubbles: int = 1) -> np.ndarray:
    U = np.empty(cfg.nx * cfg.ny * cfg.nvar, dtype=np.float64)
    c = cfg.c_struct()
    L = lib()
    if kind == "shock_bubble":
        st = L.hype_ic_shock_bubble(ctypes.byref(c), seed, nbubbles, _ptr(U))
    elif kind == "bn_discs":
        st = L.hype_ic_bn_discs(ctypes.byref(c), seed, _ptr(U))
    elif kind == "euler_quadrants":
        st = L.hype_ic_euler_quadrants(ctypes.byref(c), seed, _ptr(U))
    elif kind == "smooth_vortex":
        st = L.hype_ic_smooth_vortex(ctypes.byref(c), _ptr(U))
    else:
        raise ValueError(kind)
    if st != OK:
        raise HypeError(st, f"initial state {kind} rejected the configuration")
    return U


class Solver:
    """One grid on one GPU: hype_create / hype_destroy around the drop-in calls."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self._h = ctypes.c_void_p()
        st = lib().hype_create(ctypes.byref(cfg.c_struct()), ctypes.byref(self._h))
        if st != OK:
            msg = lib().hype_last_error(self._h).decode() if self._h else lib().hype_status_string(st).decode()
            lib().hype_destroy(self._h)
            self._h = ctypes.c_void_p()
            raise HypeError(st, msg)

    def close(self):
        if self._h:
            lib().hype_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int) -> None:
        if st != OK:
            raise HypeError(st, lib().hype_last_error(self._h).decode())

    @property
    def n(self) -> int:
        return self.cfg.nx * self.cfg.ny * self.cfg.nvar

    def rhs_function_prim(self, t: float, U: np.ndarray, RHS: np.ndarray | None = None, check: bool = True):
        """RHSFunctionPrim: returns (RHS, dt, status)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n:
            raise ValueError("U has the wrong size")
        if RHS is None:
            RHS = np.empty_like(U)
        dt = ctypes.c_double(0.0)
        st = lib().hype_rhs_prim(self._h, t, _ptr(U), _ptr(RHS), ctypes.byref(dt))
        if check and st not in (OK, ERR_INADMISSIBLE):
            self._check(st)
        return RHS, dt.value, st

    def rhs_function_prim_device(self, t: float, dU: int, dRHS: int):
        dt = ctypes.c_double(0.0)
        st = lib().hype_rhs_prim_device(self._h, t, ctypes.c_void_p(dU), ctypes.c_void_p(dRHS), ctypes.byref(dt))
        return dt.value, st

    def set_state(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n:
            raise ValueError("U has the wrong size")
        self._check(lib().hype_set_state(self._h, _ptr(U)))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        U = np.empty(self.n, dtype=np.float64) if out is None else out
        if U.size != self.n or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of the state size")
        self._check(lib().hype_get_state(self._h, _ptr(U)))
        return U

    def solve(self, t0: float, t_final: float, max_steps: int, check: bool = True):
        """Returns (steps, t_end, dt_next, status)."""
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = lib().hype_solve(self._h, t0, t_final, max_steps, ctypes.byref(steps), ctypes.byref(t), ctypes.byref(dt))
        if check and st not in (OK, ERR_INADMISSIBLE):
            self._check(st)
        return steps.value, t.value, dt.value, st

    def begin(self, t0: float, t_final: float, max_steps: int) -> None:
        self._check(lib().hype_begin(self._h, t0, t_final, max_steps))

    def advance(self, nsteps: int) -> None:
        self._check(lib().hype_advance(self._h, nsteps))

    def wait(self):
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = lib().hype_wait(self._h, ctypes.byref(steps), ctypes.byref(t), ctypes.byref(dt))
        return steps.value, t.value, dt.value, st

    def totals(self, scaled: bool = False):
        tot = np.zeros(self.cfg.nvar)
        amin = ctypes.c_double(0.0)
        amax = ctypes.c_double(0.0)
        self._check(lib().hype_totals(self._h, int(scaled), _ptr(tot), ctypes.byref(amin), ctypes.byref(amax)))
        return tot, amin.value, amax.value

    def launch_info(self) -> dict:
        gx, gy, th, bps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        smem = ctypes.c_size_t()
        self._check(lib().hype_launch_info(self._h, ctypes.byref(gx), ctypes.byref(gy), ctypes.byref(th),
                                           ctypes.byref(smem), ctypes.byref(bps)))
        return {"grid": (gx.value, gy.value), "threads": th.value, "smem": smem.value, "blocks_per_sm": bps.value}

    def time_stage(self, reps: int = 20) -> float:
        """Average milliseconds of one stage-kernel launch (CUDA events)."""
        ms = ctypes.c_double(0.0)
        self._check(lib().hype_time_stage(self._h, reps, ctypes.byref(ms)))
        return ms.value

    def autotune(self, reps: int = 3):
        """Pick the fastest stage-kernel tile shape; returns (tile width, waves)."""
        c, w = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().hype_autotune(self._h, reps, ctypes.byref(c), ctypes.byref(w)))
        return c.value, w.value

    def last_elapsed_ms(self) -> float:
        ms = ctypes.c_double(0.0)
        self._check(lib().hype_last_elapsed_ms(self._h, ctypes.byref(ms)))
        return ms.value
