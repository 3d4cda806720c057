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
PREC_FP64, PREC_MIXED, PREC_FP64_FAST = 0, 1, 2
FLAG_BN_FIX_P2 = 1
FLAG_CONSERVATIVE = 2
FLAG_VISCOUS = 4
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
                ("precision", ctypes.c_int), ("flags", ctypes.c_uint), ("device", ctypes.c_int),
                ("mu1", ctypes.c_double), ("mu2", ctypes.c_double)]


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
    mu1: float = 1.0e-2      # MU_1, MU_2 (hype.h:46-47), read with FLAG_VISCOUS
    mu2: float = 0.0

    @property
    def nvar(self) -> int:
        return NVAR[self.system]

    def c_struct(self) -> _Cfg:
        return _Cfg(**dataclasses.asdict(self))


class _BatchCfg(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_instances", ctypes.c_int), ("hbm_budget", ctypes.c_size_t),
                ("max_cells", ctypes.c_longlong)]


class _InstStatus(ctypes.Structure):
    _fields_ = [("active", ctypes.c_int), ("done", ctypes.c_int), ("steps", ctypes.c_int), ("status", ctypes.c_int),
                ("t", ctypes.c_double), ("dt_next", ctypes.c_double), ("held", ctypes.c_int), ("substeps", ctypes.c_int)]


class _Request(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("cfg", _Cfg), ("t0", ctypes.c_double), ("t_final", ctypes.c_double),
                ("max_steps", ctypes.c_int), ("ic", ctypes.c_int), ("ic_seed", ctypes.c_uint64), ("ic_param", ctypes.c_int)]


class _Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("steps", ctypes.c_int), ("t_end", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("done_s", ctypes.c_double), ("latency_s", ctypes.c_double)]


class _ServeCfg(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_instances", ctypes.c_int), ("hbm_budget", ctypes.c_size_t),
                ("max_cells", ctypes.c_longlong), ("poll_ms", ctypes.c_double), ("realtime", ctypes.c_int),
                ("autotune", ctypes.c_int), ("fetch_results", ctypes.c_int), ("active_cells", ctypes.c_longlong),
                ("substep_cells", ctypes.c_longlong)]


class _ServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int), ("failed", ctypes.c_int), ("wall_s", ctypes.c_double),
                ("p50_s", ctypes.c_double), ("p90_s", ctypes.c_double), ("p99_s", ctypes.c_double),
                ("max_s", ctypes.c_double), ("mean_s", ctypes.c_double), ("queue_p50_s", ctypes.c_double),
                ("queue_p99_s", ctypes.c_double), ("cell_updates", ctypes.c_double),
                ("cell_updates_per_s", ctypes.c_double), ("peak_instances", ctypes.c_int),
                ("peak_bytes", ctypes.c_size_t), ("polls", ctypes.c_longlong), ("steps_replayed", ctypes.c_longlong)]


_FILL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_Request),
                            ctypes.POINTER(ctypes.c_double))
_SINK_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(_Result))

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
        L.hype_advance_host.argtypes = [vp, _DP, _DP, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        L.hype_totals.argtypes = [vp, ctypes.c_int, _DP, _DP, _DP]
        L.hype_launch_info.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 3 + [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        L.hype_last_elapsed_ms.argtypes = [vp, _DP]
        L.hype_test_division.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong)]
        L.hype_test_skip_row_loads.argtypes = [vp, ctypes.c_int]
        L.hype_test_fast_rcp.argtypes = [ctypes.c_int, _DP, ctypes.c_int, _DP, _DP]
        L.hype_time_stage.argtypes = [vp, ctypes.c_int, _DP]
        L.hype_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.hype_config_default.argtypes = [ctypes.POINTER(_Cfg)]
        L.hype_get_primitive.argtypes = [vp, _DP]
        L.hype_fp64_rate.argtypes = [ctypes.c_int, ctypes.c_int, _DP]
        L.hype_fp64_fma_rate.argtypes = [ctypes.c_int, ctypes.c_int, _DP]
        L.hype_group_create.argtypes = [ctypes.POINTER(_Cfg), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(vp)]
        L.hype_group_destroy.argtypes = [vp]
        L.hype_group_last_error.argtypes = [vp]
        L.hype_group_last_error.restype = ctypes.c_char_p
        L.hype_group_slab.argtypes = [vp, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 3
        L.hype_group_set_state.argtypes = [vp, _DP]
        L.hype_group_get_state.argtypes = [vp, _DP]
        L.hype_group_begin.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.hype_group_advance.argtypes = [vp, ctypes.c_int]
        L.hype_group_wait.argtypes = [vp, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        L.hype_group_solve.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        L.hype_group_last_elapsed_ms.argtypes = [vp, _DP]
        L.hype_solver_config.argtypes = [vp, ctypes.POINTER(_Cfg)]
        for name in ("hype_write_restart", "hype_read_restart", "hype_write_vts"):
            getattr(L, name).argtypes = [vp, ctypes.c_char_p]
        L.hype_solve_monitored.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        for name in ("hype_ic_shock_bubble",):
            getattr(L, name).argtypes = [ctypes.POINTER(_Cfg), ctypes.c_uint64, ctypes.c_int, _DP]
        for name in ("hype_ic_bn_discs", "hype_ic_euler_quadrants"):
            getattr(L, name).argtypes = [ctypes.POINTER(_Cfg), ctypes.c_uint64, _DP]
        L.hype_ic_smooth_vortex.argtypes = [ctypes.POINTER(_Cfg), _DP]
        # include/hype_batch.h
        IP = ctypes.POINTER(ctypes.c_int)
        L.hype_batch_config_default.argtypes = [ctypes.POINTER(_BatchCfg)]
        L.hype_batch_create.argtypes = [ctypes.POINTER(_BatchCfg), ctypes.POINTER(vp)]
        L.hype_batch_destroy.argtypes = [vp]
        L.hype_batch_last_error.argtypes = [vp]
        L.hype_batch_last_error.restype = ctypes.c_char_p
        L.hype_batch_instance_bytes.argtypes = [ctypes.POINTER(_Cfg)]
        L.hype_batch_instance_bytes.restype = ctypes.c_size_t
        L.hype_batch_add.argtypes = [vp, ctypes.POINTER(_Cfg), _DP, ctypes.c_double, ctypes.c_double, ctypes.c_int, IP]
        L.hype_batch_remove.argtypes = [vp, ctypes.c_int]
        L.hype_batch_advance.argtypes = [vp, ctypes.c_int]
        L.hype_batch_sync.argtypes = [vp]
        L.hype_batch_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(_InstStatus)]
        L.hype_batch_get_state.argtypes = [vp, ctypes.c_int, _DP]
        L.hype_batch_hold.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.hype_batch_set_substeps.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.hype_batch_set_tiling.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.hype_batch_autotune.argtypes = [vp, ctypes.c_int, IP, IP]
        L.hype_batch_info.argtypes = [vp, IP, IP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
        L.hype_batch_last_elapsed_ms.argtypes = [vp, _DP]
        # include/hype_serve.h
        L.hype_serve_config_default.argtypes = [ctypes.POINTER(_ServeCfg)]
        L.hype_serve_run.argtypes = [ctypes.POINTER(_ServeCfg), ctypes.POINTER(_Request), ctypes.c_int, _FILL_FN, _SINK_FN,
                                     vp, ctypes.POINTER(_Result), ctypes.POINTER(_ServeStats)]
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

    def last_error(self) -> str:
        return lib().hype_last_error(self._h).decode()

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

    def get_primitive(self) -> np.ndarray:
        """Primitive variables of the device state (ComputePrimitiveVariables)."""
        W = np.empty(self.n, dtype=np.float64)
        self._check(lib().hype_get_primitive(self._h, _ptr(W)))
        return W

    def write_restart(self, path: str) -> None:
        self._check(lib().hype_write_restart(self._h, os.fsencode(path)))

    def read_restart(self, path: str) -> int:
        return lib().hype_read_restart(self._h, os.fsencode(path))

    def write_vts(self, path: str) -> None:
        self._check(lib().hype_write_vts(self._h, os.fsencode(path)))

    def solve_monitored(self, t0: float, t_final: float, max_steps: int, write_interval: int, restart_interval: int,
                        directory: str):
        """hype_solve with MonitorFunction's file schedule; returns (steps, t_end, dt_next)."""
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        self._check(lib().hype_solve_monitored(self._h, t0, t_final, max_steps, write_interval, restart_interval,
                                               os.fsencode(directory), ctypes.byref(steps), ctypes.byref(t),
                                               ctypes.byref(dt)))
        return steps.value, t.value, dt.value

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

    def advance_host(self, U_in: np.ndarray, U_out: np.ndarray, nsteps: int = 1):
        """Host state in, nsteps steps, host state out, copies overlapped with
        the first and last steps' stages (hype_advance_host); returns (steps, t, dt_next, status)."""
        for a in (U_in, U_out):
            if a.size != self.n or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("states must be contiguous float64 arrays of the state size")
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = lib().hype_advance_host(self._h, _ptr(U_in), _ptr(U_out), nsteps, ctypes.byref(steps), ctypes.byref(t),
                                     ctypes.byref(dt))
        if st not in (OK, ERR_INADMISSIBLE):
            self._check(st)
        return steps.value, t.value, dt.value, st

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

    def test_skip_row_loads(self, row: int) -> None:
        """Test hook (hype_test_skip_row_loads): issue no row load for rows >= row,
        so the kernels' bounded wait runs out; row < 0 turns it off."""
        self._check(lib().hype_test_skip_row_loads(self._h, row))


def test_fast_rcp(x: np.ndarray, device: int = 0):
    """The FP64 performance form's reciprocal and IEEE 1/x of the same values on
    the GPU (hype_test_fast_rcp): returns (fast, ieee)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    fast, ieee = np.empty_like(x), np.empty_like(x)
    st = lib().hype_test_fast_rcp(device, _ptr(x), x.size, _ptr(fast), _ptr(ieee))
    if st != OK:
        raise HypeError(st, "hype_test_fast_rcp failed")
    return fast, ieee


def fp64_rate(device: int = 0, reps: int = 5) -> float:
    """Measured rate of separately rounded FP64 multiplies and adds on `device`
    (hype_fp64_rate): the FP64 roofline of the bit-exact kernels, in ops/s."""
    r = ctypes.c_double(0.0)
    st = lib().hype_fp64_rate(device, reps, ctypes.byref(r))
    if st != OK:
        raise HypeError(st, lib().hype_status_string(st).decode())
    return r.value


def fp64_fma_rate(device: int = 0, reps: int = 5) -> float:
    """Measured FP64 rate with fused multiply-adds (hype_fp64_fma_rate), FLOP/s
    counting two per FMA: the FP64 roofline of the performance form."""
    r = ctypes.c_double(0.0)
    st = lib().hype_fp64_fma_rate(device, reps, ctypes.byref(r))
    if st != OK:
        raise HypeError(st, "hype_fp64_fma_rate failed")
    return r.value


class Group:
    """One grid split into y-slabs (include/hype_group.h): HyPE-2D's DMDA
    decomposition over ranks, here over the GPUs of one process (`devices`, one
    per slab; default: all slabs on cfg.device).  Same calls as Solver's time
    loop; the results equal a Solver's bit for bit."""

    def __init__(self, cfg: Config, nslabs: int, devices=None):
        self.cfg = cfg
        self.nslabs = nslabs
        self._h = ctypes.c_void_p()
        dev = None
        if devices is not None:
            if len(devices) != nslabs:
                raise ValueError("one device per slab")
            dev = (ctypes.c_int * nslabs)(*devices)
        st = lib().hype_group_create(ctypes.byref(cfg.c_struct()), nslabs, dev, ctypes.byref(self._h))
        if st != OK:
            msg = lib().hype_group_last_error(self._h).decode() if self._h else lib().hype_status_string(st).decode()
            lib().hype_group_destroy(self._h)
            self._h = ctypes.c_void_p()
            raise HypeError(st, msg)

    def close(self):
        if self._h:
            lib().hype_group_destroy(self._h)
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
            raise HypeError(st, lib().hype_group_last_error(self._h).decode())

    @property
    def n(self) -> int:
        return self.cfg.nx * self.cfg.ny * self.cfg.nvar

    def last_error(self) -> str:
        return lib().hype_group_last_error(self._h).decode()

    def slab(self, k: int):
        """(first global row, rows, device) of slab k."""
        r0, n, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().hype_group_slab(self._h, k, ctypes.byref(r0), ctypes.byref(n), ctypes.byref(d)))
        return r0.value, n.value, d.value

    def set_state(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n:
            raise ValueError("U has the wrong size")
        self._check(lib().hype_group_set_state(self._h, _ptr(U)))

    def get_state(self) -> np.ndarray:
        U = np.empty(self.n, dtype=np.float64)
        self._check(lib().hype_group_get_state(self._h, _ptr(U)))
        return U

    def solve(self, t0: float, t_final: float, max_steps: int, check: bool = True):
        """Returns (steps, t_end, dt_next, status)."""
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = lib().hype_group_solve(self._h, t0, t_final, max_steps, ctypes.byref(steps), ctypes.byref(t), ctypes.byref(dt))
        if check and st not in (OK, ERR_INADMISSIBLE):
            self._check(st)
        return steps.value, t.value, dt.value, st

    def begin(self, t0: float, t_final: float, max_steps: int) -> None:
        self._check(lib().hype_group_begin(self._h, t0, t_final, max_steps))

    def advance(self, nsteps: int) -> None:
        self._check(lib().hype_group_advance(self._h, nsteps))

    def wait(self):
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = lib().hype_group_wait(self._h, ctypes.byref(steps), ctypes.byref(t), ctypes.byref(dt))
        return steps.value, t.value, dt.value, st

    def last_elapsed_ms(self) -> float:
        ms = ctypes.c_double(0.0)
        self._check(lib().hype_group_last_elapsed_ms(self._h, ctypes.byref(ms)))
        return ms.value


class Batch:
    """Many independent instances stepped together (include/hype_batch.h).

    ``add(cfg, U0, t0, t_final, max_steps)`` admits an instance (its own time
    loop, as ``Solver.solve``) and returns its id; ``advance(n)`` enqueues n
    steps of every instance; ``sync()`` waits and refreshes ``status(id)``.
    """

    def __init__(self, max_instances: int = 256, hbm_budget: int = 0, max_cells: int = 2048 * 2048, device: int = 0):
        c = _BatchCfg()
        lib().hype_batch_config_default(ctypes.byref(c))
        c.device, c.max_instances, c.hbm_budget, c.max_cells = device, max_instances, hbm_budget, max_cells
        self._h = ctypes.c_void_p()
        self.cfgs = {}
        st = lib().hype_batch_create(ctypes.byref(c), ctypes.byref(self._h))
        if st != OK:
            msg = lib().hype_batch_last_error(self._h).decode() if self._h else lib().hype_status_string(st).decode()
            lib().hype_batch_destroy(self._h)
            self._h = ctypes.c_void_p()
            raise HypeError(st, msg)

    def close(self):
        if self._h:
            lib().hype_batch_destroy(self._h)
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
            raise HypeError(st, lib().hype_batch_last_error(self._h).decode())

    @staticmethod
    def instance_bytes(cfg: Config) -> int:
        return lib().hype_batch_instance_bytes(ctypes.byref(cfg.c_struct()))

    def try_add(self, cfg: Config, U0: np.ndarray, t0: float, t_final: float, max_steps: int):
        """Returns (status, id); status ERR_NOMEM / ERR_BUSY when admission refuses."""
        U0 = np.ascontiguousarray(U0, dtype=np.float64)
        if U0.size != cfg.nx * cfg.ny * cfg.nvar:
            raise ValueError("U0 has the wrong size")
        i = ctypes.c_int(-1)
        st = lib().hype_batch_add(self._h, ctypes.byref(cfg.c_struct()), _ptr(U0), t0, t_final, max_steps, ctypes.byref(i))
        if st == OK:
            self.cfgs[i.value] = cfg
        return st, i.value

    def add(self, cfg: Config, U0: np.ndarray, t0: float, t_final: float, max_steps: int) -> int:
        st, i = self.try_add(cfg, U0, t0, t_final, max_steps)
        self._check(st)
        return i

    def remove(self, i: int) -> None:
        self._check(lib().hype_batch_remove(self._h, i))
        self.cfgs.pop(i, None)

    def advance(self, nsteps: int) -> None:
        self._check(lib().hype_batch_advance(self._h, nsteps))

    def sync(self) -> None:
        self._check(lib().hype_batch_sync(self._h))

    def status(self, i: int) -> dict:
        s = _InstStatus()
        self._check(lib().hype_batch_status(self._h, i, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _InstStatus._fields_}

    def hold(self, i: int, hold: bool = True) -> None:
        self._check(lib().hype_batch_hold(self._h, i, int(hold)))

    def set_substeps(self, i: int, k: int) -> None:
        self._check(lib().hype_batch_set_substeps(self._h, i, k))

    def get_state(self, i: int) -> np.ndarray:
        c = self.cfgs[i]
        U = np.empty(c.nx * c.ny * c.nvar, dtype=np.float64)
        self._check(lib().hype_batch_get_state(self._h, i, _ptr(U)))
        return U

    def set_tiling(self, cells: int, rows: int) -> None:
        self._check(lib().hype_batch_set_tiling(self._h, cells, rows))

    def autotune(self, reps: int = 3):
        c, r = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().hype_batch_autotune(self._h, reps, ctypes.byref(c), ctypes.byref(r)))
        return c.value, r.value

    def info(self) -> dict:
        n, w = ctypes.c_int(0), ctypes.c_int(0)
        b, g = ctypes.c_size_t(0), ctypes.c_size_t(0)
        self._check(lib().hype_batch_info(self._h, ctypes.byref(n), ctypes.byref(w), ctypes.byref(b), ctypes.byref(g)))
        return {"instances": n.value, "work_items": w.value, "bytes_in_use": b.value, "budget": g.value}

    def last_elapsed_ms(self) -> float:
        ms = ctypes.c_double(0.0)
        self._check(lib().hype_batch_last_elapsed_ms(self._h, ctypes.byref(ms)))
        return ms.value


# include/hype_serve.h
IC_CALLBACK, IC_SHOCK_BUBBLE, IC_BN_DISCS, IC_EULER_QUADRANTS, IC_SMOOTH_VORTEX = range(5)


@dataclasses.dataclass
class Request:
    """One solve: configuration, time interval and step limit, initial state
    (a built-in seeded generator, or IC_CALLBACK with ``fill``)."""
    arrival_s: float
    cfg: Config
    t0: float = 0.0
    t_final: float = 1e30
    max_steps: int = 100
    ic: int = IC_SHOCK_BUBBLE
    ic_seed: int = 0
    ic_param: int = 1


def serve(requests, *, device: int = 0, max_instances: int = 256, hbm_budget: int = 0, max_cells: int = 2048 * 2048,
          poll_ms: float = 10.0, realtime: bool = True, autotune: bool = True, fetch_results: bool = True,
          active_cells: int | None = None, substep_cells: int | None = None, fill=None, sink=None):
    """Runs hype_serve_run over ``requests`` (sorted by arrival).

    fill(index, U0) fills the initial state of IC_CALLBACK requests in place;
    sink(index, U, result) receives each final state (a copy).  Returns
    (results, stats) as lists/dicts of the C structures' fields.
    """
    L = lib()
    n = len(requests)
    arr = (_Request * max(n, 1))()
    for i, r in enumerate(requests):
        arr[i] = _Request(r.arrival_s, r.cfg.c_struct(), r.t0, r.t_final, r.max_steps, r.ic, r.ic_seed, r.ic_param)
    res = (_Result * max(n, 1))()
    st = _ServeStats()
    c = _ServeCfg()
    L.hype_serve_config_default(ctypes.byref(c))
    c.device, c.max_instances, c.hbm_budget, c.max_cells = device, max_instances, hbm_budget, max_cells
    c.poll_ms, c.realtime, c.autotune, c.fetch_results = poll_ms, int(realtime), int(autotune), int(fetch_results)
    if active_cells is not None:
        c.active_cells = active_cells
    if substep_cells is not None:
        c.substep_cells = substep_cells

    def _fill(_ctx, i, _req, U):
        try:
            cfg = requests[i].cfg
            fill(i, np.ctypeslib.as_array(U, shape=(cfg.nx * cfg.ny * cfg.nvar,)))
            return 0
        except Exception:
            return 1

    def _sink(_ctx, i, _req, U, rp):
        cfg = requests[i].cfg
        out = np.ctypeslib.as_array(U, shape=(cfg.nx * cfg.ny * cfg.nvar,)).copy()
        sink(i, out, {f: getattr(rp.contents, f) for f, _ in _Result._fields_})

    fcb = _FILL_FN(_fill) if fill is not None else _FILL_FN()
    scb = _SINK_FN(_sink) if sink is not None else _SINK_FN()
    rc = L.hype_serve_run(ctypes.byref(c), arr, n, fcb, scb, None, res, ctypes.byref(st))
    if rc != OK:
        raise HypeError(rc, f"hype_serve_run: {L.hype_status_string(rc).decode()}")
    results = [{f: getattr(res[i], f) for f, _ in _Result._fields_} for i in range(n)]
    return results, {f: getattr(st, f) for f, _ in _ServeStats._fields_}
