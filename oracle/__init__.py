"""CPU checker for the hype-parallel_b200 kernels.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may use
this package; the product (``hype-parallel_b200/``) never imports it.

Two CPU implementations live here:

* ``Oracle`` -- ``hype_oracle.c``: a C restatement of HyPE-2D's
  ``RHSFunctionPrim`` / ``RHSFunction`` (``HyPE-2D/rhs_function_prim.c:12-626``,
  ``HyPE-2D/rhs_function.c:12-625``) and of the PETSc TSSSP time loop that
  ``HyPE-2D/hype.c:337-384`` sets up.  Built by ``make -C oracle``.
* ``Reference`` -- the reference's own sources compiled unmodified against a
  one-rank PETSc stand-in (``make -C oracle ref``, output in ``oracle/_ref``).
  Used to pin ``Oracle`` bit for bit and to produce tests/golden fixtures.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libhype_oracle.so")
FLOPS_LIB = os.path.join(HERE, "_build", "libhype_oracle_flops.so")   # the oracle with counted operations
REF_LIB = {0: os.path.join(HERE, "_ref", "libhype_ref_euler.so"),
           1: os.path.join(HERE, "_ref", "libhype_ref_kapila.so"),
           2: os.path.join(HERE, "_ref", "libhype_ref_bn.so")}
REF_LIB_VISCOUS = os.path.join(HERE, "_ref", "libhype_ref_kapila_visc.so")   # Kapila built with -DVISCOUS

EULER, KAPILA, BN = 0, 1, 2
NVAR = {EULER: 4, KAPILA: 6, BN: 9}
# HyPE-2D/hype.h:76 enum bndry_type
WALL, INLET, PERIODIC, REFLECTIVE, TRANSMISSIVE = 0, 1, 2, 3, 4
OK, ERR_CONFIG, ERR_INADMISSIBLE = 0, 1, 2


@dataclasses.dataclass
class Config:
    system: int = KAPILA
    order: int = 2
    nx: int = 16
    ny: int = 16
    x_min: float = 0.0
    x_max: float = 1.0
    y_min: float = 0.0
    y_max: float = 1.0
    cfl: float = 0.4
    bc_left: int = TRANSMISSIVE
    bc_right: int = TRANSMISSIVE
    bc_bottom: int = TRANSMISSIVE
    bc_top: int = TRANSMISSIVE
    gamma1: float = 4.4
    gamma2: float = 1.4
    pi1: float = 6.0e8
    pi2: float = 0.0
    bn_fixed_p2: int = 0
    conservative: int = 0
    viscous: int = 0          # the VISCOUS build (Kapila, N >= 1)
    mu1: float = 1.0e-2       # MU_1, MU_2 (hype.h:46-47)
    mu2: float = 0.0

    @property
    def nvar(self) -> int:
        return NVAR[self.system]


class _HyoConfig(ctypes.Structure):
    _fields_ = [("system", ctypes.c_int), ("order", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double), ("y_min", ctypes.c_double),
                ("y_max", ctypes.c_double), ("cfl", ctypes.c_double),
                ("bc_left", ctypes.c_int), ("bc_right", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_top", ctypes.c_int),
                ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("pi1", ctypes.c_double), ("pi2", ctypes.c_double),
                ("bn_fixed_p2", ctypes.c_int), ("conservative", ctypes.c_int), ("viscous", ctypes.c_int),
                ("mu1", ctypes.c_double), ("mu2", ctypes.c_double)]


class _RefConfig(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double), ("y_min", ctypes.c_double),
                ("y_max", ctypes.c_double), ("cfl", ctypes.c_double),
                ("bc_left", ctypes.c_int), ("bc_right", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_top", ctypes.c_int),
                ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("pi1", ctypes.c_double), ("pi2", ctypes.c_double),
                ("mu1", ctypes.c_double), ("mu2", ctypes.c_double)]


_DP = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def build(ref: bool = False) -> None:
    """Compile the checker (and, when the reference sources are present, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def reference_available() -> bool:
    return all(os.path.exists(p) for p in REF_LIB.values())


def viscous_reference_available() -> bool:
    return os.path.exists(REF_LIB_VISCOUS)


FLOP_KINDS = ("add", "mul", "div", "sqrt", "cmp", "abs", "neg", "trans")


def count_rhs_ops(cfg: Config, U: np.ndarray):
    """The floating-point operations of one oracle RHS evaluation (oracle/flops.cpp):
    returns (RHS, status, {kind: count}); "flops" = add + mul + div + sqrt."""
    if not os.path.exists(FLOPS_LIB):
        subprocess.run(["make", "-s", "-C", HERE, "flops"], check=True)
    lib = ctypes.CDLL(FLOPS_LIB, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    lib.hyo_rhs.argtypes = [ctypes.POINTER(_HyoConfig), ctypes.c_double, _DP, _DP, _DP]
    lib.hyo_flops_read.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    U = np.ascontiguousarray(U, dtype=np.float64)
    R = np.empty_like(U)
    dt = ctypes.c_double(0.0)
    lib.hyo_flops_reset()
    st = lib.hyo_rhs(ctypes.byref(Oracle._cfg(cfg)), 0.0, _ptr(U), _ptr(R), ctypes.byref(dt))
    out = (ctypes.c_ulonglong * 8)()
    lib.hyo_flops_read(out)
    counts = dict(zip(FLOP_KINDS, [int(v) for v in out]))
    counts["flops"] = counts["add"] + counts["mul"] + counts["div"] + counts["sqrt"]
    return R, st, counts


class Oracle:
    """ctypes view of hype_oracle.c."""

    def __init__(self):
        if not os.path.exists(ORACLE_LIB):
            build()
        self.lib = ctypes.CDLL(ORACLE_LIB)
        self.lib.hyo_rhs.argtypes = [ctypes.POINTER(_HyoConfig), ctypes.c_double, _DP, _DP, _DP]
        self.lib.hyo_solve.argtypes = [ctypes.POINTER(_HyoConfig), _DP, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), _DP, _DP]
        self.lib.hyo_last_pad_fallbacks.restype = ctypes.c_long

    @staticmethod
    def _cfg(cfg: Config) -> _HyoConfig:
        return _HyoConfig(**dataclasses.asdict(cfg))

    def rhs(self, cfg: Config, U: np.ndarray, t: float = 0.0):
        """RHSFunctionPrim (or RHSFunction when cfg.conservative): returns (RHS, dt, status)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty_like(U)
        dt = ctypes.c_double(0.0)
        st = self.lib.hyo_rhs(ctypes.byref(self._cfg(cfg)), t, _ptr(U), _ptr(R), ctypes.byref(dt))
        return R, dt.value, st

    def pad_fallbacks(self) -> int:
        return int(self.lib.hyo_last_pad_fallbacks())

    def solve(self, cfg: Config, U: np.ndarray, t0: float, t_final: float, max_steps: int):
        """hype.c time loop: returns (U_end, steps, t_end, dt_next, status)."""
        U = np.array(U, dtype=np.float64, order="C", copy=True)
        steps = ctypes.c_int(0)
        tt = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = self.lib.hyo_solve(ctypes.byref(self._cfg(cfg)), _ptr(U), t0, t_final, max_steps,
                                ctypes.byref(steps), ctypes.byref(tt), ctypes.byref(dt))
        return U, steps.value, tt.value, dt.value, st


class Reference:
    """The reference's own RHSFunctionPrim/RHSFunction and time loop (oracle/_ref)."""

    def __init__(self, system: int, viscous: bool = False):
        if viscous and system != KAPILA:
            raise ValueError("the reference has a viscous flux for the Kapila system only")
        path = REF_LIB_VISCOUS if viscous else REF_LIB[system]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.system = system
        self.viscous = bool(viscous)
        self.lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        self.lib.ref_setup.argtypes = [ctypes.POINTER(_RefConfig)]
        self.lib.ref_rhs.argtypes = [ctypes.c_double, _DP, _DP, _DP, ctypes.c_int]
        self.lib.ref_solve.argtypes = [_DP, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), _DP, _DP]
        self._cfg = None

    def setup(self, cfg: Config) -> None:
        if cfg.system != self.system:
            raise ValueError("reference library built for another system")
        if cfg.bn_fixed_p2:
            raise ValueError("the reference has only the shipped Baer-Nunziato flux")
        if bool(cfg.viscous) != self.viscous:
            raise ValueError("viscous configurations need the VISCOUS build and vice versa")
        rc = _RefConfig(N=cfg.order, nx=cfg.nx, ny=cfg.ny, x_min=cfg.x_min, x_max=cfg.x_max, y_min=cfg.y_min,
                        y_max=cfg.y_max, cfl=cfg.cfl, bc_left=cfg.bc_left, bc_right=cfg.bc_right,
                        bc_bottom=cfg.bc_bottom, bc_top=cfg.bc_top, gamma1=cfg.gamma1, gamma2=cfg.gamma2,
                        pi1=cfg.pi1, pi2=cfg.pi2, mu1=cfg.mu1, mu2=cfg.mu2)
        self.lib.ref_setup(ctypes.byref(rc))
        self._cfg = cfg

    def rhs(self, U: np.ndarray, t: float = 0.0):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty_like(U)
        dt = ctypes.c_double(0.0)
        st = self.lib.ref_rhs(t, _ptr(U), _ptr(R), ctypes.byref(dt), 0 if self._cfg.conservative else 1)
        return R, dt.value, st

    def solve(self, U: np.ndarray, t0: float, t_final: float, max_steps: int):
        U = np.array(U, dtype=np.float64, order="C", copy=True)
        steps = ctypes.c_int(0)
        tt = ctypes.c_double(0.0)
        dt = ctypes.c_double(0.0)
        st = self.lib.ref_solve(_ptr(U), t0, t_final, max_steps, 0 if self._cfg.conservative else 1,
                                ctypes.byref(steps), ctypes.byref(tt), ctypes.byref(dt))
        return U, steps.value, tt.value, dt.value, st
