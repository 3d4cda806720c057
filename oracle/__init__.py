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
* ``LiveReference`` -- the same sources run as several live MPI ranks (one
  process each, the stand-in's shared-memory MPI), on the DMDA split that
  ``HyPE-2D/hype.c:108-122`` asks PETSc for: what ``mpiexec -n R`` runs.
* ``initial_state`` -- the seeded workload states (``hype_oracle_ic.c``), so the
  CPU legs never load the product's library.
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


_IC_KINDS = {"shock_bubble": KAPILA, "bn_discs": BN, "euler_quadrants": EULER}


def initial_state(cfg: Config, kind: str, seed: int = 0, nbubbles: int = 1) -> np.ndarray:
    """Seeded initial state (Vec layout, nx*ny*nvar doubles) of one of the
    benchmark workloads, from the oracle's own generator: "shock_bubble"
    (Kapila), "bn_discs" (Baer-Nunziato) or "euler_quadrants" (Euler)."""
    if _IC_KINDS.get(kind) != cfg.system:
        raise ValueError(f"initial state {kind!r} does not fit system {cfg.system}")
    if not os.path.exists(ORACLE_LIB):
        build()
    lib = ctypes.CDLL(ORACLE_LIB)
    U = np.empty(cfg.nx * cfg.ny * cfg.nvar, dtype=np.float64)
    c = Oracle._cfg(cfg)
    if kind == "shock_bubble":
        lib.hyo_ic_shock_bubble.argtypes = [ctypes.POINTER(_HyoConfig), ctypes.c_uint64, ctypes.c_int, _DP]
        st = lib.hyo_ic_shock_bubble(ctypes.byref(c), seed, nbubbles, _ptr(U))
    elif kind == "bn_discs":
        lib.hyo_ic_bn_discs.argtypes = [ctypes.POINTER(_HyoConfig), ctypes.c_uint64, _DP]
        st = lib.hyo_ic_bn_discs(ctypes.byref(c), seed, _ptr(U))
    else:
        lib.hyo_ic_euler_quadrants.argtypes = [ctypes.POINTER(_HyoConfig), ctypes.c_uint64, _DP]
        st = lib.hyo_ic_euler_quadrants(ctypes.byref(c), seed, _ptr(U))
    if st != OK:
        raise ValueError(f"initial state {kind!r}: status {st}")
    return U


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

    def begin(self, U: np.ndarray, t0: float, t_final: float) -> int:
        """The time loop of solve() in chunks: loads U and seeds dt (hype.c:343)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.lib.ref_begin.argtypes = [_DP, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        return self.lib.ref_begin(_ptr(U), t0, t_final, 0 if self._cfg.conservative else 1)

    def advance(self, nsteps: int):
        """Up to nsteps more steps of the loop begin() set up: (steps, t, dt_next, status)."""
        self.lib.ref_advance.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, _DP]
        n, tt, dt = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_double(0.0)
        st = self.lib.ref_advance(nsteps, ctypes.byref(n), ctypes.byref(tt), ctypes.byref(dt))
        return n.value, tt.value, dt.value, st

    def set_output(self, write_interval: int, restart_interval: int) -> None:
        """The output schedule of the reference's MonitorFunction (post_process.c:12-64),
        written in the current directory during solve(); 0 turns a kind off."""
        self.lib.ref_set_output.argtypes = [ctypes.c_int, ctypes.c_int]
        self.lib.ref_set_output(write_interval, restart_interval)

    def write_final(self, steps: int) -> int:
        """hype.c:389-400: sol-<steps>.vts of the state the last solve() left, in the
        current directory."""
        self.lib.ref_write_final.argtypes = [ctypes.c_int]
        return self.lib.ref_write_final(steps)

    def load_restart(self):
        """hype.c:316-325: (state, status) read by VecLoad from restart1.bin in the
        current directory."""
        self.lib.ref_load_restart.argtypes = [_DP]
        U = np.empty(self._cfg.nx * self._cfg.ny * self._cfg.nvar, dtype=np.float64)
        return U, self.lib.ref_load_restart(_ptr(U))

    def state(self) -> np.ndarray:
        """The state of the loop begin() set up (Vec layout)."""
        self.lib.ref_get_state.argtypes = [_DP]
        U = np.empty(self._cfg.nx * self._cfg.ny * self._cfg.nvar, dtype=np.float64)
        self.lib.ref_get_state(_ptr(U))
        return U


# ---------------------------------------------------------------------------
# the reference as live MPI ranks
# ---------------------------------------------------------------------------
def _ref_cfg(cfg: Config) -> _RefConfig:
    return _RefConfig(N=cfg.order, nx=cfg.nx, ny=cfg.ny, x_min=cfg.x_min, x_max=cfg.x_max, y_min=cfg.y_min,
                      y_max=cfg.y_max, cfl=cfg.cfl, bc_left=cfg.bc_left, bc_right=cfg.bc_right,
                      bc_bottom=cfg.bc_bottom, bc_top=cfg.bc_top, gamma1=cfg.gamma1, gamma2=cfg.gamma2,
                      pi1=cfg.pi1, pi2=cfg.pi2, mu1=cfg.mu1, mu2=cfg.mu2)


def _live_rank_main(rank, size, px, py, cfg, seg_name, grid_name, wait_s, conn):
    """One MPI rank: joins the shared segment, sets the reference up on its block
    of the DMDA, then serves the parent's commands until "close"."""
    import time as _time
    from multiprocessing import shared_memory
    seg = shared_memory.SharedMemory(name=seg_name)
    grid = shared_memory.SharedMemory(name=grid_name)
    nv = cfg.nvar
    G = np.ndarray((cfg.ny, cfg.nx, nv), dtype=np.float64, buffer=grid.buf)
    seg_arr = np.ndarray((seg.size,), dtype=np.uint8, buffer=seg.buf)
    path = REF_LIB_VISCOUS if cfg.viscous else REF_LIB[cfg.system]
    lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    lib.ref_live_join.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
    lib.ref_live_set_wait.argtypes = [ctypes.c_double]
    lib.ref_setup.argtypes = [ctypes.POINTER(_RefConfig)]
    lib.ref_rhs.argtypes = [ctypes.c_double, _DP, _DP, _DP, ctypes.c_int]
    lib.ref_begin.argtypes = [_DP, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.ref_advance.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, _DP]
    lib.ref_get_state.argtypes = [_DP]
    lib.ref_corners.argtypes = [ctypes.POINTER(ctypes.c_int)] * 4
    prim = 0 if cfg.conservative else 1
    try:
        if lib.ref_live_join(rank, size, px, py, ctypes.c_void_p(seg_arr.ctypes.data), cfg.nx * cfg.ny * nv) != 0:
            raise RuntimeError("ref_live_join refused the rank layout")
        lib.ref_live_set_wait(wait_s)
        lib.ref_setup(ctypes.byref(_ref_cfg(cfg)))
        c4 = [ctypes.c_int(0) for _ in range(4)]
        lib.ref_corners(*[ctypes.byref(x) for x in c4])
        xs, ys, xm, ym = (x.value for x in c4)
        conn.send(("ready", (xs, ys, xm, ym)))
        B = np.empty((ym, xm, nv), dtype=np.float64)
        while True:
            cmd, arg = conn.recv()
            if cmd == "close":
                break
            t0 = _time.perf_counter()
            if cmd == "rhs":
                B[...] = G[ys:ys + ym, xs:xs + xm]
                R = np.empty_like(B)
                dt = ctypes.c_double(0.0)
                st = lib.ref_rhs(arg, _ptr(B), _ptr(R), ctypes.byref(dt), prim)
                if st == 0:
                    G[ys:ys + ym, xs:xs + xm] = R   # the parent read the input before asking
                conn.send((st, 0, 0.0, dt.value, _time.perf_counter() - t0))
            elif cmd == "begin":
                B[...] = G[ys:ys + ym, xs:xs + xm]
                st = lib.ref_begin(_ptr(B), arg[0], arg[1], prim)
                conn.send((st, 0, arg[0], 0.0, _time.perf_counter() - t0))
            elif cmd == "advance":
                n, tt, dt = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_double(0.0)
                st = lib.ref_advance(arg, ctypes.byref(n), ctypes.byref(tt), ctypes.byref(dt))
                conn.send((st, n.value, tt.value, dt.value, _time.perf_counter() - t0))
            elif cmd == "state":
                lib.ref_get_state(_ptr(B))
                G[ys:ys + ym, xs:xs + xm] = B
                conn.send((0, 0, 0.0, 0.0, _time.perf_counter() - t0))
    finally:
        del G, seg_arr
        seg.close()
        grid.close()


class LiveReference:
    """The reference's RHSFunctionPrim / RHSFunction and hype.c time loop run as
    `nranks` live MPI ranks, one process each (oracle/_ref on the stand-in's
    shared-memory MPI): the DMDA is split over a px x py process grid (0, 0: the
    PETSC_DECIDE split of HyPE-2D/hype.c:108-122), every RHS call exchanges the
    ghost strips of its neighbours (rhs_function_prim.c:44-45) and reduces dt
    with MPI_Allreduce(MIN) (rhs_function_prim.c:620-623) across the processes.
    States in and out are whole grids (Vec layout); each rank copies its block.
    A rank that aborts (MPI_Abort) ends the collective calls of all of them; the
    group is then spent."""

    def __init__(self, cfg: Config, nranks: int, px: int = 0, py: int = 0, wait_s: float = 600.0):
        import multiprocessing as mp
        from multiprocessing import shared_memory
        if cfg.bn_fixed_p2:
            raise ValueError("the reference has only the shipped Baer-Nunziato flux")
        path = REF_LIB_VISCOUS if cfg.viscous else REF_LIB[cfg.system]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.cfg = cfg
        self.nranks = nranks
        grid_doubles = cfg.nx * cfg.ny * cfg.nvar
        probe = ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        probe.ref_live_bytes.restype = ctypes.c_size_t
        probe.ref_live_bytes.argtypes = [ctypes.c_longlong]
        self._grid = None
        self._seg = shared_memory.SharedMemory(create=True, size=int(probe.ref_live_bytes(grid_doubles)))
        self._grid = shared_memory.SharedMemory(create=True, size=grid_doubles * 8)
        self.G = np.ndarray((cfg.ny, cfg.nx, cfg.nvar), dtype=np.float64, buffer=self._grid.buf)
        ctx = mp.get_context("spawn")
        self._procs, self._conns, self.blocks = [], [], []
        try:
            for r in range(nranks):
                a, b = ctx.Pipe()
                p = ctx.Process(target=_live_rank_main,
                                args=(r, nranks, px, py, cfg, self._seg.name, self._grid.name, wait_s, b), daemon=True)
                p.start()
                self._procs.append(p)
                self._conns.append(a)
            for k in range(nranks):
                tag, blk = self._recv(k)
                self.blocks.append(blk)
        except BaseException:
            self.close()
            raise

    def _recv(self, k):
        """Rank k's answer; a rank process that ended without one is an error."""
        c, p = self._conns[k], self._procs[k]
        while not c.poll(1.0):
            if not p.is_alive():
                raise RuntimeError(f"reference rank {k} ended (exit code {p.exitcode})")
        return c.recv()

    def _all(self, cmd, arg=None):
        for c in self._conns:
            c.send((cmd, arg))
        return [self._recv(k) for k in range(len(self._conns))]

    @staticmethod
    def _merge(res):
        st = next((r[0] for r in res if r[0] != 0), 0)
        return st, res[0][1], res[0][2], res[0][3], max(r[4] for r in res)

    def rhs(self, U: np.ndarray, t: float = 0.0):
        """One RHS call on every rank: returns (RHS, dt, status)."""
        self.G[...] = np.asarray(U, dtype=np.float64).reshape(self.G.shape)
        st, _, _, dt, _ = self._merge(self._all("rhs", t))
        return self.G.reshape(-1).copy(), dt, st

    def begin(self, U: np.ndarray, t0: float, t_final: float) -> int:
        """Loads U and seeds dt with one RHS call (hype.c:343)."""
        self.G[...] = np.asarray(U, dtype=np.float64).reshape(self.G.shape)
        return self._merge(self._all("begin", (t0, t_final)))[0]

    def advance(self, nsteps: int):
        """Up to nsteps more steps: returns (steps, t, dt_next, status, seconds of the slowest rank)."""
        st, n, t, dt, sec = self._merge(self._all("advance", nsteps))
        return n, t, dt, st, sec

    def state(self) -> np.ndarray:
        self._all("state")
        return self.G.reshape(-1).copy()

    def solve(self, U: np.ndarray, t0: float, t_final: float, max_steps: int):
        """hype.c time loop: returns (U_end, steps, t_end, dt_next, status)."""
        st = self.begin(U, t0, t_final)
        if st != 0:
            return None, 0, t0, 0.0, st
        n, t, dt, st, _ = self.advance(max_steps)
        return (self.state() if st == 0 else None), n, t, dt, st

    def close(self) -> None:
        if self._grid is None:
            return
        for c in self._conns:
            try:
                c.send(("close", None))
            except (BrokenPipeError, OSError):
                pass
        for p in self._procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
        self._conns, self._procs = [], []
        del self.G
        self._grid.close()
        self._grid.unlink()
        self._seg.close()
        self._seg.unlink()
        self._grid = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
