"""TEST INFRASTRUCTURE: the product's PETSc glue (petsc_glue.c, built by
tests/glue/Makefile against the PETSc stand-in) run as live MPI ranks, one
process per rank, over the stand-in's shared-memory MPI -- the way HyPE-2D runs
under mpiexec: a DMDA split over a px x py process grid (0, 0: PETSc's
PETSC_DECIDE split, hype.c:108-122), ghost strips exchanged by DMGlobalToLocal
and dt reduced with MPI_Allreduce(MIN) by the glue.  Every rank drives its own
GPU solver (hype_create_block) on the same device.  States in and out are whole
grids in the Vec layout; each rank reads and writes its own block.
"""
import ctypes
import os

import numpy as np

GLUE_BUILD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "glue", "_build")
_DP = ctypes.POINTER(ctypes.c_double)


def _lib(name):
    L = ctypes.CDLL(os.path.join(GLUE_BUILD, f"libglue_{name}.so"), mode=os.RTLD_LOCAL | os.RTLD_NOW)
    L.glue_live_bytes.restype = ctypes.c_size_t
    L.glue_live_bytes.argtypes = [ctypes.c_longlong]
    L.glue_live_join.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
    L.glue_live_set_wait.argtypes = [ctypes.c_double]
    L.glue_corners.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 4
    L.glue_rhs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP, ctypes.c_double, ctypes.POINTER(ctypes.c_int), _DP,
                           ctypes.c_int, _DP, _DP, _DP]
    L.glue_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP, ctypes.c_double, ctypes.POINTER(ctypes.c_int), _DP,
                             ctypes.c_int, _DP, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                             _DP, _DP]
    return L


def _args(c):
    dom = (ctypes.c_double * 4)(c["x_min"], c["x_max"], c["y_min"], c["y_max"])
    bc = (ctypes.c_int * 4)(c["bc_left"], c["bc_right"], c["bc_bottom"], c["bc_top"])
    eos = (ctypes.c_double * 4)(c["gamma1"], c["gamma2"], c["pi1"], c["pi2"])
    return dom, bc, eos


def _rank_main(rank, size, px, py, lib_name, c, seg_name, gin_name, gout_name, wait_s, conn):
    from multiprocessing import shared_memory
    seg = shared_memory.SharedMemory(name=seg_name)
    gin = shared_memory.SharedMemory(name=gin_name)
    gout = shared_memory.SharedMemory(name=gout_name)
    n = c["nx"] * c["ny"] * c["nvar"]
    Gin = np.ndarray((n,), dtype=np.float64, buffer=gin.buf)
    Gout = np.ndarray((n,), dtype=np.float64, buffer=gout.buf)
    segb = np.ndarray((seg.size,), dtype=np.uint8, buffer=seg.buf)
    try:
        L = _lib(lib_name)
        if "mu1" in c:
            L.glue_set_mu.argtypes = [ctypes.c_double, ctypes.c_double]
            L.glue_set_mu(c["mu1"], c["mu2"])
        if L.glue_live_join(rank, size, px, py, ctypes.c_void_p(segb.ctypes.data), n) != 0:
            raise RuntimeError("glue_live_join refused the rank layout")
        L.glue_live_set_wait(wait_s)
        q = [ctypes.c_int(0) for _ in range(4)]
        L.glue_corners(c["nx"], c["ny"], *[ctypes.byref(x) for x in q])
        conn.send(("ready", tuple(x.value for x in q)))
        dom, bc, eos = _args(c)
        while True:
            cmd, arg = conn.recv()
            if cmd == "close":
                break
            if cmd == "rhs":
                dt = ctypes.c_double(0.0)
                st = L.glue_rhs(c["order"], c["nx"], c["ny"], dom, c["cfl"], bc, eos, c["conservative"],
                                Gin.ctypes.data_as(_DP), Gout.ctypes.data_as(_DP), ctypes.byref(dt))
                conn.send((st, 0, 0.0, dt.value))
            elif cmd == "solve":
                t0, tf, nmax = arg
                k, te, dtn = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_double(0.0)
                st = L.glue_solve(c["order"], c["nx"], c["ny"], dom, c["cfl"], bc, eos, c["conservative"],
                                  Gin.ctypes.data_as(_DP), t0, tf, nmax, ctypes.byref(k), ctypes.byref(te), ctypes.byref(dtn))
                conn.send((st, k.value, te.value, dtn.value))
        L.glue_finalize()
    finally:
        del Gin, Gout, segb
        seg.close()
        gin.close()
        gout.close()


class LiveGlue:
    """`nranks` processes, each one MPI rank running the glue's RHSFunctionPrim /
    RHSFunction (and a hype.c-style TSSolve around it) on its block of the DMDA.
    cfg: an oracle.Config; lib_name: the glue library ("kapila", "bn", "euler",
    "kapila_visc")."""

    def __init__(self, cfg, lib_name, nranks, px=0, py=0, wait_s=120.0):
        import multiprocessing as mp
        from multiprocessing import shared_memory
        n = cfg.nx * cfg.ny * cfg.nvar
        self.n = n
        self._c = dict(nx=cfg.nx, ny=cfg.ny, nvar=cfg.nvar, order=cfg.order, cfl=cfg.cfl, conservative=int(cfg.conservative),
                       x_min=cfg.x_min, x_max=cfg.x_max, y_min=cfg.y_min, y_max=cfg.y_max, bc_left=cfg.bc_left,
                       bc_right=cfg.bc_right, bc_bottom=cfg.bc_bottom, bc_top=cfg.bc_top, gamma1=cfg.gamma1,
                       gamma2=cfg.gamma2, pi1=cfg.pi1, pi2=cfg.pi2)
        if cfg.viscous:
            self._c.update(mu1=cfg.mu1, mu2=cfg.mu2)
        probe = _lib(lib_name)
        self._seg = shared_memory.SharedMemory(create=True, size=int(probe.glue_live_bytes(n)))
        self._gin = shared_memory.SharedMemory(create=True, size=n * 8)
        self._gout = shared_memory.SharedMemory(create=True, size=n * 8)
        self.Gin = np.ndarray((n,), dtype=np.float64, buffer=self._gin.buf)
        self.Gout = np.ndarray((n,), dtype=np.float64, buffer=self._gout.buf)
        ctx = mp.get_context("spawn")
        self._procs, self._conns, self.blocks = [], [], []
        try:
            for r in range(nranks):
                a, b = ctx.Pipe()
                p = ctx.Process(target=_rank_main, args=(r, nranks, px, py, lib_name, self._c, self._seg.name, self._gin.name,
                                                         self._gout.name, wait_s, b), daemon=True)
                p.start()
                self._procs.append(p)
                self._conns.append(a)
            for k in range(nranks):
                self.blocks.append(self._recv(k)[1])
        except BaseException:
            self.close()
            raise

    def _recv(self, k):
        c, p = self._conns[k], self._procs[k]
        while not c.poll(1.0):
            if not p.is_alive():
                raise RuntimeError(f"glue rank {k} ended (exit code {p.exitcode})")
        try:
            return c.recv()
        except EOFError:
            p.join(timeout=10)
            raise RuntimeError(f"glue rank {k} ended (exit code {p.exitcode})") from None

    def _all(self, cmd, arg=None):
        for c in self._conns:
            c.send((cmd, arg))
        res = [self._recv(k) for k in range(len(self._conns))]
        st = next((r[0] for r in res if r[0] != 0), 0)
        return st, res

    def rhs(self, U):
        """RHSFunctionPrim on every rank: (RHS, [dt of each rank], status)."""
        self.Gin[...] = np.asarray(U, dtype=np.float64).reshape(-1)
        self.Gout[...] = np.nan
        st, res = self._all("rhs")
        return self.Gout.copy(), [r[3] for r in res], st

    def solve(self, U, t0, t_final, max_steps):
        """hype.c's time loop with the glue's RHS: (U_end, steps, t_end, dt_next, status)."""
        self.Gin[...] = np.asarray(U, dtype=np.float64).reshape(-1)
        st, res = self._all("solve", (t0, t_final, max_steps))
        return self.Gin.copy(), res[0][1], res[0][2], res[0][3], st

    def close(self):
        if getattr(self, "_seg", None) is None:
            return
        for c in self._conns:
            try:
                c.send(("close", None))
            except (BrokenPipeError, OSError):
                pass
        for p in self._procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
        del self.Gin, self.Gout
        for m in (self._gin, self._gout, self._seg):
            m.close()
            m.unlink()
        self._seg = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
