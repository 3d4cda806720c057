"""The PETSc-signature drop-in (hype-parallel_b200/csrc/petsc_glue.c).

The glue is compiled the way a HyPE-2D tree would compile it (hype.h's
AppCtx and system #define, PETSc from the one-rank stand-in of
oracle/petsc_mini) and called as hype.c calls RHSFunctionPrim.  On a GPU its
RHS and Ctx->dt must equal the reference's bit for bit; without one it must
return an error code instead of ending the process.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import cases
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GLUE = os.path.join(ROOT, "tests", "glue")
# (system, viscous) -> library; "kapila_visc" is the glue compiled with VISCOUS defined
LIBNAME = {(O.EULER, 0): "euler", (O.KAPILA, 0): "kapila", (O.BN, 0): "bn", (O.KAPILA, 1): "kapila_visc"}


@pytest.fixture(scope="module")
def glue_libs(hp):
    subprocess.run(["make", "-s", "-C", GLUE], check=True, capture_output=True)
    libs = {}
    for key, nm in LIBNAME.items():
        L = ctypes.CDLL(os.path.join(GLUE, "_build", f"libglue_{nm}.so"))
        DP = ctypes.POINTER(ctypes.c_double)
        IP = ctypes.POINTER(ctypes.c_int)
        L.glue_rhs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, DP, ctypes.c_double, IP, DP, ctypes.c_int, DP, DP, DP]
        L.glue_rhs.restype = ctypes.c_int
        if key[1]:
            L.glue_set_mu.argtypes = [ctypes.c_double, ctypes.c_double]
        libs[key] = L
    return libs


def glue_rhs(L, cfg, U):
    dom = (ctypes.c_double * 4)(cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max)
    bc = (ctypes.c_int * 4)(cfg.bc_left, cfg.bc_right, cfg.bc_bottom, cfg.bc_top)
    eos = (ctypes.c_double * 4)(cfg.gamma1, cfg.gamma2, cfg.pi1, cfg.pi2)
    if cfg.viscous:
        L.glue_set_mu(cfg.mu1, cfg.mu2)
    R = np.empty_like(U)
    dt = ctypes.c_double(0.0)
    DP = ctypes.POINTER(ctypes.c_double)
    st = L.glue_rhs(cfg.order, cfg.nx, cfg.ny, dom, cfg.cfl, bc, eos, cfg.conservative, U.ctypes.data_as(DP),
                    R.ctypes.data_as(DP), ctypes.byref(dt))
    return R, dt.value, st


def test_glue_builds_and_exports_the_reference_signature(glue_libs):
    for L in glue_libs.values():
        assert L.RHSFunctionPrim is not None and L.RHSFunction is not None and L.RHSFunctionPrimFinalize is not None


def test_glue_without_gpu_returns_an_error(hp, glue_libs):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = O.Config(system=O.KAPILA, order=2, nx=8, ny=8, **cases.KAPILA_EOS)
    R, dt, st = glue_rhs(glue_libs[(O.KAPILA, 0)], cfg, cases.state(cfg, "bubble", 1))
    assert st == hp.ERR_NO_DEVICE


GLUE_CASES = ["kapila_37x23_rough_mixed_bc", "kapila_18x14_inlet", "kapila_15x13_N3", "euler_21x19_reflective_N1",
              "bn_16x16", "bn_13x21_periodic_N1",
              # RHSFunction (Ctx.ReconsPrimitive false)
              "kapila_cons_37x23_rough", "kapila_cons_18x14_inlet", "euler_cons_17x12_periodic_N3", "bn_cons_12x10_N3",
              # a tree built with VISCOUS: MU_1, MU_2 from the globals
              "kapila_visc_37x23_rough", "kapila_visc_15x13_N3", "kapila_visc_cons_24x20_walls"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", GLUE_CASES)
def test_glue_rhs_bitwise_vs_oracle(name, hp, orc, glue_libs):
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    Ro, dto, sto = orc.rhs(cfg, U)
    assert sto == O.OK
    R, dt, st = glue_rhs(glue_libs[(cfg.system, int(cfg.viscous))], cfg, U)
    assert st == 0
    assert dt == dto
    assert R.tobytes() == Ro.tobytes()


def split_rows(ny, n):
    """PETSc's split of ny rows over n ranks: the first ny % n get one more."""
    rows = [ny // n + (1 if r < ny % n else 0) for r in range(n)]
    return [(sum(rows[:r]), rows[r]) for r in range(n)]


RANK_CASES = [("kapila_37x23_rough_mixed_bc", 3), ("kapila_24x24_periodic", 4), ("kapila_18x14_inlet", 2),
              ("kapila_15x13_N3", 2), ("bn_13x21_periodic_N1", 3), ("euler_21x19_reflective_N1", 3),
              ("kapila_cons_37x23_rough", 3), ("kapila_visc_37x23_rough", 3)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,nranks", RANK_CASES)
def test_glue_ranks_bitwise_vs_oracle(name, nranks, hp, orc, glue_libs):
    """The glue on a DMDA split in y over several ranks (petsc_mini emulates one rank
    at a time): each rank's RHS rows equal the reference's bit for bit, and the
    minimum of the ranks' dt (the glue's MPI_Allreduce) is the reference's dt."""
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    Ro, dto, sto = orc.rhs(cfg, U)
    assert sto == O.OK
    L = glue_libs[(cfg.system, int(cfg.viscous))]
    L.glue_emulate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    row = cfg.nx * cfg.nvar
    R = np.full_like(U, np.nan)
    dts = []
    try:
        for r, (ys, ym) in enumerate(split_rows(cfg.ny, nranks)):
            L.glue_emulate(r, nranks, ys, ym, U.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            Rr, dt, st = glue_rhs(L, cfg, U)
            assert st == 0, (r, st)
            R[ys * row:(ys + ym) * row] = Rr[ys * row:(ys + ym) * row]
            dts.append(dt)
    finally:
        L.glue_emulate(0, 1, 0, -1, None)
    assert R.tobytes() == Ro.tobytes()
    if cfg.viscous:
        # rhs_function_prim.c:617-623: each rank's dt has its own s_max and s_max_v, so
        # the minimum over ranks can exceed the one-rank dt
        assert min(dts) >= dto
    else:
        assert min(dts) == dto


# (case, ranks, px, py): px = py = 0 is PETSc's own PETSC_DECIDE split (hype.c:108-122)
LIVE_CASES = [("kapila_37x23_rough_mixed_bc", 4, 0, 0), ("kapila_24x24_periodic", 6, 3, 2), ("kapila_18x14_inlet", 3, 3, 1),
              ("kapila_15x13_N3", 4, 2, 2), ("bn_13x21_periodic_N1", 4, 2, 2), ("euler_21x19_reflective_N1", 6, 3, 2),
              ("kapila_cons_37x23_rough", 4, 2, 2), ("kapila_visc_37x23_rough", 4, 0, 0)]
LIVE_SOLVES = [("kapila_32x32_bubble_solve", 4, 0, 0), ("kapila_24x20_bubble_solve_N1", 6, 3, 2),
               ("kapila_16x16_solve_N3", 4, 2, 2), ("euler_32x24_solve", 6, 0, 0), ("bn_20x20_solve", 4, 4, 1),
               ("kapila_cons_32x32_solve", 4, 2, 2), ("kapila_visc_32x32_solve", 4, 0, 0)]


def _live_glue_setup():
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    subprocess.run(["make", "-s", "-C", GLUE], check=True, capture_output=True)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nranks,px,py", LIVE_CASES)
def test_glue_live_ranks_rhs_bitwise_vs_reference_ranks(name, nranks, px, py, hp):
    """The glue as live MPI ranks (one process each, all on one GPU) on a DMDA split
    in x and y -- each rank's GPU solver a block with 3 ghost rows and columns,
    corners included, from DMGlobalToLocal, dt reduced with MPI_Allreduce(MIN) --
    against the reference's RHSFunctionPrim / RHSFunction run as the same ranks
    (oracle.LiveReference): RHS and dt bit for bit."""
    import glue_live
    _live_glue_setup()
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    with O.LiveReference(cfg, nranks, px, py, wait_s=120.0) as ref:
        Rr, dtr, sr = ref.rhs(U)
        blocks = sorted(ref.blocks)
    assert sr == 0
    with glue_live.LiveGlue(cfg, LIBNAME[(cfg.system, int(cfg.viscous))], nranks, px, py) as g:
        assert sorted(g.blocks) == blocks
        if px > 1:
            assert all(b[2] < cfg.nx for b in blocks)   # the grid is split in x
        R, dts, st = g.rhs(U)
    assert st == 0
    assert all(d == dtr for d in dts)
    assert R.tobytes() == Rr.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("name,nranks,px,py", LIVE_SOLVES)
def test_glue_live_ranks_time_loop_bitwise_vs_reference_ranks(name, nranks, px, py, hp):
    """hype.c's time loop (hype.c:337-384: a direct RHS call seeds Ctx->dt, TSSolve
    with dt reset from Ctx->dt every step, post_process.c:19) with the glue's RHS on
    live ranks over a DMDA split in x and y, against the reference's loop on the
    same ranks: steps, final time, next dt and state bit for bit."""
    import glue_live
    _live_glue_setup()
    (_, cfg, kind, seed), t0, tf, nmax = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    with O.LiveReference(cfg, nranks, px, py, wait_s=120.0) as ref:
        Ur, nr, tr, dtnr, sr = ref.solve(U, t0, tf, nmax)
    assert sr == 0 and nr > 0
    with glue_live.LiveGlue(cfg, LIBNAME[(cfg.system, int(cfg.viscous))], nranks, px, py) as g:
        Ug, ng, tg, dtng, sg = g.solve(U, t0, tf, nmax)
    assert sg == 0 and (ng, tg, dtng) == (nr, tr, dtnr)
    assert Ug.tobytes() == Ur.tobytes()


def test_glue_live_ranks_without_gpu_all_return_the_error(hp, glue_libs):
    """Without a GPU every rank's solver fails to be created; the glue's reduction
    of the status (MPI_Allreduce(MAX)) makes every rank of a 2 x 2 DMDA return
    the error, RHS and time loop alike, instead of one rank aborting the job."""
    import torch
    import glue_live
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    _, cfg, kind, seed = cases.case_by_name("kapila_24x24_periodic")
    U = cases.state(cfg, kind, seed)
    with glue_live.LiveGlue(cfg, "kapila", 4, 2, 2, wait_s=60.0) as g:
        assert sorted(g.blocks) == [(0, 0, 12, 12), (0, 12, 12, 12), (12, 0, 12, 12), (12, 12, 12, 12)]
        R, dts, st = g.rhs(U)
        assert st == hp.ERR_NO_DEVICE
        _, n, _, _, st = g.solve(U, 0.0, 1.0, 3)
        assert st == hp.ERR_NO_DEVICE and n == 0
