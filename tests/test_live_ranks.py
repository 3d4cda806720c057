"""The reference run as live MPI ranks (oracle.LiveReference): several processes,
one DMDA split over them as PETSc splits it, ghost strips exchanged and dt
reduced with MPI_Allreduce(MIN) through the PETSc stand-in's shared-memory MPI.

What the reference does on R ranks (rhs_function_prim.c:44-45 halo refresh,
:620-623 dt reduction; hype.c:108-122 DMDA over PETSC_DECIDE x PETSC_DECIDE)
must give its one-rank bits for the inviscid systems: the minimum over ranks of
CFL h / (2 s_max) is CFL h / (2 max s_max), and a cell's arithmetic does not
depend on which rank owns it.  An MPI_Abort in one rank must end the run of all
of them with the abort status.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")

KAP = dict(gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)
EUL = dict(gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
T, R, P = O.TRANSMISSIVE, O.REFLECTIVE, O.PERIODIC

CASES = [
    # system, kind, eos, order, nx, ny, bcs (l r b t), ranks, px, py, conservative
    (O.KAPILA, "shock_bubble", KAP, 2, 40, 36, (T, T, T, T), 4, 0, 0, 0),
    (O.KAPILA, "shock_bubble", KAP, 2, 37, 29, (P, P, R, R), 3, 0, 0, 0),
    (O.KAPILA, "shock_bubble", KAP, 3, 30, 28, (R, T, P, P), 4, 2, 2, 0),
    (O.KAPILA, "shock_bubble", KAP, 1, 33, 40, (T, T, T, T), 2, 1, 2, 1),
    (O.BN, "bn_discs", KAP, 2, 32, 30, (R, R, T, T), 6, 0, 0, 0),
    (O.EULER, "euler_quadrants", EUL, 2, 41, 35, (P, P, P, P), 4, 4, 1, 0),
    (O.EULER, "euler_quadrants", EUL, 0, 25, 25, (T, R, T, R), 2, 2, 1, 1),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"sys{c[0]}_N{c[3]}_{c[4]}x{c[5]}_r{c[7]}_{c[8]}x{c[9]}_c{c[10]}")
def test_live_ranks_equal_one_rank(case):
    system, kind, eos, order, nx, ny, bcs, nr, px, py, cons = case
    cfg = O.Config(system=system, order=order, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                   bc_top=bcs[3], conservative=cons, **eos)
    U = O.initial_state(cfg, kind, seed=nx + ny, nbubbles=2)
    one = O.Reference(system)
    one.setup(cfg)
    R1, dt1, st1 = one.rhs(U)
    Ue, n, t, dt, st = one.solve(U, 0.0, 1.0, 3)
    assert st1 == 0 and st == 0
    with O.LiveReference(cfg, nr, px, py, wait_s=60.0) as L:
        assert len(L.blocks) == nr
        # the blocks tile the grid
        cover = np.zeros((ny, nx), dtype=int)
        for xs, ys, xm, ym in L.blocks:
            cover[ys:ys + ym, xs:xs + xm] += 1
        assert (cover == 1).all()
        Rl, dtl, stl = L.rhs(U)
        assert stl == 0 and dtl == dt1
        assert Rl.tobytes() == R1.tobytes()
        Ul, nl, tl, dtnl, stl = L.solve(U, 0.0, 1.0, 3)
    assert stl == 0 and (nl, tl, dtnl) == (n, t, dt)
    assert Ul.tobytes() == Ue.tobytes()


def test_petsc_decide_process_grid():
    """PETSC_DECIDE on a square grid: 8 ranks -> 2 x 4, 6 -> 2 x 3, 4 -> 2 x 2; on a
    wide grid the longer side gets more ranks."""
    for nr, want in ((8, (2, 4)), (6, (2, 3)), (4, (2, 2)), (3, (1, 3))):
        cfg = O.Config(system=O.EULER, order=0, nx=48, ny=48, **EUL)
        with O.LiveReference(cfg, nr, wait_s=60.0) as L:
            got = (len({b[0] for b in L.blocks}), len({b[1] for b in L.blocks}))
        assert got == want, (nr, got)
    cfg = O.Config(system=O.EULER, order=0, nx=96, ny=24, **EUL)
    with O.LiveReference(cfg, 4, wait_s=60.0) as L:
        assert len({b[0] for b in L.blocks}) == 4


def test_abort_in_one_rank_ends_all():
    """A face state the reference rejects (MPI_Abort) in one rank: every rank's
    collective call ends and the run reports the abort."""
    cfg = O.Config(system=O.KAPILA, order=2, nx=24, ny=24, **KAP)
    U = O.initial_state(cfg, "shock_bubble", seed=1, nbubbles=1).reshape(24, 24, 6)
    U[20, 20, 4] = 0.0   # no energy in one cell (negative pressure), inside rank 3's block of a 2 x 2 grid
    one = O.Reference(O.KAPILA)
    one.setup(cfg)
    assert one.rhs(U.reshape(-1))[2] == 1
    with O.LiveReference(cfg, 4, 2, 2, wait_s=60.0) as L:
        _, _, st = L.rhs(U.reshape(-1))
    assert st == 1
