"""Accuracy: the SmoothVortex advection test of kapila_5eqn.c:519-562
(periodic [-3,3]^2, final time 6.0 = one period, GAMMA 4.0/1.4, PI 20/0) with
the error norms of ErrorNorms (post_process.c:74-155: alpha_1 against its
initial cell averages, L2 = ||e||_2 / N_x, L-infinity).

The GPU path is bit-identical to the reference's code, so at a size the oracle
finishes quickly the final state must equal the oracle's bit for bit; at finer
grids the scheme must show its third order (WENO N = 2 with SSPRK(4,3)).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def vortex_cfg(hp, n, cfl=0.4):
    P = hp.BC_PERIODIC
    return hp.Config(system=hp.KAPILA_5EQN, order=2, nx=n, ny=n, x_min=-3.0, x_max=3.0, y_min=-3.0, y_max=3.0, cfl=cfl,
                     bc_left=P, bc_right=P, bc_bottom=P, bc_top=P, gamma1=4.0, gamma2=1.4, pi1=20.0, pi2=0.0)


def error_norms(U, U0, n):
    e = U0.reshape(-1, 6)[:, 5] - U.reshape(-1, 6)[:, 5]
    return float(np.sqrt(np.sum(e * e)) / n), float(np.max(np.abs(e)))


def run(hp, n, cfl=0.4):
    c = vortex_cfg(hp, n, cfl)
    U0 = hp.initial_state(c, "smooth_vortex")
    with hp.Solver(c) as s:
        s.set_state(U0)
        k, t, _, st = s.solve(0.0, 6.0, 10 ** 7)
        assert st == hp.OK and t == 6.0
        return U0, s.get_state(), k


def test_smooth_vortex_equals_reference_code(hp, orc):
    n = 32
    U0, U, k = run(hp, n)
    oc = O.Config(system=O.KAPILA, order=2, nx=n, ny=n, x_min=-3.0, x_max=3.0, y_min=-3.0, y_max=3.0, cfl=0.4,
                  bc_left=O.PERIODIC, bc_right=O.PERIODIC, bc_bottom=O.PERIODIC, bc_top=O.PERIODIC,
                  gamma1=4.0, gamma2=1.4, pi1=20.0, pi2=0.0)
    Uo, ko, to, _, sto = orc.solve(oc, U0, 0.0, 6.0, 10 ** 7)
    assert sto == O.OK and ko == k and to == 6.0
    assert U.tobytes() == Uo.tobytes()
    l2, linf = error_norms(U, U0, n)
    assert l2 == pytest.approx(0.017119652587459115, rel=1e-12)
    assert linf == pytest.approx(0.07526030231431413, rel=1e-12)


def test_smooth_vortex_third_order(hp):
    errs = {n: error_norms(*run(hp, n)[:2], n) for n in (128, 256, 512)}
    for a, b in ((128, 256), (256, 512)):
        order_l2 = np.log2(errs[a][0] / errs[b][0])
        order_inf = np.log2(errs[a][1] / errs[b][1])
        print(a, b, errs[a], errs[b], order_l2, order_inf)
    assert np.log2(errs[256][0] / errs[512][0]) > 2.8
    assert np.log2(errs[256][1] / errs[512][1]) > 2.8
