"""Mixed precision (HYPE_PREC_MIXED) for the Baer-Nunziato and Euler systems
against their FP64 paths (bit-identical to the reference, test_gpu_parity.py).

FP32 state, reconstruction and fluxes of densities and momenta; FP64 energies
(where the stiffened-gas pressure recovery cancels gamma P_inf ~ 2.6e9 against
rho e), volume fraction, cell totals and dt.  The bar is the mixed form's
specification: relative L1 error <= 1e-5 in density and volume fraction after
a run; per-field RHS errors within single-precision accuracy.  Batched and
y-slab runs equal the lone mixed solver bit for bit.
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

T_, R_, P_ = O.TRANSMISSIVE, O.REFLECTIVE, O.PERIODIC


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def vec_rel_l1(A, B, cols):
    d = np.sqrt(((A[:, cols] - B[:, cols]) ** 2).sum(axis=1)).sum()
    return float(d / max(np.sqrt((B[:, cols] ** 2).sum(axis=1)).sum(), 1e-300))


# per-system report fields: scalars (component) and vectors (momentum components)
FIELDS = {O.BN: ({"a1rho1": 0, "a1E1": 3, "a2rho2": 4, "a2E2": 7, "alpha1": 8}, {"mom1": [1, 2], "mom2": [5, 6]}),
          O.EULER: ({"rho": 0, "E": 3}, {"mom": [1, 2]})}


def field_report(M, F, system):
    sc, vc = FIELDS[system]
    out = {k: (rel_l1(M[:, c], F[:, c]), rel_linf(M[:, c], F[:, c])) for k, c in sc.items()}
    out.update({k: (vec_rel_l1(M, F, c), None) for k, c in vc.items()})
    return out


RHS_CASES = [
    # system, kind, nx, ny, bcs, fixed form, seed
    (O.BN, "discs", 144, 112, (T_, T_, R_, R_), 0, 61),
    (O.BN, "discs", 120, 96, (P_, P_, P_, P_), 1, 62),
    (O.BN, "discs", 96, 80, (R_, T_, R_, T_), 1, 63),
    (O.EULER, "quadrants", 160, 128, (T_, T_, R_, R_), 0, 64),
    (O.EULER, "quadrants", 128, 96, (P_, P_, R_, R_), 0, 65),
]


@pytest.mark.parametrize("system,kind,nx,ny,bcs,fixed,seed", RHS_CASES)
def test_mixed_rhs_close_to_fp64(hp, orc, system, kind, nx, ny, bcs, fixed, seed):
    eos = cases.KAPILA_EOS if system == O.BN else dict(gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    cfg = O.Config(system=system, order=2, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2], bc_top=bcs[3],
                   bn_fixed_p2=fixed, **eos)
    U = cases.state(cfg, kind, seed)
    Ro, dto, sto = orc.rhs(cfg, U)
    assert sto == O.OK
    pc = cases.to_pkg(cfg)
    pc.precision = hp.PREC_MIXED
    with hp.Solver(pc) as s:
        R, dt, st = s.rhs_function_prim(0.0, U)
    assert st == hp.OK
    assert abs(dt - dto) <= 1e-6 * dto
    nv = cfg.nvar
    rep = field_report(R.reshape(-1, nv), Ro.reshape(-1, nv), system)
    print(system, kind, "mixed RHS vs FP64 (rel L1, rel Linf):", rep)
    for k, (l1, _) in rep.items():
        assert l1 <= 5e-3, (k, l1)


def run_both(hp, cfg_fp64, U0, steps):
    out = {}
    for prec in (hp.PREC_FP64, hp.PREC_MIXED):
        c = hp.Config(**{**cfg_fp64.__dict__, "precision": prec})
        with hp.Solver(c) as s:
            s.set_state(U0)
            k, t, dtn, st = s.solve(0.0, 1e30, steps)
            assert st == hp.OK and k == steps, (prec, st, k)
            out[prec] = (s.get_state(), t)
    return out[hp.PREC_FP64], out[hp.PREC_MIXED]


@pytest.mark.parametrize("n,steps,seed", [(256, 60, 3), (192, 100, 4)])
def test_mixed_bn_run_error_vs_fp64(hp, n, steps, seed):
    """Baer-Nunziato discs (the 1024^2 configuration's generator), the phase-2
    flux pressure V[7]: relative L1 of mixture density and of alpha_1 <= 1e-5
    after the run."""
    cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=n, ny=n, cfl=0.4, flags=hp.FLAG_BN_FIX_P2)
    U0 = hp.initial_state(cfg, "bn_discs", seed=seed)
    (F, tf), (M, tm) = run_both(hp, cfg, U0, steps)
    F, M = F.reshape(-1, 9), M.reshape(-1, 9)
    rep = field_report(M, F, O.BN)
    rho_f, rho_m = F[:, 0] + F[:, 4], M[:, 0] + M[:, 4]
    rep["rho"] = (rel_l1(rho_m, rho_f), rel_linf(rho_m, rho_f))
    print("mixed BN vs FP64 after", steps, "steps:", rep)
    assert rep["rho"][0] <= 1e-5, rep
    assert rep["alpha1"][0] <= 1e-5, rep
    assert abs(tm - tf) <= 1e-5 * tf


def test_mixed_euler_run_error_vs_fp64(hp):
    """Euler four-quadrant states (the serving mix's generator): relative L1 of
    density and energy <= 1e-5 after 100 steps."""
    cfg = hp.Config(system=hp.EULER, order=2, nx=256, ny=256, cfl=0.4, gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    U0 = hp.initial_state(cfg, "euler_quadrants", seed=5)
    (F, tf), (M, tm) = run_both(hp, cfg, U0, 100)
    F, M = F.reshape(-1, 4), M.reshape(-1, 4)
    rep = field_report(M, F, O.EULER)
    print("mixed Euler vs FP64 after 100 steps:", rep)
    assert rep["rho"][0] <= 1e-5, rep
    assert rep["E"][0] <= 1e-5, rep
    assert abs(tm - tf) <= 1e-5 * tf


def test_mixed_bn_conserves_partial_masses(hp):
    cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=160, ny=128, cfl=0.4, flags=hp.FLAG_BN_FIX_P2,
                    precision=hp.PREC_MIXED, bc_left=hp.BC_PERIODIC, bc_right=hp.BC_PERIODIC, bc_bottom=hp.BC_PERIODIC,
                    bc_top=hp.BC_PERIODIC)
    U0 = hp.initial_state(cfg, "bn_discs", seed=9)
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        t0, _, _ = s.totals()
        k, t, dtn, st = s.solve(0.0, 1e30, 40)
        assert st == hp.OK
        t1, amin, amax = s.totals()
    assert 0.0 <= amin and amax <= 1.0
    for c in (0, 4):   # FP32 storage, FP64 accumulation
        assert abs(t1[c] - t0[c]) <= 1e-6 * abs(t0[c]), (c, t0[c], t1[c])


def test_mixed_bn_and_euler_batched_equal_lone(hp):
    """Mixed Baer-Nunziato (both flux forms) and mixed Euler instances of uneven
    sizes in one batch, beside a mixed Kapila one: each equals its lone mixed
    solver bit for bit."""
    T, R, P = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE, hp.BC_PERIODIC
    items = []
    for k, (nx, ny, fl) in enumerate(((96, 80, hp.FLAG_BN_FIX_P2), (130, 64, hp.FLAG_BN_FIX_P2), (72, 100, 0))):
        c = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=nx, ny=ny, cfl=0.4, flags=fl, precision=hp.PREC_MIXED,
                      bc_left=T, bc_right=R, bc_bottom=P, bc_top=P)
        items.append((c, hp.initial_state(c, "bn_discs", seed=70 + k), 1e30, 6))
    for k, (nx, ny) in enumerate(((120, 90), (64, 200))):
        c = hp.Config(system=hp.EULER, order=2, nx=nx, ny=ny, cfl=0.4, precision=hp.PREC_MIXED, gamma1=1.4, gamma2=1.4,
                      pi1=0.0, pi2=0.0, bc_left=T, bc_right=T, bc_bottom=R, bc_top=R)
        items.append((c, hp.initial_state(c, "euler_quadrants", seed=75 + k), 0.05, 1000))
    ck = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=100, ny=80, cfl=0.4, precision=hp.PREC_MIXED)
    items.append((ck, hp.initial_state(ck, "shock_bubble", seed=79, nbubbles=2), 1e30, 6))
    with hp.Batch(max_instances=8) as b:
        ids = [b.add(c, U0, 0.0, tf, nmax) for c, U0, tf, nmax in items]
        for _ in range(60):
            b.advance(10)
            b.sync()
            if all(b.status(i)["done"] for i in ids):
                break
        for i, (c, U0, tf, nmax) in zip(ids, items):
            with hp.Solver(c) as s:
                s.set_state(U0)
                k, t, dtn, st = s.solve(0.0, tf, nmax, check=False)
                Ul = s.get_state()
            sb = b.status(i)
            assert sb["status"] == st, (i, sb, st)
            if st != hp.OK:
                continue
            assert sb["steps"] == k and sb["t"] == t, (i, sb, k, t)
            assert b.get_state(i).tobytes() == Ul.tobytes(), i


@pytest.mark.parametrize("system,nslabs", [(2, 3), (0, 2)])
def test_mixed_bn_and_euler_slabs_equal_lone(hp, system, nslabs):
    """y-slabs of a mixed Baer-Nunziato / Euler grid (edge rows stored into the
    neighbours' FP32 and FP64 halo planes) equal the single mixed solver."""
    P = hp.BC_PERIODIC
    if system == 2:
        cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=80, ny=66, cfl=0.4, flags=hp.FLAG_BN_FIX_P2,
                        precision=hp.PREC_MIXED, bc_bottom=P, bc_top=P)
        U = hp.initial_state(cfg, "bn_discs", seed=81)
    else:
        cfg = hp.Config(system=hp.EULER, order=2, nx=90, ny=50, cfl=0.4, precision=hp.PREC_MIXED, gamma1=1.4, gamma2=1.4,
                        pi1=0.0, pi2=0.0)
        U = hp.initial_state(cfg, "euler_quadrants", seed=82)
    with hp.Solver(cfg) as s:
        s.set_state(U)
        k1, t1, dt1, st1 = s.solve(0.0, 1e30, 10)
        U1 = s.get_state()
    with hp.Group(cfg, nslabs) as grp:
        grp.set_state(U)
        k2, t2, dt2, st2 = grp.solve(0.0, 1e30, 10)
        U2 = grp.get_state()
    assert st1 == st2 == hp.OK and (k1, t1, dt1) == (k2, t2, dt2)
    assert U1.tobytes() == U2.tobytes()


HOST_BAND_CASES = [
    # system, kind, nx, ny, periodic y
    (O.KAPILA, "bubble", 640, 720, False),
    (O.KAPILA, "bubble", 600, 704, True),
    (O.BN, "discs", 480, 512, False),
    (O.EULER, "quadrants", 512, 600, True),
]


@pytest.mark.parametrize("system,kind,nx,ny,periodic", HOST_BAND_CASES)
def test_mixed_host_calls_banded_equal_unbanded(hp, system, kind, nx, ny, periodic):
    """The host-buffer calls of a mixed solver run band by band (row bands, every
    stage a wavefront on four streams, copies overlapped): hype_advance_host gives the
    bits of set_state + advance + wait + get_state (1 and 2 steps), and hype_rhs_prim
    from host arrays the bits and dt of the whole-grid call on device pointers."""
    import torch
    eos = cases.KAPILA_EOS if system != O.EULER else dict(gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    yb = P_ if periodic else R_
    cfg = O.Config(system=system, order=2, nx=nx, ny=ny, bc_left=T_, bc_right=T_, bc_bottom=yb, bc_top=yb, **eos)
    U = cases.state(cfg, kind, 70 + nx % 7)
    pc = cases.to_pkg(cfg)
    pc.precision = hp.PREC_MIXED
    for nsteps in (1, 2):
        with hp.Solver(pc) as s:
            s.set_state(U)
            s.begin(0.0, 1e30, 100)
            s.advance(nsteps)
            ref = (s.wait(), s.get_state())
        out = np.empty_like(U)
        with hp.Solver(pc) as s:
            assert s.launch_info()["grid"][1] >= 8
            s.set_state(U)
            s.begin(0.0, 1e30, 100)
            got = s.advance_host(U, out, nsteps)
        assert got[3] == hp.OK and got[:3] == ref[0][:3]
        assert out.tobytes() == ref[1].tobytes()
    dU = torch.from_numpy(U).cuda()
    dR = torch.empty_like(dU)
    torch.cuda.synchronize()
    with hp.Solver(pc) as s:
        dt_d, st_d = s.rhs_function_prim_device(0.0, dU.data_ptr(), dR.data_ptr())
        R, dt_h, st_h = s.rhs_function_prim(0.0, U)
    assert st_d == hp.OK and st_h == hp.OK and dt_h == dt_d
    assert R.tobytes() == dR.cpu().numpy().tobytes()
