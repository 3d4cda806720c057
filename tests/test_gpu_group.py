"""One grid split into y-slabs (include/hype_group.h) against the reference's bits.

HyPE-2D decomposes its grid over MPI ranks with a DMDA (hype.c:108-122) and
refreshes 3 ghost rows per rank before every RHS (rhs_function_prim.c:44-45);
dt is the global minimum (rhs_function_prim.c:620-623).  A decomposed run must
give the same bits as the undecomposed one.  Here every solve case of the golden
file is rerun with its rows split over 2 and 3 slabs, against the reference's
hashes.  Larger and uneven splits, every system, order and path, and periodic,
inlet and reflective edges are checked against a lone Solver.  The slabs share
the test's one GPU.  Their kernels never wait on each other inside a launch:
the ordering is events between streams.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))
T, R, P, I = O.TRANSMISSIVE, O.REFLECTIVE, O.PERIODIC, O.INLET


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.mark.parametrize("nslabs", [2, 3])
@pytest.mark.parametrize("name", sorted(GOLDEN["solve"]))
def test_group_solve_equals_reference(name, nslabs, hp):
    g = GOLDEN["solve"][name]
    (_, cfg, kind, seed), t0, tf, nmax = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    with hp.Group(cases.to_pkg(cfg), nslabs) as grp:
        grp.set_state(U)
        steps, te, dtn, st = grp.solve(t0, tf, nmax)
        Ue = grp.get_state()
    if g["status"] != 0:
        assert st == hp.ERR_INADMISSIBLE
        return
    assert st == hp.OK
    assert steps == g["steps"]
    assert float(te).hex() == g["t_end"]
    assert float(dtn).hex() == g["dt_next"]
    assert sha(Ue) == g["sha_U_end"]


def lone(hp, pcfg, U, t0, tf, nmax):
    with hp.Solver(pcfg) as s:
        s.set_state(U)
        k, t, dt, st = s.solve(t0, tf, nmax)
        return k, t, dt, st, s.get_state()


GROUP_CASES = [
    # (case, nslabs, steps)
    (cases._k("kapila_64x50_uneven", 64, 50, bcs=(T, T, R, R), seed=70), 3, 12),          # 17 + 17 + 16 rows
    (cases._k("kapila_48x40_periodic4", 48, 40, bcs=(P, P, P, P), seed=71), 4, 8),
    (cases._k("kapila_40x24_periodic2", 40, 24, bcs=(T, R, P, P), seed=72), 2, 8),        # both neighbours are one slab
    (cases._k("kapila_30x9_min_rows", 30, 9, bcs=(R, T, R, T), seed=73), 3, 6),   # 3 rows a slab
    # a rough field that turns inadmissible: both stop at the same step with the same state
    (cases._k("kapila_30x9_rough_stops", 30, 9, bcs=(R, T, R, T), kind="rough", seed=73), 3, 6),
    (cases._k("kapila_36x30_inlet", 36, 30, bcs=(I, T, R, R), seed=74, x_min=0.0, x_max=2.0,
              y_min=-1.0, y_max=1.0), 3, 6),
    (cases._k("kapila_32x33_N0", 32, 33, order=0, bcs=(T, T, R, R), seed=75), 3, 10),
    (cases._k("kapila_32x31_N1", 32, 31, order=1, bcs=(R, R, T, T), seed=76), 5, 10),
    (cases._k("kapila_24x27_N3", 24, 27, order=3, bcs=(T, T, P, P), seed=77), 3, 3),
    (cases._k("kapila_cons_40x30", 40, 30, bcs=(T, T, R, R), seed=78, conservative=1), 3, 8),
    (cases._k("kapila_visc_40x30", 40, 30, bcs=(T, T, R, R), seed=79, viscous=1, mu1=0.5, mu2=0.1), 3, 6),
    (cases._k("kapila_visc_cons_30x28_N3", 30, 28, order=3, bcs=(R, T, P, P), seed=80, conservative=1, viscous=1,
              mu1=2.0, mu2=0.5), 4, 3),
    (cases._b("bn_40x36_fixed", 40, 36, bcs=(T, T, R, R), seed=81, fixed=1), 3, 8),
    (cases._b("bn_cons_30x30_N3", 30, 30, order=3, bcs=(P, P, P, P), seed=82, conservative=1), 2, 3),
    (cases._e("euler_48x40_N1", 48, 40, order=1, bcs=(T, T, R, R), seed=83), 6, 100000),   # to t_final (MATCHSTEP)
    (cases._e("euler_cons_40x32", 40, 32, bcs=(R, R, P, P), seed=84, conservative=1), 4, 100000),
]


@pytest.mark.parametrize("case,nslabs,nmax", GROUP_CASES, ids=[c[0][0] for c in GROUP_CASES])
def test_group_equals_lone_solver(case, nslabs, nmax, hp):
    _, cfg, kind, seed = case
    tf = 0.02 if cfg.system == O.EULER else 1.0
    U = cases.state(cfg, kind, seed)
    pcfg = cases.to_pkg(cfg)
    k1, t1, dt1, st1, U1 = lone(hp, pcfg, U, 0.0, tf, nmax)
    with hp.Group(pcfg, nslabs) as grp:
        rows = [grp.slab(k) for k in range(nslabs)]
        assert [r[0] for r in rows] == list(np.cumsum([0] + [r[1] for r in rows])[:-1])
        assert sum(r[1] for r in rows) == cfg.ny and max(r[1] for r in rows) - min(r[1] for r in rows) <= 1
        grp.set_state(U)
        k2, t2, dt2, st2 = grp.solve(0.0, tf, nmax)
        U2 = grp.get_state()
    assert st1 == st2
    assert st1 == (hp.ERR_INADMISSIBLE if kind == "rough" else hp.OK)
    assert (k1, t1.hex(), dt1.hex()) == (k2, t2.hex(), dt2.hex())
    assert U1.tobytes() == U2.tobytes(), float(np.abs(U1 - U2).max())


def test_group_one_slab_and_split_runs(hp):
    """nslabs = 1 is the lone solver; begin / advance / wait in chunks equals one solve."""
    _, cfg, kind, seed = cases._k("kapila_40x36", 40, 36, bcs=(T, T, R, R), seed=85)
    U = cases.state(cfg, kind, seed)
    pcfg = cases.to_pkg(cfg)
    k1, t1, dt1, st1, U1 = lone(hp, pcfg, U, 0.0, 1.0, 9)
    with hp.Group(pcfg, 1) as grp:
        grp.set_state(U)
        assert grp.solve(0.0, 1.0, 9)[:3] == (k1, t1, dt1)
        assert grp.get_state().tobytes() == U1.tobytes()
    with hp.Group(pcfg, 3) as grp:
        grp.set_state(U)
        grp.begin(0.0, 1.0, 9)
        for n in (2, 3, 4, 5):           # the last chunk runs past max_steps: no extra step
            grp.advance(n)
        k, t, dt, st = grp.wait()
        assert (k, t, dt, st) == (k1, t1, dt1, hp.OK)
        assert grp.get_state().tobytes() == U1.tobytes()
        assert grp.last_elapsed_ms() > 0.0


def test_group_stops_with_the_reference_error(hp):
    """The Baer-Nunziato phase-2 pressure as written (V[8], baer_nunziato.c:271)
    makes these states inadmissible after some steps: the slabs stop at the
    same step as the lone solver, with the same first cell."""
    _, cfg, kind, seed = cases._b("bn_48x45_bug", 48, 45, bcs=(T, T, T, T), seed=86)
    U = cases.state(cfg, kind, seed)
    pcfg = cases.to_pkg(cfg)
    with hp.Solver(pcfg) as s:
        s.set_state(U)
        k1, t1, dt1, st1 = s.solve(0.0, 1.0, 400)
        msg1 = hp.lib().hype_last_error(s._h).decode()
    if st1 != hp.ERR_INADMISSIBLE:
        pytest.skip("this state did not become inadmissible within 400 steps")
    with hp.Group(pcfg, 3) as grp:
        grp.set_state(U)
        k2, t2, dt2, st2 = grp.solve(0.0, 1.0, 400)
        assert st2 == hp.ERR_INADMISSIBLE
        assert (k1, t1) == (k2, t2)
        assert grp.last_error() == msg1


def test_group_full_size(hp):
    """1024^2 Kapila as 4 slabs: 10 steps, the single solver's bits."""
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=1024, ny=1024, cfl=0.4, bc_bottom=hp.BC_REFLECTIVE,
                    bc_top=hp.BC_REFLECTIVE)
    U = hp.initial_state(cfg, "shock_bubble", seed=4, nbubbles=3)
    k1, t1, dt1, st1, U1 = lone(hp, cfg, U, 0.0, 1e30, 10)
    with hp.Group(cfg, 4) as grp:
        grp.set_state(U)
        k2, t2, dt2, st2 = grp.solve(0.0, 1e30, 10)
        U2 = grp.get_state()
    assert st1 == st2 == hp.OK and (k1, t1, dt1) == (k2, t2, dt2)
    assert U1.tobytes() == U2.tobytes()


@pytest.mark.parametrize("name,nranks", [("kapila_37x23_rough_mixed_bc", 3), ("kapila_24x24_periodic", 2),
                                         ("bn_13x21_periodic_N1", 4), ("kapila_visc_cons_15x13_N3", 2)])
def test_rhs_prim_slab_reads_only_rows(name, nranks, hp, orc):
    """hype_rhs_prim_slab on DMDA-style local arrays: owned rows plus 3 ghost rows
    from the neighbours, 3 ghost columns each side holding NaN (never read), rows
    (nx + 6) * nvar apart.  The ranks' rows make the reference's RHS bit for bit."""
    import ctypes
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    Ro, dto, _ = orc.rhs(cfg, U)
    nv, nx, ny = cfg.nvar, cfg.nx, cfg.ny
    Ug = U.reshape(ny, nx, nv)
    L = hp.lib()
    DP = ctypes.POINTER(ctypes.c_double)
    L.hype_create_slab.argtypes = [ctypes.POINTER(hp._Cfg), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.hype_rhs_prim_slab.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong, DP, DP]
    periodic = cfg.bc_bottom == O.PERIODIC
    rows = [ny // nranks + (1 if r < ny % nranks else 0) for r in range(nranks)]
    R = np.full_like(U, np.nan)
    dts = []
    for r in range(nranks):
        ys, ym = sum(rows[:r]), rows[r]
        loc = np.full((ym + 6, nx + 6, nv), np.nan)
        for j in range(-3, ym + 3):
            g = ys + j
            if 0 <= g < ny or periodic:
                loc[j + 3, 3:nx + 3] = Ug[g % ny]
        h = ctypes.c_void_p()
        st = L.hype_create_slab(ctypes.byref(cases.to_pkg(cfg).c_struct()), ys, ym, ctypes.byref(h))
        assert st == hp.OK, L.hype_last_error(h)
        Rr = np.empty(ym * nx * nv)
        dt = ctypes.c_double()
        base = loc.ctypes.data + ((3 * (nx + 6) + 3) * nv) * 8
        st = L.hype_rhs_prim_slab(h, 0.0, base, (nx + 6) * nv, Rr.ctypes.data_as(DP), ctypes.byref(dt))
        L.hype_destroy(h)
        assert st == hp.OK
        R[ys * nx * nv:(ys + ym) * nx * nv] = Rr
        dts.append(dt.value)
    assert R.tobytes() == Ro.tobytes()
    if not cfg.viscous:
        assert min(dts) == dto


@pytest.mark.parametrize("seed", range(4))
def test_group_random_configurations(seed, hp):
    """Random grids, slab counts (1 .. ny/3), orders, systems, paths and boundaries:
    the group's t, steps, dt and state equal the single solver's, bit for bit (or
    both stop with the same error at the same step)."""
    rng = np.random.default_rng(500 + seed)
    for _ in range(4):
        system = int(rng.choice([O.EULER, O.KAPILA, O.BN]))
        order = int(rng.integers(0, 4))
        nx, ny = int(rng.integers(6, 90)), int(rng.integers(6, 60))
        bcs = [int(b) for b in rng.choice([T, R], 4)]
        if rng.uniform() < 0.4:
            bcs[2] = bcs[3] = P
        if rng.uniform() < 0.3:
            bcs[0] = bcs[1] = P
        kw = dict(conservative=int(rng.uniform() < 0.3))
        if system == O.KAPILA and order >= 1 and rng.uniform() < 0.3:
            kw.update(viscous=1, mu1=float(rng.uniform(0, 0.5)), mu2=float(rng.uniform(0, 0.1)))
        if system == O.BN:
            kw["fixed"] = 1
        mk = {O.EULER: cases._e, O.KAPILA: cases._k, O.BN: cases._b}[system]
        _, cfg, kind, sd = mk("random", nx, ny, order=order, bcs=bcs, seed=int(rng.integers(1 << 20)), **kw)
        U = cases.state(cfg, kind, sd)
        pcfg = cases.to_pkg(cfg)
        nslabs = int(rng.integers(1, ny // 3 + 1))
        tf = 0.01 if system == O.EULER else 1.0
        k1, t1, dt1, st1, U1 = lone(hp, pcfg, U, 0.0, tf, 6)
        with hp.Group(pcfg, nslabs) as grp:
            grp.set_state(U)
            k2, t2, dt2, st2 = grp.solve(0.0, tf, 6)
            U2 = grp.get_state()
        what = (system, order, nx, ny, bcs, kw, nslabs)
        assert (st1, k1, t1, dt1) == (st2, k2, t2, dt2), what
        assert U1.tobytes() == U2.tobytes(), what


@pytest.mark.parametrize("bcy,nslabs,seed", [(R, 3, 0), (P, 4, 1), (T, 2, 2)])
def test_group_mixed_precision(bcy, nslabs, seed, hp):
    """The mixed-precision form as y-slabs: the stage kernel stores its edge rows
    into the neighbours' FP32 and FP64 halo planes; every bit equals the single
    mixed-precision solver's (the mixed kernel's per-cell arithmetic does not
    depend on the tiling either)."""
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=96, ny=70, cfl=0.4, precision=hp.PREC_MIXED, bc_bottom=bcy, bc_top=bcy)
    U = hp.initial_state(cfg, "shock_bubble", seed=90 + seed, nbubbles=2)
    k1, t1, dt1, st1, U1 = lone(hp, cfg, U, 0.0, 1e30, 12)
    with hp.Group(cfg, nslabs) as grp:
        grp.set_state(U)
        k2, t2, dt2, st2 = grp.solve(0.0, 1e30, 12)
        U2 = grp.get_state()
    assert st1 == st2 == hp.OK and (k1, t1, dt1) == (k2, t2, dt2)
    assert U1.tobytes() == U2.tobytes()


def test_rhs_prim_slab_mixed_precision(hp):
    """hype_rhs_prim_slab on a mixed-precision configuration: the ranks' rows make
    the single mixed solver's RHS bit for bit, and the least of their dt is its dt."""
    import ctypes
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=80, ny=45, cfl=0.4, precision=hp.PREC_MIXED, bc_bottom=P, bc_top=P)
    U = hp.initial_state(cfg, "shock_bubble", seed=95, nbubbles=3)
    with hp.Solver(cfg) as s:
        Rf, dtf, st = s.rhs_function_prim(0.0, U)
    assert st == hp.OK
    nv, nx, ny = 6, cfg.nx, cfg.ny
    Ug = U.reshape(ny, nx, nv)
    L = hp.lib()
    DP = ctypes.POINTER(ctypes.c_double)
    L.hype_create_slab.argtypes = [ctypes.POINTER(hp._Cfg), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.hype_rhs_prim_slab.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong, DP, DP]
    R = np.full_like(U, np.nan)
    dts = []
    for ys, ym in ((0, 15), (15, 15), (30, 15)):
        loc = np.full((ym + 6, nx + 6, nv), np.nan)
        for j in range(-3, ym + 3):
            loc[j + 3, 3:nx + 3] = Ug[(ys + j) % ny]
        h = ctypes.c_void_p()
        assert L.hype_create_slab(ctypes.byref(cfg.c_struct()), ys, ym, ctypes.byref(h)) == hp.OK
        Rr = np.empty(ym * nx * nv)
        dt = ctypes.c_double()
        st = L.hype_rhs_prim_slab(h, 0.0, loc.ctypes.data + ((3 * (nx + 6) + 3) * nv) * 8, (nx + 6) * nv, Rr.ctypes.data_as(DP),
                                  ctypes.byref(dt))
        L.hype_destroy(h)
        assert st == hp.OK
        R[ys * nx * nv:(ys + ym) * nx * nv] = Rr
        dts.append(dt.value)
    assert R.tobytes() == Rf.tobytes()
    assert min(dts) == dtf


BLOCK_CASES = [("kapila_37x23_rough_mixed_bc", 2, 2), ("kapila_24x24_periodic", 3, 2), ("kapila_18x14_inlet", 3, 1),
               ("kapila_15x13_N3", 2, 2), ("bn_13x21_periodic_N1", 2, 3), ("euler_21x19_reflective_N1", 3, 3),
               ("kapila_cons_37x23_rough", 4, 2), ("kapila_visc_37x23_rough", 2, 2)]


@pytest.mark.parametrize("name,px,py", BLOCK_CASES)
def test_rhs_prim_block_reads_only_its_halo(name, px, py, hp, orc):
    """hype_create_block + hype_rhs_prim_slab on DMDA-style local arrays of a grid
    split px x py: the rank's block, 3 ghost rows and columns (corners included)
    from the neighbours where a neighbour exists (periodic axes wrap), NaN in every
    ghost cell on a physical boundary -- the kernel must fill those itself.  The
    blocks' RHS make the reference's RHS bit for bit and the least of their dt is its
    dt (inviscid)."""
    import ctypes
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    Ro, dto, _ = orc.rhs(cfg, U)
    nv, nx, ny = cfg.nvar, cfg.nx, cfg.ny
    Ug = U.reshape(ny, nx, nv)
    L = hp.lib()
    DP = ctypes.POINTER(ctypes.c_double)
    L.hype_create_block.argtypes = [ctypes.POINTER(hp._Cfg), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]
    L.hype_rhs_prim_slab.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong, DP, DP]
    perx, pery = cfg.bc_left == O.PERIODIC, cfg.bc_bottom == O.PERIODIC

    def split(n, p):   # PETSc's: the first n % p ranks one more
        sizes = [n // p + (1 if r < n % p else 0) for r in range(p)]
        return [(sum(sizes[:r]), sizes[r]) for r in range(p)]
    R = np.full((ny, nx, nv), np.nan)
    dts = []
    for ys, ym in split(ny, py):
        for xs, xm in split(nx, px):
            loc = np.full((ym + 6, xm + 6, nv), np.nan)
            for j in range(-3, ym + 3):
                for i in range(-3, xm + 3):
                    gj, gi = ys + j, xs + i
                    if (0 <= gj < ny or pery) and (0 <= gi < nx or perx):
                        loc[j + 3, i + 3] = Ug[gj % ny, gi % nx]
            h = ctypes.c_void_p()
            st = L.hype_create_block(ctypes.byref(cases.to_pkg(cfg).c_struct()), xs, xm, ys, ym, ctypes.byref(h))
            assert st == hp.OK, L.hype_last_error(h)
            Rr = np.empty(ym * xm * nv)
            dt = ctypes.c_double()
            base = loc.ctypes.data + ((3 * (xm + 6) + 3) * nv) * 8
            st = L.hype_rhs_prim_slab(h, 0.0, base, (xm + 6) * nv, Rr.ctypes.data_as(DP), ctypes.byref(dt))
            L.hype_destroy(h)
            assert st == hp.OK
            R[ys:ys + ym, xs:xs + xm] = Rr.reshape(ym, xm, nv)
            dts.append(dt.value)
    assert R.reshape(-1).tobytes() == Ro.tobytes()
    if not cfg.viscous:
        assert min(dts) == dto


def _local_arrays(Ug, ys, ym, xs, xm, perx, pery):
    """DMDA-style local array of block (ys, ym) x (xs, xm): 3 ghost rows and columns
    from the neighbours (periodic axes wrap), NaN where the grid ends."""
    ny, nx, _ = Ug.shape
    rr, cc = np.arange(ys - 3, ys + ym + 3), np.arange(xs - 3, xs + xm + 3)
    loc = Ug[np.ix_(rr % ny, cc % nx)].copy()
    if not pery:
        loc[(rr < 0) | (rr >= ny)] = np.nan
    if not perx:
        loc[:, (cc < 0) | (cc >= nx)] = np.nan
    return np.ascontiguousarray(loc)


LARGE_SPLITS = [
    # system, nx, ny, px, py, periodic x, periodic y, mixed, anchor
    (O.KAPILA, 300, 420, 1, 3, False, False, False, "reference"),
    (O.BN, 260, 300, 3, 2, False, True, False, "reference"),
    (O.KAPILA, 1100, 1200, 1, 2, False, False, False, "device"),
    (O.KAPILA, 1100, 1200, 2, 2, True, True, False, "device"),
    (O.BN, 1024, 1400, 1, 2, False, True, False, "device"),
    (O.KAPILA, 1100, 1200, 1, 2, False, True, True, "device"),
]


@pytest.mark.parametrize("system,nx,ny,px,py,perx,pery,mixed,anchor", LARGE_SPLITS)
def test_rhs_prim_slab_banded_large(system, nx, ny, px, py, perx, pery, mixed, anchor, hp, orc):
    """hype_rhs_prim_slab on blocks of 130-700 rows, which run as 1-5 row bands (each
    band's rows copied from the local array, converted and launched as they arrive,
    its RHS rows copied out while later bands compute): the blocks make, bit for bit,
    the reference's RHS, or the whole-grid RHS on device pointers (itself the
    reference's bits in FP64, test_gpu_parity.py), and the least of their dt its dt."""
    import ctypes
    import torch
    bx = P if perx else T
    by = P if pery else R
    cfg = O.Config(system=system, order=2, nx=nx, ny=ny, bc_left=bx, bc_right=bx, bc_bottom=by, bc_top=by, **cases.KAPILA_EOS)
    U = cases.state(cfg, "bubble" if system == O.KAPILA else "discs", 90 + px + 3 * py)
    pc = cases.to_pkg(cfg)
    if mixed:
        pc.precision = hp.PREC_MIXED
    if anchor == "reference":
        Ro, dto, sto = orc.rhs(cfg, U)
    else:
        dU = torch.from_numpy(U).cuda()
        dR = torch.empty_like(dU)
        torch.cuda.synchronize()
        with hp.Solver(pc) as s:
            dto, sto = s.rhs_function_prim_device(0.0, dU.data_ptr(), dR.data_ptr())
        Ro = dR.cpu().numpy()
    assert sto == hp.OK
    nv = cfg.nvar
    Ug = U.reshape(ny, nx, nv)
    L = hp.lib()
    DP = ctypes.POINTER(ctypes.c_double)
    L.hype_create_block.argtypes = [ctypes.POINTER(hp._Cfg), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]
    L.hype_rhs_prim_slab.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong, DP, DP]

    def split(n, p):
        sizes = [n // p + (1 if r < n % p else 0) for r in range(p)]
        return [(sum(sizes[:r]), sizes[r]) for r in range(p)]
    Rg = np.full((ny, nx, nv), np.nan)
    dts = []
    for ys, ym in split(ny, py):
        for xs, xm in split(nx, px):
            loc = _local_arrays(Ug, ys, ym, xs, xm, perx, pery)
            h = ctypes.c_void_p()
            st = L.hype_create_block(ctypes.byref(pc.c_struct()), xs, xm, ys, ym, ctypes.byref(h))
            assert st == hp.OK, L.hype_last_error(h)
            Rr = np.empty(ym * xm * nv)
            dt = ctypes.c_double()
            base = loc.ctypes.data + ((3 * (xm + 6) + 3) * nv) * 8
            st = L.hype_rhs_prim_slab(h, 0.0, base, (xm + 6) * nv, Rr.ctypes.data_as(DP), ctypes.byref(dt))
            L.hype_destroy(h)
            assert st == hp.OK
            Rg[ys:ys + ym, xs:xs + xm] = Rr.reshape(ym, xm, nv)
            dts.append(dt.value)
    assert Rg.reshape(-1).tobytes() == Ro.tobytes()
    assert min(dts) == dto
