"""Batched instances (include/hype_batch.h) against lone solvers.

Every instance of a batch must produce exactly what a lone ``Solver`` of the
same configuration produces from the same state with the same time-loop
limits -- bit for bit, whatever else shares the batch, whichever tile shape
the persistent launches use, and whenever the instance joined.  The lone FP64
solver is itself bit-identical to the reference (test_gpu_parity.py).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def kapila(hp, nx, ny, order=2, bcs=None, **kw):
    T, R, P = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE, hp.BC_PERIODIC
    bcs = bcs or (T, T, R, R)
    return hp.Config(system=hp.KAPILA_5EQN, order=order, nx=nx, ny=ny, cfl=0.4, bc_left=bcs[0], bc_right=bcs[1],
                     bc_bottom=bcs[2], bc_top=bcs[3], **kw)


def lone(hp, cfg, U0, t0, tf, nmax):
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        k, t, dtn, st = s.solve(t0, tf, nmax, check=False)
        return s.get_state(), k, t, st


def check_same(hp, b, i, cfg, U0, t0, tf, nmax):
    U, k, t, st = lone(hp, cfg, U0, t0, tf, nmax)
    s = b.status(i)
    assert s["status"] == st, (i, s, st)
    if st != hp.OK:
        return
    assert s["done"] == 1 and s["steps"] == k and s["t"] == t, (i, s, k, t)
    Ub = b.get_state(i)
    assert Ub.tobytes() == U.tobytes(), (i, cfg.nx, cfg.ny, float(np.abs(Ub - U).max()))


def test_uneven_kapila_grids_match_lone_runs(hp):
    T, R, P = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE, hp.BC_PERIODIC
    specs = [(96, 80, (T, T, R, R), 1), (130, 64, (T, T, T, T), 2), (200, 150, (P, P, R, R), 3),
             (64, 72, (R, R, P, P), 0), (257, 33, (T, R, T, R), 4)]
    runs = []
    with hp.Batch(max_instances=8) as b:
        for n, (nx, ny, bcs, nb) in enumerate(specs):
            cfg = kapila(hp, nx, ny, bcs=bcs)
            U0 = hp.initial_state(cfg, "shock_bubble", seed=40 + n, nbubbles=nb)
            i = b.add(cfg, U0, 0.0, 1e30, 12)
            runs.append((i, cfg, U0))
        b.advance(15)   # three replays past every instance's max_steps
        b.sync()
        for i, cfg, U0 in runs:
            check_same(hp, b, i, cfg, U0, 0.0, 1e30, 12)


def test_mixed_kinds_in_one_batch(hp):
    """FP64 Kapila N = 0..3 (forward Euler copy-back, SSPRK(10,4) included), an
    inlet Kapila grid, Baer-Nunziato, Euler and the mixed-precision form, all on
    parallel branches of one step graph."""
    T, R, P = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE, hp.BC_PERIODIC
    items = []
    for order, (nx, ny) in zip(range(4), ((70, 40), (88, 64), (120, 90), (48, 40))):
        c = kapila(hp, nx, ny, order=order)
        items.append((c, hp.initial_state(c, "shock_bubble", seed=50 + order, nbubbles=1), 1e30, 6))
    ci = kapila(hp, 80, 60, bcs=(hp.BC_INLET, T, R, R), y_min=-2.0, y_max=2.0, x_max=4.0 / 3.0)
    items.append((ci, hp.initial_state(ci, "shock_bubble", seed=55, nbubbles=1), 1e30, 5))
    cb = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=72, ny=64, cfl=0.4, bc_left=T, bc_right=T, bc_bottom=R, bc_top=R,
                   gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    items.append((cb, hp.initial_state(cb, "bn_discs", seed=56), 1e30, 5))
    ce = hp.Config(system=hp.EULER, order=1, nx=100, ny=70, cfl=0.4, bc_left=T, bc_right=T, bc_bottom=T, bc_top=T,
                   gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    items.append((ce, hp.initial_state(ce, "euler_quadrants", seed=57), 0.05, 1000))
    cm = kapila(hp, 150, 110, precision=hp.PREC_MIXED)
    items.append((cm, hp.initial_state(cm, "shock_bubble", seed=58, nbubbles=2), 1e30, 8))
    with hp.Batch(max_instances=16) as b:
        ids = [b.add(c, U0, 0.0, tf, nmax) for c, U0, tf, nmax in items]
        for _ in range(40):
            b.advance(10)
            b.sync()
            if all(b.status(i)["done"] for i in ids):
                break
        for i, (c, U0, tf, nmax) in zip(ids, items):
            check_same(hp, b, i, c, U0, 0.0, tf, nmax)


def test_continuous_joins_and_leaves(hp):
    """Instances join between steps, one leaves before finishing and its slot is
    reused: the others' results do not change."""
    cfgs = [kapila(hp, 90 + 10 * k, 70 + 6 * k) for k in range(4)]
    U = [hp.initial_state(c, "shock_bubble", seed=60 + k, nbubbles=1 + k % 2) for k, c in enumerate(cfgs)]
    with hp.Batch(max_instances=3) as b:
        a = b.add(cfgs[0], U[0], 0.0, 1e30, 20)
        b.advance(7)
        bb = b.add(cfgs[1], U[1], 0.0, 1e30, 15)
        b.advance(10)
        b.sync()
        assert b.status(a)["steps"] == 17 and b.status(bb)["steps"] == 10
        b.remove(a)
        c = b.add(cfgs[2], U[2], 0.0, 1e30, 8)
        d = b.add(cfgs[3], U[3], 0.0, 1e30, 11)
        assert a in (c, d)   # the freed slot is reused
        b.advance(20)
        b.sync()
        for i, k, n in ((bb, 1, 15), (c, 2, 8), (d, 3, 11)):
            check_same(hp, b, i, cfgs[k], U[k], 0.0, 1e30, n)


def test_admission_budget_and_slots(hp):
    c = kapila(hp, 128, 128)
    U0 = hp.initial_state(c, "shock_bubble", seed=1, nbubbles=1)
    per = hp.Batch.instance_bytes(c)
    assert per == 3 * 128 * 128 * 6 * 8
    with hp.Batch(max_instances=8, hbm_budget=2 * per + per // 2) as b:
        b.add(c, U0, 0.0, 1e30, 2)
        b.add(c, U0, 0.0, 1e30, 2)
        st, _ = b.try_add(c, U0, 0.0, 1e30, 2)
        assert st == hp.ERR_NOMEM
        assert b.info()["instances"] == 2 and b.info()["bytes_in_use"] == 2 * per
    with hp.Batch(max_instances=1) as b:
        b.add(c, U0, 0.0, 1e30, 2)
        st, _ = b.try_add(c, U0, 0.0, 1e30, 2)
        assert st == hp.ERR_BUSY
    with hp.Batch(max_instances=2, max_cells=100 * 100) as b:
        with pytest.raises(hp.HypeError) as ei:
            b.add(c, U0, 0.0, 1e30, 2)
        assert ei.value.status == hp.ERR_INVALID


@pytest.mark.parametrize("prec", [0, 1])
def test_tile_shapes_and_autotune_do_not_change_results(hp, prec):
    cfgs = [kapila(hp, nx, ny, precision=prec) for nx, ny in ((300, 120), (140, 200), (77, 64))]
    U = [hp.initial_state(c, "shock_bubble", seed=70 + k, nbubbles=2) for k, c in enumerate(cfgs)]
    outs = []
    for tiling in ((64, 16), (128, 128), (128, 40), "auto"):
        with hp.Batch(max_instances=4) as b:
            ids = [b.add(c, u, 0.0, 1e30, 6) for c, u in zip(cfgs, U)]
            if tiling == "auto":
                cells, rows = b.autotune(2)
                assert cells in (64, 128) and rows in (16, 32, 64, 128)
            else:
                b.set_tiling(*tiling)
            b.advance(6)
            b.sync()
            outs.append([b.get_state(i).tobytes() for i in ids])
    for o in outs[1:]:
        assert o == outs[0]


def test_inadmissible_instance_stops_alone(hp):
    """A grid whose face states fail the admissibility test stops with
    HYPE_ERR_INADMISSIBLE; the other instances are unaffected."""
    import cases
    import oracle as O
    R = O.REFLECTIVE
    ocfg = O.Config(system=O.KAPILA, order=1, nx=24, ny=20, bc_left=R, bc_right=R, bc_bottom=R, bc_top=R, **cases.KAPILA_EOS)
    bad_cfg, bad_U = cases.to_pkg(ocfg), cases.state(ocfg, "rough", 13)
    good = kapila(hp, 100, 80)
    Ug = hp.initial_state(good, "shock_bubble", seed=80, nbubbles=1)
    with hp.Batch(max_instances=4) as b:
        ib = b.add(bad_cfg, bad_U, 0.0, 1.0, 6)
        ig = b.add(good, Ug, 0.0, 1e30, 9)
        b.advance(12)
        b.sync()
        assert b.status(ib)["status"] == hp.ERR_INADMISSIBLE and b.status(ib)["done"] == 1
        check_same(hp, b, ig, good, Ug, 0.0, 1e30, 9)


def test_held_instance_waits_and_resumes_unchanged(hp):
    """A held instance takes no steps (its state and time loop stay as they
    are) and, once released, ends exactly as a lone run."""
    ca, cb = kapila(hp, 120, 90), kapila(hp, 90, 70)
    Ua = hp.initial_state(ca, "shock_bubble", seed=90, nbubbles=2)
    Ub = hp.initial_state(cb, "shock_bubble", seed=91, nbubbles=1)
    with hp.Batch(max_instances=4) as b:
        a = b.add(ca, Ua, 0.0, 1e30, 10)
        i = b.add(cb, Ub, 0.0, 1e30, 10)
        b.advance(4)
        b.sync()
        b.hold(a)
        b.advance(5)
        b.sync()
        assert b.status(a)["steps"] == 4 and b.status(a)["held"] == 1
        assert b.status(i)["steps"] == 9
        U_mid = b.get_state(a)
        b.advance(3)
        b.sync()
        assert b.get_state(a).tobytes() == U_mid.tobytes() and b.status(a)["steps"] == 4
        b.hold(a, False)
        b.advance(8)
        b.sync()
        check_same(hp, b, a, ca, Ua, 0.0, 1e30, 10)
        check_same(hp, b, i, cb, Ub, 0.0, 1e30, 10)


def test_substeps_take_several_exact_steps_per_batch_step(hp):
    """An instance with substeps k takes k of its own steps per batch step and
    still stops exactly at its max_steps / t_final; results are a lone run's."""
    cs = [kapila(hp, 60, 50), kapila(hp, 150, 100), kapila(hp, 70, 64, precision=hp.PREC_MIXED)]
    U = [hp.initial_state(c, "shock_bubble", seed=95 + k, nbubbles=1) for k, c in enumerate(cs)]
    ce = hp.Config(system=hp.EULER, order=2, nx=40, ny=40, cfl=0.4, gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
    Ue = hp.initial_state(ce, "euler_quadrants", seed=99)
    with hp.Batch(max_instances=8) as b:
        a = b.add(cs[0], U[0], 0.0, 1e30, 23)
        c = b.add(cs[1], U[1], 0.0, 1e30, 6)
        m = b.add(cs[2], U[2], 0.0, 1e30, 13)
        e = b.add(ce, Ue, 0.0, 0.02, 100000)
        b.set_substeps(a, 4)
        b.set_substeps(m, 3)
        b.set_substeps(e, 16)
        b.advance(2)
        b.sync()
        assert b.status(a)["steps"] == 8 and b.status(c)["steps"] == 2 and b.status(m)["steps"] == 6
        assert b.status(a)["substeps"] == 4
        b.advance(6)
        b.sync()
        check_same(hp, b, a, cs[0], U[0], 0.0, 1e30, 23)
        check_same(hp, b, c, cs[1], U[1], 0.0, 1e30, 6)
        check_same(hp, b, m, cs[2], U[2], 0.0, 1e30, 13)
        check_same(hp, b, e, ce, Ue, 0.0, 0.02, 100000)


def test_conservative_and_viscous_kinds_in_one_batch(hp):
    """The conservative path (RHSFunction) and the VISCOUS build as batch kinds,
    beside primitive-path and mixed instances: each equals its lone solver bit
    for bit (the lone solvers are pinned to the reference in test_gpu_parity.py),
    with the viscous dt term carried per instance; a tile-shape change keeps them."""
    T, R, P, I = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE, hp.BC_PERIODIC, hp.BC_INLET
    CONS, VISC = hp.FLAG_CONSERVATIVE, hp.FLAG_VISCOUS
    specs = [
        (kapila(hp, 90, 70, flags=CONS), "shock_bubble"),
        (kapila(hp, 64, 50, order=3, bcs=(T, T, P, P), flags=CONS), "shock_bubble"),
        (kapila(hp, 60, 44, order=1, flags=VISC, mu1=0.4, mu2=0.05), "shock_bubble"),
        (kapila(hp, 80, 64, order=2, bcs=(R, R, R, R), flags=VISC | CONS, mu1=0.2), "shock_bubble"),
        (kapila(hp, 50, 48, order=3, bcs=(T, R, P, P), flags=VISC, mu1=1.0, mu2=0.3), "shock_bubble"),
        (kapila(hp, 72, 40, bcs=(I, T, R, R), flags=CONS, x_min=0.0, x_max=2.0, y_min=-1.0, y_max=1.0), "shock_bubble"),
        (hp.Config(system=hp.EULER, order=2, nx=70, ny=60, cfl=0.4, gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0, flags=CONS),
         "euler_quadrants"),
        (hp.Config(system=hp.BAER_NUNZIATO, order=1, nx=56, ny=56, cfl=0.4, flags=CONS | hp.FLAG_BN_FIX_P2), "bn_discs"),
        (kapila(hp, 100, 60), "shock_bubble"),
        (kapila(hp, 96, 64, precision=hp.PREC_MIXED), "shock_bubble"),
    ]
    runs = []
    with hp.Batch(max_instances=16) as b:
        for n, (cfg, ic) in enumerate(specs):
            U0 = hp.initial_state(cfg, ic, seed=300 + n, **({"nbubbles": 2} if ic == "shock_bubble" else {}))
            i = b.add(cfg, U0, 0.0, 1e30, 8)
            runs.append((i, cfg, U0))
        b.advance(4)
        b.set_tiling(64, 32)       # the conservative and viscous kinds keep 128-column tiles
        b.advance(6)
        b.sync()
        for i, cfg, U0 in runs:
            check_same(hp, b, i, cfg, U0, 0.0, 1e30, 8)
    for cfg, _ in specs[:6]:
        assert hp.Batch.instance_bytes(cfg) > 0
