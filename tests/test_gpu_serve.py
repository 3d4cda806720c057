"""The request loop (include/hype_serve.h) under continuous batching.

The central check: every request's result is the same -- bit for bit, for
the FP64 and the mixed-precision forms alike -- when it is served alone,
when it is served in a mix of Euler, Kapila and Baer-Nunziato requests that
arrive while others are on the GPU and wait for HBM budget, and when it is
solved by a lone Solver.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_trace(hp, n, seed, spacing_s):
    rng = np.random.default_rng(seed)
    T, R = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE
    reqs = []
    t = 0.0
    for i in range(n):
        u = rng.uniform()
        nx, ny = int(rng.integers(40, 180)), int(rng.integers(40, 180))
        steps = int(rng.integers(5, 40))
        if u < 0.5:
            prec = hp.PREC_MIXED if rng.uniform() < 0.4 else hp.PREC_FP64
            cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=nx, ny=ny, cfl=0.4, bc_left=T, bc_right=T, bc_bottom=R,
                            bc_top=R, precision=prec)
            r = hp.Request(t, cfg, max_steps=steps, ic=hp.IC_SHOCK_BUBBLE, ic_seed=1000 + i, ic_param=int(rng.integers(1, 5)))
        elif u < 0.8:
            # phase-2 flux pressure from V[7]: as written (V[8], baer_nunziato.c:271) these states abort within ~50 steps
            cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=nx, ny=ny, cfl=0.4, bc_left=T, bc_right=T, bc_bottom=T,
                            bc_top=T, flags=hp.FLAG_BN_FIX_P2)
            r = hp.Request(t, cfg, max_steps=steps, ic=hp.IC_BN_DISCS, ic_seed=2000 + i)
        else:
            cfg = hp.Config(system=hp.EULER, order=int(rng.integers(1, 3)), nx=nx, ny=ny, cfl=0.4, bc_left=T, bc_right=T,
                            bc_bottom=T, bc_top=T, gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)
            # end time instead of a step count: the run stops at t_final (MATCHSTEP)
            r = hp.Request(t, cfg, t_final=0.02 + 0.01 * rng.uniform(), max_steps=100000, ic=hp.IC_EULER_QUADRANTS,
                           ic_seed=3000 + i)
        reqs.append(r)
        t += rng.exponential(spacing_s)
    return reqs


def initial(hp, r):
    kind = {hp.IC_SHOCK_BUBBLE: "shock_bubble", hp.IC_BN_DISCS: "bn_discs", hp.IC_EULER_QUADRANTS: "euler_quadrants"}[r.ic]
    return hp.initial_state(r.cfg, kind, seed=r.ic_seed, nbubbles=r.ic_param)


def collect(hp, reqs, **kw):
    out = {}
    res, stats = hp.serve(reqs, sink=lambda i, U, rr: out.__setitem__(i, (U, rr)), **kw)
    return res, stats, out


@pytest.mark.parametrize("active_cells,substep_cells", [(0, 0), (20000, 0), (0, 1 << 20)])
def test_each_result_same_alone_and_in_the_mix(hp, active_cells, substep_cells):
    """active_cells 0: every resident request steps; 20000: the scheduler holds
    all but the least-remaining-work requests (a few grids' worth of cells);
    substep_cells 2^20: these small grids take 16 steps per batch step."""
    reqs = make_trace(hp, 24, seed=5, spacing_s=0.004)
    sizes = [hp.Batch.instance_bytes(r.cfg) for r in reqs]
    budget = 3 * max(sizes)   # forces waiting for memory
    res, stats, mixed = collect(hp, reqs, hbm_budget=budget, max_instances=8, poll_ms=2.0, active_cells=active_cells,
                                substep_cells=substep_cells)
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    assert stats["peak_bytes"] <= budget and stats["peak_instances"] <= 8
    assert stats["peak_instances"] >= 2          # requests overlapped on the device
    assert 0 < stats["p50_s"] <= stats["p90_s"] <= stats["p99_s"] <= stats["max_s"]
    assert stats["cell_updates"] == sum(r.cfg.nx * r.cfg.ny * res[i]["steps"] for i, r in enumerate(reqs))
    for i, r in enumerate(reqs):
        # served alone
        res1, _, alone = collect(hp, [hp.Request(0.0, r.cfg, r.t0, r.t_final, r.max_steps, r.ic, r.ic_seed, r.ic_param)])
        assert res1[0]["status"] == hp.OK
        U_mix, rr = mixed[i]
        U_alone, ra = alone[0]
        assert (rr["steps"], rr["t_end"]) == (ra["steps"], ra["t_end"]), i
        assert U_mix.tobytes() == U_alone.tobytes(), (i, float(np.abs(U_mix - U_alone).max()))
        # and by a lone solver (for FP64 requests this is the reference's arithmetic)
        if i % 3 == 0:
            with hp.Solver(r.cfg) as s:
                s.set_state(initial(hp, r))
                k, t, _, st = s.solve(r.t0, r.t_final, r.max_steps)
                assert st == hp.OK and (k, t) == (rr["steps"], rr["t_end"])
                assert s.get_state().tobytes() == U_mix.tobytes(), i


def test_queued_at_start_and_fifo_admission(hp):
    reqs = make_trace(hp, 12, seed=6, spacing_s=0.0)
    res, stats, _ = collect(hp, reqs, realtime=False, max_instances=4, autotune=False)
    assert stats["completed"] == 12 and stats["peak_instances"] == 4
    admits = [r["admit_s"] for r in res]
    assert admits == sorted(admits)   # arrival order
    for r in res:
        assert r["latency_s"] == r["done_s"] >= r["admit_s"] >= 0.0


def test_rejections_do_not_disturb_the_rest(hp):
    reqs = make_trace(hp, 6, seed=7, spacing_s=0.001)
    bad = hp.Config(system=hp.KAPILA_5EQN, nx=2, ny=2)                       # invalid grid
    big = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=400, ny=400, cfl=0.4)  # never fits the budget
    reqs.insert(2, hp.Request(reqs[1].arrival_s, bad, max_steps=3))
    reqs.insert(4, hp.Request(reqs[3].arrival_s, big, max_steps=3))
    budget = 2 * max(hp.Batch.instance_bytes(r.cfg) for r in reqs if r.cfg.nx < 300)
    res, stats, out = collect(hp, reqs, hbm_budget=budget)
    assert res[2]["status"] == hp.ERR_INVALID and res[4]["status"] == hp.ERR_NOMEM
    assert stats["failed"] == 2 and stats["completed"] == len(reqs) - 2
    assert all(res[i]["status"] == hp.OK for i in range(len(reqs)) if i not in (2, 4))


def test_callback_initial_state(hp):
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=64, ny=48, cfl=0.4)
    U0 = hp.initial_state(cfg, "shock_bubble", seed=9, nbubbles=2)
    reqs = [hp.Request(0.0, cfg, max_steps=7, ic=hp.IC_CALLBACK)]
    out = {}
    res, _ = hp.serve(reqs, fill=lambda i, U: U.__setitem__(slice(None), U0), sink=lambda i, U, r: out.__setitem__(i, U))
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        s.solve(0.0, 1e30, 7)
        assert s.get_state().tobytes() == out[0].tobytes()


def test_conservative_and_viscous_requests(hp):
    """Requests for the conservative path and the VISCOUS build are served beside
    primitive-path ones; each result equals a lone solver's bit for bit."""
    T, R = hp.BC_TRANSMISSIVE, hp.BC_REFLECTIVE
    CONS, VISC = hp.FLAG_CONSERVATIVE, hp.FLAG_VISCOUS
    cfgs = [hp.Config(system=hp.KAPILA_5EQN, order=2, nx=70, ny=60, cfl=0.4, bc_bottom=R, bc_top=R, flags=VISC, mu1=0.3),
            hp.Config(system=hp.KAPILA_5EQN, order=2, nx=64, ny=64, cfl=0.4, flags=CONS),
            hp.Config(system=hp.KAPILA_5EQN, order=1, nx=80, ny=40, cfl=0.4, flags=VISC | CONS, mu1=0.1, mu2=0.02),
            hp.Config(system=hp.KAPILA_5EQN, order=2, nx=90, ny=50, cfl=0.4),
            hp.Config(system=hp.EULER, order=2, nx=60, ny=60, cfl=0.4, gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0, flags=CONS)]
    reqs = []
    for i, c in enumerate(cfgs):
        ic = hp.IC_EULER_QUADRANTS if c.system == hp.EULER else hp.IC_SHOCK_BUBBLE
        reqs.append(hp.Request(0.002 * i, c, max_steps=10 + i, ic=ic, ic_seed=700 + i, ic_param=2))
    res, stats, out = collect(hp, reqs, max_instances=4)
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    for i, r in enumerate(reqs):
        U, rr = out[i]
        with hp.Solver(r.cfg) as s:
            s.set_state(initial(hp, r))
            k, t, _, st = s.solve(r.t0, r.t_final, r.max_steps)
            assert st == hp.OK and (k, t) == (rr["steps"], rr["t_end"]), i
            assert s.get_state().tobytes() == U.tobytes(), i
