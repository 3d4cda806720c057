"""End-to-end pins of the benchmark configurations against the reference's own
multi-step runs (tests/golden/config_runs.json, made from oracle/_ref by
tests/golden/make_golden_configs.py).

* Kapila 256^2, 1 bubble, 100 SSPRK(4,3) steps (the reference's CPU-runnable
  configuration): final state, step count, t and dt bit for bit, and after every
  step the extremes of alpha_1 and the cells where they sit.  The reference
  itself takes alpha_1 past 1 - 1e-6 at the shock from the first step on (it
  keeps alpha_1 in [0, 1] only, through its admissibility check,
  kapila_5eqn.c:450-479, and has no clipping); the GPU path leaves the band
  [1e-6, 1 - 1e-6] at the same step, in the same cell, with the same value.
* The 2048^2 benchmark workload (4 bubbles, seed 0): 10 steps bit for bit
  against the reference run as 8 live MPI ranks.
* Baer-Nunziato discs, the reference's flux form (phase-2 pressure V[8],
  baer_nunziato.c:271): at 128^2 and at 1024^2 (the Baer-Nunziato benchmark
  grid) the state after 20 / 10 steps bit for bit, and the run stops with
  HYPE_ERR_INADMISSIBLE at the step where the reference calls MPI_Abort.
* Baer-Nunziato 128^2 with the phase-2 pressure V[7]: 40 steps bit for bit
  against the oracle (the reference has only its own form).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "config_runs.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def setup(g):
    cfg = O.Config(**g["config"])
    if g["ic"] == "shock_bubble":
        U = O.initial_state(cfg, "shock_bubble", seed=g["seed"], nbubbles=g["nbubbles"])
    else:
        U = O.initial_state(cfg, g["ic"], seed=g["seed"])
    assert sha(U) == g["sha_U0"]
    return cfg, U


def test_kapila256_100_steps_and_alpha_band(hp):
    g = GOLD["kapila256_cfg0"]
    cfg, U = setup(g)
    eps = g["eps"]
    first_out = None
    with hp.Solver(cases.to_pkg(cfg)) as s:
        s.set_state(U)
        s.begin(0.0, 1e30, g["steps"])
        for k in range(1, g["steps"] + 1):
            s.advance(1)
            n, t, dt, st = s.wait()
            assert st == hp.OK and n == k
            a = s.get_state().reshape(-1, 6)[:, 5]
            lo, hi = int(np.argmin(a)), int(np.argmax(a))
            assert [float(a[lo]).hex(), lo, float(a[hi]).hex(), hi] == g["alpha_extremes_per_step"][k - 1], f"step {k}"
            assert 0.0 <= a[lo] and a[hi] <= 1.0
            if first_out is None and (a[lo] < eps or a[hi] > 1 - eps):
                cell = lo if a[lo] < eps else hi
                first_out = {"step": k, "cell": cell, "alpha1": float(a[cell]).hex(), "side": "low" if a[lo] < eps else "high"}
        Ue = s.get_state()
    assert first_out == g["first_step_outside_eps_band"]
    assert float(t).hex() == g["t_end"] and float(dt).hex() == g["dt_next"]
    assert sha(Ue) == g["sha_U_end"]


def test_headline_2048_workload_10_steps(hp):
    g = GOLD["kapila2048_headline"]
    cfg, U = setup(g)
    with hp.Solver(cases.to_pkg(cfg)) as s:
        s.set_state(U)
        n, t, dt, st = s.solve(0.0, 1e30, g["steps"])
        Ue = s.get_state()
    assert st == hp.OK and n == g["steps"]
    assert float(t).hex() == g["t_end"] and float(dt).hex() == g["dt_next"]
    a = Ue.reshape(-1, 6)[:, 5]
    assert float(a.min()).hex() == g["alpha_min"] and float(a.max()).hex() == g["alpha_max"]
    assert sha(Ue) == g["sha_U_end"]


@pytest.mark.parametrize("name", ["bn128_reference_form", "bn1024_reference_form"])
def test_bn_reference_form_stops_where_the_reference_aborts(hp, name):
    g = GOLD[name]
    cfg, U = setup(g)
    keep = g["state_at"]
    with hp.Solver(cases.to_pkg(cfg)) as s:
        s.set_state(U)
        s.begin(0.0, 1e30, 1 << 30)
        s.advance(keep["step"])
        n, t, dt, st = s.wait()
        assert st == hp.OK and n == keep["step"]
        assert float(t).hex() == keep["t"] and float(dt).hex() == keep["dt_next"]
        assert sha(s.get_state()) == keep["sha_U"]
        s.advance(g["failing_step"] + 5 - keep["step"])
        n, t, dt, st = s.wait()
    # the step counter includes the step whose RHS raised the error; the run stops there
    assert st == hp.ERR_INADMISSIBLE
    assert n == g["failing_step"] == g["completed_steps"] + 1
    assert t > float.fromhex(g["t_before_failure"])


def test_bn128_fixed_form_40_steps(hp):
    g = GOLD["bn128_fixed_p2"]
    cfg, U = setup(g)
    with hp.Solver(cases.to_pkg(cfg)) as s:
        s.set_state(U)
        n, t, dt, st = s.solve(0.0, 1e30, g["steps"])
        Ue = s.get_state()
    assert st == hp.OK and n == g["steps"]
    assert float(t).hex() == g["t_end"] and float(dt).hex() == g["dt_next"]
    assert sha(Ue) == g["sha_U_end"]
