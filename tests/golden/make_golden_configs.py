"""Generate tests/golden/config_runs.json: multi-step runs of the benchmark
configurations by the reference's own HyPE-2D sources (oracle/_ref), for the
end-to-end GPU pins in tests/test_gpu_configs.py.

Run in a container that has the reference sources (a few minutes on 8 cores):
    make -C oracle all ref && python tests/golden/make_golden_configs.py

Runs (inputs from the oracle's seeded generators, which tests/test_oracle_ic.py
holds to the library's bits):
  kapila256_cfg0       Kapila 256^2, 1 bubble, seed 0, SSPRK(4,3), CFL 0.4, 100
                       steps; per step the extremes of alpha_1 and their cells
  kapila2048_headline  the benchmark workload (2048^2, 4 bubbles, seed 0), 10
                       steps, run as 8 live MPI ranks (bitwise the one-rank run)
  bn128_reference_form Baer-Nunziato 128^2 discs (seed 0), the reference's flux
                       (phase-2 pressure V[8]), stepped until it aborts
  bn1024_reference_form  the same at 1024^2 (8 live ranks): the state after 10
                       steps and the step where it aborts
  bn128_fixed_p2       Baer-Nunziato 128^2 with the phase-2 pressure V[7], 40
                       steps; the reference has only its own flux, so this one is
                       the oracle's (pinned to the reference by test_oracle_pin.py)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle as O  # noqa: E402

KAP = dict(gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)
EPS = 1e-6


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def cfg_dict(cfg):
    import dataclasses
    return dataclasses.asdict(cfg)


def kapila256():
    cfg = O.Config(system=O.KAPILA, order=2, nx=256, ny=256, cfl=0.4, **KAP)
    U = O.initial_state(cfg, "shock_bubble", seed=0, nbubbles=1)
    ref = O.Reference(O.KAPILA)
    ref.setup(cfg)
    assert ref.begin(U, 0.0, 1e30) == 0
    per_step, first_out = [], None
    for k in range(1, 101):
        n, t, dt, st = ref.advance(1)
        assert st == 0 and n == k
        a = ref.state().reshape(-1, 6)[:, 5]
        lo, hi = int(np.argmin(a)), int(np.argmax(a))
        per_step.append([float(a[lo]).hex(), lo, float(a[hi]).hex(), hi])
        if first_out is None and (a[lo] < EPS or a[hi] > 1 - EPS):
            cell = lo if a[lo] < EPS else hi
            first_out = {"step": k, "cell": cell, "alpha1": float(a[cell]).hex(), "side": "low" if a[lo] < EPS else "high"}
    Ue = ref.state()
    return {"config": cfg_dict(cfg), "ic": "shock_bubble", "seed": 0, "nbubbles": 1, "steps": 100, "sha_U0": sha(U),
            "sha_U_end": sha(Ue), "t_end": float(t).hex(), "dt_next": float(dt).hex(), "alpha_extremes_per_step": per_step,
            "first_step_outside_eps_band": first_out, "eps": EPS, "source": "reference"}


def kapila2048():
    cfg = O.Config(system=O.KAPILA, order=2, nx=2048, ny=2048, cfl=0.4, **KAP)
    U = O.initial_state(cfg, "shock_bubble", seed=0, nbubbles=4)
    with O.LiveReference(cfg, 8) as L:
        Ue, n, t, dt, st = L.solve(U, 0.0, 1e30, 10)
        grid = f"{len({b[0] for b in L.blocks})}x{len({b[1] for b in L.blocks})}"
    assert st == 0 and n == 10
    a = Ue.reshape(-1, 6)[:, 5]
    return {"config": cfg_dict(cfg), "ic": "shock_bubble", "seed": 0, "nbubbles": 4, "steps": 10, "sha_U0": sha(U),
            "sha_U_end": sha(Ue), "t_end": float(t).hex(), "dt_next": float(dt).hex(),
            "alpha_min": float(a.min()).hex(), "alpha_max": float(a.max()).hex(),
            "source": f"reference, 8 live MPI ranks (process grid {grid})"}


def bn_reference_form(n, live, keep_step):
    cfg = O.Config(system=O.BN, order=2, nx=n, ny=n, cfl=0.4, **KAP)
    U = O.initial_state(cfg, "bn_discs", seed=0)
    runner = O.LiveReference(cfg, 8) if live else O.Reference(O.BN)
    try:
        if not live:
            runner.setup(cfg)
        assert runner.begin(U, 0.0, 1e30) == 0
        kept, done, t, dt = None, 0, 0.0, 0.0
        for k in range(1, 1000):
            r = runner.advance(1)
            st = r[3]
            if st != 0:
                break
            done, t, dt = r[0], r[1], r[2]
            if k == keep_step:
                kept = {"step": k, "sha_U": sha(runner.state()), "t": float(t).hex(), "dt_next": float(dt).hex()}
        failing = done + 1
    finally:
        if live:
            runner.close()
    return {"config": cfg_dict(cfg), "ic": "bn_discs", "seed": 0, "sha_U0": sha(U), "completed_steps": done,
            "failing_step": failing, "t_before_failure": float(t).hex(), "state_at": kept,
            "source": "reference" + (", 8 live MPI ranks" if live else "")}


def bn128_fixed():
    cfg = O.Config(system=O.BN, order=2, nx=128, ny=128, cfl=0.4, bn_fixed_p2=1, **KAP)
    U = O.initial_state(cfg, "bn_discs", seed=0)
    Ue, n, t, dt, st = O.Oracle().solve(cfg, U, 0.0, 1e30, 40)
    assert st == 0 and n == 40
    return {"config": cfg_dict(cfg), "ic": "bn_discs", "seed": 0, "steps": 40, "sha_U0": sha(U), "sha_U_end": sha(Ue),
            "t_end": float(t).hex(), "dt_next": float(dt).hex(), "source": "oracle (phase-2 pressure V[7])"}


def main():
    if not O.reference_available():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` where the reference sources exist")
    out = {"generator": "tests/golden/make_golden_configs.py"}
    for name, fn in (("kapila256_cfg0", kapila256), ("bn128_reference_form", lambda: bn_reference_form(128, False, 20)),
                     ("bn128_fixed_p2", bn128_fixed), ("kapila2048_headline", kapila2048),
                     ("bn1024_reference_form", lambda: bn_reference_form(1024, True, 10))):
        t0 = time.time()
        out[name] = fn()
        print(f"{name}: {time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "config_runs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
