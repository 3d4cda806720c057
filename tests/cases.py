"""Seeded parity cases shared by the CPU pin tests, the GPU parity tests and the
golden-fixture generator (tests/golden/make_golden.py).

Each case is (name, oracle.Config, state builder).  States come either from the
library's own seeded generators (host code, no GPU needed) or from the rough
numpy fields below, which are built to make the reconstruction's admissibility
check fail in some cells (sharp volume-fraction steps, strong pressure jumps)
so the minmod fallback of rhs_function_prim.c:407-421 is exercised.
"""
from __future__ import annotations

import dataclasses
import sys

import numpy as np

import oracle as O

hp = sys.modules["hype_parallel_b200"]

KAPILA_EOS = dict(gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)
EULER_EOS = dict(gamma1=1.4, gamma2=1.4, pi1=0.0, pi2=0.0)


def to_pkg(cfg: O.Config) -> "hp.Config":
    return hp.Config(system=cfg.system, order=cfg.order, nx=cfg.nx, ny=cfg.ny, x_min=cfg.x_min, x_max=cfg.x_max,
                     y_min=cfg.y_min, y_max=cfg.y_max, cfl=cfg.cfl, bc_left=cfg.bc_left, bc_right=cfg.bc_right,
                     bc_bottom=cfg.bc_bottom, bc_top=cfg.bc_top, gamma1=cfg.gamma1, gamma2=cfg.gamma2, pi1=cfg.pi1,
                     pi2=cfg.pi2, precision=hp.PREC_FP64,
                     flags=(hp.FLAG_BN_FIX_P2 if cfg.bn_fixed_p2 else 0) | (hp.FLAG_CONSERVATIVE if cfg.conservative else 0)
                     | (hp.FLAG_VISCOUS if cfg.viscous else 0), mu1=cfg.mu1, mu2=cfg.mu2)


def kapila_rough(cfg: O.Config, seed: int) -> np.ndarray:
    """Two-phase Kapila field with one-cell alpha steps and a pressure jump."""
    rng = np.random.default_rng(seed)
    nx, ny = cfg.nx, cfg.ny
    X, Y = np.meshgrid((np.arange(nx) + 0.5) / nx, (np.arange(ny) + 0.5) / ny)
    eps = 1e-6
    a = np.full(X.shape, 1 - eps)
    for _ in range(3):
        cx, cy, r = rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8), rng.uniform(0.1, 0.3)
        a = np.where(np.hypot(X - cx, Y - cy) < r, eps, a)
    r1 = 1000 * rng.uniform(0.95, 1.05, X.shape)
    r2 = rng.uniform(0.9, 1.1, X.shape)
    u = 20 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    v = -20 * np.cos(2 * np.pi * X) * np.sin(2 * np.pi * Y)
    p = np.where(X < 0.25, 1e6, 1e5) * rng.uniform(0.98, 1.02, X.shape)
    g1, g2, pi1, pi2 = cfg.gamma1, cfg.gamma2, cfg.pi1, cfg.pi2
    a2 = 1 - a
    rho = a * r1 + a2 * r2
    G1, G2 = g1 - 1, g2 - 1
    e = (p * (a * G2 + a2 * G1) + a * g1 * pi1 * G2 + a2 * g2 * pi2 * G1) / (G1 * G2)
    E = e + 0.5 * rho * (u * u + v * v)
    return np.ascontiguousarray(np.stack([a * r1, a2 * r2, rho * u, rho * v, E, a], -1).reshape(-1))


def state(cfg: O.Config, kind: str, seed: int) -> np.ndarray:
    if kind == "rough":
        return kapila_rough(cfg, seed)
    pc = to_pkg(cfg)
    if kind == "bubble":
        return hp.initial_state(pc, "shock_bubble", seed=seed, nbubbles=2)
    if kind == "discs":
        return hp.initial_state(pc, "bn_discs", seed=seed)
    if kind == "quadrants":
        return hp.initial_state(pc, "euler_quadrants", seed=seed)
    if kind == "vortex":
        return hp.initial_state(pc, "smooth_vortex")
    raise ValueError(kind)


T, R, P, I = O.TRANSMISSIVE, O.REFLECTIVE, O.PERIODIC, O.INLET


def _k(name, nx, ny, order=2, bcs=(T, T, T, T), kind="bubble", seed=0, **kw):
    cfg = O.Config(system=O.KAPILA, order=order, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                   bc_top=bcs[3], **KAPILA_EOS, **kw)
    return (name, cfg, kind, seed)


def _e(name, nx, ny, order=2, bcs=(T, T, T, T), seed=0, **kw):
    cfg = O.Config(system=O.EULER, order=order, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                   bc_top=bcs[3], **EULER_EOS, **kw)
    return (name, cfg, "quadrants", seed)


def _b(name, nx, ny, order=2, bcs=(T, T, T, T), seed=0, fixed=0, **kw):
    cfg = O.Config(system=O.BN, order=order, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                   bc_top=bcs[3], bn_fixed_p2=fixed, **KAPILA_EOS, **kw)
    return (name, cfg, "discs", seed)


# RHS parity cases: small enough that the oracle runs them in well under a second
RHS_CASES = [
    _k("kapila_16x16_bubble", 16, 16),
    _k("kapila_37x23_rough_mixed_bc", 37, 23, bcs=(R, T, R, R), kind="rough", seed=1),
    _k("kapila_20x12_periodic_x", 20, 12, bcs=(P, P, T, R), kind="rough", seed=2),
    _k("kapila_24x24_periodic", 24, 24, bcs=(P, P, P, P), seed=3),
    _k("kapila_3x3_min", 3, 3, kind="rough", seed=4),
    _k("kapila_251x7_three_strips", 251, 7, bcs=(R, R, T, T), kind="rough", seed=5),
    _k("kapila_130x9_two_strips", 130, 9, bcs=(T, R, P, P), seed=6),
    _k("kapila_5x67_tall", 5, 67, bcs=(R, R, R, T), kind="rough", seed=7),
    _k("kapila_18x14_inlet", 18, 14, bcs=(I, T, R, R), kind="rough", seed=8, x_min=0.0, x_max=2.0, y_min=-1.0, y_max=0.5556),
    _k("kapila_19x17_N1", 19, 17, order=1, kind="rough", seed=9),
    _k("kapila_15x13_N3", 15, 13, order=3, bcs=(R, T, P, P), kind="rough", seed=10),
    _k("kapila_11x10_N0", 11, 10, order=0, seed=11),
    _e("euler_16x16", 16, 16),
    _e("euler_21x19_reflective_N1", 21, 19, order=1, bcs=(R, R, R, R), seed=1),
    _e("euler_17x12_periodic_N3", 17, 12, order=3, bcs=(P, P, P, P), seed=2),
    _e("euler_9x8_N0", 9, 8, order=0, bcs=(T, R, T, R), seed=3),
    _b("bn_16x16", 16, 16),
    _b("bn_23x19_fixed_p2", 23, 19, fixed=1, bcs=(R, T, R, T), seed=1),
    _b("bn_13x21_periodic_N1", 13, 21, order=1, bcs=(P, P, R, R), seed=2),
    _b("bn_12x10_N3", 12, 10, order=3, seed=3),
    # conservative-variable path (RHSFunction, rhs_function.c)
    _k("kapila_cons_24x20_bubble", 24, 20, bcs=(T, T, R, R), seed=20, conservative=1),
    _k("kapila_cons_37x23_rough", 37, 23, bcs=(R, T, R, R), kind="rough", seed=21, conservative=1),
    _k("kapila_cons_18x14_inlet", 18, 14, bcs=(I, T, R, R), kind="rough", seed=22, x_min=0.0, x_max=2.0, y_min=-1.0,
       y_max=0.5556, conservative=1),
    _k("kapila_cons_19x17_N1", 19, 17, order=1, kind="rough", seed=23, conservative=1),
    _k("kapila_cons_15x13_N3", 15, 13, order=3, bcs=(R, T, P, P), seed=24, conservative=1),
    _k("kapila_cons_11x10_N0", 11, 10, order=0, seed=25, conservative=1),
    _k("kapila_cons_251x7_three_strips", 251, 7, bcs=(R, R, T, T), seed=26, conservative=1),
    _e("euler_cons_21x19_reflective", 21, 19, bcs=(R, R, R, R), seed=27, conservative=1),
    _e("euler_cons_17x12_periodic_N3", 17, 12, order=3, bcs=(P, P, P, P), seed=28, conservative=1),
    _e("euler_cons_16x16_N1", 16, 16, order=1, seed=29, conservative=1),
    _b("bn_cons_16x16", 16, 16, seed=30, conservative=1),
    _b("bn_cons_13x21_periodic_N1", 13, 21, order=1, bcs=(P, P, R, R), seed=31, conservative=1),
    _b("bn_cons_12x10_N3", 12, 10, order=3, bcs=(R, R, T, T), seed=32, conservative=1),
    # the reference's VISCOUS build (Kapila, N >= 1)
    _k("kapila_visc_24x20_walls", 24, 20, bcs=(R, R, R, R), seed=40, viscous=1, mu1=0.3, mu2=0.05),
    _k("kapila_visc_37x23_rough", 37, 23, bcs=(R, T, R, R), kind="rough", seed=41, viscous=1, mu1=0.05, mu2=0.01),
    _k("kapila_visc_19x17_N1", 19, 17, order=1, bcs=(T, T, P, P), kind="rough", seed=42, viscous=1),
    _k("kapila_visc_15x13_N3", 15, 13, order=3, bcs=(R, T, P, P), seed=43, viscous=1, mu1=2.0, mu2=0.5),
    _k("kapila_visc_18x14_inlet", 18, 14, bcs=(I, T, R, R), kind="rough", seed=44, x_min=0.0, x_max=2.0, y_min=-1.0,
       y_max=0.5556, viscous=1, mu1=0.1),
    _k("kapila_visc_251x7_three_strips", 251, 7, bcs=(R, R, T, T), seed=45, viscous=1, mu1=0.2, mu2=0.02),
    _k("kapila_visc_cons_24x20_walls", 24, 20, bcs=(R, R, R, R), seed=46, conservative=1, viscous=1, mu1=0.3, mu2=0.05),
    _k("kapila_visc_cons_19x17_N1", 19, 17, order=1, kind="rough", seed=47, conservative=1, viscous=1),
    _k("kapila_visc_cons_15x13_N3", 15, 13, order=3, bcs=(R, T, P, P), seed=48, conservative=1, viscous=1, mu1=2.0, mu2=0.5),
]

# Multi-step solve cases (hype.c time loop)
SOLVE_CASES = [
    (_k("kapila_32x32_bubble_solve", 32, 32, seed=12), 0.0, 1.0, 8),
    (_k("kapila_24x20_rough_solve_N1", 24, 20, order=1, bcs=(R, R, R, R), kind="rough", seed=13), 0.0, 1.0, 6),
    (_k("kapila_24x20_bubble_solve_N1", 24, 20, order=1, bcs=(R, R, R, R), seed=17), 0.0, 1.0, 6),
    (_k("kapila_16x16_solve_N3", 16, 16, order=3, bcs=(P, P, P, P), seed=14), 0.0, 1.0, 3),
    (_e("euler_32x24_solve", 32, 24, bcs=(T, T, R, R), seed=15), 0.0, 0.05, 1000),
    (_b("bn_20x20_solve", 20, 20, seed=16), 0.0, 1.0, 4),
    (_k("kapila_cons_32x32_solve", 32, 32, seed=33, conservative=1), 0.0, 1.0, 8),
    (_e("euler_cons_32x24_solve", 32, 24, bcs=(T, T, R, R), seed=34, conservative=1), 0.0, 0.05, 1000),
    (_b("bn_cons_20x20_solve", 20, 20, bcs=(R, R, R, R), seed=35, conservative=1), 0.0, 1.0, 4),
    (_k("kapila_visc_32x32_solve", 32, 32, bcs=(T, T, R, R), seed=49, viscous=1, mu1=0.5, mu2=0.1), 0.0, 1.0, 6),
    (_k("kapila_visc_cons_24x24_solve", 24, 24, bcs=(P, P, P, P), seed=50, conservative=1, viscous=1, mu1=0.5), 0.0, 1.0, 4),
]


def case_by_name(name: str):
    for c in RHS_CASES:
        if c[0] == name:
            return c
    for c in SOLVE_CASES:
        if c[0][0] == name:
            return c
    raise KeyError(name)


def config_to_dict(cfg: O.Config) -> dict:
    return dataclasses.asdict(cfg)
