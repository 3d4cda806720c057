"""Benchmark of the B200 SSP-RK step (one JSON line on rank 0).

Workload (the plain FP64 drop-in path): Kapila five-equation model,
2048 x 2048 cells on [0,1]^2, transmissive boundaries, stiffened gases
(gamma 4.4 / 1.4, P_inf 6e8 / 0), seeded shock + 4 gas bubbles, WENO N=2,
Rusanov, SSPRK(4,3) (4 RHS evaluations per step), CFL 0.4.  One "step" is one
full SSP-RK step of that grid; the metric is cell-updates per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1: launched with torch.distributed.run, one rank per GPU; the grids are
independent replicas (the path does not shard across GPUs here), so scaling
is weak and no collective touches the data path; timing is the max over ranks.

`--impl reference` times the reference's own HyPE-2D code on the host cores
(oracle/_ref, the unmodified sources compiled against the PETSc stand-in) on
the same 2048 x 2048 workload, as one live MPI rank per host core on the DMDA
split PETSc would choose (the stand-in's shared-memory MPI); its input comes
from the oracle's own generator, so that arm never loads this repository's
library.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "hype-parallel_b200")
METRIC = "cell-updates/s FP64 plain vs mixed+batched at L1<=1e-5; serving p50/p99 latency"
UNIT = "cell-updates/s"
NX = NY = 2048
# Algorithmic FP64 operations of one RHS evaluation of this workload (2048^2 Kapila,
# N = 2, 4-bubble shock-bubble state of seed 0): the reference's arithmetic counted
# operation by operation (oracle/flops.cpp; tests/test_flops.py recounts it):
# 8728100905 additions, 10411302998 multiplications, 894672899 divisions and
# 33570816 square roots, i.e. 4784.5 per cell.
RHS_FLOPS_2048 = 20067647618
# the SSPRK(4,3) combinations per cell: three AXPY stages (1 mul + 1 add per field)
# and the AXPBYPCZ stage (3 mul + 2 add per field), 6 fields
RK_FLOPS_PER_CELL = 3 * 2 * 6 + 5 * 6
# DRAM bytes of one stage-kernel launch on this workload, from an ncu capture of the
# kernel (dram__bytes_read.sum + dram__bytes_write.sum: 210,945,536 + 159,174,656)
STAGE_TRAFFIC_BYTES = 210945536 + 159174656
NBUB = 4
SEED = 0
BYTES_PER_CELL_UPDATE = 9 * 6 * 8    # SSPRK(4,3): 5 state reads + 4 state writes of 6 FP64 fields


def load_pkg():
    if "hype_parallel_b200" in sys.modules:
        return sys.modules["hype_parallel_b200"]
    spec = importlib.util.spec_from_file_location("hype_parallel_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hype_parallel_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline and reference arm: the reference's own code (oracle/_ref) run as
# live MPI ranks on the host cores, on this workload
# ---------------------------------------------------------------------------
def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_run(nranks: int, warmup: int, steps: int, budget_s: float, nx: int = NX, ny: int = NY):
    """The reference's RHSFunctionPrim and hype.c time loop (oracle/_ref: the
    HyPE-2D sources on the PETSc stand-in) on this workload -- the 2048^2
    4-bubble shock-bubble state of seed 0, built by the oracle's own generator --
    as `nranks` live MPI ranks on the DMDA split PETSC_DECIDE gives (what
    `mpiexec -n nranks` runs), halos and the dt reduction through shared memory.
    Times up to `steps` SSP-RK steps after `warmup`, one at a time, stopping once
    `budget_s` seconds of timed steps have passed (at least one step).
    Falls back to the oracle port on one core when oracle/_ref is absent."""
    sys.path.insert(0, ROOT)
    import oracle as O
    cfg = O.Config(system=O.KAPILA, order=2, nx=nx, ny=ny, cfl=0.4)
    U = O.initial_state(cfg, "shock_bubble", seed=SEED, nbubbles=NBUB)
    if not O.reference_available():
        orc = O.Oracle()
        t0 = time.perf_counter()
        _, n, *_ = orc.solve(cfg, U, 0.0, 1e30, 1)
        sec = time.perf_counter() - t0
        return {"value": nx * ny * n / sec, "cores": 1, "kind": "port", "timed_steps": n, "seconds": sec,
                "process_grid": "1x1", "status": 0}
    with O.LiveReference(cfg, nranks) as L:
        st = L.begin(U, 0.0, 1e30)
        if st == 0 and warmup > 0:
            st = L.advance(warmup)[3]
        done, sec = 0, 0.0
        while st == 0 and done < max(1, steps):
            n, _, _, st, s1 = L.advance(1)
            done += 1
            sec += s1
            if sec >= budget_s:
                break
        xs = sorted({b[0] for b in L.blocks})
        ys = sorted({b[1] for b in L.blocks})
    return {"value": nx * ny * done / sec if sec > 0 else None, "cores": nranks, "kind": "reference", "timed_steps": done,
            "seconds": sec, "process_grid": f"{len(xs)}x{len(ys)}", "status": st}


def cpu_baseline(budget_s: float = 20.0):
    """The reference beside the GPU number: the same workload on all host cores,
    a bounded sample (1 warm-up step, then steps until ~budget_s seconds)."""
    cores = host_cores()
    r = reference_run(cores, 1, 1 << 20, budget_s)
    return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
            "sample": f"the 2048x2048 Kapila shock-bubble workload (seed 0, 4 bubbles), {r['timed_steps']} SSPRK(4,3) "
                      f"step(s) after 1 warm-up step, {r['seconds']:.1f} s; oracle/_ref (HyPE-2D's sources on the PETSc "
                      f"stand-in) as {r['cores']} live MPI ranks, process grid {r['process_grid']} (PETSC_DECIDE)"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path on all host cores, on
    this arm's workload: oracle/_ref as one live MPI rank per core over the
    2048^2 grid (reference_run).  A run of --steps K --warmup W times up to K
    steps after min(W, 1) warm-up steps, within a time budget so the arm ends in
    minutes on any host.  Under torchrun only rank 0 runs; it never loads this
    repository's library."""
    if rank != 0:
        return 0
    cores = host_cores()
    r = reference_run(cores, min(args.warmup, 1), args.steps, args.ref_budget_s)
    value = r["value"]
    sample = (f"the 2048x2048 Kapila shock-bubble workload (seed 0, 4 bubbles), {r['timed_steps']} of {args.steps} "
              f"requested SSPRK(4,3) steps timed ({r['seconds']:.1f} s, budget {args.ref_budget_s:.0f} s) after "
              f"{min(args.warmup, 1)} warm-up step; "
              + (f"oracle/_ref (HyPE-2D's sources on the PETSc stand-in) as {cores} live MPI ranks, process grid "
                 f"{r['process_grid']} (PETSC_DECIDE)" if r["kind"] == "reference" else "oracle port, one core"))
    base = {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": sample}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": r["timed_steps"],
            "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * r["seconds"] / max(1, r["timed_steps"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded shock-bubble generator)",
            "config": {"workload": "kapila5-shock-bubble-2048x2048-fp64-weno3-ssprk43", "grid": f"{NX}x{NY}",
                       "system": "kapila5", "order": 2, "bubbles": NBUB, "cfl": 0.4, "ranks": r["cores"],
                       "process_grid": r["process_grid"], "steps_requested": args.steps, "same_config": True},
            "status": r["status"], "cpu_baseline": base,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The job's time is its slowest rank's: MAX all-reduce of a per-rank time."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, cells: int, steps: int, ms: float) -> float:
    """Whole-job cell-updates/s of `world` independent replicas that each ran
    `steps` steps of `cells` cells, the slowest taking `ms` milliseconds."""
    return world * cells * steps / (ms * 1e-3)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def batch_leg(hp, args, local_rank):
    """Batched form: 64 independent Kapila shock-bubble grids of seeded uneven
    sizes (nx, ny drawn from {128, 192, ..., 1024}) stepped together -- one persistent launch per RK
    stage over a (grid, tile) work-list, each step one CUDA graph, tile shape
    from the batch autotuner -- in FP64 and in mixed precision, against the
    plain FP64 path (one solver per grid, run one after another)."""
    rng = np.random.default_rng(2024)
    sizes = [(64 * int(a), 64 * int(b)) for a, b in rng.integers(2, 17, size=(64, 2))]   # sides in {128, 192, ..., 1024}
    nb = [int(k) for k in rng.integers(1, 5, size=64)]
    cells = sum(a * b for a, b in sizes)
    steps = args.batch_steps

    def cfg(nx, ny, prec):
        return hp.Config(system=hp.KAPILA_5EQN, order=2, nx=nx, ny=ny, cfl=0.4, device=local_rank, precision=prec)
    U0 = [hp.initial_state(cfg(nx, ny, 0), "shock_bubble", seed=100 + k, nbubbles=nb[k]) for k, (nx, ny) in enumerate(sizes)]
    out = {}
    finals = {}
    for prec, name in ((hp.PREC_FP64, "fp64"), (hp.PREC_MIXED, "mixed")):
        with hp.Batch(max_instances=64, max_cells=1024 * 1024, device=local_rank) as b:
            ids = [b.add(cfg(nx, ny, prec), U0[k], 0.0, 1e30, 1 << 30) for k, (nx, ny) in enumerate(sizes)]
            tile = b.autotune(3)
            b.advance(3)
            b.sync()
            b.advance(steps)
            b.sync()
            ms = b.last_elapsed_ms()
            st = [b.status(i) for i in ids]
            info = b.info()
            finals[name] = [b.get_state(i).reshape(-1, 6) for i in ids]
        out[name] = {"value": cells * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
                     "autotuned_tile": {"cells": tile[0], "rows": tile[1]}, "work_items_per_stage": info["work_items"],
                     "device_bytes": info["bytes_in_use"], "all_ok": all(x["status"] == hp.OK for x in st),
                     "steps_each": steps + 3}
    # plain FP64 path: one solver per grid, sequentially, a shorter run each
    plain_steps = max(3, min(steps, 20))
    tot_ms = 0.0
    for k, (nx, ny) in enumerate(sizes):
        with hp.Solver(cfg(nx, ny, hp.PREC_FP64)) as s:
            s.set_state(U0[k])
            s.begin(0.0, 1e30, 1 << 30)
            s.advance(2)
            s.wait()
            s.advance(plain_steps)
            s.wait()
            tot_ms += s.last_elapsed_ms()
    plain = cells * plain_steps / (tot_ms * 1e-3)

    def rel_l1(a, b):
        return float(np.abs(a - b).sum() / np.abs(b).sum())
    err_rho = max(rel_l1(M[:, 0] + M[:, 1], F[:, 0] + F[:, 1]) for M, F in zip(finals["mixed"], finals["fp64"]))
    err_a = max(rel_l1(M[:, 5], F[:, 5]) for M, F in zip(finals["mixed"], finals["fp64"]))
    return {"workload": "64 kapila5 shock-bubble grids, nx,ny seeded uniform in {128,192,...,1024}, N=2 SSPRK(4,3)",
            "cells_total": cells, "plain_fp64": {"value": plain, "unit": UNIT, "steps_each": plain_steps},
            "batched_fp64": out["fp64"], "batched_mixed": out["mixed"],
            "speedup_batched_mixed_vs_plain": out["mixed"]["value"] / plain,
            "speedup_batched_fp64_vs_plain": out["fp64"]["value"] / plain,
            "mixed_vs_fp64_max_rel_L1": {"rho": err_rho, "alpha1": err_a}}


def bn_leg(hp, args, local_rank):
    """Baer-Nunziato 1024 x 1024, N = 2, 200 SSPRK(4,3) steps on the seeded
    disc state (alpha_1 from 8 tanh discs, Fourier velocities |u| <= 50,
    p in [1e5, 1e7]; stiffened gases 4.4/6e8 and 1.4/0): FP64 in both flux forms,
    as the reference writes it (phase-2 flux pressure V[8]) and fixed (V[7]), and
    the fixed form in mixed precision with each field's relative L1 / L-infinity
    error against the FP64 run after the 200 steps."""
    out = {}
    n = 1024
    states = {}
    runs = (("reference_form", 0, hp.PREC_FP64), ("fixed_p2", hp.FLAG_BN_FIX_P2, hp.PREC_FP64),
            ("mixed_fixed_p2", hp.FLAG_BN_FIX_P2, hp.PREC_MIXED))
    for name, flags, prec in runs:
        cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=n, ny=n, cfl=0.4, device=local_rank, flags=flags, precision=prec)
        U0 = hp.initial_state(cfg, "bn_discs", seed=SEED)
        with hp.Solver(cfg) as s:
            s.set_state(U0)
            tile = s.autotune(3) if not args.no_autotune else None
            s.begin(0.0, 1e30, 200)
            s.advance(200)
            steps, t, dtn, st = s.wait()
            ms = s.last_elapsed_ms()
            ms_stage = s.time_stage(10)
            tot, amin, amax = s.totals()
            states[name] = s.get_state().reshape(-1, 9)
        bpc = 2 * (6 * 4 + 3 * 8) if prec == hp.PREC_MIXED else 2 * 9 * 8
        out[name] = {"steps_done": steps, "status": st, "t_end": t,
                     "value": n * n * steps / (ms * 1e-3) if steps else None, "unit": UNIT,
                     "ms_per_step": ms / steps if steps else None, "stage_ms_per_launch": ms_stage,
                     "stage_roofline_GBs": bpc * n * n / (ms_stage * 1e-3) / 1e9, "autotuned_tile": tile,
                     "alpha_min": amin, "alpha_max": amax}
    m, f = out["mixed_fixed_p2"], out["fixed_p2"]
    if m["value"] and f["value"]:
        m["speedup_vs_fp64"] = m["value"] / f["value"]
    if m["steps_done"] == f["steps_done"]:
        M, F = states["mixed_fixed_p2"], states["fixed_p2"]

        def rel(a, b):
            return [float(np.abs(a - b).sum() / np.abs(b).sum()), float(np.abs(a - b).max() / np.abs(b).max())]
        errs = {nm: rel(M[:, c], F[:, c]) for c, nm in ((0, "a1rho1"), (3, "a1E1"), (4, "a2rho2"), (7, "a2E2"), (8, "alpha1"))}
        errs["rho"] = rel(M[:, 0] + M[:, 4], F[:, 0] + F[:, 4])
        for nm, cols in (("momentum1_vector", [1, 2]), ("momentum2_vector", [5, 6])):
            dm = np.sqrt(((M[:, cols] - F[:, cols]) ** 2).sum(axis=1))
            mag = np.sqrt((F[:, cols] ** 2).sum(axis=1))
            errs[nm] = [float(dm.sum() / mag.sum()), float(dm.max() / mag.max())]
        m["rel_error_vs_fp64_after_run"] = {"fields_L1_Linf": errs, "steps": f["steps_done"]}
    m["precision"] = "FP32 partial densities, momenta, velocities, reconstruction and their fluxes; FP64 phase energies, " \
                     "alpha1, pressure recovery, totals, dt"
    out["workload"] = "bn9 discs 1024x1024, N=2 SSPRK(4,3), 200 steps"
    out["note"] = ("the reference's flux form stops where the reference would MPI_Abort (inadmissible face state); "
                   "steps after the stop are skipped on the device, so its value counts the steps taken")
    return out


def fast_leg(hp, args, local_rank, world, U0, U_ref, n_done, value_exact, ms_stage_exact):
    """The FP64 performance form (HYPE_PREC_FP64_FAST: fused multiply-adds, shared
    reciprocals; within 1e-12 of the reference per RHS call, tests/test_gpu_fast.py)
    on the same workload and step counts as the bit-exact headline: throughput, its
    stage kernel alone against the measured FMA rate, and its state after the same
    steps against the bit-exact state (per field, relative to the field's largest value)."""
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=NX, ny=NY, cfl=0.4, device=local_rank, precision=hp.PREC_FP64_FAST)
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        tile = s.autotune(3) if not args.no_autotune else None
        s.begin(0.0, 1e30, 1 << 30)
        s.advance(max(3, args.warmup))
        s.wait()
        s.advance(args.steps)
        n, t, dt, st = s.wait()
        ms = max_over_ranks(s.last_elapsed_ms(), world)
        U = s.get_state()
        ms_stage = s.time_stage(20)
        info = s.launch_info()
    F, B = U.reshape(-1, 6), U_ref.reshape(-1, 6)
    err = {}
    for nm, cols in (("a1rho1", [0]), ("a2rho2", [1]), ("momentum_vector", [2, 3]), ("E", [4]), ("alpha1", [5])):
        d = np.sqrt(((F[:, cols] - B[:, cols]) ** 2).sum(axis=1)).max()
        err[nm] = float(d / np.sqrt((B[:, cols] ** 2).sum(axis=1)).max())
    fma_peak = hp.fp64_fma_rate(local_rank, 5)
    v = replica_throughput(world, NX * NY, args.steps, ms)
    return {"value": v, "unit": UNIT, "ms_per_step": ms / args.steps, "status": st, "steps_done": n,
            "speedup_vs_bitexact": v / value_exact, "stage_ms_per_launch": ms_stage,
            "stage_speedup_vs_bitexact": ms_stage_exact / ms_stage, "autotuned_tile": tile, "launch": info,
            "fp64": {"achieved_tflops_stage": RHS_FLOPS_2048 / (ms_stage * 1e-3) / 1e12,
                     "peak_tflops_fma": fma_peak / 1e12,
                     "frac_stage": RHS_FLOPS_2048 / (ms_stage * 1e-3) / fma_peak,
                     "peak_source": "hype_fp64_fma_rate: independent FP64 fused multiply-add chains on every SM, 2 FLOPs each, "
                                    "best of 5 launches",
                     "flops": "the reference's operation count (4784.5 per cell-RHS), not the fused instruction count"},
            "state_vs_bitexact_after_run": {"steps": n_done, "fields_rel_Linf": err,
                                            "norm": "max over cells of the difference / max over cells of the bit-exact "
                                                    "field (momentum: Euclidean norm per cell)"},
            "correctness": "within 1e-12 relative L-infinity of the reference per RHS call (tests/test_gpu_fast.py)"}


def group_leg(hp, args, local_rank, U0, U_ref):
    """The FP64 workload as y-slabs on this GPU (hype_group): the cost of the
    decomposition (halo rows stored by the stage kernels into the neighbours,
    per-stage events, one reduction per step) against the single solver, and the
    final state compared with the single solver's after the same steps."""
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=NX, ny=NY, cfl=0.4, device=local_rank)
    with hp.Group(cfg, args.group_slabs) as grp:
        grp.set_state(U0)
        grp.begin(0.0, 1e30, 1 << 30)
        grp.advance(max(3, args.warmup))
        grp.wait()
        grp.advance(args.steps)
        _, _, _, st = grp.wait()
        ms = grp.last_elapsed_ms()
        same = None if U_ref is None else bool(grp.get_state().tobytes() == U_ref.tobytes())
    return {"value": NX * NY * args.steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / args.steps, "status": st,
            "slabs": args.group_slabs, "devices": [local_rank] * args.group_slabs,
            "bitwise_equal_to_single_solver": same}


def euler_rate(hp, local_rank, prec):
    """Euler N = 2 at 1024^2 (four-quadrant state) in precision `prec`,
    cell-updates/s: the serving mix's third system."""
    cfg = hp.Config(system=hp.EULER, order=2, nx=1024, ny=1024, cfl=0.4, device=local_rank, gamma1=1.4, gamma2=1.4, pi1=0.0,
                    pi2=0.0, precision=prec)
    with hp.Solver(cfg) as s:
        s.set_state(hp.initial_state(cfg, "euler_quadrants", seed=SEED))
        s.begin(0.0, 1e30, 1 << 30)
        s.advance(3)
        s.wait()
        s.advance(20)
        s.wait()
        return 1024 * 1024 * 20 / (s.last_elapsed_ms() * 1e-3)


def mix_capacity(work_share, rates):
    """Throughput of a request mix whose systems share the GPU in turn: the
    work-weighted harmonic mean of the systems' own rates."""
    return 1.0 / sum(work_share[k] / rates[k] for k in work_share)


def serve_leg(hp, args, local_rank, rates):
    """Serving: a Poisson stream of solve requests through the C request loop
    (hype_serve_run) -- 70/20/10 Kapila / Baer-Nunziato / Euler, square grids
    with side log-uniform in 64..2048, runs of 50..2000 steps (log-uniform),
    150 GB HBM budget, continuous batching.  The arrival rate is seed-drawn as
    a load factor rho ~ U[0.5, 0.8] of the batched throughput measured above."""
    rng = np.random.default_rng(7)
    n = args.serve_requests
    T = hp.BC_TRANSMISSIVE
    prec = hp.PREC_MIXED if args.serve_precision == "mixed" else hp.PREC_FP64
    reqs, work = [], []
    for i in range(n):
        u = rng.uniform()
        side = int(round(64 * 32 ** rng.uniform()))
        steps = int(round(50 * 40 ** rng.uniform()))
        if u < 0.7:
            cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=side, ny=side, cfl=0.4, device=local_rank, precision=prec)
            ic, par = hp.IC_SHOCK_BUBBLE, int(rng.integers(1, 5))
        elif u < 0.9:
            # phase-2 flux pressure from V[7]; the reference's V[8] (baer_nunziato.c:271) aborts these runs early
            cfg = hp.Config(system=hp.BAER_NUNZIATO, order=2, nx=side, ny=side, cfl=0.4, device=local_rank,
                            flags=hp.FLAG_BN_FIX_P2, precision=prec)
            ic, par = hp.IC_BN_DISCS, 0
        else:
            cfg = hp.Config(system=hp.EULER, order=2, nx=side, ny=side, cfl=0.4, device=local_rank, gamma1=1.4, gamma2=1.4,
                            pi1=0.0, pi2=0.0, precision=prec)
            ic, par = hp.IC_EULER_QUADRANTS, 0
        reqs.append(hp.Request(0.0, cfg, 0.0, 1e30, steps, ic, 5000 + i, par))
        work.append(side * side * steps)
    rho = float(rng.uniform(0.5, 0.8))
    if args.serve_load is not None:
        rho = args.serve_load
    # the load factor is of this mix's own capacity (per-system rates measured in this run)
    share = {k: 0.0 for k in rates}
    for r, w in zip(reqs, work):
        share[{hp.KAPILA_5EQN: "kapila", hp.BAER_NUNZIATO: "bn", hp.EULER: "euler"}[r.cfg.system]] += w
    total = sum(share.values())
    share = {k: v / total for k, v in share.items()}
    capacity = mix_capacity(share, rates)
    rate = rho * capacity / float(np.mean(work))
    t = 0.0
    for r in reqs:
        r.arrival_s = t
        t += float(rng.exponential(1.0 / rate))
    res, st = hp.serve(reqs, device=local_rank, hbm_budget=150 * 10 ** 9, max_instances=1024, max_cells=2048 * 2048,
                       poll_ms=args.serve_poll_ms, realtime=True, active_cells=args.serve_active_cells,
                       substep_cells=args.serve_substep_cells)
    lat = np.array([r["latency_s"] for r in res])
    by_sys = {}
    for nm, sysid in (("kapila", hp.KAPILA_5EQN), ("bn", hp.BAER_NUNZIATO), ("euler", hp.EULER)):
        sel = np.array([r.cfg.system == sysid for r in reqs])
        if sel.any():
            fails = {}
            for i in np.nonzero(sel)[0]:
                if res[i]["status"] != hp.OK:
                    key = hp.lib().hype_status_string(res[i]["status"]).decode()
                    fails[key] = fails.get(key, 0) + 1
            by_sys[nm] = {"n": int(sel.sum()), "p50_s": float(np.percentile(lat[sel], 50)),
                          "p99_s": float(np.percentile(lat[sel], 99)), "failed": fails}
    # the first failed requests: which grid, how many steps asked and done
    failures = [{"i": i, "system": int(r.cfg.system), "side": r.cfg.nx, "steps": r.max_steps, "steps_done": res[i]["steps"],
                 "status": res[i]["status"]} for i, r in enumerate(reqs) if res[i]["status"] != hp.OK][:40]
    return {"workload": f"Poisson stream of {n} solves: 70/20/10 kapila5/bn/euler, square grids 64..2048 log-uniform, "
                        "50..2000 steps log-uniform, N=2 SSPRK(4,3), 150 GB HBM budget",
            "requests": n, "precision": args.serve_precision, "active_cells": args.serve_active_cells,
            "capacity_estimate": capacity, "capacity_from": {"rates": rates, "work_share": share,
                                                             "rule": "work-weighted harmonic mean of the systems' rates"},
            "substep_cells": args.serve_substep_cells, "bn_form": "phase-2 flux pressure from V[7]", "load_factor": rho, "rate_per_s": rate,
            "offered_cell_updates": float(np.sum(work)),
            "p50_s": st["p50_s"], "p90_s": st["p90_s"], "p99_s": st["p99_s"], "max_s": st["max_s"], "mean_s": st["mean_s"],
            "queue_p50_s": st["queue_p50_s"], "queue_p99_s": st["queue_p99_s"],
            "value": st["cell_updates_per_s"], "unit": UNIT, "wall_s": st["wall_s"],
            "completed": st["completed"], "failed": st["failed"], "peak_instances": st["peak_instances"],
            "peak_bytes": st["peak_bytes"], "polls": st["polls"], "batch_steps": st["steps_replayed"],
            "by_system": by_sys, "failures": failures}


def run_gpu(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    hp = load_pkg()
    torch.cuda.set_device(local_rank)
    cfg = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=NX, ny=NY, cfl=0.4, device=local_rank)
    U0 = hp.initial_state(cfg, "shock_bubble", seed=SEED + rank, nbubbles=NBUB)
    solver = hp.Solver(cfg)
    solver.set_state(U0)
    tile = solver.autotune(3) if not args.no_autotune else None
    solver.begin(0.0, 1e30, 1 << 30)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up steps (untimed)
    solver.advance(max(3, args.warmup))
    steps, t_end, dt_next, st = solver.wait()
    if st != hp.OK:
        raise RuntimeError(f"warm-up failed: status {st}")
    # timed: exactly K steps, CUDA events on the solver's stream
    barrier()
    with ClockSampler(local_rank) as clk:
        solver.advance(args.steps)
        steps2, t2, dt2, st = solver.wait()
    barrier()
    if st != hp.OK:
        raise RuntimeError(f"timed run failed: status {st}")
    ms = max_over_ranks(solver.last_elapsed_ms(), world)
    cells = NX * NY
    value = replica_throughput(world, cells, args.steps, ms)
    U_fp64 = solver.get_state()   # the y-slab leg compares with it
    n_done = max(3, args.warmup) + args.steps
    err_steps = max(args.error_steps, n_done)
    # the FP64 state after err_steps steps, for the mixed form's error (500 steps of
    # the 2048^2 mixed-precision configuration); before the host-buffer leg, which
    # restarts the device state from a fixed input
    U_err = U_fp64
    if not args.no_mixed and err_steps > n_done:
        solver.advance(err_steps - n_done)
        solver.wait()
        U_err = solver.get_state()

    # dominant kernel: the stage kernel, timed alone (CUDA events, same stream)
    ms_stage = solver.time_stage(20)
    alg_bytes_launch = (2 * 6 * 8) * cells                # an AXPY stage: read one state, write one state
    achieved = alg_bytes_launch / (ms_stage * 1e-3) / 1e9
    peak, peak_src = peaks()
    totals, amin, amax = solver.totals()
    # FP64 roofline: the reference's operation count per cell-update against the
    # measured rate of separately rounded FP64 multiplies and adds
    flops_cu = 4 * RHS_FLOPS_2048 / (NX * NY) + RK_FLOPS_PER_CELL
    fp64_peak = hp.fp64_rate(local_rank, 5)
    stage_flops = RHS_FLOPS_2048 + 12 * cells   # one stage: an RHS plus the AXPY combination (1 mul + 1 add per field)
    fp64 = {"flops_per_cell_update": flops_cu, "achieved_tflops": value / world * flops_cu / 1e12,
            "peak_tflops": fp64_peak / 1e12, "frac": (value / world * flops_cu) / fp64_peak,
            "stage_kernel_frac": (NX * NY * RHS_FLOPS_2048 / (NX * NY) / (ms_stage * 1e-3)) / fp64_peak,
            "peak_source": "hype_fp64_rate: independent FP64 multiply and add chains on every SM, no FMA (as the bit-exact "
                           "kernels), best of 5 launches",
            "note": "divisions and square roots count one operation each (213.3 and 8.0 per cell-RHS) but run as "
                    "multi-instruction sequences on the FP64 pipe"}

    # end to end through the C ABI with host buffers: per step the state goes
    # host (pinned) -> device, one SSP-RK step runs, the state comes back.
    pin_in = torch.from_numpy(solver.get_state()).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.advance_host(pin_in.numpy(), pin_out.numpy(), 1)
    barrier()
    e2e_s = max_over_ranks(max(time.perf_counter() - t0, 1e-9), world)
    state_bytes = cells * 6 * 8
    e2e = {"value": (world * cells * e2e_steps / e2e_s) if e2e_steps else None, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
           "d2h_bytes_per_step": state_bytes,
           "how": "per step: hype_advance_host(U_in, U_out, 1): the state from pinned host memory, one SSPRK(4,3) "
                  "step, the state back to pinned host memory (every stage a wavefront of row bands behind the "
                  "band-by-band upload, bands copied out as they finish); wall clock"}
    # the drop-in's per-stage call: RHSFunctionPrim through the C ABI with host
    # buffers (petsc_glue.c makes this call once per TS stage)
    rhs_host = None
    if e2e_steps:
        pin_rhs = torch.empty_like(pin_in).pin_memory()
        solver.rhs_function_prim(0.0, pin_in.numpy(), pin_rhs.numpy())
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            solver.rhs_function_prim(0.0, pin_in.numpy(), pin_rhs.numpy())
        barrier()
        rhs_s = max_over_ranks(max(time.perf_counter() - t0, 1e-9), world)
        # the same call on pageable arrays (as PETSc's Vec arrays are): staged through pinned buffers
        pg_in, pg_rhs = pin_in.numpy().copy(), np.empty(pin_in.numel())
        solver.rhs_function_prim(0.0, pg_in, pg_rhs)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            solver.rhs_function_prim(0.0, pg_in, pg_rhs)
        barrier()
        rhs_pg_s = max_over_ranks(max(time.perf_counter() - t0, 1e-9), world)
        rhs_host = {"ms_per_call": rhs_s / e2e_steps * 1e3, "value": world * cells * e2e_steps / rhs_s, "unit": "cell-RHS/s",
                    "pageable_ms_per_call": rhs_pg_s / e2e_steps * 1e3,
                    "calls": e2e_steps, "h2d_bytes_per_call": state_bytes, "d2h_bytes_per_call": state_bytes,
                    "how": "hype_rhs_prim(t, U, RHS, &dt) from and to pinned host memory, the call RHSFunctionPrim "
                           "(petsc_glue.c) makes once per TS stage: row bands of U stream in, each band's RHS launch "
                           "runs once its rows are there, RHS rows stream out; wall clock.  pageable_ms_per_call: the "
                           "same from pageable arrays, staged through the solver's pinned buffers by host threads"}
    info = solver.launch_info()
    solver.close()

    # mixed-precision form on the same workload and step count, and its error
    # against the FP64 run (relative L1 / L-infinity per field)
    mixed = None
    if not args.no_mixed:
        cm = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=NX, ny=NY, cfl=0.4, device=local_rank, precision=hp.PREC_MIXED)
        sm = hp.Solver(cm)
        sm.set_state(U0)
        mtile = sm.autotune(3) if not args.no_autotune else None
        sm.begin(0.0, 1e30, 1 << 30)
        sm.advance(max(3, args.warmup))
        sm.wait()
        barrier()
        sm.advance(args.steps)
        _, tm, _, stm = sm.wait()
        barrier()
        ms_m = max_over_ranks(sm.last_elapsed_ms(), world)
        if err_steps > n_done:
            sm.advance(err_steps - n_done)
            sm.wait()
        M = sm.get_state().reshape(-1, 6)
        F = U_err.reshape(-1, 6)
        ms_stage_m = sm.time_stage(20)
        e2e_m = None
        if e2e_steps:   # host buffers, as the FP64 e2e leg: FP64 cell-major state in and out per step
            min_ = torch.from_numpy(M.reshape(-1).copy()).pin_memory()
            mout = torch.empty_like(min_).pin_memory()
            sm.advance_host(min_.numpy(), mout.numpy(), 1)
            barrier()
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                sm.advance_host(min_.numpy(), mout.numpy(), 1)
            barrier()
            em_s = max_over_ranks(max(time.perf_counter() - t0, 1e-9), world)
            e2e_m = {"value": world * cells * e2e_steps / em_s, "unit": UNIT, "ms_per_step": em_s / e2e_steps * 1e3,
                     "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                     "how": "hype_advance_host(U_in, U_out, 1) of the mixed solver, FP64 host state converted band by "
                            "band on the device; wall clock"}
        sm.close()

        def rel(a, b):
            return [float(np.abs(a - b).sum() / np.abs(b).sum()), float(np.abs(a - b).max() / np.abs(b).max())]
        errs = {"rho": rel(M[:, 0] + M[:, 1], F[:, 0] + F[:, 1]), "alpha1": rel(M[:, 5], F[:, 5])}
        for c, nm in ((0, "a1rho1"), (1, "a2rho2"), (4, "E")):
            errs[nm] = rel(M[:, c], F[:, c])
        dm = np.hypot(M[:, 2] - F[:, 2], M[:, 3] - F[:, 3])
        mag = np.hypot(F[:, 2], F[:, 3])
        errs["momentum_vector"] = [float(dm.sum() / mag.sum()), float(dm.max() / mag.max())]
        vm = replica_throughput(world, cells, args.steps, ms_m)
        mixed = {"value": vm, "unit": UNIT, "ms_per_step": ms_m / args.steps, "speedup_vs_fp64": vm / value,
                 "status": stm, "stage_ms_per_launch": ms_stage_m, "autotuned_tile": mtile,
                 "bytes_per_cell_update": 9 * (4 * 4 + 2 * 8),
                 "rel_error_vs_fp64_after_run": {"fields_L1_Linf": errs, "steps": err_steps},
                 "precision": "FP32 state/recon/flux; FP64 E, alpha1, pressure recovery, totals, dt", "e2e": e2e_m}

    fast = None if args.no_fast else fast_leg(hp, args, local_rank, world, U0, U_fp64, n_done, value, ms_stage)
    group = None if args.group_slabs <= 1 else group_leg(hp, args, local_rank, U0, U_fp64)
    bn = None if args.no_bn else bn_leg(hp, args, local_rank)
    batched = None if args.no_batch else batch_leg(hp, args, local_rank)
    serving = None
    if args.serve_requests > 0:
        # per-system rates of this run in the requests' precision: batched Kapila, BN in
        # the fixed flux form, Euler measured here (fallbacks when a leg was skipped)
        mixed_serve = args.serve_precision == "mixed"
        kap = None
        if batched:
            kap = batched["batched_mixed" if mixed_serve else "batched_fp64"]["value"]
        rates = {"kapila": kap or (value * (2.0 if mixed_serve else 1.0)),
                 "bn": (bn or {}).get("mixed_fixed_p2" if mixed_serve else "fixed_p2", {}).get("value") or 0.5 * value,
                 "euler": euler_rate(hp, local_rank, hp.PREC_MIXED if mixed_serve else hp.PREC_FP64)}
        serving = serve_leg(hp, args, local_rank, rates)

    if rank != 0:
        return 0
    cpu = None if args.no_cpu_baseline else cpu_baseline()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded shock-bubble generator, random-init)",
            "config": {"workload": "kapila5-shock-bubble-2048x2048-fp64-weno3-ssprk43", "grid": f"{NX}x{NY}",
                       "system": "kapila5", "order": 2, "bubbles": NBUB, "cfl": 0.4, "precision": "fp64-bitexact",
                       "parallelism": f"replicas{world}", "l2": "state 201 MB per buffer > 126 MB L2 (no flush needed)"},
            "roofline": {"bound": "fp64", "achieved": stage_flops / (ms_stage * 1e-3) / 1e12, "peak": fp64_peak / 1e12,
                         "unit": "TFLOP/s", "frac": stage_flops / (ms_stage * 1e-3) / fp64_peak,
                         "traffic": STAGE_TRAFFIC_BYTES, "traffic_source": "one ncu capture of the stage kernel (profiles/)",
                         "algorithmic_flops": stage_flops,
                         "peak_source": "measured in this run: hype_fp64_rate, independent FP64 multiply and add chains on "
                                        "every SM without FMA (the bit-exact kernel's instruction mix), best of 5 launches",
                         "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                                 "algorithmic_bytes": alg_bytes_launch, "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_src})"},
                         "step": fp64,
                         "note": "stage kernel alone, one SSPRK(4,3) stage of 2048^2 cells per launch: the reference's "
                                 "operation count (4784.5 per cell-RHS, oracle/flops.cpp, plus 12 for the stage combination) "
                                 "over the CUDA-event time; 96 B/cell algorithmic HBM bytes per launch (one FP64 state read + "
                                 "one write).  The kernel is FP64-pipe bound (profiles/stage_kernel_kapila2048_fp64.md)"},
            "stage_kernel": {"ms_per_launch": ms_stage, "launch": info, "autotuned_tile": tile},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps * 6,
            "clocks": clk.summary(),
            "checks": {"alpha_min": amin, "alpha_max": amax, "steps_done": steps2, "t": t2},
            "forms": {"fp64_fast": fast, "mixed": mixed, "bn1024": bn, "batched": batched, "serving": serving,
                      "y_slabs": group, "rhs_host": rhs_host}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=120.0,
                    help="reference arm: seconds of timed reference steps after which it stops early")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default stage tile shape")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-fast", action="store_true", help="skip the FP64 performance-form leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-grids leg")
    ap.add_argument("--no-bn", action="store_true", help="skip the Baer-Nunziato 1024^2 leg")
    ap.add_argument("--error-steps", type=int, default=500,
                    help="steps after which the mixed form's error against FP64 is measured (at least warm-up + timed steps)")
    ap.add_argument("--group-slabs", type=int, default=2, help="y-slabs of the decomposed leg on this GPU (<= 1: skip)")
    ap.add_argument("--batch-steps", type=int, default=300, help="steps of the batched-grids leg")
    ap.add_argument("--serve-requests", type=int, default=64, help="requests of the serving leg (0: skip)")
    ap.add_argument("--serve-precision", default="mixed", choices=["mixed", "fp64"], help="precision of the served requests")
    ap.add_argument("--serve-poll-ms", type=float, default=10.0)
    ap.add_argument("--serve-active-cells", type=int, default=4 << 20,
                    help="scheduler: cells stepped at once, least remaining work first (0: all resident requests)")
    ap.add_argument("--serve-load", type=float, default=None, help="load factor of the arrival rate (default: seed-drawn)")
    ap.add_argument("--serve-substep-cells", type=int, default=0,
                    help="scheduler: a grid of c cells takes up to this/c steps per batch step (0: one)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        return run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
