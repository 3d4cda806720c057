"""The algorithmic operation count behind bench.py's FP64 roofline.

oracle/flops.cpp compiles the oracle with every double operation counted.  The
counted build must compute the oracle's own bits, and its count for the bench
workload's RHS (2048^2 Kapila, N = 2, 4-bubble shock-bubble, seed 0) must be the
constant bench.py reports against.
"""
import os
import sys

import pytest

import cases
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["kapila_37x23_rough_mixed_bc", "bn_16x16", "euler_21x19_reflective_N1", "kapila_cons_37x23_rough",
                                  "kapila_visc_37x23_rough"])
def test_counted_oracle_computes_the_oracle_bits(name, orc):
    _, cfg, kind, seed = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    R, st, counts = O.count_rhs_ops(cfg, U)
    Ro, _, sto = orc.rhs(cfg, U)
    assert st == sto and R.tobytes() == Ro.tobytes()
    assert counts["flops"] > 0 and counts["div"] > 0


def test_bench_flop_constant(hp):
    sys.path.insert(0, ROOT)
    import bench
    cfg = O.Config(system=O.KAPILA, order=2, nx=bench.NX, ny=bench.NY, cfl=0.4, **cases.KAPILA_EOS)
    pc = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=bench.NX, ny=bench.NY, cfl=0.4)
    U = hp.initial_state(pc, "shock_bubble", seed=bench.SEED, nbubbles=bench.NBUB)
    _, st, counts = O.count_rhs_ops(cfg, U)
    assert st == O.OK
    assert counts["flops"] == bench.RHS_FLOPS_2048
