"""The bounded waits of the stage kernels, driven to expiry.

hype_test_skip_row_loads makes the kernels issue no TMA load for the rows from a
given one on, so nothing ever completes the wait on such a row: no copy is in
flight for it and nothing faults.  The block waits out its limit (about 2 s of
GPU time), waits for the loads it did issue, raises the timeout bit and returns;
the call reports HYPE_ERR_TIMEOUT.  With the hook off again the same solver --
same context, same device buffers -- must give the oracle's bits.
"""
import time

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mixed", [False, True])
def test_lost_row_load_times_out_and_the_solver_recovers(hp, orc, mixed):
    cfg = O.Config(system=O.KAPILA, order=2, nx=100, ny=16, **cases.KAPILA_EOS)
    U = cases.state(cfg, "bubble", 3)
    pc = cases.to_pkg(cfg)
    if mixed:
        pc.precision = hp.PREC_MIXED
    with hp.Solver(pc) as s:
        R0, dt0, st0 = s.rhs_function_prim(0.0, U)
        assert st0 == hp.OK
        s.test_skip_row_loads(12)
        t0 = time.perf_counter()
        _, _, st = s.rhs_function_prim(0.0, U, check=False)
        waited = time.perf_counter() - t0
        assert st == hp.ERR_TIMEOUT
        assert waited < 30.0
        s.test_skip_row_loads(-1)
        R1, dt1, st1 = s.rhs_function_prim(0.0, U)
    assert st1 == hp.OK
    assert R1.tobytes() == R0.tobytes() and dt1 == dt0
    if not mixed:
        Ro, dto, _ = orc.rhs(cfg, U)
        assert R1.tobytes() == Ro.tobytes() and dt1 == dto


def test_time_loop_reports_the_timeout(hp, orc):
    cfg = O.Config(system=O.KAPILA, order=2, nx=100, ny=16, **cases.KAPILA_EOS)
    U = cases.state(cfg, "bubble", 4)
    with hp.Solver(cases.to_pkg(cfg)) as s:
        s.test_skip_row_loads(9)
        s.set_state(U)
        _, _, _, st = s.solve(0.0, 1.0, 2, check=False)
        assert st == hp.ERR_TIMEOUT
        assert "TMA" in s.last_error()
        s.test_skip_row_loads(-1)
        s.set_state(U)
        n, t, dt, st = s.solve(0.0, 1.0, 2)
        Ue = s.get_state()
    Uo, no, to, dto, sto = orc.solve(cfg, U, 0.0, 1.0, 2)
    assert st == hp.OK and (n, t, dt) == (no, to, dto)
    assert Ue.tobytes() == Uo.tobytes()
