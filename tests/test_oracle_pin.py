"""Pin the CPU oracle (oracle/hype_oracle.c) to the reference's own outputs.

* Against tests/golden/reference_outputs.json: SHA-256 of the RHS / final
  state and the exact dt, steps and final time that the reference's own
  HyPE-2D sources produced (tests/golden/make_golden.py).
* Against the reference itself (oracle/_ref) on fresh seeds, when it has been
  built here (`make -C oracle ref`; needs the reference sources).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cases
import oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(GOLDEN["rhs"]))
def test_oracle_rhs_matches_reference_bits(name, orc):
    g = GOLDEN["rhs"][name]
    _, cfg, kind, seed = cases.case_by_name(name)
    assert cases.config_to_dict(cfg) == g["config"]
    U = cases.state(cfg, kind, seed)
    assert sha(U) == g["sha_U"], "seeded input generator drifted; regenerate the golden file"
    R, dt, st = orc.rhs(cfg, U)
    assert st == g["status"]
    assert float(dt).hex() == g["dt"]
    assert sha(R) == g["sha_RHS"]


@pytest.mark.parametrize("name", sorted(GOLDEN["solve"]))
def test_oracle_solve_matches_reference_bits(name, orc):
    g = GOLDEN["solve"][name]
    (_, cfg, kind, seed), t0, tf, nmax = cases.case_by_name(name)
    U = cases.state(cfg, kind, seed)
    assert sha(U) == g["sha_U"]
    Ue, steps, te, dtn, st = orc.solve(cfg, U, t0, tf, nmax)
    if g["status"] != 0:
        # the reference aborts (MPI_Abort) on an inadmissible face state; the oracle reports it
        assert st == O.ERR_INADMISSIBLE
        return
    assert st == 0
    assert steps == g["steps"]
    assert float(te).hex() == g["t_end"]
    assert float(dtn).hex() == g["dt_next"]
    assert sha(Ue) == g["sha_U_end"]


def test_small_arrays_present():
    arr = np.load(os.path.join(os.path.dirname(__file__), "golden", "rhs_small.npz"))
    for name in ("kapila_16x16_bubble", "euler_16x16", "bn_16x16"):
        U, R = arr[name + "__U"], arr[name + "__RHS"]
        assert sha(R) == GOLDEN["rhs"][name]["sha_RHS"]
        assert U.shape == R.shape


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("seed", [101, 102, 103])
@pytest.mark.parametrize("system", [O.EULER, O.KAPILA, O.BN])
@pytest.mark.parametrize("order", [1, 2, 3])
def test_oracle_vs_live_reference(system, order, seed, orc):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(5, 30)), int(rng.integers(5, 30))
    bcs = [int(b) for b in rng.choice([O.TRANSMISSIVE, O.REFLECTIVE], 4)]
    if rng.uniform() < 0.3:
        bcs[0] = bcs[1] = O.PERIODIC
    eos = cases.EULER_EOS if system == O.EULER else cases.KAPILA_EOS
    cfg = O.Config(system=system, order=order, nx=nx, ny=ny, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                   bc_top=bcs[3], **eos)
    kind = {O.EULER: "quadrants", O.KAPILA: "rough", O.BN: "discs"}[system]
    U = cases.state(cfg, kind, seed)
    ref = O.Reference(system)
    ref.setup(cfg)
    R1, dt1, s1 = ref.rhs(U)
    R2, dt2, s2 = orc.rhs(cfg, U)
    assert (s1 != 0) == (s2 != 0)
    if s1 == 0:
        assert dt1 == dt2
        assert R1.tobytes() == R2.tobytes()
    U1, n1, t1, d1, st1 = ref.solve(U, 0.0, 1e9, 3)
    U2, n2, t2, d2, st2 = orc.solve(cfg, U, 0.0, 1e9, 3)
    assert (st1 != 0) == (st2 != 0)
    if st1 == 0:
        assert (n1, t1, d1) == (n2, t2, d2)
        assert U1.tobytes() == U2.tobytes()


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (needs the reference sources)")
def test_oracle_conservative_path_vs_live_reference(orc):
    for system, kind in ((O.EULER, "quadrants"), (O.KAPILA, "rough"), (O.BN, "discs")):
        eos = cases.EULER_EOS if system == O.EULER else cases.KAPILA_EOS
        cfg = O.Config(system=system, order=2, nx=14, ny=11, conservative=1, bc_left=O.REFLECTIVE, **eos)
        U = cases.state(cfg, kind, 7)
        ref = O.Reference(system)
        ref.setup(cfg)
        R1, dt1, s1 = ref.rhs(U)
        R2, dt2, s2 = orc.rhs(cfg, U)
        assert s1 == 0 and s2 == 0
        assert dt1 == dt2 and R1.tobytes() == R2.tobytes()


@pytest.mark.skipif(not O.viscous_reference_available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("conservative", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3])
def test_oracle_viscous_vs_live_reference(conservative, order, orc):
    """The VISCOUS build of the reference (Kapila; hype.h:36 leaves it off):
    face gradients from the unlimited coefficients, ViscRiemannSolver[Prim],
    tangential reflection at walls and the viscous dt."""
    T, R, P, I = O.TRANSMISSIVE, O.REFLECTIVE, O.PERIODIC, O.INLET
    ref = O.Reference(O.KAPILA, viscous=True)
    for bcs, kind, mu in (((R, R, R, R), "rough", (0.3, 0.05)), ((T, T, P, P), "bubble", (1e-2, 0.0)),
                          ((R, T, R, T), "bubble", (2.0, 0.5)), ((I, T, R, R), "rough", (0.1, 0.0))):
        ext = dict(x_min=0.0, x_max=2.0, y_min=-1.0, y_max=0.6) if bcs[0] == I else {}
        cfg = O.Config(system=O.KAPILA, order=order, nx=23, ny=17, bc_left=bcs[0], bc_right=bcs[1], bc_bottom=bcs[2],
                       bc_top=bcs[3], conservative=conservative, viscous=1, mu1=mu[0], mu2=mu[1], **cases.KAPILA_EOS, **ext)
        U = cases.state(cfg, kind, 5 + order)
        ref.setup(cfg)
        R1, dt1, s1 = ref.rhs(U)
        R2, dt2, s2 = orc.rhs(cfg, U)
        assert (s1 == 0) == (s2 == 0)
        if s1 == 0:
            assert dt1 == dt2 and R1.tobytes() == R2.tobytes()
        if kind == "bubble":
            U1, n1, t1, d1, st1 = ref.solve(U, 0.0, 1.0, 3)
            U2, n2, t2, d2, st2 = orc.solve(cfg, U, 0.0, 1.0, 3)
            assert st1 == 0 and st2 == 0 and (n1, t1, d1) == (n2, t2, d2) and U1.tobytes() == U2.tobytes()
