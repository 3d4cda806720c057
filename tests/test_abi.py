"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/*.h declares, validates configurations before touching a device, and
its seeded initial-data generators are deterministic and admissible."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import cases
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        names |= set(re.findall(r"HYPE_API\s+[\w\s\*]*?\b(hype_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(hp):
    assert os.path.exists(hp.LIB_PATH)
    out = subprocess.run(["nm", "-D", "--defined-only", hp.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (hype_\w+)", out))
    declared = declared_symbols()
    assert len(declared) >= 20
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    lib = hp.lib()
    for name in declared:
        assert getattr(lib, name) is not None


def test_nvar_and_status_strings(hp):
    L = hp.lib()
    assert [L.hype_nvar(s) for s in (0, 1, 2, 7)] == [4, 6, 9, 0]
    for st in range(8):
        assert L.hype_status_string(st)


def test_config_defaults_follow_reference_main(hp):
    c = hp.default_config()
    # HyPE-2D/hype.c:32-49 and hype.h:42-45
    assert (c.order, c.nx, c.ny, c.cfl) == (1, 128, 128, 0.9)
    assert (c.x_max, c.y_max) == (12.0, 12.0)
    assert (c.bc_left, c.bc_right, c.bc_bottom, c.bc_top) == (4, 4, 3, 3)
    assert (c.gamma1, c.gamma2, c.pi1, c.pi2) == (4.4, 1.4, 6000.0, 0.0)


@pytest.mark.parametrize("change,needle", [
    (dict(bc_left=0), "wall"),
    (dict(bc_right=1), "inlet"),
    (dict(system=0, bc_left=1), "inlet"),
    (dict(nx=2), "3x3"),
    (dict(order=4), "order"),
    (dict(system=5), "system"),
    (dict(bc_left=2), "periodic"),
    (dict(cfl=0.0), "CFL"),
    (dict(x_max=0.0), "domain"),
    (dict(precision=7), "precision"),
    (dict(precision=1, system=2, order=3), "N = 2"),
    (dict(precision=1, order=1), "N = 2"),
    (dict(precision=1, order=2, flags=2), "FP64 only"),
    (dict(flags=8), "unknown flags"),
    (dict(flags=4, system=2), "viscous"),
    (dict(flags=4, order=0), "viscous"),
    (dict(flags=4, precision=1), "viscous"),
])
def test_invalid_configs_rejected_before_device(hp, change, needle):
    cfg = hp.Config(nx=16, ny=16)
    for k, v in change.items():
        setattr(cfg, k, v)
    with pytest.raises(hp.HypeError) as ei:
        hp.Solver(cfg)
    assert ei.value.status == hp.ERR_INVALID
    assert needle.lower() in str(ei.value).lower()


def test_valid_config_without_gpu_reports_no_device(hp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hp.HypeError) as ei:
        hp.Solver(hp.Config(nx=16, ny=16))
    assert ei.value.status in (hp.ERR_NO_DEVICE, hp.ERR_CUDA)


@pytest.mark.parametrize("change,nslabs,needle", [
    (dict(), 0, "nslabs"),
    (dict(ny=12), 5, "ny/3"),
    (dict(precision=1, order=1), 2, "N = 2"),
    (dict(nx=2), 1, "3x3"),
])
def test_group_rejects_before_device(hp, change, nslabs, needle):
    """y-slab groups: 1..ny/3 slabs of a valid configuration, checked before any device call."""
    cfg = hp.Config(nx=16, ny=16)
    for k, v in change.items():
        setattr(cfg, k, v)
    with pytest.raises(hp.HypeError) as ei:
        hp.Group(cfg, nslabs)
    assert ei.value.status == hp.ERR_INVALID
    assert needle.lower() in str(ei.value).lower()


def test_group_without_gpu_reports_no_device(hp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hp.HypeError) as ei:
        hp.Group(hp.Config(nx=16, ny=16), 2)
    assert ei.value.status == hp.ERR_NO_DEVICE


def test_initial_states_deterministic_and_admissible(hp):
    c = hp.Config(nx=64, ny=48)
    a = hp.initial_state(c, "shock_bubble", seed=3, nbubbles=4)
    b = hp.initial_state(c, "shock_bubble", seed=3, nbubbles=4)
    d = hp.initial_state(c, "shock_bubble", seed=4, nbubbles=4)
    assert a.tobytes() == b.tobytes() and a.tobytes() != d.tobytes()
    Q = a.reshape(48, 64, 6)
    assert np.all(Q[..., 5] >= 1e-6 - 1e-18) and np.all(Q[..., 5] <= 1 - 1e-6 + 1e-18)
    assert np.all(Q[..., 0] > 0) and np.all(Q[..., 1] > 0) and np.all(Q[..., 4] > 0)
    cb = hp.Config(system=hp.BAER_NUNZIATO, nx=40, ny=40)
    B = hp.initial_state(cb, "bn_discs", seed=1).reshape(40, 40, 9)
    assert np.all(B[..., 8] >= 0.01 - 1e-15) and np.all(B[..., 8] <= 0.99 + 1e-15)
    ce = hp.Config(system=hp.EULER, nx=10, ny=10, gamma1=1.4)
    E = hp.initial_state(ce, "euler_quadrants", seed=1).reshape(10, 10, 4)
    assert len(np.unique(E[..., 0])) == 4
    with pytest.raises(hp.HypeError):
        hp.initial_state(cb, "shock_bubble")


def test_shock_bubble_rankine_hugoniot(hp):
    """The post-shock state satisfies the stiffened-gas jump conditions for phase 1."""
    c = hp.Config(nx=100, ny=4)
    Q = hp.initial_state(c, "shock_bubble", seed=0, nbubbles=0).reshape(4, 100, 6)
    g, pi = c.gamma1, c.pi1
    # post-shock cell (x < 0.1) and pre-shock cell
    orc = O.Oracle()

    def prim(q):
        # kapila_5eqn.c:14-35 via numpy
        a1 = q[5]; a2 = 1 - a1; rho = q[0] + q[1]; u = q[2] / rho; v = q[3] / rho
        e = q[4] - 0.5 * rho * (u * u + v * v)
        G1, G2 = c.gamma1 - 1, c.gamma2 - 1
        p = (e * G1 * G2 - a1 * c.gamma1 * c.pi1 * G2 - a2 * c.gamma2 * c.pi2 * G1) / (a1 * G2 + a2 * G1)
        return q[0] / a1, u, p
    r1, u1, p1 = prim(Q[0, 0])
    r0, u0, p0 = prim(Q[0, 50])
    assert u0 == 0.0 and abs(p0 - 1e5) < 1e-3 and abs(r0 - 1000) < 1e-9
    assert 10 * 1e5 * (1 - 1e-9) <= p1 <= 1000 * 1e5 * (1 + 1e-9)
    # Hugoniot: e1 - e0 = (p1 + p0)/2 (1/r0 - 1/r1), with stiffened-gas e = (p + g pi)/((g-1) rho)
    e0 = (p0 + g * pi) / ((g - 1) * r0)
    e1 = (p1 + g * pi) / ((g - 1) * r1)
    assert abs((e1 - e0) - 0.5 * (p1 + p0) * (1 / r0 - 1 / r1)) < 1e-6 * abs(e1)
    # mass and momentum across a shock of speed s: r0 s = r1 (s - u1)
    s = r1 * u1 / (r1 - r0)
    assert abs((p1 - p0) - r0 * s * u1) < 1e-6 * p1
    assert orc is not None


def test_serve_validates_before_device(hp):
    """The request loop rejects a trace whose arrivals go backwards before it
    touches a device; without a GPU it reports that instead of running."""
    import torch
    c = hp.Config(nx=16, ny=16)
    with pytest.raises(hp.HypeError) as ei:
        hp.serve([hp.Request(1.0, c), hp.Request(0.5, c)])
    assert ei.value.status == hp.ERR_INVALID
    if not torch.cuda.is_available():
        with pytest.raises(hp.HypeError) as ei:
            hp.serve([hp.Request(0.0, c, max_steps=2)])
        assert ei.value.status in (hp.ERR_NO_DEVICE, hp.ERR_CUDA)


def test_batch_instance_bytes(hp):
    k = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=100, ny=30)
    assert hp.Batch.instance_bytes(k) == 3 * 112 * 30 * 6 * 8                # pitch 112, U/S0/S1
    k3 = hp.Config(system=hp.KAPILA_5EQN, order=3, nx=100, ny=30)
    assert hp.Batch.instance_bytes(k3) == 4 * 112 * 30 * 6 * 8               # + S2 for SSPRK(10,4)
    km = hp.Config(system=hp.KAPILA_5EQN, order=2, nx=100, ny=30, precision=hp.PREC_MIXED)
    assert hp.Batch.instance_bytes(km) == 3 * 128 * 30 * (4 * 4 + 2 * 8)     # FP32 x4 + FP64 x2 planes
    assert hp.Batch.instance_bytes(hp.Config(nx=2, ny=2)) == 0                # invalid
