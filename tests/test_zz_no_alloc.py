"""hype_rhs_prim_noalloc: the RHSFunctionPrim entry point for callers that
cannot allocate device memory (a plug-in inside an application whose memory
pool owns the GPU, or a time loop that must not pay for cudaMalloc/cudaFree).

It must give the same result as the allocating entry point
(hype_rhs_prim_device): bit for bit, which is the tolerance of this suite, on
two calls in a row (the second call finds the first call's leftovers in the
shared static scratch); on the golden cases that is also the reference's own
SHA-256.  Its calls must leave the device's free memory unchanged, and its size
limit is exact: Kapila 590 x 590 fits the 16 MiB scratch, 591 x 591 is
refused.  This file is named to be collected last.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))


def _bind(hp):
    L = hp.lib()
    L.hype_rhs_prim_noalloc.argtypes = [ctypes.POINTER(hp._Cfg), ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_double)]
    L.hype_rhs_prim_noalloc.restype = ctypes.c_int
    return L


def _noalloc(hp, L, pcfg, dU, dR):
    dt = ctypes.c_double(0.0)
    st = L.hype_rhs_prim_noalloc(ctypes.byref(pcfg.c_struct()), 0.0, ctypes.c_void_p(dU.data_ptr()),
                                 ctypes.c_void_p(dR.data_ptr()), ctypes.byref(dt))
    return st, dt.value


def _allocating(hp, pcfg, dU):
    import torch
    dR = torch.full_like(dU, float("nan"))
    with hp.Solver(pcfg) as s:
        dt, st = s.rhs_function_prim_device(0.0, dU.data_ptr(), dR.data_ptr())
    assert st == hp.OK
    return dR.cpu().numpy(), dt


@pytest.mark.parametrize("name", ["kapila_37x23_rough_mixed_bc", "bn_23x19_fixed_p2", "kapila_24x24_periodic"])
def test_noalloc_matches_allocating_entry_point_two_calls_in_a_row(hp, name):
    import torch
    L = _bind(hp)
    _, cfg, kind, seed = cases.case_by_name(name)
    pcfg = cases.to_pkg(cfg)
    U = cases.state(cfg, kind, seed)
    dU = torch.from_numpy(U).cuda()
    ref, dt_ref = _allocating(hp, pcfg, dU)
    for call in range(2):
        dR = torch.full_like(dU, float("nan"))
        st, dt = _noalloc(hp, L, pcfg, dU, dR)
        assert st == hp.OK, (name, call, st)
        assert dt == dt_ref, (name, call)
        out = dR.cpu().numpy()
        assert out.tobytes() == ref.tobytes(), (name, call)
        assert hashlib.sha256(out.tobytes()).hexdigest() == GOLDEN["rhs"][name]["sha_RHS"]
        assert float(dt).hex() == GOLDEN["rhs"][name]["dt"]


def test_noalloc_calls_leave_free_device_memory_unchanged(hp):
    import torch
    L = _bind(hp)
    _, cfg, kind, seed = cases.case_by_name("kapila_37x23_rough_mixed_bc")
    pcfg = cases.to_pkg(cfg)
    dU = torch.from_numpy(cases.state(cfg, kind, seed)).cuda()
    dR = torch.empty_like(dU)
    assert _noalloc(hp, L, pcfg, dU, dR)[0] == hp.OK   # the first call on the device loads the module
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert _noalloc(hp, L, pcfg, dU, dR)[0] == hp.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_size_limit_is_exact(hp):
    """256 + ceil16(nx) * ny * nvar * 8 <= 16 MiB: Kapila 590^2 (592 * 590 * 48 + 256
    bytes) fits, 591^2 does not."""
    import torch
    L = _bind(hp)
    cfg = O.Config(system=O.KAPILA, order=2, nx=590, ny=590, **cases.KAPILA_EOS)
    pcfg = cases.to_pkg(cfg)
    dU = torch.from_numpy(O.initial_state(cfg, "shock_bubble", seed=5, nbubbles=2)).cuda()
    ref, dt_ref = _allocating(hp, pcfg, dU)
    dR = torch.full_like(dU, float("nan"))
    st, dt = _noalloc(hp, L, pcfg, dU, dR)
    assert st == hp.OK and dt == dt_ref
    assert dR.cpu().numpy().tobytes() == ref.tobytes()
    over = cases.to_pkg(O.Config(system=O.KAPILA, order=2, nx=591, ny=591, **cases.KAPILA_EOS))
    assert _noalloc(hp, L, over, dU, dR)[0] == hp.ERR_NOMEM


def test_noalloc_rejects_grids_beyond_its_scratch(hp):
    L = _bind(hp)
    big = hp.Config(system=hp.KAPILA_5EQN, nx=1024, ny=1024)   # 48 MiB of planes > 16 MiB
    dt = ctypes.c_double(0.0)
    st = L.hype_rhs_prim_noalloc(ctypes.byref(big.c_struct()), 0.0, None, None, ctypes.byref(dt))
    assert st == hp.ERR_NOMEM
    inlet = hp.Config(system=hp.KAPILA_5EQN, nx=32, ny=32, bc_left=hp.BC_INLET)
    st = L.hype_rhs_prim_noalloc(ctypes.byref(inlet.c_struct()), 0.0, None, None, ctypes.byref(dt))
    assert st == hp.ERR_INVALID
