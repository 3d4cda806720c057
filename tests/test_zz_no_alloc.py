"""hype_rhs_prim_noalloc: the RHSFunctionPrim entry point for callers that
cannot allocate device memory (a plug-in inside an application whose memory
pool owns the GPU, or a time loop that must not pay for cudaMalloc/cudaFree).

It must give the same result as the allocating entry point
(hype_rhs_prim_device): bit for bit, which is the tolerance of this suite, on
two calls in a row (the second call finds the first call's leftovers in the
shared static scratch).  This file is named to be collected last.
"""
import ctypes

import pytest

import cases

pytestmark = pytest.mark.gpu


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


def test_noalloc_matches_allocating_entry_point_two_calls_in_a_row(hp):
    import torch
    L = _bind(hp)
    runs = [cases.case_by_name("kapila_37x23_rough_mixed_bc"), cases.case_by_name("bn_23x19_fixed_p2")]
    for name, cfg, kind, seed in runs:
        pcfg = cases.to_pkg(cfg)
        U = cases.state(cfg, kind, seed)
        dU = torch.from_numpy(U).cuda()
        dR_ref = torch.full_like(dU, float("nan"))
        with hp.Solver(pcfg) as s:
            dt_ref, st_ref = s.rhs_function_prim_device(0.0, dU.data_ptr(), dR_ref.data_ptr())
        assert st_ref == hp.OK
        ref = dR_ref.cpu().numpy()
        for call in range(2):
            dR = torch.full_like(dU, float("nan"))
            st, dt = _noalloc(hp, L, pcfg, dU, dR)
            assert st == hp.OK, (name, call, st)
            assert dt == dt_ref, (name, call)
            assert dR.cpu().numpy().tobytes() == ref.tobytes(), (name, call)


def test_noalloc_rejects_grids_beyond_its_scratch(hp):
    L = _bind(hp)
    big = hp.Config(system=hp.KAPILA_5EQN, nx=1024, ny=1024)   # 48 MiB of planes > 16 MiB
    dt = ctypes.c_double(0.0)
    st = L.hype_rhs_prim_noalloc(ctypes.byref(big.c_struct()), 0.0, None, None, ctypes.byref(dt))
    assert st == hp.ERR_NOMEM
    inlet = hp.Config(system=hp.KAPILA_5EQN, nx=32, ny=32, bc_left=hp.BC_INLET)
    st = L.hype_rhs_prim_noalloc(ctypes.byref(inlet.c_struct()), 0.0, None, None, ctypes.byref(dt))
    assert st == hp.ERR_INVALID
