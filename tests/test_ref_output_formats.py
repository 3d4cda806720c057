"""The reference's own output and restart path, run through the PETSc stand-in.

MonitorFunction (post_process.c:12-64) writes restart1.bin / restart2.bin with
VecView on a binary viewer and sol-%08d.vts with VecView on a VTK viewer;
hype.c:316-325 reads restart1.bin back with VecLoad.  The stand-in's binary
viewer follows PETSc's published binary Vec layout (big-endian class id
1211214, length, big-endian doubles in natural order; "-vecload_block_size
<dof>" in <name>.info); its VTK viewer writes the viewed Vec's values as raw
doubles, the numbers a .vts file carries.  These tests pin that the reference's
schedule and values come out of the stand-in, so that the GPU's files can be
compared with them (tests/test_gpu_io.py).
"""
import os
import struct

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")

KAP = dict(gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)


def read_petsc_vec(path):
    raw = open(path, "rb").read()
    cid, n = struct.unpack(">ii", raw[:8])
    assert cid == 1211214 and len(raw) == 8 + 8 * n
    return np.frombuffer(raw[8:], dtype=">f8").astype(np.float64)


def run_in(d, fn):
    here = os.getcwd()
    os.chdir(d)
    try:
        return fn()
    finally:
        os.chdir(here)


def test_reference_monitor_schedule_and_restart_roundtrip(tmp_path):
    cfg = O.Config(system=O.KAPILA, order=2, nx=32, ny=24, cfl=0.4, **KAP)
    U0 = O.initial_state(cfg, "shock_bubble", seed=5, nbubbles=1)
    ref = O.Reference(O.KAPILA)
    ref.setup(cfg)
    ref.set_output(5, 4)
    Ue, n, t, dt, st = run_in(tmp_path, lambda: ref.solve(U0, 0.0, 1e30, 12))
    assert st == 0 and n == 12
    assert run_in(tmp_path, lambda: ref.write_final(n)) == 0
    assert sorted(os.listdir(tmp_path)) == ["restart1.bin", "restart1.bin.info", "restart2.bin", "restart2.bin.info",
                                           "sol-00000000.vts", "sol-00000005.vts", "sol-00000010.vts",
                                           "sol-00000012.vts"]
    assert open(tmp_path / "restart1.bin.info").read() == "-vecload_block_size 6\n"
    # restart1 last written at step 12, restart2 at step 9: the same run cut there
    assert read_petsc_vec(tmp_path / "restart1.bin").tobytes() == Ue.tobytes()
    ref.set_output(0, 0)
    U9, *_ = ref.solve(U0, 0.0, 1e30, 9)
    assert read_petsc_vec(tmp_path / "restart2.bin").tobytes() == U9.tobytes()
    # the solution file holds the primitive variables (post_process.c:165-200) of the final state
    W = np.fromfile(tmp_path / "sol-00000012.vts", dtype="<f8")
    assert W.size == Ue.size and np.isfinite(W).all()
    assert W.reshape(-1, 6)[:, 5].tobytes() == Ue.reshape(-1, 6)[:, 5].tobytes()   # phi = alpha_1
    # hype.c:316-325 reads restart1.bin back bit for bit
    Ul, rc = run_in(tmp_path, ref.load_restart)
    assert rc == 0 and Ul.tobytes() == Ue.tobytes()


def test_reference_load_rejects_another_grid(tmp_path):
    cfg = O.Config(system=O.KAPILA, order=2, nx=20, ny=16, cfl=0.4, **KAP)
    U0 = O.initial_state(cfg, "shock_bubble", seed=1, nbubbles=1)
    ref = O.Reference(O.KAPILA)
    ref.setup(cfg)
    ref.set_output(0, 1)
    run_in(tmp_path, lambda: ref.solve(U0, 0.0, 1e30, 1))
    ref.setup(O.Config(system=O.KAPILA, order=2, nx=21, ny=16, cfl=0.4, **KAP))
    _, rc = run_in(tmp_path, ref.load_restart)
    assert rc == 1
