"""The reference's file formats from the device state (hype_io.cu).

Restart files are PETSc binary Vecs (big-endian class id 1211214, length,
doubles in Vec order); solution files are VTK XML structured grids of the
primitive variables with the DMDA's cell-centre coordinates, which
HyPE-2D/plot.py reads field by field.  The files are parsed here byte by byte.
"""
import os
import re
import shutil
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture
def outdir(request):
    d = os.path.join(ROOT, "tests", "_scratch", request.node.name.replace("[", "_").replace("]", ""))
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    yield d
    shutil.rmtree(d, ignore_errors=True)


def kapila_cfg(hp, nx=40, ny=30, **kw):
    return hp.Config(system=hp.KAPILA_5EQN, order=2, nx=nx, ny=ny, cfl=0.4, **kw)


def read_petsc_vec(path):
    raw = open(path, "rb").read()
    cid, n = struct.unpack(">ii", raw[:8])
    assert cid == 1211214 and len(raw) == 8 + 8 * n
    return np.frombuffer(raw[8:], dtype=">f8").astype(np.float64)


def read_vts(path):
    raw = open(path, "rb").read()
    head, _, data = raw.partition(b"<AppendedData encoding=\"raw\">\n_")
    text = head.decode()
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', text).group(1).split()]
    arrays = re.findall(r'<DataArray type="Float64" Name="([^"]+)" NumberOfComponents="(\d)" format="appended" offset="(\d+)"',
                        text)
    out = {}
    for name, ncomp, off in arrays:
        off = int(off)
        nbytes = struct.unpack("<Q", data[off:off + 8])[0]
        out[name] = np.frombuffer(data[off + 8:off + 8 + nbytes], dtype="<f8").reshape(-1, int(ncomp))
    return ext, [a[0] for a in arrays], out


def test_restart_roundtrip_and_layout(hp, outdir):
    cfg = kapila_cfg(hp)
    U0 = hp.initial_state(cfg, "shock_bubble", seed=3, nbubbles=2)
    path = os.path.join(outdir, "restart1.bin")
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        s.solve(0.0, 1e30, 5)
        U5 = s.get_state()
        s.write_restart(path)
    assert read_petsc_vec(path).tobytes() == U5.tobytes()
    assert open(path + ".info").read() == "-vecload_block_size 6\n"
    with hp.Solver(cfg) as s:
        assert s.read_restart(path) == hp.OK
        assert s.get_state().tobytes() == U5.tobytes()
    with hp.Solver(kapila_cfg(hp, 41, 30)) as s:   # another grid: VecLoad size mismatch
        assert s.read_restart(path) == hp.ERR_INVALID


def cons2prim_kapila(U, g1, g2, pi1, pi2):
    """kapila_5eqn.c:14-35 in numpy, same operation order."""
    Q = U.reshape(-1, 6)
    a1 = Q[:, 5]
    a2 = 1.0 - a1
    rho = Q[:, 0] + Q[:, 1]
    u = Q[:, 2] / rho
    v = Q[:, 3] / rho
    ei = Q[:, 4] - 0.5 * rho * (u * u + v * v)
    G1, G2 = g1 - 1.0, g2 - 1.0
    p = (ei * G1 * G2 - a1 * g1 * pi1 * G2 - a2 * g2 * pi2 * G1) / (a1 * G2 + a2 * G1)
    return np.stack([Q[:, 0] / a1, Q[:, 1] / a2, u, v, p, a1], -1)


@pytest.mark.parametrize("periodic", [False, True])
def test_vts_fields_and_dmda_coordinates(hp, outdir, periodic):
    T, P = hp.BC_TRANSMISSIVE, hp.BC_PERIODIC
    b = P if periodic else T
    cfg = kapila_cfg(hp, 40, 30, x_min=0.0, x_max=2.0, y_min=-1.0, y_max=0.5, bc_left=b, bc_right=b, bc_bottom=b, bc_top=b)
    U0 = hp.initial_state(cfg, "shock_bubble", seed=4, nbubbles=1)
    path = os.path.join(outdir, "sol.vts")
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        W = s.get_primitive()
        s.write_vts(path)
    np.testing.assert_array_equal(W.reshape(-1, 6), cons2prim_kapila(U0, cfg.gamma1, cfg.gamma2, cfg.pi1, cfg.pi2))
    ext, names, arr = read_vts(path)
    assert ext == [0, 39, 0, 29, 0, 0]
    assert names == ["Position", "sol.density1", "sol.density2", "sol.x-velocity", "sol.y-velocity", "sol.pressure",
                     "sol.phi"]
    for c, nm in enumerate(names[1:]):
        assert arr[nm][:, 0].tobytes() == W.reshape(-1, 6)[:, c].tobytes()
    h = 2.0 / 40
    hx = 2.0 / (40 if periodic else 39)
    hy = 1.5 / (30 if periodic else 29)
    X = arr["Position"].reshape(30, 40, 3)
    np.testing.assert_array_equal(X[0, :, 0], (0.0 + 0.5 * h) + hx * np.arange(40))
    np.testing.assert_array_equal(X[:, 0, 1], (-1.0 + 0.5 * h) + hy * np.arange(30))
    assert np.all(X[..., 2] == 0.0)


def test_solve_monitored_writes_the_monitor_schedule(hp, outdir):
    cfg = kapila_cfg(hp, 32, 24)
    U0 = hp.initial_state(cfg, "shock_bubble", seed=5, nbubbles=1)
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        steps, t, _ = s.solve_monitored(0.0, 1e30, 12, 5, 4, outdir)
    assert steps == 12
    files = sorted(os.listdir(outdir))
    assert files == ["restart1.bin", "restart1.bin.info", "restart2.bin", "restart2.bin.info", "sol-00000000.vts",
                     "sol-00000005.vts", "sol-00000010.vts", "sol-00000012.vts"]
    # restart1 last written at step 12 (12 % 4 == 0), restart2 at step 9 ((9 + 7) % 4 == 0)
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        s.solve(0.0, 1e30, 12)
        assert read_petsc_vec(os.path.join(outdir, "restart1.bin")).tobytes() == s.get_state().tobytes()
        s.set_state(U0)
        s.solve(0.0, 1e30, 9)
        assert read_petsc_vec(os.path.join(outdir, "restart2.bin")).tobytes() == s.get_state().tobytes()


def test_monitor_files_equal_the_reference_files(hp, outdir):
    """The GPU's monitored solve against the reference's own MonitorFunction
    (post_process.c:12-64) and final write (hype.c:389-400) run through the PETSc
    stand-in on the same state: the same file names, restart files equal byte for
    byte (header, big-endian data, .info), and each .vts data array equal to the
    primitive variables the reference hands its VTK viewer.  Then each side reads
    the other's restart1.bin (hype.c:316-325 VecLoad; hype_read_restart) and both
    resume 6 steps from it to the same bits."""
    import cases
    import oracle as O
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    ocfg = O.Config(system=O.KAPILA, order=2, nx=36, ny=26, cfl=0.4, gamma1=4.4, gamma2=1.4, pi1=6.0e8, pi2=0.0)
    U0 = O.initial_state(ocfg, "shock_bubble", seed=11, nbubbles=2)
    gdir, rdir = os.path.join(outdir, "gpu"), os.path.join(outdir, "ref")
    os.makedirs(gdir)
    os.makedirs(rdir)
    cfg = cases.to_pkg(ocfg)
    with hp.Solver(cfg) as s:
        s.set_state(U0)
        steps, t, _ = s.solve_monitored(0.0, 1e30, 14, 4, 3, gdir)
        Ug = s.get_state()
    ref = O.Reference(O.KAPILA)
    ref.setup(ocfg)
    ref.set_output(4, 3)
    here = os.getcwd()
    os.chdir(rdir)
    try:
        Ur, n, tr, _, st = ref.solve(U0, 0.0, 1e30, 14)
        assert st == 0 and ref.write_final(n) == 0
    finally:
        os.chdir(here)
    assert (steps, float(t).hex()) == (n, float(tr).hex())
    assert Ug.tobytes() == Ur.tobytes()
    gfiles, rfiles = sorted(os.listdir(gdir)), sorted(os.listdir(rdir))
    assert gfiles == rfiles
    for f in gfiles:
        if f.startswith("restart"):
            assert open(os.path.join(gdir, f), "rb").read() == open(os.path.join(rdir, f), "rb").read(), f
        else:
            _, names, arr = read_vts(os.path.join(gdir, f))
            W = np.fromfile(os.path.join(rdir, f), dtype="<f8").reshape(-1, 6)
            for c, nm in enumerate(names[1:]):
                assert arr[nm][:, 0].tobytes() == W[:, c].tobytes(), (f, nm)
    # cross reads of the GPU's restart1.bin (last written at step 12), then 6 more
    # steps from the restart state on each side
    U12 = read_petsc_vec(os.path.join(gdir, "restart1.bin"))
    os.replace(os.path.join(gdir, "restart1.bin"), os.path.join(rdir, "restart1.bin"))
    os.chdir(rdir)
    try:
        Ul, rc = ref.load_restart()
    finally:
        os.chdir(here)
    assert rc == 0 and Ul.tobytes() == U12.tobytes()
    ref.set_output(0, 0)
    Ur6, n6, t6, dt6, st6 = ref.solve(Ul, 0.0, 1e30, 6)
    with hp.Solver(cfg) as s:
        assert s.read_restart(os.path.join(rdir, "restart1.bin")) == hp.OK
        assert s.get_state().tobytes() == U12.tobytes()
        g6, tg6, dtg6, stg6 = s.solve(0.0, 1e30, 6)
        assert stg6 == hp.OK and (g6, float(tg6).hex(), float(dtg6).hex()) == (n6, float(t6).hex(), float(dt6).hex())
        assert s.get_state().tobytes() == Ur6.tobytes()
