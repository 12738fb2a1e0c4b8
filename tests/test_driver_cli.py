"""The command-line drivers: nebula_b200/nebula_b200_gpu, a drop-in for the
reference's GPU executable (gpu_main.cu): same positional arguments and
options, 36-byte detected-electron records on stdout; and
nebula_b200/nebula_b200_edep, the same for its energy-deposit executable
(cpu_energydep.cpp): 28-byte deposit records and a detected-record file.

CPU: usage and argument errors (exit status 1, nothing on stdout), the
material-count check of gpu_main.cu:322-343.  GPU: the records it writes
are exactly the records the library's API gives for the same primaries and
seed (counter-based random numbers make the run independent of how it is
driven), and its physics switches reach the transport.
"""
import os
import subprocess

import numpy as np
import pytest

import nebula_b200 as nb
from nebula_b200 import build
from conftest import has_gpu

DRIVER = build.DRIVER


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(DRIVER):
        build.build()
    assert os.path.exists(DRIVER)
    return DRIVER


@pytest.fixture(scope="module")
def slab_files(tmp_path_factory):
    from nebula_b200.synth import workloads, geometry, materials, nmat, primaries
    d = tmp_path_factory.mktemp("cli")
    w = workloads.slab(n_primaries=50_000)
    tri = str(d / "slab.tri")
    geometry.write_tri(tri, w.triangles)
    mat = str(d / "si.nmat")
    nmat.write(mat, materials.build_raw_material(w.material_specs[0]))
    pri = str(d / "slab.pri")
    p = w.primaries.copy()
    p["px"] = np.arange(len(p)) % 100
    primaries.write_pri(pri, p)
    return tri, pri, mat, p


def _run(args, timeout=300):
    return subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)


def test_usage_and_bad_arguments(driver, slab_files):
    tri, pri, mat, _ = slab_files
    r = _run([driver])
    assert r.returncode == 1 and r.stdout == b"" and b"Usage: nebula_b200_gpu" in r.stderr
    assert b"--record-buffer" in r.stderr and b"--workers-per-device" in r.stderr
    r = _run([driver, "--no-such-option", "1", tri, pri, mat])
    assert r.returncode == 1 and b"unknown option --no-such-option" in r.stderr
    # the slab needs material 0: none given
    r = _run([driver, tri, pri])
    assert r.returncode == 1 and r.stdout == b""
    # the physics banner reports the selection (before any device call)
    r = _run([driver, "--inelastic-model", "1", "--interface-absorption", "1", tri, pri, mat])
    assert b"inelastic: kieft_inelastic" in r.stderr and b"interface absorption 1" in r.stderr
    # the reference parser's other forms: --key=value and --key = value
    r = _run([driver, "--inelastic-model=1", "--interface-absorption", "=", "1", tri, pri, mat])
    assert b"inelastic: kieft_inelastic" in r.stderr and b"interface absorption 1" in r.stderr


def test_not_enough_materials(driver, tmp_path):
    from nebula_b200.synth import workloads, geometry, materials, nmat, primaries
    w = workloads.grating(nx=2, ny=2, per_pixel=10)
    tri = str(tmp_path / "g.tri")
    geometry.write_tri(tri, w.triangles)
    mat = str(tmp_path / "si.nmat")
    nmat.write(mat, materials.build_raw_material(w.material_specs[0]))
    pri = str(tmp_path / "g.pri")
    primaries.write_pri(pri, w.primaries)
    r = _run([driver, tri, pri, mat])
    assert r.returncode == 1 and b"not enough materials" in r.stderr and r.stdout == b""


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_records_equal_the_api_run(driver, slab_files):
    """The default page-locked record buffers; buffers of 3 000 records over
    ranges of 20 000 primaries (steps stop on a full buffer, records that did
    not fit carried into the next one, several times within a graph); and
    the device buffer drained between steps: the same records each time."""
    tri, pri, mat, p = slab_files
    sim = nb.Simulation(nb.Geometry.from_tri_file(tri), [nb.Material.load(mat)], capacity=1 << 20, seed=4242)
    sim.push(p)
    sim.run()
    ref = sim.flush_detected()
    sim.close()
    key = lambda a: np.sort(a.view(np.dtype((np.void, 36))).ravel()).tobytes()
    for extra in ([], ["--record-buffer", "3000", "--chunk", "20000"], ["--record-buffer", "0"]):
        r = _run([driver, "--seed", "4242", "--capacity", "65536"] + extra + [tri, pri, mat])
        assert r.returncode == 0, r.stderr[-2000:]
        assert b"Simulation successful" in r.stderr and b"Timing (seconds):" in r.stderr
        got = np.frombuffer(r.stdout, dtype=nb.PRI_DTYPE)
        assert len(got) == len(ref) > 0.5 * len(p), extra
        assert key(got) == key(ref), extra
        assert ("%d detected electrons written" % len(ref)).encode() in r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_physics_switches_and_sorting(driver, slab_files):
    tri, pri, mat, p = slab_files
    base = _run([driver, "--seed", "7", tri, pri, mat])
    assert base.returncode == 0
    a = np.frombuffer(base.stdout, dtype=nb.PRI_DTYPE)
    # no secondaries: no SE peak below 50 eV beyond what backscatter leaves
    nose = _run([driver, "--seed", "7", "--generate-secondaries", "0", tri, pri, mat])
    assert nose.returncode == 0
    b = np.frombuffer(nose.stdout, dtype=nb.PRI_DTYPE)
    assert (b["E"] < 50).sum() < 0.2 * (a["E"] < 50).sum()
    # sorted primaries: a different assignment of random streams, same physics
    srt = _run([driver, "--seed", "7", "--sort-primaries", "1", tri, pri, mat])
    assert srt.returncode == 0
    c = np.frombuffer(srt.stdout, dtype=nb.PRI_DTYPE)
    n = len(p)
    for sel in (lambda x: x["E"] < 50, lambda x: x["E"] >= 50):
        ya, yc = sel(a).sum(), sel(c).sum()
        assert abs(ya - yc) < 5 * np.sqrt(2.0 * max(ya, 1)) * 1.5, (ya, yc, n)


def test_edep_usage(driver):
    edep = build.DRIVER_EDEP
    assert os.path.exists(edep)
    r = _run([edep])
    assert r.returncode == 1 and b"Usage: nebula_b200_edep" in r.stderr
    assert b"--deposit-filename" in r.stderr and b"--detect-filename" in r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_edep_outputs_equal_the_api_run(driver, slab_files, tmp_path):
    """nebula_b200_edep (cpu_energydep.cpp's command line): the deposit
    stream (default stdout) and the detected file are exactly the API's
    deposit records and detected records of the same run."""
    tri, pri, mat, p = slab_files
    det = str(tmp_path / "det.bin")
    r = _run([build.DRIVER_EDEP, "--seed", "99", "--detect-filename", det, tri, pri, mat])
    assert r.returncode == 0, r.stderr[-2000:]
    dep = np.frombuffer(r.stdout, dtype=nb.DEPOSIT_DTYPE)
    got_det = np.fromfile(det, dtype=nb.PRI_DTYPE)
    sim = nb.Simulation(nb.Geometry.from_tri_file(tri), [nb.Material.load(mat)], capacity=1 << 20, seed=99,
                        deposit_capacity=1 << 24)
    sim.push(p)
    sim.run()
    ref_dep = sim.drain_deposits()
    ref_det = sim.flush_detected()
    sim.close()
    key = lambda a, n: np.sort(a.view(np.dtype((np.void, n))).ravel()).tobytes()
    assert len(dep) == len(ref_dep) > 10 * len(p)
    assert key(dep, 28) == key(ref_dep, 28)
    assert key(got_det, 36) == key(ref_det, 36)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_split_files_with_first_primary_equal_one_run(driver, slab_files, tmp_path):
    """Two processes on the two halves of the primaries, the second with
    --first-primary, write together exactly the records of one run."""
    from nebula_b200.synth import primaries
    tri, pri, mat, p = slab_files
    k = len(p) // 2 + 3
    a, b = str(tmp_path / "a.pri"), str(tmp_path / "b.pri")
    primaries.write_pri(a, p[:k])
    primaries.write_pri(b, p[k:])
    whole = _run([driver, "--seed", "5", tri, pri, mat])
    ra = _run([driver, "--seed", "5", tri, a, mat])
    rb = _run([driver, "--seed", "5", "--first-primary", str(k), tri, b, mat])
    assert whole.returncode == ra.returncode == rb.returncode == 0
    key = lambda buf: np.sort(np.frombuffer(buf, dtype=np.dtype((np.void, 36)))).tobytes()
    assert key(ra.stdout + rb.stdout) == key(whole.stdout)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error(driver, slab_files):
    tri, pri, mat, _ = slab_files
    r = _run([driver, tri, pri, mat])
    assert r.returncode == 1 and r.stdout == b"" and b"no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_workers_sharing_the_primaries_equal_one_run(driver, slab_files, tmp_path):
    """The worker-per-device fan-out (gpu_main.cu:284-295), run here as two
    workers on device 0 taking 7001-primary ranges from the shared cursor:
    the records equal, as a set, one worker's run over the whole file; the
    same for the energy-deposit executable's two outputs."""
    tri, pri, mat, p = slab_files
    one = _run([driver, "--seed", "13", "--device", "0", tri, pri, mat])
    two = _run([driver, "--seed", "13", "--devices", "0", "--workers-per-device", "2", "--chunk", "7001",
                tri, pri, mat])
    assert one.returncode == two.returncode == 0, two.stderr[-2000:]
    assert b"2 worker(s)" in two.stderr
    key = lambda buf, n: np.sort(np.frombuffer(buf, dtype=np.dtype((np.void, n)))).tobytes()
    assert len(one.stdout) == len(two.stdout) > 0
    assert key(two.stdout, 36) == key(one.stdout, 36)
    d1, d2 = str(tmp_path / "d1.bin"), str(tmp_path / "d2.bin")
    e1 = _run([build.DRIVER_EDEP, "--seed", "3", "--detect-filename", d1, tri, pri, mat])
    e2 = _run([build.DRIVER_EDEP, "--seed", "3", "--detect-filename", d2, "--devices", "0",
               "--workers-per-device", "2", "--chunk", "9000", tri, pri, mat])
    assert e1.returncode == e2.returncode == 0, e2.stderr[-2000:]
    assert key(e2.stdout, 28) == key(e1.stdout, 28)
    assert key(open(d2, "rb").read(), 36) == key(open(d1, "rb").read(), 36)
