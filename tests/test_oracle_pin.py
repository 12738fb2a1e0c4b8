"""The oracle (oracle/nbl_oracle.cpp, a CPU restatement of the reference
path) against golden fixtures made by the reference itself
(tests/golden/make_golden.py), and against the reference build when
oracle/_ref is present.  CPU only."""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_inputs_match_fixture_generation(inputs):
    g = load_golden("inputs_sha256.npz")
    for k in ("slab.tri", "grating.tri", "si.nmat", "pmma.nmat"):
        assert _sha(inputs[k]) == str(g[k.replace(".", "_")]), "synthetic generator changed: " + k


@pytest.mark.parametrize("name", ["si", "pmma"])
def test_oracle_tables_match_reference(inputs, name):
    g = load_golden("tables_%s.npz" % name)
    m = O.Material(inputs[name + ".nmat"])
    for t in O.TABLE_NAMES:
        data, scale = m.table(t)
        assert list(data.shape) == list(g[t + "_shape"])
        assert hashlib.sha256(np.ascontiguousarray(data).tobytes()).hexdigest() == str(g[t + "_sha256"]), t
        assert np.array_equal(scale.view(np.uint32), g[t + "_scale"].view(np.uint32)), t
    assert np.array_equal(m.constants().view(np.uint32), g["constants"].view(np.uint32))


def _golden_geometry(name):
    o = load_golden("octree_%s.npz" % name)
    return O.Geometry(o["octree_data"], o["tri11"], o["center"], o["halfsize"], float(o["max_extent"]))


@pytest.mark.parametrize("name", ["slab", "grating"])
def test_oracle_octree_walk_bit_exact(name):
    g = _golden_geometry(name)
    r = load_golden("rays_%s.npz" % name)
    od, ot = g.propagate(r["pos"], r["dir"], r["dist"], r["ignore_tri"], r["ignore_mat"])
    assert np.array_equal(ot, r["out_tri"])
    assert np.array_equal(od.view(np.uint32), r["out_dist"].view(np.uint32))


def test_oracle_driver_records_bit_exact(inputs):
    """Single-threaded CPU driver loop: the oracle reproduces the reference's
    detected-electron records byte for byte (400 primaries, 1 keV, slab)."""
    gold = load_golden("records_slab.npz")
    g = _golden_geometry("slab")
    m = O.Material(inputs["si.nmat"])
    from nebula_b200.synth import primaries
    pri = primaries.point_beam(int(gold["n_primaries"]))
    rec, tot, ev = O.simulate(g, [m], pri, int(gold["seed"]))
    assert ev == int(gold["n_events"])
    assert tot == int(gold["n_total"])
    assert rec.view(np.uint8).tobytes() == gold["records"].tobytes()


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_events_bit_exact_vs_reference(inputs):
    """Single events with the reference mt19937 stream: identical outputs."""
    rg = O.RefGeometry(inputs["grating.tri"])
    og = rg.oracle_geometry()
    rms = [O.RefMaterial(inputs["si.nmat"]), O.RefMaterial(inputs["pmma.nmat"])]
    oms = [O.Material(inputs["si.nmat"]), O.Material(inputs["pmma.nmat"])]
    rng = np.random.default_rng(5)
    for it in range(600):
        E = float(np.exp(rng.uniform(np.log(13), np.log(9000))))
        d = rng.standard_normal(3)
        st = np.array([rng.uniform(-60, 60), rng.uniform(-60, 60), rng.uniform(-50, 30), *d, E], np.float32)
        kind = int(rng.integers(1, 4))
        mat = int(rng.integers(0, 2))
        tri = int(rng.integers(0, len(rg.tri11))) if kind == 3 else -1
        if kind == 3:
            mat = int(rng.choice([0, 1, -123]))
        seed = int(rng.integers(0, 2 ** 32))
        a = O.ref_event(rg, rms, kind, st, mat, seed, tri)
        h = O.lib().orc_rng_mt(seed)
        b = O.event(og, oms, kind, st, mat, h, tri)
        O.lib().orc_rng_free(h)
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)), (kind, st, mat, tri)
        assert a[1:3] == b[1:3]
        assert (a[3] is None) == (b[3] is None)
        if a[3] is not None:
            assert np.array_equal(a[3].view(np.uint32), b[3].view(np.uint32))


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_grating_records_bit_exact_vs_reference(inputs):
    rg = O.RefGeometry(inputs["grating.tri"])
    og = rg.oracle_geometry()
    rms = [O.RefMaterial(inputs["si.nmat"]), O.RefMaterial(inputs["pmma.nmat"])]
    oms = [O.Material(inputs["si.nmat"]), O.Material(inputs["pmma.nmat"])]
    from nebula_b200.synth import workloads
    w = workloads.grating(pixels=[(100, 120), (101, 120), (140, 30)], per_pixel=60)
    a = O.ref_simulate(rg, rms, w.primaries, 77)
    b = O.simulate(og, oms, w.primaries, 77)
    assert a[2] == b[2] and a[1] == b[1]
    assert a[0].tobytes() == b[0].tobytes()


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_deposits_bit_exact_vs_reference(inputs):
    """Energy-deposit driver (energydeposit_cpu_driver.h:44-93): the oracle's
    deposit records equal the reference's byte for byte (grating, 2 pixels x
    30 primaries, one thread)."""
    rg = O.RefGeometry(inputs["grating.tri"])
    og = rg.oracle_geometry()
    rms = [O.RefMaterial(inputs["si.nmat"]), O.RefMaterial(inputs["pmma.nmat"])]
    oms = [O.Material(inputs["si.nmat"]), O.Material(inputs["pmma.nmat"])]
    from nebula_b200.synth import workloads
    w = workloads.grating(pixels=[(100, 120), (140, 30)], per_pixel=30)
    a = O.ref_simulate_deposits(rg, rms, w.primaries, 41)
    b, ev = O.simulate_deposits(og, oms, w.primaries, 41)
    assert len(a) > 1000
    assert a.tobytes() == b.tobytes()
    assert np.all(a["loss"] != 0)
