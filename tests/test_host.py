"""Host side of the library: it loads, exports every C-ABI symbol the header
declares, prepares materials and builds octrees exactly like the reference,
and rejects bad inputs with the documented status codes.  CPU only (no
compute call reaches a GPU here)."""
import hashlib
import os
import re
import subprocess

import numpy as np
import pytest

import nebula_b200 as nb
from nebula_b200 import _capi
from conftest import ROOT, load_golden, has_gpu

HEADER = os.path.join(ROOT, "include", "nebula_b200.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nbl_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = nb.lib()
    assert lib.nbl_abi_version() == 1
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (nbl_[a-z0-9_]+)", out))
    declared = header_functions()
    assert declared, "no declarations parsed"
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # the Python binding declares exactly the header's functions
    assert sorted(_capi.declared_symbols()) == declared


def test_library_is_built_for_sm100a_only():
    # every CUDA translation unit is compiled with exactly one -gencode:
    # sm_100a code, no PTX for other targets (the device-side check of the
    # loaded kernel's architecture is test_gpu_edge.py's)
    from nebula_b200 import build as nbuild
    gencodes = [nbuild.NVCC_FLAGS[i + 1] for i, f in enumerate(nbuild.NVCC_FLAGS) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"], gencodes
    assert not any(f.startswith(("-arch", "--gpu-architecture", "-code")) for f in nbuild.NVCC_FLAGS)


@pytest.mark.parametrize("name", ["si", "pmma"])
def test_material_tables_match_reference(inputs, name):
    g = load_golden("tables_%s.npz" % name)
    t = nb.Material.load(inputs[name + ".nmat"]).tables()
    for k in _capi.TABLE_NAMES:
        data, scale = t[k]
        assert list(data.shape) == list(g[k + "_shape"])
        assert hashlib.sha256(np.ascontiguousarray(data).tobytes()).hexdigest() == str(g[k + "_sha256"]), k
        assert np.array_equal(scale.view(np.uint32), g[k + "_scale"].view(np.uint32)), k
    assert np.array_equal(t["constants"].view(np.uint32), g["constants"].view(np.uint32))


@pytest.mark.parametrize("name", ["slab", "grating"])
def test_octree_builder_matches_reference(inputs, name):
    g = nb.Geometry.from_tri_file(inputs[name + ".tri"])
    od, tr = g.export()
    ref = load_golden("octree_%s.npz" % name)
    assert np.array_equal(od, ref["octree_data"])
    mine = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                           tr["r0"], tr["e1"], tr["e2"]], 1)
    assert np.array_equal(mine.view(np.uint32), ref["tri11"].view(np.uint32))
    inf = g.info()
    assert np.array_equal(inf["center"], ref["center"]) and np.array_equal(inf["halfsize"], ref["halfsize"])
    assert np.float32(inf["max_extent"]) == ref["max_extent"]


def test_octree_builder_random_soup_matches_oracle_reference():
    """Random triangle soup with duplicates, slivers and axis-aligned faces,
    against the reference builder when its build is present."""
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference build not present")
    import tempfile
    from nebula_b200.synth import geometry
    rng = np.random.default_rng(3)
    n = 2000
    # small triangles (a point is covered by few of them, so cells do not
    # split without bound), some in the plane z = 0 or on lattice points
    c = rng.uniform(-50, 50, (n, 1, 3))
    v = c + rng.normal(0, 2.0, (n, 3, 3))
    v[:200, :, 2] = 0.0
    v[200:300] = np.round(v[200:300])
    rows = np.concatenate([rng.integers(-1, 3, (n, 2)), v.reshape(n, 9)], 1)
    rows = np.concatenate([rows, rows[:20]])   # duplicates
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "soup.tri")
        geometry.write_tri(p, rows)
        rg = O.RefGeometry(p)
        g = nb.Geometry.from_tri_file(p)
    od, tr = g.export()
    assert np.array_equal(od, rg.octree_data)
    assert np.array_equal(tr["r0"], rg.tri11[:, 2:5])


def test_tri_loader_rejects_bad_rows(tmp_path):
    p = tmp_path / "bad.tri"
    p.write_text("0 -123 0 0 0 1 0 0 0 1 0\n0 -123 0 0 0 1\n")
    with pytest.raises(nb.NblError) as e:
        nb.Geometry.from_tri_file(str(p))
    assert e.value.status == 7


def test_pri_loader(tmp_path):
    """nbl_load_pri_file: whole 36-byte records round-trip; a file whose size
    is not a multiple of 36 is an IO error (load_pri_file.cpp:106-107); a
    missing file too."""
    import ctypes as C
    from nebula_b200 import _capi
    from nebula_b200.synth import primaries
    rec = primaries.point_beam(5)
    good = tmp_path / "good.pri"
    primaries.write_pri(str(good), rec)
    out = C.POINTER(_capi.Record)()
    n = C.c_int64()
    L = nb.lib()
    assert L.nbl_load_pri_file(str(good).encode(), C.byref(out), C.byref(n)) == 0 and n.value == 5
    got = np.frombuffer(C.string_at(out, 36 * n.value), dtype=nb.PRI_DTYPE)
    L.nbl_free(out)
    assert got.tobytes() == rec.tobytes()
    bad = tmp_path / "bad.pri"
    bad.write_bytes(rec.tobytes()[:-5])
    assert L.nbl_load_pri_file(str(bad).encode(), C.byref(out), C.byref(n)) == 7
    assert L.nbl_load_pri_file(b"/nonexistent/file.pri", C.byref(out), C.byref(n)) == 7


def test_missing_material_file():
    with pytest.raises(nb.NblError) as e:
        nb.Material.load("/nonexistent/file.nmat")
    assert e.value.status == 7


def test_truncated_material_file(inputs, tmp_path):
    data = open(inputs["si.nmat"], "rb").read()
    p = tmp_path / "trunc.nmat"
    p.write_bytes(data[: len(data) // 2])
    with pytest.raises(nb.NblError) as e:
        nb.Material.load(str(p))
    assert e.value.status == 7


def test_linearized_octree_validation():
    tr = np.zeros(1, nb.TRI_DTYPE)
    # child offset pointing past the end must be rejected, not walked
    od = np.array([9, 9, 9, 9, 9, 9, 9, 500, -1], np.int32)
    with pytest.raises(nb.NblError) as e:
        nb.Geometry.from_linearized(od, tr, [0, 0, 0], [1, 1, 1])
    assert e.value.status == 1
    # a cycle back to the root
    od = np.array([0, -8, -8, -8, -8, -8, -8, -8, -1], np.int32)
    with pytest.raises(nb.NblError):
        nb.Geometry.from_linearized(od, tr, [0, 0, 0], [1, 1, 1])
    # triangle id out of range
    od = np.array([-8, -8, -8, -8, -8, -8, -8, -8, 3, -1], np.int32)
    with pytest.raises(nb.NblError):
        nb.Geometry.from_linearized(od, tr, [0, 0, 0], [1, 1, 1])
    # a valid one is accepted
    od = np.array([-8, -8, -8, -8, -8, -8, -8, -8, 0, -1], np.int32)
    g = nb.Geometry.from_linearized(od, tr, [0, 0, 0], [1, 1, 1])
    assert g.info()["n_octree"] == 10


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_is_an_error_not_a_fallback(inputs):
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    with pytest.raises(nb.NblError) as e:
        nb.Simulation(g, [m], capacity=1024)
    assert e.value.status in (3, 8)
    with pytest.raises(nb.NblError):
        g.ray_query(np.zeros((1, 3)), np.array([[0, 0, -1.0]]), np.ones(1))


def test_material_count_checked(inputs):
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    with pytest.raises(nb.NblError) as e:
        nb.Simulation(g, [m], capacity=1024)
    assert e.value.status == 1


def test_batch_limits_checked_before_any_device_work(inputs):
    """A batch takes at most 64 geometries (its geometry table lives in each
    block's shared memory): more are an argument error, on any machine."""
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    with pytest.raises(nb.NblError) as e:
        nb.Batch([g] * 65, [m], capacity=1024)
    assert e.value.status == 1 and "64 geometries" in str(e.value)


def test_octree_builder_rough_lines_matches_reference(tmp_path):
    """Line-edge-roughness grating (the large-mesh geometry at reduced
    length: 4 lines, 40 nm long, ~25 k triangles): the multithreaded top-down
    builder gives the reference's incremental builder's octree exactly."""
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference build not present")
    from nebula_b200.synth import geometry
    rows = geometry.rough_grating(n_lines=4, line_length=40.0, size=200.0)
    p = str(tmp_path / "rough.tri")
    geometry.write_tri(p, rows)
    rg = O.RefGeometry(p)
    g = nb.Geometry.from_tri_file(p)
    od, tr = g.export()
    assert len(tr) > 10000
    assert np.array_equal(od, rg.octree_data)
    assert np.array_equal(tr["r0"], rg.tri11[:, 2:5])
    assert np.array_equal(tr["e2"], rg.tri11[:, 8:11])
