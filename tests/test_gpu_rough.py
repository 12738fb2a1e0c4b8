"""Large-mesh plain method: the line-edge-roughness grating (16 lines, 1.2 M
triangles, octree depth <= 12, <= 16 triangles per leaf) at 300 eV.

The octree comes from this library's multithreaded builder (shown identical
to the reference builder in tests/test_host.py); the oracle runs the
reference's CPU driver loop on the same octree.  SE/BSE yields of a 32 x 32
pixel block agree within 3 sigma, the detected energy and polar-angle
distributions pass a two-sample KS test at p > 0.01, and events per primary
agree within 3 %.
"""
import numpy as np
import pytest

import nebula_b200 as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rough(tmp_path_factory):
    from nebula_b200.synth import geometry, materials, nmat
    d = tmp_path_factory.mktemp("rough")
    rows = geometry.rough_grating()
    t = nb.triangles_from_vertices(rows)
    g = nb.Geometry.from_triangles(t, max_depth=12, split_count=16)
    mats = []
    paths = []
    for sp in (materials.silicon(), materials.pmma()):
        p = str(d / (sp.name + ".nmat"))
        nmat.write(p, materials.build_raw_material(sp))
        paths.append(p)
        mats.append(nb.Material.load(p))
    return g, mats, paths


def _yield_and_sigma(rec, pri):
    key = pri["px"].astype(np.int64) * 100000 + pri["py"]
    uk, n_per = np.unique(key, return_counts=True)
    rk = rec["px"].astype(np.int64) * 100000 + rec["py"]
    pos = np.searchsorted(uk, rk)
    out = []
    for sel in (rec["E"] < 50, rec["E"] >= 50):
        c = np.bincount(pos[sel], minlength=len(uk)).astype(np.float64)
        y = c.sum() / len(pri)
        per = c / n_per
        out.append((y, per.std(ddof=1) / np.sqrt(len(uk))))
    return out


def test_rough_lines_yields_match_oracle(rough):
    from scipy.stats import ks_2samp
    from nebula_b200.synth import primaries
    g, mats, paths = rough
    inf = g.info()
    assert inf["n_octree"] > 10_000_000
    px = np.arange(240, 272)
    pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
    pri = primaries.raster_scan(512, 512, 200, 0.5, 300.0, 40.0, spot_sigma=1.0, seed=11, pixels=pixels)
    sim = nb.Simulation(g, mats, capacity=1 << 20, seed=4242, record_capacity=1 << 22)
    sim.push(pri)
    sim.run()
    rec = sim.flush_detected()
    c = sim.counters()
    assert c["walk_overflow"] == 0 and c["queue_overflow"] == 0 and c["nan_state"] == 0
    sim.close()

    od_, tr = g.export()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    oms = [O.Material(p) for p in paths]
    sub = pri.reshape(len(pixels), 200)[:, :100].reshape(-1)         # 100 primaries per pixel
    import os
    orec, _, oev = O.simulate(og, oms, sub, 77, threads=min(16, os.cpu_count() or 1))

    (ys, ss), (yb, sb) = _yield_and_sigma(rec, pri)
    (ors, oss), (orb, osb) = _yield_and_sigma(orec, sub)
    assert abs(ys - ors) < 3 * np.hypot(ss, oss), (ys, ors, ss, oss)
    assert abs(yb - orb) < 3 * np.hypot(sb, osb), (yb, orb, sb, osb)
    assert ks_2samp(rec["E"], orec["E"]).pvalue > 0.01
    d = rec["dir"].astype(np.float64)
    od = orec["dir"].astype(np.float64)
    assert ks_2samp(d[:, 2] / np.linalg.norm(d, axis=1), od[:, 2] / np.linalg.norm(od, axis=1)).pvalue > 0.01
    ev_gpu = c["flights"] / len(pri)
    ev_cpu = oev / len(sub)
    assert abs(ev_gpu - ev_cpu) / ev_cpu < 0.03, (ev_gpu, ev_cpu)
