"""Per-pixel SE / BSE images with a detector acceptance cone.

1. Against the oracle (the CPU restatement pinned bit for bit to the
   reference CPU driver): the device images of a 64 x 64-pixel block of the
   grating scan, with and without the cone, against the oracle's detected
   records for the same primaries binned into the same pixels with the same
   cut.  Different random numbers, so the comparison is statistical: over
   16 x 16-pixel blocks, z = (GPU - oracle) / sigma, with sigma from
   independent groups of each pixel's primaries (each pixel's primaries are
   tallied into 4 sub-grids, so the spatial structure of the yield does not
   enter the error); chi^2 over the blocks must give p > 0.01 and no block
   may be beyond 3.5 sigma (16 blocks: a 1 % family-wise chance).
2. Internal consistency: the device images equal the same run's detected
   records binned on the host (up to records within 1e-5 of the cut, where
   the device's fast division may round the other way), and the records do
   not depend on the image filter.
"""
import os

import numpy as np
import pytest
from scipy import stats

import nebula_b200 as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

K = 4           # sub-grids per pixel (independent primary groups)
NX = 64         # block of the 256 x 256 raster: pixels 96..159 in x and y
BLOCK = 16


def _bin(rec, sel, nx, ny):
    img = np.zeros((ny, nx), np.int64)
    np.add.at(img, (rec["py"][sel], rec["px"][sel]), 1)
    return img


def _cos_z(rec):
    d = rec["dir"].astype(np.float32)
    return d[:, 2] / np.sqrt((d * d).sum(1, dtype=np.float32))


def _grating(inputs, per_pixel):
    from nebula_b200.synth import workloads
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    px = np.arange(96, 96 + NX)
    pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
    w = workloads.grating(pixels=pixels, per_pixel=per_pixel)
    return g, ms, w.primaries


def _subgrid(pri):
    """Tally pixel of each primary: (px - 96, py - 96 + 64 k), k = index
    within its pixel mod K (the beam positions are unchanged)."""
    p = pri.copy()
    k = np.arange(len(p)) % K
    p["px"] = p["px"] - 96
    p["py"] = p["py"] - 96 + NX * k
    return p


def _blocks(img):
    """(NX * K, NX) sub-grid image -> block totals and their variances from
    the spread over the K groups of each pixel."""
    sub = img.reshape(K, NX, NX).astype(np.float64)             # [k, y, x]
    pix_var = K * sub.var(axis=0, ddof=1)                       # variance of each pixel's total
    tot = sub.sum(0)
    nb_ = NX // BLOCK
    t = tot.reshape(nb_, BLOCK, nb_, BLOCK).sum((1, 3))
    v = pix_var.reshape(nb_, BLOCK, nb_, BLOCK).sum((1, 3))
    return t.ravel(), v.ravel()


def test_images_match_oracle(inputs):
    g, ms, pri0 = _grating(inputs, per_pixel=200)
    pri = _subgrid(pri0)
    cone = (0.8, 1.0)
    imgs = {}
    for name, c in (("all", None), ("cone", cone)):
        sim = nb.Simulation(g, ms, capacity=1 << 20, seed=31, tally=(NX, NX * K), image_cos_range=c,
                            record_capacity=1 << 22)
        sim.push(pri)
        sim.run()
        se, bse, _ = sim.tallies()
        imgs[name] = (se, bse)
        sim.close()
    od, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    orec, _, _ = O.simulate(og, [O.Material(inputs["si.nmat"]), O.Material(inputs["pmma.nmat"])], pri, 8,
                            threads=os.cpu_count() or 1)
    c = _cos_z(orec)
    se_o = orec["E"] < 50.0
    for name in ("all", "cone"):
        keep = np.ones(len(orec), bool) if name == "all" else (c >= cone[0]) & (c <= cone[1])
        for kind, sel in (("SE", se_o), ("BSE", ~se_o)):
            gpu = imgs[name][0 if kind == "SE" else 1].astype(np.int64)
            ora = _bin(orec, sel & keep, NX, NX * K)
            tg, vg = _blocks(gpu)
            to, vo = _blocks(ora)
            z = (tg - to) / np.sqrt(vg + vo)
            chi2 = float((z * z).sum())
            p = stats.chi2.sf(chi2, z.size)
            assert p > 0.01 and np.abs(z).max() < 3.5, (name, kind, chi2, p, np.round(z, 2))
            assert tg.sum() > 1000
        if name == "cone":
            assert imgs["cone"][0].sum() < imgs["all"][0].sum()


def test_image_filter_matches_records(inputs):
    g, ms, pri = _grating(inputs, per_pixel=50)
    imgs = {}
    recs = {}
    for name, cone in (("all", None), ("cone", (0.8, 1.0))):
        sim = nb.Simulation(g, ms, capacity=1 << 18, seed=12, tally=(256, 256), image_cos_range=cone)
        sim.push(pri)
        sim.run()
        recs[name] = sim.flush_detected()
        imgs[name] = sim.tallies()
        sim.close()
    rec = recs["all"]
    # the filter applies to the images only: the records are the same
    key = lambda a: np.sort(a.view(np.dtype((np.void, 36))).ravel()).tobytes()
    assert key(rec) == key(recs["cone"])
    c = _cos_z(rec)
    se = rec["E"] < 50
    for k, sel in ((0, se), (1, ~se)):
        assert np.array_equal(imgs["all"][k], _bin(rec, sel, 256, 256))
        inside = sel & (c >= 0.8) & (c <= 1.0)
        near = sel & (np.abs(c - 0.8) < 1e-5)
        diff = np.abs(imgs["cone"][k].astype(np.int64) - _bin(rec, inside, 256, 256)).sum()
        assert diff <= near.sum()
        assert imgs["cone"][k].sum() < imgs["all"][k].sum()
