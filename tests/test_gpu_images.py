"""Per-pixel SE / BSE images with a detector acceptance cone: the device
images equal the detected records binned on the host with the same cut
(up to records within 1e-5 of the cut, where the device's fast division may
round the other way), and the unfiltered images equal all records."""
import numpy as np
import pytest

import nebula_b200 as nb

pytestmark = pytest.mark.gpu


def _bin(rec, sel, nx, ny):
    img = np.zeros((ny, nx), np.int64)
    np.add.at(img, (rec["py"][sel], rec["px"][sel]), 1)
    return img


def test_image_filter_matches_records(inputs):
    from nebula_b200.synth import workloads
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    px = np.arange(96, 160)
    pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
    w = workloads.grating(pixels=pixels, per_pixel=50)
    imgs = {}
    recs = {}
    for name, cone in (("all", None), ("cone", (0.8, 1.0))):
        sim = nb.Simulation(g, ms, capacity=1 << 18, seed=12, tally=(256, 256), image_cos_range=cone)
        sim.push(w.primaries)
        sim.run()
        recs[name] = sim.flush_detected()
        imgs[name] = sim.tallies()
        sim.close()
    rec = recs["all"]
    assert rec.tobytes() == recs["cone"].tobytes() or len(rec) == len(recs["cone"])
    d = rec["dir"].astype(np.float32)
    c = d[:, 2] / np.sqrt((d * d).sum(1, dtype=np.float32))
    se = rec["E"] < 50
    for k, sel in ((0, se), (1, ~se)):
        assert np.array_equal(imgs["all"][k], _bin(rec, sel, 256, 256))
        inside = sel & (c >= 0.8) & (c <= 1.0)
        near = sel & (np.abs(c - 0.8) < 1e-5)
        diff = np.abs(imgs["cone"][k].astype(np.int64) - _bin(rec, inside, 256, 256)).sum()
        assert diff <= near.sum()
        assert imgs["cone"][k].sum() < imgs["all"][k].sum()
