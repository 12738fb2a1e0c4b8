"""Energy deposits on the GPU (the reference's energy-deposit driver,
drivers/cpu/energydeposit_cpu_driver.h:44-93, record cpu_energydep.cpp:197-204)
through the C ABI, against the oracle's deposit loop (pinned bit for bit to
the reference in tests/test_oracle_pin.py):

* deposit events and deposited energy per primary within 3 sigma;
* depth, lateral position, loss and energy distributions (one deposit per
  primary, so the samples are independent): two-sample KS at p > 0.01;
* the device voxel grid equals the records binned on the host (FP64 sums,
  relative 1e-9);
* records independent of capacity (counter-based random numbers).
"""
import os

import numpy as np
import pytest

import nebula_b200 as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _slab(inputs, n):
    from nebula_b200.synth import primaries
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    pri = primaries.point_beam(n)
    idx = np.arange(n)
    pri["px"] = idx % 1000
    pri["py"] = idx // 1000
    return g, m, pri


def _per_group(dep, n_groups):
    key = dep["py"].astype(np.int64) * 1000 + dep["px"]
    cnt = np.bincount(key, minlength=n_groups).astype(np.float64)
    e = np.bincount(key, weights=dep["loss"].astype(np.float64), minlength=n_groups)
    return cnt, e


def _one_per_primary(dep, seed):
    key = dep["py"].astype(np.int64) * 1000 + dep["px"]
    order = np.argsort(key, kind="stable")
    k = key[order]
    starts = np.flatnonzero(np.r_[True, k[1:] != k[:-1]])
    ends = np.r_[starts[1:], len(k)]
    rng = np.random.default_rng(seed)
    pick = starts + (rng.random(len(starts)) * (ends - starts)).astype(np.int64)
    return dep[order[pick]]


def _z(a, b):
    return abs(a.mean() - b.mean()) / np.hypot(a.std(ddof=1) / np.sqrt(len(a)), b.std(ddof=1) / np.sqrt(len(b)))


def test_deposits_match_oracle(inputs):
    from scipy.stats import ks_2samp
    n = 50000
    g, m, pri = _slab(inputs, n)
    sim = nb.Simulation(g, [m], capacity=1 << 16, seed=8, deposit_capacity=1 << 24)
    sim.push(pri)
    sim.run()
    dep = sim.drain_deposits()
    c = sim.counters()
    sim.close()
    assert c["deposits"] == len(dep) and c["deposit_overflow"] == 0
    assert np.all(dep["loss"] != 0) and np.all(dep["E"] > 0)

    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    odep, _ = O.simulate_deposits(og, [O.Material(inputs["si.nmat"])], pri, 19,
                                  threads=min(16, os.cpu_count() or 1))
    ng = (n + 999) // 1000 * 1000
    gc, ge = _per_group(dep, ng)
    oc, oe = _per_group(odep, ng)
    assert _z(gc, oc) < 3, (gc.mean(), oc.mean())
    assert _z(ge, oe) < 3, (ge.mean(), oe.mean())
    # one deposit per primary (deposits of one track are correlated; the KS
    # test needs independent samples)
    a = _one_per_primary(dep, 1)
    b = _one_per_primary(odep, 2)
    for name, x, y in (("z", a["pos"][:, 2], b["pos"][:, 2]), ("x", a["pos"][:, 0], b["pos"][:, 0]),
                       ("loss", a["loss"], b["loss"]), ("E", a["E"], b["E"])):
        p = ks_2samp(x, y).pvalue
        assert p > 0.01, (name, p)


def test_deposit_grid_equals_binned_records(inputs):
    n = 5000
    g, m, pri = _slab(inputs, n)
    origin, voxel, dims = (-50.0, -50.0, -100.0), (2.0, 2.5, 1.0), (50, 40, 100)
    sim = nb.Simulation(g, [m], capacity=1 << 14, seed=3, deposit_capacity=1 << 21,
                        deposit_grid=(origin, voxel, dims))
    sim.push(pri)
    sim.run()
    dep = sim.drain_deposits()
    grid = sim.deposit_grid()
    sim.close()
    # bin on the host exactly as the device does: floor((x - origin) * (1/voxel)) in float32
    pos = dep["pos"]
    idx = []
    for k in range(3):
        inv = np.float32(1.0) / np.float32(voxel[k])
        idx.append(np.floor((pos[:, k] - np.float32(origin[k])) * inv).astype(np.int64))
    inside = np.ones(len(dep), bool)
    for k in range(3):
        inside &= (idx[k] >= 0) & (idx[k] < dims[k])
    ref = np.zeros(dims[::-1], np.float64)
    np.add.at(ref, (idx[2][inside], idx[1][inside], idx[0][inside]), dep["loss"][inside].astype(np.float64))
    assert inside.sum() > 0.5 * len(dep)
    assert np.allclose(grid, ref, rtol=1e-9, atol=1e-9)


def test_deposits_independent_of_capacity(inputs):
    g, m, pri = _slab(inputs, 3000)
    out = []
    for cap in (1 << 10, 1 << 16):
        sim = nb.Simulation(g, [m], capacity=cap, seed=5, deposit_capacity=1 << 20)
        sim.push(pri)
        sim.run()
        d = sim.drain_deposits()
        sim.close()
        out.append(np.sort(d.view(np.dtype((np.void, 28))).ravel()))
    assert len(out[0]) > 0 and np.array_equal(out[0], out[1])
