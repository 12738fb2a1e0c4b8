"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Run here (where the reference sources are) after ``make -C oracle``:

    python tests/golden/make_golden.py

Everything comes from the reference's own code built by oracle/Makefile:
``oracle/_ref/libnbl_ref.so`` (its octree walk, its table transforms, its
single-threaded CPU driver loop) and ``oracle/_ref/nebula_cpu_mt`` (its
unmodified multithreaded CPU driver).  Inputs are the deterministic synthetic
workloads of nebula_b200.synth; the sha256 of each input file is stored so
tests can detect a change of the generators.

Fixtures:
  rays_<geom>.npz       rays incl. axis-parallel, zero-length, ignore cases,
                        and the reference octree<false>::propagate results
  octree_<geom>.npz     the reference's linearised octree (node array, triangles)
  tables_si.npz / tables_pmma.npz   sha256, shape and axes of the reference's
                        transformed tables, and its material constants
  records_slab.npz      36-byte records of the single-threaded reference
                        driver, 400 primaries, seed 5489 (oracle pin)
  stats_slab.npz        reference nebula_cpu_mt, 10^6 primaries at 1 keV:
                        yields with the per-primary sum of squared counts
                        (variance), energy histogram,
                        a 20 000-record subsample for KS tests
  stats_grating.npz     same for a 100 x 100 pixel subset of the grating scan
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.dirname(os.path.abspath(__file__))

from oracle import oracle as O  # noqa: E402
from nebula_b200.synth import workloads, geometry, materials, nmat, primaries  # noqa: E402


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def make_rays(g, rng, n, zlo, zhi):
    """Random rays inside the domain plus edge cases."""
    c, h = g.center, g.halfsize
    pos = np.empty((n, 3), np.float32)
    pos[:, 0] = rng.uniform(c[0] - h[0] * 0.9, c[0] + h[0] * 0.9, n)
    pos[:, 1] = rng.uniform(c[1] - h[1] * 0.9, c[1] + h[1] * 0.9, n)
    pos[:, 2] = rng.uniform(zlo, zhi, n)
    d = rng.standard_normal((n, 3))
    # a quarter axis-parallel (zero components: infinite slab distances)
    k = n // 4
    axis = rng.integers(0, 3, k)
    d[:k] = 0.0
    d[np.arange(k), axis] = rng.choice([-1.0, 1.0], k)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    dirs = d.astype(np.float32)
    dist = rng.exponential(50.0, n).astype(np.float32)
    dist[rng.random(n) < 0.05] = 0.0
    dist[rng.random(n) < 0.1] = np.float32(g.max_extent)
    ignore_tri = np.where(rng.random(n) < 0.2, rng.integers(0, len(g.tri11), n), -1).astype(np.int32)
    ignore_mat = rng.choice(np.array([-123, 0, 1, -126], np.int32), n)
    return pos, dirs, dist, ignore_tri, ignore_mat


def rays_on_triangles(g, rng, n):
    """Rays that start on triangle surfaces (the case after a boundary event)."""
    t = g.tri11
    idx = rng.integers(0, len(t), n)
    u = rng.random(n)
    v = rng.random(n) * (1 - u)
    r0, e1, e2 = t[idx, 2:5], t[idx, 5:8], t[idx, 8:11]
    pos = (r0 + u[:, None] * e1 + v[:, None] * e2).astype(np.float32)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    dist = rng.exponential(30.0, n).astype(np.float32)
    ign_mat = rng.choice(np.array([-123, 0, 1], np.int32), n)
    return pos, d.astype(np.float32), dist, idx.astype(np.int32), ign_mat


def stats_from_records(rec, n_pri, pixel_of_primary, rng, sub=20000):
    E = rec["E"]
    se = E < 50
    # per-primary (or per-pixel) counts for the variance of the yields
    key = rec["px"].astype(np.int64) * 100000 + rec["py"]
    uk = np.unique(pixel_of_primary)
    n_groups = len(uk)
    cnt_se = np.zeros(n_groups)
    cnt_bse = np.zeros(n_groups)
    pos_of = {int(k): i for i, k in enumerate(uk)}
    for k, s in zip(key, se):
        if s:
            cnt_se[pos_of[int(k)]] += 1
        else:
            cnt_bse[pos_of[int(k)]] += 1
    pick = rng.choice(len(rec), size=min(sub, len(rec)), replace=False)
    d = rec["dir"][pick].astype(np.float64)
    cos_t = d[:, 2] / np.linalg.norm(d, axis=1)
    hist, _ = np.histogram(E, bins=200, range=(0, 1000))
    return dict(n_primaries=n_pri, n_groups=n_groups, se=int(se.sum()), bse=int((~se).sum()),
                se_group_sumsq=float((cnt_se ** 2).sum()), bse_group_sumsq=float((cnt_bse ** 2).sum()),
                hist=hist.astype(np.int64), sub_E=E[pick].astype(np.float32), sub_cos=cos_t.astype(np.float32),
                sub_x=rec["pos"][pick, 0].astype(np.float32), sub_y=rec["pos"][pick, 1].astype(np.float32))


def run_cpu_mt(tri, pri, mats, workdir, seed=0x78C7E39B):
    outp = os.path.join(workdir, "out.bin")
    with open(outp, "wb") as fo:
        r = subprocess.run([O.REF_CPU_MT, "--seed=%d" % seed, tri, pri] + mats, stdout=fo,
                           stderr=subprocess.PIPE, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return np.fromfile(outp, dtype=O.PRI_DTYPE), r.stderr


def main():
    rng = np.random.default_rng(20261203)
    work = tempfile.mkdtemp(prefix="nbl_golden_")
    files = {}
    slab = workloads.slab()
    geometry.write_tri(os.path.join(work, "slab.tri"), slab.triangles)
    geometry.write_tri(os.path.join(work, "grating.tri"), workloads.grating_geometry())
    nmat.write(os.path.join(work, "si.nmat"), materials.build_raw_material(materials.silicon()))
    nmat.write(os.path.join(work, "pmma.nmat"), materials.build_raw_material(materials.pmma()))
    for k in ("slab.tri", "grating.tri", "si.nmat", "pmma.nmat"):
        files[k] = os.path.join(work, k)
    hashes = {k: sha(v) for k, v in files.items()}
    np.savez_compressed(os.path.join(OUT, "inputs_sha256.npz"), **{k.replace(".", "_"): np.array(v) for k, v in hashes.items()})

    # materials
    rms = {}
    for name in ("si", "pmma"):
        rm = O.RefMaterial(files[name + ".nmat"])
        rms[name] = rm
        d = {}
        for t in O.TABLE_NAMES:
            data, scale = rm.table(t)
            d[t + "_sha256"] = np.array(hashlib.sha256(np.ascontiguousarray(data, np.float32).tobytes()).hexdigest())
            d[t + "_shape"] = np.array(data.shape, np.int32)
            d[t + "_scale"] = scale
        d["constants"] = rm.constants()
        np.savez_compressed(os.path.join(OUT, "tables_%s.npz" % name), **d)

    # geometry: octree + rays
    for gname, zlo, zhi in (("slab", -1000.0, 10.0), ("grating", -60.0, 49.0)):
        rg = O.RefGeometry(files[gname + ".tri"])
        np.savez_compressed(os.path.join(OUT, "octree_%s.npz" % gname), octree_data=rg.octree_data, tri11=rg.tri11,
                            center=rg.center, halfsize=rg.halfsize, max_extent=np.float32(rg.max_extent))
        p1, d1, s1, it1, im1 = make_rays(rg, rng, 3000, zlo, zhi)
        p2, d2, s2, it2, im2 = rays_on_triangles(rg, rng, 1000)
        pos = np.concatenate([p1, p2]); dirs = np.concatenate([d1, d2]); dist = np.concatenate([s1, s2])
        it = np.concatenate([it1, it2]); im = np.concatenate([im1, im2])
        od, ot = rg.propagate(pos, dirs, dist, it, im)
        np.savez_compressed(os.path.join(OUT, "rays_%s.npz" % gname), pos=pos, dir=dirs, dist=dist, ignore_tri=it,
                            ignore_mat=im, out_dist=od, out_tri=ot)
        print(gname, "rays", len(pos), "hits", int((ot >= 0).sum()))

    # single-threaded reference driver records (pins the oracle bit for bit)
    rg = O.RefGeometry(files["slab.tri"])
    pri = primaries.point_beam(400)
    rec, tot, ev = O.ref_simulate(rg, [rms["si"]], pri, 5489)
    np.savez_compressed(os.path.join(OUT, "records_slab.npz"), records=rec.view(np.uint8).reshape(-1, 36),
                        n_total=tot, n_events=ev, n_primaries=len(pri), seed=5489)
    print("records_slab", len(rec), ev)

    # reference nebula_cpu_mt statistics: slab, 10^6 primaries, unique pixel per primary
    n = 1_000_000
    pri = primaries.point_beam(n)
    idx = np.arange(n)
    pri["px"] = idx % 1000
    pri["py"] = idx // 1000
    primaries.write_pri(os.path.join(work, "slab.pri"), pri)
    rec, log = run_cpu_mt(files["slab.tri"], os.path.join(work, "slab.pri"), [files["si.nmat"]], work)
    st = stats_from_records(rec, n, pri["px"].astype(np.int64) * 100000 + pri["py"], rng)
    np.savez_compressed(os.path.join(OUT, "stats_slab.npz"), **st)
    print("stats_slab SE %.4f BSE %.4f" % (st["se"] / n, st["bse"] / n))

    # grating: 100 x 100 pixel subset of the 256 x 256 scan, 100 primaries each
    px = np.arange(78, 178)
    pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
    w = workloads.grating(pixels=pixels)
    primaries.write_pri(os.path.join(work, "grating.pri"), w.primaries)
    rec, log = run_cpu_mt(files["grating.tri"], os.path.join(work, "grating.pri"),
                          [files["si.nmat"], files["pmma.nmat"]], work)
    st = stats_from_records(rec, len(w.primaries), w.primaries["px"].astype(np.int64) * 100000 + w.primaries["py"], rng)
    st["pixels"] = pixels.astype(np.int32)
    np.savez_compressed(os.path.join(OUT, "stats_grating.npz"), **st)
    print("stats_grating SE %.4f BSE %.4f" % (st["se"] / len(w.primaries), st["bse"] / len(w.primaries)))


if __name__ == "__main__":
    main()
