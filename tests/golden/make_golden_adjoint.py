"""Reference-driver finite-difference gradients of the SE yield, from the
REFERENCE itself (its single-threaded CPU driver, oracle/_ref/libnbl_ref.so
ref_simulate), for checking the GPU adjoint.

Run here (where the reference sources are) after ``make -C oracle``:

    python tests/golden/make_golden_adjoint.py

Scan: the grating, 16 x 16 pixels (0.5 nm) x 4000 primaries at 500 eV.  For
each of the 6 parameters (inelastic and elastic inverse-mean-free-path scale,
work function; Si then PMMA) the material files are rewritten with the
parameter moved by +-delta (1 % of a scale: the imfp dataset times 1 +- 0.01;
0.05 eV of a work function: the barrier property +- 0.05), and the reference
driver runs the scan in 32 chunks, its mt19937 generator reseeded for every
primary (seed 5000 + primary index; ref_simulate_reseeded), the same in the
+ and - runs, so that the two runs share random numbers primary by primary
(common random numbers; one stream per chunk would let a perturbation shift
every later primary's numbers).  Saved: tests/golden/adjoint_ref_fd.npz with the per-pixel
SE counts of every run, the per-pixel primary counts and the deltas.
"""
from __future__ import annotations

import copy
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.dirname(os.path.abspath(__file__))

NX = 16
PER_PIXEL = 4000
CHUNKS = 32
DELTA_SCALE = 0.01
DELTA_W = 0.05
PARAMS = ["s_inel_si", "s_el_si", "W_si", "s_inel_pmma", "s_el_pmma", "W_pmma"]


def perturbed_raw(spec, k_local, sign):
    from nebula_b200.synth import materials
    raw = copy.deepcopy(materials.build_raw_material(spec))
    if k_local == 0:
        raw["datasets"]["/full_penn/imfp"]["data"] = raw["datasets"]["/full_penn/imfp"]["data"] * (1 + sign * DELTA_SCALE)
    elif k_local == 1:
        raw["datasets"]["/elastic/imfp"]["data"] = raw["datasets"]["/elastic/imfp"]["data"] * (1 + sign * DELTA_SCALE)
    else:
        b, u = raw["properties"]["barrier"]
        raw["properties"]["barrier"] = (b + sign * DELTA_W, u)
        w, u = raw["properties"]["work_function"]
        raw["properties"]["work_function"] = (w + sign * DELTA_W, u)
    return raw


def _work(args):
    work, k, sign, chunk = args
    from oracle import oracle as O
    from nebula_b200.synth import workloads
    rg = O.RefGeometry(os.path.join(work, "grating.tri"))
    names = []
    for m in range(2):
        tag = "%d_%d_%d" % (m, k, sign) if (k // 3) == m else "%d_base" % m
        names.append(os.path.join(work, "mat_%s.nmat" % tag))
    rms = [O.RefMaterial(p) for p in names]
    w = workloads.grating(nx=NX, ny=NX, per_pixel=PER_PIXEL)
    part = np.array_split(w.primaries, CHUNKS)[chunk]
    first = chunk * len(part)   # chunks are equal (the scan size is a multiple of CHUNKS)
    rec, tot = O.ref_simulate_reseeded(rg, rms, part, 5000 + first, max_records=8 * len(part) + 1024)
    se = rec["E"] < 50
    img = np.zeros((NX, NX), np.int64)
    np.add.at(img, (rec["py"][se], rec["px"][se]), 1)
    return k, sign, img


def main():
    from nebula_b200.synth import workloads, geometry, materials, nmat
    work = tempfile.mkdtemp(prefix="nbl_golden_adj_")
    geometry.write_tri(os.path.join(work, "grating.tri"), workloads.grating_geometry())
    specs = [materials.silicon(), materials.pmma()]
    for m, sp in enumerate(specs):
        nmat.write(os.path.join(work, "mat_%d_base.nmat" % m), materials.build_raw_material(sp))
        for kl in range(3):
            for sign in (-1, 1):
                nmat.write(os.path.join(work, "mat_%d_%d_%d.nmat" % (m, 3 * m + kl, sign)),
                           perturbed_raw(sp, kl, sign))
    w = workloads.grating(nx=NX, ny=NX, per_pixel=PER_PIXEL)
    per_pixel = np.zeros((NX, NX), np.int64)
    np.add.at(per_pixel, (w.primaries["py"], w.primaries["px"]), 1)
    tasks = [(work, k, sign, c) for k in range(6) for sign in (-1, 1) for c in range(CHUNKS)]
    counts = np.zeros((6, 2, NX, NX), np.int64)
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        for k, sign, img in pool.imap_unordered(_work, tasks):
            counts[k, (sign + 1) // 2] += img
    deltas = np.array([DELTA_SCALE, DELTA_SCALE, DELTA_W] * 2)
    np.savez_compressed(os.path.join(OUT, "adjoint_ref_fd.npz"), counts_se=counts, per_pixel=per_pixel,
                        deltas=deltas, params=np.array(PARAMS), nx=NX, per_pixel_n=PER_PIXEL)
    N = per_pixel.sum()
    for k in range(6):
        fd_pix = (counts[k, 1] - counts[k, 0]) / (2 * deltas[k])
        fd = fd_pix.sum() / N
        se = fd_pix.std(ddof=1) * np.sqrt(fd_pix.size) / N
        print("%-12s reference FD dY/dtheta = %+.5f +- %.5f" % (PARAMS[k], fd, se))


if __name__ == "__main__":
    main()
