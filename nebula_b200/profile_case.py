"""A bounded transport run for profilers and timing sweeps.

``python -m nebula_b200.profile_case --pixels 64 --per-pixel 100`` runs the
line-space grating scan (the 4 144-triangle, 8-line PMMA-on-Si grating) on a
``pixels x pixels`` block of the 256 x 256 raster at 500 eV, ``--repeat``
times after one warm-up run, and prints one JSON line with the transport
kernel time, primaries/s and events per primary.  ``--workload rough`` runs
the 16 rough lines (1.2 M triangles, octree depth <= 12) on a ``pixels x
pixels`` block at the centre of their 512 x 512 raster (300 eV unless
``--energy`` is given); ``--workload slab`` the 1 um Si slab; ``--workload
batch`` the 64-job mixed batch, every job's primaries scaled by ``--scale``,
in the batched persistent kernel (one launch per run; ``--block`` and
``--capacity`` set its launch shape and pool).  It is small enough for a full
ncu capture of a few launches (``-k regex:k_step -s <n> -c <m>``) and keeps
its whole state on one GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--pixels", type=int, default=64)
    ap.add_argument("--per-pixel", type=int, default=100)
    ap.add_argument("--energy", type=float, default=500.0)
    ap.add_argument("--capacity", type=int, default=1 << 18)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--workload", default="grating", choices=["grating", "slab", "rough", "batch"])
    ap.add_argument("--scale", type=float, default=0.02, help="batch: fraction of every job's primaries")
    ap.add_argument("--block", type=int, default=0, help="threads per block of the step kernel (0: default)")
    args = ap.parse_args(argv)

    import numpy as np
    import nebula_b200 as nb
    from nebula_b200.synth import workloads, geometry, materials, nmat

    if args.workload == "batch":
        return run_batch(args)
    with tempfile.TemporaryDirectory() as d:
        if args.workload == "grating":
            px = np.arange(128 - args.pixels // 2, 128 - args.pixels // 2 + args.pixels)
            pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
            w = workloads.grating(pixels=pixels, per_pixel=args.per_pixel, energy=args.energy)
        elif args.workload == "rough":
            px = np.arange(256 - args.pixels // 2, 256 - args.pixels // 2 + args.pixels)
            pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
            args.energy = args.energy if args.energy != ap.get_default("energy") else 300.0
            w = workloads.rough(pixels=pixels, per_pixel=args.per_pixel, energy=args.energy, pixel_streams=False)
        else:
            w = workloads.slab(n_primaries=args.pixels * args.pixels * args.per_pixel, energy=args.energy)
        ms = []
        for sp in w.material_specs:
            p = os.path.join(d, sp.name + ".nmat")
            nmat.write(p, materials.build_raw_material(sp))
            ms.append(nb.Material.load(p))
        if args.workload == "rough":
            g = nb.Geometry.from_triangles(nb.triangles_from_vertices(w.triangles), max_depth=12, split_count=16)
        else:
            tri = os.path.join(d, "g.tri")
            geometry.write_tri(tri, w.triangles)
            g = nb.Geometry.from_tri_file(tri)
        sim = nb.Simulation(g, ms, capacity=args.capacity, seed=args.seed, record_capacity=1 << 22,
                            block_size=args.block)
        runs = []
        for r in range(args.repeat + 1):
            sim.reset()
            sim.push(w.primaries)
            t0 = time.perf_counter()
            sim.run()
            wall = time.perf_counter() - t0
            c = sim.counters()
            sim.flush_detected()
            if r > 0:
                runs.append((sim.kernel_ms(), wall, c["flights"], c["iterations"]))
        sim.close()
    n = len(w.primaries)
    kms = float(np.mean([r[0] for r in runs]))
    print(json.dumps({"workload": "%s %dx%dx%d at %g eV" % (args.workload, args.pixels, args.pixels, args.per_pixel,
                                                            args.energy),
                      "primaries": n, "kernel_ms": kms, "primaries_per_s": n / (kms / 1e3),
                      "events_per_primary": runs[-1][2] / n, "iterations": runs[-1][3],
                      "wall_s": float(np.mean([r[1] for r in runs]))}))


def run_batch(args):
    import numpy as np
    import nebula_b200 as nb
    from nebula_b200.tune_mixed_batch import load_mixed_batch

    with tempfile.TemporaryDirectory() as d:
        geoms, mats, jobs, _ = load_mixed_batch(d, scale=args.scale)
        b = nb.Batch(geoms, mats, capacity=args.capacity, block_size=args.block or 512, refill_threshold=0.5)
        b.set_jobs(jobs)
        runs = []
        for r in range(args.repeat + 1):
            b.run()
            if r > 0:
                runs.append(b.kernel_ms())
        c = b.counters()
        b.close()
    n = sum(len(p) for _, _, p in jobs)
    kms = float(np.mean(runs))
    print(json.dumps({"workload": "mixed batch x %g (%d jobs)" % (args.scale, len(jobs)), "primaries": n,
                      "kernel_ms": kms, "primaries_per_s": n / (kms / 1e3),
                      "events_per_primary": c["flights"] / n, "iterations": c["iterations"]}))


if __name__ == "__main__":
    main()
