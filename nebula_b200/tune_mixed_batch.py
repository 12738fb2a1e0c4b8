"""Run the batch autotuner on the mixed 64-job batch and store the choice.

    python -m nebula_b200.tune_mixed_batch [--scale 0.1]

Writes nebula_b200/tuned/mixed_batch.json (the chosen capacity, block size
and refill threshold, plus every timed point); bench.py reads it.
"""
import argparse
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "tuned", "mixed_batch.json")


def load_mixed_batch(workdir, scale=1.0):
    import nebula_b200 as nb
    from nebula_b200.synth import workloads, geometry, materials, nmat
    gt, specs, jobs, desc = workloads.batch(scale=scale)
    geoms = []
    for i, t in enumerate(gt):
        p = os.path.join(workdir, "g%d.tri" % i)
        geometry.write_tri(p, t)
        geoms.append(nb.Geometry.from_tri_file(p))
    mats = []
    for sp in specs:
        p = os.path.join(workdir, sp.name + ".nmat")
        nmat.write(p, materials.build_raw_material(sp))
        mats.append(nb.Material.load(p))
    return geoms, mats, jobs, desc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.1, help="fraction of each job's primaries timed")
    ap.add_argument("--passes", type=int, default=1)
    args = ap.parse_args()
    from nebula_b200 import autotune
    with tempfile.TemporaryDirectory() as d:
        geoms, mats, jobs, _ = load_mixed_batch(d)
        best, table = autotune.tune_batch(geoms, mats, jobs, sample_scale=args.scale, passes=args.passes,
                                          log=lambda r: print(r, flush=True))
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    autotune.save(OUT, best, table)
    print("best", best)


if __name__ == "__main__":
    sys.exit(main())
