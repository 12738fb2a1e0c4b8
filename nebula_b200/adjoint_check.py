"""Adjoint gradients against common-random-number finite differences over
several independent seeds (a check with more statistics than one scan).

    python -m nebula_b200.adjoint_check --seeds 10 --params 0,4

For each seed, the grating scan of 64 x 64 pixels x 10^4 primaries at 500 eV
(4.1 x 10^7 primaries) is run forward, replayed for the adjoint (per-pixel
gradients of the SE yield), and differenced centrally for each chosen
parameter with the same seed (steps: 1 % and 5 % of a mean-free-path scale,
0.05 eV of a work function).  Prints one JSON line per seed and a summary:
means over seeds with their standard errors, and adjoint - difference.
Parameters: 0 s_inel Si, 1 s_el Si, 2 W Si, 3 s_inel PMMA, 4 s_el PMMA,
5 W PMMA.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile

import numpy as np

NAMES = ["s_inel_si", "s_el_si", "W_si", "s_inel_pmma", "s_el_pmma", "W_pmma"]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=10)
    ap.add_argument("--params", default="0,4", help="comma-separated parameter indices")
    ap.add_argument("--pixels", type=int, default=64)
    ap.add_argument("--per-pixel", type=int, default=10_000)
    ap.add_argument("--first-seed", type=int, default=1000)
    args = ap.parse_args(argv)
    import nebula_b200 as nb
    from nebula_b200.synth import workloads, geometry, materials, nmat
    from nebula_b200.torch_adjoint import ScanProblem

    params = [int(x) for x in args.params.split(",") if x.strip()]
    rows = []
    with tempfile.TemporaryDirectory() as d:
        w = workloads.grating(nx=args.pixels, ny=args.pixels, per_pixel=args.per_pixel)
        tri = os.path.join(d, "grating.tri")
        geometry.write_tri(tri, w.triangles)
        ms = []
        for sp in w.material_specs:
            p = os.path.join(d, sp.name + ".nmat")
            nmat.write(p, materials.build_raw_material(sp))
            ms.append(nb.Material.load(p))
        g = nb.Geometry.from_tri_file(tri)
        for rep in range(args.seeds):
            prob = ScanProblem(g, ms, w.primaries, (args.pixels, args.pixels), seed=args.first_seed + rep,
                               capacity=1 << 22)
            th0 = prob.theta0().numpy()
            prob.forward(th0)
            J = prob.jacobian(th0)
            W = prob.per_pixel
            N = W.sum()
            row = {}
            for k in params:
                row["adjoint_" + NAMES[k]] = float((J[..., k] * W).sum() / N)
                steps = (("0.05eV", 0.05),) if k % 3 == 2 else (("1%", 0.01 * float(th0[k])),
                                                                  ("5%", 0.05 * float(th0[k])))
                for label, dl in steps:
                    tp, tm = th0.copy(), th0.copy()
                    tp[k] += dl
                    tm[k] -= dl
                    row["fd%s_%s" % (label, NAMES[k])] = float(((prob.forward(tp) - prob.forward(tm)) * W).sum()
                                                             / N / (2 * dl))
            prob.close()
            rows.append(row)
            print(json.dumps({"seed": args.first_seed + rep, **row}), flush=True)
    summary = {}
    for key in rows[0]:
        v = np.array([r[key] for r in rows])
        summary[key] = [float(v.mean()), float(v.std(ddof=1) / np.sqrt(len(v))) if len(v) > 1 else None]
    for k in params:
        for key in rows[0]:
            if key.startswith("fd") and key.endswith(NAMES[k]):
                dv = np.array([r["adjoint_" + NAMES[k]] - r[key] for r in rows])
                summary["adjoint-" + key] = [float(dv.mean()),
                                             float(dv.std(ddof=1) / np.sqrt(len(dv))) if len(dv) > 1 else None]
    print(json.dumps({"summary": summary, "seeds": args.seeds,
                      "primaries_per_seed": int(args.pixels * args.pixels * args.per_pixel)}))


if __name__ == "__main__":
    main()
