"""Golden statistics for the non-default physics selections, from the
REFERENCE itself (its driver templates instantiated with each selection in
oracle/_ref/libnbl_ref.so, ref_simulate).

Run here (where the reference sources are) after ``make -C oracle``:

    python tests/golden/make_golden_physics.py

For each preset (the option dictionaries of tests/test_physics_options.py):
the 100 x 100 pixel subset (pixels 78..177) of the 256 x 256 grating scan,
100 primaries per pixel at 500 eV, split into chunks run in parallel with
seeds 1000 + chunk.  Saved as stats_physics_<preset>.npz with the same keys
as stats_grating.npz (yields, per-pixel sums of squared counts, a 20 000
record subsample for KS tests).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.dirname(os.path.abspath(__file__))

PRESETS = {
    "kieft": {"inelastic_model": 1},
    "classical_boundary": {"acoustic_phonon_loss": 0, "atomic_recoil_loss": 0, "quantum_transmission": 0,
                           "interface_refraction": 0, "interface_absorption": 1},
    "kieft_plain": {"inelastic_model": 1, "optical_phonon_loss": 0, "instantaneous_momentum": 0,
                    "momentum_conservation": 0},
}
PIXELS = np.stack(np.meshgrid(np.arange(78, 178), np.arange(78, 178), indexing="xy"), -1).reshape(-1, 2)
CHUNKS = 32


def _work(args):
    work, preset, chunk = args
    from oracle import oracle as O
    from nebula_b200.synth import workloads
    ph = PRESETS[preset]
    suffix = "_kieft.nmat" if ph.get("inelastic_model") == 1 else ".nmat"
    rg = O.RefGeometry(os.path.join(work, "grating.tri"))
    rms = [O.RefMaterial(os.path.join(work, "si" + suffix)), O.RefMaterial(os.path.join(work, "pmma" + suffix))]
    w = workloads.grating(pixels=PIXELS)
    part = np.array_split(w.primaries, CHUNKS)[chunk]
    rec, tot, ev = O.ref_simulate(rg, rms, part, 1000 + chunk, phys=O.physics_bits(ph),
                                  max_records=8 * len(part) + 1024)
    assert tot == len(rec)
    return rec, ev


def main():
    from make_golden import stats_from_records
    from nebula_b200.synth import workloads, geometry, materials, nmat
    work = tempfile.mkdtemp(prefix="nbl_golden_phys_")
    geometry.write_tri(os.path.join(work, "grating.tri"), workloads.grating_geometry())
    for sp, name in ((materials.silicon(), "si"), (materials.pmma(), "pmma")):
        nmat.write(os.path.join(work, name + ".nmat"), materials.build_raw_material(sp))
        nmat.write(os.path.join(work, name + "_kieft.nmat"), materials.build_raw_material(sp, inelastic="kieft"))
    w = workloads.grating(pixels=PIXELS)
    rng = np.random.default_rng(20261204)
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(CHUNKS, os.cpu_count() or 1)) as pool:
        for preset in sorted(PRESETS):
            parts = pool.map(_work, [(work, preset, c) for c in range(CHUNKS)])
            rec = np.concatenate([p[0] for p in parts])
            ev = sum(p[1] for p in parts)
            n = len(w.primaries)
            st = stats_from_records(rec, n, w.primaries["px"].astype(np.int64) * 100000 + w.primaries["py"], rng)
            st["pixels"] = PIXELS.astype(np.int32)
            st["events"] = np.int64(ev)
            np.savez_compressed(os.path.join(OUT, "stats_physics_%s.npz" % preset), **st)
            print(preset, "SE %.4f BSE %.4f events/primary %.1f" % (st["se"] / n, st["bse"] / n, ev / n))


if __name__ == "__main__":
    main()
