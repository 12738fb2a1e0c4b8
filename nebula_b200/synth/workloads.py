"""The five workloads the path is measured and checked on.

* ``slab``: Si-like 1 um cube, top at z=0, detector plane at z=+10 nm,
  10^4 primaries at (0, 0, +5 nm), normal incidence, 1 keV.
* ``grating``: 8 trapezoidal PMMA-like lines (pitch 32 nm, top CD 16 nm,
  86 deg sidewalls, 30 nm high, ~4.1 k triangles) on the slab substrate;
  256 x 256 pixels at 0.5 nm, 100 primaries per pixel, 500 eV, Gaussian spot
  sigma 1 nm; detector plane at z = 50 nm.
* ``rough``: 16 lines with line-edge roughness (sigma 1.5 nm, exponential
  correlation length 20 nm, 0.25 nm vertex spacing; ~1.2 M triangles);
  512 x 512 pixels x 200 primaries at 300 eV.
* ``batch``: 64 jobs drawn from a seed (slab, or grating with pitch 20-64 nm;
  energy log-uniform 200 eV-20 keV; primaries log-uniform 10^3-10^6).
* ``adjoint``: the grating at 64 x 64 pixels x 10^4 primaries at 500 eV.

Material 0 is always the Si-like substrate, material 1 the PMMA-like lines.
"""
from __future__ import annotations

import dataclasses
import numpy as np

from . import geometry, materials, primaries


@dataclasses.dataclass
class Workload:
    name: str
    triangles: np.ndarray            # (N, 11) float64
    material_specs: list
    primaries: np.ndarray            # PRI_DTYPE records
    detector_z: float
    n_pixels: tuple = (1, 1)
    extra: dict = dataclasses.field(default_factory=dict)


def slab(n_primaries=10_000, energy=1000.0, e_max=10e3):
    return Workload("slab", geometry.slab(), [materials.silicon(e_max)],
                    primaries.point_beam(n_primaries, energy=energy), detector_z=10.0)


GRATING_Z0 = 40.0   # primaries start between the line tops (30 nm) and the detector (50 nm)


def grating_geometry(pitch=32.0):
    # the top CD scales with the pitch (half pitch), as in a 1:1 line-space
    return geometry.grating(pitch=pitch, top_cd=pitch / 2)


def grating(nx=256, ny=256, per_pixel=100, energy=500.0, pixels=None, seed=7, e_max=10e3):
    pri = primaries.raster_scan(nx, ny, per_pixel, 0.5, energy, GRATING_Z0, spot_sigma=1.0,
                                seed=seed, pixels=pixels)
    return Workload("grating", grating_geometry(), [materials.silicon(e_max), materials.pmma(e_max)],
                    pri, detector_z=50.0, n_pixels=(nx, ny))


def rough(nx=512, ny=512, per_pixel=200, energy=300.0, pixels=None, seed=11, pixel_streams=True):
    tris = geometry.rough_grating()
    pri = primaries.raster_scan(nx, ny, per_pixel, 0.5, energy, GRATING_Z0, spot_sigma=1.0,
                                seed=seed, pixels=pixels, pixel_streams=pixel_streams)
    return Workload("rough", tris, [materials.silicon(), materials.pmma()], pri,
                    detector_z=50.0, n_pixels=(nx, ny))


def batch_jobs(n_jobs=64, seed=2024, e_lo=200.0, e_hi=20e3, n_lo=1e3, n_hi=1e6):
    """Job descriptions for the mixed batch: list of dicts with geometry kind,
    pitch, energy and primary count, all drawn from ``seed``."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        kind = "slab" if rng.random() < 0.5 else "grating"
        pitch = float(rng.uniform(20.0, 64.0))
        energy = float(np.exp(rng.uniform(np.log(e_lo), np.log(e_hi))))
        count = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        jobs.append(dict(job=j, kind=kind, pitch=pitch if kind == "grating" else None,
                         energy=energy, n_primaries=count, seed=int(rng.integers(1, 2**31))))
    return jobs


def adjoint(nx=64, ny=64, per_pixel=10_000, energy=500.0):
    return grating(nx=nx, ny=ny, per_pixel=per_pixel, energy=energy)


def batch(seed=2024, n_jobs=64, scale=1.0, e_max=30e3):
    """The mixed batch: geometries (slab first, then one grating per distinct
    pitch), material specs covering the energy range, and jobs as
    (geometry index, seed, primaries).  ``scale`` multiplies every job's
    primary count (a bounded sample of the batch keeps its energy and
    geometry mix).  Slab jobs: a point beam at (0, 0, +5 nm); grating jobs:
    primaries spread uniformly over a 64 x 64 nm field centred on the lines,
    starting at z = 40 nm; all at normal incidence."""
    desc = batch_jobs(n_jobs=n_jobs, seed=seed)
    geoms = [geometry.slab()]
    pitch_index = {}
    jobs = []
    for d in desc:
        n = max(1, int(round(d["n_primaries"] * scale)))
        rng = np.random.default_rng([seed, d["job"]])
        if d["kind"] == "slab":
            gi = 0
            pri = primaries.point_beam(n, energy=d["energy"], pixel=(d["job"], 0))
        else:
            key = round(d["pitch"], 6)
            if key not in pitch_index:
                pitch_index[key] = len(geoms)
                geoms.append(grating_geometry(pitch=d["pitch"]))
            gi = pitch_index[key]
            pri = np.zeros(n, dtype=primaries.PRI_DTYPE)
            pri["pos"][:, 0] = rng.uniform(-32.0, 32.0, n)
            pri["pos"][:, 1] = rng.uniform(-32.0, 32.0, n)
            pri["pos"][:, 2] = GRATING_Z0
            pri["dir"] = (0.0, 0.0, -1.0)
            pri["E"] = d["energy"]
            pri["px"] = d["job"]
        jobs.append((gi, d["seed"], pri))
    return geoms, [materials.silicon(e_max), materials.pmma(e_max)], jobs, desc
