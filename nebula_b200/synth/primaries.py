"""Primary electrons in Nebula's ``.pri`` layout.

One record is 36 bytes, little-endian: ``float pos[3], dir[3], E; int px, py``
(``io/load_pri_file.cpp:112-121``).  The detected-electron output uses the
same record layout (``gpu_main.cu:216-223``).
"""
from __future__ import annotations

import numpy as np

PRI_DTYPE = np.dtype([("pos", "<f4", 3), ("dir", "<f4", 3), ("E", "<f4"),
                      ("px", "<i4"), ("py", "<i4")])
assert PRI_DTYPE.itemsize == 36


def point_beam(n, pos=(0.0, 0.0, 5.0), direction=(0.0, 0.0, -1.0), energy=1000.0,
               pixel=(0, 0)):
    """``n`` identical primaries (a point beam at normal incidence)."""
    rec = np.zeros(n, dtype=PRI_DTYPE)
    rec["pos"] = pos
    rec["dir"] = direction
    rec["E"] = energy
    rec["px"] = pixel[0]
    rec["py"] = pixel[1]
    return rec


def raster_scan(nx, ny, per_pixel, pixel_size, energy, z0, spot_sigma=0.0, seed=0,
                center=(0.0, 0.0), pixel_offset=(0, 0), pixels=None, pixel_streams=True):
    """Raster scan: ``per_pixel`` primaries at each pixel centre with a
    Gaussian spot of ``spot_sigma`` nm, normal incidence, pixel-major order.

    ``pixels`` optionally restricts the scan to a list of (px, py) pairs
    (used for bounded CPU samples of a large scan); the positions of those
    pixels are exactly the ones the full scan would give them.  With
    ``pixel_streams=False`` the spot offsets come from one stream for the
    whole scan instead (much faster for 10^5+ pixels; subsets then differ).
    """
    if pixels is None:
        px, py = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
        pixels = np.stack([px.ravel(), py.ravel()], axis=1)
    pixels = np.asarray(pixels, dtype=np.int64).reshape(-1, 2)
    n = len(pixels) * per_pixel
    rec = np.zeros(n, dtype=PRI_DTYPE)
    pxr = np.repeat(pixels[:, 0], per_pixel)
    pyr = np.repeat(pixels[:, 1], per_pixel)
    x = center[0] + (pxr - (nx - 1) / 2.0) * pixel_size
    y = center[1] + (pyr - (ny - 1) / 2.0) * pixel_size
    if spot_sigma > 0 and not pixel_streams:
        off = np.random.default_rng([seed, 0x5CA9]).standard_normal((n, 2)) * spot_sigma
        x = x + off[:, 0]
        y = y + off[:, 1]
    elif spot_sigma > 0:
        # one independent stream per pixel keeps subsets identical to the full scan
        off = np.empty((n, 2))
        for k, (a, b) in enumerate(pixels):
            r = np.random.default_rng([seed, int(a), int(b)])
            off[k * per_pixel:(k + 1) * per_pixel] = r.standard_normal((per_pixel, 2)) * spot_sigma
        x = x + off[:, 0]
        y = y + off[:, 1]
    # filled column by column through a plain (n, 9) word view of the records
    # (assigning the structured fields directly is far slower)
    words = rec.view(np.float32).reshape(n, 9)
    words[:, 0] = x
    words[:, 1] = y
    words[:, 2] = z0
    words[:, 5] = -1.0
    words[:, 6] = energy
    iw = words.view(np.int32)
    iw[:, 7] = pxr + pixel_offset[0]
    iw[:, 8] = pyr + pixel_offset[1]
    return rec


def write_pri(path, rec: np.ndarray) -> None:
    np.ascontiguousarray(rec, dtype=PRI_DTYPE).tofile(path)


def read_pri(path) -> np.ndarray:
    return np.fromfile(path, dtype=PRI_DTYPE)
