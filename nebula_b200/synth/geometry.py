"""Synthetic triangle meshes in Nebula's ``.tri`` convention.

A triangle is ``(material_in, material_out, A, B, C)`` with its normal
``(B - A) x (C - A)`` pointing from ``material_in`` towards ``material_out``
(``core/triangle.h:66-67``; ``io/load_tri_file.cpp:8-60`` reads 11 columns:
in, out, then 9 coordinates in nm).  Special material ids are the
reference's (``core/material_manager.h:77-86``).

Arrays returned here are float64 of shape (N, 11); ``write_tri`` prints them
with round-trip precision so that ``std::stod`` followed by a cast to float
gives the same float32 vertices as ``np.float32`` of these values.
"""
from __future__ import annotations

import numpy as np

NOP = -128
TERMINATOR = -127
DETECTOR = -126
DETECTOR_LT50 = -125
DETECTOR_GE50 = -124
VACUUM = -123
MIRROR = -122


def _quad(out, mi, mo, p0, p1, p2, p3):
    """Two triangles for the planar quad p0-p1-p2-p3 (counter-clockwise seen
    from the side the normal points to)."""
    out.append([mi, mo, *p0, *p1, *p2])
    out.append([mi, mo, *p0, *p2, *p3])


def box(out, lo, hi, mat_in, mat_out, skip_top=False):
    """Axis-aligned box with outward normals."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    # bottom (-z)
    _quad(out, mat_in, mat_out, (x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0))
    if not skip_top:
        _quad(out, mat_in, mat_out, (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1))
    # -x
    _quad(out, mat_in, mat_out, (x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0))
    # +x
    _quad(out, mat_in, mat_out, (x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1))
    # -y
    _quad(out, mat_in, mat_out, (x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1))
    # +y
    _quad(out, mat_in, mat_out, (x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0))


def detector_plane(out, z, half_x, half_y):
    _quad(out, VACUUM, DETECTOR, (-half_x, -half_y, z), (half_x, -half_y, z),
          (half_x, half_y, z), (-half_x, half_y, z))


def slab(size=1000.0, detector_z=10.0):
    """The slab: a ``size``^3 material-0 cube with its top at z=0,
    vacuum outside, and a detector plane at ``detector_z`` over the footprint."""
    h = size / 2
    out = []
    box(out, (-h, -h, -size), (h, h, 0.0), 0, VACUUM)
    detector_plane(out, detector_z, h, h)
    return np.asarray(out, dtype=np.float64)


def _line_profile(center, top_cd, height, sidewall_deg):
    """x of the left/right edges at bottom and top of a trapezoidal line."""
    run = height / np.tan(np.deg2rad(sidewall_deg))
    bl, br = center - top_cd / 2 - run, center + top_cd / 2 + run
    tl, tr = center - top_cd / 2, center + top_cd / 2
    return bl, br, tl, tr


def grating(n_lines=8, pitch=32.0, top_cd=16.0, sidewall_deg=86.0, height=30.0,
            size=1000.0, y_segments=50, detector_z=50.0, line_mat=1, sub_mat=0,
            edge_fn=None, z_rows=1, line_length=None):
    """Line-space grating of trapezoidal lines on the slab substrate.

    Lines run along y, centred on x=0.  Each line is cut into ``y_segments``
    segments along y (and its sidewalls into ``z_rows`` rows) so that the
    mesh has the requested triangle density.  ``edge_fn(line, side, y)``
    (optional) returns an x displacement of the sidewall at ``y`` (nm),
    used for line-edge roughness.
    """
    h = size / 2
    L = size if line_length is None else line_length
    out = []
    # substrate: all faces but the top, which is tessellated below
    box(out, (-h, -h, -size), (h, h, 0.0), sub_mat, VACUUM, skip_top=True)

    centers = (np.arange(n_lines) - (n_lines - 1) / 2) * pitch
    ys = np.linspace(-L / 2, L / 2, y_segments + 1)
    zs = np.linspace(0.0, height, z_rows + 1)

    def edges(i, y):
        bl, br, tl, tr = _line_profile(centers[i], top_cd, height, sidewall_deg)
        dl = edge_fn(i, 0, y) if edge_fn else 0.0
        dr = edge_fn(i, 1, y) if edge_fn else 0.0
        return bl + dl, br + dr, tl + dl, tr + dr

    def xz(i, y, side, z):
        bl, br, tl, tr = edges(i, y)
        t = z / height
        if side == 0:
            return bl + (tl - bl) * t
        return br + (tr - br) * t

    # substrate top outside the line region (y beyond the lines)
    if L < size:
        _quad(out, sub_mat, VACUUM, (-h, -h, 0.0), (h, -h, 0.0), (h, -L / 2, 0.0), (-h, -L / 2, 0.0))
        _quad(out, sub_mat, VACUUM, (-h, L / 2, 0.0), (h, L / 2, 0.0), (h, h, 0.0), (-h, h, 0.0))

    for s in range(y_segments):
        y0, y1 = ys[s], ys[s + 1]
        # substrate top strip: gaps to vacuum, line footprints to line material
        xs0 = [-h]
        xs1 = [-h]
        for i in range(n_lines):
            bl0, br0, _, _ = edges(i, y0)
            bl1, br1, _, _ = edges(i, y1)
            xs0 += [bl0, br0]
            xs1 += [bl1, br1]
        xs0.append(h)
        xs1.append(h)
        for k in range(len(xs0) - 1):
            mo = line_mat if (k % 2 == 1) else VACUUM
            _quad(out, sub_mat, mo, (xs0[k], y0, 0.0), (xs0[k + 1], y0, 0.0),
                  (xs1[k + 1], y1, 0.0), (xs1[k], y1, 0.0))
        for i in range(n_lines):
            for r in range(z_rows):
                za, zb = zs[r], zs[r + 1]
                # left sidewall (normal towards -x)
                _quad(out, line_mat, VACUUM,
                      (xz(i, y0, 0, za), y0, za), (xz(i, y0, 0, zb), y0, zb),
                      (xz(i, y1, 0, zb), y1, zb), (xz(i, y1, 0, za), y1, za))
                # right sidewall (normal towards +x)
                _quad(out, line_mat, VACUUM,
                      (xz(i, y0, 1, za), y0, za), (xz(i, y1, 1, za), y1, za),
                      (xz(i, y1, 1, zb), y1, zb), (xz(i, y0, 1, zb), y0, zb))
            # top
            _, _, tl0, tr0 = edges(i, y0)
            _, _, tl1, tr1 = edges(i, y1)
            _quad(out, line_mat, VACUUM, (tl0, y0, height), (tr0, y0, height),
                  (tr1, y1, height), (tl1, y1, height))
    # line end caps at y = -L/2 (normal -y) and y = +L/2 (normal +y)
    for i in range(n_lines):
        for y, sgn in ((ys[0], -1), (ys[-1], 1)):
            bl, br, tl, tr = edges(i, y)
            if sgn < 0:
                _quad(out, line_mat, VACUUM, (bl, y, 0.0), (br, y, 0.0), (tr, y, height), (tl, y, height))
            else:
                _quad(out, line_mat, VACUUM, (bl, y, 0.0), (tl, y, height), (tr, y, height), (br, y, 0.0))
    detector_plane(out, detector_z, h, h)
    return np.asarray(out, dtype=np.float64)


def gaussian_random_field_1d(n, spacing, sigma, corr_len, rng):
    """Stationary Gaussian process with exponential correlation
    sigma^2 exp(-|dy|/corr_len) sampled on a regular grid: an AR(1) recursion,
    which is exact for this covariance."""
    rho = np.exp(-spacing / corr_len)
    x = np.empty(n)
    x[0] = rng.standard_normal() * sigma
    noise = rng.standard_normal(n) * sigma * np.sqrt(1 - rho * rho)
    for i in range(1, n):
        x[i] = rho * x[i - 1] + noise[i]
    return x


def rough_grating(n_lines=16, pitch=32.0, top_cd=16.0, sidewall_deg=86.0, height=30.0,
                  size=1000.0, line_length=500.0, vertex_spacing=0.25, sigma=1.5,
                  corr_len=20.0, z_rows=8, seed=1234, detector_z=50.0):
    """Grating with line-edge roughness (about 1.2 M triangles
    at the defaults)."""
    rng = np.random.default_rng(seed)
    nseg = int(round(line_length / vertex_spacing))
    ys = np.linspace(-line_length / 2, line_length / 2, nseg + 1)
    fields = {(i, s): gaussian_random_field_1d(nseg + 1, vertex_spacing, sigma, corr_len, rng)
              for i in range(n_lines) for s in range(2)}

    def edge_fn(i, side, y):
        k = int(round((y - ys[0]) / vertex_spacing))
        return fields[(i, side)][k]

    return grating(n_lines=n_lines, pitch=pitch, top_cd=top_cd, sidewall_deg=sidewall_deg,
                   height=height, size=size, y_segments=nseg, detector_z=detector_z,
                   edge_fn=edge_fn, z_rows=z_rows, line_length=line_length)


def write_tri(path, tris: np.ndarray) -> None:
    with open(path, "w") as f:
        for t in tris:
            f.write("%d %d %s\n" % (int(t[0]), int(t[1]), " ".join(repr(float(v)) for v in t[2:])))


def read_tri(path) -> np.ndarray:
    rows = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            v = s.split()
            if len(v) != 11:
                raise ValueError("invalid number of columns")
            rows.append([float(x) for x in v])
    return np.asarray(rows, dtype=np.float64).reshape(-1, 11)
