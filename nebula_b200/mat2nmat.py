"""Convert Nebula HDF5 material files (``.mat``) to ``.nmat``.

    python -m nebula_b200.mat2nmat material.mat material.nmat

A ``.mat`` file as ``nbl::hdf5_file`` reads it (``io/hdf5_file.cpp``):

* quantities as attributes of the root group, a compound of a double
  ``value`` and a string ``unit`` (``read_attribute_quantity``,
  hdf5_file.cpp:72-101); string-valued attributes are not material data and
  are left out;
* tables as float datasets with a ``units`` string attribute, each axis
  optionally carrying a dimension scale: a 1-D double dataset with its own
  ``units`` attribute, the first scale attached being the one used
  (``get_dimscale``, hdf5_file.cpp:108-151).

``.nmat`` (``nebula_b200/synth/nmat.py``) holds exactly these: every
quantity, every non-scale dataset under its full path with its unit, data
and per-axis scales.  Reading needs ``h5py``, imported only when converting a
file; ``read_mat`` itself works on any object with h5py's ``File`` interface.
"""
from __future__ import annotations

import sys

import numpy as np

from .synth import nmat


def _text(v) -> str:
    if isinstance(v, bytes):
        return v.decode()
    if isinstance(v, np.ndarray) and v.shape == ():
        return _text(v[()])
    return str(v)


def _quantity(v):
    """(value, unit) of a compound attribute, or None for any other kind."""
    names = getattr(getattr(v, "dtype", None), "names", None)
    if not names or "value" not in names or "unit" not in names:
        return None
    return float(v["value"]), _text(v["unit"])


def read_mat(f) -> dict:
    """The raw material content (``properties``, ``datasets``) of an open
    HDF5 material file, in the structure ``nmat.write`` takes."""
    props = {}
    for name, v in f.attrs.items():
        q = _quantity(v)
        if q is not None:
            props[name] = q
    datasets = {}

    def visit(name, obj):
        if not hasattr(obj, "dims") or getattr(obj, "is_scale", False):
            return
        data = np.asarray(obj[()], dtype=np.float32)
        unit = _text(obj.attrs["units"]) if "units" in obj.attrs else ""
        scales = []
        for ax in range(data.ndim):
            attached = obj.dims[ax]
            if len(attached) == 0:
                scales.append(None)
                continue
            sc = attached[0]
            vals = np.asarray(sc[()], dtype=np.float64).reshape(-1)
            if vals.shape[0] != data.shape[ax]:
                raise ValueError("%s: dimension scale %d has %d values for an axis of %d"
                                 % (name, ax, vals.shape[0], data.shape[ax]))
            scales.append((_text(sc.attrs["units"]) if "units" in sc.attrs else "", vals))
        datasets["/" + name.lstrip("/")] = dict(unit=unit, data=data, scales=scales)

    f.visititems(visit)
    return dict(properties=props, datasets=datasets)


def convert(src: str, dst: str) -> dict:
    try:
        import h5py
    except ImportError as e:  # pragma: no cover - depends on the installation
        raise RuntimeError("reading .mat files needs h5py") from e
    with h5py.File(src, "r") as f:
        raw = read_mat(f)
    nmat.write(dst, raw)
    return raw


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print("usage: python -m nebula_b200.mat2nmat <material.mat> <material.nmat>", file=sys.stderr)
        return 1
    raw = convert(argv[0], argv[1])
    print("%s: %d quantities, %d tables" % (argv[1], len(raw["properties"]), len(raw["datasets"])), file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
