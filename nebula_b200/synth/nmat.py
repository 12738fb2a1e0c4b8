"""``.nmat``: a self-describing binary stand-in for Nebula's HDF5 material files.

Nebula reads materials through ``nbl::hdf5_file`` (``io/hdf5_file.h:27-177``):
quantity attributes with units, float datasets with an optional dimension
scale (double values + unit string) per axis, and a ``units`` attribute per
dataset.  ``.nmat`` carries exactly that content, little-endian:

    magic   8 bytes  b"NBLMAT01"
    u32     number of properties
      str name, f64 value, str unit
    u32     number of datasets
      str name, str unit, u32 ndim, u64 dims[ndim]
      per axis: u8 has_scale; if 1: str unit, f64 values[dims[axis]]
      f32 data[prod(dims)]          (row-major, last axis fastest)
    str = u32 byte length + UTF-8 bytes

The C++ reader is ``nebula_b200/csrc/nmat.cpp``; the same format is what the
in-memory HDF5 stand-in used to build the reference CPU driver parses.
"""
from __future__ import annotations

import struct
import numpy as np

MAGIC = b"NBLMAT01"


def _wstr(f, s: str):
    b = s.encode()
    f.write(struct.pack("<I", len(b)))
    f.write(b)


def _rstr(buf, off):
    (n,) = struct.unpack_from("<I", buf, off)
    off += 4
    return buf[off:off + n].decode(), off + n


def write(path, raw: dict) -> None:
    with open(path, "wb") as f:
        f.write(MAGIC)
        props = raw["properties"]
        f.write(struct.pack("<I", len(props)))
        for name, (value, unit) in props.items():
            _wstr(f, name)
            f.write(struct.pack("<d", float(value)))
            _wstr(f, unit)
        ds = raw["datasets"]
        f.write(struct.pack("<I", len(ds)))
        for name, d in ds.items():
            data = np.ascontiguousarray(d["data"], dtype=np.float32)
            _wstr(f, name)
            _wstr(f, d["unit"])
            f.write(struct.pack("<I", data.ndim))
            f.write(struct.pack("<%dQ" % data.ndim, *data.shape))
            scales = d.get("scales") or [None] * data.ndim
            for ax, sc in enumerate(scales):
                if sc is None:
                    f.write(b"\x00")
                    continue
                unit, vals = sc
                vals = np.asarray(vals, dtype=np.float64)
                assert vals.shape == (data.shape[ax],)
                f.write(b"\x01")
                _wstr(f, unit)
                f.write(vals.astype("<f8").tobytes())
            f.write(data.astype("<f4").tobytes())


def read(path) -> dict:
    buf = open(path, "rb").read()
    if buf[:8] != MAGIC:
        raise ValueError("%s: not an .nmat file" % path)
    off = 8
    (n,) = struct.unpack_from("<I", buf, off)
    off += 4
    props = {}
    for _ in range(n):
        name, off = _rstr(buf, off)
        (value,) = struct.unpack_from("<d", buf, off)
        off += 8
        unit, off = _rstr(buf, off)
        props[name] = (value, unit)
    (n,) = struct.unpack_from("<I", buf, off)
    off += 4
    ds = {}
    for _ in range(n):
        name, off = _rstr(buf, off)
        unit, off = _rstr(buf, off)
        (ndim,) = struct.unpack_from("<I", buf, off)
        off += 4
        dims = struct.unpack_from("<%dQ" % ndim, buf, off)
        off += 8 * ndim
        scales = []
        for ax in range(ndim):
            has = buf[off]
            off += 1
            if not has:
                scales.append(None)
                continue
            su, off = _rstr(buf, off)
            vals = np.frombuffer(buf, dtype="<f8", count=dims[ax], offset=off).copy()
            off += 8 * dims[ax]
            scales.append((su, vals))
        cnt = int(np.prod(dims))
        data = np.frombuffer(buf, dtype="<f4", count=cnt, offset=off).reshape(dims).copy()
        off += 4 * cnt
        ds[name] = dict(unit=unit, data=data, scales=scales)
    return dict(properties=props, datasets=ds)
