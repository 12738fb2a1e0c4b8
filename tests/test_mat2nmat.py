"""The .mat -> .nmat converter (nebula_b200/mat2nmat.py) on an in-memory
object with h5py's File interface laid out as Nebula's HDF5 material files
are (quantity attributes on the root group, tables with a ``units``
attribute and attached dimension scales, a string attribute that is not
material data): the content read back equals what was laid out, and the
written .nmat loads to the same transformed tables as the original."""
import numpy as np

import nebula_b200 as nb
from nebula_b200 import mat2nmat
from nebula_b200.synth import materials, nmat

QDTYPE = np.dtype([("value", "<f8"), ("unit", object)])


class _Attrs(dict):
    pass


class _Dataset:
    def __init__(self, data, unit=None, is_scale=False):
        self._data = np.asarray(data)
        self.attrs = _Attrs()
        if unit is not None:
            self.attrs["units"] = unit.encode()          # HDF5 strings arrive as bytes
        self.is_scale = is_scale
        self.dims = [[] for _ in range(self._data.ndim)]

    @property
    def ndim(self):
        return self._data.ndim

    def __getitem__(self, key):
        assert key == ()
        return self._data


class _File:
    """Just the parts of h5py.File that the converter touches."""

    def __init__(self, raw):
        self.attrs = _Attrs()
        for name, (value, unit) in raw["properties"].items():
            self.attrs[name] = np.array((value, unit.encode()), dtype=QDTYPE)[()]
        self.attrs["name"] = np.bytes_(b"silicon")          # not a quantity: skipped
        self._items = []
        for name, d in raw["datasets"].items():
            ds = _Dataset(d["data"].astype(np.float32), d["unit"])
            for ax, sc in enumerate(d.get("scales") or []):
                if sc is None:
                    continue
                scale = _Dataset(np.asarray(sc[1], np.float64), sc[0], is_scale=True)
                ds.dims[ax].append(scale)
                self._items.append((name.lstrip("/") + "_scale%d" % ax, scale))
            self._items.append((name.lstrip("/"), ds))

    def visititems(self, fn):
        for name, obj in self._items:
            fn(name, obj)


def _same(a, b):
    assert a["properties"].keys() == b["properties"].keys()
    for k, (v, u) in a["properties"].items():
        assert b["properties"][k] == (v, u)
    assert a["datasets"].keys() == b["datasets"].keys()
    for k, d in a["datasets"].items():
        e = b["datasets"][k]
        assert d["unit"] == e["unit"]
        assert np.array_equal(np.asarray(d["data"], np.float32), e["data"])
        for s, t in zip(d.get("scales") or [], e["scales"]):
            assert (s is None) == (t is None)
            if s is not None:
                assert s[0] == t[0] and np.array_equal(np.asarray(s[1], np.float64), t[1])


def test_read_mat_recovers_the_material_content():
    for spec, model in ((materials.silicon(), "full_penn"), (materials.pmma(), "kieft")):
        raw = materials.build_raw_material(spec, inelastic=model)
        got = mat2nmat.read_mat(_File(raw))
        _same(raw, got)
        assert "name" not in got["properties"]


def test_converted_file_loads_to_the_same_tables(tmp_path):
    raw = materials.build_raw_material(materials.silicon())
    a, b = str(tmp_path / "direct.nmat"), str(tmp_path / "converted.nmat")
    nmat.write(a, raw)
    nmat.write(b, mat2nmat.read_mat(_File(raw)))
    ta, tb = nb.Material.load(a).tables(), nb.Material.load(b).tables()
    assert ta.keys() == tb.keys()
    for k in ta:
        x, y = ta[k], tb[k]
        if isinstance(x, tuple):
            for u, v in zip(x, y):
                assert np.array_equal(np.asarray(u), np.asarray(v))
        elif isinstance(x, dict):
            assert x == y
        else:
            assert np.array_equal(np.asarray(x), np.asarray(y))


def test_usage():
    assert mat2nmat.main([]) == 1
