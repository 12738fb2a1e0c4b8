"""Test infrastructure (oracle), not product code.

ctypes bindings for
  * ``libnbl_oracle.so`` -- the CPU restatement of the reference path
    (oracle/nbl_oracle.cpp), the model the parity tests compare against;
  * ``_ref/libnbl_ref.so`` -- the reference's own code compiled from its
    sources (oracle/ref_harness.cpp), used to pin the restatement and to make
    golden fixtures; optional (absent where the reference sources are not).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libnbl_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnbl_ref.so")
REF_CPU_MT = os.path.join(HERE, "_ref", "nebula_cpu_mt")
REF_GPU = os.path.join(HERE, "_ref", "nebula_gpu")
REF_GPU_JOBS = os.path.join(HERE, "_ref", "ref_gpu_jobs")

TABLE_NAMES = ("el_imfp", "el_icdf", "in_imfp", "in_omega", "in_q", "in_binding")
TABLE_DIMS = (1, 2, 1, 2, 3, 3)
KIEFT_TABLE_NAMES = ("ki_imfp", "ki_w0", "ki_binding")
KIEFT_TABLE_DIMS = (1, 2, 2)

# Physics selection bits (nbl_oracle.h orc_set_physics; the option bools of
# physics_config.h:20-46 and the models it names).
PHYSICS_BITS = {"generate_secondaries": 1, "acoustic_phonon_loss": 2, "atomic_recoil_loss": 4,
                "quantum_transmission": 8, "interface_refraction": 16, "interface_absorption": 32,
                "optical_phonon_loss": 64, "instantaneous_momentum": 128, "momentum_conservation": 256}
KIEFT_BIT = 65536
PHYS_DEFAULT = 0x1DF


def physics_bits(physics=None):
    """Bits for a dict of nbl_physics_opts overrides (the library's names)."""
    b = PHYS_DEFAULT
    for k, v in (physics or {}).items():
        if k == "inelastic_model":
            b = (b | KIEFT_BIT) if int(v) == 1 else (b & ~KIEFT_BIT)
        elif v:
            b |= PHYSICS_BITS[k]
        else:
            b &= ~PHYSICS_BITS[k]
    return b
PRI_DTYPE = np.dtype([("pos", "<f4", 3), ("dir", "<f4", 3), ("E", "<f4"),
                      ("px", "<i4"), ("py", "<i4")])
DEPOSIT_DTYPE = np.dtype([("pos", "<f4", 3), ("E", "<f4"), ("loss", "<f4"), ("px", "<i4"), ("py", "<i4")])

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)


def _p(a, t):
    return a.ctypes.data_as(t)


class OrcTable(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("x_min", C.c_float), ("x_step", C.c_float),
                ("y_min", C.c_float), ("y_step", C.c_float),
                ("z_min", C.c_float), ("z_step", C.c_float),
                ("data", f32p)]


class OrcMaterial(C.Structure):
    _fields_ = [(n, OrcTable) for n in TABLE_NAMES] + [
        ("fermi", C.c_float), ("band_gap", C.c_float), ("barrier", C.c_float),
        ("phonon_loss", C.c_float), ("recoil_const", C.c_float), ("models", C.c_int32)] + [
        (n, OrcTable) for n in KIEFT_TABLE_NAMES]


class OrcGeometry(C.Structure):
    _fields_ = [("octree_data", i32p), ("n_octree", C.c_int64), ("tri11", f32p),
                ("n_tri", C.c_int64), ("center", C.c_float * 3), ("halfsize", C.c_float * 3),
                ("max_extent", C.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(ORACLE_SO)
        L.orc_material_load.restype = C.c_void_p
        L.orc_material_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_material_view.restype = C.POINTER(OrcMaterial)
        L.orc_material_view.argtypes = [C.c_void_p]
        L.orc_material_free.argtypes = [C.c_void_p]
        L.orc_table_get.restype = C.c_float
        L.orc_table_get.argtypes = [C.POINTER(OrcTable), C.c_int, C.c_float, C.c_float, C.c_float]
        L.orc_table_rounddown.restype = C.c_float
        L.orc_table_rounddown.argtypes = [C.POINTER(OrcTable), C.c_int, C.c_float, C.c_float, C.c_float]
        L.orc_propagate.argtypes = [C.POINTER(OrcGeometry), f32p, f32p, C.c_float, C.c_int32,
                                    C.c_int32, f32p, i32p]
        L.orc_rng_mt.restype = C.c_void_p
        L.orc_rng_mt.argtypes = [C.c_uint32]
        L.orc_rng_list.restype = C.c_void_p
        L.orc_rng_list.argtypes = [f32p, C.c_int64]
        L.orc_rng_used.restype = C.c_int64
        L.orc_rng_used.argtypes = [C.c_void_p]
        L.orc_rng_free.argtypes = [C.c_void_p]
        L.orc_rng_unit.restype = C.c_float
        L.orc_rng_unit.argtypes = [C.c_void_p]
        L.orc_event.restype = C.c_int
        L.orc_event.argtypes = [C.POINTER(OrcGeometry), C.POINTER(OrcMaterial), C.c_int, C.c_int,
                                C.c_int32, C.c_void_p, f32p, i32p, f32p, i32p]
        for fn in (L.orc_simulate,):
            fn.restype = C.c_int64
            fn.argtypes = [C.POINTER(OrcGeometry), C.POINTER(OrcMaterial), C.c_int, C.c_void_p,
                           C.c_int64, C.c_uint32, C.c_float, C.c_void_p, C.c_int64, i64p, i64p]
        L.orc_simulate_deposits.restype = C.c_int64
        L.orc_simulate_deposits.argtypes = [C.POINTER(OrcGeometry), C.POINTER(OrcMaterial), C.c_int,
                                            C.c_void_p, C.c_int64, C.c_uint32, C.c_float, C.c_int,
                                            C.c_void_p, C.c_int64, i64p, i64p]
        L.orc_set_physics.argtypes = [C.c_uint32]
        L.orc_get_physics.restype = C.c_uint32
        L.orc_simulate_mt.restype = C.c_int64
        L.orc_simulate_mt.argtypes = [C.POINTER(OrcGeometry), C.POINTER(OrcMaterial), C.c_int,
                                      C.c_void_p, C.c_int64, C.c_uint32, C.c_float, C.c_int,
                                      C.c_void_p, C.c_int64, i64p, i64p]
        _lib = L
    return _lib


class Material:
    """Prepared material tables computed by the oracle from a .nmat file."""

    def __init__(self, path):
        err = C.create_string_buffer(512)
        self._h = lib().orc_material_load(path.encode(), err, 512)
        if not self._h:
            raise RuntimeError(err.value.decode())
        self.view = lib().orc_material_view(self._h).contents

    def table(self, name):
        t = getattr(self.view, name)
        n = t.nx * t.ny * t.nz
        data = np.ctypeslib.as_array(t.data, shape=(n,)).copy()
        scale = np.array([t.x_min, t.x_step, t.y_min, t.y_step, t.z_min, t.z_step], np.float32)
        return data.reshape(t.nx, t.ny, t.nz), scale

    def constants(self):
        v = self.view
        return np.array([v.fermi, v.band_gap, v.barrier, v.phonon_loss, v.recoil_const], np.float32)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_material_free(self._h)


def materials_array(mats):
    arr = (OrcMaterial * len(mats))()
    for i, m in enumerate(mats):
        arr[i] = m.view
    return arr


class Geometry:
    """Linearized octree (as the reference lays it out) held for the oracle."""

    def __init__(self, octree_data, tri11, center, halfsize, max_extent):
        self.octree_data = np.ascontiguousarray(octree_data, np.int32)
        self.tri11 = np.ascontiguousarray(tri11, np.float32).reshape(-1, 11)
        self.s = OrcGeometry()
        self.s.octree_data = _p(self.octree_data, i32p)
        self.s.n_octree = len(self.octree_data)
        self.s.tri11 = _p(self.tri11, f32p)
        self.s.n_tri = len(self.tri11)
        self.s.center[:] = [float(x) for x in center]
        self.s.halfsize[:] = [float(x) for x in halfsize]
        self.s.max_extent = float(max_extent)

    def propagate(self, pos, dirs, dist, ignore_tri=None, ignore_mat=None):
        n = len(pos)
        pos = np.ascontiguousarray(pos, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        dist = np.ascontiguousarray(dist, np.float32)
        it = np.full(n, -1, np.int32) if ignore_tri is None else np.asarray(ignore_tri, np.int32)
        im = np.full(n, -123, np.int32) if ignore_mat is None else np.asarray(ignore_mat, np.int32)
        od = np.empty(n, np.float32)
        ot = np.empty(n, np.int32)
        L = lib()
        d1 = np.empty(1, np.float32)
        t1 = np.empty(1, np.int32)
        for i in range(n):
            L.orc_propagate(C.byref(self.s), _p(pos[i], f32p), _p(dirs[i], f32p), float(dist[i]),
                            int(it[i]), int(im[i]), _p(d1, f32p), _p(t1, i32p))
            od[i] = d1[0]
            ot[i] = t1[0]
        return od, ot


class _physics:
    """Select the oracle's physics bits for the duration of a call."""

    def __init__(self, bits):
        self.bits = bits

    def __enter__(self):
        self.old = lib().orc_get_physics()
        lib().orc_set_physics(self.bits)

    def __exit__(self, *a):
        lib().orc_set_physics(self.old)


def event(geom, mats, kind, state, material, rng_handle, tri=-1, phys=PHYS_DEFAULT):
    """One event through the oracle; returns (state, material, status, se or None)."""
    st = np.ascontiguousarray(state, np.float32).copy()
    m = np.array([material], np.int32)
    se = np.zeros(7, np.float32)
    status = np.zeros(1, np.int32)
    arr = materials_array(mats)
    with _physics(phys):
        n = lib().orc_event(C.byref(geom.s) if geom is not None else None, arr, len(mats), kind, tri,
                            rng_handle, _p(st, f32p), _p(m, i32p), _p(se, f32p), _p(status, i32p))
    return st, int(m[0]), int(status[0]), (se if n else None)


def simulate(geom, mats, pri, seed, energy_threshold=0.0, threads=1, max_records=None, phys=PHYS_DEFAULT):
    """Run the oracle driver loop; returns (records, n_total, n_events)."""
    with _physics(phys):
        return _simulate(geom, mats, pri, seed, energy_threshold, threads, max_records)


def _simulate(geom, mats, pri, seed, energy_threshold, threads, max_records):
    pri = np.ascontiguousarray(pri, PRI_DTYPE)
    cap = max_records if max_records is not None else max(16, 4 * len(pri) + 1024)
    out = np.zeros(cap, PRI_DTYPE)
    tot = C.c_int64(0)
    ev = C.c_int64(0)
    arr = materials_array(mats)
    L = lib()
    if threads == 1:
        n = L.orc_simulate(C.byref(geom.s), arr, len(mats), pri.ctypes.data, len(pri), seed,
                           energy_threshold, out.ctypes.data, cap, C.byref(tot), C.byref(ev))
    else:
        n = L.orc_simulate_mt(C.byref(geom.s), arr, len(mats), pri.ctypes.data, len(pri), seed,
                              energy_threshold, threads, out.ctypes.data, cap, C.byref(tot),
                              C.byref(ev))
    return out[:n], tot.value, ev.value


# ----------------------------------------------------------------------------
# reference build (optional)
_ref = None


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        L.ref_last_error.restype = C.c_char_p
        L.ref_geometry_load.restype = C.c_void_p
        L.ref_geometry_load.argtypes = [C.c_char_p]
        L.ref_geometry_free.argtypes = [C.c_void_p]
        L.ref_geometry_sizes.argtypes = [C.c_void_p, i64p]
        L.ref_geometry_dump.argtypes = [C.c_void_p, i32p, f32p, f32p]
        L.ref_propagate.argtypes = [C.c_void_p, C.c_int64, f32p, f32p, f32p, i32p, i32p, f32p, i32p]
        L.ref_material_load.restype = C.c_void_p
        L.ref_material_load.argtypes = [C.c_char_p]
        L.ref_material_free.argtypes = [C.c_void_p]
        L.ref_material_table_shape.argtypes = [C.c_void_p, C.c_int, i32p, f32p]
        L.ref_material_table_data.argtypes = [C.c_void_p, C.c_int, f32p]
        L.ref_material_constants.argtypes = [C.c_void_p, f32p]
        L.ref_table_lookup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int64, f32p, f32p, f32p, f32p]
        L.ref_event.restype = C.c_int
        L.ref_event.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_uint32, C.c_int, C.c_int32,
                                C.c_uint32, f32p, i32p, f32p, C.c_int, i32p]
        L.ref_simulate_reseeded.restype = C.c_int64
        L.ref_simulate_reseeded.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.c_int64,
                                            C.c_uint32, C.c_float, C.c_void_p, C.c_int64, i64p]
        L.ref_simulate_deposits.restype = C.c_int64
        L.ref_simulate_deposits.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.c_int64,
                                            C.c_uint32, C.c_float, C.c_void_p, C.c_int64, i64p]
        L.ref_simulate.restype = C.c_int64
        L.ref_simulate.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_uint32, C.c_void_p,
                                   C.c_int64, C.c_uint32, C.c_float, C.c_void_p, C.c_int64, i64p, i64p]
        _ref = L
    return _ref


class RefGeometry:
    """The reference's octree built from a .tri file by its own builder."""

    def __init__(self, tri_path):
        L = ref()
        self.h = L.ref_geometry_load(tri_path.encode())
        if not self.h:
            raise RuntimeError(L.ref_last_error().decode())
        sz = np.zeros(2, np.int64)
        L.ref_geometry_sizes(self.h, _p(sz, i64p))
        self.octree_data = np.zeros(sz[0], np.int32)
        self.tri11 = np.zeros((sz[1], 11), np.float32)
        chx = np.zeros(7, np.float32)
        L.ref_geometry_dump(self.h, _p(self.octree_data, i32p), _p(self.tri11, f32p), _p(chx, f32p))
        self.center, self.halfsize, self.max_extent = chx[0:3], chx[3:6], float(chx[6])

    def oracle_geometry(self):
        return Geometry(self.octree_data, self.tri11, self.center, self.halfsize, self.max_extent)

    def propagate(self, pos, dirs, dist, ignore_tri=None, ignore_mat=None):
        n = len(pos)
        pos = np.ascontiguousarray(pos, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        dist = np.ascontiguousarray(dist, np.float32)
        it = np.full(n, -1, np.int32) if ignore_tri is None else np.ascontiguousarray(ignore_tri, np.int32)
        im = np.full(n, -123, np.int32) if ignore_mat is None else np.ascontiguousarray(ignore_mat, np.int32)
        od = np.empty(n, np.float32)
        ot = np.empty(n, np.int32)
        ref().ref_propagate(self.h, n, _p(pos, f32p), _p(dirs, f32p), _p(dist, f32p), _p(it, i32p),
                            _p(im, i32p), _p(od, f32p), _p(ot, i32p))
        return od, ot

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_geometry_free(self.h)


class RefMaterial:
    def __init__(self, path):
        L = ref()
        self.h = L.ref_material_load(path.encode())
        if not self.h:
            raise RuntimeError(L.ref_last_error().decode())

    def table(self, name):
        which = (TABLE_NAMES + KIEFT_TABLE_NAMES).index(name)
        shape = np.zeros(3, np.int32)
        scale = np.zeros(6, np.float32)
        ref().ref_material_table_shape(self.h, which, _p(shape, i32p), _p(scale, f32p))
        data = np.zeros(int(np.prod(shape)), np.float32)
        ref().ref_material_table_data(self.h, which, _p(data, f32p))
        return data.reshape(tuple(shape)), scale

    def constants(self):
        out = np.zeros(5, np.float32)
        ref().ref_material_constants(self.h, _p(out, f32p))
        return out

    def lookup(self, name, x, y=None, z=None, rounddown=False):
        n = len(x)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(np.zeros(n) if y is None else y, np.float32)
        z = np.ascontiguousarray(np.zeros(n) if z is None else z, np.float32)
        out = np.empty(n, np.float32)
        ref().ref_table_lookup(self.h, (TABLE_NAMES + KIEFT_TABLE_NAMES).index(name), int(rounddown), n, _p(x, f32p),
                               _p(y, f32p), _p(z, f32p), _p(out, f32p))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_material_free(self.h)


def ref_event(geom, mats, kind, state, material, seed, tri=-1, phys=PHYS_DEFAULT):
    st = np.ascontiguousarray(state, np.float32).copy()
    m = np.array([material], np.int32)
    se = np.zeros(7 * 4, np.float32)
    status = np.zeros(1, np.int32)
    hs = (C.c_void_p * len(mats))(*[x.h for x in mats])
    n = ref().ref_event(geom.h if geom is not None else None, hs, len(mats), phys, kind, tri, seed,
                        _p(st, f32p), _p(m, i32p), _p(se, f32p), 4, _p(status, i32p))
    return st, int(m[0]), int(status[0]), (se[:7].copy() if n else None)


def ref_simulate(geom, mats, pri, seed, energy_threshold=0.0, max_records=None, phys=PHYS_DEFAULT):
    pri = np.ascontiguousarray(pri, PRI_DTYPE)
    cap = max_records if max_records is not None else max(16, 4 * len(pri) + 1024)
    out = np.zeros(cap, PRI_DTYPE)
    tot = C.c_int64(0)
    ev = C.c_int64(0)
    hs = (C.c_void_p * len(mats))(*[x.h for x in mats])
    n = ref().ref_simulate(geom.h, hs, len(mats), phys, pri.ctypes.data, len(pri), seed, energy_threshold,
                           out.ctypes.data, cap, C.byref(tot), C.byref(ev))
    if n < 0:
        raise RuntimeError(ref().ref_last_error().decode())
    return out[:n], tot.value, ev.value


def simulate_deposits(geom, mats, pri, seed, energy_threshold=0.0, threads=1, max_records=None, phys=PHYS_DEFAULT):
    """The oracle's energy-deposit driver loop; returns (deposits, n_events)."""
    pri = np.ascontiguousarray(pri, PRI_DTYPE)
    cap = max_records if max_records is not None else max(1024, 600 * len(pri))
    out = np.zeros(cap, DEPOSIT_DTYPE)
    tot = C.c_int64(0)
    ev = C.c_int64(0)
    arr = materials_array(mats)
    with _physics(phys):
        n = lib().orc_simulate_deposits(C.byref(geom.s), arr, len(mats), pri.ctypes.data, len(pri), seed,
                                        energy_threshold, threads, out.ctypes.data, cap, C.byref(tot), C.byref(ev))
    if tot.value > cap:
        raise RuntimeError("deposit buffer too small")
    return out[:n], ev.value


def ref_simulate_deposits(geom, mats, pri, seed, energy_threshold=0.0, max_records=None):
    """The reference's energy-deposit driver (default physics, one thread)."""
    pri = np.ascontiguousarray(pri, PRI_DTYPE)
    cap = max_records if max_records is not None else max(1024, 600 * len(pri))
    out = np.zeros(cap, DEPOSIT_DTYPE)
    tot = C.c_int64(0)
    hs = (C.c_void_p * len(mats))(*[x.h for x in mats])
    n = ref().ref_simulate_deposits(geom.h, hs, len(mats), pri.ctypes.data, len(pri), seed, energy_threshold,
                                    out.ctypes.data, cap, C.byref(tot))
    if tot.value > cap:
        raise RuntimeError("deposit buffer too small")
    return out[:n]


def ref_simulate_reseeded(geom, mats, pri, base_seed, energy_threshold=0.0, max_records=None):
    """Reference driver with its generator reseeded per primary (base_seed + i)."""
    pri = np.ascontiguousarray(pri, PRI_DTYPE)
    cap = max_records if max_records is not None else max(16, 8 * len(pri) + 1024)
    out = np.zeros(cap, PRI_DTYPE)
    tot = C.c_int64(0)
    hs = (C.c_void_p * len(mats))(*[x.h for x in mats])
    n = ref().ref_simulate_reseeded(geom.h, hs, len(mats), pri.ctypes.data, len(pri), base_seed, energy_threshold,
                                    out.ctypes.data, cap, C.byref(tot))
    return out[:n], tot.value
