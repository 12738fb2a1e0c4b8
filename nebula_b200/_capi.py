"""ctypes declarations of the C ABI in include/nebula_b200.h.

Loading the library is strict: ``lib()`` raises if ``libnebula_b200.so`` is
missing (there is no fallback implementation of any entry point).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnebula_b200.so")

NBL_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "BUDGET_EXCEEDED",
                5: "NAN_STATE", 6: "POOL_OVERFLOW", 7: "IO", 8: "NO_DEVICE"}

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
i64p = C.POINTER(C.c_int64)


class NblError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


class Record(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("dir", C.c_float * 3), ("energy", C.c_float),
                ("px", C.c_int32), ("py", C.c_int32)]


class Triangle(C.Structure):
    _fields_ = [("material_in", C.c_int32), ("material_out", C.c_int32),
                ("r0", C.c_float * 3), ("e1", C.c_float * 3), ("e2", C.c_float * 3)]


class Table(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("x_min", C.c_float), ("x_step", C.c_float), ("y_min", C.c_float),
                ("y_step", C.c_float), ("z_min", C.c_float), ("z_step", C.c_float),
                ("data", f32p)]


TABLE_NAMES = ("el_imfp", "el_icdf", "in_imfp", "in_omega", "in_q", "in_binding")
KIEFT_TABLE_NAMES = ("ki_imfp", "ki_w0", "ki_binding")


class MaterialTables(C.Structure):
    _fields_ = [(n, Table) for n in TABLE_NAMES] + [
        ("fermi", C.c_float), ("band_gap", C.c_float), ("barrier", C.c_float),
        ("phonon_loss", C.c_float), ("recoil_const", C.c_float), ("models", C.c_int32)] + [
        (n, Table) for n in KIEFT_TABLE_NAMES]


PHYSICS_OPTION_NAMES = ("inelastic_model", "generate_secondaries", "acoustic_phonon_loss", "atomic_recoil_loss",
                        "quantum_transmission", "interface_refraction", "interface_absorption",
                        "optical_phonon_loss", "instantaneous_momentum", "momentum_conservation")


class PhysicsOpts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in PHYSICS_OPTION_NAMES]


class DepositGrid(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("voxel", C.c_float * 3), ("n", C.c_int32 * 3)]


class ImageFilter(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("cos_min", C.c_float), ("cos_max", C.c_float)]


class Params(C.Structure):
    _fields_ = [("device", C.c_int32), ("capacity", C.c_uint32), ("energy_threshold", C.c_float),
                ("seed", C.c_uint64), ("block_size", C.c_uint32), ("grid_size", C.c_uint32),
                ("iterations_per_graph", C.c_uint32), ("record_capacity", C.c_uint32),
                ("tally_nx", C.c_int32), ("tally_ny", C.c_int32), ("hist_bins", C.c_int32),
                ("hist_emax", C.c_float), ("max_events", C.c_uint32), ("stream", C.c_void_p),
                ("physics", PhysicsOpts), ("adjoint", C.c_int32), ("adjoint_w_step", C.c_float),
                ("deposit_capacity", C.c_uint32), ("deposit_grid", DepositGrid),
                ("image_filter", ImageFilter), ("walk_cells", C.c_uint32)]


class BatchJob(C.Structure):
    _fields_ = [("geometry", C.c_int32), ("reserved", C.c_uint32), ("seed", C.c_uint64), ("first", C.c_int64),
                ("count", C.c_int64)]


class BatchParams(C.Structure):
    _fields_ = [("device", C.c_int32), ("capacity", C.c_uint32), ("refill_threshold", C.c_float),
                ("block_size", C.c_uint32), ("queue_factor", C.c_uint32), ("energy_threshold", C.c_float),
                ("max_events", C.c_uint32), ("max_iterations", C.c_uint32), ("use_graph", C.c_int32),
                ("stream", C.c_void_p), ("physics", PhysicsOpts), ("walk_cells", C.c_uint32),
                ("record_capacity", C.c_uint32)]


COUNTER_NAMES = ("flights", "boundary", "elastic", "inelastic", "spawned", "detected", "terminated",
                 "primaries_started", "walk_overflow", "nan_state", "queue_overflow",
                 "record_overflow", "event_budget", "spilled", "iterations", "primaries_total",
                 "records_pending", "deposits", "deposit_overflow", "deposits_pending", "walk_resumes")


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in COUNTER_NAMES]


# (name, restype, argtypes); restype None means void
_DECLS = [
    ("nbl_last_error_string", C.c_char_p, []),
    ("nbl_abi_version", C.c_int, []),
    ("nbl_device_count", C.c_int, [C.POINTER(C.c_int32)]),
    ("nbl_free", None, [C.c_void_p]),
    ("nbl_host_alloc", C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    ("nbl_host_free", None, [C.c_void_p]),
    ("nbl_host_register", C.c_int, [C.c_void_p, C.c_int64]),
    ("nbl_host_unregister", C.c_int, [C.c_void_p]),
    ("nbl_load_tri_file", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(Triangle)), i64p]),
    ("nbl_load_pri_file", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(Record)), i64p]),
    ("nbl_material_load", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("nbl_material_create", C.c_int, [C.POINTER(MaterialTables), C.POINTER(C.c_void_p)]),
    ("nbl_material_get_tables", C.c_int, [C.c_void_p, C.POINTER(MaterialTables)]),
    ("nbl_material_max_energy", C.c_int, [C.c_void_p, f32p]),
    ("nbl_material_destroy", None, [C.c_void_p]),
    ("nbl_geometry_build", C.c_int, [C.POINTER(Triangle), C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("nbl_geometry_from_linearized", C.c_int, [i32p, C.c_int64, C.POINTER(Triangle), C.c_int64, f32p, f32p,
                                                C.POINTER(C.c_void_p)]),
    ("nbl_geometry_info", C.c_int, [C.c_void_p, i64p, i64p, f32p, f32p, f32p]),
    ("nbl_geometry_export", C.c_int, [C.c_void_p, i32p, C.POINTER(Triangle)]),
    ("nbl_geometry_destroy", None, [C.c_void_p]),
    ("nbl_ray_query", C.c_int, [C.c_void_p, C.c_int, C.c_int64, f32p, f32p, f32p, i32p, i32p, f32p, i32p]),
    ("nbl_physics_defaults", None, [C.POINTER(PhysicsOpts)]),
    ("nbl_params_defaults", None, [C.POINTER(Params)]),
    ("nbl_sim_create", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, C.POINTER(Params),
                                 C.POINTER(C.c_void_p)]),
    ("nbl_sim_push_primaries", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("nbl_sim_push_primaries_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("nbl_sim_push_primaries_streamed", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("nbl_sim_set_primary_offset", C.c_int, [C.c_void_p, C.c_uint64]),
    ("nbl_debug_kernel_arch", C.c_int, [C.c_int, C.POINTER(C.c_int32)]),
    ("nbl_debug_philox", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("nbl_sim_step", C.c_int, [C.c_void_p, C.c_uint32, i64p]),
    ("nbl_sim_run", C.c_int, [C.c_void_p]),
    ("nbl_sim_drain_detected", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, i64p]),
    ("nbl_sim_detected_count", C.c_int, [C.c_void_p, i64p]),
    ("nbl_sim_tallies", C.c_int, [C.c_void_p, u32p, u32p, u32p]),
    ("nbl_sim_counters", C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    ("nbl_sim_reset", C.c_int, [C.c_void_p]),
    ("nbl_sim_set_seed", C.c_int, [C.c_void_p, C.c_uint64]),
    ("nbl_sim_set_theta", C.c_int, [C.c_void_p, f32p, C.c_int32]),
    ("nbl_sim_get_theta", C.c_int, [C.c_void_p, f32p, C.c_int32]),
    ("nbl_sim_gradients", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("nbl_sim_drain_deposits", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, i64p]),
    ("nbl_sim_set_record_sink", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("nbl_sim_sink_count", C.c_int, [C.c_void_p, i64p]),
    ("nbl_sim_deposit_grid", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("nbl_sim_kernel_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("nbl_sim_destroy", None, [C.c_void_p]),
    ("nbl_batch_params_defaults", None, [C.POINTER(BatchParams)]),
    ("nbl_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p), C.c_int32,
                                   C.POINTER(BatchParams), C.POINTER(C.c_void_p)]),
    ("nbl_batch_set_jobs", C.c_int, [C.c_void_p, C.POINTER(BatchJob), C.c_int32, C.c_void_p, C.c_int64]),
    ("nbl_batch_run", C.c_int, [C.c_void_p]),
    ("nbl_batch_job_yields", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("nbl_batch_records", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    ("nbl_batch_counters", C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    ("nbl_batch_kernel_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("nbl_batch_destroy", None, [C.c_void_p]),
    ("nbl_run_noalloc", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, C.POINTER(Params), C.c_void_p,
                                  C.c_int64, C.c_void_p, C.c_int64, i64p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(Counters)]),
    ("nbl_debug_table_lookup", C.c_int, [C.c_void_p, C.c_int, C.c_int32, C.c_int32, C.c_int64, f32p, f32p, f32p,
                                         f32p]),
    ("nbl_debug_event", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, C.c_int, C.POINTER(PhysicsOpts),
                                  C.c_int32, C.c_int64,
                                  f32p, i32p, i32p, f32p, C.c_int32, f32p, i32p, i32p, f32p, i32p, i32p]),
]

_lib = None


def lib():
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("nebula_b200 native library not built: %s (run python -m nebula_b200.build)"
                              % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, res, args in _DECLS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return [d[0] for d in _DECLS]


def check(status):
    if status != NBL_OK:
        raise NblError(status, lib().nbl_last_error_string().decode())
