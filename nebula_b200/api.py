"""Python host API over the C ABI.

Names follow the reference's driver (drivers/gpu/gpu_driver.h:56-178:
``push``, ``do_iteration``, ``get_running_count``, ``get_detected_count``,
``flush_buffered``) and its inputs (``.tri`` triangles, material files,
``.pri`` records).  Every call goes through ``libnebula_b200.so``; there is
no Python or CPU implementation behind these classes.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from . import _capi
from ._capi import lib, check

PRI_DTYPE = np.dtype([("pos", "<f4", 3), ("dir", "<f4", 3), ("E", "<f4"), ("px", "<i4"), ("py", "<i4")])
# nbl_deposit_record: position, energy before the event, energy lost, pixel (28 bytes)
DEPOSIT_DTYPE = np.dtype([("pos", "<f4", 3), ("E", "<f4"), ("loss", "<f4"), ("px", "<i4"), ("py", "<i4")])
assert PRI_DTYPE.itemsize == C.sizeof(_capi.Record) == 36
TRI_DTYPE = np.dtype([("material_in", "<i4"), ("material_out", "<i4"), ("r0", "<f4", 3), ("e1", "<f4", 3),
                      ("e2", "<f4", 3)])
assert TRI_DTYPE.itemsize == C.sizeof(_capi.Triangle) == 44


def _fp(a):
    return a.ctypes.data_as(_capi.f32p)


def _ip(a):
    return a.ctypes.data_as(_capi.i32p)


def triangles_from_vertices(tri11: np.ndarray) -> np.ndarray:
    """(N, 11) rows ``in, out, A, B, C`` (as a .tri file holds them) to the
    triangle layout: vertices rounded to float32, edges r1-r0 and r2-r0
    computed in float32 (core/triangle.inl:1-5)."""
    tri11 = np.asarray(tri11, dtype=np.float64).reshape(-1, 11)
    out = np.zeros(len(tri11), TRI_DTYPE)
    out["material_in"] = tri11[:, 0].astype(np.int32)
    out["material_out"] = tri11[:, 1].astype(np.int32)
    a = tri11[:, 2:5].astype(np.float32)
    b = tri11[:, 5:8].astype(np.float32)
    c = tri11[:, 8:11].astype(np.float32)
    out["r0"] = a
    out["e1"] = b - a
    out["e2"] = c - a
    return out


class Geometry:
    """Triangle mesh indexed by the linearised octree."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    @classmethod
    def from_triangles(cls, tris, max_depth=0, split_count=0):
        """Build from ``TRI_DTYPE`` records or (N, 11) vertex rows."""
        if not (isinstance(tris, np.ndarray) and tris.dtype == TRI_DTYPE):
            tris = triangles_from_vertices(tris)
        tris = np.ascontiguousarray(tris)
        h = C.c_void_p()
        check(lib().nbl_geometry_build(tris.ctypes.data_as(C.POINTER(_capi.Triangle)), len(tris), max_depth,
                                       split_count, C.byref(h)))
        return cls(h)

    @classmethod
    def from_tri_file(cls, path, max_depth=0, split_count=0):
        p = C.POINTER(_capi.Triangle)()
        n = C.c_int64()
        check(lib().nbl_load_tri_file(path.encode(), C.byref(p), C.byref(n)))
        try:
            buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(n.value * 44,)).copy()
        finally:
            lib().nbl_free(p)
        return cls.from_triangles(buf.view(TRI_DTYPE), max_depth, split_count)

    @classmethod
    def from_linearized(cls, octree_data, tris, center, halfsize):
        od = np.ascontiguousarray(octree_data, np.int32)
        tris = np.ascontiguousarray(tris, TRI_DTYPE)
        c = np.ascontiguousarray(center, np.float32)
        hs = np.ascontiguousarray(halfsize, np.float32)
        h = C.c_void_p()
        check(lib().nbl_geometry_from_linearized(_ip(od), len(od), tris.ctypes.data_as(C.POINTER(_capi.Triangle)),
                                                 len(tris), _fp(c), _fp(hs), C.byref(h)))
        return cls(h)

    def info(self):
        n_oct, n_tri = C.c_int64(), C.c_int64()
        c = np.zeros(3, np.float32)
        hs = np.zeros(3, np.float32)
        ext = np.zeros(1, np.float32)
        check(lib().nbl_geometry_info(self._h, C.byref(n_oct), C.byref(n_tri), _fp(c), _fp(hs), _fp(ext)))
        return dict(n_octree=n_oct.value, n_triangles=n_tri.value, center=c, halfsize=hs, max_extent=float(ext[0]))

    def export(self):
        """(octree_data int32, triangles TRI_DTYPE) in the linearised order."""
        inf = self.info()
        od = np.zeros(inf["n_octree"], np.int32)
        tr = np.zeros(inf["n_triangles"], TRI_DTYPE)
        check(lib().nbl_geometry_export(self._h, _ip(od), tr.ctypes.data_as(C.POINTER(_capi.Triangle))))
        return od, tr

    def ray_query(self, pos, dirs, dist, ignore_tri=None, ignore_mat=None, device=0):
        """Nearest triangle hit for each ray on the device (bit-exact with the
        reference's octree walk).  Returns (distance, triangle or -1)."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        n = len(pos)
        dirs = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        dist = np.ascontiguousarray(dist, np.float32).reshape(-1)
        it = np.full(n, -1, np.int32) if ignore_tri is None else np.ascontiguousarray(ignore_tri, np.int32)
        im = np.full(n, -123, np.int32) if ignore_mat is None else np.ascontiguousarray(ignore_mat, np.int32)
        od = np.empty(n, np.float32)
        ot = np.empty(n, np.int32)
        check(lib().nbl_ray_query(self._h, device, n, _fp(pos), _fp(dirs), _fp(dist), _ip(it), _ip(im), _fp(od),
                                  _ip(ot)))
        return od, ot

    def close(self):
        if self._h:
            lib().nbl_geometry_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Material:
    """Scatter tables and constants of one material."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        check(lib().nbl_material_load(path.encode(), C.byref(h)))
        return cls(h)

    def tables(self):
        """Tables in the transformed domain, by name, as (data, scale) pairs,
        plus "constants" and "models" (bit 0 Full Penn, bit 1 Kieft-Bosch).
        Only the tables of the models the material carries are returned."""
        t = _capi.MaterialTables()
        check(lib().nbl_material_get_tables(self._h, C.byref(t)))
        out = {"models": int(t.models)}
        names = list(_capi.TABLE_NAMES[:2])
        if t.models & 1:
            names += list(_capi.TABLE_NAMES[2:])
        if t.models & 2:
            names += list(_capi.KIEFT_TABLE_NAMES)
        for name in names:
            tb = getattr(t, name)
            n = tb.nx * tb.ny * tb.nz
            data = np.ctypeslib.as_array(tb.data, shape=(n,)).copy().reshape(tb.nx, tb.ny, tb.nz)
            scale = np.array([tb.x_min, tb.x_step, tb.y_min, tb.y_step, tb.z_min, tb.z_step], np.float32)
            out[name] = (data, scale)
        out["constants"] = np.array([t.fermi, t.band_gap, t.barrier, t.phonon_loss, t.recoil_const], np.float32)
        return out

    def max_energy(self):
        v = np.zeros(1, np.float32)
        check(lib().nbl_material_max_energy(self._h, _fp(v)))
        return float(v[0])

    def table_lookup(self, which, x, y=None, z=None, rounddown=False, device=0):
        if isinstance(which, str):
            which = (_capi.TABLE_NAMES + _capi.KIEFT_TABLE_NAMES).index(which)
        x = np.ascontiguousarray(x, np.float32)
        n = len(x)
        y = np.ascontiguousarray(np.zeros(n) if y is None else y, np.float32)
        z = np.ascontiguousarray(np.zeros(n) if z is None else z, np.float32)
        out = np.empty(n, np.float32)
        check(lib().nbl_debug_table_lookup(self._h, device, which, int(rounddown), n, _fp(x), _fp(y), _fp(z), _fp(out)))
        return out

    def close(self):
        if self._h:
            lib().nbl_material_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def page_lock(array):
    """Page-lock the memory of a contiguous numpy array in place (for record
    sinks and streamed pushes without a staging copy); undo with
    page_unlock before the array is freed."""
    if not array.flags.c_contiguous or array.nbytes == 0:
        raise ValueError("page_lock needs a non-empty contiguous array")
    check(lib().nbl_host_register(array.ctypes.data, array.nbytes))


def page_unlock(array):
    check(lib().nbl_host_unregister(array.ctypes.data))


def physics_options(physics=None):
    """``nbl_physics_opts`` from the reference defaults (physics_config.h)
    with the entries of the dict ``physics`` overriding them, e.g.
    ``{"inelastic_model": 1, "interface_refraction": 0}``."""
    o = _capi.PhysicsOpts()
    lib().nbl_physics_defaults(C.byref(o))
    for k, v in (physics or {}).items():
        if k not in _capi.PHYSICS_OPTION_NAMES:
            raise KeyError("unknown physics option %r" % k)
        setattr(o, k, int(v))
    return o


def debug_events(kind, materials, states, mats, uniforms, geometry=None, tris=None, device=0, physics=None):
    """Run one event per case on the device with given uniforms.
    Returns (state_out, material_out, status, se_state, has_se, uniforms_used)."""
    ph = physics_options(physics)
    states = np.ascontiguousarray(states, np.float32).reshape(-1, 7)
    n = len(states)
    mats_in = np.ascontiguousarray(mats, np.int32)
    uniforms = np.ascontiguousarray(uniforms, np.float32).reshape(n, -1)
    tri = None if tris is None else np.ascontiguousarray(tris, np.int32)
    arr = (C.c_void_p * len(materials))(*[m._h.value if isinstance(m._h, C.c_void_p) else m._h for m in materials])
    so = np.empty_like(states)
    mo = np.empty(n, np.int32)
    st = np.empty(n, np.int32)
    se = np.empty_like(states)
    hs = np.empty(n, np.int32)
    us = np.empty(n, np.int32)
    check(lib().nbl_debug_event(geometry._h if geometry is not None else None, arr, len(materials), device,
                                C.byref(ph), kind, n,
                                _fp(states), _ip(mats_in), _ip(tri) if tri is not None else None, _fp(uniforms),
                                uniforms.shape[1], _fp(so), _ip(mo), _ip(st), _fp(se), _ip(hs), _ip(us)))
    return so, mo, st, se, hs, us


class Simulation:
    """One plain wavefront run on one device (the gpu_driver equivalent)."""

    def __init__(self, geometry, materials, capacity=1 << 20, seed=0x78C7E39B, energy_threshold=0.0, device=0,
                 tally=(0, 0), hist_bins=200, hist_emax=1000.0, record_capacity=0, block_size=0, grid_size=0,
                 iterations_per_graph=0, max_events=0, adjoint=False, stream=None, physics=None,
                 adjoint_w_step=0.0, deposit_capacity=0, deposit_grid=None, image_cos_range=None, walk_cells=0):
        p = _capi.Params()
        lib().nbl_params_defaults(C.byref(p))
        p.physics = physics_options(physics)
        p.device = device
        p.capacity = capacity
        p.seed = seed
        p.energy_threshold = energy_threshold
        p.tally_nx, p.tally_ny = tally
        p.hist_bins = hist_bins
        p.hist_emax = hist_emax
        p.record_capacity = record_capacity
        p.block_size = block_size
        p.grid_size = grid_size
        p.iterations_per_graph = iterations_per_graph
        p.max_events = max_events
        p.adjoint = int(bool(adjoint))
        p.adjoint_w_step = adjoint_w_step
        p.deposit_capacity = deposit_capacity
        p.walk_cells = walk_cells
        if image_cos_range is not None:
            p.image_filter.enabled = 1
            p.image_filter.cos_min, p.image_filter.cos_max = (float(v) for v in image_cos_range)
        self.deposit_grid_shape = None
        if deposit_grid is not None:
            origin, voxel, n = deposit_grid
            p.deposit_grid.origin[:] = [float(v) for v in origin]
            p.deposit_grid.voxel[:] = [float(v) for v in voxel]
            p.deposit_grid.n[:] = [int(v) for v in n]
            self.deposit_grid_shape = (int(n[2]), int(n[1]), int(n[0]))
        p.stream = stream
        p.record_capacity = record_capacity
        self.params = p
        self.tally = tuple(tally)
        self.hist_bins = hist_bins
        self.materials = list(materials)
        self.geometry = geometry
        arr = (C.c_void_p * len(self.materials))(*[m._h.value if isinstance(m._h, C.c_void_p) else m._h
                                                    for m in self.materials])
        h = C.c_void_p()
        check(lib().nbl_sim_create(geometry._h, arr, len(self.materials), C.byref(p), C.byref(h)))
        self._h = h

    # gpu_driver::push / push_to_buffer
    def push(self, records):
        records = np.ascontiguousarray(records, PRI_DTYPE)
        check(lib().nbl_sim_push_primaries(self._h, records.ctypes.data, len(records)))

    def push_streamed(self, records):
        """Queue primaries from page-locked host memory (a PRI_DTYPE array,
        e.g. a view of a pinned torch tensor) without waiting for the copy:
        the next run admits them as their chunks land.  The array must stay
        unchanged until the run returns; it is kept referenced until then."""
        records = np.asarray(records, PRI_DTYPE)
        if not records.flags.c_contiguous:
            raise ValueError("streamed primaries must be one contiguous array")
        check(lib().nbl_sim_push_primaries_streamed(self._h, records.ctypes.data, len(records)))
        self._streamed = getattr(self, "_streamed", []) + [records]

    def push_device(self, ptr, n):
        check(lib().nbl_sim_push_primaries_device(self._h, C.c_void_p(ptr), n))

    def set_primary_offset(self, first):
        """Index of the first primary pushed within a larger scan: a resumed
        or sharded scan then gives exactly the whole scan's records.  Only
        while no primaries are queued (after creation or reset())."""
        check(lib().nbl_sim_set_primary_offset(self._h, int(first)))

    # gpu_driver::do_iteration (rounded up to whole graphs)
    def do_iteration(self, n=1):
        running = C.c_int64()
        check(lib().nbl_sim_step(self._h, n, C.byref(running)))
        return running.value

    def run(self):
        check(lib().nbl_sim_run(self._h))

    def get_running_count(self):
        """Electrons in flight (started + spawned - detected - terminated)."""
        c = self.counters()
        return int(c["primaries_started"] - c["detected"] - c["terminated"] + c["spawned"])

    def get_detected_count(self):
        n = C.c_int64()
        check(lib().nbl_sim_detected_count(self._h, C.byref(n)))
        return n.value

    # gpu_driver::flush_buffered: detected electrons as 36-byte records
    def flush_detected(self, out=None):
        """Detected records; ``out`` (a PRI_DTYPE array, e.g. over pinned
        memory) receives them directly when given and large enough."""
        n = self.get_detected_count()
        if out is None or len(out) < n:
            out = np.zeros(max(n, 1), PRI_DTYPE)
        got = C.c_int64()
        check(lib().nbl_sim_drain_detected(self._h, out.ctypes.data, n, C.byref(got)))
        return out[:got.value]

    def tallies(self):
        nx, ny = self.tally
        se = np.zeros(max(nx * ny, 1), np.uint32)
        bse = np.zeros(max(nx * ny, 1), np.uint32)
        hist = np.zeros(self.hist_bins, np.uint32)
        check(lib().nbl_sim_tallies(self._h, se.ctypes.data_as(_capi.u32p), bse.ctypes.data_as(_capi.u32p),
                                    hist.ctypes.data_as(_capi.u32p)))
        if nx * ny:
            return se.reshape(ny, nx), bse.reshape(ny, nx), hist
        return None, None, hist

    def counters(self):
        c = _capi.Counters()
        check(lib().nbl_sim_counters(self._h, C.byref(c)))
        return {n: int(getattr(c, n)) for n in _capi.COUNTER_NAMES}

    def kernel_ms(self):
        v = C.c_double()
        check(lib().nbl_sim_kernel_ms(self._h, C.byref(v)))
        return v.value

    def set_seed(self, seed):
        check(lib().nbl_sim_set_seed(self._h, seed))

    def n_theta(self):
        return 3 * min(len(self.materials), 2)

    def set_theta(self, theta):
        """(inelastic scale, elastic scale, work function) per material."""
        t = np.ascontiguousarray(theta, np.float32).ravel()
        check(lib().nbl_sim_set_theta(self._h, _fp(t), len(t)))

    def get_theta(self):
        t = np.zeros(self.n_theta(), np.float32)
        check(lib().nbl_sim_get_theta(self._h, _fp(t), len(t)))
        return t

    def gradients(self, forward=None):
        """Per-pixel FP64 sums of d(SE count)/d theta and d(BSE count)/d
        theta, shape (ny, nx, 6) each (adjoint simulations only).  With
        ``adjoint_w_step > 0`` the work-function entries need ``forward``,
        the adjoint=False run of the same primaries and seed."""
        nx, ny = self.tally
        gs = np.zeros((ny, nx, 6), np.float64)
        gb = np.zeros((ny, nx, 6), np.float64)
        check(lib().nbl_sim_gradients(self._h, forward._h if forward is not None else None,
                                      gs.ctypes.data_as(C.POINTER(C.c_double)),
                                      gb.ctypes.data_as(C.POINTER(C.c_double))))
        return gs, gb

    def set_record_sink(self, out):
        """Stream detected records into ``out`` (a PRI_DTYPE array, ideally in
        page-locked memory) during later runs; None removes the sink."""
        if out is None:
            check(lib().nbl_sim_set_record_sink(self._h, None, 0))
            self._sink = None
            return
        self._sink = out
        check(lib().nbl_sim_set_record_sink(self._h, out.ctypes.data, len(out)))

    def sink_records(self):
        """The records streamed into the sink so far (a view of it)."""
        n = C.c_int64()
        check(lib().nbl_sim_sink_count(self._h, C.byref(n)))
        return self._sink[:n.value]

    def drain_deposits(self):
        """Energy-deposit records of the run so far (DEPOSIT_DTYPE), removed
        from the simulation."""
        parts = []
        chunk = 1 << 22
        while True:
            out = np.empty(chunk, DEPOSIT_DTYPE)
            n = C.c_int64()
            check(lib().nbl_sim_drain_deposits(self._h, out.ctypes.data, chunk, C.byref(n)))
            parts.append(out[:n.value])
            if n.value < chunk:
                break
        return np.concatenate(parts)

    def deposit_grid(self):
        """Deposited energy per voxel (eV, float64), shape (nz, ny, nx)."""
        g = np.zeros(self.deposit_grid_shape, np.float64)
        check(lib().nbl_sim_deposit_grid(self._h, g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    def reset(self):
        check(lib().nbl_sim_reset(self._h))
        self._streamed = []

    def close(self):
        if getattr(self, "_h", None):
            lib().nbl_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scan jobs (own geometry, primaries and seed each) in one
    persistent launch.  A job's electrons draw the random numbers a plain
    ``Simulation`` of that job alone with the job's seed draws, so per-job
    results equal the plain run's."""

    def __init__(self, geometries, materials, capacity=1 << 20, refill_threshold=1.0, block_size=256,
                 queue_factor=4, device=0, use_graph=True, energy_threshold=0.0, max_events=0, stream=None,
                 physics=None, record_capacity=0, walk_cells=0):
        p = _capi.BatchParams()
        lib().nbl_batch_params_defaults(C.byref(p))
        p.physics = physics_options(physics)
        p.device = device
        p.capacity = capacity
        p.refill_threshold = refill_threshold
        p.block_size = block_size
        p.queue_factor = queue_factor
        p.use_graph = int(bool(use_graph))
        p.energy_threshold = energy_threshold
        p.max_events = max_events
        p.stream = stream
        p.record_capacity = record_capacity
        p.walk_cells = walk_cells
        self.params = p
        self.geometries = list(geometries)
        self.materials = list(materials)
        ga = (C.c_void_p * len(self.geometries))(*[g._h.value if isinstance(g._h, C.c_void_p) else g._h
                                                   for g in self.geometries])
        ma = (C.c_void_p * len(self.materials))(*[m._h.value if isinstance(m._h, C.c_void_p) else m._h
                                                  for m in self.materials])
        h = C.c_void_p()
        check(lib().nbl_batch_create(ga, len(self.geometries), ma, len(self.materials), C.byref(p), C.byref(h)))
        self._h = h
        self.n_jobs = 0

    def set_jobs(self, jobs, primaries=None):
        """``jobs``: list of (geometry index, seed, PRI_DTYPE primaries).
        ``primaries``: optionally, the jobs' primaries already laid end to
        end in one PRI_DTYPE array (then only the lengths of the jobs'
        arrays are used)."""
        arr = (_capi.BatchJob * len(jobs))()
        first = 0
        for i, (gi, seed, pri) in enumerate(jobs):
            arr[i].geometry = gi
            arr[i].seed = seed
            arr[i].first = first
            arr[i].count = len(pri)
            first += len(pri)
        if primaries is None:
            allp = np.ascontiguousarray(np.concatenate([np.asarray(p, PRI_DTYPE) for _, _, p in jobs]), PRI_DTYPE)
        else:
            allp = np.ascontiguousarray(primaries, PRI_DTYPE)
            if len(allp) != first:
                raise ValueError("primaries hold %d records, the jobs %d" % (len(allp), first))
        check(lib().nbl_batch_set_jobs(self._h, arr, len(jobs), allp.ctypes.data, len(allp)))
        self.n_jobs = len(jobs)
        self.n_primaries = len(allp)

    def run(self):
        check(lib().nbl_batch_run(self._h))

    def job_yields(self):
        se = (C.c_uint64 * self.n_jobs)()
        bse = (C.c_uint64 * self.n_jobs)()
        check(lib().nbl_batch_job_yields(self._h, se, bse))
        return np.array(se[:], np.int64), np.array(bse[:], np.int64)

    def records(self):
        """The last run's detected records (PRI_DTYPE) and the job of each
        (uint8), in detection order; needs ``record_capacity``."""
        n = C.c_int64()
        check(lib().nbl_batch_records(self._h, None, None, 0, C.byref(n)))
        rec = np.empty(n.value, PRI_DTYPE)
        job = np.empty(n.value, np.uint8)
        if n.value:
            check(lib().nbl_batch_records(self._h, rec.ctypes.data, job.ctypes.data, n.value, C.byref(n)))
        return rec, job

    def job_records(self):
        """The last run's detected records split by job: a list of n_jobs
        PRI_DTYPE arrays (each in detection order)."""
        rec, job = self.records()
        order = np.argsort(job, kind="stable")
        bounds = np.searchsorted(job[order], np.arange(self.n_jobs + 1))
        return [rec[order[bounds[i]:bounds[i + 1]]] for i in range(self.n_jobs)]

    def counters(self):
        c = _capi.Counters()
        check(lib().nbl_batch_counters(self._h, C.byref(c)))
        return {n: int(getattr(c, n)) for n in _capi.COUNTER_NAMES}

    def kernel_ms(self):
        v = C.c_double()
        check(lib().nbl_batch_kernel_ms(self._h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            lib().nbl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
