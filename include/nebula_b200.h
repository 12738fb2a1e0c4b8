/*
 * nebula_b200 -- C ABI of the B200 electron-transport library.
 *
 * Plain C types only: every entry point returns an nbl_status, never throws,
 * and copies caller arrays during the call (the library owns all device
 * memory; the caller owns host arrays).  A simulation handle is bound to one
 * device and one CUDA stream; calls on one handle are not thread-safe,
 * distinct handles are independent and may be driven from different host
 * threads at the same time (graphs are captured in thread-local mode).
 *
 * Reference interfaces each group replaces (paths relative to the
 * reference's source/ directory):
 *   materials   material<scatter_list<full_penn, kieft_elastic>>(hdf5_file)
 *               core/material.inl:13-18, physics/full_penn.h:294-406,
 *               physics/kieft/elastic.h:120-166
 *   geometry    nbl::load_tri_file io/load_tri_file.cpp:8-60;
 *               octree_builder::octree_root + linearized_octree
 *               geometry/octree/octree_builder.cpp:171-352;
 *               octree<true>::create geometry/octree.inl:3-7, 279-313
 *   ray query   octree<gpu_flag>::propagate geometry/octree.inl:33-192
 *   simulation  gpu_driver<scatter_physics, intersect_t, octree>
 *               drivers/gpu/gpu_driver.h:56-178 (constructor, push,
 *               push_to_simulation, do_iteration, buffer_detected,
 *               flush_buffered, get_running_count, get_detected_count)
 *   records     36-byte primary / detected records io/load_pri_file.cpp:112-121,
 *               gpu_main.cu:216-223
 *   physics     compile-time physics selection physics_config.h:20-46
 */
#ifndef NEBULA_B200_H
#define NEBULA_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBL_ABI_VERSION 1

typedef enum nbl_status {
	NBL_OK = 0,
	NBL_ERR_INVALID_ARG = 1,
	NBL_ERR_OOM = 2,
	NBL_ERR_CUDA = 3,
	NBL_ERR_BUDGET_EXCEEDED = 4,   /* iteration / event budget ran out */
	NBL_ERR_NAN_STATE = 5,         /* an electron reached a NaN state */
	NBL_ERR_POOL_OVERFLOW = 6,     /* an event queue or the record buffer overflowed */
	NBL_ERR_IO = 7,                /* file missing or malformed */
	NBL_ERR_NO_DEVICE = 8
} nbl_status;

/* Message of the last failing call on this thread (never NULL). */
const char* nbl_last_error_string(void);
int nbl_abi_version(void);
/* CUDA devices this process can use (0 without a driver or device); the
 * reference's worker-per-GPU loop counts them the same way (gpu_main.cu:284-295). */
nbl_status nbl_device_count(int32_t* n);

/* Special material ids (core/material_manager.h:77-86). */
#define NBL_MAT_NOP (-128)
#define NBL_MAT_TERMINATOR (-127)
#define NBL_MAT_DETECTOR (-126)
#define NBL_MAT_DETECTOR_LT50 (-125)
#define NBL_MAT_DETECTOR_GE50 (-124)
#define NBL_MAT_VACUUM (-123)
#define NBL_MAT_MIRROR (-122)

/* ------------------------------------------------------------ records */
/* Primary electron / detected electron, 36 bytes little-endian:
 * position (nm), direction (unnormalised), kinetic energy (eV), pixel. */
typedef struct nbl_record {
	float pos[3];
	float dir[3];
	float energy;
	int32_t px, py;
} nbl_record;

/* Triangle, the reference member layout (core/triangle.h:66-76): the normal
 * (r1-r0)x(r2-r0) points from material_in to material_out; e1 = r1-r0 and
 * e2 = r2-r0 are computed in float. */
typedef struct nbl_triangle {
	int32_t material_in;
	int32_t material_out;
	float r0[3];
	float e1[3];
	float e2[3];
} nbl_triangle;

/* Read a .tri file (11 columns: in out x0 y0 z0 x1 y1 z1 x2 y2 z2, nm).
 * *out is allocated by the library; release with nbl_free. */
nbl_status nbl_load_tri_file(const char* path, nbl_triangle** out, int64_t* n);
/* Read a .pri file of 36-byte records; release with nbl_free. */
nbl_status nbl_load_pri_file(const char* path, nbl_record** out, int64_t* n);
void nbl_free(void* p);
/* Page-locked host memory for record sinks and streamed pushes: allocate
 * (release with nbl_host_free), or page-lock memory the caller owns (undo
 * with nbl_host_unregister before freeing it; a range already page-locked
 * is NBL_ERR_INVALID_ARG).  Thin wrappers of the CUDA runtime's
 * cudaMallocHost / cudaHostRegister, so a host program needs no CUDA
 * headers; no counterpart in the reference. */
nbl_status nbl_host_alloc(int64_t bytes, void** out);
void nbl_host_free(void* p);
nbl_status nbl_host_register(void* p, int64_t bytes);
nbl_status nbl_host_unregister(void* p);

/* ------------------------------------------------------------ materials */
/* A table in the reference's transformed domain (common/util/table_{1,2,3}D):
 * dense row-major data[nx][ny][nz] (ny = nz = 1 for 1-D, nz = 1 for 2-D),
 * index along each axis = (value - min) * step. */
typedef struct nbl_table {
	int32_t nx, ny, nz;
	float x_min, x_step, y_min, y_step, z_min, z_step;
	const float* data;
} nbl_table;

/* Tables and constants of one material after the reference's create()
 * transforms (full_penn::create, kieft_inelastic::create, kieft_elastic::create):
 *   el_imfp   log(elastic 1/lambda / nm^-1)      over log(E/eV)
 *   el_icdf   cos(theta)                          over log(E/eV) x P
 * Full-Penn inelastic model (full_penn.h:294-406; present when models & 1):
 *   in_imfp   log(inelastic 1/lambda / nm^-1)    over log(E/eV)
 *   in_omega  log(omega/eV)                       over log(E/eV) x P
 *   in_q      hbar q / sqrt(2m) in eV^1/2         over log(E/eV) x omega/E x P
 *   in_binding binding energy in eV, -1 = none    over log(E/eV) x log(omega/E) x P
 * Kieft-Bosch inelastic model (kieft/inelastic.h:215-331; present when models & 2):
 *   ki_imfp   log(inelastic 1/lambda / nm^-1)    over log(E/eV)
 *   ki_w0     log(omega'/eV) zero-momentum loss   over log(E/eV) x P
 *   ki_binding binding energy in eV, -1 = none    over log(E/eV) x P (get_rounddown)
 * barrier = fermi + work function (eV); band_gap -1 for metals;
 * recoil_const = 4 m_e / M (elastic.h:161-163). */
typedef struct nbl_material_tables {
	nbl_table el_imfp, el_icdf, in_imfp, in_omega, in_q, in_binding;
	float fermi, band_gap, barrier, phonon_loss, recoil_const;
	int32_t models;              /* bit 0: Full-Penn tables, bit 1: Kieft-Bosch tables */
	nbl_table ki_imfp, ki_w0, ki_binding;
} nbl_material_tables;

typedef struct nbl_material nbl_material;

/* Load a material file (.nmat: the self-describing binary equivalent of the
 * reference's HDF5 material file) and apply the reference's table transforms. */
nbl_status nbl_material_load(const char* path, nbl_material** out);
/* Create from tables already in the transformed domain (copied). */
nbl_status nbl_material_create(const nbl_material_tables* tables, nbl_material** out);
/* Views of the material's tables (valid while the material lives). */
nbl_status nbl_material_get_tables(const nbl_material* m, nbl_material_tables* out);
/* Largest energy all tables cover (scatter_list::get_max_energy). */
nbl_status nbl_material_max_energy(const nbl_material* m, float* out);
void nbl_material_destroy(nbl_material* m);

/* ------------------------------------------------------------ geometry */
typedef struct nbl_geometry nbl_geometry;

/* Build the octree from triangles the way octree_builder does: cells split
 * above `split_count` triangles until `max_depth` (reference: 16 and 21;
 * pass 0 for those defaults), triangle-box overlap on 1.01x inflated cells,
 * root box = triangle bounds + 1 nm, breadth-first linearisation with
 * triangles in first-leaf order. */
nbl_status nbl_geometry_build(const nbl_triangle* tris, int64_t n, int32_t max_depth, int32_t split_count,
	nbl_geometry** out);
/* Use an already linearised octree (octree_builder.h:209-248 layout). */
nbl_status nbl_geometry_from_linearized(const int32_t* octree_data, int64_t n_octree,
	const nbl_triangle* tris, int64_t n_tri, const float center[3], const float halfsize[3],
	nbl_geometry** out);
/* Sizes and domain of a geometry. */
nbl_status nbl_geometry_info(const nbl_geometry* g, int64_t* n_octree, int64_t* n_tri,
	float center[3], float halfsize[3], float* max_extent);
/* Copy out the linearised octree and its triangle order. */
nbl_status nbl_geometry_export(const nbl_geometry* g, int32_t* octree_data, nbl_triangle* tris);
void nbl_geometry_destroy(nbl_geometry* g);

/* Device batch of octree walks on host arrays (n rays): nearest triangle hit
 * within dist[i] along the normalised dir, ignoring triangle ignore_tri[i]
 * (-1: none) and triangles whose outgoing material is ignore_mat[i].
 * Results equal octree<false>::propagate bit for bit: out_dist is dist[i]
 * and out_tri -1 when nothing is hit. */
nbl_status nbl_ray_query(const nbl_geometry* g, int device, int64_t n, const float* pos, const float* dir,
	const float* dist, const int32_t* ignore_tri, const int32_t* ignore_mat, float* out_dist, int32_t* out_tri);

/* ------------------------------------------------------------ physics */
/* Physics selection, mirroring physics_config.h:20-46 and the option bools of
 * the models it names (full_penn.h:15-19, kieft/inelastic.h:12-23,
 * kieft/elastic.h:17-22, boundary_intersect.h:11-19).  The reference picks
 * these at compile time; here they are run-time values of one build.  Each
 * flag is 0 or 1; nbl_physics_defaults sets the reference's selection. */
typedef struct nbl_physics_opts {
	int32_t inelastic_model;        /* 0: Full Penn (default), 1: Kieft-Bosch */
	int32_t generate_secondaries;   /* 1  (both inelastic models) */
	int32_t acoustic_phonon_loss;   /* 1  elastic */
	int32_t atomic_recoil_loss;     /* 1  elastic */
	int32_t quantum_transmission;   /* 1  boundary */
	int32_t interface_refraction;   /* 1  boundary */
	int32_t interface_absorption;   /* 0  boundary (Kieft-Bosch empirical absorption) */
	int32_t optical_phonon_loss;    /* 1  Kieft-Bosch inelastic only */
	int32_t instantaneous_momentum; /* 1  Kieft-Bosch inelastic only */
	int32_t momentum_conservation;  /* 1  Kieft-Bosch inelastic only */
} nbl_physics_opts;
void nbl_physics_defaults(nbl_physics_opts* o);

/* ------------------------------------------------------------ simulation */
/* Energy deposits (the reference's energy-deposit driver,
 * drivers/cpu/energydeposit_cpu_driver.h:44-93 with the record of
 * cpu_energydep.cpp:197-204): every scatter event (not a boundary crossing)
 * that changes the kinetic energy deposits the difference at its position. */
typedef struct nbl_deposit_record {
	float pos[3];                /* nm, where the event happened */
	float energy;                /* eV, kinetic energy before the event */
	float loss;                  /* eV, energy lost in the event */
	int32_t px, py;              /* pixel of the primary */
} nbl_deposit_record;
/* Voxel grid the losses are summed into on the device (FP64, eV per voxel,
 * layout [n[2]][n[1]][n[0]]); voxel (i, j, k) covers
 * origin + (i, j, k) * voxel ... origin + (i+1, j+1, k+1) * voxel.  n = 0: off. */
typedef struct nbl_deposit_grid {
	float origin[3];
	float voxel[3];
	int32_t n[3];
} nbl_deposit_grid;

/* Detector acceptance of the per-pixel SE / BSE images (the records are not
 * filtered): a detected electron counts when the cosine of the angle between
 * its direction and +z lies in [cos_min, cos_max].  enabled = 0: all count. */
typedef struct nbl_image_filter {
	int32_t enabled;
	float cos_min, cos_max;
} nbl_image_filter;

typedef struct nbl_params {
	int32_t device;              /* CUDA device ordinal */
	uint32_t capacity;           /* refill target: primaries are added while fewer electrons are in
	                                flight; queues hold up to 8x this (secondaries); 0: 1 << 20 */
	float energy_threshold;      /* eV above the vacuum level, gpu_driver.h:56-59 */
	uint64_t seed;
	uint32_t block_size;         /* 0: 256 */
	uint32_t grid_size;          /* 0: all SMs at full occupancy */
	uint32_t iterations_per_graph; /* 0: 24 (multiple of 3) */
	uint32_t record_capacity;    /* detected records buffered on the device; 0: max(4 * capacity, 2^20) */
	int32_t tally_nx, tally_ny;  /* per-pixel SE / BSE tallies over px in [0,nx), py in [0,ny); 0: off */
	int32_t hist_bins;           /* detected-energy histogram; 0: 200 */
	float hist_emax;             /* eV; 0: 1000 */
	uint32_t max_events;         /* per-electron flight budget; 0: 1 << 22 */
	void* stream;                /* cudaStream_t to run on; NULL: a library-owned stream */
	nbl_physics_opts physics;
	int32_t adjoint;             /* 1: accumulate score functions (see nbl_sim_gradients) */
	float adjoint_w_step;        /* eV; > 0: work-function derivative by a shifted replay
	                                (see nbl_sim_gradients); 0: transmission score only */
	uint32_t deposit_capacity;   /* deposit records buffered on the device; 0: no records */
	nbl_deposit_grid deposit_grid; /* voxel grid of the losses; n = 0: none */
	nbl_image_filter image_filter; /* detector acceptance of the per-pixel images */
	uint32_t walk_cells;         /* leaf cells a flight's octree walk takes per iteration; a longer walk
	                                continues in the next iteration from where it stopped (same cells,
	                                same float values, same results); 0: 1 */
} nbl_params;
void nbl_params_defaults(nbl_params* p);

typedef struct nbl_sim nbl_sim;

typedef struct nbl_counters {
	uint64_t flights;            /* free flights = driver iterations of the reference */
	uint64_t boundary, elastic, inelastic;
	uint64_t spawned, detected, terminated, primaries_started;
	uint64_t walk_overflow, nan_state, queue_overflow, record_overflow, event_budget;
	uint64_t spilled;            /* secondaries parked in the overflow ring for lack of queue room */
	uint64_t iterations;         /* wavefront iterations launched */
	uint64_t primaries_total;    /* primaries pushed */
	uint64_t records_pending;    /* detected records not yet drained */
	uint64_t deposits;           /* scatter events that deposited energy */
	uint64_t deposit_overflow;   /* deposit records lost for lack of buffer room */
	uint64_t deposits_pending;   /* deposit records not yet drained */
	uint64_t walk_resumes;       /* flights whose walk continued in a later iteration (walk_cells) */
} nbl_counters;

nbl_status nbl_sim_create(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials,
	const nbl_params* params, nbl_sim** out);
/* Queue primaries (host records; tag = running index; pixel kept for the
 * detected records).  Mirrors gpu_driver::push / push_to_buffer. */
nbl_status nbl_sim_push_primaries(nbl_sim* s, const nbl_record* recs, int64_t n);
/* Same from device memory (records already resident in HBM). */
nbl_status nbl_sim_push_primaries_device(nbl_sim* s, const void* d_recs, int64_t n);
/* The same from page-locked host memory without waiting for the copy: the
 * records are copied in chunks on a copy stream, and the next run admits
 * each primary once its chunk has landed, so the copy overlaps the
 * transport (the reference streams its input buffer frame by frame,
 * gpu_driver.inl:215-254).  `recs` must stay valid and unchanged until the
 * next nbl_sim_run / nbl_sim_step returns or nbl_sim_reset; pageable memory
 * is rejected (use nbl_sim_push_primaries). */
nbl_status nbl_sim_push_primaries_streamed(nbl_sim* s, const nbl_record* recs, int64_t n);
/* Index of the first primary pushed within a larger scan (default 0).  A
 * primary's random numbers are keyed by the seed and this index, so a scan
 * resumed at primary k (first = k, pushing primaries k..) or split over
 * devices (each with its range's first index) gives exactly the records the
 * whole scan gives in one run (work_pool's primary cursor, work_pool.h:69-88,
 * made reproducible).  Only while no primaries are queued (after create or
 * reset); it stays set across nbl_sim_reset; first + primaries pushed must
 * stay below 2^32. */
nbl_status nbl_sim_set_primary_offset(nbl_sim* s, uint64_t first);
/* Run `iterations` wavefront iterations (rounded up to whole graphs); the
 * number still in flight or queued is returned (gpu_driver::do_iteration,
 * get_running_count).  With a record sink, stops early after a graph whose
 * records the sink could not all take: nbl_sim_sink_count then equals the
 * sink's capacity, the rest wait in the simulation, and the next
 * nbl_sim_set_record_sink delivers them first (so a caller can step a run of
 * any size through two alternating sinks). */
nbl_status nbl_sim_step(nbl_sim* s, uint32_t iterations, int64_t* running);
/* Run until every queued primary and its cascade is done. */
nbl_status nbl_sim_run(nbl_sim* s);
/* Copy detected records out (flush_buffered); *n gets the number written. */
nbl_status nbl_sim_drain_detected(nbl_sim* s, nbl_record* out, int64_t cap, int64_t* n);
/* Pending detected records on the device. */
nbl_status nbl_sim_detected_count(nbl_sim* s, int64_t* n);
/* Tallies: se/bse per pixel (tally_nx * tally_ny each, may be NULL),
 * histogram (hist_bins, may be NULL). */
nbl_status nbl_sim_tallies(nbl_sim* s, uint32_t* se_img, uint32_t* bse_img, uint32_t* hist);
nbl_status nbl_sim_counters(nbl_sim* s, nbl_counters* out);
/* Clear tallies, counters and records, forget pushed primaries, keep geometry
 * and materials (a new scan on the same sample). */
nbl_status nbl_sim_reset(nbl_sim* s);
/* Change the random-number key for the next run (e.g. a new scan on the same
 * sample); call between runs. */
nbl_status nbl_sim_set_seed(nbl_sim* s, uint64_t seed);
/* Device time of the transport iterations run so far (CUDA events around
 * each graph launch), milliseconds. */
nbl_status nbl_sim_kernel_ms(nbl_sim* s, double* ms);
void nbl_sim_destroy(nbl_sim* s);

/* Record sink: page-locked host memory (pageable memory is page-locked here)
 * that receives the detected records of later runs while they run: the
 * records each graph of iterations adds to the device buffer are copied into
 * it on a copy stream while the next graph runs, so when nbl_sim_run returns
 * only the last graph's copy has been waited for.  Records of a run start at
 * host[0] after a reset (or after this call), in the order
 * nbl_sim_drain_detected would return them; nbl_sim_run with more records
 * than `capacity` fails with NBL_ERR_POOL_OVERFLOW (nbl_sim_step stops
 * instead, see there).  Records a stepped run could not fit into the previous
 * sink go first into this one (with capacity 0, to nbl_sim_drain_detected).
 * capacity 0 removes the sink (records stay in the device buffer for
 * nbl_sim_drain_detected again).  No counterpart in the reference (its
 * flush_buffered copies the whole pool per frame). */
nbl_status nbl_sim_set_record_sink(nbl_sim* s, nbl_record* host, int64_t capacity);
/* Records in the sink so far. */
nbl_status nbl_sim_sink_count(nbl_sim* s, int64_t* n);

/* Deposit records of the run so far (host copies first, in arrival order
 * within a graph); the returned ones are removed.  Needs deposit_capacity > 0. */
nbl_status nbl_sim_drain_deposits(nbl_sim* s, nbl_deposit_record* out, int64_t cap, int64_t* n);
/* The voxel grid (n[0] * n[1] * n[2] doubles, eV). */
nbl_status nbl_sim_deposit_grid(nbl_sim* s, double* out);

/* ------------------------------------------------------------ adjoint */
/* Continuous material parameters theta, 3 per material for up to 2 materials:
 * theta[3m+0] inelastic inverse-mean-free-path scale, theta[3m+1] elastic
 * scale (both 1 as loaded), theta[3m+2] work function in eV (barrier minus
 * Fermi energy as loaded).  No counterpart in the reference (its parameters
 * are fixed at material load). */
nbl_status nbl_sim_set_theta(nbl_sim* s, const float* theta, int32_t n);
nbl_status nbl_sim_get_theta(nbl_sim* s, float* theta, int32_t n);
/* Gradients of the per-pixel SE and BSE counts with respect to theta.  A
 * simulation created with params.adjoint = 1 replays each primary with the
 * same random numbers as an adjoint = 0 run with the same seed while every
 * electron carries the score d log p(path)/d theta of its own free flights
 * (chosen event and survival densities) and of its ancestry up to its
 * creation; every detection adds it to its pixel.  Output: FP64 sums,
 * [tally_ny][tally_nx][6] each; divide by the primaries of a pixel for the
 * yield gradient.
 *
 * The mean-free-path scales enter the path density only: their entries are
 * score-function (likelihood-ratio) estimates.  The work function also moves
 * the crossing deterministically (energy shift, refraction, the escape
 * threshold), which a score cannot carry.  So:
 *   adjoint_w_step = 0: the work-function entries are the score of the
 *     transmission probability alone (the replay's tallies equal the
 *     forward run's; `forward` may be NULL);
 *   adjoint_w_step = h > 0: each primary's cascade is replayed with the work
 *     functions shifted by h * r_m, r_m = +-1 drawn per primary and material,
 *     on the same random numbers; the work-function entries are
 *     (sum of r_m over the replay's detections - the same sum over `forward`'s)
 *     / h, `forward` being the adjoint = 0 run with the same seed, primaries
 *     and tally grid.  This is a central difference in expectation (the odd
 *     moments of r vanish), in the same single replay.
 * No counterpart in the reference. */
nbl_status nbl_sim_gradients(nbl_sim* s, const nbl_sim* forward, double* grad_se, double* grad_bse);

/* ------------------------------------------------------------ batched runs */
/* Many scan jobs -- each with its own geometry, primaries and seed -- fed
 * into one electron pool by a persistent kernel: every wavefront iteration of
 * the whole batch runs inside ONE cooperative launch (a grid barrier between
 * iterations instead of a kernel boundary), captured in a CUDA graph.  The
 * reference runs one scan at a time through gpu_driver (gpu_main.cu:92-232);
 * a job's electrons here draw exactly the random numbers a plain run of that
 * job alone with the same seed draws, so per-job results equal the plain
 * run's. */
typedef struct nbl_batch_job {
	int32_t geometry;          /* index into the geometries given to nbl_batch_create */
	uint32_t reserved;
	uint64_t seed;             /* the job's random-number key (as nbl_params.seed) */
	int64_t first;             /* first primary of the job in the batch's primary array */
	int64_t count;             /* its number of primaries (< 2^24) */
} nbl_batch_job;

typedef struct nbl_batch_params {
	int32_t device;
	uint32_t capacity;         /* refill target (electrons); 0: 1 << 20 */
	float refill_threshold;    /* refill only while fewer than threshold x capacity are in flight; 0: 1 */
	uint32_t block_size;       /* 128, 256 or 512; 0: 256 */
	uint32_t queue_factor;     /* population bound = factor x capacity; 0: 4 */
	float energy_threshold;
	uint32_t max_events;       /* per-electron flight budget; 0: 1 << 22 */
	uint32_t max_iterations;   /* iteration bound of one launch; 0: 1 << 20 */
	int32_t use_graph;         /* capture the launch in a CUDA graph; 0: plain launch */
	void* stream;              /* NULL: a library-owned stream */
	nbl_physics_opts physics;  /* one selection for every job */
	uint32_t walk_cells;       /* leaf cells a flight's walk takes per iteration (as nbl_params); 0: 1 */
	uint32_t record_capacity;  /* detected records kept on the device for the whole batch, each with
	                              its job (nbl_batch_records); 0: per-job yields only */
} nbl_batch_params;
void nbl_batch_params_defaults(nbl_batch_params* p);

typedef struct nbl_batch nbl_batch;
/* 1..64 geometries (staged in each block's shared memory), 1..127 materials. */
nbl_status nbl_batch_create(const nbl_geometry* const* geometries, int32_t n_geometries,
	nbl_material* const* materials, int32_t n_materials, const nbl_batch_params* params, nbl_batch** out);
/* 1..255 jobs and the batch's primary array (host records, copied; each
 * job's range [first, first+count) must lie inside it, ranges in increasing
 * order). */
nbl_status nbl_batch_set_jobs(nbl_batch* b, const nbl_batch_job* jobs, int32_t n_jobs, const nbl_record* primaries,
	int64_t n_primaries);
/* Run every job to completion in one persistent launch. */
nbl_status nbl_batch_run(nbl_batch* b);
/* Detected electrons per job: se (E < 50 eV) and bse (E >= 50 eV), n_jobs each. */
nbl_status nbl_batch_job_yields(nbl_batch* b, uint64_t* se, uint64_t* bse);
/* The last run's detected records (the 36-byte records of gpu_main.cu:216-223,
 * every job's, in detection order) and the job of each: n = how many; with
 * cap = 0 only n is returned.  Needs record_capacity > 0. */
nbl_status nbl_batch_records(nbl_batch* b, nbl_record* out, uint8_t* job, int64_t cap, int64_t* n);
nbl_status nbl_batch_counters(nbl_batch* b, nbl_counters* out);
/* Device time of the last run (CUDA events around the launch), ms. */
nbl_status nbl_batch_kernel_ms(nbl_batch* b, double* ms);
void nbl_batch_destroy(nbl_batch* b);

/* ------------------------------------------------------------ run without allocation */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (an embedding host whose allocator owns the device, a real-time loop
 * where an allocation could block or fail): the same transport as
 * nbl_sim_run, with all scratch -- queues, overflow ring, control words,
 * counters, device copies of geometry and tables -- in one fixed array of
 * NBL_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit.  No cudaMalloc/cudaFree or other allocating call is made.
 *   inputs : geometry and materials (host handles), primaries in device memory
 *   outputs: detected records (device, records_cap of them) and their count,
 *            optional per-pixel SE/BSE images (tally_nx x tally_ny, device) and
 *            histogram (hist_bins, device), all cleared first; counters (host)
 * The image filter (detector acceptance) applies as in nbl_sim_create.
 * Limits: capacity <= NBL_NOALLOC_MAX_CAPACITY (0 selects it), at most
 * NBL_NOALLOC_MAX_MATERIALS materials, geometry <= 2 MiB and tables <= 4 MiB
 * in device layout, no adjoint, no energy deposits (deposit_capacity and
 * deposit_grid must be zero); other requests are rejected.  The first call on
 * a device looks up the array's address and keeps it for the process; make it
 * before any stream capture, and make no call on a device after resetting it
 * (cudaDeviceReset).  With CUDA's default lazy module loading the array is
 * reserved at the first call on a device, not when the library is loaded:
 * make one call before giving the device to another allocator.  A call waits
 * on its stream and returns when the run is complete.
 * Calls share the array and it keeps the previous call's contents: each call
 * clears what must start at zero, and calls that overlap on the GPU race. */
#define NBL_NOALLOC_MAX_CAPACITY 2048
#define NBL_NOALLOC_MAX_MATERIALS 4
#define NBL_NOALLOC_SCRATCH_BYTES 17565696
nbl_status nbl_run_noalloc(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials,
	const nbl_params* params, const nbl_record* d_primaries, int64_t n_primaries, nbl_record* d_records,
	int64_t records_cap, int64_t* n_records, uint32_t* d_se_img, uint32_t* d_bse_img, uint32_t* d_hist,
	nbl_counters* counters);

/* ------------------------------------------------------------ debug entry points */
/* Architecture the transport kernel was loaded for on `device`, as the CUDA
 * runtime reports it (cudaFuncAttributes::binaryVersion: 100 = sm_100). */
nbl_status nbl_debug_kernel_arch(int device, int32_t* binary_version);
/* The Philox4x32-10 bijection the transport draws its random numbers from
 * (host evaluation of the same code): out = philox(counter, key). */
nbl_status nbl_debug_philox(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]);
/* Table lookups on the device (which: 0 el_imfp 1 el_icdf 2 in_imfp 3 in_omega
 * 4 in_q 5 in_binding 6 ki_imfp 7 ki_w0 8 ki_binding) for n points;
 * `rounddown` selects get_rounddown. */
nbl_status nbl_debug_table_lookup(const nbl_material* m, int device, int32_t which, int32_t rounddown,
	int64_t n, const float* x, const float* y, const float* z, float* out);
/* One event per case on the device with caller-supplied uniforms (n_uniforms
 * per case).  kind 1 inelastic, 2 elastic, 3 boundary crossing of triangle
 * tri[i] (geometry g).  state: 7 floats (pos, dir, E) in, out. */
nbl_status nbl_debug_event(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials,
	int device, const nbl_physics_opts* physics /* NULL: defaults */, int32_t kind, int64_t n, const float* state_in, const int32_t* mat_in, const int32_t* tri,
	const float* uniforms, int32_t n_uniforms, float* state_out, int32_t* mat_out, int32_t* status,
	float* se_out, int32_t* has_se, int32_t* used);

#ifdef __cplusplus
}
#endif
#endif
