// Host-visible declarations of the device-side run state and the kernel
// launchers (implemented in transport.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "nbl_device_types.h"

namespace nbl {

// Electron state in structure-of-arrays form, one set per queue.  Three
// 16-byte vectors and one word per electron (52 B), so each field of a warp's
// 32 electrons is one fully coalesced 512-byte transaction.
struct Queue {
	float4* a;      // x, y, z, kinetic energy (eV)
	float4* b;      // direction x, y, z (unnormalised), material id (int bits)
	uint4* c;       // last triangle (-1 none), primary tag, event counter, lineage lo
	uint32_t* d;    // lineage hi
	float4* s;      // adjoint: scores d log p / d theta, parameters 0..3 (null if off)
	float2* s2;     // adjoint: parameters 4..5
	float4* w0;     // EV_WALK only: walk point x, y, z, distance left
	uint4* w1;      //   location code lo, hi, flight length (float bits), type | hop << 2 | cells << 4
};

// Counters kept on the device (64-bit).
enum : int {
	CNT_FLIGHTS = 0, CNT_BOUNDARY, CNT_ELASTIC, CNT_INELASTIC, CNT_SPAWNED, CNT_DETECTED,
	CNT_TERMINATED, CNT_PRIMARIES, CNT_WALK_OVERFLOW, CNT_NAN, CNT_QUEUE_OVERFLOW,
	CNT_RECORD_OVERFLOW, CNT_EVENT_BUDGET, CNT_SPILLED, CNT_DEPOSITS, CNT_DEPOSIT_OVERFLOW, CNT_RESUMED, N_COUNTERS
};

// Per-iteration control words, three rotating slots of 16 words:
// [queue counts x N_QUEUES, primary cursor, secondary budget, spill head,
//  spill tail at iteration start, spill pushes this iteration, work, pad].
// The flight queue's count also hands out the secondaries' tickets, so it
// can exceed the entries written: those are min(count, budget).
constexpr int SLOT_WORDS = 16;
constexpr int SLOT_CURSOR = N_QUEUES;
constexpr int SLOT_NEW_BUDGET = N_QUEUES + 1;
constexpr int SLOT_SPILL_HEAD = N_QUEUES + 2;
constexpr int SLOT_SPILL_TAIL = N_QUEUES + 3;
constexpr int SLOT_SPILL_PUSHED = N_QUEUES + 4;
constexpr int SLOT_WORK = N_QUEUES + 5;   // items handed out so far in the iteration that reads the slot
constexpr int SLOT_AVAIL = N_QUEUES + 6;  // primaries in device memory (streamed pushes), as the previous iteration saw
static_assert(SLOT_WORK < SLOT_WORDS, "control slot too small");

struct Tallies {
	uint32_t* se_img;        // per pixel counts of detected E < 50 eV (null: off)
	uint32_t* bse_img;       // per pixel counts of detected E >= 50 eV
	uint32_t* hist;          // energy histogram [n_bins]
	double* grad_se;         // adjoint: per pixel d(SE count)/d theta [n_pix][6] (null: off)
	double* grad_bse;
	int32_t* wsign_se;       // per pixel sum over detected SE of the primary's work-function
	int32_t* wsign_bse;      //   signs r_m = +-1, m = 0, 1 [n_pix][2] (null: off)
	int32_t nx, ny;          // pixel grid
	int32_t n_bins;
	float hist_emax;
	int32_t filter;          // images count only detections with cos(polar angle) in [cos_min, cos_max]
	float cos_min, cos_max;
};

struct StepParams {
	DevGeometry geom;
	const DevMaterial* mats;
	int32_t n_mat;
	float energy_threshold;
	PhiloxKey key;
	Queue q[2][N_QUEUES];
	uint32_t qcap;            // queue capacity = population bound
	uint32_t capacity;        // refill target: active electrons per iteration
	uint32_t ramp;            // most primaries refilled per iteration
	Queue spill;              // ring of secondaries that did not fit (power-of-two size)
	uint32_t spill_mask;      // ring size - 1
	uint32_t* ctrl;           // 3 slots x SLOT_WORDS
	const Record36* primaries;
	uint32_t n_primaries;
	const uint32_t* n_avail;  // primaries copied so far by a streamed push (null: all n_primaries are there)
	uint32_t tag_base;        // random-stream tag of primaries[0] (a resumed or sharded scan)
	Record36* detected;
	uint32_t* n_detected;
	uint32_t det_cap;
	uint8_t* det_job;         // batched runs: job of each detected record (null: none)
	Tallies tal;
	unsigned long long* counters;
	uint32_t max_events;      // per-electron event budget
	int32_t adjoint;          // accumulate score functions
	uint32_t refill_below;    // refill primaries only while fewer electrons are in flight
	uint32_t phys;            // physics selection (PH_* bits)
	float wstep;              // adjoint replay: work functions shifted by wstep * r_m(primary) (0: off)
	// energy deposits of scatter events (null: off)
	DepositRecord* dep;       // records [dep_cap]
	uint32_t* n_dep;
	uint32_t dep_cap;
	double* grid;             // eV per voxel [gn[2]][gn[1]][gn[0]]
	float g_org[3], g_inv[3]; // grid origin, 1 / voxel size
	int32_t gn[3];
	uint32_t walk_cells;      // leaf cells a flight's walk takes per iteration before it continues in the next
};

// Work-function sign of a primary for material m (0 or 1): +1 or -1 from a
// hash of the primary's tag and the run's key, the same in every run with
// that seed.
__device__ __forceinline__ float wsign(const PhiloxKey& key, uint32_t tag, int m)
{
	uint32_t h = tag * 0x9E3779B1u ^ key.k0 ^ (key.k1 * 0x85EBCA77u);
	h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
	return ((h >> m) & 1u) ? 1.0f : -1.0f;
}

// One job of a batched run: its geometry, its primaries (a contiguous range
// of the batch's primary array) and its random-number key.
struct DevJob {
	uint32_t geom;
	uint32_t first;
	uint32_t count;
	PhiloxKey key;
	uint32_t pad;
};

// Per-job state of a batched (persistent) run.
// A batch's geometry and job tables are staged in each block's shared memory.
constexpr int NBL_BATCH_MAX_GEOMS = 64;
constexpr int NBL_BATCH_MAX_JOBS = 255;

struct BatchParams {
	const DevGeometry* geoms;
	const DevJob* jobs;
	int32_t n_geoms;
	int32_t n_jobs;
	unsigned long long* job_se;     // detected with E < 50 eV, per job
	unsigned long long* job_bse;    // detected with E >= 50 eV, per job
	uint32_t* bar_count;            // grid barrier arrival counter
	uint32_t* bar_gen;              // grid barrier generation
	uint32_t* err;                  // bit 0: barrier timeout, bit 1: iteration bound
	uint32_t* iterations;           // iterations the launch ran
	uint32_t max_iterations;
};

// launchers
cudaError_t launch_ray_query(const DevGeometry& g, const float* pos, const float* dir, const float* dist,
	const int32_t* ignore_tri, const int32_t* ignore_mat, int64_t n, float* out_dist, int32_t* out_tri,
	cudaStream_t s);
cudaError_t launch_table_kat(const DevMaterial* mat, int which, int rounddown, int64_t n,
	const float* x, const float* y, const float* z, float* out, cudaStream_t s);
cudaError_t launch_event_kat(const DevGeometry& g, const DevMaterial* mats, uint32_t phys, int kind, int64_t n,
	const float* state_in, const int32_t* mat_in, const int32_t* tri, const float* uniforms, int32_t n_uniforms,
	float* state_out, int32_t* mat_out, int32_t* status, float* se_out, int32_t* has_se, int32_t* used,
	cudaStream_t s);
cudaError_t launch_step(const StepParams& p, uint32_t iteration, int grid, int block, cudaStream_t s);
// blocks for `block` threads at full occupancy of the step kernel that `p` selects
int step_grid_size(int device, int block, const StepParams& p);
// binary architecture (major * 10 + minor) of the loaded transport kernel
cudaError_t step_binary_version(int device, int* version);
cudaError_t launch_batch(const StepParams& p, const BatchParams& b, int grid, int block, cudaStream_t s);
int batch_grid_size(int device, int block, const StepParams& p);

}  // namespace nbl
