// Electron-transport kernels for sm_100a.
//
// The plain method is a wavefront: every iteration is ONE launch of k_step,
// which walks a combined index space
//
//     [ boundary | elastic | inelastic | new secondaries | continued walks |
//       drained spill ring | new primaries ]
//
// where the first five segments are this iteration's queues, then the
// secondaries parked in the overflow ring, then the refill from the
// device-resident primary buffer (filled so that at most `capacity`
// electrons are in flight, at most `ramp` per iteration).  Each item performs
// the interaction that ended its previous free flight, then its next free
// flight (free-path sampling + octree walk), and is appended to the next
// iteration's queue for the event that flight ended in.  A walk stops after
// `walk_cells` leaf cells (default 1); an unfinished one is appended to the
// continued-walk queue with its exact state and goes on in the next
// iteration, so a warp never waits on its lane with the longest walk.  Queues are
// structure-of-arrays and double-buffered; appends are warp-aggregated
// (one ballot and one atomic per warp and queue), so each queue segment a
// warp reads or writes is contiguous and coalesced.  Sorting items by event
// kind this way replaces the reference's per-iteration radix sort of the
// whole pool (drivers/gpu/gpu_particle_manager.inl:237-246) and keeps the
// interaction code of a warp uniform (all lanes in one segment).
//
// The reference kernels this replaces: kernels::init / intersect / elastic /
// inelastic and the pool management (drivers/gpu/gpu_driver.inl:403-566,
// gpu_particle_manager.inl:354-376).  The per-iteration control words live
// in three rotating slots so a kernel can read its counts, append to the next
// slot and clear the one after without any host round trip; a run is a
// sequence of iterations captured in CUDA graphs.
#include "kernels.cuh"
#include "device/rng.cuh"
#include "device/geometry.cuh"
#include "device/tables.cuh"
#include "device/physics.cuh"

#include <cooperative_groups.h>
#include <algorithm>
namespace cg = cooperative_groups;

#ifndef NBL_STEP_MIN_BLOCKS
#define NBL_STEP_MIN_BLOCKS 4
#endif

namespace nbl {

__device__ __forceinline__ unsigned lanemask_lt()
{
	unsigned m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

// Reserve one slot per lane with `pred` from `counter`; all 32 lanes must
// call.  Returns the lane's slot (undefined where pred is false).
__device__ __forceinline__ uint32_t warp_reserve(uint32_t* counter, bool pred)
{
	const unsigned mask = __ballot_sync(0xffffffffu, pred);
	uint32_t base = 0;
	if (mask) {
		const int leader = __ffs(mask) - 1;
		if ((int)(threadIdx.x & 31) == leader)
			base = atomicAdd(counter, (uint32_t)__popc(mask));
		base = __shfl_sync(0xffffffffu, base, leader);
	}
	return base + (uint32_t)__popc(mask & lanemask_lt());
}

// Reserve one slot per lane in the queue `q` it names (0..4, -1: none) from
// the five consecutive counters at `counters`; all 32 lanes must call.  The
// atomics of the different queues are issued together (lane t issues queue
// t's), so a warp that appends to several queues waits for one round trip
// instead of one per queue.  Returns the lane's slot (undefined for q = -1).
__device__ __forceinline__ uint32_t warp_reserve5(uint32_t* counters, int q)
{
	const unsigned m0 = __ballot_sync(0xffffffffu, q == 0), m1 = __ballot_sync(0xffffffffu, q == 1);
	const unsigned m2 = __ballot_sync(0xffffffffu, q == 2), m3 = __ballot_sync(0xffffffffu, q == 3);
	const unsigned m4 = __ballot_sync(0xffffffffu, q == 4);
	const uint32_t lane = threadIdx.x & 31u;
	const unsigned issue = lane == 0u ? m0 : lane == 1u ? m1 : lane == 2u ? m2 : lane == 3u ? m3 : m4;
	uint32_t base = 0;
	if (lane < 5u && issue)
		base = atomicAdd(counters + lane, (uint32_t)__popc(issue));
	base = __shfl_sync(0xffffffffu, base, q > 0 ? q : 0);
	const unsigned mq = q == 0 ? m0 : q == 1 ? m1 : q == 2 ? m2 : q == 3 ? m3 : m4;
	return base + (uint32_t)__popc(mq & lanemask_lt());
}

/* --------------------------------------------------------- streamed queue traffic */
// Every queue entry is written once and read once, in the next iteration:
// the event queues and the primaries stream through the 126 MB L2 at several
// hundred MB per iteration.  They are loaded and stored with an evict-first
// L2 policy and without allocating in L1, so that the caches keep the data
// that is read over and over -- octree nodes, triangles, tables.  The loads
// are ordered like the __ldcg loads they replace (the batched kernel reads
// entries that other SMs wrote before its grid barrier).
__device__ __forceinline__ uint64_t stream_policy()
{
	uint64_t p;
	asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
	return p;
}
__device__ __forceinline__ float4 ld_stream(const float4* a)
{
	float4 v;
	asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
		: "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a), "l"(stream_policy()) : "memory");
	return v;
}
__device__ __forceinline__ uint4 ld_stream(const uint4* a)
{
	uint4 v;
	asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
		: "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(a), "l"(stream_policy()) : "memory");
	return v;
}
__device__ __forceinline__ float2 ld_stream(const float2* a)
{
	float2 v;
	asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;"
		: "=f"(v.x), "=f"(v.y) : "l"(a), "l"(stream_policy()) : "memory");
	return v;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* a)
{
	uint32_t v;
	asm volatile("ld.global.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
		: "=r"(v) : "l"(a), "l"(stream_policy()) : "memory");
	return v;
}
__device__ __forceinline__ float ld_stream(const float* a)
{
	float v;
	asm volatile("ld.global.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
		: "=f"(v) : "l"(a), "l"(stream_policy()) : "memory");
	return v;
}
__device__ __forceinline__ void st_stream(float4* a, float4 v)
{
	asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
		:: "l"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(stream_policy()) : "memory");
}
__device__ __forceinline__ void st_stream(uint4* a, uint4 v)
{
	asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.u32 [%0], {%1,%2,%3,%4}, %5;"
		:: "l"(a), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "l"(stream_policy()) : "memory");
}
__device__ __forceinline__ void st_stream(float2* a, float2 v)
{
	asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f32 [%0], {%1,%2}, %3;"
		:: "l"(a), "f"(v.x), "f"(v.y), "l"(stream_policy()) : "memory");
}
__device__ __forceinline__ void st_stream(uint32_t* a, uint32_t v)
{
	asm volatile("st.global.L1::no_allocate.L2::cache_hint.u32 [%0], %1, %2;"
		:: "l"(a), "r"(v), "l"(stream_policy()) : "memory");
}

/* --------------------------------------------------------------- ray query */
__global__ void k_ray_query(const DevGeometry g, const float* __restrict__ pos, const float* __restrict__ dir,
	const float* __restrict__ dist, const int32_t* __restrict__ ignore_tri, const int32_t* __restrict__ ignore_mat,
	int64_t n, float* __restrict__ out_dist, int32_t* __restrict__ out_tri)
{
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	float d;
	const int t = propagate(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], dir[3 * i], dir[3 * i + 1], dir[3 * i + 2],
		dist[i], ignore_tri[i], ignore_mat[i], d);
	out_dist[i] = d;
	out_tri[i] = t;
}

cudaError_t launch_ray_query(const DevGeometry& g, const float* pos, const float* dir, const float* dist,
	const int32_t* ignore_tri, const int32_t* ignore_mat, int64_t n, float* out_dist, int32_t* out_tri,
	cudaStream_t s)
{
	if (n <= 0)
		return cudaSuccess;
	const int block = 128;
	const int64_t grid = (n + block - 1) / block;
	k_ray_query<<<(unsigned)grid, block, 0, s>>>(g, pos, dir, dist, ignore_tri, ignore_mat, n, out_dist, out_tri);
	return cudaGetLastError();
}

/* --------------------------------------------------------- table lookups */
__global__ void k_table_kat(const DevMaterial* __restrict__ mat, int which, int rounddown, int64_t n,
	const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ out)
{
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const DevMaterial& m = *mat;
	float v;
	switch (which) {
	case 0: v = table1_get(m.el_imfp, x[i]); break;
	case 2: v = table1_get(m.in_imfp, x[i]); break;
	case 1: v = rounddown ? table2_rounddown(m.el_icdf, x[i], y[i]) : table2_get(m.el_icdf, x[i], y[i]); break;
	case 3: v = rounddown ? table2_rounddown(m.in_omega, x[i], y[i]) : table2_get(m.in_omega, x[i], y[i]); break;
	case 4: v = rounddown ? table3_rounddown(m.in_q, x[i], y[i], z[i]) : table3_get(m.in_q, x[i], y[i], z[i]); break;
	case 5: v = rounddown ? table3_rounddown(m.in_binding, x[i], y[i], z[i]) : table3_get(m.in_binding, x[i], y[i], z[i]); break;
	case 6: v = table1_get(m.in_imfp, x[i]); break;
	case 7: v = rounddown ? table2_rounddown(m.in_omega, x[i], y[i]) : table2_get(m.in_omega, x[i], y[i]); break;
	default: v = rounddown ? table2_rounddown(m.in_binding, x[i], y[i]) : table2_get(m.in_binding, x[i], y[i]); break;
	}
	out[i] = v;
}

cudaError_t launch_table_kat(const DevMaterial* mat, int which, int rounddown, int64_t n,
	const float* x, const float* y, const float* z, float* out, cudaStream_t s)
{
	if (n <= 0)
		return cudaSuccess;
	k_table_kat<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mat, which, rounddown, n, x, y, z, out);
	return cudaGetLastError();
}

/* ---------------------------------------------------------- single events */
__global__ void k_event_kat(const DevGeometry g, const DevMaterial* __restrict__ mats, uint32_t ph, int kind, int64_t n,
	const float* __restrict__ state_in, const int32_t* __restrict__ mat_in, const int32_t* __restrict__ tri,
	const float* __restrict__ uniforms, int32_t n_uniforms, float* __restrict__ state_out,
	int32_t* __restrict__ mat_out, int32_t* __restrict__ status, float* __restrict__ se_out,
	int32_t* __restrict__ has_se, int32_t* __restrict__ used)
{
	const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	ListStream rng{ uniforms + i * n_uniforms, 0u, (uint32_t)n_uniforms };
	Electron p;
	const float* s = state_in + 7 * i;
	p.pos = v3(s[0], s[1], s[2]);
	p.dir = v3(s[3], s[4], s[5]);
	p.E = s[6];
	int mat = mat_in[i];
	int st = ST_RUNNING;
	bool spawned = false;
	Electron se;
	se.pos = v3(0, 0, 0); se.dir = v3(0, 0, 0); se.E = 0;
	if (kind == 3) {
		const DevTriangle T = load_tri(g.tris, tri[i]);
		st = boundary_event(T, mats, p, mat, rng, nullptr, ph);
	} else if (kind == 1) {
		spawned = inelastic_event(mats[mat], p, se, rng, ph);
	} else {
		elastic_event(mats[mat], p, rng, ph);
	}
	float* o = state_out + 7 * i;
	o[0] = p.pos.x; o[1] = p.pos.y; o[2] = p.pos.z; o[3] = p.dir.x; o[4] = p.dir.y; o[5] = p.dir.z; o[6] = p.E;
	float* so = se_out + 7 * i;
	so[0] = se.pos.x; so[1] = se.pos.y; so[2] = se.pos.z; so[3] = se.dir.x; so[4] = se.dir.y; so[5] = se.dir.z; so[6] = se.E;
	mat_out[i] = mat;
	status[i] = st;
	has_se[i] = spawned ? 1 : 0;
	used[i] = (int32_t)rng.n;
}

cudaError_t launch_event_kat(const DevGeometry& g, const DevMaterial* mats, uint32_t phys, int kind, int64_t n,
	const float* state_in, const int32_t* mat_in, const int32_t* tri, const float* uniforms, int32_t n_uniforms,
	float* state_out, int32_t* mat_out, int32_t* status, float* se_out, int32_t* has_se, int32_t* used,
	cudaStream_t s)
{
	if (n <= 0)
		return cudaSuccess;
	k_event_kat<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(g, mats, phys, kind, n, state_in, mat_in, tri, uniforms,
		n_uniforms, state_out, mat_out, status, se_out, has_se, used);
	return cudaGetLastError();
}

/* ----------------------------------------------------------- transport */
// Event counters of one block, in shared memory (one shared atomic per
// counted event), flushed to the device counters once per block and launch.
struct LocalCounters {
	uint32_t* c;   // shared, N_COUNTERS words
	// one shared atomic per group of lanes counting together
	__device__ __forceinline__ void add(int k)
	{
		const cg::coalesced_group g = cg::coalesced_threads();
		if (g.thread_rank() == 0)
			atomicAdd(c + k, g.size());
	}
};

// What one electron needs to know about the run it belongs to: its geometry
// and its random-number key (a batched run holds one of each per job).
struct RunView {
	const DevGeometry* geom;
	PhiloxKey key;
};

// What a flight whose walk stopped at the cell budget carries to the next
// iteration (the EV_WALK queue's w0 / w1 words).
struct FlightResume {
	WalkState w;
	float dist;      // the flight's length (sampled, or the domain extent in vacuum)
	int type;        // what ends it if no triangle does: 0 nothing (vacuum), 1 inelastic, 2 elastic
	int hop;
};

__device__ __forceinline__ void load_resume(const Queue& q, uint32_t i, FlightResume& fr)
{
	const float4 w0 = ld_stream(q.w0 + i);
	const uint4 w1 = ld_stream(q.w1 + i);
	fr.w.cx = w0.x; fr.w.cy = w0.y; fr.w.cz = w0.z; fr.w.to_go = w0.w;
	fr.w.location = ((uint64_t)w1.y << 32) | w1.x;
	fr.dist = __uint_as_float(w1.z);
	fr.type = (int)(w1.w & 3u);
	fr.hop = (int)((w1.w >> 2) & 3u);
	fr.w.steps = (int)(w1.w >> 4);
}

__device__ __forceinline__ void store_resume(const Queue& q, uint32_t i, const FlightResume& fr)
{
	st_stream(q.w0 + i, make_float4(fr.w.cx, fr.w.cy, fr.w.cz, fr.w.to_go));
	st_stream(q.w1 + i, make_uint4((uint32_t)fr.w.location, (uint32_t)(fr.w.location >> 32), __float_as_uint(fr.dist),
		(uint32_t)fr.type | ((uint32_t)fr.hop << 2) | ((uint32_t)fr.w.steps << 4)));
}

// Free flight(s) from the electron's current state: domain and energy cut,
// free-path sampling, octree walk, move.  Flights in vacuum that hit nothing
// end without an event and are repeated (the next one leaves the domain).
// Returns the queue of the event the flight ends in, -1 when the electron is
// terminated, or EV_WALK when the walk reached the run's per-iteration cell
// budget (`fr` then holds where it stands).  With `resume` non-null, the
// flight stored at entry `resume_i` of that walk queue continues (its checks,
// event count and random draws are behind it).
// Mirrors cpu_driver::init / kernels::init
// (drivers/cpu/cpu_driver.inl:74-130, drivers/gpu/gpu_driver.inl:403-480).
template<bool ADJ>
__device__ __forceinline__ int free_flight(const StepParams& P, const RunView& rv, Electron& p, int mat, int& last_tri,
	uint32_t& event, uint32_t stream_tag, uint64_t lineage, float* sc, LocalCounters& lc, const float* dbar,
	FlightResume& fr, const Queue* resume, uint32_t resume_i, const DevMaterial* mats)
{
	const DevGeometry& G = *rv.geom;
	if (resume) {
		load_resume(*resume, resume_i, fr);
		lc.add(CNT_RESUMED);
	}
	for (int hop = resume ? fr.hop : 0; hop < 4; ++hop) {
		int type = 0;
		float dist;
		float mu_el = 0.0f, mu_in = 0.0f;
		const DevMaterial* m = nullptr;
		WalkState w;
		if (resume) {
			resume = nullptr;
			type = fr.type;
			dist = fr.dist;
			w = fr.w;
			if (mat >= 0) {
				m = mats + mat;
				if (ADJ) {
					// the inverse mean free paths the flight was sampled with
					mu_el = imfp_at(m->el_imfp, m->el_scale, p.E);
					mu_in = imfp_at(m->in_imfp, m->in_scale, p.E);
				}
			}
		} else {
			lc.add(CNT_FLIGHTS);
			if (!(p.E == p.E) || !(p.pos.x == p.pos.x)) { lc.add(CNT_NAN); return -1; }
			if (!in_domain(G, p.pos.x, p.pos.y, p.pos.z))
				return -1;
			if (event >= P.max_events) { lc.add(CNT_EVENT_BUDGET); return -1; }
			++event;
			dist = G.max_extent;
			if (mat >= 0) {
				m = mats + mat;
				const float barrier = (ADJ && dbar && mat < 2) ? fa(m->barrier, dbar[mat]) : m->barrier;
				if (p.E < fa(barrier, P.energy_threshold))
					return -1;
				PhiloxStream r;
				r.init(rv.key, event, 0u, stream_tag, lineage);
				const float pe = sample_path(m->el_imfp, m->el_scale, p.E, r, mu_el);
				const float pi = sample_path(m->in_imfp, m->in_scale, p.E, r, mu_in);
				dist = __int_as_float(0x7f800000);
				if (pe < dist) { dist = pe; type = 2; }
				if (pi < dist) { dist = pi; type = 1; }
			}
			w = walk_start(p.pos.x, p.pos.y, p.pos.z, dist);
		}
		const V3 d = vnormalised(p.dir);
		float idist;
		const int hit = propagate_cells(G, w, d.x, d.y, d.z, dist, last_tri, mat, idist, (int)P.walk_cells);
		if (hit == NBL_WALK_PENDING) {
			fr.w = w;
			fr.dist = dist;
			fr.type = type;
			fr.hop = hop;
			return EV_WALK;
		}
		if (hit == -2) { lc.add(CNT_WALK_OVERFLOW); return -1; }
		if (ADJ && mat >= 0 && mat < 2) {
			// score of the flight: density mu_k exp(-(mu_in+mu_el) d) of the
			// chosen event k at distance d, or survival exp(-(mu_in+mu_el) d)
			// when a boundary cuts the flight; derivative w.r.t. the scales
			const float travel = hit >= 0 ? idist : dist;
			const float in_k = (hit < 0 && type == 1) ? 1.0f : 0.0f;
			const float el_k = (hit < 0 && type == 2) ? 1.0f : 0.0f;
			sc[3 * mat + 0] += (in_k - mu_in * travel) / m->in_scale;
			sc[3 * mat + 1] += (el_k - mu_el * travel) / m->el_scale;
		}
		if (hit >= 0) {
			p.pos = vadd(p.pos, vmul(d, idist));
			last_tri = hit;
			return EV_BOUNDARY;
		}
		p.pos = vadd(p.pos, vmul(d, dist));
		if (type == 1) return EV_INELASTIC;
		if (type == 2) return EV_ELASTIC;
	}
	return -1;
}

__device__ __forceinline__ void store_electron(const Queue& q, uint32_t slot, const Electron& p, int mat, int last_tri,
	uint32_t tag, uint32_t event, uint64_t lineage)
{
	st_stream(q.a + slot, make_float4(p.pos.x, p.pos.y, p.pos.z, p.E));
	st_stream(q.b + slot, make_float4(p.dir.x, p.dir.y, p.dir.z, __int_as_float(mat)));
	st_stream(q.c + slot, make_uint4((uint32_t)last_tri, tag, event, (uint32_t)lineage));
	st_stream(q.d + slot, (uint32_t)(lineage >> 32));
}

// Loads of data written during the same launch by other SMs bypass L1
// (the persistent kernel keeps running across iterations).
__device__ __forceinline__ uint32_t ld_ctrl(const uint32_t* p) { return __ldcg(p); }

// Job of a batched primary (global index g): the last job whose first
// primary is <= g (`jobs`: the block's shared copy of the job table).
__device__ __forceinline__ uint32_t job_of(const DevJob* jobs, int n_jobs, uint32_t g)
{
	int lo = 0, hi = n_jobs - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (jobs[mid].first <= g) lo = mid; else hi = mid - 1;
	}
	return (uint32_t)lo;
}

// The six adjoint scores of an electron, by value.
struct Scores {
	float v[6];
};

// Detection output of the lanes of a warp that detected an electron
// (`det`): per-pixel SE / BSE tallies (with the detector acceptance cone),
// adjoint gradient sums, the energy histogram and the 36-byte record
// (gpu_main.cu:216-223).  Called by every lane of a warp in which any lane
// detected; kept out of line so that the hot loop's instructions stay few.
template<bool ADJ, bool BATCH>
__device__ __noinline__ void detection_output(const StepParams* Pp, const BatchParams* Bp, bool det, Electron p,
	uint32_t rec_index, uint32_t job, PhiloxKey key, uint32_t stream_tag, Scores sc, bool wshift, uint32_t* s_counters)
{
	const StepParams& P = *Pp;
	LocalCounters lc{ s_counters };
	if (det) {
		lc.add(CNT_DETECTED);
		const Tallies& T = P.tal;
		if (BATCH) {
			atomicAdd((p.E < 50.0f ? Bp->job_se : Bp->job_bse) + job, 1ull);
		} else {
			const Record36* pr = P.primaries + rec_index;
			const int px = pr->px, py = pr->py;
			bool seen = true;
			if (T.filter) {
				// detector acceptance: polar angle of the detected direction to +z
				const float c = fdf(p.dir.z, __fsqrt_rn(vmag2(p.dir)));
				seen = c >= T.cos_min && c <= T.cos_max;
			}
			if (seen && T.se_img && px >= 0 && py >= 0 && px < T.nx && py < T.ny) {
				const size_t pix = (size_t)py * T.nx + px;
				atomicAdd((p.E < 50.0f ? T.se_img : T.bse_img) + pix, 1u);
				if (ADJ && T.grad_se) {
					double* g = (p.E < 50.0f ? T.grad_se : T.grad_bse) + pix * 6;
#pragma unroll
					for (int k = 0; k < 6; ++k)
						if (k % 3 != 2 || !wshift)
							atomicAdd(g + k, (double)sc.v[k]);
				}
				if (T.wsign_se) {
					int32_t* w = (p.E < 50.0f ? T.wsign_se : T.wsign_bse) + pix * 2;
					atomicAdd(w, (int32_t)wsign(key, stream_tag, 0));
					atomicAdd(w + 1, (int32_t)wsign(key, stream_tag, 1));
				}
			}
		}
		if (T.hist && p.E >= 0.0f && p.E < T.hist_emax) {
			int bin = (int)(p.E / T.hist_emax * (float)T.n_bins);
			bin = bin < T.n_bins ? bin : T.n_bins - 1;
			atomicAdd(T.hist + bin, 1u);
		}
	}
	if (P.detected) {
		const uint32_t rslot = warp_reserve(P.n_detected, det);
		if (det) {
			if (rslot < P.det_cap) {
				Record36 rec;
				const Record36* pr = P.primaries + rec_index;
				rec.x = p.pos.x; rec.y = p.pos.y; rec.z = p.pos.z;
				rec.dx = p.dir.x; rec.dy = p.dir.y; rec.dz = p.dir.z; rec.E = p.E;
				rec.px = pr->px; rec.py = pr->py;
				P.detected[rslot] = rec;
				if (BATCH && P.det_job)
					P.det_job[rslot] = (uint8_t)job;
			} else {
				lc.add(CNT_RECORD_OVERFLOW);
			}
		}
	}
}

// One wavefront iteration over the index space
//   [boundary | elastic | inelastic | new secondaries | drained ring | primaries].
// Returns false when there was no work at all (the run is finished); every
// thread of every block sees the same control words and returns the same.
// BATCH: electrons carry their job in the tag's top 8 bits (the low 24 bits
// are the primary's index within its job, which keys its random numbers, as
// in a run of that job alone); geometry, key and yield tallies are per job.
// Energy deposit of one scatter event (energydeposit_cpu_driver.h:44-93):
// a 28-byte record and / or the loss added to its voxel.  Called by the whole
// warp together; `s_loss` is the warp's 32 floats of shared memory.  Lanes
// that hit the same voxel are summed first (one double atomic per voxel).
__device__ __forceinline__ void deposit(const StepParams& P, bool scat, const Electron& p, float e_before,
	const Record36* pr, float* s_loss, LocalCounters& lc)
{
	const uint32_t lane = threadIdx.x & 31u;
	const float loss = scat ? fs(e_before, p.E) : 0.0f;
	if (P.dep) {
		const uint32_t slot = warp_reserve(P.n_dep, scat);
		if (scat) {
			if (slot < P.dep_cap) {
				DepositRecord r;
				r.x = p.pos.x; r.y = p.pos.y; r.z = p.pos.z; r.E = e_before; r.dE = loss;
				r.px = pr->px; r.py = pr->py;
				P.dep[slot] = r;
			} else {
				lc.add(CNT_DEPOSIT_OVERFLOW);
			}
		}
	}
	if (P.grid) {
		int v = -1;
		if (scat) {
			const int i = __float2int_rd(fm(fs(p.pos.x, P.g_org[0]), P.g_inv[0]));
			const int j = __float2int_rd(fm(fs(p.pos.y, P.g_org[1]), P.g_inv[1]));
			const int k = __float2int_rd(fm(fs(p.pos.z, P.g_org[2]), P.g_inv[2]));
			if (i >= 0 && j >= 0 && k >= 0 && i < P.gn[0] && j < P.gn[1] && k < P.gn[2])
				v = (k * P.gn[1] + j) * P.gn[0] + i;
		}
		const unsigned peers = __match_any_sync(0xFFFFFFFFu, v);
		s_loss[lane] = loss;
		__syncwarp();
		if (v >= 0 && (int)lane == __ffs(peers) - 1) {
			double sum = 0.0;
			for (unsigned m = peers; m; m &= m - 1u)
				sum += (double)s_loss[__ffs(m) - 1];
			atomicAdd(P.grid + v, sum);
		}
		__syncwarp();
	}
	if (scat)
		lc.add(CNT_DEPOSITS);
}

template<bool ADJ, bool BATCH, bool DEP = false, uint32_t PHC = 0u>
__device__ __forceinline__ bool step_iteration(const StepParams& P, const BatchParams& B, uint32_t it, LocalCounters& lc,
	const DevMaterial* mats, float* s_lane = nullptr, const DevGeometry* s_geoms = nullptr,
	const DevJob* s_jobs = nullptr)
{
	// physics selection bits: a compile-time constant in the instantiations
	// for the default selection (its option tests fold away, and the code of
	// the unselected inelastic model drops out), the run-time word otherwise
	const uint32_t phys = PHC ? PHC : P.phys;
	const uint32_t rs = it % 3u, ws = (it + 1u) % 3u, zs = (it + 2u) % 3u;
	const uint32_t* cr = P.ctrl + rs * SLOT_WORDS;
	uint32_t* cw = P.ctrl + ws * SLOT_WORDS;
	// counts are clamped to the queue capacity (the secondary budget below
	// keeps them there; the clamp makes an out-of-range read impossible)
	const uint32_t n0 = min(ld_ctrl(cr + 0), P.qcap), n1 = min(ld_ctrl(cr + 1), P.qcap);
	const uint32_t n2 = min(ld_ctrl(cr + 2), P.qcap);
	const uint32_t n3 = min(min(ld_ctrl(cr + EV_NEW), ld_ctrl(cr + SLOT_NEW_BUDGET)), P.qcap);
	const uint32_t n4 = min(ld_ctrl(cr + 4), P.qcap);
	const uint32_t cursor = ld_ctrl(cr + SLOT_CURSOR);
	const uint32_t e1 = n0 + n1, e2 = e1 + n2, e2n = e2 + n3, active = e2n + n4;
	// spill ring: secondaries that found no room earlier, drained (oldest
	// first) ahead of new primaries while the population has room
	const uint32_t sp_head = ld_ctrl(cr + SLOT_SPILL_HEAD);
	const uint32_t sp_tail = ld_ctrl(cr + SLOT_SPILL_TAIL) + ld_ctrl(cr + SLOT_SPILL_PUSHED);
	const uint32_t sp_room = active < P.qcap ? P.qcap - active : 0u;
	const uint32_t n_drain = min(sp_tail - sp_head, sp_room);
	const uint32_t e3 = active + n_drain;
	// no new primaries while secondaries are still parked in the ring, nor
	// while the population is above the refill threshold
	const bool parked = sp_tail - sp_head > n_drain;
	const uint32_t room = (e3 < P.refill_below && !parked) ? P.capacity - min(e3, P.capacity) : 0u;
	// a streamed push: only the primaries whose copy had landed when the
	// previous iteration started (the same snapshot for every thread)
	const uint32_t avail = P.n_avail ? min(ld_ctrl(cr + SLOT_AVAIL), P.n_primaries) : P.n_primaries;
	const uint32_t left = avail > cursor ? avail - cursor : 0u;
	const uint32_t nr = min(min(room, left), P.ramp);
	const uint32_t total = e3 + nr;
	// Secondary budget: every item leaves at most one electron in the next
	// queues plus at most one secondary, so queueing at most qcap - total
	// secondaries keeps the next population, and hence every queue, within
	// qcap.  Secondaries beyond the budget go to the spill ring (the
	// reference instead holds the parent back, PENDING in
	// drivers/gpu/gpu_driver.inl:522-527, which can deadlock a full pool).
	const uint32_t se_budget = P.qcap > total ? P.qcap - total : 0u;
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		cw[SLOT_CURSOR] = cursor + nr;
		cw[SLOT_SPILL_HEAD] = sp_head + n_drain;
		cw[SLOT_SPILL_TAIL] = sp_tail;
		cw[SLOT_NEW_BUDGET] = se_budget;
		if (P.n_avail)
			cw[SLOT_AVAIL] = max(ld_ctrl(P.n_avail), ld_ctrl(cr + SLOT_AVAIL));
		uint32_t* cz = P.ctrl + zs * SLOT_WORDS;
#pragma unroll
		for (int k = 0; k < SLOT_WORDS; ++k)
			cz[k] = 0u;
	}
	// an iteration without work still carries cursor and ring state forward
	// (above), so iterations launched after the end stay empty
	if (total == 0u)
		return false;
	const Queue* qin = P.q[it & 1u];
	const Queue* qout = P.q[(it + 1u) & 1u];

	const uint32_t lane = threadIdx.x & 31u;
	// Warps take 32 items at a time from a counter in the read slot (zeroed
	// two iterations ago, untouched since), so the iteration ends when the
	// work does rather than when the slowest warp's fixed share does.
	uint32_t* const work = P.ctrl + rs * SLOT_WORDS + SLOT_WORK;
	uint32_t base = 0u;
	if (lane == 0u) base = atomicAdd(work, 32u);
	base = __shfl_sync(0xFFFFFFFFu, base, 0);

	for (; base < total; ) {
		const uint32_t item = base + lane;
		// item kinds: the queues EV_BOUNDARY .. EV_WALK, then K_RING (a
		// secondary drained from the spill ring) and K_PRIMARY (a new primary)
		constexpr int K_RING = N_QUEUES, K_PRIMARY = N_QUEUES + 1;
		int kind = -1;
		uint32_t qi = 0;
		if (item < total) {
			if (item < n0) { kind = EV_BOUNDARY; qi = item; }
			else if (item < e1) { kind = EV_ELASTIC; qi = item - n0; }
			else if (item < e2) { kind = EV_INELASTIC; qi = item - e1; }
			else if (item < e2n) { kind = EV_NEW; qi = item - e2; }
			else if (item < active) { kind = EV_WALK; qi = item - e2n; }
			else if (item < e3) { kind = K_RING; qi = (sp_head + (item - active)) & P.spill_mask; }
			else { kind = K_PRIMARY; qi = cursor + (item - e3); }
		}

		Electron p;
		int mat = MAT_VACUUM, last_tri = -1;
		uint32_t tag = 0, event = 0;
		uint64_t lineage = 0;
		float sc[6];
#pragma unroll
		for (int k = 0; k < 6; ++k) sc[k] = 0.0f;
		FlightResume fr;
		if (kind == K_RING || (kind >= 0 && kind < N_QUEUES)) {
			const Queue& q = kind == K_RING ? P.spill : qin[kind];
			const float4 a = ld_stream(q.a + qi), b = ld_stream(q.b + qi);
			const uint4 c = ld_stream(q.c + qi);
			p.pos = v3(a.x, a.y, a.z); p.E = a.w;
			p.dir = v3(b.x, b.y, b.z); mat = __float_as_int(b.w);
			last_tri = (int)c.x; tag = c.y; event = c.z;
			lineage = ((uint64_t)ld_stream(q.d + qi) << 32) | c.w;
			if (ADJ) {
				const float4 s = ld_stream(q.s + qi);
				const float2 s2 = ld_stream(q.s2 + qi);
				sc[0] = s.x; sc[1] = s.y; sc[2] = s.z; sc[3] = s.w; sc[4] = s2.x; sc[5] = s2.y;
			}
		} else if (kind == K_PRIMARY) {
			const Record36* r = P.primaries + qi;
			p.pos = v3(ld_stream(&r->x), ld_stream(&r->y), ld_stream(&r->z));
			p.dir = v3(ld_stream(&r->dx), ld_stream(&r->dy), ld_stream(&r->dz));
			p.E = ld_stream(&r->E);
			if (BATCH) {
				const uint32_t j = job_of(s_jobs, B.n_jobs, qi);
				tag = (j << 24) | (qi - s_jobs[j].first);
			} else {
				tag = P.tag_base + qi;
			}
			lc.add(CNT_PRIMARIES);
		}
		const float e_before = p.E;
		// run context: job geometry / key, the primary's record, the tag that
		// keys the random numbers
		RunView rv;
		uint32_t job = 0, stream_tag = tag, rec_index = BATCH ? tag : tag - P.tag_base;
		if (BATCH) {
			job = tag >> 24;
			stream_tag = tag & 0xFFFFFFu;
			const DevJob& J = s_jobs[kind >= 0 ? job : 0u];
			rv.geom = s_geoms + J.geom;
			rv.key = J.key;
			rec_index = J.first + stream_tag;
		} else {
			rv.geom = &P.geom;
			rv.key = P.key;
		}

		// adjoint replay with wstep > 0: this primary's cascade runs with the
		// work functions shifted by wstep * r_m (the same random numbers as the
		// forward run otherwise); the work-function derivative is then the
		// difference of the signed tallies of the two runs, and the
		// transmission score is not accumulated
		float dbar[2] = { 0.0f, 0.0f };
		const bool wshift = ADJ && P.wstep > 0.0f;
		if (wshift) {
			dbar[0] = fm(P.wstep, wsign(rv.key, stream_tag, 0));
			dbar[1] = fm(P.wstep, wsign(rv.key, stream_tag, 1));
		}

		// interaction that ended the previous flight
		int status = (kind >= 0) ? ST_RUNNING : ST_TERMINATED;
		bool spawn = false;
		Electron se;
		if (kind == EV_BOUNDARY) {
			lc.add(CNT_BOUNDARY);
			PhiloxStream r;
			r.init(rv.key, event, 1u, stream_tag, lineage);
			const DevTriangle T = load_tri(rv.geom->tris, last_tri);
			if (ADJ) {
				BoundaryScore bs = { 0.0f, 0.0f, -1, -1 };
				status = boundary_event(T, mats, p, mat, r, &bs, phys, wshift ? dbar : nullptr);
				// the work function enters through barrier = fermi + W of the
				// materials on either side of the crossing
				if (!wshift) {
					if (bs.mat_in >= 0 && bs.mat_in < 2) sc[3 * bs.mat_in + 2] += bs.d_in;
					if (bs.mat_out >= 0 && bs.mat_out < 2) sc[3 * bs.mat_out + 2] += bs.d_out;
				}
			} else {
				status = boundary_event(T, mats, p, mat, r, nullptr, phys);
			}
		} else if (kind == EV_ELASTIC) {
			lc.add(CNT_ELASTIC);
			last_tri = -1;
			PhiloxStream r;
			r.init(rv.key, event, 1u, stream_tag, lineage);
			elastic_event(mats[mat], p, r, phys);
		} else if (kind == EV_INELASTIC) {
			lc.add(CNT_INELASTIC);
			last_tri = -1;
			PhiloxStream r;
			r.init(rv.key, event, 1u, stream_tag, lineage);
			spawn = inelastic_event(mats[mat], p, se, r, phys);
		}

		// energy deposit of a scatter event that changed the energy
		if (DEP)
			deposit(P, (kind == EV_ELASTIC || kind == EV_INELASTIC) && p.E != e_before, p, e_before,
				P.primaries + rec_index, s_lane + (threadIdx.x & ~31u), lc);

		// detection output: record + tallies (out of line: a warp has a
		// detection in a small fraction of its chunks)
		if (__any_sync(0xFFFFFFFFu, status == ST_DETECTED)) {
			Scores scs;
#pragma unroll
			for (int k = 0; k < 6; ++k) scs.v[k] = ADJ ? sc[k] : 0.0f;
			detection_output<ADJ, BATCH>(&P, BATCH ? &B : nullptr, status == ST_DETECTED, p, rec_index, job, rv.key,
				stream_tag, scs, wshift, lc.c);
		}

		// secondary: inherits material, tag and the parent's scores; its
		// lineage id is derived from the parent's and the spawning event
		uint64_t se_lineage = 0;
		if (spawn) {
			lc.add(CNT_SPAWNED);
			se_lineage = child_lineage(lineage, event);
			// A secondary below its material's escape threshold ends at its
			// first free flight (energy cut, before any random draw or
			// event): count that flight and termination here instead of
			// queueing it.  Counter-based random numbers make this change
			// nothing for any other electron.
			const float barrier = (wshift && mat < 2) ? fa(mats[mat].barrier, dbar[mat]) : mats[mat].barrier;
			if (se.E < fa(barrier, P.energy_threshold)) {
				spawn = false;
				lc.add(CNT_FLIGHTS);
				lc.add(CNT_TERMINATED);
			}
		}
		// The flight queue's counter hands out the tickets: the first
		// se_budget secondaries are queued, later ones go to the spill ring
		// (their slots stay unwritten; the next iteration reads at most
		// se_budget entries).
		const uint32_t sslot = warp_reserve(cw + EV_NEW, spawn);
		const bool queued = spawn && sslot < se_budget;
		const bool spilled = spawn && !queued;
		const uint32_t pslot = warp_reserve(cw + SLOT_SPILL_PUSHED, spilled);
		if (queued || spilled) {
			const Queue* dst = nullptr;
			uint32_t at = 0;
			if (queued) {
				if (sslot < P.qcap) { dst = &qout[EV_NEW]; at = sslot; }
				else lc.add(CNT_QUEUE_OVERFLOW);
			} else {
				lc.add(CNT_SPILLED);
				// the ring holds at most spill_mask + 1 electrons, counting the
				// ones being drained during this iteration
				if (sp_tail + pslot - sp_head <= P.spill_mask) { dst = &P.spill; at = (sp_tail + pslot) & P.spill_mask; }
				else lc.add(CNT_QUEUE_OVERFLOW);
			}
			if (dst) {
				store_electron(*dst, at, se, mat, -1, tag, 0u, se_lineage);
				if (ADJ) {
					st_stream(dst->s + at, make_float4(sc[0], sc[1], sc[2], sc[3]));
					st_stream(dst->s2 + at, make_float2(sc[4], sc[5]));
				}
			}
		}

		// next free flight (or the rest of a walk cut short last iteration)
		int qtype = -1;
		if (status == ST_RUNNING)
			qtype = free_flight<ADJ>(P, rv, p, mat, last_tri, event, stream_tag, lineage, sc, lc,
				wshift ? dbar : nullptr, fr, kind == EV_WALK ? &qin[EV_WALK] : nullptr, qi, mats);
		if (kind >= 0 && status != ST_DETECTED && qtype < 0)
			lc.add(CNT_TERMINATED);
		{
			// the warp's next chunk is claimed (lane 5) together with the
			// queue slots (lanes 0-4): one atomic round trip for both
			uint32_t next = 0u;
			if (lane == 5u)
				next = atomicAdd(work, 32u);
			const uint32_t slot = warp_reserve5(cw, qtype);
			if (qtype >= 0 && slot >= P.qcap)
				lc.add(CNT_QUEUE_OVERFLOW);
			// compile-time queue indices (a run-time index into the kernel
			// parameters would copy them to local memory)
#pragma unroll
			for (int t = 0; t < N_QUEUES; ++t) {
				if (qtype == t && slot < P.qcap) {
					store_electron(qout[t], slot, p, mat, last_tri, tag, event, lineage);
					if (ADJ) {
						st_stream(qout[t].s + slot, make_float4(sc[0], sc[1], sc[2], sc[3]));
						st_stream(qout[t].s2 + slot, make_float2(sc[4], sc[5]));
					}
					if (t == EV_WALK)
						store_resume(qout[t], slot, fr);
				}
			}
			base = __shfl_sync(0xFFFFFFFFu, next, 5);
		}
	}
	return true;
}

// The material descriptors (table pointers, sizes and axis scales, and the
// constants), which every table lookup reads on the event's chain of
// dependent loads, copied into the block's dynamic shared memory
// (n_mat x 320 bytes, sized by the launch) for the batched kernel's whole
// launch: shared loads are the shorter ones.  The caller synchronises the
// block before use.
__device__ __forceinline__ const DevMaterial* stage_materials(const StepParams& P)
{
	extern __shared__ __align__(16) unsigned char s_dynamic[];
	DevMaterial* s_mats = reinterpret_cast<DevMaterial*>(s_dynamic);
	for (int k = threadIdx.x; k < P.n_mat; k += blockDim.x)
		s_mats[k] = P.mats[k];
	return s_mats;
}

// dynamic shared memory of a batched launch: the staged materials
// (127 materials at most: 40.6 KB)
static size_t batch_shared_bytes(const StepParams& p)
{
	return (size_t)p.n_mat * sizeof(DevMaterial);
}

// lets a kernel take that much dynamic shared memory next to its static
// arrays (above 48 KB per block the limit is raised explicitly)
static void allow_shared_bytes(const void* kernel, size_t bytes)
{
	if (bytes > 0 && cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
		cudaGetLastError();
}

__device__ __forceinline__ void flush_counters(const StepParams& P, uint32_t* s_counters)
{
	__syncthreads();
	for (int k = threadIdx.x; k < N_COUNTERS; k += blockDim.x)
		if (s_counters[k])
			atomicAdd(P.counters + k, (unsigned long long)s_counters[k]);
}

// One wavefront iteration per launch (the plain method).  Four resident
// blocks of 256 threads per SM (at most 64 registers): the kernel is latency
// bound, so warps in flight matter more than registers.
// DEP: energy deposits on (a separate instantiation, so the plain step keeps
// none of their code).  PHC: nonzero = the physics selection fixed at
// compile time (PH_DEFAULT only).
template<bool ADJ, bool DEP, uint32_t PHC = 0u>
__global__ void __launch_bounds__(256, NBL_STEP_MIN_BLOCKS) k_step(const __grid_constant__ StepParams P, uint32_t it)
{
	__shared__ uint32_t s_counters[N_COUNTERS];
	__shared__ float s_lane[DEP ? 256 : 1];
	for (int k = threadIdx.x; k < N_COUNTERS; k += blockDim.x)
		s_counters[k] = 0u;
	__syncthreads();
	LocalCounters lc{ s_counters };
	const BatchParams none{};
	// materials read from global memory: staged in shared memory as the
	// batched kernel stages them, this kernel measured slower (-0.4 % on the
	// grating scan, -1.5 % on the 1.2 M-triangle mesh)
	step_iteration<ADJ, false, DEP, PHC>(P, none, it, lc, P.mats, s_lane);
	flush_counters(P, s_counters);
}

// Grid-wide barrier of the persistent kernel (all blocks co-resident by the
// cooperative launch).  Arrival counter + generation word; waiting is bounded
// (2^22 polls, a few seconds; one iteration takes milliseconds); on timeout,
// or if any block already timed out, it records the error and returns false
// so every block leaves.
__device__ __forceinline__ bool grid_barrier(const BatchParams& B)
{
	__shared__ int s_ok;
	__syncthreads();
	if (threadIdx.x == 0) {
		const unsigned gen0 = atomicAdd(B.bar_gen, 0u);
		__threadfence();
		const unsigned arrived = atomicAdd(B.bar_count, 1u) + 1u;
		int ok = 1;
		if (arrived == gridDim.x) {
			atomicExch(B.bar_count, 0u);
			__threadfence();
			atomicAdd(B.bar_gen, 1u);
		} else {
			unsigned polls = 0;
			while (atomicAdd(B.bar_gen, 0u) == gen0) {
				if (atomicAdd(B.err, 0u)) { ok = 0; break; }
				__nanosleep(64);
				if (++polls > (1u << 22)) { atomicOr(B.err, 1u); ok = 0; break; }
			}
		}
		__threadfence();
		s_ok = ok && atomicAdd(B.err, 0u) == 0u;
	}
	__syncthreads();
	return s_ok != 0;
}

// The batched method: one persistent launch runs every iteration of a whole
// batch of jobs, with a grid barrier between iterations instead of a kernel
// boundary; it ends when an iteration finds no work (all blocks see the same
// control words) or after max_iterations (error word set).
template<bool ADJ, uint32_t PHC = 0u>
__global__ void __launch_bounds__(512, 2) k_batch(const __grid_constant__ StepParams P,
	const __grid_constant__ BatchParams B)
{
	__shared__ uint32_t s_counters[N_COUNTERS];
	// the geometry and job tables every item looks up, staged in shared
	// memory for the whole launch: the walk reads the geometry's fields on
	// its chain of dependent loads, and shared loads are the shorter ones
	__shared__ DevGeometry s_geoms[NBL_BATCH_MAX_GEOMS];
	__shared__ DevJob s_jobs[NBL_BATCH_MAX_JOBS];
	for (int k = threadIdx.x; k < N_COUNTERS; k += blockDim.x)
		s_counters[k] = 0u;
	for (int k = threadIdx.x; k < B.n_geoms; k += blockDim.x)
		s_geoms[k] = B.geoms[k];
	for (int k = threadIdx.x; k < B.n_jobs; k += blockDim.x)
		s_jobs[k] = B.jobs[k];
	const DevMaterial* s_mats = stage_materials(P);
	__syncthreads();
	LocalCounters lc{ s_counters };
	uint32_t it = 0;
	for (; it < B.max_iterations; ++it) {
		if (!step_iteration<ADJ, true, false, PHC>(P, B, it, lc, s_mats, nullptr, s_geoms, s_jobs))
			break;
		if (!grid_barrier(B))
			break;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		*B.iterations = it;
		if (it >= B.max_iterations)
			atomicOr(B.err, 2u);
	}
	flush_counters(P, s_counters);
}

// The step kernel instantiation a run's parameters select: adjoint or not,
// deposits or not, the default physics selection fixed at compile time or the
// run-time word.
static const void* step_kernel(const StepParams& p)
{
	const bool dep = p.dep || p.grid;
	const bool fixed = p.phys == PH_DEFAULT;
	if (p.adjoint) {
		if (dep) return (const void*)k_step<true, true>;
		if (fixed) return (const void*)k_step<true, false, PH_DEFAULT>;
		return (const void*)k_step<true, false>;
	}
	if (dep) return (const void*)k_step<false, true>;
	if (fixed) return (const void*)k_step<false, false, PH_DEFAULT>;
	return (const void*)k_step<false, false>;
}

cudaError_t launch_step(const StepParams& p, uint32_t iteration, int grid, int block, cudaStream_t s)
{
	void* args[] = { const_cast<StepParams*>(&p), &iteration };
	return cudaLaunchKernel(step_kernel(p), dim3(grid), dim3(block), args, 0, s);
}

int step_grid_size(int device, int block, const StepParams& p)
{
	int sms = 148, per_sm = 1;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	// occupancy of the instantiation these parameters launch
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel(p), block, 0);
	if (per_sm < 1)
		per_sm = 1;
	return sms * per_sm;
}

cudaError_t step_binary_version(int device, int* version)
{
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess)
		return e;
	cudaFuncAttributes a{};
	e = cudaFuncGetAttributes(&a, k_step<false, false, PH_DEFAULT>);
	*version = a.binaryVersion;
	return e;
}

int batch_grid_size(int device, int block, const StepParams& p)
{
	int sms = 148, per_sm = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	// the cooperative grid must be co-resident for whichever instantiation runs
	// (batches run without the adjoint: the host never sets it for them)
	const void* kernels[] = { (const void*)k_batch<false>, (const void*)k_batch<false, PH_DEFAULT> };
	for (const void* k : kernels) {
		int n = 0;
		allow_shared_bytes(k, batch_shared_bytes(p));
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, batch_shared_bytes(p));
		per_sm = per_sm == 0 ? n : std::min(per_sm, n);
	}
	return sms * per_sm;
}

cudaError_t launch_batch(const StepParams& p, const BatchParams& b, int grid, int block, cudaStream_t s)
{
	void* args[] = { const_cast<StepParams*>(&p), const_cast<BatchParams*>(&b) };
	if (p.adjoint)
		return cudaErrorInvalidValue;           // no batched adjoint
	const void* k = p.phys == PH_DEFAULT ? (const void*)k_batch<false, PH_DEFAULT> : (const void*)k_batch<false>;
	return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(block), args, batch_shared_bytes(p), s);
}

}  // namespace nbl
