// Transport run that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host that hands the library a fixed
// device-memory budget up front (an embedding framework whose allocator owns
// the whole device), a real-time acquisition loop where an allocation could
// block or fail in the middle of a scan, or code that must not touch the
// driver's allocator for any other reason.  nbl_run_noalloc serves them: it
// runs the same wavefront transport kernel as nbl_sim_run, but keeps all of
// its scratch memory -- event queues, overflow ring, control words, counters,
// and the device copies of geometry and material tables -- in one
// file-scope __device__ array of fixed size, NBL_NOALLOC_SCRATCH_BYTES, that
// every GPU which loads the library holds until the process exits.  The
// caller provides the primaries and every output buffer in device memory.
//
// Limits (rejected with NBL_ERR_INVALID_ARG beyond them): capacity at most
// NBL_NOALLOC_MAX_CAPACITY electrons, at most NBL_NOALLOC_MAX_MATERIALS
// materials, geometry and tables within the byte budgets below, no adjoint,
// no energy deposits.  The first call on a device looks the array's device
// address up (cudaGetSymbolAddress) and keeps it for the life of the process,
// so make that first call before any stream capture, and make no call on a
// device after the caller has reset it (cudaDeviceReset): the kept address
// belongs to the context that the reset destroyed.  Under CUDA's default lazy
// module loading the array is reserved when the library's kernels are first
// used on a device, not when the library is loaded: a caller that hands the
// device to its own allocator afterwards should make one call first (or load
// modules eagerly, CUDA_MODULE_LOADING=EAGER).  A call waits on its stream:
// it reads the run's progress from the device between rounds of iterations
// and returns when the run is complete.  All calls share the one array and it
// keeps the previous call's contents: each call clears the parts that must
// start at zero, and two calls whose work overlaps on the GPU (different
// streams, different threads) race on it.
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include <string>
#include <algorithm>

#include "kernels.cuh"
#include "host/internal.hpp"

namespace nbl {
namespace {

constexpr uint32_t NA_CAPACITY = NBL_NOALLOC_MAX_CAPACITY;
constexpr uint32_t NA_QCAP = 8 * NA_CAPACITY;                  // population bound
constexpr uint32_t NA_RING = 16 * NA_CAPACITY;                 // overflow ring (power of two)
constexpr size_t NA_GEOM_BYTES = (size_t)2 << 20;               // octree + triangles
constexpr size_t NA_TABLE_BYTES = (size_t)4 << 20;              // all material tables
constexpr size_t ALIGN = 256;

constexpr size_t align_up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }
constexpr size_t QUEUE_BYTES(uint32_t n) { return align_up((size_t)n * 16) * 3 + align_up((size_t)n * 4); }
constexpr size_t OFF_CTRL = 0;
constexpr size_t OFF_COUNTERS = align_up(OFF_CTRL + 3 * SLOT_WORDS * sizeof(uint32_t));
constexpr size_t OFF_NDET = align_up(OFF_COUNTERS + N_COUNTERS * sizeof(unsigned long long));
constexpr size_t OFF_MATS = align_up(OFF_NDET + sizeof(uint32_t));
constexpr size_t OFF_GEOM = align_up(OFF_MATS + NBL_NOALLOC_MAX_MATERIALS * sizeof(DevMaterial));
constexpr size_t OFF_TABLES = OFF_GEOM + NA_GEOM_BYTES;
constexpr size_t OFF_QUEUES = OFF_TABLES + NA_TABLE_BYTES;
// the event, flight and walk-continuation queues; the last also carries the
// walk state of a flight that continues (two more 16-byte words per entry)
constexpr size_t WALK_BYTES(uint32_t n) { return 2 * align_up((size_t)n * 16); }
constexpr size_t OFF_WALK = OFF_QUEUES + 2 * N_QUEUES * QUEUE_BYTES(NA_QCAP);
constexpr size_t OFF_SPILL = OFF_WALK + 2 * WALK_BYTES(NA_QCAP);
constexpr size_t SCRATCH_BYTES = OFF_SPILL + QUEUE_BYTES(NA_RING);
static_assert(SCRATCH_BYTES == NBL_NOALLOC_SCRATCH_BYTES, "NBL_NOALLOC_SCRATCH_BYTES out of date");
static_assert((NA_RING & (NA_RING - 1)) == 0, "ring size must be a power of two");

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

// Device address of the scratch array, looked up once per device.
constexpr int MAX_DEVICES = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[MAX_DEVICES] = {};

unsigned char* scratch_address(int device)
{
	require(device >= 0 && device < MAX_DEVICES, "device ordinal out of range");
	std::lock_guard<std::mutex> lock(g_scratch_mu);
	if (!g_scratch_addr[device]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess)
			throw Error(NBL_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
		g_scratch_addr[device] = p;
	}
	return static_cast<unsigned char*>(g_scratch_addr[device]);
}

Queue carve_queue(unsigned char* base, uint32_t n)
{
	Queue q;
	q.a = reinterpret_cast<float4*>(base);
	q.b = reinterpret_cast<float4*>(base + align_up((size_t)n * 16));
	q.c = reinterpret_cast<uint4*>(base + 2 * align_up((size_t)n * 16));
	q.d = reinterpret_cast<uint32_t*>(base + 3 * align_up((size_t)n * 16));
	q.s = nullptr;
	q.s2 = nullptr;
	q.w0 = nullptr;
	q.w1 = nullptr;
	return q;
}

void cuda_ok(cudaError_t e, const char* what)
{
	if (e != cudaSuccess)
		throw Error(NBL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace nbl

using namespace nbl;

extern "C" nbl_status nbl_run_noalloc(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials,
	const nbl_params* params, const nbl_record* d_primaries, int64_t n_primaries, nbl_record* d_records,
	int64_t records_cap, int64_t* n_records, uint32_t* d_se_img, uint32_t* d_bse_img, uint32_t* d_hist,
	nbl_counters* counters)
{
	return guard([&] {
		require(g && materials && params && n_records, "null argument");
		require(n_primaries >= 0 && n_primaries < 0xFFFFFFFFll, "primaries count out of range");
		require(n_primaries == 0 || d_primaries, "null primaries");
		require(records_cap >= 0 && records_cap <= 0xFFFFFFFFll && (records_cap == 0 || d_records), "bad record buffer");
		require(n_materials >= 1 && n_materials <= NBL_NOALLOC_MAX_MATERIALS,
			"nbl_run_noalloc: at most " + std::to_string(NBL_NOALLOC_MAX_MATERIALS) + " materials");
		require(params->adjoint == 0, "nbl_run_noalloc: the adjoint is not available without allocation");
		require(params->walk_cells <= (1u << 20), "walk_cells must be at most 2^20");
		const nbl_deposit_grid& dgp = params->deposit_grid;
		require(params->deposit_capacity == 0 && dgp.n[0] == 0 && dgp.n[1] == 0 && dgp.n[2] == 0,
			"nbl_run_noalloc: energy deposits are not available without allocation");
		const nbl_image_filter& flt = params->image_filter;
		require(!flt.enabled || (flt.cos_min <= flt.cos_max && flt.cos_min >= -1.0f && flt.cos_max <= 1.0f),
			"image filter needs -1 <= cos_min <= cos_max <= 1");
		const uint32_t phys = physics_bits(params->physics);
		const bool kieft = (phys & PH_KIEFT) != 0;
		const uint32_t cap = params->capacity ? params->capacity : NA_CAPACITY;
		require(cap >= 32 && cap <= NA_CAPACITY, "nbl_run_noalloc: capacity must be 32.." + std::to_string(NA_CAPACITY));
		int max_mat = -1;
		for (const nbl_triangle& t : g->g.tris)
			max_mat = std::max(max_mat, std::max(t.material_in, t.material_out));
		require(max_mat < n_materials, "geometry uses more materials than given");
		const HostGeometry& hg = g->g;
		const size_t oct_bytes = align_up(hg.octree.size() * sizeof(int32_t));
		require(oct_bytes + hg.tris.size() * sizeof(DevTriangle) <= NA_GEOM_BYTES,
			"nbl_run_noalloc: geometry exceeds its " + std::to_string(NA_GEOM_BYTES >> 20) + " MiB budget");
		size_t table_bytes = 0;
		for (int i = 0; i < n_materials; ++i) {
			require(materials[i] != nullptr, "null material");
			const HostMaterial& m = materials[i]->m;
			const InelasticTables it = inelastic_tables(m, kieft);
			for (const HostTable* t : { &m.el_imfp, &m.el_icdf, it.imfp, it.omega, it.q, it.binding })
				table_bytes += align_up(t->data.size() * sizeof(float));
		}
		require(table_bytes <= NA_TABLE_BYTES,
			"nbl_run_noalloc: material tables exceed their " + std::to_string(NA_TABLE_BYTES >> 20) + " MiB budget");
		const int32_t nx = params->tally_nx, ny = params->tally_ny;
		require(nx >= 0 && ny >= 0, "bad tally grid");
		const bool tally = nx > 0 && ny > 0;
		require(!tally || (d_se_img && d_bse_img), "tally grid given without image buffers");
		const int32_t n_bins = params->hist_bins > 0 ? params->hist_bins : 200;

		int n_dev = 0;
		if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
			throw Error(NBL_ERR_NO_DEVICE, "no CUDA device available");
		require(params->device >= 0 && params->device < n_dev, "device ordinal out of range");
		cuda_ok(cudaSetDevice(params->device), "cudaSetDevice");
		unsigned char* base = scratch_address(params->device);
		cudaStream_t s = static_cast<cudaStream_t>(params->stream);

		// device copies of the geometry (64-byte triangles with normals) and tables
		unsigned char* geom = base + OFF_GEOM;
		cuda_ok(cudaMemcpyAsync(geom, hg.octree.data(), hg.octree.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s),
			"copy octree");
		DevTriangle chunk[256];
		for (size_t i = 0; i < hg.tris.size(); i += 256) {
			const size_t k = std::min<size_t>(256, hg.tris.size() - i);
			for (size_t j = 0; j < k; ++j) {
				const nbl_triangle& t = hg.tris[i + j];
				DevTriangle& d = chunk[j];
				d.r0x = t.r0[0]; d.r0y = t.r0[1]; d.r0z = t.r0[2]; d.mat_in = t.material_in;
				d.e1x = t.e1[0]; d.e1y = t.e1[1]; d.e1z = t.e1[2]; d.mat_out = t.material_out;
				d.e2x = t.e2[0]; d.e2y = t.e2[1]; d.e2z = t.e2[2]; d.pad0 = 0;
				d.nx = t.e1[1] * t.e2[2] - t.e1[2] * t.e2[1];
				d.ny = t.e1[2] * t.e2[0] - t.e1[0] * t.e2[2];
				d.nz = t.e1[0] * t.e2[1] - t.e1[1] * t.e2[0];
				d.pad1 = 0;
			}
			cuda_ok(cudaMemcpyAsync(geom + oct_bytes + i * sizeof(DevTriangle), chunk, k * sizeof(DevTriangle),
				cudaMemcpyHostToDevice, s), "copy triangles");
			cuda_ok(cudaStreamSynchronize(s), "copy triangles");
		}
		DevMaterial dm[NBL_NOALLOC_MAX_MATERIALS];
		unsigned char* tab = base + OFF_TABLES;
		size_t toff = 0;
		for (int i = 0; i < n_materials; ++i) {
			const HostMaterial& m = materials[i]->m;
			auto put = [&](const HostTable& t) {
				DevTable d;
				d.data = reinterpret_cast<const float*>(tab + toff);
				d.nx = t.nx; d.ny = t.ny; d.nz = t.nz; d.pad = 0;
				d.x_min = t.x_min; d.x_step = t.x_step; d.y_min = t.y_min; d.y_step = t.y_step;
				d.z_min = t.z_min; d.z_step = t.z_step;
				cuda_ok(cudaMemcpyAsync(tab + toff, t.data.data(), t.data.size() * sizeof(float), cudaMemcpyHostToDevice, s),
					"copy table");
				toff += align_up(t.data.size() * sizeof(float));
				return d;
			};
			DevMaterial& d = dm[i];
			const InelasticTables it = inelastic_tables(m, kieft);
			d.el_imfp = put(m.el_imfp); d.el_icdf = put(m.el_icdf); d.in_imfp = put(*it.imfp);
			d.in_omega = put(*it.omega); d.in_q = put(*it.q); d.in_binding = put(*it.binding);
			d.fermi = m.fermi; d.band_gap = m.band_gap; d.barrier = m.barrier;
			d.phonon_loss = m.phonon_loss; d.recoil_const = m.recoil_const;
			d.in_scale = 1.0f; d.el_scale = 1.0f; d.pad = 0;
		}
		cuda_ok(cudaMemcpyAsync(base + OFF_MATS, dm, n_materials * sizeof(DevMaterial), cudaMemcpyHostToDevice, s),
			"copy materials");

		// the state every run must start from: control words, counters,
		// record count and the caller's tallies at zero
		cuda_ok(cudaMemsetAsync(base + OFF_CTRL, 0, OFF_MATS - OFF_CTRL, s), "clear control words");
		if (tally) {
			cuda_ok(cudaMemsetAsync(d_se_img, 0, (size_t)nx * ny * sizeof(uint32_t), s), "clear tallies");
			cuda_ok(cudaMemsetAsync(d_bse_img, 0, (size_t)nx * ny * sizeof(uint32_t), s), "clear tallies");
		}
		if (d_hist)
			cuda_ok(cudaMemsetAsync(d_hist, 0, (size_t)n_bins * sizeof(uint32_t), s), "clear histogram");

		StepParams sp{};
		sp.geom.octree = reinterpret_cast<const int32_t*>(geom);
		sp.geom.tris = reinterpret_cast<const DevTriangle*>(geom + oct_bytes);
		sp.geom.cx = hg.center[0]; sp.geom.cy = hg.center[1]; sp.geom.cz = hg.center[2];
		sp.geom.hx = hg.halfsize[0]; sp.geom.hy = hg.halfsize[1]; sp.geom.hz = hg.halfsize[2];
		sp.geom.max_extent = hg.max_extent;
		sp.geom.n_tri = (int32_t)hg.tris.size();
		sp.geom.n_octree = (int64_t)hg.octree.size();
		sp.mats = reinterpret_cast<const DevMaterial*>(base + OFF_MATS);
		sp.n_mat = n_materials;
		sp.energy_threshold = params->energy_threshold;
		sp.key.k0 = (uint32_t)params->seed;
		sp.key.k1 = (uint32_t)(params->seed >> 32);
		unsigned char* qb = base + OFF_QUEUES;
		for (int b = 0; b < 2; ++b)
			for (int q = 0; q < N_QUEUES; ++q, qb += QUEUE_BYTES(NA_QCAP))
				sp.q[b][q] = carve_queue(qb, NA_QCAP);
		for (int b = 0; b < 2; ++b) {
			unsigned char* wb = base + OFF_WALK + b * WALK_BYTES(NA_QCAP);
			sp.q[b][EV_WALK].w0 = reinterpret_cast<float4*>(wb);
			sp.q[b][EV_WALK].w1 = reinterpret_cast<uint4*>(wb + align_up((size_t)NA_QCAP * 16));
		}
		sp.qcap = 8 * cap;
		sp.capacity = cap;
		sp.ramp = std::max<uint32_t>(cap / 16, 256);
		sp.refill_below = cap;
		sp.phys = phys;
		sp.spill = carve_queue(base + OFF_SPILL, NA_RING);
		sp.spill_mask = NA_RING - 1;
		sp.ctrl = reinterpret_cast<uint32_t*>(base + OFF_CTRL);
		sp.primaries = reinterpret_cast<const Record36*>(d_primaries);
		sp.n_primaries = (uint32_t)n_primaries;
		sp.detected = reinterpret_cast<Record36*>(d_records);
		sp.n_detected = reinterpret_cast<uint32_t*>(base + OFF_NDET);
		sp.det_cap = (uint32_t)records_cap;
		sp.tal.se_img = tally ? d_se_img : nullptr;
		sp.tal.bse_img = tally ? d_bse_img : nullptr;
		sp.tal.hist = d_hist;
		sp.tal.grad_se = sp.tal.grad_bse = nullptr;
		sp.tal.nx = nx; sp.tal.ny = ny;
		sp.tal.n_bins = n_bins;
		sp.tal.hist_emax = params->hist_emax > 0 ? params->hist_emax : 1000.0f;
		// detector acceptance of the images, as nbl_sim_create applies it
		sp.tal.filter = flt.enabled ? 1 : 0;
		sp.tal.cos_min = flt.enabled ? flt.cos_min : 0.0f;
		sp.tal.cos_max = flt.enabled ? flt.cos_max : 0.0f;
		sp.counters = reinterpret_cast<unsigned long long*>(base + OFF_COUNTERS);
		sp.max_events = params->max_events ? params->max_events : (1u << 22);
		require(sp.max_events < (1u << 24), "max_events must be < 2^24");
		sp.adjoint = 0;

		const int block = params->block_size ? (int)params->block_size : 256;
		require(block % 32 == 0 && block >= 32 && block <= 256, "block_size must be a multiple of 32 in 32..256");
		sp.walk_cells = params->walk_cells ? params->walk_cells : 1u;
		const int grid = params->grid_size ? (int)params->grid_size : step_grid_size(params->device, block, sp);
		const uint32_t check_every = 24;
		const uint64_t bound = ((uint64_t)sp.max_events + 1) * 64 + (uint64_t)n_primaries + 64;
		uint32_t ctrl[SLOT_WORDS];
		unsigned long long flights = 0, last_flights = ~0ull;
		int stalled = 0;
		bool done = false;
		uint64_t it = 0;
		for (; it < bound && !done; ) {
			for (uint32_t k = 0; k < check_every; ++k, ++it)
				cuda_ok(launch_step(sp, (uint32_t)(it % 6), grid, block, s), "transport launch");
			const uint32_t slot = (uint32_t)(it % 3);
			cuda_ok(cudaMemcpyAsync(ctrl, sp.ctrl + slot * SLOT_WORDS, sizeof(ctrl), cudaMemcpyDeviceToHost, s), "read state");
			cuda_ok(cudaMemcpyAsync(&flights, sp.counters + CNT_FLIGHTS, sizeof(flights), cudaMemcpyDeviceToHost, s),
				"read state");
			cuda_ok(cudaStreamSynchronize(s), "transport");
			uint64_t active = (uint32_t)(ctrl[SLOT_SPILL_TAIL] + ctrl[SLOT_SPILL_PUSHED] - ctrl[SLOT_SPILL_HEAD]);
			for (int q = 0; q < N_QUEUES; ++q)
				active += q == EV_NEW ? std::min(ctrl[q], ctrl[SLOT_NEW_BUDGET]) : ctrl[q];
			done = active == 0 && ctrl[SLOT_CURSOR] == (uint32_t)n_primaries;
			if (!done) {
				stalled = flights == last_flights ? stalled + 1 : 0;
				if (stalled >= 2)
					throw Error(NBL_ERR_POOL_OVERFLOW, "no electron moved for two rounds of iterations");
				last_flights = flights;
			}
		}
		if (!done)
			throw Error(NBL_ERR_BUDGET_EXCEEDED, "run did not finish within its iteration bound");

		unsigned long long c[N_COUNTERS];
		uint32_t ndet = 0;
		cuda_ok(cudaMemcpyAsync(c, sp.counters, sizeof(c), cudaMemcpyDeviceToHost, s), "read counters");
		cuda_ok(cudaMemcpyAsync(&ndet, sp.n_detected, sizeof(ndet), cudaMemcpyDeviceToHost, s), "read counters");
		cuda_ok(cudaStreamSynchronize(s), "read counters");
		*n_records = std::min<int64_t>(ndet, records_cap);
		if (counters) {
			std::memset(counters, 0, sizeof(*counters));
			counters->flights = c[CNT_FLIGHTS]; counters->boundary = c[CNT_BOUNDARY]; counters->elastic = c[CNT_ELASTIC];
			counters->inelastic = c[CNT_INELASTIC]; counters->spawned = c[CNT_SPAWNED]; counters->detected = c[CNT_DETECTED];
			counters->terminated = c[CNT_TERMINATED]; counters->primaries_started = c[CNT_PRIMARIES];
			counters->walk_overflow = c[CNT_WALK_OVERFLOW]; counters->nan_state = c[CNT_NAN];
			counters->queue_overflow = c[CNT_QUEUE_OVERFLOW]; counters->record_overflow = c[CNT_RECORD_OVERFLOW];
			counters->event_budget = c[CNT_EVENT_BUDGET]; counters->spilled = c[CNT_SPILLED];
			counters->primaries_total = (uint64_t)n_primaries;
			counters->iterations = it;
			counters->records_pending = *n_records;
		}
		if (c[CNT_QUEUE_OVERFLOW] || c[CNT_RECORD_OVERFLOW] || ndet > records_cap)
			throw Error(NBL_ERR_POOL_OVERFLOW, "record buffer or overflow ring too small: " +
				std::to_string(c[CNT_RECORD_OVERFLOW]) + " records and " + std::to_string(c[CNT_QUEUE_OVERFLOW]) +
				" electrons dropped");
		if (c[CNT_NAN])
			throw Error(NBL_ERR_NAN_STATE, std::to_string(c[CNT_NAN]) + " electrons reached a NaN state");
		if (c[CNT_EVENT_BUDGET] || c[CNT_WALK_OVERFLOW])
			throw Error(NBL_ERR_BUDGET_EXCEEDED, "event budget or octree step bound exceeded");
	});
}
