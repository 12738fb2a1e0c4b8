// Batched runs: many jobs in one persistent launch (k_batch).
#include "internal.hpp"
#include "device.hpp"

#include <algorithm>
#include <cstring>
#include <memory>

using namespace nbl;

struct nbl_batch {
	int device = 0;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	nbl_batch_params params{};
	std::vector<std::unique_ptr<DeviceGeometry>> geoms;
	DevBuf geom_views;
	DeviceMaterials mats;
	DevBuf queues[2][N_QUEUES][6];
	DevBuf spill[4];
	DevBuf ctrl, counters, primaries, jobs, job_se, job_bse, words;
	DevBuf detected, det_job, n_detected;     // detected records of the last run and their jobs
	StepParams sp{};
	BatchParams bp{};
	int n_jobs = 0;
	int grid = 0, block = 256;
	cudaGraphExec_t graph = nullptr;
	bool graph_dirty = true;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	double last_ms = 0;
	uint32_t last_iterations = 0;

	~nbl_batch()
	{
		if (graph) cudaGraphExecDestroy(graph);
		if (ev0) cudaEventDestroy(ev0);
		if (ev1) cudaEventDestroy(ev1);
		if (own_stream && stream) cudaStreamDestroy(stream);
	}

	// clear run state, then the persistent launch
	void enqueue()
	{
		CU(cudaMemsetAsync(ctrl.p, 0, ctrl.bytes, stream));
		CU(cudaMemsetAsync(counters.p, 0, counters.bytes, stream));
		CU(cudaMemsetAsync(words.p, 0, words.bytes, stream));
		if (n_detected.p)
			CU(cudaMemsetAsync(n_detected.p, 0, n_detected.bytes, stream));
		if (n_jobs) {
			CU(cudaMemsetAsync(job_se.p, 0, job_se.bytes, stream));
			CU(cudaMemsetAsync(job_bse.p, 0, job_bse.bytes, stream));
		}
		CU(launch_batch(sp, bp, grid, block, stream));
	}

	void run()
	{
		if (params.use_graph) {
			if (graph_dirty) {
				if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
				cudaGraph_t g = nullptr;
				CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
				try {
					enqueue();
				} catch (...) {
					cudaStreamEndCapture(stream, &g);
					if (g) cudaGraphDestroy(g);
					throw;
				}
				CU(cudaStreamEndCapture(stream, &g));
				const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
				cudaGraphDestroy(g);
				CU(e);
				graph_dirty = false;
			}
			CU(cudaEventRecord(ev0, stream));
			CU(cudaGraphLaunch(graph, stream));
			CU(cudaEventRecord(ev1, stream));
		} else {
			CU(cudaEventRecord(ev0, stream));
			enqueue();
			CU(cudaEventRecord(ev1, stream));
		}
		CU(cudaStreamSynchronize(stream));
		float ms = 0;
		CU(cudaEventElapsedTime(&ms, ev0, ev1));
		last_ms = ms;
		uint32_t w[4];
		CU(cudaMemcpy(w, words.p, sizeof(w), cudaMemcpyDeviceToHost));
		last_iterations = w[3];
		unsigned long long cnt[N_COUNTERS];
		CU(cudaMemcpy(cnt, counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
		if (w[2] & 1u)
			throw Error(NBL_ERR_CUDA, "batched launch: grid barrier timed out");
		if (w[2] & 2u)
			throw Error(NBL_ERR_BUDGET_EXCEEDED, "batched launch reached its iteration bound");
		if (cnt[CNT_RECORD_OVERFLOW])
			throw Error(NBL_ERR_POOL_OVERFLOW, std::to_string(cnt[CNT_RECORD_OVERFLOW]) +
				" detected records did not fit; raise record_capacity");
		if (cnt[CNT_QUEUE_OVERFLOW])
			throw Error(NBL_ERR_POOL_OVERFLOW, std::to_string(cnt[CNT_QUEUE_OVERFLOW]) +
				" electrons did not fit the overflow ring; raise capacity or queue_factor");
		if (cnt[CNT_NAN])
			throw Error(NBL_ERR_NAN_STATE, std::to_string(cnt[CNT_NAN]) + " electrons reached a NaN state");
		if (cnt[CNT_EVENT_BUDGET] || cnt[CNT_WALK_OVERFLOW])
			throw Error(NBL_ERR_BUDGET_EXCEEDED, "event budget or octree step bound exceeded");
	}
};

extern "C" {

void nbl_batch_params_defaults(nbl_batch_params* p)
{
	if (!p) return;
	std::memset(p, 0, sizeof(*p));
	p->use_graph = 1;
	nbl_physics_defaults(&p->physics);
}

nbl_status nbl_batch_create(const nbl_geometry* const* geometries, int32_t n_geometries, nbl_material* const* materials,
	int32_t n_materials, const nbl_batch_params* params, nbl_batch** out)
{
	return guard([&] {
		require(geometries && materials && params && out, "null argument");
		require(n_geometries >= 1 && n_materials >= 1 && n_materials <= 127, "bad counts");
		require(n_geometries <= NBL_BATCH_MAX_GEOMS, "at most " + std::to_string(NBL_BATCH_MAX_GEOMS) +
			" geometries per batch");
		for (int i = 0; i < n_geometries; ++i) {
			require(geometries[i] != nullptr, "null geometry");
			for (const nbl_triangle& t : geometries[i]->g.tris)
				require(std::max(t.material_in, t.material_out) < n_materials, "geometry uses a missing material");
		}
		auto b = std::make_unique<nbl_batch>();
		b->params = *params;
		b->device = params->device;
		set_device(b->device);
		if (params->stream) {
			b->stream = static_cast<cudaStream_t>(params->stream);
		} else {
			CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
			b->own_stream = true;
		}
		CU(cudaEventCreate(&b->ev0));
		CU(cudaEventCreate(&b->ev1));
		const uint32_t cap = params->capacity ? params->capacity : (1u << 20);
		const uint32_t factor = params->queue_factor ? params->queue_factor : 4;
		require(cap >= 32 && factor >= 2 && factor <= 16 && (uint64_t)cap * factor < (1ull << 30), "bad capacity / queue_factor");
		const float thr = params->refill_threshold > 0 ? params->refill_threshold : 1.0f;
		require(thr <= 1.0f, "refill_threshold must be in (0, 1]");
		b->block = params->block_size ? (int)params->block_size : 256;
		require(b->block == 128 || b->block == 256 || b->block == 512, "block_size must be 128, 256 or 512");

		std::vector<DevGeometry> views;
		for (int i = 0; i < n_geometries; ++i) {
			b->geoms.emplace_back(new DeviceGeometry());
			b->geoms.back()->upload(geometries[i]->g, b->stream);
			views.push_back(b->geoms.back()->view);
		}
		b->geom_views.alloc(views.size() * sizeof(DevGeometry));
		CU(cudaMemcpy(b->geom_views.p, views.data(), views.size() * sizeof(DevGeometry), cudaMemcpyHostToDevice));
		std::vector<const HostMaterial*> ms;
		for (int i = 0; i < n_materials; ++i) {
			require(materials[i] != nullptr, "null material");
			ms.push_back(&materials[i]->m);
		}
		const uint32_t phys = physics_bits(params->physics);
		b->mats.upload(ms, b->stream, phys);

		StepParams& sp = b->sp;
		sp.mats = b->mats.mats.as<DevMaterial>();
		sp.n_mat = n_materials;
		// co-resident grid with the staged materials' shared memory
		b->grid = batch_grid_size(b->device, b->block, sp);
		require(b->grid > 0, "the batched kernel does not fit on this device with that block size");
		sp.energy_threshold = params->energy_threshold;
		sp.capacity = cap;
		sp.qcap = factor * cap;
		sp.ramp = std::max<uint32_t>(cap / 16, 256);
		sp.refill_below = std::max<uint32_t>(1u, (uint32_t)((double)thr * cap));
		sp.phys = phys;
		require(params->walk_cells <= (1u << 20), "walk_cells must be at most 2^20");
		sp.walk_cells = params->walk_cells ? params->walk_cells : 1u;
		for (int k = 0; k < 2; ++k)
			for (int q = 0; q < N_QUEUES; ++q) {
				DevBuf* qb = b->queues[k][q];
				qb[0].alloc((size_t)sp.qcap * sizeof(float4));
				qb[1].alloc((size_t)sp.qcap * sizeof(float4));
				qb[2].alloc((size_t)sp.qcap * sizeof(uint4));
				qb[3].alloc((size_t)sp.qcap * sizeof(uint32_t));
				Queue& Q = sp.q[k][q];
				Q.a = qb[0].as<float4>(); Q.b = qb[1].as<float4>(); Q.c = qb[2].as<uint4>(); Q.d = qb[3].as<uint32_t>();
				Q.s = nullptr; Q.s2 = nullptr; Q.w0 = nullptr; Q.w1 = nullptr;
				if (q == EV_WALK) {
					qb[4].alloc((size_t)sp.qcap * sizeof(float4));
					qb[5].alloc((size_t)sp.qcap * sizeof(uint4));
					Q.w0 = qb[4].as<float4>(); Q.w1 = qb[5].as<uint4>();
				}
			}
		uint32_t ring = 1u << 20;
		while (ring < 2 * sp.qcap) ring <<= 1;
		b->spill[0].alloc((size_t)ring * sizeof(float4));
		b->spill[1].alloc((size_t)ring * sizeof(float4));
		b->spill[2].alloc((size_t)ring * sizeof(uint4));
		b->spill[3].alloc((size_t)ring * sizeof(uint32_t));
		sp.spill.a = b->spill[0].as<float4>(); sp.spill.b = b->spill[1].as<float4>();
		sp.spill.c = b->spill[2].as<uint4>(); sp.spill.d = b->spill[3].as<uint32_t>();
		sp.spill.s = nullptr; sp.spill.s2 = nullptr; sp.spill.w0 = nullptr; sp.spill.w1 = nullptr;
		sp.spill_mask = ring - 1;
		b->ctrl.alloc(3 * SLOT_WORDS * sizeof(uint32_t));
		sp.ctrl = b->ctrl.as<uint32_t>();
		b->counters.alloc(N_COUNTERS * sizeof(unsigned long long));
		sp.counters = b->counters.as<unsigned long long>();
		// detected records of every job in one buffer, each with its job
		// beside it (the batch runs in one launch: the buffer holds the
		// whole batch's records)
		sp.detected = nullptr;
		sp.n_detected = nullptr;
		sp.det_cap = 0;
		sp.det_job = nullptr;
		if (params->record_capacity) {
			b->detected.alloc((size_t)params->record_capacity * sizeof(Record36));
			b->det_job.alloc((size_t)params->record_capacity);
			b->n_detected.alloc(sizeof(uint32_t));
			sp.detected = b->detected.as<Record36>();
			sp.det_job = b->det_job.as<uint8_t>();
			sp.n_detected = b->n_detected.as<uint32_t>();
			sp.det_cap = params->record_capacity;
		}
		sp.tal = Tallies{};
		sp.max_events = params->max_events ? params->max_events : (1u << 22);
		require(sp.max_events < (1u << 24), "max_events must be < 2^24");
		sp.adjoint = 0;
		b->words.alloc(4 * sizeof(uint32_t));   // barrier count, generation, error, iterations
		BatchParams& bp = b->bp;
		bp.geoms = b->geom_views.as<DevGeometry>();
		bp.n_geoms = (int32_t)b->geoms.size();
		bp.bar_count = b->words.as<uint32_t>();
		bp.bar_gen = bp.bar_count + 1;
		bp.err = bp.bar_count + 2;
		bp.iterations = bp.bar_count + 3;
		bp.max_iterations = params->max_iterations ? params->max_iterations : (1u << 20);
		*out = b.release();
	});
}

nbl_status nbl_batch_set_jobs(nbl_batch* b, const nbl_batch_job* jobs, int32_t n_jobs, const nbl_record* primaries,
	int64_t n_primaries)
{
	return guard([&] {
		require(b && jobs && (primaries || n_primaries == 0), "null argument");
		require(n_jobs >= 1 && n_jobs <= 255, "1..255 jobs per batch");
		require(n_primaries >= 0 && n_primaries < 0xFFFFFFFFll, "primaries count out of range");
		std::vector<DevJob> dj(n_jobs);
		int64_t prev_end = 0;
		for (int i = 0; i < n_jobs; ++i) {
			const nbl_batch_job& j = jobs[i];
			require(j.geometry >= 0 && j.geometry < (int)b->geoms.size(), "job geometry out of range");
			require(j.count >= 0 && j.count < (1 << 24), "a job holds fewer than 2^24 primaries");
			require(j.first >= prev_end && j.first + j.count <= n_primaries, "job ranges must be increasing and inside the array");
			// a primary between jobs would be picked up by the previous job
			require(i == 0 ? j.first == 0 : j.first == prev_end, "job ranges must tile the primary array");
			prev_end = j.first + j.count;
			dj[i].geom = (uint32_t)j.geometry;
			dj[i].first = (uint32_t)j.first;
			dj[i].count = (uint32_t)j.count;
			dj[i].key.k0 = (uint32_t)j.seed;
			dj[i].key.k1 = (uint32_t)(j.seed >> 32);
			dj[i].pad = 0;
		}
		require(prev_end == n_primaries, "job ranges must cover the primary array");
		set_device(b->device);
		// device buffers are reused while large enough (a batch object is
		// typically given job lists of similar size run after run)
		auto fit = [](DevBuf& buf, size_t n) { if (buf.bytes < n) buf.alloc(n); };
		fit(b->jobs, dj.size() * sizeof(DevJob));
		CU(cudaMemcpy(b->jobs.p, dj.data(), dj.size() * sizeof(DevJob), cudaMemcpyHostToDevice));
		fit(b->primaries, std::max<int64_t>(n_primaries, 1) * sizeof(Record36));
		if (n_primaries)
			CU(cudaMemcpy(b->primaries.p, primaries, n_primaries * sizeof(Record36), cudaMemcpyHostToDevice));
		fit(b->job_se, n_jobs * sizeof(unsigned long long));
		fit(b->job_bse, n_jobs * sizeof(unsigned long long));
		b->n_jobs = n_jobs;
		b->sp.primaries = b->primaries.as<Record36>();
		b->sp.n_primaries = (uint32_t)n_primaries;
		b->bp.jobs = b->jobs.as<DevJob>();
		b->bp.n_jobs = n_jobs;
		b->bp.job_se = b->job_se.as<unsigned long long>();
		b->bp.job_bse = b->job_bse.as<unsigned long long>();
		b->graph_dirty = true;
	});
}

nbl_status nbl_batch_run(nbl_batch* b)
{
	return guard([&] {
		require(b != nullptr, "null batch");
		require(b->n_jobs > 0, "no jobs set");
		set_device(b->device);
		b->run();
	});
}

nbl_status nbl_batch_job_yields(nbl_batch* b, uint64_t* se, uint64_t* bse)
{
	return guard([&] {
		require(b && se && bse, "null argument");
		set_device(b->device);
		CU(cudaMemcpy(se, b->job_se.p, b->n_jobs * sizeof(uint64_t), cudaMemcpyDeviceToHost));
		CU(cudaMemcpy(bse, b->job_bse.p, b->n_jobs * sizeof(uint64_t), cudaMemcpyDeviceToHost));
	});
}

nbl_status nbl_batch_records(nbl_batch* b, nbl_record* out, uint8_t* job, int64_t cap, int64_t* n)
{
	return guard([&] {
		require(b && n, "null argument");
		require(cap >= 0 && (cap == 0 || (out && job)), "bad output buffers");
		require(b->n_detected.p != nullptr, "the batch keeps no records (record_capacity = 0)");
		set_device(b->device);
		uint32_t nd = 0;
		CU(cudaMemcpy(&nd, b->n_detected.p, sizeof(nd), cudaMemcpyDeviceToHost));
		const int64_t have = std::min<int64_t>(nd, b->sp.det_cap);
		*n = have;
		if (cap == 0)
			return;
		require(cap >= have, "output buffer holds " + std::to_string(cap) + " records, the run detected " +
			std::to_string(have));
		CU(cudaMemcpyAsync(out, b->detected.p, (size_t)have * sizeof(nbl_record), cudaMemcpyDeviceToHost, b->stream));
		CU(cudaMemcpyAsync(job, b->det_job.p, (size_t)have, cudaMemcpyDeviceToHost, b->stream));
		CU(cudaStreamSynchronize(b->stream));
	});
}

nbl_status nbl_batch_counters(nbl_batch* b, nbl_counters* out)
{
	return guard([&] {
		require(b && out, "null argument");
		set_device(b->device);
		unsigned long long c[N_COUNTERS];
		CU(cudaMemcpy(c, b->counters.p, sizeof(c), cudaMemcpyDeviceToHost));
		std::memset(out, 0, sizeof(*out));
		out->flights = c[CNT_FLIGHTS]; out->boundary = c[CNT_BOUNDARY]; out->elastic = c[CNT_ELASTIC];
		out->inelastic = c[CNT_INELASTIC]; out->spawned = c[CNT_SPAWNED]; out->detected = c[CNT_DETECTED];
		out->terminated = c[CNT_TERMINATED]; out->primaries_started = c[CNT_PRIMARIES];
		out->walk_overflow = c[CNT_WALK_OVERFLOW]; out->nan_state = c[CNT_NAN];
		out->queue_overflow = c[CNT_QUEUE_OVERFLOW]; out->record_overflow = c[CNT_RECORD_OVERFLOW];
		out->event_budget = c[CNT_EVENT_BUDGET]; out->spilled = c[CNT_SPILLED];
		out->iterations = b->last_iterations;
		out->primaries_total = b->sp.n_primaries;
		if (b->n_detected.p) {
			uint32_t nd = 0;
			CU(cudaMemcpy(&nd, b->n_detected.p, sizeof(nd), cudaMemcpyDeviceToHost));
			out->records_pending = std::min(nd, b->sp.det_cap);
		}
	});
}

nbl_status nbl_batch_kernel_ms(nbl_batch* b, double* ms)
{
	return guard([&] {
		require(b && ms, "null argument");
		*ms = b->last_ms;
	});
}

void nbl_batch_destroy(nbl_batch* b)
{
	if (!b) return;
	cudaSetDevice(b->device);
	if (b->stream) cudaStreamSynchronize(b->stream);
	delete b;
}

}  // extern "C"
