// C ABI: geometry, materials, device uploads, the wavefront run loop and the
// debug entry points.  See include/nebula_b200.h for the contract.
#include "internal.hpp"
#include "device.hpp"

#include <cuda_runtime.h>
#include "../device/rng.cuh"
#include <cmath>
#include <cstring>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <memory>

using namespace nbl;

namespace nbl {

static thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }

uint32_t physics_bits(const nbl_physics_opts& o)
{
	const int32_t flags[9] = { o.generate_secondaries, o.acoustic_phonon_loss, o.atomic_recoil_loss,
		o.quantum_transmission, o.interface_refraction, o.interface_absorption, o.optical_phonon_loss,
		o.instantaneous_momentum, o.momentum_conservation };
	const uint32_t bits[9] = { PH_GEN_SE, PH_PHONON, PH_RECOIL, PH_QT, PH_REFRACT, PH_ABSORB, PH_OPT_PHONON,
		PH_INST_MOM, PH_MOM_CONS };
	require(o.inelastic_model == 0 || o.inelastic_model == 1, "inelastic_model must be 0 (Full Penn) or 1 (Kieft-Bosch)");
	uint32_t r = o.inelastic_model == 1 ? PH_KIEFT : 0u;
	for (int i = 0; i < 9; ++i) {
		require(flags[i] == 0 || flags[i] == 1, "physics options are 0 or 1");
		if (flags[i]) r |= bits[i];
	}
	return r;
}

namespace {

void check_table(const nbl_table& t, int rank, const char* name)
{
	require(t.data != nullptr, std::string("table ") + name + " has no data");
	require(t.nx >= 2 && t.ny >= 1 && t.nz >= 1, std::string("table ") + name + " too small");
	if (rank >= 2) require(t.ny >= 2, std::string("table ") + name + " needs >= 2 rows");
	if (rank >= 3) require(t.nz >= 2, std::string("table ") + name + " needs >= 2 planes");
	if (rank < 3) require(t.nz == 1, std::string("table ") + name + " has the wrong rank");
	if (rank < 2) require(t.ny == 1, std::string("table ") + name + " has the wrong rank");
}

HostTable copy_table(const nbl_table& t)
{
	HostTable h;
	h.nx = t.nx; h.ny = t.ny; h.nz = t.nz;
	h.x_min = t.x_min; h.x_step = t.x_step; h.y_min = t.y_min; h.y_step = t.y_step; h.z_min = t.z_min; h.z_step = t.z_step;
	h.data.assign(t.data, t.data + (size_t)t.nx * t.ny * t.nz);
	return h;
}

}  // namespace
}  // namespace nbl

/* ======================================================================= */
/* simulation object                                                        */
struct nbl_sim {
	int device = 0;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	nbl_params params{};
	DeviceGeometry geom;
	DeviceMaterials mats;
	DevBuf queues[2][N_QUEUES][8];
	DevBuf spill[6];
	DevBuf ctrl, counters, detected, n_detected, se_img, bse_img, hist, grad_se, grad_bse, wsign_se, wsign_bse;
	DevBuf deposits, n_deposits, dep_grid;
	std::vector<nbl_deposit_record> host_deposits;   // deposit records drained during runs
	uint32_t deposits_seen = 0, deposit_growth = 0;
	DevBuf primaries;
	uint64_t pri_cap = 0, n_pri = 0;
	StepParams sp{};
	int grid = 0, block = 256;
	uint32_t graph_iters = 24;
	uint64_t iteration = 0;
	cudaGraphExec_t graph = nullptr;
	bool graph_dirty = true;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	double kernel_ms = 0;
	std::vector<nbl_record> host_records;   // records drained from the device during runs
	uint32_t records_seen = 0;              // device record count at the last graph boundary
	uint32_t record_growth = 0;             // most records one graph has added
	uint32_t* pinned_ctrl = nullptr;        // control slot, record count, then the counters
	static constexpr size_t PINNED_COUNTERS_OFFSET = ((SLOT_WORDS + 4) * sizeof(uint32_t) + 7) & ~(size_t)7;
	static constexpr size_t PINNED_BYTES = PINNED_COUNTERS_OFFSET + N_COUNTERS * sizeof(unsigned long long);
	unsigned long long* pinned_counters()
	{
		return reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(pinned_ctrl) + PINNED_COUNTERS_OFFSET);
	}

	// Record sink: page-locked host memory that receives a run's detected
	// records while it runs.  The kernel appends them to the device buffer;
	// after each graph the records that graph added are copied into the sink
	// on a copy stream while the next graph runs, so only the last graph's
	// copy is left when the run ends (the kernel's own 36-byte stores stay in
	// device memory instead of crossing the bus one by one).
	nbl_record* sink = nullptr;
	int64_t sink_cap = 0;
	bool sink_registered = false;           // page-locked by this library
	uint32_t dev_det_cap = 0;               // capacity of the device record buffer
	cudaStream_t cstream = nullptr;         // the copies into the sink
	// Streamed pushes: primaries copied from page-locked host memory in
	// chunks on the copy stream; after each chunk the count of primaries in
	// device memory is copied to `avail`, and the refill admits only those.
	DevBuf avail;                           // one word: primaries in device memory
	uint32_t* avail_host = nullptr;         // page-locked counts, one per chunk in flight
	static constexpr int AVAIL_SLOTS = 64;
	cudaEvent_t ev_first = nullptr;         // the first chunk of a streamed push has landed
	bool stream_pending = false;            // a streamed push may still be copying
	uint64_t sink_fill = 0;                 // records copied (or on their way) into the sink
	uint32_t dev_copied = 0;                // of the device buffer, records already sent to the sink
	bool sink_overflow = false;             // a run had more records than the sink holds
	bool sink_full = false;                 // records wait in the device buffer for room in a sink
	bool timing_pending = false;            // the last graph's events not yet read
	uint32_t last_ndet = 0;                 // device buffer records as of the last completed graph

	void release_sink()
	{
		if (cstream) cudaStreamSynchronize(cstream);
		if (sink_registered && sink) cudaHostUnregister(sink);
		sink_registered = false;
		sink = nullptr;
		sink_cap = 0;
	}

	// Send the device buffer's records [dev_copied, ndet) to the sink (they
	// were written by graphs that have completed).  What the sink has no
	// room for stays in the device buffer (sink_full) for the next sink.
	void sink_copy(uint32_t ndet)
	{
		ndet = std::min(ndet, sp.det_cap);
		if (ndet <= dev_copied)
			return;
		uint64_t n = ndet - dev_copied;
		if (sink_fill + n > (uint64_t)sink_cap) {
			sink_full = true;
			n = sink_fill < (uint64_t)sink_cap ? (uint64_t)sink_cap - sink_fill : 0;
		}
		if (n)
			CU(cudaMemcpyAsync(sink + sink_fill, detected.as<nbl_record>() + dev_copied, (size_t)n * sizeof(nbl_record),
				cudaMemcpyDeviceToHost, cstream));
		sink_fill += n;
		dev_copied += (uint32_t)n;
	}

	~nbl_sim()
	{
		release_sink();
		if (cstream) cudaStreamSynchronize(cstream);
		if (cstream) cudaStreamDestroy(cstream);
		if (avail_host) cudaFreeHost(avail_host);
		if (ev_first) cudaEventDestroy(ev_first);
		if (graph) cudaGraphExecDestroy(graph);
		if (ev0) cudaEventDestroy(ev0);
		if (ev1) cudaEventDestroy(ev1);
		if (pinned_ctrl) cudaFreeHost(pinned_ctrl);
		if (own_stream && stream) cudaStreamDestroy(stream);
	}

	void build_graph()
	{
		if (graph) {
			cudaGraphExecDestroy(graph);
			graph = nullptr;
		}
		cudaGraph_t g = nullptr;
		CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
		cudaError_t err = cudaSuccess;
		for (uint32_t i = 0; i < graph_iters && err == cudaSuccess; ++i)
			err = launch_step(sp, i, grid, block, stream);
		cudaError_t e2 = cudaStreamEndCapture(stream, &g);
		CU(err);
		CU(e2);
		err = cudaGraphInstantiate(&graph, g, 0);
		cudaGraphDestroy(g);
		CU(err);
		graph_dirty = false;
	}

	// Launch one graph of `graph_iters` iterations (iteration index is a
	// multiple of 6 here, so the rotating slots and queue parity line up).
	void launch_graph()
	{
		if (graph_dirty)
			build_graph();
		CU(cudaEventRecord(ev0, stream));
		CU(cudaGraphLaunch(graph, stream));
		CU(cudaEventRecord(ev1, stream));
		timing_pending = true;
		iteration += graph_iters;
	}

	// Queue counts + cursor of the next iteration's read slot.
	void read_ctrl(uint32_t out[SLOT_WORDS])
	{
		const uint32_t slot = (uint32_t)(iteration % 3);
		CU(cudaMemcpyAsync(pinned_ctrl, ctrl.as<uint32_t>() + slot * SLOT_WORDS, SLOT_WORDS * sizeof(uint32_t),
			cudaMemcpyDeviceToHost, stream));
		CU(cudaMemcpyAsync(pinned_ctrl + SLOT_WORDS, n_detected.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
		CU(cudaMemcpyAsync(pinned_counters(), counters.p, N_COUNTERS * sizeof(unsigned long long),
			cudaMemcpyDeviceToHost, stream));
		CU(cudaStreamSynchronize(stream));
		// each graph's device time counted once
		float ms = 0;
		if (timing_pending && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess)
			kernel_ms += ms;
		timing_pending = false;
		std::memcpy(out, pinned_ctrl, SLOT_WORDS * sizeof(uint32_t));
	}

	// Move device records to the host store.
	void drain_to_host(uint32_t n_dev)
	{
		const uint32_t n = std::min(n_dev, sp.det_cap);
		if (n == 0) return;
		const size_t old = host_records.size();
		host_records.resize(old + n);
		CU(cudaMemcpyAsync(host_records.data() + old, detected.p, (size_t)n * sizeof(nbl_record), cudaMemcpyDeviceToHost, stream));
		CU(cudaMemsetAsync(n_detected.p, 0, sizeof(uint32_t), stream));
		CU(cudaStreamSynchronize(stream));
	}

	// Move device deposit records to the host store.
	void drain_deposits_to_host(uint32_t n_dev)
	{
		const uint32_t n = std::min(n_dev, sp.dep_cap);
		if (n == 0) return;
		const size_t old = host_deposits.size();
		host_deposits.resize(old + n);
		CU(cudaMemcpyAsync(host_deposits.data() + old, deposits.p, (size_t)n * sizeof(nbl_deposit_record),
			cudaMemcpyDeviceToHost, stream));
		CU(cudaMemsetAsync(n_deposits.p, 0, sizeof(uint32_t), stream));
		CU(cudaStreamSynchronize(stream));
	}

	// Run graphs until done (or `max_graphs` graphs); returns electrons still
	// in flight plus primaries not yet started.  With `stop_when_sink_full`,
	// stops after the graph whose records the sink could not all take (the
	// rest wait in the device buffer for the next sink); otherwise records
	// beyond the sink are dropped and the run reports the overflow.
	int64_t advance(uint64_t max_graphs, bool stop_when_sink_full = false)
	{
		uint32_t c[SLOT_WORDS + 1];
		uint64_t stalled = 0, last_progress = ~0ull;
		// Records of a finished graph go to the sink once the next graph has
		// been launched: the copy then runs beside that graph, and the small
		// reads of the control words (queued behind the graph) never wait
		// behind a large copy on the copy engine, which would hold back the
		// next launch for the whole copy.
		bool sink_pending = false;
		uint32_t sink_upto = 0;
		if (stop_when_sink_full && sink_full) {
			// records still wait for a sink: no graph until they have one
			read_ctrl(c);
			return (int64_t)(queued(c) + spill_occupancy(c) + (n_pri - c[SLOT_CURSOR]));
		}
		for (uint64_t k = 0; k < max_graphs; ++k) {
			launch_graph();
			if (sink_pending) {
				sink_copy(sink_upto);
				sink_pending = false;
			}
			read_ctrl(c);
			// records stay on the device until the buffer could not take two
			// more graphs' worth (the most one graph has added so far, at
			// least a quarter of the buffer: a run's early graphs detect less
			// than its later ones); then they are parked on the host
			const uint32_t ndet = pinned_ctrl[SLOT_WORDS];
			last_ndet = ndet;
			record_growth = std::max(record_growth, ndet >= records_seen ? ndet - records_seen : ndet);
			const uint64_t reserve = std::max<uint64_t>(2ull * record_growth, sp.det_cap / 4);
			if (sink) {
				if ((uint64_t)ndet + reserve > sp.det_cap) {
					// the buffer is reused from its start once its records
					// are in the sink
					sink_copy(ndet);
					if (sink_full && stop_when_sink_full)
						return (int64_t)(queued(c) + spill_occupancy(c) + (n_pri - c[SLOT_CURSOR]));
					if (sink_full)
						sink_overflow = true;       // the rest is dropped
					CU(cudaStreamSynchronize(cstream));
					CU(cudaMemsetAsync(n_detected.p, 0, sizeof(uint32_t), stream));
					dev_copied = 0;
					last_ndet = 0;
					records_seen = 0;
				} else {
					sink_pending = true;
					sink_upto = ndet;
					records_seen = ndet;
				}
			} else if ((uint64_t)ndet + reserve > sp.det_cap) {
				drain_to_host(ndet);
				records_seen = 0;
			} else {
				records_seen = ndet;
			}
			if (sp.dep) {
				// deposit records: the same rule
				uint32_t ndep = 0;
				CU(cudaMemcpyAsync(&ndep, n_deposits.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
				CU(cudaStreamSynchronize(stream));
				deposit_growth = std::max(deposit_growth, ndep >= deposits_seen ? ndep - deposits_seen : ndep);
				const uint64_t dres = std::max<uint64_t>(2ull * deposit_growth, sp.dep_cap / 8);
				if ((uint64_t)ndep + dres > sp.dep_cap) {
					drain_deposits_to_host(ndep);
					deposits_seen = 0;
				} else {
					deposits_seen = ndep;
				}
			}
			const uint64_t active = queued(c) + spill_occupancy(c);
			const uint64_t left = n_pri - c[SLOT_CURSOR];
			if (active == 0 && left == 0) {
				if (sink_pending)
					sink_copy(sink_upto);
				return 0;
			}
			if (sink_full && stop_when_sink_full) {
				if (sink_pending)
					sink_copy(sink_upto);          // nothing more fits; the rest waits
				return (int64_t)(active + left);
			}
			// every iteration with work makes flights; none for two whole
			// graphs means the run cannot progress: report it, never spin
			const uint64_t progress = flights_done();
			if (progress == last_progress && stream_pending) {
				// nothing to do until more primaries land: wait for the copies
				CU(cudaStreamSynchronize(cstream));
				stream_pending = false;
				stalled = 0;
			} else if (progress == last_progress) {
				if (++stalled >= 2)
					throw Error(NBL_ERR_POOL_OVERFLOW, "no electron moved for two graphs of iterations");
			} else {
				stalled = 0;
			}
			last_progress = progress;
		}
		if (sink_pending)
			sink_copy(sink_upto);
		read_ctrl(c);
		return (int64_t)(queued(c) + spill_occupancy(c) + (n_pri - c[SLOT_CURSOR]));
	}

	// electrons in the queues of a control slot (the flight queue's count
	// also counts the tickets of secondaries that went to the spill ring)
	static uint64_t queued(const uint32_t* c)
	{
		uint64_t n = 0;
		for (int q = 0; q < N_QUEUES; ++q) n += q == EV_NEW ? std::min(c[q], c[SLOT_NEW_BUDGET]) : c[q];
		return n;
	}

	static uint32_t spill_occupancy(const uint32_t* c)
	{
		return c[SLOT_SPILL_TAIL] + c[SLOT_SPILL_PUSHED] - c[SLOT_SPILL_HEAD];
	}

	// flights started plus walks continued (as of the last read_ctrl): grows
	// in every iteration that has work
	uint64_t flights_done()
	{
		const unsigned long long* c = pinned_counters();
		return c[CNT_FLIGHTS] + c[CNT_RESUMED];
	}

	// the copies into the sink of the graphs run so far have landed
	void sink_wait()
	{
		if (sink)
			CU(cudaStreamSynchronize(cstream));
	}

	void check_errors()
	{
		if (sink_overflow)
			throw Error(NBL_ERR_POOL_OVERFLOW, "the record sink holds " + std::to_string(sink_cap) +
				" records, the run detected more; pass a larger sink");
		unsigned long long cnt[N_COUNTERS];
		CU(cudaMemcpyAsync(cnt, counters.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
		CU(cudaStreamSynchronize(stream));
		if (cnt[CNT_DEPOSIT_OVERFLOW])
			throw Error(NBL_ERR_POOL_OVERFLOW, std::to_string(cnt[CNT_DEPOSIT_OVERFLOW]) +
				" deposit records dropped; raise deposit_capacity");
		if (cnt[CNT_QUEUE_OVERFLOW] || cnt[CNT_RECORD_OVERFLOW])
			throw Error(NBL_ERR_POOL_OVERFLOW, "secondary overflow ring, record buffer or record sink full (" +
				std::to_string(cnt[CNT_QUEUE_OVERFLOW]) + " electrons, " + std::to_string(cnt[CNT_RECORD_OVERFLOW]) +
				" records dropped); raise capacity / record_capacity");
		if (cnt[CNT_NAN])
			throw Error(NBL_ERR_NAN_STATE, std::to_string(cnt[CNT_NAN]) + " electrons reached a NaN state");
		if (cnt[CNT_EVENT_BUDGET] || cnt[CNT_WALK_OVERFLOW])
			throw Error(NBL_ERR_BUDGET_EXCEEDED, std::to_string(cnt[CNT_EVENT_BUDGET]) +
				" electrons exceeded the event budget, " + std::to_string(cnt[CNT_WALK_OVERFLOW]) + " octree walks the step bound");
	}

	void reset_device_state()
	{
		if (cstream)
			CU(cudaStreamSynchronize(cstream));   // no copy may still land in the buffers
		CU(cudaMemsetAsync(ctrl.p, 0, ctrl.bytes, stream));
		CU(cudaMemsetAsync(counters.p, 0, counters.bytes, stream));
		CU(cudaMemsetAsync(n_detected.p, 0, n_detected.bytes, stream));
		if (se_img.p) CU(cudaMemsetAsync(se_img.p, 0, se_img.bytes, stream));
		if (bse_img.p) CU(cudaMemsetAsync(bse_img.p, 0, bse_img.bytes, stream));
		if (hist.p) CU(cudaMemsetAsync(hist.p, 0, hist.bytes, stream));
		if (grad_se.p) CU(cudaMemsetAsync(grad_se.p, 0, grad_se.bytes, stream));
		if (grad_bse.p) CU(cudaMemsetAsync(grad_bse.p, 0, grad_bse.bytes, stream));
		if (wsign_se.p) CU(cudaMemsetAsync(wsign_se.p, 0, wsign_se.bytes, stream));
		if (wsign_bse.p) CU(cudaMemsetAsync(wsign_bse.p, 0, wsign_bse.bytes, stream));
		if (n_deposits.p) CU(cudaMemsetAsync(n_deposits.p, 0, n_deposits.bytes, stream));
		if (dep_grid.p) CU(cudaMemsetAsync(dep_grid.p, 0, dep_grid.bytes, stream));
		CU(cudaStreamSynchronize(stream));
		host_deposits.clear();
		deposits_seen = 0;
		iteration = 0;
		kernel_ms = 0;
		host_records.clear();
		records_seen = 0;
		sink_fill = 0;
		dev_copied = 0;
		sink_overflow = false;
		sink_full = false;
		last_ndet = 0;
		sp.n_avail = nullptr;
		stream_pending = false;
	}

	void ensure_primary_capacity(uint64_t need)
	{
		if (need <= pri_cap) return;
		uint64_t cap = std::max<uint64_t>(need, pri_cap * 2);
		cap = std::max<uint64_t>(cap, 1024);
		DevBuf nb(cap * sizeof(Record36));
		if (n_pri)
			CU(cudaMemcpyAsync(nb.p, primaries.p, n_pri * sizeof(Record36), cudaMemcpyDeviceToDevice, stream));
		CU(cudaStreamSynchronize(stream));
		std::swap(primaries.p, nb.p);
		std::swap(primaries.bytes, nb.bytes);
		pri_cap = cap;
		sp.primaries = primaries.as<Record36>();
		graph_dirty = true;
	}
};

/* ======================================================================= */
extern "C" {

const char* nbl_last_error_string(void) { return g_last_error.c_str(); }

nbl_status nbl_device_count(int32_t* n)
{
	return guard([&] {
		require(n != nullptr, "null argument");
		int c = 0;
		const cudaError_t e = cudaGetDeviceCount(&c);
		if (e != cudaSuccess) {
			cudaGetLastError();
			c = 0;
		}
		*n = c;
	});
}
int nbl_abi_version(void) { return NBL_ABI_VERSION; }
void nbl_free(void* p) { std::free(p); }

nbl_status nbl_host_alloc(int64_t bytes, void** out)
{
	return guard([&] {
		require(out != nullptr && bytes > 0, "bad page-locked allocation");
		*out = nullptr;
		if (cudaMallocHost(out, (size_t)bytes) != cudaSuccess) {
			cudaGetLastError();
			*out = nullptr;
			throw Error(NBL_ERR_OOM, "cannot allocate " + std::to_string(bytes) + " bytes of page-locked host memory");
		}
	});
}

void nbl_host_free(void* p)
{
	if (p) cudaFreeHost(p);
}

nbl_status nbl_host_register(void* p, int64_t bytes)
{
	return guard([&] {
		require(p != nullptr && bytes > 0, "bad host range");
		const cudaError_t e = cudaHostRegister(p, (size_t)bytes, cudaHostRegisterDefault);
		if (e != cudaSuccess) {
			cudaGetLastError();
			if (e == cudaErrorHostMemoryAlreadyRegistered)
				throw Error(NBL_ERR_INVALID_ARG, "the host range is already page-locked");
			throw Error(NBL_ERR_OOM, "cannot page-lock " + std::to_string(bytes) + " bytes of host memory");
		}
	});
}

nbl_status nbl_host_unregister(void* p)
{
	return guard([&] {
		require(p != nullptr, "null pointer");
		CU(cudaHostUnregister(p));
	});
}

nbl_status nbl_load_tri_file(const char* path, nbl_triangle** out, int64_t* n)
{
	return guard([&] {
		require(path && out && n, "null argument");
		std::ifstream f(path);
		require(bool(f), std::string("cannot open ") + path, NBL_ERR_IO);
		std::vector<nbl_triangle> v;
		std::string line;
		size_t line_num = 0;
		while (std::getline(f, line)) {
			++line_num;
			const size_t i = line.find_first_not_of(" \t\r");
			if (i == std::string::npos || line[i] == '#')
				continue;
			std::istringstream ss(line);
			std::vector<std::string> cols;
			std::string c;
			while (ss >> c) cols.push_back(c);
			require(cols.size() == 11, "invalid number of columns in line " + std::to_string(line_num), NBL_ERR_IO);
			nbl_triangle t;
			t.material_in = std::stoi(cols[0]);
			t.material_out = std::stoi(cols[1]);
			float r[3][3];
			for (int k = 0; k < 9; ++k) r[k / 3][k % 3] = (float)std::stod(cols[2 + k]);
			for (int k = 0; k < 3; ++k) {
				t.r0[k] = r[0][k];
				t.e1[k] = r[1][k] - r[0][k];
				t.e2[k] = r[2][k] - r[0][k];
			}
			v.push_back(t);
		}
		*n = (int64_t)v.size();
		*out = static_cast<nbl_triangle*>(std::malloc(std::max<size_t>(v.size(), 1) * sizeof(nbl_triangle)));
		if (!*out) throw std::bad_alloc();
		std::memcpy(*out, v.data(), v.size() * sizeof(nbl_triangle));
	});
}

nbl_status nbl_load_pri_file(const char* path, nbl_record** out, int64_t* n)
{
	return guard([&] {
		require(path && out && n, "null argument");
		std::ifstream f(path, std::ios::binary | std::ios::ate);
		require(bool(f), std::string("cannot open ") + path, NBL_ERR_IO);
		const std::streamsize sz = f.tellg();
		require(sz % 36 == 0, "Unexpected end of primaries file", NBL_ERR_IO);
		f.seekg(0);
		*n = sz / 36;
		*out = static_cast<nbl_record*>(std::malloc(std::max<std::streamsize>(sz, 1)));
		if (!*out) throw std::bad_alloc();
		f.read(reinterpret_cast<char*>(*out), sz);
	});
}

/* materials */
nbl_status nbl_material_load(const char* path, nbl_material** out)
{
	return guard([&] {
		require(path && out, "null argument");
		auto m = std::make_unique<nbl_material>();
		m->m = load_material_file(path);
		*out = m.release();
	});
}

nbl_status nbl_material_create(const nbl_material_tables* t, nbl_material** out)
{
	return guard([&] {
		require(t && out, "null argument");
		require(t->models >= 1 && t->models <= 3, "models must name the Full-Penn (1) and/or Kieft-Bosch (2) tables");
		check_table(t->el_imfp, 1, "el_imfp"); check_table(t->el_icdf, 2, "el_icdf");
		auto m = std::make_unique<nbl_material>();
		m->m.el_imfp = copy_table(t->el_imfp); m->m.el_icdf = copy_table(t->el_icdf);
		if (t->models & 1) {
			check_table(t->in_imfp, 1, "in_imfp"); check_table(t->in_omega, 2, "in_omega");
			check_table(t->in_q, 3, "in_q"); check_table(t->in_binding, 3, "in_binding");
			m->m.in_imfp = copy_table(t->in_imfp); m->m.in_omega = copy_table(t->in_omega);
			m->m.in_q = copy_table(t->in_q); m->m.in_binding = copy_table(t->in_binding);
		}
		if (t->models & 2) {
			check_table(t->ki_imfp, 1, "ki_imfp"); check_table(t->ki_w0, 2, "ki_w0");
			check_table(t->ki_binding, 2, "ki_binding");
			m->m.ki_imfp = copy_table(t->ki_imfp); m->m.ki_w0 = copy_table(t->ki_w0);
			m->m.ki_binding = copy_table(t->ki_binding);
		}
		m->m.models = t->models;
		m->m.fermi = t->fermi; m->m.band_gap = t->band_gap; m->m.barrier = t->barrier;
		m->m.phonon_loss = t->phonon_loss; m->m.recoil_const = t->recoil_const;
		*out = m.release();
	});
}

nbl_status nbl_material_get_tables(const nbl_material* m, nbl_material_tables* out)
{
	return guard([&] {
		require(m && out, "null argument");
		out->el_imfp = m->m.el_imfp.view(); out->el_icdf = m->m.el_icdf.view();
		out->in_imfp = m->m.in_imfp.view(); out->in_omega = m->m.in_omega.view();
		out->in_q = m->m.in_q.view(); out->in_binding = m->m.in_binding.view();
		out->fermi = m->m.fermi; out->band_gap = m->m.band_gap; out->barrier = m->m.barrier;
		out->phonon_loss = m->m.phonon_loss; out->recoil_const = m->m.recoil_const;
		out->models = m->m.models;
		out->ki_imfp = m->m.ki_imfp.view(); out->ki_w0 = m->m.ki_w0.view(); out->ki_binding = m->m.ki_binding.view();
	});
}

nbl_status nbl_material_max_energy(const nbl_material* m, float* out)
{
	return guard([&] {
		require(m && out, "null argument");
		// get_max_energy: exp of the last IMFP abscissa (full_penn.h:42-45, elastic.h:46-49)
		auto emax = [](const HostTable& t) { return std::exp(t.x_min + (t.nx - 1) / t.x_step); };
		// (over the inelastic tables of every model the material carries)
		float e = emax(m->m.el_imfp);
		if (m->m.models & 1) e = std::min(e, emax(m->m.in_imfp));
		if (m->m.models & 2) e = std::min(e, emax(m->m.ki_imfp));
		*out = e;
	});
}

void nbl_material_destroy(nbl_material* m) { delete m; }

/* geometry */
nbl_status nbl_geometry_build(const nbl_triangle* tris, int64_t n, int32_t max_depth, int32_t split_count,
	nbl_geometry** out)
{
	return guard([&] {
		require(tris && out, "null argument");
		auto g = std::make_unique<nbl_geometry>();
		g->g = build_octree(tris, n, max_depth, split_count);
		*out = g.release();
	});
}

nbl_status nbl_geometry_from_linearized(const int32_t* octree_data, int64_t n_octree, const nbl_triangle* tris,
	int64_t n_tri, const float center[3], const float halfsize[3], nbl_geometry** out)
{
	return guard([&] {
		require(octree_data && tris && center && halfsize && out, "null argument");
		require(n_octree >= 9 && n_tri >= 0, "octree too small");
		// validate the whole structure so that no walk can read out of bounds:
		// inner nodes hold 8 in-range child offsets, leaves a -1 terminated
		// list of triangle ids, depth <= 21 (63-bit location codes)
		{
			std::vector<uint8_t> seen((size_t)n_octree, 0);
			std::vector<std::pair<int64_t, int>> stack{ { 0, 0 } };
			while (!stack.empty()) {
				const int64_t at = stack.back().first;
				const int depth = stack.back().second;
				stack.pop_back();
				require(at >= 0 && at + 8 <= n_octree, "octree inner node out of range");
				require(!seen[at], "octree has a shared or cyclic node");
				seen[at] = 1;
				require(depth < 21, "octree deeper than 21 levels");
				for (int o = 0; o < 8; ++o) {
					const int64_t v = octree_data[at + o];
					require(v != 0, "octree child offset is zero");
					if (v > 0) {
						stack.push_back({ v, depth + 1 });
					} else {
						int64_t k = -v;
						for (;; ++k) {
							require(k < n_octree, "octree leaf runs past the end");
							const int32_t t = octree_data[k];
							if (t < 0) {
								require(t == -1, "octree leaf must end with -1");
								break;
							}
							require(t < n_tri, "octree leaf names a triangle out of range");
						}
					}
				}
			}
		}
		auto g = std::make_unique<nbl_geometry>();
		g->g.octree.assign(octree_data, octree_data + n_octree);
		g->g.tris.assign(tris, tris + n_tri);
		for (int k = 0; k < 3; ++k) {
			g->g.center[k] = center[k];
			g->g.halfsize[k] = halfsize[k];
		}
		g->g.max_extent = max_extent_of(g->g.halfsize);
		*out = g.release();
	});
}

nbl_status nbl_geometry_info(const nbl_geometry* g, int64_t* n_octree, int64_t* n_tri, float center[3],
	float halfsize[3], float* max_extent)
{
	return guard([&] {
		require(g != nullptr, "null geometry");
		if (n_octree) *n_octree = (int64_t)g->g.octree.size();
		if (n_tri) *n_tri = (int64_t)g->g.tris.size();
		for (int k = 0; k < 3; ++k) {
			if (center) center[k] = g->g.center[k];
			if (halfsize) halfsize[k] = g->g.halfsize[k];
		}
		if (max_extent) *max_extent = g->g.max_extent;
	});
}

nbl_status nbl_geometry_export(const nbl_geometry* g, int32_t* octree_data, nbl_triangle* tris)
{
	return guard([&] {
		require(g != nullptr, "null geometry");
		if (octree_data) std::memcpy(octree_data, g->g.octree.data(), g->g.octree.size() * sizeof(int32_t));
		if (tris) std::memcpy(tris, g->g.tris.data(), g->g.tris.size() * sizeof(nbl_triangle));
	});
}

void nbl_geometry_destroy(nbl_geometry* g)
{
	if (!g) return;
	for (auto& kv : g->dev) {
		if (cudaSetDevice(kv.first) == cudaSuccess) {
			cudaFree(kv.second.octree);
			cudaFree(kv.second.tris);
		}
	}
	delete g;
}

nbl_status nbl_ray_query(const nbl_geometry* g, int device, int64_t n, const float* pos, const float* dir,
	const float* dist, const int32_t* ignore_tri, const int32_t* ignore_mat, float* out_dist, int32_t* out_tri)
{
	return guard([&] {
		require(g && pos && dir && dist && ignore_tri && ignore_mat && out_dist && out_tri, "null argument");
		require(n >= 0, "negative count");
		for (int64_t i = 0; i < n; ++i)
			require(ignore_tri[i] < (int64_t)g->g.tris.size(), "ignore_tri out of range");
		set_device(device);
		if (n == 0) return;
		cudaStream_t s;
		CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		struct S { cudaStream_t s; ~S() { cudaStreamDestroy(s); } } sg{ s };
		DeviceGeometry dg;
		dg.upload(g->g, s);
		DevBuf b(n * (3 * 4 + 3 * 4 + 4 + 4 + 4 + 4 + 4));
		char* p = b.as<char>();
		float* d_pos = (float*)p; p += n * 12;
		float* d_dir = (float*)p; p += n * 12;
		float* d_dist = (float*)p; p += n * 4;
		int32_t* d_it = (int32_t*)p; p += n * 4;
		int32_t* d_im = (int32_t*)p; p += n * 4;
		float* d_od = (float*)p; p += n * 4;
		int32_t* d_ot = (int32_t*)p;
		CU(cudaMemcpyAsync(d_pos, pos, n * 12, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(d_dir, dir, n * 12, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(d_dist, dist, n * 4, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(d_it, ignore_tri, n * 4, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(d_im, ignore_mat, n * 4, cudaMemcpyHostToDevice, s));
		CU(launch_ray_query(dg.view, d_pos, d_dir, d_dist, d_it, d_im, n, d_od, d_ot, s));
		CU(cudaMemcpyAsync(out_dist, d_od, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(out_tri, d_ot, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaStreamSynchronize(s));
	});
}

void nbl_physics_defaults(nbl_physics_opts* o)
{
	if (!o) return;
	o->inelastic_model = 0;
	o->generate_secondaries = 1;
	o->acoustic_phonon_loss = 1;
	o->atomic_recoil_loss = 1;
	o->quantum_transmission = 1;
	o->interface_refraction = 1;
	o->interface_absorption = 0;
	o->optical_phonon_loss = 1;
	o->instantaneous_momentum = 1;
	o->momentum_conservation = 1;
}

void nbl_params_defaults(nbl_params* p)
{
	if (!p) return;
	std::memset(p, 0, sizeof(*p));
	p->seed = 0x78c7e39bull;   // gpu_main.cu --seed default
	nbl_physics_defaults(&p->physics);
}

nbl_status nbl_sim_create(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials,
	const nbl_params* params, nbl_sim** out)
{
	return guard([&] {
		require(g && materials && params && out, "null argument");
		require(n_materials >= 1 && n_materials <= 127, "need 1..127 materials");
		const uint32_t phys = physics_bits(params->physics);
		int max_mat = -1;
		for (const nbl_triangle& t : g->g.tris)
			max_mat = std::max(max_mat, std::max(t.material_in, t.material_out));
		require(max_mat < n_materials, "geometry uses material " + std::to_string(max_mat) + " but only " +
			std::to_string(n_materials) + " materials were given");
		require(params->adjoint == 0 || n_materials <= 2, "the adjoint covers at most 2 materials (6 parameters)");

		auto s = std::make_unique<nbl_sim>();
		s->params = *params;
		s->device = params->device;
		set_device(s->device);
		if (params->stream) {
			s->stream = static_cast<cudaStream_t>(params->stream);
		} else {
			CU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
			s->own_stream = true;
		}
		CU(cudaEventCreate(&s->ev0));
		CU(cudaEventCreate(&s->ev1));
		CU(cudaMallocHost(&s->pinned_ctrl, nbl_sim::PINNED_BYTES));

		const uint32_t cap = params->capacity ? params->capacity : (1u << 20);
		require(cap >= 32 && cap <= (1u << 28), "capacity must be 32..2^28");
		s->block = params->block_size ? (int)params->block_size : 256;
		require(s->block % 32 == 0 && s->block >= 32 && s->block <= 256, "block_size must be a multiple of 32 in 32..256");
		uint32_t gi = params->iterations_per_graph ? params->iterations_per_graph : 24;
		gi = (gi + 5) / 6 * 6;
		s->graph_iters = gi;

		s->geom.upload(g->g, s->stream);
		std::vector<const HostMaterial*> ms;
		for (int i = 0; i < n_materials; ++i) {
			require(materials[i] != nullptr, "null material");
			ms.push_back(&materials[i]->m);
		}
		s->mats.upload(ms, s->stream, phys);

		StepParams& sp = s->sp;
		sp.geom = s->geom.view;
		sp.mats = s->mats.mats.as<DevMaterial>();
		sp.n_mat = n_materials;
		sp.energy_threshold = params->energy_threshold;
		sp.key.k0 = (uint32_t)params->seed;
		sp.key.k1 = (uint32_t)(params->seed >> 32);
		sp.capacity = cap;
		// population bound: a cascade grows the population well past the
		// number of primaries refilled, so every queue is sized for 8x the
		// refill target; the secondary budget keeps the population below it
		require((uint64_t)cap * 8 < (1ull << 30), "capacity too large");
		sp.qcap = 8 * cap;
		// refill at most 1/16 of the target per iteration, so the population
		// ramps up while the cascades of the first primaries develop
		sp.ramp = std::max<uint32_t>(cap / 16, 256);
		sp.refill_below = cap;
		sp.phys = phys;
		const bool adj = params->adjoint != 0;
		require(params->walk_cells <= (1u << 20), "walk_cells must be at most 2^20");
		sp.walk_cells = params->walk_cells ? params->walk_cells : 1u;
		for (int b = 0; b < 2; ++b)
			for (int q = 0; q < N_QUEUES; ++q) {
				DevBuf* qb = s->queues[b][q];
				qb[0].alloc((size_t)sp.qcap * sizeof(float4));
				qb[1].alloc((size_t)sp.qcap * sizeof(float4));
				qb[2].alloc((size_t)sp.qcap * sizeof(uint4));
				qb[3].alloc((size_t)sp.qcap * sizeof(uint32_t));
				if (adj) {
					qb[4].alloc((size_t)sp.qcap * sizeof(float4));
					qb[5].alloc((size_t)sp.qcap * sizeof(float2));
				}
				Queue& Q = sp.q[b][q];
				Q.a = qb[0].as<float4>(); Q.b = qb[1].as<float4>(); Q.c = qb[2].as<uint4>(); Q.d = qb[3].as<uint32_t>();
				Q.s = qb[4].as<float4>(); Q.s2 = qb[5].as<float2>();
				if (q == EV_WALK) {
					qb[6].alloc((size_t)sp.qcap * sizeof(float4));
					qb[7].alloc((size_t)sp.qcap * sizeof(uint4));
				}
				Q.w0 = qb[6].as<float4>(); Q.w1 = qb[7].as<uint4>();
			}
		{
			// overflow ring: at least twice the population bound, >= 2^20
			uint32_t ring = 1u << 20;
			while (ring < 2 * sp.qcap) ring <<= 1;
			DevBuf* qb = s->spill;
			qb[0].alloc((size_t)ring * sizeof(float4));
			qb[1].alloc((size_t)ring * sizeof(float4));
			qb[2].alloc((size_t)ring * sizeof(uint4));
			qb[3].alloc((size_t)ring * sizeof(uint32_t));
			if (adj) {
				qb[4].alloc((size_t)ring * sizeof(float4));
				qb[5].alloc((size_t)ring * sizeof(float2));
			}
			Queue& Q = sp.spill;
			Q.a = qb[0].as<float4>(); Q.b = qb[1].as<float4>(); Q.c = qb[2].as<uint4>(); Q.d = qb[3].as<uint32_t>();
			Q.s = qb[4].as<float4>(); Q.s2 = qb[5].as<float2>();
			Q.w0 = nullptr; Q.w1 = nullptr;
			sp.spill_mask = ring - 1;
		}
		s->ctrl.alloc(3 * SLOT_WORDS * sizeof(uint32_t));
		sp.ctrl = s->ctrl.as<uint32_t>();
		s->counters.alloc(N_COUNTERS * sizeof(unsigned long long));
		sp.counters = s->counters.as<unsigned long long>();
		sp.det_cap = params->record_capacity ? params->record_capacity : std::max<uint32_t>(4 * cap, 1u << 20);
		s->detected.alloc((size_t)sp.det_cap * sizeof(Record36));
		s->dev_det_cap = sp.det_cap;
		sp.detected = s->detected.as<Record36>();
		s->n_detected.alloc(sizeof(uint32_t));
		sp.n_detected = s->n_detected.as<uint32_t>();
		Tallies& T = sp.tal;
		T.nx = params->tally_nx; T.ny = params->tally_ny;
		require(T.nx >= 0 && T.ny >= 0 && (int64_t)T.nx * T.ny < (int64_t)1 << 28, "tally grid too large");
		if (T.nx > 0 && T.ny > 0) {
			const size_t np = (size_t)T.nx * T.ny;
			s->se_img.alloc(np * sizeof(uint32_t));
			s->bse_img.alloc(np * sizeof(uint32_t));
			T.se_img = s->se_img.as<uint32_t>();
			T.bse_img = s->bse_img.as<uint32_t>();
			if (adj) {
				s->grad_se.alloc(np * 6 * sizeof(double));
				s->grad_bse.alloc(np * 6 * sizeof(double));
				T.grad_se = s->grad_se.as<double>();
				T.grad_bse = s->grad_bse.as<double>();
			}
			// signed tallies of the work-function signs (forward and replay
			// alike) for the work-function derivative of a shifted replay
			s->wsign_se.alloc(np * 2 * sizeof(int32_t));
			s->wsign_bse.alloc(np * 2 * sizeof(int32_t));
			T.wsign_se = s->wsign_se.as<int32_t>();
			T.wsign_bse = s->wsign_bse.as<int32_t>();
		}
		require(params->adjoint_w_step >= 0.0f && params->adjoint_w_step <= 1.0f,
			"adjoint_w_step must be in [0, 1] eV");
		sp.wstep = adj ? params->adjoint_w_step : 0.0f;
		if (params->deposit_capacity) {
			sp.dep_cap = params->deposit_capacity;
			s->deposits.alloc((size_t)sp.dep_cap * sizeof(DepositRecord));
			s->n_deposits.alloc(sizeof(uint32_t));
			sp.dep = s->deposits.as<DepositRecord>();
			sp.n_dep = s->n_deposits.as<uint32_t>();
		}
		{
			const nbl_deposit_grid& dg = params->deposit_grid;
			const int64_t nv = (int64_t)dg.n[0] * dg.n[1] * dg.n[2];
			if (dg.n[0] || dg.n[1] || dg.n[2]) {
				require(dg.n[0] > 0 && dg.n[1] > 0 && dg.n[2] > 0 && nv < ((int64_t)1 << 31),
					"deposit grid dimensions must be positive and below 2^31 voxels in all");
				for (int k = 0; k < 3; ++k) {
					require(dg.voxel[k] > 0 && std::isfinite(dg.voxel[k]) && std::isfinite(dg.origin[k]),
						"deposit grid voxels must be positive and finite");
					sp.g_org[k] = dg.origin[k];
					sp.g_inv[k] = 1.0f / dg.voxel[k];
					sp.gn[k] = dg.n[k];
				}
				s->dep_grid.alloc((size_t)nv * sizeof(double));
				sp.grid = s->dep_grid.as<double>();
			}
		}
		if (params->image_filter.enabled) {
			const nbl_image_filter& f = params->image_filter;
			require(f.cos_min <= f.cos_max && f.cos_min >= -1.0f && f.cos_max <= 1.0f,
				"image filter needs -1 <= cos_min <= cos_max <= 1");
			T.filter = 1;
			T.cos_min = f.cos_min;
			T.cos_max = f.cos_max;
		}
		T.n_bins = params->hist_bins > 0 ? params->hist_bins : 200;
		T.hist_emax = params->hist_emax > 0 ? params->hist_emax : 1000.0f;
		s->hist.alloc((size_t)T.n_bins * sizeof(uint32_t));
		T.hist = s->hist.as<uint32_t>();
		sp.max_events = params->max_events ? params->max_events : (1u << 22);
		require(sp.max_events < (1u << 24), "max_events must be < 2^24");
		sp.adjoint = adj ? 1 : 0;
		s->grid = params->grid_size ? (int)params->grid_size : step_grid_size(s->device, s->block, sp);
		s->ensure_primary_capacity(1024);
		sp.n_primaries = 0;
		s->reset_device_state();
		*out = s.release();
	});
}

static void push_common(nbl_sim* s, const void* src, int64_t n, cudaMemcpyKind kind)
{
	require(s != nullptr, "null simulation");
	require(n >= 0, "negative count");
	require(s->n_pri + (uint64_t)n < 0xFFFFFFFFull, "at most 2^32-1 primaries per simulation");
	require(s->sp.tag_base + s->n_pri + (uint64_t)n <= 0xFFFFFFFFull,
		"primary offset + primaries must stay below 2^32");
	if (n == 0) return;
	set_device(s->device);
	if (s->cstream)
		CU(cudaStreamSynchronize(s->cstream));    // a streamed push before this one has landed
	s->ensure_primary_capacity(s->n_pri + n);
	CU(cudaMemcpyAsync(s->primaries.as<Record36>() + s->n_pri, src, (size_t)n * sizeof(Record36), kind, s->stream));
	CU(cudaStreamSynchronize(s->stream));
	s->n_pri += n;
	s->sp.n_primaries = (uint32_t)s->n_pri;
	s->sp.n_avail = nullptr;                      // every pushed primary is in device memory
	s->stream_pending = false;
	s->graph_dirty = true;
}

nbl_status nbl_sim_push_primaries(nbl_sim* s, const nbl_record* recs, int64_t n)
{
	return guard([&] {
		require(recs != nullptr || n == 0, "null records");
		push_common(s, recs, n, cudaMemcpyHostToDevice);
	});
}

nbl_status nbl_sim_push_primaries_streamed(nbl_sim* s, const nbl_record* recs, int64_t n)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		require(recs != nullptr || n == 0, "null records");
		require(n >= 0, "negative count");
		require(s->n_pri + (uint64_t)n < 0xFFFFFFFFull, "at most 2^32-1 primaries per simulation");
		require(s->sp.tag_base + s->n_pri + (uint64_t)n <= 0xFFFFFFFFull,
			"primary offset + primaries must stay below 2^32");
		if (n == 0) return;
		set_device(s->device);
		cudaPointerAttributes a{};
		if (!(cudaPointerGetAttributes(&a, recs) == cudaSuccess && a.type == cudaMemoryTypeHost)) {
			cudaGetLastError();
			throw Error(NBL_ERR_INVALID_ARG, "streamed pushes copy from page-locked host memory; "
				"use nbl_sim_push_primaries for pageable memory");
		}
		if (!s->cstream)
			CU(cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking));
		if (!s->avail_host)
			CU(cudaMallocHost(&s->avail_host, nbl_sim::AVAIL_SLOTS * sizeof(uint32_t)));
		if (!s->avail.p)
			s->avail.alloc(sizeof(uint32_t));
		if (!s->ev_first)
			CU(cudaEventCreateWithFlags(&s->ev_first, cudaEventDisableTiming));
		CU(cudaStreamSynchronize(s->cstream));    // earlier copies and their count slots are done
		s->ensure_primary_capacity(s->n_pri + n);
		const uint64_t first = s->n_pri;
		Record36* dst = s->primaries.as<Record36>() + first;
		// chunks of at least 2^16 primaries, at most AVAIL_SLOTS - 1 of them
		const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(nbl_sim::AVAIL_SLOTS - 1, n >> 16));
		const int64_t per = (n + chunks - 1) / chunks;
		s->avail_host[0] = (uint32_t)first;
		CU(cudaMemcpyAsync(s->avail.p, s->avail_host, sizeof(uint32_t), cudaMemcpyHostToDevice, s->cstream));
		int slot = 1;
		for (int64_t off = 0; off < n; off += per, ++slot) {
			const int64_t len = std::min(per, n - off);
			CU(cudaMemcpyAsync(dst + off, recs + off, (size_t)len * sizeof(Record36), cudaMemcpyHostToDevice, s->cstream));
			s->avail_host[slot] = (uint32_t)(first + off + len);
			CU(cudaMemcpyAsync(s->avail.p, s->avail_host + slot, sizeof(uint32_t), cudaMemcpyHostToDevice, s->cstream));
			if (off == 0)
				CU(cudaEventRecord(s->ev_first, s->cstream));
		}
		// the run's first graph starts once the first chunk is in
		CU(cudaStreamWaitEvent(s->stream, s->ev_first, 0));
		s->n_pri += n;
		s->sp.n_primaries = (uint32_t)s->n_pri;
		s->sp.n_avail = s->avail.as<uint32_t>();
		s->stream_pending = true;
		s->graph_dirty = true;
	});
}

nbl_status nbl_sim_set_primary_offset(nbl_sim* s, uint64_t first)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		require(s->n_pri == 0, "the primary offset is set while no primaries are queued (after create or reset)");
		require(first < 0xFFFFFFFFull, "the primary offset must be below 2^32 - 1");
		s->sp.tag_base = (uint32_t)first;
		s->graph_dirty = true;
	});
}

nbl_status nbl_sim_push_primaries_device(nbl_sim* s, const void* d_recs, int64_t n)
{
	return guard([&] {
		require(d_recs != nullptr || n == 0, "null records");
		push_common(s, d_recs, n, cudaMemcpyDeviceToDevice);
	});
}

nbl_status nbl_sim_step(nbl_sim* s, uint32_t iterations, int64_t* running)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		set_device(s->device);
		const uint64_t graphs = (iterations + s->graph_iters - 1) / s->graph_iters;
		const int64_t r = s->advance(std::max<uint64_t>(graphs, 1), true);
		s->sink_wait();
		if (running) *running = r;
		s->check_errors();
	});
}

nbl_status nbl_sim_run(nbl_sim* s)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		set_device(s->device);
		// a safety bound on the iterations (the stall check and the walk's
		// step bound are what end a run that cannot progress): an electron
		// cannot outlive max_events flights, a flight's walk continues over
		// cells / walk_cells iterations (64 covers the walks met here many
		// times over), and the pool refills at least one primary per
		// iteration while primaries are left
		const uint64_t bound = ((uint64_t)s->sp.max_events + 1) * 64 + s->n_pri + 16;
		const uint64_t max_graphs = bound / s->graph_iters + 2;
		const int64_t left = s->advance(max_graphs);
		s->sink_wait();
		if (s->sink_full)
			s->sink_overflow = true;
		s->check_errors();
		if (left != 0)
			throw Error(NBL_ERR_BUDGET_EXCEEDED, "run did not finish within its iteration bound");
	});
}

nbl_status nbl_sim_set_record_sink(nbl_sim* s, nbl_record* host, int64_t capacity)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		require(capacity >= 0 && capacity <= 0xFFFFFFFFll && (host || capacity == 0), "bad record sink");
		set_device(s->device);
		CU(cudaStreamSynchronize(s->stream));
		// records a stepped run could not fit into the previous sink wait in
		// the device buffer after the ones it took: they go first into the new
		// sink (or, with no new sink, to the host store)
		const bool carry = s->sink && s->dev_copied < s->last_ndet;
		s->release_sink();
		if (capacity > 0) {
			cudaPointerAttributes a{};
			if (!(cudaPointerGetAttributes(&a, host) == cudaSuccess && a.type == cudaMemoryTypeHost)) {
				cudaGetLastError();
				const cudaError_t e = cudaHostRegister(host, (size_t)capacity * sizeof(nbl_record), cudaHostRegisterDefault);
				if (e != cudaSuccess) {
					cudaGetLastError();
					throw Error(NBL_ERR_INVALID_ARG, "the record sink could not be page-locked");
				}
				s->sink_registered = true;
			}
			if (!s->cstream)
				CU(cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking));
			s->sink = host;
			s->sink_cap = capacity;
		}
		s->sink_fill = 0;
		s->sink_overflow = false;
		s->sink_full = false;
		if (carry && s->sink) {
			s->sink_copy(s->last_ndet);
			CU(cudaStreamSynchronize(s->cstream));
			return;
		}
		if (carry) {
			const uint32_t n = s->last_ndet - s->dev_copied;
			const size_t old = s->host_records.size();
			s->host_records.resize(old + n);
			CU(cudaMemcpyAsync(s->host_records.data() + old, s->detected.as<nbl_record>() + s->dev_copied,
				(size_t)n * sizeof(nbl_record), cudaMemcpyDeviceToHost, s->stream));
		}
		// records of later runs go to the device buffer either way
		s->sp.detected = s->detected.as<Record36>();
		s->sp.det_cap = s->dev_det_cap;
		s->dev_copied = 0;
		s->last_ndet = 0;
		CU(cudaMemsetAsync(s->n_detected.p, 0, sizeof(uint32_t), s->stream));
		CU(cudaStreamSynchronize(s->stream));
		s->records_seen = 0;
	});
}

nbl_status nbl_sim_sink_count(nbl_sim* s, int64_t* n)
{
	return guard([&] {
		require(s && n, "null argument");
		set_device(s->device);
		s->sink_wait();
		*n = s->sink ? (int64_t)s->sink_fill : 0;
	});
}

nbl_status nbl_sim_detected_count(nbl_sim* s, int64_t* n)
{
	return guard([&] {
		require(s && n, "null argument");
		set_device(s->device);
		uint32_t d = 0;
		CU(cudaMemcpyAsync(&d, s->n_detected.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
		// with a record sink the device buffer's records are the sink's
		*n = (int64_t)s->host_records.size() + (s->sink ? 0u : std::min(d, s->sp.det_cap));
	});
}

nbl_status nbl_sim_drain_detected(nbl_sim* s, nbl_record* out, int64_t cap, int64_t* n)
{
	return guard([&] {
		require(s && n && (out || cap == 0) && cap >= 0, "null argument");
		set_device(s->device);
		// records parked on the host during the run come first, then the
		// device buffer is copied straight into the caller's array
		const int64_t k = std::min<int64_t>(cap, (int64_t)s->host_records.size());
		if (k > 0) std::memcpy(out, s->host_records.data(), (size_t)k * sizeof(nbl_record));
		s->host_records.erase(s->host_records.begin(), s->host_records.begin() + k);
		if (s->sink) {
			// with a record sink every record is already in it
			*n = k;
			return;
		}
		uint32_t d = 0;
		CU(cudaMemcpyAsync(&d, s->n_detected.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
		d = std::min(d, s->sp.det_cap);
		int64_t m = 0;
		if (s->host_records.empty()) {
			m = std::min<int64_t>(cap - k, (int64_t)d);
			if (m > 0)
				CU(cudaMemcpyAsync(out + k, s->detected.p, (size_t)m * sizeof(nbl_record), cudaMemcpyDeviceToHost, s->stream));
		}
		if ((int64_t)d > m) {
			const size_t old = s->host_records.size();
			s->host_records.resize(old + (d - m));
			CU(cudaMemcpyAsync(s->host_records.data() + old, s->detected.as<nbl_record>() + m, (size_t)(d - m) * sizeof(nbl_record),
				cudaMemcpyDeviceToHost, s->stream));
		}
		CU(cudaMemsetAsync(s->n_detected.p, 0, sizeof(uint32_t), s->stream));
		CU(cudaStreamSynchronize(s->stream));
		s->records_seen = 0;
		*n = k + m;
	});
}

nbl_status nbl_sim_tallies(nbl_sim* s, uint32_t* se_img, uint32_t* bse_img, uint32_t* hist)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		set_device(s->device);
		const Tallies& T = s->sp.tal;
		if (se_img && s->se_img.p)
			CU(cudaMemcpyAsync(se_img, s->se_img.p, s->se_img.bytes, cudaMemcpyDeviceToHost, s->stream));
		if (bse_img && s->bse_img.p)
			CU(cudaMemcpyAsync(bse_img, s->bse_img.p, s->bse_img.bytes, cudaMemcpyDeviceToHost, s->stream));
		if (hist)
			CU(cudaMemcpyAsync(hist, T.hist, (size_t)T.n_bins * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
	});
}

nbl_status nbl_sim_counters(nbl_sim* s, nbl_counters* out)
{
	return guard([&] {
		require(s && out, "null argument");
		set_device(s->device);
		unsigned long long c[N_COUNTERS];
		uint32_t d = 0;
		CU(cudaMemcpyAsync(c, s->counters.p, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
		CU(cudaMemcpyAsync(&d, s->n_detected.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
		out->flights = c[CNT_FLIGHTS]; out->boundary = c[CNT_BOUNDARY]; out->elastic = c[CNT_ELASTIC];
		out->inelastic = c[CNT_INELASTIC]; out->spawned = c[CNT_SPAWNED]; out->detected = c[CNT_DETECTED];
		out->terminated = c[CNT_TERMINATED]; out->primaries_started = c[CNT_PRIMARIES];
		out->walk_overflow = c[CNT_WALK_OVERFLOW]; out->nan_state = c[CNT_NAN];
		out->queue_overflow = c[CNT_QUEUE_OVERFLOW]; out->record_overflow = c[CNT_RECORD_OVERFLOW];
		out->event_budget = c[CNT_EVENT_BUDGET];
		out->spilled = c[CNT_SPILLED];
		out->iterations = s->iteration;
		out->primaries_total = s->n_pri;
		out->records_pending = s->host_records.size() + (s->sink ? 0u : std::min(d, s->sp.det_cap));
		out->deposits = c[CNT_DEPOSITS];
		out->deposit_overflow = c[CNT_DEPOSIT_OVERFLOW];
		uint32_t nd = 0;
		if (s->n_deposits.p) {
			CU(cudaMemcpyAsync(&nd, s->n_deposits.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
			CU(cudaStreamSynchronize(s->stream));
		}
		out->deposits_pending = s->host_deposits.size() + std::min(nd, s->sp.dep_cap);
		out->walk_resumes = c[CNT_RESUMED];
	});
}

nbl_status nbl_sim_drain_deposits(nbl_sim* s, nbl_deposit_record* out, int64_t cap, int64_t* n)
{
	return guard([&] {
		require(s && n && (out || cap == 0) && cap >= 0, "null argument");
		require(s->sp.dep != nullptr, "the simulation was created without deposit records (deposit_capacity = 0)");
		set_device(s->device);
		s->drain_deposits_to_host([&] {
			uint32_t d = 0;
			CU(cudaMemcpyAsync(&d, s->n_deposits.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
			CU(cudaStreamSynchronize(s->stream));
			return d;
		}());
		s->deposits_seen = 0;
		const int64_t k = std::min<int64_t>(cap, (int64_t)s->host_deposits.size());
		if (k > 0) std::memcpy(out, s->host_deposits.data(), (size_t)k * sizeof(nbl_deposit_record));
		s->host_deposits.erase(s->host_deposits.begin(), s->host_deposits.begin() + k);
		*n = k;
	});
}

nbl_status nbl_sim_deposit_grid(nbl_sim* s, double* out)
{
	return guard([&] {
		require(s && out, "null argument");
		require(s->sp.grid != nullptr, "the simulation was created without a deposit grid");
		set_device(s->device);
		CU(cudaMemcpyAsync(out, s->dep_grid.p, s->dep_grid.bytes, cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
	});
}

nbl_status nbl_sim_reset(nbl_sim* s)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		set_device(s->device);
		s->n_pri = 0;
		s->sp.n_primaries = 0;
		s->graph_dirty = true;
		s->reset_device_state();
	});
}

nbl_status nbl_sim_set_theta(nbl_sim* s, const float* theta, int32_t n)
{
	return guard([&] {
		require(s && theta, "null argument");
		require(n == 3 * std::min(s->mats.n, 2), "theta holds 3 values per material (at most 2 materials)");
		set_device(s->device);
		std::vector<DevMaterial>& h = s->mats.host;
		for (int m = 0; m < n / 3; ++m) {
			require(theta[3 * m] > 0 && theta[3 * m + 1] > 0, "mean-free-path scales must be positive");
			h[m].in_scale = theta[3 * m];
			h[m].el_scale = theta[3 * m + 1];
			h[m].barrier = h[m].fermi + theta[3 * m + 2];
		}
		CU(cudaMemcpyAsync(s->mats.mats.p, h.data(), h.size() * sizeof(DevMaterial), cudaMemcpyHostToDevice, s->stream));
		CU(cudaStreamSynchronize(s->stream));
	});
}

nbl_status nbl_sim_get_theta(nbl_sim* s, float* theta, int32_t n)
{
	return guard([&] {
		require(s && theta, "null argument");
		require(n == 3 * std::min(s->mats.n, 2), "theta holds 3 values per material (at most 2 materials)");
		const std::vector<DevMaterial>& h = s->mats.host;
		for (int m = 0; m < n / 3; ++m) {
			theta[3 * m] = h[m].in_scale;
			theta[3 * m + 1] = h[m].el_scale;
			theta[3 * m + 2] = h[m].barrier - h[m].fermi;
		}
	});
}

nbl_status nbl_sim_gradients(nbl_sim* s, const nbl_sim* forward, double* grad_se, double* grad_bse)
{
	return guard([&] {
		require(s && grad_se && grad_bse, "null argument");
		require(s->params.adjoint && s->grad_se.p, "gradients need adjoint = 1 and a tally grid");
		const float step = s->sp.wstep;
		if (step > 0.0f) {
			require(forward != nullptr, "a replay with adjoint_w_step > 0 needs its forward run");
			require(forward != s && !forward->params.adjoint && forward->wsign_se.p &&
				forward->sp.tal.nx == s->sp.tal.nx && forward->sp.tal.ny == s->sp.tal.ny &&
				forward->sp.key.k0 == s->sp.key.k0 && forward->sp.key.k1 == s->sp.key.k1,
				"the forward run must be an adjoint = 0 simulation with the same seed and tally grid");
		}
		set_device(s->device);
		CU(cudaMemcpyAsync(grad_se, s->grad_se.p, s->grad_se.bytes, cudaMemcpyDeviceToHost, s->stream));
		CU(cudaMemcpyAsync(grad_bse, s->grad_bse.p, s->grad_bse.bytes, cudaMemcpyDeviceToHost, s->stream));
		CU(cudaStreamSynchronize(s->stream));
		if (step > 0.0f) {
			// d(count)/dW_m = (sum of r_m over the shifted replay's detections
			// - the same sum over the forward run's) / step
			const size_t np = (size_t)s->sp.tal.nx * s->sp.tal.ny;
			std::vector<int32_t> a(np * 2), f(np * 2);
			for (int which = 0; which < 2; ++which) {
				const DevBuf& sa = which ? s->wsign_bse : s->wsign_se;
				const DevBuf& sf = which ? forward->wsign_bse : forward->wsign_se;
				CU(cudaMemcpyAsync(a.data(), sa.p, np * 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
				CU(cudaStreamSynchronize(s->stream));
				set_device(forward->device);
				CU(cudaMemcpyAsync(f.data(), sf.p, np * 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, forward->stream));
				CU(cudaStreamSynchronize(forward->stream));
				set_device(s->device);
				double* g = which ? grad_bse : grad_se;
				for (size_t i = 0; i < np; ++i) {
					g[i * 6 + 2] = (double)(a[2 * i] - f[2 * i]) / step;
					g[i * 6 + 5] = (double)(a[2 * i + 1] - f[2 * i + 1]) / step;
				}
			}
		}
	});
}

nbl_status nbl_sim_set_seed(nbl_sim* s, uint64_t seed)
{
	return guard([&] {
		require(s != nullptr, "null simulation");
		s->sp.key.k0 = (uint32_t)seed;
		s->sp.key.k1 = (uint32_t)(seed >> 32);
		s->params.seed = seed;
		s->graph_dirty = true;
	});
}

nbl_status nbl_sim_kernel_ms(nbl_sim* s, double* ms)
{
	return guard([&] {
		require(s && ms, "null argument");
		*ms = s->kernel_ms;
	});
}

void nbl_sim_destroy(nbl_sim* s)
{
	if (!s) return;
	cudaSetDevice(s->device);
	if (s->stream) cudaStreamSynchronize(s->stream);
	delete s;
}

/* debug entry points */
nbl_status nbl_debug_kernel_arch(int device, int32_t* binary_version)
{
	return guard([&] {
		require(binary_version != nullptr, "null argument");
		set_device(device);
		int v = 0;
		CU(step_binary_version(device, &v));
		*binary_version = v;
	});
}

nbl_status nbl_debug_philox(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4])
{
	return guard([&] {
		require(counter && key && out, "null argument");
		uint32_t c[4] = { counter[0], counter[1], counter[2], counter[3] };
		nbl::PhiloxKey k;
		k.k0 = key[0];
		k.k1 = key[1];
		nbl::philox4x32_10(c, k);
		for (int i = 0; i < 4; ++i) out[i] = c[i];
	});
}

nbl_status nbl_debug_table_lookup(const nbl_material* m, int device, int32_t which, int32_t rounddown, int64_t n,
	const float* x, const float* y, const float* z, float* out)
{
	return guard([&] {
		require(m && x && y && z && out, "null argument");
		require(which >= 0 && which <= 8 && n >= 0, "bad arguments");
		// 6..8: the Kieft-Bosch tables, uploaded in the inelastic slots
		// (ki_imfp -> in_imfp, ki_w0 -> in_omega, ki_binding -> in_binding, 2-D)
		const bool kieft = which >= 6;
		set_device(device);
		if (n == 0) return;
		cudaStream_t s;
		CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		struct S { cudaStream_t s; ~S() { cudaStreamDestroy(s); } } sg{ s };
		DeviceMaterials dm;
		dm.upload({ &m->m }, s, kieft ? (PH_DEFAULT | PH_KIEFT) : PH_DEFAULT);
		DevBuf b(n * 16);
		float* dx = b.as<float>();
		float* dy = dx + n;
		float* dz = dy + n;
		float* dout = dz + n;
		CU(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(dy, y, n * 4, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(dz, z, n * 4, cudaMemcpyHostToDevice, s));
		CU(launch_table_kat(dm.mats.as<DevMaterial>(), which, rounddown, n, dx, dy, dz, dout, s));
		CU(cudaMemcpyAsync(out, dout, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaStreamSynchronize(s));
	});
}

nbl_status nbl_debug_event(const nbl_geometry* g, nbl_material* const* materials, int32_t n_materials, int device,
	const nbl_physics_opts* physics, int32_t kind, int64_t n, const float* state_in, const int32_t* mat_in, const int32_t* tri, const float* uniforms,
	int32_t n_uniforms, float* state_out, int32_t* mat_out, int32_t* status, float* se_out, int32_t* has_se,
	int32_t* used)
{
	return guard([&] {
		require(materials && state_in && mat_in && uniforms && state_out && mat_out && status && se_out && has_se && used,
			"null argument");
		require(kind >= 1 && kind <= 3 && n >= 0 && n_uniforms > 0 && n_materials >= 1, "bad arguments");
		if (kind == 3) {
			require(g && tri, "boundary events need a geometry and triangles");
			for (int64_t i = 0; i < n; ++i)
				require(tri[i] >= 0 && tri[i] < (int64_t)g->g.tris.size(), "triangle index out of range");
		} else {
			for (int64_t i = 0; i < n; ++i)
				require(mat_in[i] >= 0 && mat_in[i] < n_materials, "scatter events need a physical material");
		}
		nbl_physics_opts def;
		nbl_physics_defaults(&def);
		const uint32_t phys = physics_bits(physics ? *physics : def);
		set_device(device);
		if (n == 0) return;
		cudaStream_t s;
		CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		struct S { cudaStream_t s; ~S() { cudaStreamDestroy(s); } } sg{ s };
		std::vector<const HostMaterial*> ms;
		for (int i = 0; i < n_materials; ++i) ms.push_back(&materials[i]->m);
		DeviceMaterials dm;
		dm.upload(ms, s, phys);
		DeviceGeometry dg;
		if (g) dg.upload(g->g, s);
		const size_t nu = (size_t)n * n_uniforms;
		DevBuf b(n * (7 * 4 * 3 + 4 * 6) + nu * 4);
		char* p = b.as<char>();
		float* d_si = (float*)p; p += n * 28;
		float* d_so = (float*)p; p += n * 28;
		float* d_se = (float*)p; p += n * 28;
		int32_t* d_mi = (int32_t*)p; p += n * 4;
		int32_t* d_tri = (int32_t*)p; p += n * 4;
		int32_t* d_mo = (int32_t*)p; p += n * 4;
		int32_t* d_st = (int32_t*)p; p += n * 4;
		int32_t* d_hs = (int32_t*)p; p += n * 4;
		int32_t* d_us = (int32_t*)p; p += n * 4;
		float* d_u = (float*)p;
		CU(cudaMemcpyAsync(d_si, state_in, n * 28, cudaMemcpyHostToDevice, s));
		CU(cudaMemcpyAsync(d_mi, mat_in, n * 4, cudaMemcpyHostToDevice, s));
		if (tri) CU(cudaMemcpyAsync(d_tri, tri, n * 4, cudaMemcpyHostToDevice, s));
		else CU(cudaMemsetAsync(d_tri, 0, n * 4, s));
		CU(cudaMemcpyAsync(d_u, uniforms, nu * 4, cudaMemcpyHostToDevice, s));
		CU(launch_event_kat(dg.view, dm.mats.as<DevMaterial>(), phys, kind, n, d_si, d_mi, d_tri, d_u, n_uniforms, d_so, d_mo,
			d_st, d_se, d_hs, d_us, s));
		CU(cudaMemcpyAsync(state_out, d_so, n * 28, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(mat_out, d_mo, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(status, d_st, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(se_out, d_se, n * 28, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(has_se, d_hs, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaMemcpyAsync(used, d_us, n * 4, cudaMemcpyDeviceToHost, s));
		CU(cudaStreamSynchronize(s));
	});
}

}  // extern "C"
