// nebula_b200_gpu: the command-line driver, a drop-in for the reference's
// GPU executable (gpu_main.cu).  Same arguments and outputs:
//
//   nebula_b200_gpu [options] <geometry.tri> <primaries.pri> [material0] .. [materialN]
//
// detected electrons go to stdout as the reference writes them
// (gpu_main.cu:216-223: float pos[3], dir[3], E; int px, py; 36 bytes,
// little-endian), progress and a "Timing (seconds):" block to stderr.
// Options of gpu_main.cu:247-253 (--energy-threshold, --capacity,
// --prescan-size, --batch-factor, --seed, --sort-primaries; --key=value or
// --key value) plus --device and the physics selection of physics_config.h
// as run-time switches.  Material files are .nmat (the content of the
// reference's HDF5 .mat files).
//
// Built a second time with NBL_DRIVER_EDEP as nebula_b200_edep, a drop-in
// for the reference's energy-deposit executable (cpu_energydep.cpp): its
// options --energy-threshold, --seed, --detect-filename (default
// detected.bin) and --deposit-filename (default stdout, "stdout" meaning
// standard output), 28-byte deposit records (position after the event,
// energy before it, energy lost; pixel: cpu_energydep.cpp:197-204) and the
// 36-byte detected records.
//
// Like gpu_main.cu:284-295 it runs one worker thread per GPU (--devices:
// all visible devices by default, or a list), each with its own simulation
// handle; the workers pull contiguous ranges of the primary array from one
// shared cursor (the reference's work_pool, gpu_main.cu:213) and each range
// runs with its first primary's index as the primary offset, so every
// primary draws the random numbers it draws in a one-GPU run and the records
// are those of that run (in another order).  Records of all workers go out
// through one writer thread (the reference's mutexed output stream).
//
// It uses only the C ABI of include/nebula_b200.h.  Other differences from
// the reference drivers: no prescan (--prescan-size and --batch-factor are
// accepted and ignored: the library keeps its pool full by itself), and
// every primary is simulated (gpu_main.cu:228-229 can end a run one input
// batch early when a frame starts with nothing in flight).
#include "nebula_b200.h"

#include <algorithm>
#include <atomic>
#include <deque>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

#ifdef NBL_DRIVER_EDEP
constexpr bool kEdep = true;
constexpr const char* kProgram = "nebula_b200_edep";
#else
constexpr bool kEdep = false;
constexpr const char* kProgram = "nebula_b200_gpu";
#endif

struct Option {
	std::string value;
	const char* help;
};

struct Cli {
	std::map<std::string, Option> opts;
	std::vector<std::string> positional;

	void add(const char* key, const char* def, const char* help) { opts[key] = { def, help }; }

	// --key=value, --key value, --key = value (the forms gpu_main.cu's
	// cli_params accepts, common/cli_params.h:55-90)
	void parse(int argc, char** argv)
	{
		for (int i = 1; i < argc; ++i) {
			const std::string a = argv[i];
			if (a.size() > 2 && a[0] == '-' && a[1] == '-') {
				std::string key = a.substr(2), value;
				const size_t eq = key.find('=');
				if (eq != std::string::npos) {
					value = key.substr(eq + 1);
					key = key.substr(0, eq);
				} else if (i + 1 < argc) {
					value = argv[++i];
					if (value == "=" && i + 1 < argc)
						value = argv[++i];
				}
				auto it = opts.find(key);
				if (it == opts.end())
					throw std::invalid_argument("unknown option --" + key);
				it->second.value = value;
			} else {
				positional.push_back(a);
			}
		}
	}

	const std::string& get(const char* key) const { return opts.at(key).value; }
	double num(const char* key) const { return std::stod(get(key)); }
	uint64_t u64(const char* key) const { return std::stoull(get(key), nullptr, 0); }
	bool flag(const char* key) const
	{
		const std::string& v = get(key);
		return !(v.empty() || v == "0" || v == "false" || v == "no");
	}

	void usage(FILE* f) const
	{
		std::fprintf(f, "Usage: %s [options] <geometry.tri> <primaries.pri> [material0] .. [materialN]\n"
			"Options:\n", kProgram);
		for (const auto& kv : opts)
			std::fprintf(f, "\t--%s: %s [default: %s]\n", kv.first.c_str(), kv.second.help, kv.second.value.c_str());
	}
};

struct Timer {
	std::vector<std::pair<std::string, double>> phases;
	std::chrono::steady_clock::time_point t0;
	void start() { t0 = std::chrono::steady_clock::now(); }
	void stop(const char* name)
	{
		phases.emplace_back(name, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
	}
	void print(FILE* f) const
	{
		size_t w = 0;
		for (const auto& p : phases) w = std::max(w, p.first.size());
		std::fprintf(f, "Timing (seconds):\n");
		for (const auto& p : phases)
			std::fprintf(f, "%*s: %.3f\n", (int)w, p.first.c_str(), p.second);
	}
};

// Writes record buffers to a stream on its own thread, in the order they
// are handed over (from any number of worker threads).  A buffer must not
// change until its `done` flag is set (wait()).
template<class T>
class RecordWriter {
public:
	explicit RecordWriter(FILE* f) : f_(f), thread_([this] { loop(); }) {}
	~RecordWriter()
	{
		{
			std::lock_guard<std::mutex> l(m_);
			stop_ = true;
		}
		cv_.notify_all();
		thread_.join();
	}
	void submit(const std::vector<T>* b, bool* done) { submit(b->data(), b->size(), done); }
	void submit(const T* data, size_t n, bool* done)
	{
		std::lock_guard<std::mutex> l(m_);
		rethrow();
		*done = false;
		jobs_.push_back({ data, n, done });
		cv_.notify_all();
	}
	// wait until the buffer whose flag this is has been written
	void wait(const bool* done)
	{
		std::unique_lock<std::mutex> l(m_);
		cv_.wait(l, [&] { return *done || !error_.empty(); });
		rethrow();
	}
	void finish()
	{
		{
			std::unique_lock<std::mutex> l(m_);
			cv_.wait(l, [this] { return jobs_.empty() || !error_.empty(); });
			rethrow();
		}
		if (std::fflush(f_) != 0)
			throw std::runtime_error("writing records failed");
	}

private:
	struct Job {
		const T* data;
		size_t n;
		bool* done;
	};
	void rethrow()
	{
		if (!error_.empty())
			throw std::runtime_error(error_);
	}
	void loop()
	{
		std::unique_lock<std::mutex> l(m_);
		for (;;) {
			cv_.wait(l, [this] { return !jobs_.empty() || stop_; });
			if (jobs_.empty())
				return;
			const Job j = jobs_.front();
			l.unlock();
			const bool ok = j.n == 0 || std::fwrite(j.data, sizeof(T), j.n, f_) == j.n;
			l.lock();
			if (!ok)
				error_ = "writing records failed";
			jobs_.pop_front();
			*j.done = true;
			cv_.notify_all();
		}
	}

	FILE* f_;
	std::mutex m_;
	std::condition_variable cv_;
	std::deque<Job> jobs_;
	bool stop_ = false;
	std::string error_;
	std::thread thread_;
};

void check(nbl_status s, const char* what)
{
	if (s != NBL_OK)
		throw std::runtime_error(std::string(what) + ": " + nbl_last_error_string());
}

// Interleave the low 16 bits of x, y, z (bit i of x -> bit 3i).
uint64_t spread3(uint64_t v)
{
	v &= 0xFFFF;
	v = (v | (v << 32)) & 0x001F00000000FFFFull;
	v = (v | (v << 16)) & 0x001F0000FF0000FFull;
	v = (v | (v << 8)) & 0x100F00F00F00F00Full;
	v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
	v = (v | (v << 2)) & 0x1249249249249249ull;
	return v;
}

// --sort-primaries: Morton order of the start positions over their bounding
// box, 16 bits per axis (the ordering of load_pri_file.cpp's sort_pri_file).
void sort_primaries(nbl_record* r, int64_t n)
{
	if (n < 2) return;
	float lo[3], hi[3];
	for (int a = 0; a < 3; ++a) lo[a] = hi[a] = r[0].pos[a];
	for (int64_t i = 1; i < n; ++i)
		for (int a = 0; a < 3; ++a) {
			lo[a] = std::min(lo[a], r[i].pos[a]);
			hi[a] = std::max(hi[a], r[i].pos[a]);
		}
	std::vector<uint64_t> key(n);
	for (int64_t i = 0; i < n; ++i) {
		uint64_t c[3];
		for (int a = 0; a < 3; ++a) {
			const float span = hi[a] - lo[a];
			const float t = span > 0 ? (r[i].pos[a] - lo[a]) / span : 0.0f;
			c[a] = (uint64_t)(t * 65535.0f);
		}
		key[i] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
	}
	std::vector<int64_t> order(n);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
	std::vector<nbl_record> sorted(n);
	for (int64_t i = 0; i < n; ++i) sorted[i] = r[order[i]];
	std::memcpy(r, sorted.data(), (size_t)n * sizeof(nbl_record));
}

// The reference loader's checks (load_pri_file.cpp:110-181): counted and
// reported with an example, never filtered.
void report_primaries(const nbl_record* r, int64_t n, const float lo[3], const float hi[3], float max_energy)
{
	const float eps = 10.0f * 1.1920928955078125e-07f;
	int64_t outside = 0, low = 0, high = 0, dir = 0;
	int64_t ex_out = -1, ex_low = -1, ex_high = -1, ex_dir = -1;
	for (int64_t i = 0; i < n; ++i) {
		const nbl_record& p = r[i];
		if (!(p.pos[0] > lo[0] && p.pos[1] > lo[1] && p.pos[2] > lo[2] && p.pos[0] < hi[0] && p.pos[1] < hi[1]
				&& p.pos[2] < hi[2])) {
			if (!outside++) ex_out = i;
		}
		if (!(p.energy > eps) && !low++) ex_low = i;
		if (p.energy > max_energy && !high++) ex_high = i;
		if (!(std::fabs(p.dir[0]) > eps || std::fabs(p.dir[1]) > eps || std::fabs(p.dir[2]) > eps) && !dir++)
			ex_dir = i;
	}
	if (outside)
		std::fprintf(stderr, "WARNING: %lld primary electrons start outside the geometry, e.g. (%g, %g, %g) nm.\n",
			(long long)outside, r[ex_out].pos[0], r[ex_out].pos[1], r[ex_out].pos[2]);
	if (low)
		std::fprintf(stderr, "WARNING: %lld primary electrons start with no kinetic energy, e.g. %g eV.\n",
			(long long)low, r[ex_low].energy);
	if (high)
		std::fprintf(stderr, "WARNING: %lld primary electrons start above the %g keV the material files cover, "
			"e.g. %g keV.\n", (long long)high, max_energy / 1000, r[ex_high].energy / 1000);
	if (dir)
		std::fprintf(stderr, "WARNING: %lld primary electrons have a zero direction vector, e.g. (%g, %g, %g).\n",
			(long long)dir, r[ex_dir].dir[0], r[ex_dir].dir[1], r[ex_dir].dir[2]);
}

int run(int argc, char** argv)
{
	Cli cli;
	cli.add("energy-threshold", "0", "Lowest energy to simulate (eV above the vacuum level)");
	cli.add("capacity", "8388608", "Electrons kept in flight on the GPU");
	cli.add("prescan-size", "1000", "Accepted for compatibility; no prescan is needed");
	cli.add("batch-factor", "0.9", "Accepted for compatibility; no input batches are sized");
	cli.add("seed", "0x78c7e39b", "Random seed");
	cli.add("sort-primaries", "0", "Sort primary electrons (Morton order of their positions) before simulation");
	cli.add("device", "", "CUDA device to run on (one; overrides --devices)");
	cli.add("devices", "all", "CUDA devices to run on, one worker thread each: all, or a comma-separated list");
	cli.add("workers-per-device", "1", "Worker threads (simulation handles) per device");
	cli.add("chunk", "0", "Primaries a worker takes from the shared queue at a time; 0: a quarter of an even share, "
		"at least 65536");
	cli.add("record-buffer", "4194304", "Detected records per page-locked host buffer (two per worker) that receive "
		"the records while the run goes; 0: drain the device buffer between steps instead");
	cli.add("first-primary", "0", "Index of the file's first primary within a larger scan (resume, or one process "
		"per GPU on disjoint files: the records equal one run over the whole scan)");
	if (kEdep) {
		cli.add("detect-filename", "detected.bin", "Filename for detected electrons");
		cli.add("deposit-filename", "stdout", "Filename for energy deposits");
		cli.add("deposit-buffer", "16777216", "Deposit records buffered on the GPU between drains");
	}
	cli.add("inelastic-model", "0", "0: full_penn, 1: kieft_inelastic");
	cli.add("generate-secondaries", "1", "Inelastic events create secondary electrons");
	cli.add("acoustic-phonon-loss", "1", "kieft_elastic acoustic phonon loss below 200 eV");
	cli.add("atomic-recoil-loss", "1", "kieft_elastic atomic recoil loss above 200 eV");
	cli.add("optical-phonon-loss", "1", "kieft_inelastic optical phonon loss");
	cli.add("instantaneous-momentum", "1", "kieft_inelastic instantaneous momentum");
	cli.add("momentum-conservation", "1", "kieft_inelastic momentum conservation");
	cli.add("quantum-transmission", "1", "boundary_intersect quantum-mechanical transmission");
	cli.add("interface-refraction", "1", "boundary_intersect refraction");
	cli.add("interface-absorption", "0", "boundary_intersect empirical absorption");
	try {
		cli.parse(argc, argv);
	} catch (const std::exception& e) {
		std::fprintf(stderr, "%s\n", e.what());
		cli.usage(stderr);
		return 1;
	}
	if (cli.positional.size() < 3) {
		cli.usage(stderr);
		return 1;
	}
	std::fprintf(stderr, "nebula_b200 (C ABI version %d): B200 electron transport\n\n", nbl_abi_version());
	// the selected physics, as the reference's print_info lines report its
	// compiled-in models (gpu_main.cu:239-243)
	std::fprintf(stderr, "Physics models:\n");
	if (cli.u64("inelastic-model") == 1)
		std::fprintf(stderr, "  inelastic: kieft_inelastic (optical phonon loss %d, generate secondaries %d, "
			"instantaneous momentum %d, momentum conservation %d)\n", (int)cli.flag("optical-phonon-loss"),
			(int)cli.flag("generate-secondaries"), (int)cli.flag("instantaneous-momentum"),
			(int)cli.flag("momentum-conservation"));
	else
		std::fprintf(stderr, "  inelastic: full_penn (generate secondaries %d)\n", (int)cli.flag("generate-secondaries"));
	std::fprintf(stderr, "  elastic:   kieft_elastic (acoustic phonon loss %d, atomic recoil loss %d)\n",
		(int)cli.flag("acoustic-phonon-loss"), (int)cli.flag("atomic-recoil-loss"));
	std::fprintf(stderr, "  boundary:  boundary_intersect (quantum transmission %d, interface refraction %d, "
		"interface absorption %d)\n\n", (int)cli.flag("quantum-transmission"), (int)cli.flag("interface-refraction"),
		(int)cli.flag("interface-absorption"));
	static char stdout_buffer[1 << 22];
	std::setvbuf(stdout, stdout_buffer, _IOFBF, sizeof(stdout_buffer));

	Timer timer;
	std::fprintf(stderr, "Loading geometry...\n");
	timer.start();
	nbl_triangle* tris = nullptr;
	int64_t n_tri = 0;
	check(nbl_load_tri_file(cli.positional[0].c_str(), &tris, &n_tri), "loading triangles");
	timer.stop("Loading triangles");
	if (n_tri == 0) {
		std::fprintf(stderr, "Error: could not load triangles!\n");
		nbl_free(tris);
		return 1;
	}
	const int n_mat = (int)cli.positional.size() - 2;
	int max_material = -1;
	for (int64_t i = 0; i < n_tri; ++i)
		max_material = std::max({ max_material, tris[i].material_in, tris[i].material_out });
	if (max_material >= n_mat) {
		std::fprintf(stderr, "Error: not enough materials provided for this geometry!\n"
			"  Expected %d materials, %d provided.\n", max_material + 1, n_mat);
		nbl_free(tris);
		return 1;
	}
	if (max_material < n_mat - 1)
		std::fprintf(stderr, "Warning: too many materials provided for this geometry!\n"
			"  Expected %d materials, %d provided.\n", max_material + 1, n_mat);
	timer.start();
	nbl_geometry* geom = nullptr;
	const nbl_status gs = nbl_geometry_build(tris, n_tri, 0, 0, &geom);
	nbl_free(tris);
	check(gs, "building the octree");
	timer.stop("Building acceleration structure");

	std::fprintf(stderr, "Loading materials...\n");
	timer.start();
	std::vector<nbl_material*> mats(n_mat, nullptr);
	float max_energy = INFINITY;
	for (int i = 0; i < n_mat; ++i) {
		check(nbl_material_load(cli.positional[2 + i].c_str(), &mats[i]), "loading a material");
		float e = 0;
		check(nbl_material_max_energy(mats[i], &e), "material energy range");
		max_energy = std::min(max_energy, e);
	}
	timer.stop("Loading materials");

	std::fprintf(stderr, "Loading primary electrons...\n");
	timer.start();
	nbl_record* pri = nullptr;
	int64_t n_pri = 0;
	check(nbl_load_pri_file(cli.positional[1].c_str(), &pri, &n_pri), "loading primaries");
	int64_t n_oct = 0, n_t = 0;
	float center[3], half[3], max_extent = 0;
	check(nbl_geometry_info(geom, &n_oct, &n_t, center, half, &max_extent), "geometry info");
	float lo[3], hi[3];
	for (int a = 0; a < 3; ++a) {
		lo[a] = center[a] - half[a];
		hi[a] = center[a] + half[a];
	}
	report_primaries(pri, n_pri, lo, hi, max_energy);
	if (cli.flag("sort-primaries"))
		sort_primaries(pri, n_pri);
	timer.stop("Loading primary electrons");
	if (n_pri == 0) {
		std::fprintf(stderr, "Error: could not load primary electrons!\n");
		return 1;
	}
	std::fprintf(stderr, "\nLoaded %lld triangles.\n  min = {%g, %g, %g}\n  max = {%g, %g, %g}\n"
		"Loaded %lld primaries.\nLoaded %d materials.\n\n", (long long)n_tri, lo[0], lo[1], lo[2], hi[0], hi[1],
		hi[2], (long long)n_pri, n_mat);

	nbl_params p;
	nbl_params_defaults(&p);
	p.capacity = (uint32_t)cli.u64("capacity");
	p.energy_threshold = (float)cli.num("energy-threshold");
	p.seed = cli.u64("seed");
	p.physics.inelastic_model = (int32_t)cli.u64("inelastic-model");
	p.physics.generate_secondaries = cli.flag("generate-secondaries");
	p.physics.acoustic_phonon_loss = cli.flag("acoustic-phonon-loss");
	p.physics.atomic_recoil_loss = cli.flag("atomic-recoil-loss");
	p.physics.optical_phonon_loss = cli.flag("optical-phonon-loss");
	p.physics.instantaneous_momentum = cli.flag("instantaneous-momentum");
	p.physics.momentum_conservation = cli.flag("momentum-conservation");
	p.physics.quantum_transmission = cli.flag("quantum-transmission");
	p.physics.interface_refraction = cli.flag("interface-refraction");
	p.physics.interface_absorption = cli.flag("interface-absorption");
	if (kEdep)
		p.deposit_capacity = (uint32_t)cli.u64("deposit-buffer");

	// devices and workers (gpu_main.cu:284-295: one worker per visible GPU)
	std::vector<int> devices;
	if (!cli.get("device").empty()) {
		devices.push_back((int)cli.u64("device"));
	} else if (cli.get("devices") == "all") {
		int32_t n_dev = 0;
		check(nbl_device_count(&n_dev), "counting devices");
		for (int d = 0; d < n_dev; ++d) devices.push_back(d);
	} else {
		const std::string& list = cli.get("devices");
		size_t at = 0;
		for (;;) {
			const size_t comma = list.find(',', at);
			const std::string item = list.substr(at, comma == std::string::npos ? std::string::npos : comma - at);
			if (!item.empty()) devices.push_back(std::stoi(item));
			if (comma == std::string::npos) break;
			at = comma + 1;
		}
	}
	if (devices.empty())
		throw std::runtime_error("no CUDA device to run on");
	const int per_device = std::max(1, (int)cli.u64("workers-per-device"));
	std::vector<int> worker_device;
	for (int d : devices)
		for (int k = 0; k < per_device; ++k) worker_device.push_back(d);
	const int n_workers = (int)worker_device.size();
	int64_t chunk = (int64_t)cli.u64("chunk");
	if (chunk <= 0)
		chunk = std::max<int64_t>(65536, (n_pri + 4 * n_workers - 1) / (4 * n_workers));
	std::vector<nbl_sim*> sims(n_workers, nullptr);
	for (int w = 0; w < n_workers; ++w) {
		p.device = worker_device[w];
		check(nbl_sim_create(geom, mats.data(), n_mat, &p, &sims[w]), "creating the simulation");
	}
	std::fprintf(stderr, "Running on %d device(s), %d worker(s), %lld primaries per range.\n", (int)devices.size(),
		n_workers, (long long)chunk);

	// output streams: stdout for the detected records (gpu_main.cu) or the
	// two files of cpu_energydep.cpp:169-170 ("stdout" = standard output)
	FILE* detect_f = stdout;
	FILE* deposit_f = nullptr;
	auto open_out = [](const std::string& name) {
		if (name == "stdout") return stdout;
		FILE* f = std::fopen(name.c_str(), "wb");
		if (!f) throw std::runtime_error("cannot open " + name + " for writing");
		return f;
	};
	if (kEdep) {
		detect_f = open_out(cli.get("detect-filename"));
		deposit_f = open_out(cli.get("deposit-filename"));
	}

	// the run, records streamed out as it goes (gpu_main.cu:191-231): each
	// worker's records of one step are written by the writer threads while
	// that worker runs its next step
	timer.start();
	const uint64_t first_primary = cli.u64("first-primary");
	std::atomic<int64_t> cursor{ 0 }, started{ 0 }, written{ 0 }, deposited{ 0 };
	std::atomic<bool> failed{ false };
	std::mutex err_m;
	std::string error;
	{
		RecordWriter<nbl_record> writer(detect_f);
		RecordWriter<nbl_deposit_record> dep_writer(deposit_f ? deposit_f : stdout);
		std::mutex progress_m;
		const int64_t record_buffer = (int64_t)cli.u64("record-buffer");
		auto worker = [&](int w) {
			nbl_sim* sim = sims[w];
			std::vector<nbl_record> buf[2];
			std::vector<nbl_deposit_record> dbuf[2];
			bool done[2] = { true, true }, ddone[2] = { true, true };
			// two page-locked record sinks: the run copies its records into one
			// while the writer writes the other (the device buffer drained
			// between steps when they cannot be had)
			nbl_record* sink[2] = { nullptr, nullptr };
			bool use_sink = record_buffer > 0;
			for (int k = 0; k < 2 && use_sink; ++k) {
				void* m = nullptr;
				if (nbl_host_alloc(record_buffer * (int64_t)sizeof(nbl_record), &m) == NBL_OK)
					sink[k] = static_cast<nbl_record*>(m);
				else
					use_sink = false;
			}
			try {
				int cur = 0, dcur = 0;
				if (use_sink)
					check(nbl_sim_set_record_sink(sim, sink[cur], record_buffer), "record sink");
				// hand the current sink's records to the writer and continue
				// into the other one (records that did not fit go there first)
				auto rotate = [&]() {
					int64_t n = 0;
					check(nbl_sim_sink_count(sim, &n), "record count");
					writer.submit(sink[cur], (size_t)n, &done[cur]);
					written += n;
					cur ^= 1;
					writer.wait(&done[cur]);
					check(nbl_sim_set_record_sink(sim, sink[cur], record_buffer), "record sink");
				};
				auto drain = [&](std::vector<nbl_record>& out) {
					int64_t pending = 0;
					check(nbl_sim_detected_count(sim, &pending), "record count");
					out.resize((size_t)pending);
					int64_t got = 0;
					while (got < pending) {
						int64_t n = 0;
						check(nbl_sim_drain_detected(sim, out.data() + got, pending - got, &n), "draining records");
						if (n == 0) break;
						got += n;
					}
					out.resize((size_t)got);
					written += got;
				};
				auto drain_deposits = [&](std::vector<nbl_deposit_record>& out) {
					nbl_counters c;
					check(nbl_sim_counters(sim, &c), "counters");
					out.resize((size_t)c.deposits_pending);
					int64_t got = 0;
					while (got < (int64_t)out.size()) {
						int64_t n = 0;
						check(nbl_sim_drain_deposits(sim, out.data() + got, (int64_t)out.size() - got, &n),
							"draining deposits");
						if (n == 0) break;
						got += n;
					}
					out.resize((size_t)got);
					deposited += got;
				};
				// ranges of the shared primary array, in turn
				for (;;) {
					const int64_t a = cursor.fetch_add(chunk);
					if (a >= n_pri || failed)
						break;
					const int64_t n = std::min<int64_t>(chunk, n_pri - a);
					check(nbl_sim_reset(sim), "reset");
					check(nbl_sim_set_primary_offset(sim, first_primary + (uint64_t)a), "primary offset");
					check(nbl_sim_push_primaries(sim, pri + a, n), "pushing primaries");
					int64_t running = 1, seen = 0;
					for (bool full = false; !failed && (running > 0 || full);) {
						check(nbl_sim_step(sim, 240, &running), "transport");
						if (use_sink) {
							// a step stops early when the sink is full (the records
							// that did not fit go into the next one); a range's end
							// hands its records over before the next reset
							int64_t n = 0;
							check(nbl_sim_sink_count(sim, &n), "record count");
							full = n >= record_buffer;
							if (full || running == 0)
								rotate();
						} else {
							writer.wait(&done[cur]);        // this buffer's previous records are out
							drain(buf[cur]);
							writer.submit(&buf[cur], &done[cur]);
							cur ^= 1;
						}
						if (kEdep) {
							dep_writer.wait(&ddone[dcur]);
							drain_deposits(dbuf[dcur]);
							dep_writer.submit(&dbuf[dcur], &ddone[dcur]);
							dcur ^= 1;
						}
						nbl_counters c;
						check(nbl_sim_counters(sim, &c), "counters");
						started += (int64_t)c.primaries_started - seen;
						seen = (int64_t)c.primaries_started;
						std::lock_guard<std::mutex> l(progress_m);
						std::fprintf(stderr, " \rProgress %.2f%% | Running: %lld",
							100.0 * (double)started / (double)std::max<int64_t>(n_pri, 1), (long long)running);
					}
				}
			} catch (const std::exception& e) {
				std::lock_guard<std::mutex> l(err_m);
				if (error.empty())
					error = "device " + std::to_string(worker_device[w]) + ": " + e.what();
				failed = true;
			}
			// the writers may still hold this worker's buffers
			for (int k = 0; k < 2; ++k) {
				try { writer.wait(&done[k]); } catch (const std::exception&) { failed = true; }
				if (kEdep)
					try { dep_writer.wait(&ddone[k]); } catch (const std::exception&) { failed = true; }
			}
			// the simulation lets go of the sinks (its copies done) before they are freed
			if (sink[0] || sink[1]) {
				nbl_sim_set_record_sink(sim, nullptr, 0);
				nbl_host_free(sink[0]);
				nbl_host_free(sink[1]);
			}
		};
		std::vector<std::thread> threads;
		for (int w = 0; w < n_workers; ++w)
			threads.emplace_back(worker, w);
		for (std::thread& t : threads)
			t.join();
		if (failed)
			throw std::runtime_error(error.empty() ? std::string("writing records failed") : error);
		writer.finish();
		if (kEdep)
			dep_writer.finish();
	}
	if (detect_f != stdout) std::fclose(detect_f);
	if (deposit_f && deposit_f != stdout) std::fclose(deposit_f);
	timer.stop("Simulation");
	std::fprintf(stderr, "\nSimulation successful!\n%lld detected electrons written.\n", (long long)written.load());
	if (kEdep)
		std::fprintf(stderr, "%lld energy deposits written.\n", (long long)deposited.load());
	std::fprintf(stderr, "\n");
	timer.print(stderr);

	for (nbl_sim* sim : sims) nbl_sim_destroy(sim);
	nbl_free(pri);
	for (nbl_material* m : mats) nbl_material_destroy(m);
	nbl_geometry_destroy(geom);
	return 0;
}

}  // namespace

int main(int argc, char** argv)
{
	try {
		return run(argc, argv);
	} catch (const std::exception& e) {
		std::fprintf(stderr, "\nError: %s\n", e.what());
		return 1;
	}
}
