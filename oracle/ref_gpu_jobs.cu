/*
 * Test infrastructure (oracle), not product code.
 *
 * The reference's plain GPU driver run job after job, for the comparison
 * with the batched kernel on the mixed batch.  One process runs a list of
 * jobs (geometry, primaries, seed) against one set of material files; for
 * each job it performs the steps of the reference's per-GPU worker
 * (gpu_main.cu:92-232) on one GPU: build the octree and upload it, construct
 * the reference's `gpu_driver` (capacity 10^6 as gpu_main.cu:249), run the
 * prescan on the first 1 000 primaries and derive frame and batch sizes from
 * it (gpu_main.cu:130-186), then loop over frames -- buffer_detected,
 * push_to_simulation, frame_size x do_iteration, push_to_buffer,
 * flush_buffered -- until the work pool is empty and nothing runs
 * (gpu_main.cu:191-231).  Every call is the reference's own code
 * (drivers/gpu/gpu_driver.inl); this file only sequences them.
 *
 * Differences from gpu_main.cu, all outside the driver:
 *   - one worker, no threads: the main thread's once-a-second progress poll
 *     (gpu_main.cu:398-415) is absent, so a job ends when its frame loop does;
 *   - phases are timed with a steady clock after cudaDeviceSynchronize
 *     (driver construction, prescan, frames) instead of the whole-second
 *     time_log;
 *   - detected electrons are counted (SE: E < 50 eV, BSE otherwise) instead
 *     of written to stdout;
 *   - degenerate prescans of very small jobs are clamped (frame size within
 *     the prescan, batch size within [1, capacity]), where gpu_main.cu would
 *     index past its statistics or divide by zero;
 *   - the frame loop ends after two consecutive frames that start with
 *     nothing running and take nothing from the work pool.  gpu_main.cu's own
 *     test (running_count == 0 && primaries.done(), gpu_main.cu:228-229)
 *     reads a running count snapshotted before the frame's push, so a frame
 *     that starts empty and drains the pool into the input buffer ends the
 *     loop with that batch never simulated -- after the prescan (which leaves
 *     nothing running) every job whose remaining primaries fit in one batch
 *     would run its 1 000 prescan primaries only.
 *
 * Usage: ref_gpu_jobs <jobs.txt> <material0> [material1 ...]
 *   jobs.txt: one job per line, "<geometry.tri> <primaries.pri> <seed>".
 * Output: one JSON object per job on stdout.
 */
#include "config/config.h"
#include "physics_config.h"
#include "core/material.h"
#include "common/work_pool.h"
#include "io/load_tri_file.h"
#include "io/load_pri_file.h"
#include "drivers/gpu/gpu_driver.h"
#include "geometry/octree.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <limits>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

using geometry_t = nbl::geometry::octree<true>;
using cpu_material_t = material<scatter_physics<false>>;
using gpu_material_t = material<scatter_physics<true>>;
using driver_t = nbl::drivers::gpu_driver<scatter_physics<true>, intersect_t, geometry_t>;

static double seconds_since(std::chrono::steady_clock::time_point t0)
{
	cudaDeviceSynchronize();
	return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int main(int argc, char** argv)
{
	if (argc < 3) {
		std::fprintf(stderr, "usage: %s <jobs.txt> <material0> [material1 ...]\n", argv[0]);
		return 1;
	}
	const uint32_t capacity = 1000000;     // gpu_main.cu:249 default
	const uint32_t prescan_size = 1000;    // gpu_main.cu:250
	const real batch_factor = 0.9f;        // gpu_main.cu:251
	const real energy_threshold = 0;       // gpu_main.cu:248

	std::vector<cpu_material_t> cpu_materials;
	for (int i = 2; i < argc; ++i)
		cpu_materials.push_back(cpu_material_t(nbl::hdf5_file(argv[i])));
	real max_energy = std::numeric_limits<real>::infinity();
	for (auto const& m : cpu_materials)
		max_energy = std::min(max_energy, (real)m.get_max_energy());
	std::vector<gpu_material_t> gpu_materials;
	for (auto const& m : cpu_materials)
		gpu_materials.push_back(gpu_material_t(m));

	std::ifstream jobs_file(argv[1]);
	std::string line;
	int job = 0;
	while (std::getline(jobs_file, line)) {
		std::istringstream ls(line);
		std::string tri_path, pri_path;
		unsigned long long seed = 0;
		if (!(ls >> tri_path >> pri_path >> seed))
			continue;

		const auto t_load = std::chrono::steady_clock::now();
		std::vector<triangle> triangles = nbl::load_tri_file(tri_path);
		const auto lin = nbl::geometry::octree_builder::linearized_octree(
			nbl::geometry::octree_builder::octree_root(triangles));
		geometry_t geometry = geometry_t::create(lin);
		std::vector<particle> primaries;
		std::vector<int2> pixels;
		std::tie(primaries, pixels) = nbl::load_pri_file(pri_path, lin.AABB_min(), lin.AABB_max(), max_energy);
		nbl::prescan_shuffle(primaries, pixels, prescan_size);
		std::vector<uint32_t> tags(primaries.size());
		std::iota(tags.begin(), tags.end(), 0);
		work_pool pool(primaries.data(), tags.data(), primaries.size());
		const double load_s = seconds_since(t_load);

		uint64_t n_se = 0, n_bse = 0;
		double construct_s, prescan_s, frames_s;
		uint32_t frame_size = 0, batch_size = 0, iterations = 0;
		{
			auto t0 = std::chrono::steady_clock::now();
			intersect_t inter;
			driver_t d(capacity, geometry, inter, gpu_materials, energy_threshold, (driver_t::seed_t)seed);
			construct_s = seconds_since(t0);

			// prescan (gpu_main.cu:130-186)
			t0 = std::chrono::steady_clock::now();
			std::vector<std::pair<uint32_t, uint32_t>> stats;
			{
				auto w = pool.get_work(prescan_size);
				stats.push_back({ d.push(std::get<0>(w), std::get<1>(w), std::get<2>(w)), 0 });
			}
			while (stats.back().first > 0) {
				d.do_iteration();
				++iterations;
				stats.push_back({ d.get_running_count(), d.get_detected_count() });
			}
			frame_size = 1 + (uint32_t)std::distance(stats.begin(), std::max_element(stats.begin(), stats.end(),
				[](std::pair<uint32_t, uint32_t> a, std::pair<uint32_t, uint32_t> b) { return a.first < b.first; }));
			frame_size = std::max<uint32_t>(1, std::min<uint32_t>(frame_size, (uint32_t)stats.size() - 1));
			if (stats.size() < 2)
				stats.push_back(stats.back());
			real acc = 0;
			for (size_t i = 2 * (size_t)frame_size; i < stats.size(); i += frame_size)
				acc += stats[i].first / real(prescan_size);
			acc += 2 * stats[frame_size].first / real(prescan_size);
			acc += 2 * stats[frame_size].second / real(prescan_size);
			const double bs = acc > 0 ? batch_factor * capacity / acc : (double)capacity;
			batch_size = (uint32_t)std::max(1.0, std::min(bs, (double)capacity));
			prescan_s = seconds_since(t0);

			// frames (gpu_main.cu:191-231); detections of the prescan are
			// still in the pool and come out with the first flush
			t0 = std::chrono::steady_clock::now();
			d.allocate_input_buffers(batch_size);
			int idle_frames = 0;
			for (;;) {
				d.buffer_detected();
				d.push_to_simulation();
				cudaDeviceSynchronize();
				for (uint32_t i = 0; i < frame_size; ++i)
					d.do_iteration();
				iterations += frame_size;
				const size_t to_go = pool.get_primaries_to_go();
				d.push_to_buffer(pool);
				const bool took = pool.get_primaries_to_go() != to_go;
				const auto running = d.flush_buffered([&](particle p, uint32_t) {
					if (p.kin_energy < 50) ++n_se; else ++n_bse;
				});
				cudaDeviceSynchronize();
				idle_frames = (running == 0 && !took && pool.done()) ? idle_frames + 1 : 0;
				if (idle_frames == 2)
					break;
			}
			frames_s = seconds_since(t0);
		}
		geometry_t::destroy(geometry);
		const cudaError_t err = cudaDeviceSynchronize();
		std::printf("{\"job\": %d, \"primaries\": %zu, \"seed\": %llu, \"load_s\": %.6f, \"construct_s\": %.6f, "
			"\"prescan_s\": %.6f, \"frames_s\": %.6f, \"frame_size\": %u, \"batch_size\": %u, \"iterations\": %u, "
			"\"se\": %llu, \"bse\": %llu, \"cuda_error\": %d}\n",
			job, primaries.size(), seed, load_s, construct_s, prescan_s, frames_s, frame_size, batch_size,
			iterations, (unsigned long long)n_se, (unsigned long long)n_bse, (int)err);
		std::fflush(stdout);
		if (err != cudaSuccess)
			return 2;
		++job;
	}
	return 0;
}
