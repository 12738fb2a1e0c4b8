/*
 * Test infrastructure (oracle), not product code.
 *
 * A thin C-callable harness around the reference's OWN code, compiled from
 * the reference sources where they lie (see oracle/Makefile) into
 * oracle/_ref/libnbl_ref.so.  Nothing here re-implements physics: every
 * entry point calls the reference's templates as its CPU driver
 * instantiates them (physics_config.h:20-46, cpu_mt_main.cpp:24-31):
 *
 *   ref_geometry_*   load_tri_file (io/load_tri_file.cpp:8-60),
 *                    octree_root + linearized_octree
 *                    (geometry/octree/octree_builder.cpp:171-352) and
 *                    octree<false>::create (geometry/octree.inl:3-7)
 *   ref_propagate    octree<false>::propagate (geometry/octree.inl:33-192)
 *   ref_material_*   material<scatter_physics<false>>(hdf5_file)
 *                    (core/material.inl:13-18): full_penn::create,
 *                    kieft_elastic::create, kieft_inelastic::create; table
 *                    dumps and table lookups
 *   ref_event        one scatter (the model's execute) or one boundary
 *                    crossing (boundary_intersect::execute) on one electron
 *                    held by the reference cpu_particle_manager, with the
 *                    reference mt19937 generator seeded by the caller, for
 *                    any combination of the models' option bools
 *   ref_simulate     the cpu_mt_main.cpp sim_loop (lines 167-201) run on ONE
 *                    thread with one seed, so the run is deterministic:
 *                    push one primary, simulate_to_end, flush_detected; for
 *                    the reference's physics selection and three others.
 *
 * Private/protected members are opened with the preprocessor so that the
 * tables can be dumped and the driver's init/intersect/scatter steps counted.
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <string>
#include <map>
#include <queue>
#include <array>
#include <iostream>
#include <sstream>
#include <fstream>
#include <random>
#include <algorithm>
#include <numeric>
#include <mutex>
#include <thread>
#include <limits>
#include <cmath>
#include <stdexcept>
#include <functional>
#include <cstdio>
#include <cstdlib>
#include <memory>

#define private public
#define protected public
#include "hdf5_standin.h"
#include "physics_config.h"
#include "core/material.h"
#include "io/load_tri_file.h"
#include "drivers/cpu/simple_cpu_driver.h"
#include "drivers/cpu/energydeposit_cpu_driver.h"
#include "geometry/octree.h"
#undef private
#undef protected

using geometry_t = nbl::geometry::octree<false>;
using material_t = material<scatter_physics<false>>;
using driver_t = nbl::drivers::simple_cpu_driver<scatter_physics<false>, intersect_t, geometry_t>;

namespace {
struct ref_geometry
{
	std::vector<triangle> input;
	nbl::geometry::octree_builder::linearized_octree lin;
	geometry_t oct;
};
thread_local std::string g_err;
}

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

/* Build from a .tri file.  Returns nullptr on error. */
void* ref_geometry_load(const char* tri_path)
{
	try {
		auto* g = new ref_geometry;
		g->input = nbl::load_tri_file(tri_path);
		if (g->input.empty())
			throw std::runtime_error("no triangles");
		g->lin = nbl::geometry::octree_builder::linearized_octree(
			nbl::geometry::octree_builder::octree_root(g->input));
		g->oct = geometry_t::create(g->lin);
		return g;
	} catch (std::exception const & e) {
		g_err = e.what();
		return nullptr;
	}
}

void ref_geometry_free(void* h)
{
	auto* g = static_cast<ref_geometry*>(h);
	geometry_t::destroy(g->oct);
	delete g;
}

/* sizes: [n_octree_data, n_triangles] */
void ref_geometry_sizes(void* h, int64_t* out)
{
	auto* g = static_cast<ref_geometry*>(h);
	out[0] = (int64_t)g->lin.octree_data.size();
	out[1] = (int64_t)g->lin.triangle_data.size();
}

/* octree_data (int32), triangles as 11 floats each in the reference member
 * order (material_in, material_out as float values, r0, e1, e2), center,
 * halfsize, max_extent. */
void ref_geometry_dump(void* h, int32_t* octree_data, float* tri11, float* center_halfsize_ext)
{
	auto* g = static_cast<ref_geometry*>(h);
	std::memcpy(octree_data, g->lin.octree_data.data(), g->lin.octree_data.size() * sizeof(int));
	for (size_t i = 0; i < g->lin.triangle_data.size(); ++i)
	{
		triangle const & t = g->lin.triangle_data[i];
		float* o = tri11 + 11 * i;
		o[0] = (float)t.material_in; o[1] = (float)t.material_out;
		o[2] = t._r0.x; o[3] = t._r0.y; o[4] = t._r0.z;
		o[5] = t._e1.x; o[6] = t._e1.y; o[7] = t._e1.z;
		o[8] = t._e2.x; o[9] = t._e2.y; o[10] = t._e2.z;
	}
	center_halfsize_ext[0] = g->oct._AABB_center.x;
	center_halfsize_ext[1] = g->oct._AABB_center.y;
	center_halfsize_ext[2] = g->oct._AABB_center.z;
	center_halfsize_ext[3] = g->oct._AABB_halfsize.x;
	center_halfsize_ext[4] = g->oct._AABB_halfsize.y;
	center_halfsize_ext[5] = g->oct._AABB_halfsize.z;
	center_halfsize_ext[6] = g->oct._max_extent;
}

/* Batch of octree<false>::propagate calls.  ignore_tri < 0 means none.
 * out_tri = -1 when no triangle is hit. */
void ref_propagate(void* h, int64_t n, const float* pos, const float* dir, const float* dist,
	const int32_t* ignore_tri, const int32_t* ignore_mat, float* out_dist, int32_t* out_tri)
{
	auto* g = static_cast<ref_geometry*>(h);
	for (int64_t i = 0; i < n; ++i)
	{
		const vec3 p{ pos[3*i], pos[3*i+1], pos[3*i+2] };
		const vec3 d{ dir[3*i], dir[3*i+1], dir[3*i+2] };
		const triangle* ign = ignore_tri[i] >= 0 ? g->oct._triangles + ignore_tri[i] : nullptr;
		intersect_event ev = g->oct.propagate(p, d, dist[i], ign, ignore_mat[i]);
		out_dist[i] = ev.isect_distance;
		out_tri[i] = ev.isect_triangle ? int32_t(ev.isect_triangle - g->oct._triangles) : -1;
	}
}

int ref_in_domain(void* h, const float* pos)
{
	auto* g = static_cast<ref_geometry*>(h);
	return g->oct.in_domain(vec3{ pos[0], pos[1], pos[2] }) ? 1 : 0;
}

/* ---------------------------------------------------------------- materials */
/* A material handle keeps the material file (the in-memory stand-in) and
 * creates the reference's objects from it: the default-physics material
 * (when the file carries Full-Penn tables) and, on demand, the scatter
 * models with other option bools or the Kieft-Bosch inelastic model. */
namespace {
using kieft_default_t = nbl::scatter::kieft_inelastic<false>;
struct ref_material
{
	nbl::hdf5_file file;
	bool penn = false, kieft = false;
	std::unique_ptr<material_t> def;
	std::unique_ptr<kieft_default_t> ki;
	float barrier = 0;
	explicit ref_material(const char* path) : file(path)
	{
		penn = file.exists("/full_penn");
		kieft = file.exists("/inelastic_kieft");
		if (penn)
			def.reset(new material_t(file));
		if (kieft)
			ki.reset(new kieft_default_t(kieft_default_t::create(file)));
		barrier = static_cast<float>(file.get_property_quantity("barrier") / nbl::units::eV);
	}
	~ref_material() { if (ki) kieft_default_t::destroy(*ki); }
};
}

void* ref_material_load(const char* path)
{
	try {
		return new ref_material(path);
	} catch (std::exception const & e) {
		g_err = e.what();
		return nullptr;
	}
}
void ref_material_free(void* h) { delete static_cast<ref_material*>(h); }

/* Table geometry: which = 0 el_imfp, 1 el_icdf, 2 in_imfp, 3 in_omega, 4 in_q,
 * 5 in_binding (Full Penn), 6 ki_imfp, 7 ki_w0, 8 ki_binding (Kieft-Bosch).
 * shape[3] (1 for absent axes), scale[6] (x_min, x_step, y_min, y_step, z_min, z_step). */
extern "C++" {
namespace {
struct table_desc { int32_t* shape; float* scale; const float** data; int64_t* pitch; };
template<class T> void desc1(const T& t, table_desc d)
{
	d.shape[0] = t._n; d.scale[0] = t._x_min; d.scale[1] = t._x_step; *d.data = t._data;
}
template<class T> void desc2(const T& t, table_desc d)
{
	d.shape[0] = t._width; d.shape[1] = t._height;
	d.scale[0] = t._x_min; d.scale[1] = t._x_step; d.scale[2] = t._y_min; d.scale[3] = t._y_step;
	*d.data = t._data; *d.pitch = (int64_t)(t._pitch / sizeof(float));
}
template<class T> void desc3(const T& t, table_desc d)
{
	d.shape[0] = t._width; d.shape[1] = t._height; d.shape[2] = t._depth;
	d.scale[0] = t._x_min; d.scale[1] = t._x_step; d.scale[2] = t._y_min; d.scale[3] = t._y_step;
	d.scale[4] = t._z_min; d.scale[5] = t._z_step;
	*d.data = t._data; *d.pitch = (int64_t)(t._pitch / sizeof(float));
}
}
}  // extern "C++"

static void table_info(ref_material* rm, int which, int32_t* shape, float* scale, const float** data, int64_t* pitch_floats)
{
	shape[0] = shape[1] = shape[2] = 1;
	for (int k = 0; k < 6; ++k) scale[k] = 0;
	*pitch_floats = 0;
	*data = nullptr;
	const table_desc d{ shape, scale, data, pitch_floats };
	if (which >= 6) {
		if (!rm->ki) throw std::runtime_error("no Kieft-Bosch tables");
		if (which == 6) desc1(rm->ki->_log_imfp_table, d);
		else if (which == 7) desc2(rm->ki->_log_icdf_table, d);
		else desc2(rm->ki->_ionisation_table, d);
		return;
	}
	if (!rm->def) {
		if (which > 1) throw std::runtime_error("no Full-Penn tables");
		// elastic tables of a Kieft-Bosch-only file
		static thread_local std::unique_ptr<nbl::scatter::kieft_elastic<false>> el;
		el.reset(new nbl::scatter::kieft_elastic<false>(nbl::scatter::kieft_elastic<false>::create(rm->file)));
		if (which == 0) desc1(el->_log_imfp_table, d); else desc2(el->_icdf_table, d);
		return;
	}
	auto& inel = nbl::tuple::get<0>(*rm->def);
	auto& el = nbl::tuple::get<1>(*rm->def);
	switch (which) {
	case 0: desc1(el._log_imfp_table, d); break;
	case 2: desc1(inel._log_imfp_table, d); break;
	case 1: desc2(el._icdf_table, d); break;
	case 3: desc2(inel._log_omega_icdf_table, d); break;
	case 4: desc3(inel._q_icdf_table, d); break;
	default: desc3(inel._ionisation_table, d); break;
	}
}

void ref_material_table_shape(void* h, int which, int32_t* shape, float* scale)
{
	const float* data; int64_t pitch;
	table_info(static_cast<ref_material*>(h), which, shape, scale, &data, &pitch);
}

/* Dense row-major copy of a table (rows are contiguous on the CPU). */
void ref_material_table_data(void* h, int which, float* out)
{
	int32_t shape[3]; float scale[6]; const float* data; int64_t pitch;
	table_info(static_cast<ref_material*>(h), which, shape, scale, &data, &pitch);
	std::memcpy(out, data, sizeof(float) * (size_t)shape[0] * shape[1] * shape[2]);
}

/* [fermi, band_gap, barrier, phonon_loss, recoil_const] */
void ref_material_constants(void* h, float* out)
{
	auto* rm = static_cast<ref_material*>(h);
	auto el = nbl::scatter::kieft_elastic<false>::create(rm->file);
	if (rm->def) {
		auto& inel = nbl::tuple::get<0>(*rm->def);
		out[0] = inel._fermi; out[1] = inel._band_gap;
	} else {
		out[0] = rm->ki->_fermi; out[1] = rm->ki->_band_gap;
	}
	out[2] = rm->barrier;
	out[3] = el._phonon_loss; out[4] = el._recoil_const;
	nbl::scatter::kieft_elastic<false>::destroy(el);
}

/* Table lookups through the reference table classes (get / get_rounddown). */
void ref_table_lookup(void* h, int which, int rounddown, int64_t n, const float* x, const float* y,
	const float* z, float* out)
{
	auto* rm = static_cast<ref_material*>(h);
	for (int64_t i = 0; i < n; ++i)
	{
		if (which >= 6) {
			auto& k = *rm->ki;
			if (which == 6) out[i] = k._log_imfp_table.get(x[i]);
			else if (which == 7) out[i] = rounddown ? k._log_icdf_table.get_rounddown(x[i], y[i]) : k._log_icdf_table.get(x[i], y[i]);
			else out[i] = rounddown ? k._ionisation_table.get_rounddown(x[i], y[i]) : k._ionisation_table.get(x[i], y[i]);
			continue;
		}
		auto& inel = nbl::tuple::get<0>(*rm->def);
		auto& el = nbl::tuple::get<1>(*rm->def);
		switch (which) {
		case 0: out[i] = el._log_imfp_table.get(x[i]); break;
		case 2: out[i] = inel._log_imfp_table.get(x[i]); break;
		case 1: out[i] = rounddown ? el._icdf_table.get_rounddown(x[i], y[i]) : el._icdf_table.get(x[i], y[i]); break;
		case 3: out[i] = rounddown ? inel._log_omega_icdf_table.get_rounddown(x[i], y[i]) : inel._log_omega_icdf_table.get(x[i], y[i]); break;
		case 4: out[i] = rounddown ? inel._q_icdf_table.get_rounddown(x[i], y[i], z[i]) : inel._q_icdf_table.get(x[i], y[i], z[i]); break;
		default: out[i] = rounddown ? inel._ionisation_table.get_rounddown(x[i], y[i], z[i]) : inel._ionisation_table.get(x[i], y[i], z[i]); break;
		}
	}
}

/* ------------------------------------------------------------------- events */
/* Physics bits (the oracle's numbering): 1 generate_secondary, 2
 * acoustic_phonon_loss, 4 atomic_recoil_loss, 8 quantum_transmission, 16
 * interface_refraction, 32 interface_absorption, 64 optical_phonon_loss, 128
 * instantaneous_momentum, 256 momentum_conservation, 65536 Kieft-Bosch
 * inelastic model.  Each bit selects the reference template argument of the
 * same name; one instantiation per combination. */
extern "C++" {
namespace {
template<class T, class PM>
void run_scatter(ref_material* rm, PM& pm, nbl::util::random_generator<false>& rng)
{
	T obj = T::create(rm->file);
	obj.execute(pm, 0, rng);
	T::destroy(obj);
}

template<class PM>
void elastic_dispatch(uint32_t b, ref_material* rm, PM& pm, nbl::util::random_generator<false>& rng)
{
	using namespace nbl::scatter;
	switch ((b >> 1) & 3) {
	case 0: run_scatter<kieft_elastic<false, false, false>>(rm, pm, rng); break;
	case 1: run_scatter<kieft_elastic<false, true, false>>(rm, pm, rng); break;
	case 2: run_scatter<kieft_elastic<false, false, true>>(rm, pm, rng); break;
	default: run_scatter<kieft_elastic<false, true, true>>(rm, pm, rng); break;
	}
}

template<bool gen, class PM>
void kieft_dispatch2(uint32_t b, ref_material* rm, PM& pm, nbl::util::random_generator<false>& rng)
{
	using namespace nbl::scatter;
	switch ((((b >> 6) & 1) << 2) | (((b >> 7) & 1) << 1) | ((b >> 8) & 1)) {
	case 0: run_scatter<kieft_inelastic<false, false, gen, false, false>>(rm, pm, rng); break;
	case 1: run_scatter<kieft_inelastic<false, false, gen, false, true>>(rm, pm, rng); break;
	case 2: run_scatter<kieft_inelastic<false, false, gen, true, false>>(rm, pm, rng); break;
	case 3: run_scatter<kieft_inelastic<false, false, gen, true, true>>(rm, pm, rng); break;
	case 4: run_scatter<kieft_inelastic<false, true, gen, false, false>>(rm, pm, rng); break;
	case 5: run_scatter<kieft_inelastic<false, true, gen, false, true>>(rm, pm, rng); break;
	case 6: run_scatter<kieft_inelastic<false, true, gen, true, false>>(rm, pm, rng); break;
	default: run_scatter<kieft_inelastic<false, true, gen, true, true>>(rm, pm, rng); break;
	}
}

template<class PM>
void inelastic_dispatch(uint32_t b, ref_material* rm, PM& pm, nbl::util::random_generator<false>& rng)
{
	using namespace nbl::scatter;
	if (b & 65536) {
		if (b & 1) kieft_dispatch2<true>(b, rm, pm, rng);
		else kieft_dispatch2<false>(b, rm, pm, rng);
	} else {
		if (b & 1) run_scatter<full_penn<false, true>>(rm, pm, rng);
		else run_scatter<full_penn<false, false>>(rm, pm, rng);
	}
}

template<class MM, class PM>
void boundary_dispatch(uint32_t b, MM& mm, PM& pm, nbl::util::random_generator<false>& rng)
{
	switch ((b >> 3) & 7) {
	case 0: { boundary_intersect<false, false, false> i; i.execute(mm, pm, 0, rng); break; }
	case 1: { boundary_intersect<true, false, false> i; i.execute(mm, pm, 0, rng); break; }
	case 2: { boundary_intersect<false, true, false> i; i.execute(mm, pm, 0, rng); break; }
	case 3: { boundary_intersect<true, true, false> i; i.execute(mm, pm, 0, rng); break; }
	case 4: { boundary_intersect<false, false, true> i; i.execute(mm, pm, 0, rng); break; }
	case 5: { boundary_intersect<true, false, true> i; i.execute(mm, pm, 0, rng); break; }
	case 6: { boundary_intersect<false, true, true> i; i.execute(mm, pm, 0, rng); break; }
	default: { boundary_intersect<true, true, true> i; i.execute(mm, pm, 0, rng); break; }
	}
}

// Material list for the managers: the boundary step only reads `barrier`, so
// a material made of the elastic model alone serves every file.
using bmat_phys = scatter_list<nbl::scatter::kieft_elastic<false>>;
using bdriver_t = nbl::drivers::simple_cpu_driver<bmat_phys, intersect_t, geometry_t>;
}
}  // extern "C++"

/* Electron in/out: [pos3, dir3, E] plus material index.
 * kind: 1 inelastic, 2 elastic (scatter_list order), 3 boundary crossing on
 * triangle `tri` of geometry `gh`.  The generator is the reference
 * random_generator<false> seeded with `seed`; `phys` selects the models and
 * options (bits above).
 * Returns the number of secondaries written to se_out (7 floats each) and sets
 * *status: 0 running, 1 detected, 2 terminated. */
int ref_event(void* gh, void** mats, int n_mat, uint32_t phys, int kind, int32_t tri, uint32_t seed,
	float* state, int32_t* material, float* se_out, int max_se, int32_t* status)
{
	std::vector<::material<bmat_phys>> materials;
	for (int i = 0; i < n_mat; ++i)
		materials.emplace_back(static_cast<ref_material*>(mats[i])->file);
	using pm_t = bdriver_t::particle_manager_t;
	using mm_t = bdriver_t::material_manager_t;
	pm_t pm = pm_t::create();
	mm_t mm = mm_t::create(materials);
	particle p{ { state[0], state[1], state[2] }, { state[3], state[4], state[5] }, state[6] };
	uint32_t tag = 0;
	pm.push(&p, &tag, 1);
	pm.set_material_index(0, *material);
	nbl::util::random_generator<false> rng(seed);
	if (kind == 3)
	{
		auto* g = static_cast<ref_geometry*>(gh);
		pm.particles[0].last_triangle = g->oct._triangles + tri;
		pm.particles[0].status = pm_t::INTERSECT_EVENT;
		boundary_dispatch(phys, mm, pm, rng);
	}
	else
	{
		auto* rm = static_cast<ref_material*>(mats[*material]);
		if (kind == 1) inelastic_dispatch(phys, rm, pm, rng);
		else elastic_dispatch(phys, rm, pm, rng);
	}
	particle q = pm[0];
	state[0] = q.pos.x; state[1] = q.pos.y; state[2] = q.pos.z;
	state[3] = q.dir.x; state[4] = q.dir.y; state[5] = q.dir.z; state[6] = q.kin_energy;
	*material = pm.get_material_index(0);
	*status = pm.particles[0].status == pm_t::DETECTED ? 1 : (pm.particles[0].status == pm_t::TERMINATED ? 2 : 0);
	int n_se = 0;
	for (size_t i = 1; i < pm.particles.size() && n_se < max_se; ++i, ++n_se)
	{
		particle s = pm.particles[i].particle_data;
		float* o = se_out + 7 * n_se;
		o[0] = s.pos.x; o[1] = s.pos.y; o[2] = s.pos.z;
		o[3] = s.dir.x; o[4] = s.dir.y; o[5] = s.dir.z; o[6] = s.kin_energy;
	}
	mm_t::destroy(mm);
	pm_t::destroy(pm);
	return n_se;
}

/* --------------------------------------------------------------- simulation */
/* Single-threaded sim_loop of cpu_mt_main.cpp:167-201 with one driver seeded
 * with `seed`: for each primary push it, run simulate_to_end
 * (drivers/cpu/simple_cpu_driver.h:53-65) counting init() calls (= events),
 * and flush detected electrons as 36-byte records (pixel = the primary's).
 * Returns the number of records (capped at max_records; *n_total gets the
 * uncapped count). */
extern "C++" {
namespace {
template<class Phys, class Isect>
int64_t simulate_impl(void* gh, void** mats, int n_mat, const void* pri_records, int64_t n_pri,
	uint32_t seed, float energy_threshold, void* out_records, int64_t max_records,
	int64_t* n_total, int64_t* n_events)
{
	using drv_t = nbl::drivers::simple_cpu_driver<Phys, Isect, geometry_t>;
	auto* g = static_cast<ref_geometry*>(gh);
	std::vector<material<Phys>> materials;
	for (int i = 0; i < n_mat; ++i)
		materials.emplace_back(static_cast<ref_material*>(mats[i])->file);
	Isect inter;
	drv_t d(g->oct, inter, materials, energy_threshold, seed);
	int64_t written = 0, total = 0, events = 0;
	const char* in = static_cast<const char*>(pri_records);
	char* out = static_cast<char*>(out_records);
	for (int64_t i = 0; i < n_pri; ++i)
	{
		float f[7]; int32_t px[2];
		std::memcpy(f, in + 36 * i, 28);
		std::memcpy(px, in + 36 * i + 28, 8);
		particle p{ { f[0], f[1], f[2] }, { f[3], f[4], f[5] }, f[6] };
		uint32_t tag = 0;
		d.push(&p, &tag, 1);
		for (size_t idx = 0; idx < d._particles.get_total_count(); ++idx)
		{
			while (d._particles.active(idx))
			{
				d.init(idx);
				d.intersect(idx);
				d.scatter(idx);
				++events;
			}
		}
		d.flush_detected([&](particle q, uint32_t) {
			if (written < max_records)
			{
				float r[7] = { q.pos.x, q.pos.y, q.pos.z, q.dir.x, q.dir.y, q.dir.z, q.kin_energy };
				std::memcpy(out + 36 * written, r, 28);
				std::memcpy(out + 36 * written + 28, px, 8);
				++written;
			}
			++total;
		});
	}
	*n_total = total;
	*n_events = events;
	return written;
}
}
}  // extern "C++"

/* Physics presets with a compiled driver (bits as for ref_event):
 *   0x1DF      the reference's selection (physics_config.h)
 *   0x101DF    Kieft-Bosch inelastic, every option on
 *   0x1E1      Full Penn; no phonon or recoil loss; classical transmission,
 *              no refraction, empirical absorption
 *   0x1001F    Kieft-Bosch without optical-phonon loss, instantaneous
 *              momentum or momentum conservation
 * Any other value returns -1. */
int64_t ref_simulate(void* gh, void** mats, int n_mat, uint32_t phys, const void* pri_records, int64_t n_pri,
	uint32_t seed, float energy_threshold, void* out_records, int64_t max_records,
	int64_t* n_total, int64_t* n_events)
{
	using namespace nbl::scatter;
	switch (phys) {
	case 0x1DF:
		return simulate_impl<scatter_physics<false>, intersect_t>(gh, mats, n_mat, pri_records, n_pri, seed,
			energy_threshold, out_records, max_records, n_total, n_events);
	case 0x101DF:
		return simulate_impl<scatter_list<kieft_inelastic<false, true, true, true, true>, kieft_elastic<false, true, true>>,
			intersect_t>(gh, mats, n_mat, pri_records, n_pri, seed, energy_threshold, out_records, max_records,
			n_total, n_events);
	case 0x1E1:
		return simulate_impl<scatter_list<full_penn<false, true>, kieft_elastic<false, false, false>>,
			boundary_intersect<false, false, true>>(gh, mats, n_mat, pri_records, n_pri, seed, energy_threshold,
			out_records, max_records, n_total, n_events);
	case 0x1001F:
		return simulate_impl<scatter_list<kieft_inelastic<false, false, true, false, false>, kieft_elastic<false, true, true>>,
			intersect_t>(gh, mats, n_mat, pri_records, n_pri, seed, energy_threshold, out_records, max_records,
			n_total, n_events);
	default:
		g_err = "physics preset not compiled in the harness";
		return -1;
	}
}

/* ref_simulate with the driver's generator reseeded for every primary
 * (seed = base_seed + index), so each primary's cascade has its own mt19937
 * stream: runs of the same primaries with slightly different material
 * parameters then share random numbers primary by primary (common random
 * numbers for finite differences).  Default physics.  Writes the detected
 * records; returns how many. */
int64_t ref_simulate_reseeded(void* gh, void** mats, int n_mat, const void* pri_records, int64_t n_pri,
	uint32_t base_seed, float energy_threshold, void* out_records, int64_t max_records, int64_t* n_total)
{
	auto* g = static_cast<ref_geometry*>(gh);
	std::vector<material_t> materials;
	for (int i = 0; i < n_mat; ++i)
		materials.emplace_back(static_cast<ref_material*>(mats[i])->file);
	intersect_t inter;
	driver_t d(g->oct, inter, materials, energy_threshold, base_seed);
	int64_t written = 0, total = 0;
	const char* in = static_cast<const char*>(pri_records);
	char* out = static_cast<char*>(out_records);
	for (int64_t i = 0; i < n_pri; ++i)
	{
		d.rand_state = nbl::util::random_generator<false>((uint32_t)(base_seed + (uint32_t)i));
		float f[7]; int32_t px[2];
		std::memcpy(f, in + 36 * i, 28);
		std::memcpy(px, in + 36 * i + 28, 8);
		particle p{ { f[0], f[1], f[2] }, { f[3], f[4], f[5] }, f[6] };
		uint32_t tag = 0;
		d.push(&p, &tag, 1);
		d.simulate_to_end();
		d.flush_detected([&](particle q, uint32_t) {
			if (written < max_records)
			{
				float r[7] = { q.pos.x, q.pos.y, q.pos.z, q.dir.x, q.dir.y, q.dir.z, q.kin_energy };
				std::memcpy(out + 36 * written, r, 28);
				std::memcpy(out + 36 * written + 28, px, 8);
				++written;
			}
			++total;
		});
	}
	*n_total = total;
	return written;
}

/* The reference's energy-deposit driver (energydeposit_cpu_driver.h:44-93),
 * default physics, one driver seeded with `seed`, primaries one at a time as
 * cpu_energydep.cpp:170-205 does on one thread; writes its 28-byte deposit
 * records (after.pos, before.kin_energy, before - after, pixel).  Returns
 * records written; *n_total all of them. */
int64_t ref_simulate_deposits(void* gh, void** mats, int n_mat, const void* pri_records, int64_t n_pri,
	uint32_t seed, float energy_threshold, void* out_records, int64_t max_records, int64_t* n_total)
{
	using dep_driver_t = nbl::drivers::energydeposit_cpu_driver<scatter_physics<false>, intersect_t, geometry_t>;
	auto* g = static_cast<ref_geometry*>(gh);
	std::vector<material_t> materials;
	for (int i = 0; i < n_mat; ++i)
		materials.emplace_back(static_cast<ref_material*>(mats[i])->file);
	intersect_t inter;
	dep_driver_t d(g->oct, inter, materials, energy_threshold, seed);
	int64_t written = 0, total = 0;
	const char* in = static_cast<const char*>(pri_records);
	char* out = static_cast<char*>(out_records);
	for (int64_t i = 0; i < n_pri; ++i)
	{
		float f[7]; int32_t px[2];
		std::memcpy(f, in + 36 * i, 28);
		std::memcpy(px, in + 36 * i + 28, 8);
		particle p{ { f[0], f[1], f[2] }, { f[3], f[4], f[5] }, f[6] };
		uint32_t tag = 0;
		d.push(&p, &tag, 1);
		d.simulate_to_end([&](particle const & before, particle const & after, uint32_t) {
			if (written < max_records)
			{
				const float r[5] = { after.pos.x, after.pos.y, after.pos.z,
					before.kin_energy, before.kin_energy - after.kin_energy };
				std::memcpy(out + 28 * written, r, 20);
				std::memcpy(out + 28 * written + 20, px, 8);
				++written;
			}
			++total;
		});
		d.flush_detected([](particle, uint32_t) {});
	}
	*n_total = total;
	return written;
}

} // extern "C"
