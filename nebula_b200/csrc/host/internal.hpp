// Host-side internals shared by the C-ABI implementation files.
#pragma once
#include <string>
#include <vector>
#include <map>
#include <stdexcept>
#include <cstdint>
#include "nebula_b200.h"

namespace nbl {

// Error carried to the C ABI as a status code plus message.
struct Error : std::runtime_error {
	nbl_status code;
	Error(nbl_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& m);

// Run `f`, mapping exceptions to status codes.
template<class F> nbl_status guard(F&& f)
{
	try {
		f();
		return NBL_OK;
	} catch (const Error& e) {
		set_last_error(e.what());
		return e.code;
	} catch (const std::bad_alloc&) {
		set_last_error("out of host memory");
		return NBL_ERR_OOM;
	} catch (const std::exception& e) {
		set_last_error(e.what());
		return NBL_ERR_INVALID_ARG;
	}
}

inline void require(bool cond, const std::string& msg, nbl_status code = NBL_ERR_INVALID_ARG)
{
	if (!cond)
		throw Error(code, msg);
}

// A table in the transformed domain, owning its data.
struct HostTable {
	int32_t nx = 1, ny = 1, nz = 1;
	float x_min = 0, x_step = 0, y_min = 0, y_step = 0, z_min = 0, z_step = 0;
	std::vector<float> data;
	nbl_table view() const
	{
		nbl_table t;
		t.nx = nx; t.ny = ny; t.nz = nz;
		t.x_min = x_min; t.x_step = x_step; t.y_min = y_min; t.y_step = y_step; t.z_min = z_min; t.z_step = z_step;
		t.data = data.data();
		return t;
	}
};

// Material (core/material.h:19-46): the scatter-model tables and constants.
// Full-Penn tables (in_*) and Kieft-Bosch inelastic tables (ki_*) are each
// present when `models` has bit 0 / bit 1 set.
struct HostMaterial {
	HostTable el_imfp, el_icdf, in_imfp, in_omega, in_q, in_binding;
	float fermi = 0, band_gap = -1, barrier = 0, phonon_loss = 0, recoil_const = 0;
	int32_t models = 0;
	HostTable ki_imfp, ki_w0, ki_binding;
};

// The inelastic tables a run of the selected model reads, in the order of
// DevMaterial's in_imfp, in_omega, in_q, in_binding (the Kieft-Bosch model
// reads no q table: a one-point placeholder stands in).
struct InelasticTables { const HostTable *imfp, *omega, *q, *binding; };
inline InelasticTables inelastic_tables(const HostMaterial& m, bool kieft)
{
	static const HostTable unused = [] { HostTable t; t.data.assign(1, 0.0f); return t; }();
	if (kieft) {
		require(m.models & 2, "material has no Kieft-Bosch inelastic tables");
		return { &m.ki_imfp, &m.ki_w0, &unused, &m.ki_binding };
	}
	require(m.models & 1, "material has no Full-Penn inelastic tables");
	return { &m.in_imfp, &m.in_omega, &m.in_q, &m.in_binding };
}

// nbl_physics_opts -> PH_* bits; every option must be 0 or 1.
uint32_t physics_bits(const nbl_physics_opts& o);

HostMaterial load_material_file(const std::string& path);

// Linearised octree (octree_builder.h:209-248), triangles in its order.
struct HostGeometry {
	std::vector<int32_t> octree;
	std::vector<nbl_triangle> tris;
	float center[3] = { 0, 0, 0 }, halfsize[3] = { 0, 0, 0 };
	float max_extent = 0;
};

HostGeometry build_octree(const nbl_triangle* tris, int64_t n, int max_depth, int split_count);
float max_extent_of(const float halfsize[3]);

}  // namespace nbl

struct nbl_material { nbl::HostMaterial m; };

struct nbl_geometry {
	nbl::HostGeometry g;
	// device copies per device ordinal (ray queries)
	struct Dev { void* octree = nullptr; void* tris = nullptr; };
	mutable std::map<int, Dev> dev;
};
