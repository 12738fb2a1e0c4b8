// Device-side data layouts shared by the CUDA kernels and the host code that
// uploads them.  Plain structs only (no CUDA types), so host .cpp files can
// include this header.
#pragma once
#include <stdint.h>

namespace nbl {

// Special material ids (reference core/material_manager.h:77-86).
enum : int32_t {
	MAT_NOP = -128, MAT_TERMINATOR = -127, MAT_DETECTOR = -126, MAT_DETECTOR_LT50 = -125,
	MAT_DETECTOR_GE50 = -124, MAT_VACUUM = -123, MAT_MIRROR = -122
};

// Philox4x32-10 key (the run seed).
struct PhiloxKey { uint32_t k0, k1; };

// Event kinds.  The queue order is the order events are laid out in the
// per-iteration index space of the transport kernel.  EV_NEW holds electrons
// whose next action is a free flight (new secondaries; in split iterations
// also electrons after their interaction); EV_WALK flights whose octree walk
// stopped at the per-iteration cell budget and continues.
enum : int32_t { EV_BOUNDARY = 0, EV_ELASTIC = 1, EV_INELASTIC = 2, EV_NEW = 3, EV_WALK = 4, N_QUEUES = 5 };

// One triangle, 64 bytes, four 16-byte vectors so a warp fetches it with
// 128-bit loads: (r0, material_in) (e1, material_out) (e2, 0) (normal, 0).
// r0/e1/e2 are the reference triangle's members (core/triangle.h:70-76);
// normal = cross(e1, e2) computed once in float on the host with the same
// operations as triangle::get_normal (core/triangle.inl:75-78), so it is the
// value the reference recomputes per test.
struct DevTriangle {
	float r0x, r0y, r0z; int32_t mat_in;
	float e1x, e1y, e1z; int32_t mat_out;
	float e2x, e2y, e2z; int32_t pad0;
	float nx, ny, nz; int32_t pad1;
};
static_assert(sizeof(DevTriangle) == 64, "DevTriangle must be 64 bytes");

struct DevGeometry {
	const int32_t* octree;       // reference linearized layout (octree_builder.h:222-231)
	const DevTriangle* tris;
	float cx, cy, cz;            // root AABB centre
	float hx, hy, hz;            // root AABB half size
	float max_extent;            // 2 |halfsize| as the reference computes it
	int32_t n_tri;
	int64_t n_octree;
};

// A table in the reference's transformed domain: row-major data, index per
// axis = (v - v_min) * v_step (common/util/table_{1,2,3}D).
struct DevTable {
	const float* data;
	int32_t nx, ny, nz, pad;
	float x_min, x_step, y_min, y_step, z_min, z_step;
};

// Physics selection (physics_config.h:20-46 and the option bools of the
// models it names), one bit per option, read by every event.
enum : uint32_t {
	PH_GEN_SE = 1u << 0,        // full_penn / kieft_inelastic generate_secondary
	PH_PHONON = 1u << 1,        // kieft_elastic acoustic_phonon_loss
	PH_RECOIL = 1u << 2,        // kieft_elastic atomic_recoil_loss
	PH_QT = 1u << 3,            // boundary_intersect quantum_transmission
	PH_REFRACT = 1u << 4,       // boundary_intersect interface_refraction
	PH_ABSORB = 1u << 5,        // boundary_intersect interface_absorption
	PH_OPT_PHONON = 1u << 6,    // kieft_inelastic optical_phonon_loss
	PH_INST_MOM = 1u << 7,      // kieft_inelastic instantaneous_momentum
	PH_MOM_CONS = 1u << 8,      // kieft_inelastic momentum_conservation
	PH_KIEFT = 1u << 16,        // inelastic model: kieft_inelastic instead of full_penn
	PH_DEFAULT = PH_GEN_SE | PH_PHONON | PH_RECOIL | PH_QT | PH_REFRACT | PH_OPT_PHONON | PH_INST_MOM | PH_MOM_CONS,
};

// Inelastic tables by model: Full Penn uses in_imfp, in_omega (log omega
// ICDF), in_q and in_binding (3-D); Kieft-Bosch uses in_imfp, in_omega (log
// omega' ICDF) and in_binding (2-D), in_q unused.
struct DevMaterial {
	DevTable el_imfp, el_icdf, in_imfp, in_omega, in_q, in_binding;
	float fermi, band_gap, barrier, phonon_loss, recoil_const;
	// adjoint parameters: multiplicative scales on the inelastic / elastic
	// inverse mean free paths (1 = the tables as given)
	float in_scale, el_scale, pad;
};

// 36-byte primary / detected-electron record (reference .pri layout,
// io/load_pri_file.cpp:112-121; output gpu_main.cu:216-223).
struct Record36 {
	float x, y, z, dx, dy, dz, E;
	int32_t px, py;
};
static_assert(sizeof(Record36) == 36, "Record36 must be 36 bytes");

// 28-byte energy-deposit record of a scatter event (cpu_energydep.cpp:197-204):
// position, kinetic energy before the event, energy lost, pixel.
struct DepositRecord {
	float x, y, z, E, dE;
	int32_t px, py;
};
static_assert(sizeof(DepositRecord) == 28, "DepositRecord must be 28 bytes");

}  // namespace nbl
