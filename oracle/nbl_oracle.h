/*
 * Test infrastructure (oracle), not product code: a CPU restatement of the
 * reference's electron-transport path, used only by tests/, smoke() and
 * bench.py's CPU baseline, as the model results are compared against.
 * Nothing in nebula_b200/ links it.
 *
 * It restates, operation by operation and in float32 like the reference's
 * CPU build (config/config.h:13), the functions its CPU driver runs:
 * table lookups, Moller-Trumbore intersection, the octree walk, Kieft-Bosch
 * elastic, Full-Penn and Kieft-Bosch inelastic and boundary crossing, with
 * the option bools of each, and the simple CPU driver loop.  With the reference mt19937 generator it reproduces the
 * reference's detected-electron records bit for bit (checked in
 * tests/test_oracle_pin.py against oracle/_ref built from the reference).
 */
#ifndef NBL_ORACLE_H
#define NBL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Table in the transformed domain the reference keeps after create():
 * row-major data[nx][ny][nz], index = (v - v_min) * v_step per axis. */
typedef struct orc_table {
	int32_t nx, ny, nz;
	float x_min, x_step, y_min, y_step, z_min, z_step;
	const float* data;
} orc_table;

/* models: bit 0 Full-Penn tables (in_*) present, bit 1 Kieft-Bosch tables
 * (ki_*: imfp 1-D, w0 ICDF 2-D, binding 2-D) present. */
typedef struct orc_material {
	orc_table el_imfp, el_icdf, in_imfp, in_omega, in_q, in_binding;
	float fermi, band_gap, barrier, phonon_loss, recoil_const;
	int32_t models;
	orc_table ki_imfp, ki_w0, ki_binding;
} orc_material;

/* Physics selection (physics_config.h:20-46 and the option bools of the
 * models), one bit per option, for every later event and run:
 *   1 generate_secondary   2 acoustic_phonon_loss   4 atomic_recoil_loss
 *   8 quantum_transmission 16 interface_refraction  32 interface_absorption
 *   64 optical_phonon_loss 128 instantaneous_momentum 256 momentum_conservation
 *   65536 Kieft-Bosch inelastic model instead of Full Penn.
 * Default 1|2|4|8|16|64|128|256 (the reference's selection). */
void orc_set_physics(uint32_t bits);
uint32_t orc_get_physics(void);

/* Linearized octree as octree_builder.h:209-248 lays it out; triangles as
 * 11 floats (material_in, material_out, r0, e1, e2). */
typedef struct orc_geometry {
	const int32_t* octree_data;
	int64_t n_octree;
	const float* tri11;
	int64_t n_tri;
	float center[3], halfsize[3], max_extent;
} orc_geometry;

/* Load a .nmat material file and apply the reference's create() transforms.
 * Returns an owning handle (nullptr on error, message in err). */
void* orc_material_load(const char* path, char* err, int errlen);
const orc_material* orc_material_view(void* handle);
void orc_material_free(void* handle);

/* Table lookups: which 0 el_imfp 1 el_icdf 2 in_imfp 3 in_omega 4 in_q 5 in_binding */
float orc_table_get(const orc_table* t, int dims, float x, float y, float z);
float orc_table_rounddown(const orc_table* t, int dims, float x, float y, float z);

/* One octree walk (octree.inl:33-192).  ignore_tri < 0: none. */
void orc_propagate(const orc_geometry* g, const float* pos, const float* dir, float dist,
	int32_t ignore_tri, int32_t ignore_mat, float* out_dist, int32_t* out_tri);

/* Uniform source: mt19937 (reference CPU generator) or a caller list. */
typedef struct orc_rng orc_rng;
orc_rng* orc_rng_mt(uint32_t seed);
orc_rng* orc_rng_list(const float* u, int64_t n);
int64_t orc_rng_used(const orc_rng* r);
void orc_rng_free(orc_rng* r);
float orc_rng_unit(orc_rng* r);

/* One event on one electron (state: pos3, dir3, E; material).  kind 1
 * inelastic, 2 elastic, 3 boundary on triangle `tri`.  Returns the number of
 * secondaries (0/1) written to se (7 floats); *status 0 running, 1 detected,
 * 2 terminated. */
int orc_event(const orc_geometry* g, const orc_material* mats, int n_mat, int kind, int32_t tri,
	orc_rng* rng, float* state, int32_t* material, float* se, int32_t* status);

/* Single-threaded run of the reference CPU driver loop on 36-byte primary
 * records.  Returns records written (36 B each); *n_total counts all
 * detected electrons, *n_events the driver iterations. */
int64_t orc_simulate(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events);

/* Same loop over `n_threads` threads pulling one primary at a time, the
 * mt19937 reseeded for every primary from (seed, primary index), so the set
 * of records depends on neither the thread count nor the scheduling (the
 * reference's cpu_mt_main.cpp:79,210 gives each thread one stream instead,
 * which makes its runs irreproducible).  Output order is not deterministic.
 * Returns records written. */
int64_t orc_simulate_mt(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold, int n_threads,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events);

/* The energy-deposit driver loop (energydeposit_cpu_driver.h:44-93) over
 * `n_threads` threads (1: the primaries in order with mt19937(seed), as the
 * reference run on one thread; more: reseeded per primary as orc_simulate_mt).
 * Writes 28-byte deposit records (after.pos, before.E, before.E - after.E,
 * pixel) for every scatter event that changed the energy; returns records
 * written, *n_total all of them. */
int64_t orc_simulate_deposits(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold, int n_threads,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events);

#ifdef __cplusplus
}
#endif
#endif
