// Scatter and boundary physics for one electron, templated on the uniform
// source (Philox stream in production, a fixed list in known-answer tests).
//
// Each function restates the reference's model with its float operation
// order and its random-draw order, so that given the same uniforms the GPU
// and the reference CPU build differ only by the last-ulp differences of the
// transcendental functions (logf, expf, sinf/cosf, atan2f, cbrtf):
//   * kieft_elastic<gpu,phonon,recoil>::execute    (physics/kieft/elastic.h:67-115)
//   * full_penn<gpu,gen_se>::execute               (physics/full_penn.h:62-288)
//   * kieft_inelastic<gpu,opl,gen_se,im,mc>::execute (physics/kieft/inelastic.h:63-209)
//   * boundary_intersect<qt,refraction,absorption>::execute (physics/boundary_intersect.h:38-155)
//   with the option bools taken from a run-time word of PH_* bits.
//   * free-path sampling: scatter_list::sample_path visits the processes with
//     tuple::for_each, which runs last-to-first (core/scatter_list.h:101-107,
//     common/tuple.h:113-118), so the elastic path is drawn before the
//     inelastic one and a tie goes to elastic.
//   * random_generator::uniform_vector draws the azimuth before the polar
//     cosine (its call arguments are evaluated right to left by the
//     reference's g++ build; common/util/random.h:72-76).
// Directions are carried unnormalised, as the reference CPU driver stores
// them, and normalised (sqrt, then multiply by the reciprocal) where used
// (common/vector_math.h:141-158).
//
// Transcendentals use the SFU forms (__logf, __expf, __sincosf; relative
// errors ~1e-6 for the arguments met here: log of energies and of uniforms,
// exp of log inverse mean free paths, angles in [-pi, 2 pi]), and divisions
// the fast hardware quotient.  The sampled
// distributions are unchanged at that level; the octree walk and the table
// lookups, which must match the reference bit for bit, use none of them.
#pragma once
#include "../nbl_device_types.h"
#include "geometry.cuh"
#include "tables.cuh"

namespace nbl {

// Division in the physics: the fast hardware quotient (within 2 ulp).  The
// physics is compared with the reference statistically and per event to
// 1e-4; the octree walk and the table lookups keep IEEE division.
__device__ __forceinline__ float fdf(float a, float b) { return __fdividef(a, b); }

#define NBL_PI 3.1415926535897932f

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return v3(fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return v3(fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)); }
__device__ __forceinline__ V3 vmul(V3 a, float b) { return v3(fm(a.x, b), fm(a.y, b), fm(a.z, b)); }
__device__ __forceinline__ V3 smul(float a, V3 b) { return v3(fm(a, b.x), fm(a, b.y), fm(a, b.z)); }
__device__ __forceinline__ V3 vcross(V3 a, V3 b)
{
	return v3(fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x)));
}
__device__ __forceinline__ float vdot(V3 a, V3 b) { return dot3(a.x, a.y, a.z, b.x, b.y, b.z); }
__device__ __forceinline__ float vmag2(V3 a) { return dot3(a.x, a.y, a.z, a.x, a.y, a.z); }
__device__ __forceinline__ V3 vnormalised(V3 a)
{
	const float s = __fsqrt_rn(vmag2(a));
	return vmul(a, fdf(1.0f, s));
}
__device__ __forceinline__ float clampf(float i, float lo, float hi) { return i < lo ? lo : (i > hi ? hi : i); }
// std::min / std::max argument semantics
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct Electron {
	V3 pos, dir;
	float E;
};

template<class R> __device__ __forceinline__ float draw_phi(R& rng) { return fm(2.0f * NBL_PI, rng.unit()); }

// make_unit_vec (vector_math.h:194-206)
__device__ __forceinline__ V3 make_unit_vec(float cos_theta, float phi)
{
	float sp, cp;
	__sincosf(phi, &sp, &cp);
	cos_theta = clampf(cos_theta, -1.0f, 1.0f);
	const float st = __fsqrt_rn(fs(1.0f, fm(cos_theta, cos_theta)));
	return v3(fm(st, cp), fm(st, sp), cos_theta);
}
template<class R> __device__ __forceinline__ V3 uniform_vector(R& rng)
{
	const float phi = draw_phi(rng);
	const float ct = fs(fm(2.0f, rng.unit()), 1.0f);
	return make_unit_vec(ct, phi);
}
// make_normal_vec (vector_math.h:171-186)
__device__ __forceinline__ V3 make_normal_vec(V3 dir, float phi)
{
	float sa, ca;
	__sincosf(atan2f(dir.y, dir.x), &sa, &ca);
	const V3 unit_v = v3(fm(dir.z, ca), fm(dir.z, sa), -__fsqrt_rn(fa(fm(dir.x, dir.x), fm(dir.y, dir.y))));
	const V3 unit_u = vcross(unit_v, dir);
	float sp, cp;
	__sincosf(phi, &sp, &cp);
	return vadd(vmul(unit_u, cp), vmul(unit_v, sp));
}

// Inverse mean free path scale * exp(table(log E)).
__device__ __forceinline__ float imfp_at(const DevTable& imfp_tab, float scale, float E)
{
	return fm(scale, __expf(table1_get(imfp_tab, __logf(E))));
}

// One exponential free path: -tau * log(U), tau = 1 / (scale * exp(table(log E)))
template<class R> __device__ __forceinline__ float sample_path(const DevTable& imfp_tab, float scale, float E, R& rng, float& mu)
{
	mu = imfp_at(imfp_tab, scale, E);
	const float tau = fdf(1.0f, mu);
	return fm(-tau, __logf(rng.unit()));
}

// Elastic event (elastic.h:67-115), acoustic-phonon and atomic-recoil loss
// as selected.
template<class R> __device__ __forceinline__ void elastic_event(const DevMaterial& m, Electron& p, R& rng,
	uint32_t ph = PH_DEFAULT)
{
	const float x = __logf(p.E);
	const float y = rng.unit();
	const float cos_theta = clampf(table2_get(m.el_icdf, x, y), -1.0f, 1.0f);
	const float sin_theta = __fsqrt_rn(fs(1.0f, fm(cos_theta, cos_theta)));
	p.dir = vnormalised(p.dir);
	const V3 normal_dir = vnormalised(make_normal_vec(p.dir, draw_phi(rng)));
	p.dir = vadd(vmul(p.dir, cos_theta), vmul(normal_dir, sin_theta));
	if (p.E < 200.0f) {
		if (ph & PH_PHONON)
			p.E = fs(p.E, smin(50e-3f, m.phonon_loss));
	} else if (ph & PH_RECOIL) {
		p.E = fs(p.E, fm(fm(m.recoil_const, fs(1.0f, cos_theta)), p.E));
	}
}

// Inelastic event (full_penn.h:62-288).  Returns true and fills `se` when a
// secondary electron is created.  The plasmon-decay rejection loop is capped
// at 64 trials (the last trial is kept); the reference loop is unbounded but
// its acceptance rate is above one half.
template<class R> __device__ __forceinline__ bool penn_event(const DevMaterial& m, Electron& p, Electron& se, R& rng,
	uint32_t ph)
{
	float omega;
	{
		const float x = __logf(p.E);
		const float y = rng.unit();
		omega = __expf(table2_get(m.in_omega, x, y));
	}
	float binding;
	{
		const float x = __logf(p.E);
		const float y = __logf(fdf(omega, p.E));
		const float z = rng.unit();
		binding = table3_rounddown(m.in_binding, x, y, z);
	}
	p.dir = vnormalised(p.dir);
	if (binding <= 0.0f) {
		if (omega > m.band_gap) {
			float q;
			{
				const float x = __logf(p.E);
				const float y = fdf(omega, p.E);
				const float z = rng.unit();
				q = table3_get(m.in_q, x, y, z);
			}
			const V3 prim_normal_dir = vnormalised(make_normal_vec(p.dir, draw_phi(rng)));
			V3 q_dir, q_normal_dir;
			{
				const float c = clampf(fdf(fa(omega, fm(q, q)), fm(fm(2.0f, __fsqrt_rn(p.E)), q)), -1.0f, 1.0f);
				const float s = __fsqrt_rn(fs(1.0f, fm(c, c)));
				q_dir = vnormalised(vadd(vmul(p.dir, c), vmul(prim_normal_dir, s)));
				q_normal_dir = vnormalised(make_normal_vec(q_dir, draw_phi(rng)));
			}
			const float c2 = clampf(fdf(fs(fs(fm(2.0f, p.E), omega), fm(q, q)),
				fm(2.0f, __fsqrt_rn(fm(p.E, fs(p.E, omega))))), -1.0f, 1.0f);
			const float s2 = __fsqrt_rn(fs(1.0f, fm(c2, c2)));
			p.E = fs(p.E, omega);
			p.dir = vadd(vmul(p.dir, c2), vmul(prim_normal_dir, s2));
			if (!(ph & PH_GEN_SE))
				return false;

			se.pos = p.pos;
			const float k_fermi = __fsqrt_rn(m.fermi);
			const float k_fermi_omega = __fsqrt_rn(fa(m.fermi, omega));
			if (q < fs(k_fermi_omega, k_fermi)) {
				// plasmon decay
				const float f = fdf(m.fermi, omega);
				float x;
				if (f < 0.1f) {
					const float U = cbrtf(rng.unit());
					x = fm(fm(f, U), U);
				} else {
					const float lower = smax(0.0f, fs(f, 1.0f));
					const float upper = f;
					const float d1 = fs(upper, lower);
					const float d2 = fs(fm(upper, upper), fm(lower, lower));
					const float alpha = fdf(d2, fa(d1, d2));
					int trial = 0;
					for (;;) {
						const float U1 = rng.unit();
						const float U2 = rng.unit();
						x = (U1 < alpha) ? __fsqrt_rn(fa(fm(d2, U2), fm(lower, lower))) : fa(fm(d1, U2), lower);
						const float acc = fdf(__fsqrt_rn(fa(fm(x, x), x)), fa(x, 0.5f));
						if (!(rng.unit() > acc) || ++trial >= 64)
							break;
					}
				}
				se.E = fa(fm(x, omega), omega);
				se.dir = uniform_vector(rng);
			} else if (q < fa(k_fermi_omega, k_fermi)) {
				// single excitation from the Fermi sphere
				const float ki_parr = fdf(fs(omega, fm(q, q)), fm(2.0f, q));
				const float kf_parr = fa(ki_parr, q);
				const float ki_perp_min_sq = smax(0.0f, fs(m.fermi, fm(kf_parr, kf_parr)));
				const float ki_perp_max_sq = fs(m.fermi, fm(ki_parr, ki_parr));
				const float ki_perp_sq = smax(0.0f, fa(ki_perp_min_sq, fm(fs(ki_perp_max_sq, ki_perp_min_sq), rng.unit())));
				const V3 ki = vadd(smul(ki_parr, q_dir), smul(__fsqrt_rn(ki_perp_sq), q_normal_dir));
				se.E = fa(vmag2(ki), omega);
				se.dir = vadd(ki, smul(q, q_dir));
			} else {
				return false;
			}
			return true;
		} else {
			p.E = fs(p.E, omega);
			return false;
		}
	}
	// inner-shell ionisation (Ivanchenko angles)
	const V3 normal_dir = vnormalised(make_normal_vec(p.dir, draw_phi(rng)));
	const float K = fa(fs(p.E, m.fermi), fm(2.0f, binding));
	const float dK = fa(binding, omega);
	const float cos_theta = __fsqrt_rn(fdf(dK, K));
	const float sin_theta = __fsqrt_rn(fs(1.0f, clampf(fm(cos_theta, cos_theta), 0.0f, 1.0f)));
	V3 sdir = vadd(vmul(p.dir, cos_theta), vmul(normal_dir, sin_theta));
	sdir = vnormalised(sdir);
	sdir = vadd(sdir, smul(__fsqrt_rn(fdf(binding, dK)), uniform_vector(rng)));
	sdir = vnormalised(sdir);
	se.E = fs(fa(m.fermi, omega), binding);
	se.pos = p.pos;
	se.dir = sdir;
	p.E = fs(p.E, omega);
	p.dir = vsub(p.dir, smul(cos_theta, sdir));
	return (ph & PH_GEN_SE) != 0;
}

// Kieft-Bosch inelastic event (kieft/inelastic.h:63-209): zero-momentum loss
// omega' from its ICDF, a binding energy from the ionisation ICDF (rounddown),
// the total loss omega from Ashley's distribution between the kinematic
// limits, Ivanchenko angles for the secondary.  The two logarithms and the
// expm1 of the omega draw take arguments close to 1 and 0, so they use the
// accurate library functions rather than the SFU forms.
template<class R> __device__ __forceinline__ bool kieft_event(const DevMaterial& m, Electron& p, Electron& se, R& rng,
	uint32_t ph)
{
	float omega0;
	{
		const float x = __logf(p.E);
		const float y = rng.unit();
		omega0 = __expf(table2_get(m.in_omega, x, y));
	}
	float binding;
	{
		const float x = __logf(omega0);
		const float y = rng.unit();
		binding = table2_rounddown(m.in_binding, x, y);
	}
	float omega;
	{
		const float omega_max = fm(0.5f, fs(fa(p.E, omega0), m.fermi));
		float omega_min = omega0;
		float w0 = smin(fs(omega0, 1.0f), fs(smax(0.0f, binding), m.fermi));
		if (p.E > fm(2.0f, omega0)) {
			omega_min = fm(0.5f, fs(fa(p.E, omega0), __fsqrt_rn(fm(p.E, fs(p.E, fm(2.0f, omega0))))));
			w0 = omega0;
		}
		const float U = rng.unit();
		if ((w0 > 0.0f) && (omega_min > w0) && (omega_min < omega_max)) {
			const float f_min = fm(fdf(1.0f, w0), logf(fdf(fs(omega_min, w0), omega_min)));
			const float f_max = fm(fdf(1.0f, w0), logf(fdf(fs(omega_max, w0), omega_max)));
			omega = fdf(-w0, expm1f(fm(w0, fa(fm(f_min, fs(1.0f, U)), fm(f_max, U)))));
		} else {
			omega = fdf(fm(omega0, omega_max), fa(fm(omega0, fs(1.0f, U)), fm(omega_max, U)));
		}
	}
	if (binding < 0.0f) {
		if (m.band_gap < 0.0f) {
			// metals: the reference leaves the Fermi-sea excitation open
		} else if (omega0 > m.band_gap) {
			binding = m.band_gap;
		} else {
			if (ph & PH_OPT_PHONON)
				p.E = fs(p.E, omega0);
			return false;
		}
	}
	binding = smax(0.0f, binding);
	p.dir = vnormalised(p.dir);
	const V3 normal_dir = vnormalised(make_normal_vec(p.dir, draw_phi(rng)));
	const float K = fa(fs(p.E, m.fermi), fm(2.0f, binding));
	const float dK = fa(binding, omega);
	const float cos_theta = __fsqrt_rn(fdf(dK, K));
	const float sin_theta = __fsqrt_rn(fs(1.0f, clampf(fm(cos_theta, cos_theta), 0.0f, 1.0f)));
	V3 sdir = vadd(vmul(p.dir, cos_theta), vmul(normal_dir, sin_theta));
	if (ph & PH_INST_MOM) {
		sdir = vnormalised(sdir);
		sdir = vadd(sdir, smul(__fsqrt_rn(fdf(binding, dK)), uniform_vector(rng)));
	}
	sdir = vnormalised(sdir);
	se.E = fs(fa(m.fermi, omega), binding);
	se.pos = p.pos;
	se.dir = sdir;
	p.E = fs(p.E, omega);
	if (ph & PH_MOM_CONS)
		p.dir = vsub(p.dir, smul(cos_theta, sdir));
	return (ph & PH_GEN_SE) != 0;
}

// Inelastic event of the selected model.  Returns true and fills `se` when a
// secondary electron is created.
template<class R> __device__ __forceinline__ bool inelastic_event(const DevMaterial& m, Electron& p, Electron& se, R& rng,
	uint32_t ph = PH_DEFAULT)
{
	if (ph & PH_KIEFT)
		return kieft_event(m, p, se, rng, ph);
	return penn_event(m, p, se, rng, ph);
}

enum : int { ST_RUNNING = 0, ST_DETECTED = 1, ST_TERMINATED = 2 };

// Boundary crossing (boundary_intersect.h:38-155) with quantum transmission,
// refraction and the Kieft-Bosch empirical absorption as selected.  `score`
// (optional) receives d log P(outcome) / d barrier_out and d / d barrier_in
// for the adjoint.
struct BoundaryScore { float d_in, d_out; int mat_in, mat_out; };

template<class R> __device__ __forceinline__ int boundary_event(const DevTriangle& T, const DevMaterial* __restrict__ mats,
	Electron& p, int& material, R& rng, BoundaryScore* score = nullptr, uint32_t ph = PH_DEFAULT,
	const float* dbar = nullptr)
{
	const V3 nd = vnormalised(p.dir);
	const V3 n = vnormalised(v3(T.nx, T.ny, T.nz));
	const float c = vdot(n, nd);
	int min_, mout;
	if (c > 0.0f) { min_ = T.mat_in; mout = T.mat_out; } else { min_ = T.mat_out; mout = T.mat_in; }
	switch (mout) {
	case MAT_DETECTOR: return ST_DETECTED;
	case MAT_DETECTOR_LT50: return p.E < 50.0f ? ST_DETECTED : ST_RUNNING;
	case MAT_DETECTOR_GE50: return p.E >= 50.0f ? ST_DETECTED : ST_RUNNING;
	case MAT_TERMINATOR: return ST_TERMINATED;
	case MAT_MIRROR: p.dir = vsub(nd, vmul(smul(2.0f, n), c)); return ST_RUNNING;
	case MAT_NOP: return ST_RUNNING;
	default: break;
	}
	if (score) { score->mat_in = min_; score->mat_out = mout; }
	// `dbar` (adjoint replay): barrier shifts of materials 0 and 1
	float dU = 0.0f;
	if (min_ >= 0) dU = fs(dU, (dbar && min_ < 2) ? fa(mats[min_].barrier, dbar[min_]) : mats[min_].barrier);
	if (mout >= 0) dU = fa(dU, (dbar && mout < 2) ? fa(mats[mout].barrier, dbar[mout]) : mats[mout].barrier);
	const float Ec2 = fm(fm(p.E, c), c);
	float g = 0.0f;                                          // d log P(outcome) / d dU
	if (fa(Ec2, dU) > 0.0f) {
		const float s = __fsqrt_rn(fa(1.0f, fdf(dU, Ec2)));
		const bool qt = (ph & PH_QT) != 0;
		const float Tr = qt ? fdf(fm(4.0f, s), fm(fa(1.0f, s), fa(1.0f, s))) : 1.0f;
		const bool transmit = rng.unit() < Tr;
		if (score && qt) {
			// T(s) = 4s/(1+s)^2, s^2 = 1 + dU/(E c^2):
			// dlogT/ddU = (1-s)/(s(1+s)) * ds/ddU, ds/ddU = 1/(2 s E c^2)
			const float dlogT_ds = fdf(fs(1.0f, s), fm(s, fa(1.0f, s)));
			const float ds_ddU = fdf(1.0f, fm(fm(2.0f, s), Ec2));
			g = fm(dlogT_ds, ds_ddU);                         // d log T / d dU
			if (!transmit) g = fm(-g, fdf(Tr, fs(1.0f, Tr)));  // d log(1-T) / d dU
		}
		if (transmit) {
			if (ph & PH_REFRACT)
				p.dir = vadd(vsub(nd, vmul(n, c)), vmul(smul(s, n), c));
			p.E = fa(p.E, dU);
			material = mout;
			if (score) { score->d_out = g; score->d_in = -g; }   // dU = +barrier_out - barrier_in
			return ST_RUNNING;
		}
	}
	if ((ph & PH_ABSORB) && dU < 0.0f) {
		// empirical absorption with probability exp(1 + E / (2 dU))
		const float pa = expf(fa(1.0f, fdf(fm(0.5f, p.E), dU)));
		if (rng.unit() < pa)
			return ST_TERMINATED;
		if (score) {
			// d log(1 - pa) / d dU = pa / (1 - pa) * E / (2 dU^2)
			g = fa(g, fm(fdf(pa, fs(1.0f, pa)), fdf(fm(0.5f, p.E), fm(dU, dU))));
		}
	}
	if (score) { score->d_out = g; score->d_in = -g; }
	p.dir = vsub(nd, vmul(smul(2.0f, n), c));
	return ST_RUNNING;
}

}  // namespace nbl
