/*
 * Test infrastructure (oracle), not product code.  See nbl_oracle.h.
 *
 * Every function restates one reference function, in float32 with the same
 * operation order (the reference's CPU build contracts nothing into FMAs:
 * x86-64 baseline, -O2), so that outputs match the reference bit for bit.
 * Reference file:line citations are given per function (paths relative to
 * the reference's source/ directory).
 */
#include "nbl_oracle.h"

#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <string>
#include <map>
#include <fstream>
#include <stdexcept>
#include <thread>
#include <mutex>
#include <atomic>
#include <limits>
#include <algorithm>
#include <functional>

namespace {

const float EPS = 10 * std::numeric_limits<float>::epsilon();  // config/data_types.h:58
const float PI = 3.1415926535897932f;                            // config/config.h:33

// special materials, core/material_manager.h:77-86
enum { NOP = -128, TERMINATOR = -127, DETECTOR = -126, DETECTOR_LT50 = -125,
	DETECTOR_GE50 = -124, VACUUM = -123, MIRROR = -122 };

struct v3 { float x, y, z; };
// common/vector_math.h:10-114 (component-wise, no contraction)
inline v3 add(v3 a, v3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline v3 sub(v3 a, v3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline v3 mul(v3 a, float b) { return { a.x * b, a.y * b, a.z * b }; }   // vec*real
inline v3 smul(float a, v3 b) { return { a * b.x, a * b.y, a * b.z }; }  // real*vec
inline v3 cross(v3 a, v3 b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float mag2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// CPU normalised(a) = a / sqrt(|a|^2) and operator/ multiplies by 1/b
// (vector_math.h:33-37, 141-158)
inline v3 normalised(v3 a) { float s = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); float inv = 1 / s; return mul(a, inv); }
inline float minr(float a, float b) { return std::min(a, b); }   // scalar_math.h:57-68 (CPU branch)
inline float maxr(float a, float b) { return std::max(a, b); }
inline float clampr(float i, float lo, float hi) { return i < lo ? lo : (i > hi ? hi : i); }  // :21-24
inline int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }
inline int floorr(float x) { return (int)std::floor(x); }        // :43-55 CPU branch

}  // namespace

/* ------------------------------------------------------------------ RNG */
struct orc_rng {
	int kind;                 // 0 mt19937, 1 list
	uint32_t mt[624];
	int mti;
	const float* list;
	int64_t n, used;
};

static uint32_t mt_next(orc_rng* r)
{
	// std::mt19937 (Matsumoto & Nishimura 1998), as std::mersenne_twister_engine
	if (r->mti >= 624) {
		for (int i = 0; i < 624; ++i) {
			uint32_t y = (r->mt[i] & 0x80000000u) | (r->mt[(i + 1) % 624] & 0x7fffffffu);
			r->mt[i] = r->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		}
		r->mti = 0;
	}
	uint32_t y = r->mt[r->mti++];
	y ^= y >> 11;
	y ^= (y << 7) & 0x9d2c5680u;
	y ^= (y << 15) & 0xefc60000u;
	y ^= y >> 18;
	return y;
}

static void mt_seed(orc_rng* r, uint32_t seed)
{
	r->kind = 0;
	r->mt[0] = seed;
	for (int i = 1; i < 624; ++i)
		r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i;
	r->mti = 624;
}

extern "C" orc_rng* orc_rng_mt(uint32_t seed)
{
	orc_rng* r = new orc_rng();
	mt_seed(r, seed);
	return r;
}

// Seed of primary i in the multithreaded loops: the splitmix64 finaliser
// (Steele, Lea and Flood 2014) of the run seed and the primary index, so a
// primary's random numbers depend on neither the thread that takes it nor
// the thread count.
static uint32_t primary_seed(uint32_t seed, int64_t i)
{
	uint64_t z = (uint64_t)seed * 0x9E3779B97F4A7C15ull + (uint64_t)i;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	z ^= z >> 31;
	return (uint32_t)(z ^ (z >> 32));
}
extern "C" orc_rng* orc_rng_list(const float* u, int64_t n)
{
	orc_rng* r = new orc_rng();
	r->kind = 1; r->list = u; r->n = n; r->used = 0;
	return r;
}
extern "C" int64_t orc_rng_used(const orc_rng* r) { return r->used; }
extern "C" void orc_rng_free(orc_rng* r) { delete r; }

/* random_state<false>::unit (common/util/random.inl:19-26):
 * std::generate_canonical<float, 24>(mt19937): one 32-bit draw, converted to
 * float and scaled by 2^-32; a result of 1 becomes the largest float < 1. */
extern "C" float orc_rng_unit(orc_rng* r)
{
	if (r->kind == 1) {
		float u = r->used < r->n ? r->list[r->used] : 0.5f;
		++r->used;
		return u;
	}
	++r->used;
	float sum = (float)mt_next(r);
	float tmp = 4294967296.0f;
	float ret = sum / tmp;
	if (ret >= 1.0f)
		ret = std::nextafter(1.0f, 0.0f);
	return ret;
}

namespace {
// random_generator (common/util/random.h:56-83)
inline float rphi(orc_rng* r) { return 2 * PI * orc_rng_unit(r); }
inline float rexponential(orc_rng* r, float tau) { return -tau * std::log(orc_rng_unit(r)); }

// make_unit_vec (vector_math.h:194-206)
inline v3 make_unit_vec(float cos_theta, float phi)
{
	float sin_phi = std::sin(phi), cos_phi = std::cos(phi);
	cos_theta = clampr(cos_theta, -1, 1);
	const float sin_theta = std::sqrt(1 - cos_theta * cos_theta);
	return { sin_theta * cos_phi, sin_theta * sin_phi, cos_theta };
}
// uniform_vector (random.h:72-76): make_unit_vec(2*unit() - 1, phi()).  The
// reference's g++ build evaluates the call's arguments right to left, so the
// azimuth is drawn first.
inline v3 uniform_vector(orc_rng* r)
{
	const float phi = rphi(r);
	const float ct = 2 * orc_rng_unit(r) - 1;
	return make_unit_vec(ct, phi);
}
// make_normal_vec (vector_math.h:171-186)
inline v3 make_normal_vec(v3 dir, float phi)
{
	const float az = std::atan2(dir.y, dir.x);
	const float sin_az = std::sin(az), cos_az = std::cos(az);
	const v3 unit_v{ dir.z * cos_az, dir.z * sin_az, -std::sqrt(dir.x * dir.x + dir.y * dir.y) };
	const v3 unit_u = cross(unit_v, dir);
	const float sin_phi = std::sin(phi), cos_phi = std::cos(phi);
	return add(mul(unit_u, cos_phi), mul(unit_v, sin_phi));
}

/* ------------------------------------------------------------ tables */
inline float tget(const orc_table& t, int i, int j, int k) { return t.data[((size_t)i * t.ny + j) * t.nz + k]; }

// table_1D::get (common/util/table_1D.inl:66-81)
float t1_get(const orc_table& t, float x)
{
	const float xi = (x - t.x_min) * t.x_step;
	const int lo = clampi(floorr(xi), 0, t.nx - 2);
	const float a = t.data[lo], b = t.data[lo + 1];
	const float f = xi - lo;
	return (1 - f) * a + f * b;
}
// table_2D::get (table_2D.inl:73-94)
float t2_get(const orc_table& t, float x, float y)
{
	const float xi = (x - t.x_min) * t.x_step;
	const float yi = (y - t.y_min) * t.y_step;
	const int lx = clampi(floorr(xi), 0, t.nx - 2);
	const int ly = clampi(floorr(yi), 0, t.ny - 2);
	const float v00 = tget(t, lx, ly, 0), v10 = tget(t, lx + 1, ly, 0);
	const float v01 = tget(t, lx, ly + 1, 0), v11 = tget(t, lx + 1, ly + 1, 0);
	const float fx = xi - lx, fy = yi - ly;
	return (1 - fx) * (1 - fy) * v00 + fx * (1 - fy) * v10 + (1 - fx) * fy * v01 + fx * fy * v11;
}
// table_2D::get_rounddown (table_2D.inl:96-104)
float t2_rd(const orc_table& t, float x, float y)
{
	const float xi = (x - t.x_min) * t.x_step;
	const float yi = (y - t.y_min) * t.y_step;
	return tget(t, clampi(floorr(xi), 0, t.nx - 1), clampi(floorr(yi), 0, t.ny - 1), 0);
}
// table_3D::get (table_3D.inl:79-110)
float t3_get(const orc_table& t, float x, float y, float z)
{
	const float xi = (x - t.x_min) * t.x_step;
	const float yi = (y - t.y_min) * t.y_step;
	const float zi = (z - t.z_min) * t.z_step;
	const int lx = clampi(floorr(xi), 0, t.nx - 2);
	const int ly = clampi(floorr(yi), 0, t.ny - 2);
	const int lz = clampi(floorr(zi), 0, t.nz - 2);
	const float v000 = tget(t, lx, ly, lz), v100 = tget(t, lx + 1, ly, lz);
	const float v010 = tget(t, lx, ly + 1, lz), v110 = tget(t, lx + 1, ly + 1, lz);
	const float v001 = tget(t, lx, ly, lz + 1), v101 = tget(t, lx + 1, ly, lz + 1);
	const float v011 = tget(t, lx, ly + 1, lz + 1), v111 = tget(t, lx + 1, ly + 1, lz + 1);
	const float fx = xi - lx, fy = yi - ly, fz = zi - lz;
	return (1 - fx) * (1 - fy) * (1 - fz) * v000
		+ fx * (1 - fy) * (1 - fz) * v100
		+ (1 - fx) * fy * (1 - fz) * v010
		+ fx * fy * (1 - fz) * v110
		+ (1 - fx) * (1 - fy) * fz * v001
		+ fx * (1 - fy) * fz * v101
		+ (1 - fx) * fy * fz * v011
		+ fx * fy * fz * v111;
}
// table_3D::get_rounddown (table_3D.inl:112-122)
float t3_rd(const orc_table& t, float x, float y, float z)
{
	const float xi = (x - t.x_min) * t.x_step;
	const float yi = (y - t.y_min) * t.y_step;
	const float zi = (z - t.z_min) * t.z_step;
	return tget(t, clampi(floorr(xi), 0, t.nx - 1), clampi(floorr(yi), 0, t.ny - 1), clampi(floorr(zi), 0, t.nz - 1));
}

/* ------------------------------------------------------------ geometry */
struct tri { int mi, mo; v3 r0, e1, e2; };
inline tri get_tri(const orc_geometry* g, int i)
{
	const float* t = g->tri11 + 11 * (size_t)i;
	return { (int)t[0], (int)t[1], { t[2], t[3], t[4] }, { t[5], t[6], t[7] }, { t[8], t[9], t[10] } };
}

// triangle::intersect_ray (core/triangle.inl:7-28)
float intersect_ray(const tri& T, v3 start, v3 dir)
{
	const v3 pvec = cross(dir, T.e2);
	const float det = dot(T.e1, pvec);
	if (std::abs(det) < EPS)
		return -1;
	const float u = dot(sub(start, T.r0), pvec) / det;
	if ((u < -EPS) || (u > 1 + EPS))
		return -1;
	const v3 qvec = cross(sub(start, T.r0), T.e1);
	const float v = dot(dir, qvec) / det;
	if ((v < -EPS) || (u + v > 1 + EPS))
		return -1;
	const float t = dot(T.e2, qvec) / det;
	if (t < 0)
		return -1;
	return t;
}

// octree::in_domain (geometry/octree.inl:25-30)
bool in_domain(const orc_geometry* g, v3 p)
{
	const float* c = g->center; const float* h = g->halfsize;
	return (p.x > c[0] - h[0]) && (p.x < c[0] + h[0]) && (p.y > c[1] - h[1]) && (p.y < c[1] + h[1])
		&& (p.z > c[2] - h[2]) && (p.z < c[2] + h[2]);
}

inline int clz64(uint64_t x) { return __builtin_clzll(x); }

// octree::propagate (geometry/octree.inl:33-192), AABB_intersect (:212-220)
void propagate(const orc_geometry* g, v3 start, v3 direction, float distance,
	int ignore_tri, int ignore_material, float* out_dist, int* out_tri)
{
	const int* od = g->octree_data;
	const v3 hs{ g->halfsize[0], g->halfsize[1], g->halfsize[2] };
	v3 cur = start;
	float to_go = distance;
	uint64_t location = 1;
	do {
		float ax = g->center[0], ay = g->center[1], az = g->center[2], aw = 1;
		int index = 0;
		for (int i = 60 - clz64(location); i >= 0; i -= 3) {
			const unsigned int octant = (location >> i) & 7;
			index = od[index + octant];
			ax += aw * hs.x * ((octant & 1) - 0.5f);
			ay += aw * hs.y * (((octant & 2) >> 1) - 0.5f);
			az += aw * hs.z * (((octant & 4) >> 2) - 0.5f);
			aw *= 0.5f;
		}
		while (index >= 0) {
			unsigned int octant = 0;
			octant ^= (cur.x > ax) ? 1 : 0;
			octant ^= (cur.y > ay) ? 2 : 0;
			octant ^= (cur.z > az) ? 4 : 0;
			location = (location << 3) | octant;
			index = od[index + octant];
			ax += aw * hs.x * ((octant & 1) - 0.5f);
			ay += aw * hs.y * (((octant & 2) >> 1) - 0.5f);
			az += aw * hs.z * (((octant & 4) >> 2) - 0.5f);
			aw *= 0.5f;
		}
		index = -index;

		float intersect;
		int target;
		{
			const v3 h = smul(aw, hs);
			const float tx = (ax + std::copysign(h.x + EPS, direction.x) - cur.x) / direction.x;
			const float ty = (ay + std::copysign(h.y + EPS, direction.y) - cur.y) / direction.y;
			const float tz = (az + std::copysign(h.z + EPS, direction.z) - cur.z) / direction.z;
			if ((tx < ty) && (tx < tz)) { intersect = tx; target = -1; }
			else if ((ty < tx) && (ty < tz)) { intersect = ty; target = -2; }
			else { intersect = tz; target = -4; }
		}

		while (true) {
			const int ti = od[index++];
			if (ti < 0)
				break;
			if (ti == ignore_tri)
				continue;
			const tri T = get_tri(g, ti);
			const int mat_out = dot(cross(T.e1, T.e2), direction) < 0 ? T.mi : T.mo;
			if (mat_out == ignore_material)
				continue;
			const float t = intersect_ray(T, cur, direction);
			if ((t > 0) && (t <= intersect + EPS)) {
				intersect = t;
				target = ti;
			}
		}

		if (intersect >= to_go) {
			*out_dist = distance; *out_tri = -1;
			return;
		}
		else if (target >= 0) {
			*out_dist = distance - to_go + intersect; *out_tri = target;
			return;
		}
		to_go -= intersect;
		cur = add(cur, mul(direction, intersect));

		unsigned int mask = -target;
		unsigned int value;
		if (mask == 1) value = (direction.x >= 0) ? 0 : 1;
		else if (mask == 2) value = (direction.y >= 0) ? 0 : 2;
		else value = (direction.z >= 0) ? 0 : 4;
		while (location > 1) {
			if ((location & mask) == value) {
				location ^= mask;
				break;
			}
			location >>= 3;
		}
	} while (location > 1);
	*out_dist = distance; *out_tri = -1;
}

/* ------------------------------------------------------------ particles */
// drivers/cpu/cpu_particle_manager.h:73-97
enum status_t { SCATTER_EVENT, INTERSECT_EVENT, NO_EVENT, DETECTED, TERMINATED };
struct pstate {
	status_t status;
	uint8_t next_scatter;
	int material;
	v3 pos, dir;
	float E;
	int last_tri;
};

struct manager {
	std::vector<pstate> p;
	// create_secondary (cpu_particle_manager.inl:181-196)
	void create_secondary(size_t parent, v3 pos, v3 dir, float E)
	{
		p.push_back({ NO_EVENT, 0, p[parent].material, pos, dir, E, -1 });
	}
};

/* ------------------------------------------------------------ physics */
enum : uint32_t {
	PH_GEN_SE = 1, PH_PHONON = 2, PH_RECOIL = 4, PH_QT = 8, PH_REFRACT = 16, PH_ABSORB = 32,
	PH_OPT_PHONON = 64, PH_INST_MOM = 128, PH_MOM_CONS = 256, PH_KIEFT = 65536,
	PH_DEFAULT = 1 | 2 | 4 | 8 | 16 | 64 | 128 | 256
};
uint32_t g_phys = PH_DEFAULT;

// kieft_elastic<cpu, acoustic_phonon_loss, atomic_recoil_loss>::execute
// (physics/kieft/elastic.h:67-115)
void elastic(const orc_material& m, pstate& ps, orc_rng* rng)
{
	pstate p = ps;
	const float x = std::log(ps.E);
	const float y = orc_rng_unit(rng);
	const float cos_theta = clampr(t2_get(m.el_icdf, x, y), -1, 1);
	const float sin_theta = std::sqrt(1 - cos_theta * cos_theta);
	p.dir = normalised(p.dir);
	const v3 normal_dir = normalised(make_normal_vec(p.dir, rphi(rng)));
	p.dir = add(mul(p.dir, cos_theta), mul(normal_dir, sin_theta));
	if (p.E < 200) {
		if (g_phys & PH_PHONON)
			p.E -= minr(50e-3f, m.phonon_loss);
	} else if (g_phys & PH_RECOIL) {
		p.E -= m.recoil_const * (1 - cos_theta) * p.E;
	}
	ps = p;
}

// full_penn<cpu, generate_secondary>::execute (physics/full_penn.h:62-288)
void inelastic_penn(const orc_material& m, manager& mgr, size_t idx, orc_rng* rng)
{
	pstate p = mgr.p[idx];
	float omega;
	{
		const float x = std::log(p.E);
		const float y = orc_rng_unit(rng);
		omega = std::exp(t2_get(m.in_omega, x, y));
	}
	float binding;
	{
		const float x = std::log(p.E);
		const float y = std::log(omega / p.E);
		const float z = orc_rng_unit(rng);
		binding = t3_rd(m.in_binding, x, y, z);
	}
	p.dir = normalised(p.dir);
	if (binding <= 0) {
		if (omega > m.band_gap) {
			float q;
			{
				const float x = std::log(p.E);
				const float y = omega / p.E;
				const float z = orc_rng_unit(rng);
				q = t3_get(m.in_q, x, y, z);
			}
			const v3 prim_normal_dir = normalised(make_normal_vec(p.dir, rphi(rng)));
			v3 q_dir, q_normal_dir;
			{
				const float c = clampr((omega + q * q) / (2 * std::sqrt(p.E) * q), -1, 1);
				const float s = std::sqrt(1 - c * c);
				q_dir = normalised(add(mul(p.dir, c), mul(prim_normal_dir, s)));
				q_normal_dir = normalised(make_normal_vec(q_dir, rphi(rng)));
			}
			const float c2 = clampr((2 * p.E - omega - q * q) / (2 * std::sqrt(p.E * (p.E - omega))), -1, 1);
			const float s2 = std::sqrt(1 - c2 * c2);
			p.E -= omega;
			p.dir = add(mul(p.dir, c2), mul(prim_normal_dir, s2));
			mgr.p[idx] = p;
			if (!(g_phys & PH_GEN_SE))
				return;

			const v3 se_pos = p.pos;
			v3 se_dir;
			float se_E;
			const float k_fermi = std::sqrt(m.fermi);
			const float k_fermi_omega = std::sqrt(m.fermi + omega);
			if (q < k_fermi_omega - k_fermi) {
				const float f = m.fermi / omega;
				float x;
				if (f < 0.1f) {
					const float U = std::cbrt(orc_rng_unit(rng));
					x = f * U * U;
				} else {
					const float lower = maxr(0, f - 1);
					const float upper = f;
					const float d1 = upper - lower;
					const float d2 = upper * upper - lower * lower;
					const float alpha = d2 / (d1 + d2);
					do {
						const float U1 = orc_rng_unit(rng);
						const float U2 = orc_rng_unit(rng);
						x = (U1 < alpha) ? std::sqrt(d2 * U2 + lower * lower) : d1 * U2 + lower;
					} while (orc_rng_unit(rng) > std::sqrt(x * x + x) / (x + .5f));
				}
				se_E = x * omega + omega;
				se_dir = uniform_vector(rng);
			} else if (q < k_fermi_omega + k_fermi) {
				const float ki_parr = (omega - q * q) / (2 * q);
				const float kf_parr = ki_parr + q;
				const float ki_perp_min_sq = maxr(0, m.fermi - kf_parr * kf_parr);
				const float ki_perp_max_sq = m.fermi - ki_parr * ki_parr;
				const float ki_perp_sq = maxr(0, ki_perp_min_sq + (ki_perp_max_sq - ki_perp_min_sq) * orc_rng_unit(rng));
				const v3 ki = add(smul(ki_parr, q_dir), smul(std::sqrt(ki_perp_sq), q_normal_dir));
				se_E = mag2(ki) + omega;
				se_dir = add(ki, smul(q, q_dir));
			} else {
				return;
			}
			mgr.create_secondary(idx, se_pos, se_dir, se_E);
			return;
		} else {
			p.E -= omega;
			mgr.p[idx] = p;
			return;
		}
	}
	// inner shell
	const v3 normal_dir = normalised(make_normal_vec(p.dir, rphi(rng)));
	const float K = p.E - m.fermi + 2 * binding;
	const float dK = binding + omega;
	const float cos_theta = std::sqrt(dK / K);
	const float sin_theta = std::sqrt(1 - clampr(cos_theta * cos_theta, 0, 1));
	v3 sdir = add(mul(p.dir, cos_theta), mul(normal_dir, sin_theta));
	sdir = normalised(sdir);
	sdir = add(sdir, smul(std::sqrt(binding / dK), uniform_vector(rng)));
	sdir = normalised(sdir);
	if (g_phys & PH_GEN_SE)
		mgr.create_secondary(idx, p.pos, sdir, m.fermi + omega - binding);
	p.E -= omega;
	p.dir = sub(p.dir, smul(cos_theta, sdir));
	mgr.p[idx] = p;
}

// kieft_inelastic<cpu, optical_phonon_loss, generate_secondary,
// instantaneous_momentum, momentum_conservation>::execute
// (physics/kieft/inelastic.h:63-209)
void inelastic_kieft(const orc_material& m, manager& mgr, size_t idx, orc_rng* rng)
{
	pstate p = mgr.p[idx];
	float omega0;
	{	// zero-momentum loss (thesis T.V. eq. 3.82)
		const float x = std::log(p.E);
		const float y = orc_rng_unit(rng);
		omega0 = std::exp(t2_get(m.ki_w0, x, y));
	}
	float binding;
	{
		const float x = std::log(omega0);
		const float y = orc_rng_unit(rng);
		binding = t2_rd(m.ki_binding, x, y);
	}
	float omega;
	{	// Ashley's total loss between the kinematic limits (eq. 3.85)
		const float omega_max = 0.5f * (p.E + omega0 - m.fermi);
		float omega_min = omega0;
		float w0 = minr(omega0 - 1, maxr(0, binding) - m.fermi);
		if (p.E > 2 * omega0) {
			omega_min = 0.5f * (p.E + omega0 - std::sqrt(p.E * (p.E - 2 * omega0)));
			w0 = omega0;
		}
		const float U = orc_rng_unit(rng);
		if ((w0 > 0) && (omega_min > w0) && (omega_min < omega_max)) {
			const float f_min = 1 / w0 * std::log((omega_min - w0) / omega_min);
			const float f_max = 1 / w0 * std::log((omega_max - w0) / omega_max);
			omega = -w0 / std::expm1(w0 * (f_min * (1 - U) + f_max * U));
		} else {
			omega = omega0 * omega_max / (omega0 * (1 - U) + omega_max * U);
		}
	}
	if (binding < 0) {
		if (m.band_gap < 0) {
			// metals: left open by the reference
		} else if (omega0 > m.band_gap) {
			binding = m.band_gap;
		} else {
			if (g_phys & PH_OPT_PHONON) {
				p.E -= omega0;
				mgr.p[idx] = p;
			}
			return;
		}
	}
	binding = maxr(0, binding);
	p.dir = normalised(p.dir);
	const v3 normal_dir = normalised(make_normal_vec(p.dir, rphi(rng)));
	const float K = p.E - m.fermi + 2 * binding;
	const float dK = binding + omega;
	const float cos_theta = std::sqrt(dK / K);
	const float sin_theta = std::sqrt(1 - clampr(cos_theta * cos_theta, 0, 1));
	v3 sdir = add(mul(p.dir, cos_theta), mul(normal_dir, sin_theta));
	if (g_phys & PH_INST_MOM) {
		sdir = normalised(sdir);
		sdir = add(sdir, smul(std::sqrt(binding / dK), uniform_vector(rng)));
	}
	sdir = normalised(sdir);
	if (g_phys & PH_GEN_SE)
		mgr.create_secondary(idx, p.pos, sdir, m.fermi + omega - binding);
	p.E -= omega;
	if (g_phys & PH_MOM_CONS)
		p.dir = sub(p.dir, smul(cos_theta, sdir));
	mgr.p[idx] = p;
}

void inelastic(const orc_material& m, manager& mgr, size_t idx, orc_rng* rng)
{
	if (g_phys & PH_KIEFT) inelastic_kieft(m, mgr, idx, rng);
	else inelastic_penn(m, mgr, idx, rng);
}

// boundary_intersect<quantum_transmission, interface_refraction,
// interface_absorption>::execute (physics/boundary_intersect.h:38-155)
void boundary(const orc_geometry* g, const orc_material* mats, pstate& ps, orc_rng* rng)
{
	pstate p = ps;
	const tri T = get_tri(g, ps.last_tri);
	const v3 nd = normalised(p.dir);
	const v3 n = normalised(cross(T.e1, T.e2));
	const float c = dot(n, nd);
	int min_, mout;
	if (c > 0) { min_ = T.mi; mout = T.mo; } else { min_ = T.mo; mout = T.mi; }
	switch (mout) {
	case DETECTOR: ps.status = DETECTED; return;
	case DETECTOR_LT50: if (p.E < 50) ps.status = DETECTED; return;
	case DETECTOR_GE50: if (p.E >= 50) ps.status = DETECTED; return;
	case TERMINATOR: ps.status = TERMINATED; return;
	case MIRROR: p.dir = sub(nd, mul(smul(2, n), c)); ps = p; return;
	case NOP: return;
	default: break;
	}
	float dU = 0;
	if (min_ >= 0) dU -= mats[min_].barrier;
	if (mout >= 0) dU += mats[mout].barrier;
	if (p.E * c * c + dU > 0) {
		const float s = std::sqrt(1 + dU / (p.E * c * c));
		const float Tr = (g_phys & PH_QT) ? 4 * s / ((1 + s) * (1 + s)) : 1;
		if (orc_rng_unit(rng) < Tr) {
			if (g_phys & PH_REFRACT)
				p.dir = add(sub(nd, mul(n, c)), mul(smul(s, n), c));
			p.E += dU;
			p.material = mout;
			ps = p;
			return;
		}
	}
	if (g_phys & PH_ABSORB) {
		if (dU < 0 && orc_rng_unit(rng) < std::exp(1 + 0.5f * p.E / dU)) {
			ps.status = TERMINATED;
			return;
		}
	}
	p.dir = sub(nd, mul(smul(2, n), c));
	ps = p;
}

/* ------------------------------------------------------------ driver */
struct driver {
	const orc_geometry* g;
	const orc_material* mats;
	float threshold;
	orc_rng* rng;
	manager mgr;

	// cpu_driver::init (drivers/cpu/cpu_driver.inl:74-130)
	void init(size_t idx)
	{
		pstate p = mgr.p[idx];
		if (!in_domain(g, p.pos)) { mgr.p[idx].status = TERMINATED; return; }
		uint8_t type = 0;
		float distance = g->max_extent;
		const int mi = p.material;
		if (mi >= 0) {
			const orc_material& m = mats[mi];
			if (p.E < m.barrier + threshold) { mgr.p[idx].status = TERMINATED; return; }
			// scatter_list::sample_path (core/scatter_list.h:101-107) visits the
			// processes with tuple::for_each, which runs from the last element
			// to the first (common/tuple.h:113-118): elastic (type 2) draws
			// first, then inelastic (type 1); the strictly shorter path wins.
			distance = std::numeric_limits<float>::infinity();
			{
				const float imfp = std::exp(t1_get(m.el_imfp, std::log(p.E)));
				const float path = rexponential(rng, 1 / imfp);
				if (path < distance) { distance = path; type = 2; }
			}
			{
				const orc_table& it = (g_phys & PH_KIEFT) ? m.ki_imfp : m.in_imfp;
				const float imfp = std::exp(t1_get(it, std::log(p.E)));
				const float path = rexponential(rng, 1 / imfp);
				if (path < distance) { distance = path; type = 1; }
			}
		}
		const v3 d = normalised(p.dir);
		float idist; int itri;
		propagate(g, p.pos, d, distance, mgr.p[idx].last_tri, mi, &idist, &itri);
		pstate& s = mgr.p[idx];
		if (itri < 0) {
			// set_scatter_event (cpu_particle_manager.inl:211-224)
			if (type != 0) { s.status = SCATTER_EVENT; s.next_scatter = type; }
			else s.status = NO_EVENT;
			s.pos = add(s.pos, mul(normalised(s.dir), distance));
		} else {
			// set_intersect_event (:225-232)
			s.status = INTERSECT_EVENT;
			s.last_tri = itri;
			s.pos = add(s.pos, mul(normalised(s.dir), idist));
		}
	}
	// cpu_driver::intersect (:136-143)
	void intersect(size_t idx)
	{
		if (mgr.p[idx].status != INTERSECT_EVENT) return;
		boundary(g, mats, mgr.p[idx], rng);
	}
	// cpu_driver::scatter (:148-160)
	void scatter(size_t idx)
	{
		if (mgr.p[idx].status != SCATTER_EVENT) return;
		mgr.p[idx].last_tri = -1;
		const orc_material& m = mats[mgr.p[idx].material];
		if (mgr.p[idx].next_scatter == 1) inelastic(m, mgr, idx, rng);
		else elastic(m, mgr.p[idx], rng);
	}
	bool active(size_t idx) const { return mgr.p[idx].status != TERMINATED && mgr.p[idx].status != DETECTED; }

	// energy-deposit driver (energydeposit_cpu_driver.h:44-93): called for a
	// scatter event (not a crossing) that changed the kinetic energy
	std::function<void(const pstate& before, const pstate& after)> on_deposit;

	// push one primary, simulate_to_end (simple_cpu_driver.h:53-65), flush
	template<typename F>
	void run_one(const float* f, int64_t& events, F emit)
	{
		mgr.p.clear();
		// cpu_particle_manager::push (cpu_particle_manager.inl:22-43): vacuum
		mgr.p.push_back({ NO_EVENT, 0, VACUUM, { f[0], f[1], f[2] }, { f[3], f[4], f[5] }, f[6], -1 });
		for (size_t i = 0; i < mgr.p.size(); ++i)
			while (active(i)) {
				init(i);
				if (on_deposit) {
					const bool track = mgr.p[i].status == SCATTER_EVENT;
					const pstate before = mgr.p[i];
					intersect(i); scatter(i); ++events;
					const pstate after = mgr.p[i];
					if (track && before.E != after.E)
						on_deposit(before, after);
				} else {
					intersect(i); scatter(i); ++events;
				}
				if (std::getenv("NBL_TRACE")) {
					const pstate& q = mgr.p[i];
					std::fprintf(stderr, "O %zu %d %d %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n", i, (int)q.status, q.material,
						q.pos.x, q.pos.y, q.pos.z, q.dir.x, q.dir.y, q.dir.z, q.E);
				}
			}
		for (auto& q : mgr.p)
			if (q.status == DETECTED) emit(q);
	}
};

}  // namespace


/* ------------------------------------------------------------ materials */
/* Loads a .nmat material file and applies the reference's table transforms:
 * kieft_elastic::create (physics/kieft/elastic.h:120-166), full_penn::create
 * (physics/full_penn.h:294-406) and material(hdf5_file)
 * (core/material.inl:13-18).  Dimension scales become geomspace/linspace
 * ranges (common/util/range.h:210-327) whose first/last values set the
 * table axes; double arithmetic follows units::quantity
 * (common/units/quantity.h), where eV, nm and dimensionless are 1 and g is
 * 6.2415e15 (common/units/unit_system.h:16-36). */
namespace {
struct nm_scale { bool present = false; std::string unit; std::vector<double> v; };
struct nm_set { std::string unit; std::vector<uint64_t> dims; std::vector<nm_scale> scales; std::vector<float> data; };
struct nm_file { std::map<std::string, std::pair<double, std::string>> props; std::map<std::string, nm_set> sets; };

// HDF5 resolves "a/b" and "/a/b" to the same dataset
std::string canonical(const std::string& name)
{
	size_t i = 0;
	while (i < name.size() && name[i] == '/') ++i;
	return name.substr(i);
}

nm_file read_nmat(const char* path)
{
	std::ifstream f(path, std::ios::binary);
	if (!f) throw std::runtime_error(std::string("cannot open ") + path);
	std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	size_t off = 0;
	auto need = [&](size_t n) { if (off + n > b.size()) throw std::runtime_error("truncated .nmat"); };
	auto u32 = [&]() { need(4); uint32_t v; std::memcpy(&v, &b[off], 4); off += 4; return v; };
	auto u64 = [&]() { need(8); uint64_t v; std::memcpy(&v, &b[off], 8); off += 8; return v; };
	auto f64 = [&]() { need(8); double v; std::memcpy(&v, &b[off], 8); off += 8; return v; };
	auto str = [&]() { uint32_t n = u32(); need(n); std::string s(&b[off], n); off += n; return s; };
	need(8);
	if (std::memcmp(b.data(), "NBLMAT01", 8)) throw std::runtime_error("not an .nmat file");
	off = 8;
	nm_file out;
	for (uint32_t i = 0, n = u32(); i < n; ++i) { std::string k = str(); double v = f64(); out.props[k] = { v, str() }; }
	for (uint32_t i = 0, n = u32(); i < n; ++i) {
		nm_set s; std::string k = str(); s.unit = str();
		uint32_t nd = u32();
		for (uint32_t a = 0; a < nd; ++a) s.dims.push_back(u64());
		for (uint32_t a = 0; a < nd; ++a) {
			need(1); nm_scale sc; sc.present = b[off++] != 0;
			if (sc.present) { sc.unit = str(); sc.v.resize(s.dims[a]); need(8 * s.dims[a]); std::memcpy(sc.v.data(), &b[off], 8 * s.dims[a]); off += 8 * s.dims[a]; }
			s.scales.push_back(sc);
		}
		size_t cnt = 1; for (auto d : s.dims) cnt *= d;
		s.data.resize(cnt); need(4 * cnt); std::memcpy(s.data.data(), &b[off], 4 * cnt); off += 4 * cnt;
		out.sets[canonical(k)] = s;
	}
	return out;
}

double unit_value(const std::string& u)
{
	// the units these files use: eV, nm, nm^-1, g, dimensionless
	if (u.empty() || u == "eV" || u == "nm" || u == "nm^-1") return 1.0;
	if (u == "g") return 6.2415e15;
	throw std::runtime_error("unknown unit " + u);
}

// geomspace(front, back, n): first value and the recomputed last value
void log_range(const nm_scale& s, double& first, double& last)
{
	const double u = unit_value(s.unit);
	const double a = s.v.front() * u, b = s.v.back() * u;
	const size_t n = s.v.size();
	const double step = std::log(b / a) / (n - 1);
	first = a;
	last = a * std::exp((n - 1) * step);
}
// linspace(front, back, n) (absent scale: [0, 1])
void lin_range(const nm_scale& s, size_t n, double& first, double& last)
{
	double a = 0, b = 1;
	if (s.present) { const double u = unit_value(s.unit); a = s.v.front() * u; b = s.v.back() * u; }
	const double step = (b - a) / (n - 1);
	first = a;
	last = a + (n - 1) * step;
}

struct owned_material {
	orc_material m;
	std::vector<float> store[9];
};


void set_axis(int32_t n, double lo, double hi, bool log_axis, float& vmin, float& vstep)
{
	const float a = (float)(log_axis ? std::log(lo) : lo);
	const float b = (float)(log_axis ? std::log(hi) : hi);
	vmin = a;
	vstep = (n - 1) / (b - a);
}
}  // namespace

extern "C" void* orc_material_load(const char* path, char* err, int errlen)
{
	try {
		nm_file f = read_nmat(path);
		auto* o = new owned_material();
		std::memset(&o->m, 0, sizeof(o->m));
		auto prop = [&](const char* k) -> double {
			auto it = f.props.find(k);
			if (it == f.props.end()) throw std::runtime_error(std::string("missing property ") + k);
			return it->second.first * unit_value(it->second.second);
		};
		auto set = [&](const char* k) -> nm_set& {
			auto it = f.sets.find(canonical(k));
			if (it == f.sets.end()) throw std::runtime_error(std::string("missing dataset ") + k);
			return it->second;
		};
		const bool penn = f.sets.count("full_penn/imfp") != 0, kieft = f.sets.count("inelastic_kieft/imfp") != 0;
		if (!penn && !kieft) throw std::runtime_error("no inelastic model tables");
		o->m.models = (penn ? 1 : 0) | (kieft ? 2 : 0);
		double lo, hi;
		// elastic imfp (elastic.h:129-140), inelastic imfp (full_penn.h:306-317,
		// kieft/inelastic.h:226-238)
		const char* imfp_names[3] = { "/elastic/imfp", "/full_penn/imfp", "/inelastic_kieft/imfp" };
		orc_table* imfp_tabs[3] = { &o->m.el_imfp, &o->m.in_imfp, &o->m.ki_imfp };
		const int imfp_store[3] = { 0, 2, 6 };
		for (int k = 0; k < 3; ++k) {
			if ((k == 1 && !penn) || (k == 2 && !kieft)) continue;
			nm_set& s = set(imfp_names[k]);
			std::vector<float>& st = o->store[imfp_store[k]];
			st = s.data;
			const float unit = (float)(unit_value(s.unit) * 1.0);
			for (auto& v : st) v = std::log(v * unit);
			orc_table& t = *imfp_tabs[k];
			t.nx = (int32_t)s.dims[0]; t.ny = t.nz = 1;
			log_range(s.scales[0], lo, hi);
			set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			t.data = st.data();
		}
		{	// elastic costheta icdf (elastic.h:144-157)
			nm_set& s = set("/elastic/costheta_icdf");
			std::vector<float>& st = o->store[1];
			st = s.data;
			for (auto& v : st) v = std::max(-1.0f, std::min(1.0f, v));
			orc_table& t = o->m.el_icdf;
			t.nx = (int32_t)s.dims[0]; t.ny = (int32_t)s.dims[1]; t.nz = 1;
			log_range(s.scales[0], lo, hi); set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			lin_range(s.scales[1], t.ny, lo, hi); set_axis(t.ny, lo, hi, false, t.y_min, t.y_step);
			t.data = st.data();
		}
		const double fermi_q = prop("fermi");
		// omega icdf (full_penn.h:321-344) / omega' icdf (kieft/inelastic.h:240-261)
		for (int k = 0; k < 2; ++k) {
			if ((k == 0 && !penn) || (k == 1 && !kieft)) continue;
			nm_set& s = set(k == 0 ? "/full_penn/omega_icdf" : "/inelastic_kieft/w0_icdf");
			std::vector<float>& st = o->store[k == 0 ? 3 : 7];
			st = s.data;
			const float unit = (float)(unit_value(s.unit) / 1.0);
			const nm_scale& ks = s.scales[0];
			const double u = unit_value(ks.unit);
			const double first = ks.v.front() * u;
			const double step = std::log((ks.v.back() * u) / first) / (ks.v.size() - 1);
			for (size_t x = 0; x < s.dims[0]; ++x) {
				const double K = first * std::exp(x * step);
				for (size_t y = 0; y < s.dims[1]; ++y) {
					float& v = st[x * s.dims[1] + y];
					v = (float)std::log(std::max(0.0, std::min<double>((K - fermi_q) / 1.0, v * unit)));
				}
			}
			orc_table& t = k == 0 ? o->m.in_omega : o->m.ki_w0;
			t.nx = (int32_t)s.dims[0]; t.ny = (int32_t)s.dims[1]; t.nz = 1;
			log_range(s.scales[0], lo, hi); set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			lin_range(s.scales[1], t.ny, lo, hi); set_axis(t.ny, lo, hi, false, t.y_min, t.y_step);
			t.data = st.data();
		}
		if (kieft) {	// ionisation table (kieft/inelastic.h:262-327)
			nm_set& s = set("ionization/binding_icdf");
			nm_set& sh = set("ionization/outer_shells");
			if (s.dims.size() != 2) throw std::runtime_error("Kieft binding table must be 2-D");
			std::vector<float>& st = o->store[8];
			st = s.data;
			orc_table& t = o->m.ki_binding;
			t.nx = (int32_t)s.dims[0]; t.ny = (int32_t)s.dims[1]; t.nz = 1;
			log_range(s.scales[0], lo, hi); set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			lin_range(s.scales[1], t.ny, lo, hi); set_axis(t.ny, lo, hi, false, t.y_min, t.y_step);
			t.data = st.data();
			std::vector<double> shells;
			for (float v : sh.data) {
				const double e = (double)v * unit_value(sh.unit);
				if (e < 100) shells.push_back(e);
			}
			std::sort(shells.begin(), shells.end());
			const double unit = unit_value(s.unit);
			const nm_scale& ks = s.scales[0];
			const double kf = ks.v.front() * unit_value(ks.unit);
			const double kstep = std::log((ks.v.back() * unit_value(ks.unit)) / kf) / (ks.v.size() - 1);
			double pa = 0, pb = 1;
			if (s.scales[1].present) { pa = s.scales[1].v.front() * unit_value(s.scales[1].unit); pb = s.scales[1].v.back() * unit_value(s.scales[1].unit); }
			const double pstep = (pb - pa) / (t.ny - 1);
			// rewritten in place in row order while being read (as the reference does)
			for (int32_t x = 0; x < t.nx; ++x) {
				const double K = kf * std::exp(x * kstep);
				for (int32_t y = 0; y < t.ny; ++y) {
					const float P = (float)(pa + y * pstep);
					double b = -1;
					if (K > 100) {
						b = (double)t2_rd(t, (float)std::log((K + 10) / 1.0), P) * unit;
						if (b < 50 || !std::isfinite(b)) b = -1;
					}
					if (b < 0) {
						const auto it = std::lower_bound(shells.rbegin(), shells.rend(), K, std::greater<double>());
						if (it != shells.rend()) b = *it;
					}
					st[(size_t)x * t.ny + y] = (float)(b / 1.0);
				}
			}
		}
		if (penn) {
		{	// q icdf (full_penn.h:348-369)
			nm_set& s = set("/full_penn/q_icdf");
			std::vector<float>& st = o->store[4];
			st = s.data;
			const float unit = (float)(unit_value(s.unit) * 0.19519 * 1.0);
			for (auto& v : st) v = v * unit;
			orc_table& t = o->m.in_q;
			t.nx = (int32_t)s.dims[0]; t.ny = (int32_t)s.dims[1]; t.nz = (int32_t)s.dims[2];
			log_range(s.scales[0], lo, hi); set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			lin_range(s.scales[1], t.ny, lo, hi); set_axis(t.ny, lo, hi, false, t.y_min, t.y_step);
			lin_range(s.scales[2], t.nz, lo, hi); set_axis(t.nz, lo, hi, false, t.z_min, t.z_step);
			t.data = st.data();
		}
		{	// binding icdf (full_penn.h:374-402)
			nm_set& s = set("/ionization/binding_icdf");
			std::vector<float>& st = o->store[5];
			st = s.data;
			const float unit = (float)(unit_value(s.unit) / 1.0);
			for (auto& v : st) { float b = v * unit; if (b < 50 || !std::isfinite(b)) b = -1; v = b; }
			orc_table& t = o->m.in_binding;
			t.nx = (int32_t)s.dims[0]; t.ny = (int32_t)s.dims[1]; t.nz = (int32_t)s.dims[2];
			log_range(s.scales[0], lo, hi); set_axis(t.nx, lo, hi, true, t.x_min, t.x_step);
			log_range(s.scales[1], lo, hi); set_axis(t.ny, lo, hi, true, t.y_min, t.y_step);
			lin_range(s.scales[2], t.nz, lo, hi); set_axis(t.nz, lo, hi, false, t.z_min, t.z_step);
			t.data = st.data();
		}
		}
		o->m.fermi = (float)(fermi_q / 1.0);
		{
			auto it = f.props.find("band_gap");
			o->m.band_gap = (float)((it == f.props.end() ? -1.0 : it->second.first * unit_value(it->second.second)) / 1.0);
		}
		o->m.barrier = (float)(prop("barrier") / 1.0);
		o->m.phonon_loss = (float)(prop("phonon_loss") / 1.0);
		o->m.recoil_const = 2 * (float)(((6.2415e15 * 9.109383e-28) * 2) / prop("effective_A"));
		return o;
	} catch (std::exception const & e) {
		if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
		return nullptr;
	}
}
extern "C" const orc_material* orc_material_view(void* h) { return &static_cast<owned_material*>(h)->m; }
extern "C" void orc_set_physics(uint32_t bits) { g_phys = bits; }
extern "C" uint32_t orc_get_physics(void) { return g_phys; }
extern "C" void orc_material_free(void* h) { delete static_cast<owned_material*>(h); }

extern "C" float orc_table_get(const orc_table* t, int dims, float x, float y, float z)
{
	return dims == 1 ? t1_get(*t, x) : dims == 2 ? t2_get(*t, x, y) : t3_get(*t, x, y, z);
}
extern "C" float orc_table_rounddown(const orc_table* t, int dims, float x, float y, float z)
{
	return dims == 2 ? t2_rd(*t, x, y) : t3_rd(*t, x, y, z);
}

extern "C" void orc_propagate(const orc_geometry* g, const float* pos, const float* dir, float dist,
	int32_t ignore_tri, int32_t ignore_mat, float* out_dist, int32_t* out_tri)
{
	int t;
	propagate(g, { pos[0], pos[1], pos[2] }, { dir[0], dir[1], dir[2] }, dist, ignore_tri, ignore_mat, out_dist, &t);
	*out_tri = t;
}

extern "C" int orc_event(const orc_geometry* g, const orc_material* mats, int n_mat, int kind, int32_t tri,
	orc_rng* rng, float* state, int32_t* material, float* se, int32_t* status)
{
	(void)n_mat;
	manager mgr;
	mgr.p.push_back({ NO_EVENT, 0, *material, { state[0], state[1], state[2] }, { state[3], state[4], state[5] }, state[6], tri });
	if (kind == 3) {
		mgr.p[0].status = INTERSECT_EVENT;
		boundary(g, mats, mgr.p[0], rng);
	} else if (kind == 1) {
		inelastic(mats[*material], mgr, 0, rng);
	} else {
		elastic(mats[*material], mgr.p[0], rng);
	}
	const pstate& p = mgr.p[0];
	state[0] = p.pos.x; state[1] = p.pos.y; state[2] = p.pos.z;
	state[3] = p.dir.x; state[4] = p.dir.y; state[5] = p.dir.z; state[6] = p.E;
	*material = p.material;
	*status = p.status == DETECTED ? 1 : (p.status == TERMINATED ? 2 : 0);
	if (mgr.p.size() > 1) {
		const pstate& s = mgr.p[1];
		se[0] = s.pos.x; se[1] = s.pos.y; se[2] = s.pos.z;
		se[3] = s.dir.x; se[4] = s.dir.y; se[5] = s.dir.z; se[6] = s.E;
		return 1;
	}
	return 0;
}

static void write_record(char* out, const pstate& q, const int32_t* px)
{
	const float r[7] = { q.pos.x, q.pos.y, q.pos.z, q.dir.x, q.dir.y, q.dir.z, q.E };
	std::memcpy(out, r, 28);
	std::memcpy(out + 28, px, 8);
}

extern "C" int64_t orc_simulate(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events)
{
	(void)n_mat;
	orc_rng* rng = orc_rng_mt(seed);
	driver d{ g, mats, energy_threshold, rng, {} };
	int64_t written = 0, total = 0, events = 0;
	const char* in = static_cast<const char*>(pri);
	char* o = static_cast<char*>(out);
	for (int64_t i = 0; i < n_pri; ++i) {
		float f[7]; int32_t px[2];
		std::memcpy(f, in + 36 * i, 28);
		std::memcpy(px, in + 36 * i + 28, 8);
		d.run_one(f, events, [&](const pstate& q) {
			if (written < max_out) write_record(o + 36 * written++, q, px);
			++total;
		});
	}
	orc_rng_free(rng);
	*n_total = total;
	*n_events = events;
	return written;
}

extern "C" int64_t orc_simulate_deposits(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold, int n_threads,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events)
{
	(void)n_mat;
	if (n_threads < 1) n_threads = 1;
	std::vector<uint32_t> seeds;
	if (n_threads == 1) {
		seeds.push_back(seed);
	} else {
		orc_rng* master = orc_rng_mt(seed);
		for (int t = 0; t < n_threads; ++t) seeds.push_back(mt_next(master));
		orc_rng_free(master);
	}
	std::atomic<int64_t> cursor(0), written(0), events(0);
	const char* in = static_cast<const char*>(pri);
	char* o = static_cast<char*>(out);
	std::vector<std::thread> th;
	for (int t = 0; t < n_threads; ++t) {
		th.emplace_back([&, t]() {
			orc_rng* rng = orc_rng_mt(seeds[t]);
			driver d{ g, mats, energy_threshold, rng, {} };
			int64_t ev = 0;
			int32_t px[2] = { 0, 0 };
			// record of cpu_energydep.cpp:197-204: after.pos, before.E, before.E - after.E, pixel
			d.on_deposit = [&](const pstate& before, const pstate& after) {
				const int64_t w = written++;
				if (w < max_out) {
					const float r[5] = { after.pos.x, after.pos.y, after.pos.z, before.E, before.E - after.E };
					std::memcpy(o + 28 * w, r, 20);
					std::memcpy(o + 28 * w + 20, px, 8);
				}
			};
			for (;;) {
				const int64_t i = cursor++;
				if (i >= n_pri) break;
				if (n_threads > 1)
					mt_seed(rng, primary_seed(seed, i));
				float f[7];
				std::memcpy(f, in + 36 * i, 28);
				std::memcpy(px, in + 36 * i + 28, 8);
				d.run_one(f, ev, [](const pstate&) {});
			}
			events += ev;
			orc_rng_free(rng);
		});
	}
	for (auto& x : th) x.join();
	*n_total = written;
	*n_events = events;
	return std::min<int64_t>(written, max_out);
}

extern "C" int64_t orc_simulate_mt(const orc_geometry* g, const orc_material* mats, int n_mat,
	const void* pri, int64_t n_pri, uint32_t seed, float energy_threshold, int n_threads,
	void* out, int64_t max_out, int64_t* n_total, int64_t* n_events)
{
	(void)n_mat;
	if (n_threads < 1) n_threads = 1;
	orc_rng* master = orc_rng_mt(seed);
	std::vector<uint32_t> seeds;
	for (int t = 0; t < n_threads; ++t) seeds.push_back(mt_next(master));
	orc_rng_free(master);
	std::atomic<int64_t> cursor(0), written(0), total(0), events(0);
	std::mutex mu;
	const char* in = static_cast<const char*>(pri);
	char* o = static_cast<char*>(out);
	std::vector<std::thread> th;
	for (int t = 0; t < n_threads; ++t) {
		th.emplace_back([&, t]() {
			orc_rng* rng = orc_rng_mt(seeds[t]);
			driver d{ g, mats, energy_threshold, rng, {} };
			int64_t ev = 0;
			for (;;) {
				const int64_t i = cursor++;
				if (i >= n_pri) break;
				mt_seed(rng, primary_seed(seed, i));
				float f[7]; int32_t px[2];
				std::memcpy(f, in + 36 * i, 28);
				std::memcpy(px, in + 36 * i + 28, 8);
				d.run_one(f, ev, [&](const pstate& q) {
					++total;
					const int64_t w = written++;
					if (w < max_out) write_record(o + 36 * w, q, px);
				});
			}
			events += ev;
			orc_rng_free(rng);
		});
	}
	for (auto& x : th) x.join();
	*n_total = total;
	*n_events = events;
	return std::min<int64_t>(written, max_out);
}
