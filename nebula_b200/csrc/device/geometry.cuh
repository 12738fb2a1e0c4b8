// Octree ray walk and ray-triangle test, bit-exact with the reference CPU
// build on identical float32 inputs.
//
// The walk visits the same leaf cells in the same order as
// octree<gpu_flag>::propagate (reference geometry/octree.inl:33-192), because
// the returned distance accumulates float roundoff along that exact cell
// sequence.  Every float operation is written as an explicitly rounded
// intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn ...), so the compiler can neither
// contract a multiply-add into an FMA nor reorder: the result equals the
// x86-64 SSE evaluation of the reference's expressions, which is what the
// parity tests check.
//
// What is B200-specific is the data path: triangles are 64-byte records read
// with four 128-bit read-only loads (one L2 sector pair), their normal is
// precomputed, and the node array is read through the read-only cache; the
// whole structure stays L2-resident for the workloads of interest.
#pragma once
#include "../nbl_device_types.h"

namespace nbl {

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

// dot(a, b) = a.x*b.x + a.y*b.y + a.z*b.z evaluated left to right
// (reference common/vector_math.h:107-110)
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz)
{
	return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

// 10 * FLT_EPSILON (reference config/data_types.h:58)
#define NBL_EPS (10.0f * 1.1920928955078125e-07f)

struct TriHit { float t; };

// Moller-Trumbore as triangle::intersect_ray (reference core/triangle.inl:7-28):
// -1 on miss.
__device__ __forceinline__ float intersect_ray(const DevTriangle& T, float sx, float sy, float sz,
	float dx, float dy, float dz)
{
	// pvec = cross(dir, e2)
	const float px = fs(fm(dy, T.e2z), fm(dz, T.e2y));
	const float py = fs(fm(dz, T.e2x), fm(dx, T.e2z));
	const float pz = fs(fm(dx, T.e2y), fm(dy, T.e2x));
	const float det = dot3(T.e1x, T.e1y, T.e1z, px, py, pz);
	if (fabsf(det) < NBL_EPS)
		return -1.0f;
	const float tx = fs(sx, T.r0x), ty = fs(sy, T.r0y), tz = fs(sz, T.r0z);
	const float u = fd(dot3(tx, ty, tz, px, py, pz), det);
	if ((u < -NBL_EPS) || (u > 1.0f + NBL_EPS))
		return -1.0f;
	// qvec = cross(start - r0, e1)
	const float qx = fs(fm(ty, T.e1z), fm(tz, T.e1y));
	const float qy = fs(fm(tz, T.e1x), fm(tx, T.e1z));
	const float qz = fs(fm(tx, T.e1y), fm(ty, T.e1x));
	const float v = fd(dot3(dx, dy, dz, qx, qy, qz), det);
	if ((v < -NBL_EPS) || (fa(u, v) > 1.0f + NBL_EPS))
		return -1.0f;
	const float t = fd(dot3(T.e2x, T.e2y, T.e2z, qx, qy, qz), det);
	if (t < 0.0f)
		return -1.0f;
	return t;
}

__device__ __forceinline__ DevTriangle load_tri(const DevTriangle* __restrict__ tris, int i)
{
	const float4* p = reinterpret_cast<const float4*>(tris + i);
	const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), n = __ldg(p + 3);
	DevTriangle t;
	t.r0x = a.x; t.r0y = a.y; t.r0z = a.z; t.mat_in = __float_as_int(a.w);
	t.e1x = b.x; t.e1y = b.y; t.e1z = b.z; t.mat_out = __float_as_int(b.w);
	t.e2x = c.x; t.e2y = c.y; t.e2z = c.z; t.pad0 = 0;
	t.nx = n.x; t.ny = n.y; t.nz = n.z; t.pad1 = 0;
	return t;
}

// octree::in_domain (reference geometry/octree.inl:25-30)
__device__ __forceinline__ bool in_domain(const DevGeometry& g, float x, float y, float z)
{
	return (x > fs(g.cx, g.hx)) && (x < fa(g.cx, g.hx)) && (y > fs(g.cy, g.hy)) && (y < fa(g.cy, g.hy))
		&& (z > fs(g.cz, g.hz)) && (z < fa(g.cz, g.hz));
}

// Where a walk stands between leaf cells: the current point, the distance
// left, the location code of the cell it is about to enter and the cells
// walked so far.  A walk cut short after some cells resumes from this state
// with exactly the float values it would have carried on with.
struct WalkState {
	float cx, cy, cz, to_go;
	uint64_t location;
	int steps;
};

__device__ __forceinline__ WalkState walk_start(float sx, float sy, float sz, float distance)
{
	WalkState w;
	w.cx = sx; w.cy = sy; w.cz = sz; w.to_go = distance;
	w.location = 1;
	w.steps = 0;
	return w;
}

// Status of a walk that stopped at its cell budget (propagate_cells).
#define NBL_WALK_PENDING (-3)

// Nearest triangle hit within `distance` along a (normalised) direction,
// ignoring `ignore_tri` and triangles whose outgoing material equals
// `ignore_mat`, walking from state `w` (walk_start for a new walk).  Returns
// the triangle index (or -1) and the distance (or `distance` itself when
// nothing is hit).  A walk longer than `max_steps` leaf cells in all stops
// early and reports -2 (the host counts these as errors; the reference has no
// such bound).  With `max_cells` > 0, a walk that has not ended after
// `max_cells` cells in this call returns NBL_WALK_PENDING with `w` holding
// where it stands; calling again with that state continues the same cell
// sequence with the same float values.
__device__ __forceinline__ int propagate_cells(const DevGeometry& g, WalkState& w,
	float dx, float dy, float dz, float distance, int ignore_tri, int ignore_mat, float& out_dist,
	int max_cells = 0, int max_steps = 1 << 20)
{
	const int32_t* __restrict__ od = g.octree;
	float cx = w.cx, cy = w.cy, cz = w.cz;
	float to_go = w.to_go;
	uint64_t location = w.location;
	int steps = w.steps;
	int cells = 0;
	do {
		// Cell centre update of the reference, c += (aw * h) * (bit - 0.5)
		// with aw = 2^-level: both products are exact (power-of-two
		// scalings of h, far from underflow), so the offset is carried as
		// +-h 2^-(level+1), halved per level, and only the addition rounds.
		float ax = g.cx, ay = g.cy, az = g.cz, aw = 1.0f;
		float ox = fm(g.hx, 0.5f), oy = fm(g.hy, 0.5f), oz = fm(g.hz, 0.5f);
		int index = 0;
		// descend to the current location code from the root
		for (int i = 60 - __clzll((long long)location); i >= 0; i -= 3) {
			const unsigned int octant = (unsigned int)(location >> i) & 7u;
			index = __ldg(od + index + octant);
			ax = fa(ax, (octant & 1u) ? ox : -ox);
			ay = fa(ay, (octant & 2u) ? oy : -oy);
			az = fa(az, (octant & 4u) ? oz : -oz);
			aw = fm(aw, 0.5f);
			ox = fm(ox, 0.5f); oy = fm(oy, 0.5f); oz = fm(oz, 0.5f);
		}
		// continue to the leaf that contains the current position
		while (index >= 0) {
			const bool bx = cx > ax, by = cy > ay, bz = cz > az;
			const unsigned int octant = (bx ? 1u : 0u) | (by ? 2u : 0u) | (bz ? 4u : 0u);
			location = (location << 3) | octant;
			index = __ldg(od + index + octant);
			ax = fa(ax, bx ? ox : -ox);
			ay = fa(ay, by ? oy : -oy);
			az = fa(az, bz ? oz : -oz);
			aw = fm(aw, 0.5f);
			ox = fm(ox, 0.5f); oy = fm(oy, 0.5f); oz = fm(oz, 0.5f);
		}
		index = -index;

		// exit distance through the leaf's faces (AABB_intersect, octree.inl:212-220)
		float intersect;
		int target;
		{
			const float hx = fm(aw, g.hx), hy = fm(aw, g.hy), hz = fm(aw, g.hz);
			const float tx = fd(fs(fa(ax, copysignf(fa(hx, NBL_EPS), dx)), cx), dx);
			const float ty = fd(fs(fa(ay, copysignf(fa(hy, NBL_EPS), dy)), cy), dy);
			const float tz = fd(fs(fa(az, copysignf(fa(hz, NBL_EPS), dz)), cz), dz);
			if ((tx < ty) && (tx < tz)) { intersect = tx; target = -1; }
			else if ((ty < tx) && (ty < tz)) { intersect = ty; target = -2; }
			else { intersect = tz; target = -4; }
		}

		// triangles of the leaf
		for (;;) {
			const int ti = __ldg(od + index);
			++index;
			if (ti < 0)
				break;
			if (ti == ignore_tri)
				continue;
			const DevTriangle T = load_tri(g.tris, ti);
			const int mat_out = dot3(T.nx, T.ny, T.nz, dx, dy, dz) < 0.0f ? T.mat_in : T.mat_out;
			if (mat_out == ignore_mat)
				continue;
			const float t = intersect_ray(T, cx, cy, cz, dx, dy, dz);
			if ((t > 0.0f) && (t <= fa(intersect, NBL_EPS))) {
				intersect = t;
				target = ti;
			}
		}

		if (intersect >= to_go) {
			out_dist = distance;
			return -1;
		} else if (target >= 0) {
			out_dist = fa(fs(distance, to_go), intersect);
			return target;
		}
		to_go = fs(to_go, intersect);
		cx = fa(cx, fm(dx, intersect));
		cy = fa(cy, fm(dy, intersect));
		cz = fa(cz, fm(dz, intersect));

		// neighbour cell by location-code arithmetic
		const unsigned int mask = (unsigned int)(-target);
		unsigned int value;
		if (mask == 1u) value = (dx >= 0.0f) ? 0u : 1u;
		else if (mask == 2u) value = (dy >= 0.0f) ? 0u : 2u;
		else value = (dz >= 0.0f) ? 0u : 4u;
		while (location > 1) {
			if ((location & mask) == value) {
				location ^= mask;
				break;
			}
			location >>= 3;
		}
		if (++steps > max_steps) {
			out_dist = distance;
			return -2;
		}
		if (++cells == max_cells && location > 1) {
			w.cx = cx; w.cy = cy; w.cz = cz; w.to_go = to_go;
			w.location = location;
			w.steps = steps;
			out_dist = distance;
			return NBL_WALK_PENDING;
		}
	} while (location > 1);
	out_dist = distance;
	return -1;
}

// The whole walk in one call (octree<gpu_flag>::propagate).
__device__ __forceinline__ int propagate(const DevGeometry& g, float sx, float sy, float sz,
	float dx, float dy, float dz, float distance, int ignore_tri, int ignore_mat, float& out_dist,
	int max_steps = 1 << 20)
{
	WalkState w = walk_start(sx, sy, sz, distance);
	return propagate_cells(g, w, dx, dy, dz, distance, ignore_tri, ignore_mat, out_dist, 0, max_steps);
}

}  // namespace nbl
