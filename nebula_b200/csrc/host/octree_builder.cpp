// Host octree builder producing the reference's linearised layout.
//
// Same construction rules as octree_builder (reference
// geometry/octree/octree_builder.cpp:93-352), so that a mesh gives the same
// node array and triangle order, and therefore bit-identical octree walks:
//   * root box: bounds of the triangles' corners (r0, r0+e1, r0+e2 in float)
//     with 1 nm added to the half size (:171-209);
//   * a triangle enters a cell when it overlaps the cell inflated by 1.01
//     (:31-42), tested in double;
//   * a leaf with more than `split_count` triangles splits while its depth is
//     below `max_depth` (:112-113; the reference fixes 16 and 21,
//     octree_builder.h:157-158); duplicates within a leaf are dropped (:103-109);
//   * breadth-first node order; a leaf stores its triangle indices then -1, an
//     inner node eight child offsets, negated for leaf children; triangles
//     are renumbered in order of first appearance in the leaves (:252-352).
// The triangle-box overlap is the separating-axis test of Akenine-Moller,
// "Fast 3D triangle-box overlap testing" (J. Graphics Tools 6(1), 2001):
// nine edge-cross-axis tests, the box-vs-triangle-bounds test and the
// plane-vs-box test, written here from that description.
#include "internal.hpp"

#include <cmath>
#include <deque>
#include <algorithm>
#include <iostream>

namespace nbl {
namespace {

struct F3 { float x, y, z; };
inline F3 f3add(F3 a, F3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline F3 f3sub(F3 a, F3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline F3 f3scale(float s, F3 a) { return { s * a.x, s * a.y, s * a.z }; }

struct Tri {
	F3 r0, r1, r2;   // r1 = r0 + e1, r2 = r0 + e2 (triangle::r1/r2, core/triangle.inl:35-42)
};

inline bool f3eq(F3 a, F3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// triangle::perfect_overlap (core/triangle.inl:89-103)
bool perfect_overlap(const Tri& a, const Tri& b)
{
	return (f3eq(a.r0, b.r0) && f3eq(a.r1, b.r1) && f3eq(a.r2, b.r2)) ||
		(f3eq(a.r0, b.r1) && f3eq(a.r1, b.r2) && f3eq(a.r2, b.r0)) ||
		(f3eq(a.r0, b.r2) && f3eq(a.r1, b.r0) && f3eq(a.r2, b.r1)) ||
		(f3eq(a.r0, b.r0) && f3eq(a.r1, b.r2) && f3eq(a.r2, b.r1)) ||
		(f3eq(a.r0, b.r1) && f3eq(a.r1, b.r0) && f3eq(a.r2, b.r2)) ||
		(f3eq(a.r0, b.r2) && f3eq(a.r1, b.r1) && f3eq(a.r2, b.r0));
}

// Separating-axis triangle / axis-aligned box test in double.
bool tri_box_overlap(const double c[3], const double h[3], const Tri& t)
{
	const double v[3][3] = {
		{ t.r0.x - c[0], t.r0.y - c[1], t.r0.z - c[2] },
		{ t.r1.x - c[0], t.r1.y - c[1], t.r1.z - c[2] },
		{ t.r2.x - c[0], t.r2.y - c[1], t.r2.z - c[2] } };
	double e[3][3];
	for (int k = 0; k < 3; ++k) {
		e[0][k] = v[1][k] - v[0][k];
		e[1][k] = v[2][k] - v[1][k];
		e[2][k] = v[0][k] - v[2][k];
	}
	// Axis (unit_i x edge): project two vertices (the third projects like the
	// one that shares the edge) and compare with the box's projected radius.
	// Coordinates (j, k) are the two axes other than i.
	auto axis_test = [&](const double* ed, int j, int k, int va, int vb) -> bool {
		const double a = ed[k], b = ed[j];
		const double pa = a * v[va][j] - b * v[va][k];
		const double pb = a * v[vb][j] - b * v[vb][k];
		const double mn = std::min(pa, pb), mx = std::max(pa, pb);
		const double rad = std::fabs(a) * h[j] + std::fabs(b) * h[k];
		return !(mn > rad || mx < -rad);
	};
	// edge 0 (v1 - v0): vertices 0 and 2; edge 1 (v2 - v1): 0 and 1 for x/y,
	// edge 2 (v0 - v2): 0 and 1
	if (!axis_test(e[0], 1, 2, 0, 2)) return false;   // x
	if (!axis_test(e[0], 2, 0, 0, 2)) return false;   // y
	if (!axis_test(e[0], 0, 1, 1, 2)) return false;   // z
	if (!axis_test(e[1], 1, 2, 0, 2)) return false;
	if (!axis_test(e[1], 2, 0, 0, 2)) return false;
	if (!axis_test(e[1], 0, 1, 0, 1)) return false;
	if (!axis_test(e[2], 1, 2, 0, 1)) return false;
	if (!axis_test(e[2], 2, 0, 0, 1)) return false;
	if (!axis_test(e[2], 0, 1, 1, 2)) return false;
	// box vs triangle bounds
	for (int k = 0; k < 3; ++k) {
		const double mn = std::min(std::min(v[0][k], v[1][k]), v[2][k]);
		const double mx = std::max(std::max(v[0][k], v[1][k]), v[2][k]);
		if (mn > h[k] || mx < -h[k])
			return false;
	}
	// triangle plane vs box, with the box corners taken relative to vertex 0
	// (the paper's 2001-06 revision of the plane test)
	const double n[3] = {
		e[0][1] * e[1][2] - e[0][2] * e[1][1],
		e[0][2] * e[1][0] - e[0][0] * e[1][2],
		e[0][0] * e[1][1] - e[0][1] * e[1][0] };
	double vmin[3], vmax[3];
	for (int k = 0; k < 3; ++k) {
		const double o = v[0][k];
		if (n[k] > 0) { vmin[k] = -h[k] - o; vmax[k] = h[k] - o; }
		else { vmin[k] = h[k] - o; vmax[k] = -h[k] - o; }
	}
	if (n[0] * vmin[0] + n[1] * vmin[1] + n[2] * vmin[2] > 0)
		return false;
	return n[0] * vmax[0] + n[1] * vmax[1] + n[2] * vmax[2] >= 0;
}

struct Node {
	int32_t first_child = -1;   // index of 8 consecutive children, -1 for a leaf
	int32_t depth = 0;
	std::vector<int32_t> tris;
};

struct Builder {
	std::vector<Tri> tris;
	std::vector<Node> nodes;
	int max_depth, split_count;
	size_t duplicates = 0;

	static void octant_box(int octant, F3 c, F3 h, F3& oc, F3& oh)
	{
		// get_octant_center_halfsize (octree_builder.cpp:44-62)
		oh = f3scale(0.5f, h);
		oc.x = c.x + (float)(((octant & 1) << 1) - 1) * oh.x;
		oc.y = c.y + (float)((octant & 2) - 1) * oh.y;
		oc.z = c.z + (float)(((octant & 4) >> 1) - 1) * oh.z;
	}
	bool overlaps(int32_t ti, F3 c, F3 h) const
	{
		const double dc[3] = { c.x, c.y, c.z };
		const double dh[3] = { 1.01 * h.x, 1.01 * h.y, 1.01 * h.z };
		return tri_box_overlap(dc, dh, tris[ti]);
	}
	void split(int32_t node, F3 c, F3 h)
	{
		const int32_t first = (int32_t)nodes.size();
		const int32_t depth = nodes[node].depth + 1;
		nodes.resize(nodes.size() + 8);
		for (int o = 0; o < 8; ++o)
			nodes[first + o].depth = depth;
		std::vector<int32_t> mine;
		mine.swap(nodes[node].tris);
		nodes[node].first_child = first;
		for (int o = 0; o < 8; ++o) {
			F3 oc, oh;
			octant_box(o, c, h, oc, oh);
			for (int32_t ti : mine)
				insert(first + o, ti, oc, oh);
		}
	}
	// octree_child::insert (octree_builder.cpp:93-126)
	void insert(int32_t node, int32_t ti, F3 c, F3 h)
	{
		if (!overlaps(ti, c, h))
			return;
		if (nodes[node].first_child < 0) {
			for (int32_t o : nodes[node].tris)
				if (perfect_overlap(tris[ti], tris[o])) {
					++duplicates;
					return;
				}
			nodes[node].tris.push_back(ti);
			if ((int)nodes[node].tris.size() > split_count && nodes[node].depth < max_depth)
				split(node, c, h);
		} else {
			const int32_t first = nodes[node].first_child;
			for (int o = 0; o < 8; ++o) {
				F3 oc, oh;
				octant_box(o, c, h, oc, oh);
				insert(first + o, ti, oc, oh);
			}
		}
	}
};

}  // namespace

float max_extent_of(const float h[3])
{
	// 2 * magnitude(halfsize), CPU magnitude = sqrt(x*x + y*y + z*z) (vector_math.h:116-127)
	return 2 * std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
}

HostGeometry build_octree(const nbl_triangle* in, int64_t n, int max_depth, int split_count)
{
	require(n > 0, "geometry has no triangles");
	require(n < (int64_t)1 << 31, "too many triangles for a linearized octree");
	if (max_depth <= 0) max_depth = 21;
	if (split_count <= 0) split_count = 16;
	require(max_depth <= 21, "max_depth must be <= 21 (63-bit location codes)");

	Builder b;
	b.max_depth = max_depth;
	b.split_count = split_count;
	b.tris.resize(n);
	F3 lo{ 0, 0, 0 }, hi{ 0, 0, 0 };
	for (int64_t i = 0; i < n; ++i) {
		const F3 r0{ in[i].r0[0], in[i].r0[1], in[i].r0[2] };
		const F3 e1{ in[i].e1[0], in[i].e1[1], in[i].e1[2] };
		const F3 e2{ in[i].e2[0], in[i].e2[1], in[i].e2[2] };
		Tri t{ r0, f3add(r0, e1), f3add(r0, e2) };
		b.tris[i] = t;
		// triangle::AABB_min/max (triangle.inl:44-72) with std::min/max
		const F3 tmin{ std::min(std::min(t.r0.x, t.r1.x), t.r2.x), std::min(std::min(t.r0.y, t.r1.y), t.r2.y),
			std::min(std::min(t.r0.z, t.r1.z), t.r2.z) };
		const F3 tmax{ std::max(std::max(t.r0.x, t.r1.x), t.r2.x), std::max(std::max(t.r0.y, t.r1.y), t.r2.y),
			std::max(std::max(t.r0.z, t.r1.z), t.r2.z) };
		if (i == 0) { lo = tmin; hi = tmax; }
		else {
			lo = { std::min(lo.x, tmin.x), std::min(lo.y, tmin.y), std::min(lo.z, tmin.z) };
			hi = { std::max(hi.x, tmax.x), std::max(hi.y, tmax.y), std::max(hi.z, tmax.z) };
		}
	}
	const F3 center = f3scale(0.5f, f3add(lo, hi));
	const F3 halfsize = f3add(f3scale(0.5f, f3sub(hi, lo)), F3{ 1, 1, 1 });

	// root with eight leaf children (octree_builder.cpp:160-169, 200-208)
	b.nodes.reserve(1024);
	b.nodes.emplace_back();
	b.nodes[0].first_child = 1;
	b.nodes.resize(9);
	for (int o = 1; o < 9; ++o) b.nodes[o].depth = 1;
	for (int32_t ti = 0; ti < (int32_t)n; ++ti) {
		if (!b.overlaps(ti, center, halfsize))
			continue;
		for (int o = 0; o < 8; ++o) {
			F3 oc, oh;
			Builder::octant_box(o, center, halfsize, oc, oh);
			b.insert(1 + o, ti, oc, oh);
		}
	}
	if (b.duplicates)
		std::clog << "WARNING: ignored " << b.duplicates << " duplicate triangle(s)" << std::endl;

	// breadth-first order
	std::vector<int32_t> order;
	order.reserve(b.nodes.size());
	{
		std::deque<int32_t> q;
		q.push_back(0);
		while (!q.empty()) {
			const int32_t nd = q.front();
			q.pop_front();
			order.push_back(nd);
			if (b.nodes[nd].first_child >= 0)
				for (int o = 0; o < 8; ++o)
					q.push_back(b.nodes[nd].first_child + o);
		}
	}
	HostGeometry g;
	std::vector<int32_t> remap(n, -1);
	for (int32_t nd : order) {
		if (b.nodes[nd].first_child >= 0)
			continue;
		for (int32_t ti : b.nodes[nd].tris) {
			if (remap[ti] >= 0)
				continue;
			remap[ti] = (int32_t)g.tris.size();
			g.tris.push_back(in[ti]);
		}
	}
	std::vector<int64_t> start(b.nodes.size(), 0);
	for (int32_t nd : order) {
		start[nd] = (int64_t)g.octree.size();
		if (b.nodes[nd].first_child < 0) {
			for (int32_t ti : b.nodes[nd].tris)
				g.octree.push_back(remap[ti]);
			g.octree.push_back(-1);
		} else {
			g.octree.insert(g.octree.end(), 8, 0);
		}
	}
	require(g.octree.size() < (size_t)1 << 31, "octree is too large");
	for (int32_t nd : order) {
		if (b.nodes[nd].first_child < 0)
			continue;
		for (int o = 0; o < 8; ++o) {
			const int32_t ch = b.nodes[nd].first_child + o;
			const int32_t s = (int32_t)start[ch];
			g.octree[start[nd] + o] = b.nodes[ch].first_child < 0 ? -s : s;
		}
	}
	g.center[0] = center.x; g.center[1] = center.y; g.center[2] = center.z;
	g.halfsize[0] = halfsize.x; g.halfsize[1] = halfsize.y; g.halfsize[2] = halfsize.z;
	g.max_extent = max_extent_of(g.halfsize);
	return g;
}

}  // namespace nbl
