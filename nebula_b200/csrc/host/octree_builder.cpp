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
//   * the reference reaches its tree by inserting the triangles one at a
//     time; the same tree is built here top-down, level by level, on all host
//     threads (the argument is at the build loop);
//   * breadth-first node order; a leaf stores its triangle indices then -1, an
//     inner node eight child offsets, negated for leaf children; triangles
//     are renumbered in order of first appearance in the leaves (:252-352).
// The triangle-box overlap is the separating-axis test of Akenine-Moller,
// "Fast 3D triangle-box overlap testing" (J. Graphics Tools 6(1), 2001):
// nine edge-cross-axis tests, the box-vs-triangle-bounds test and the
// plane-vs-box test, written here from that description.
#include "internal.hpp"

#include <cmath>
#include <algorithm>
#include <atomic>
#include <iostream>
#include <thread>

namespace nbl {
namespace {

struct F3 { float x, y, z; };
inline F3 f3add(F3 a, F3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline F3 f3sub(F3 a, F3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline F3 f3scale(float s, F3 a) { return { s * a.x, s * a.y, s * a.z }; }

struct Tri {
	F3 r0, r1, r2;   // r1 = r0 + e1, r2 = r0 + e2 (triangle::r1/r2, core/triangle.inl:35-42)
};

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

// Duplicate classes (triangle::perfect_overlap: the same three vertices in
// any order): the reference drops a triangle from a leaf that already holds
// one of its duplicates, and duplicates overlap exactly the same cells, so
// only the lowest-index member of a class ever appears in a leaf.  Found once
// by sorting canonical vertex keys (-0 folded into +0, as float == does;
// triangles with a NaN vertex equal nothing and stay).
std::vector<uint8_t> duplicate_flags(const std::vector<Tri>& tris, size_t& n_dup)
{
	struct Key { float v[9]; int32_t idx; };
	auto canon = [](float x) { return x == 0.0f ? 0.0f : x; };
	std::vector<Key> keys;
	keys.reserve(tris.size());
	for (size_t i = 0; i < tris.size(); ++i) {
		const Tri& t = tris[i];
		F3 p[3] = { t.r0, t.r1, t.r2 };
		bool nan = false;
		for (auto& q : p) {
			q = { canon(q.x), canon(q.y), canon(q.z) };
			nan |= q.x != q.x || q.y != q.y || q.z != q.z;
		}
		if (nan) continue;
		auto less = [](const F3& a, const F3& b) {
			return a.x < b.x || (a.x == b.x && (a.y < b.y || (a.y == b.y && a.z < b.z)));
		};
		std::sort(p, p + 3, less);
		Key k;
		for (int j = 0; j < 3; ++j) { k.v[3 * j] = p[j].x; k.v[3 * j + 1] = p[j].y; k.v[3 * j + 2] = p[j].z; }
		k.idx = (int32_t)i;
		keys.push_back(k);
	}
	auto key_less = [](const Key& a, const Key& b) {
		for (int j = 0; j < 9; ++j)
			if (a.v[j] != b.v[j]) return a.v[j] < b.v[j];
		return a.idx < b.idx;
	};
	std::sort(keys.begin(), keys.end(), key_less);
	std::vector<uint8_t> dup(tris.size(), 0);
	n_dup = 0;
	for (size_t i = 1; i < keys.size(); ++i) {
		bool same = true;
		for (int j = 0; j < 9 && same; ++j) same = keys[i].v[j] == keys[i - 1].v[j];
		if (same) { dup[keys[i].idx] = 1; ++n_dup; }
	}
	return dup;
}

// get_octant_center_halfsize (octree_builder.cpp:44-62)
inline void octant_box(int octant, F3 c, F3 h, F3& oc, F3& oh)
{
	oh = f3scale(0.5f, h);
	oc.x = c.x + (float)(((octant & 1) << 1) - 1) * oh.x;
	oc.y = c.y + (float)((octant & 2) - 1) * oh.y;
	oc.z = c.z + (float)(((octant & 4) >> 1) - 1) * oh.z;
}

inline bool overlaps(const Tri& t, F3 c, F3 h)
{
	const double dc[3] = { c.x, c.y, c.z };
	const double dh[3] = { 1.01 * h.x, 1.01 * h.y, 1.01 * h.z };
	return tri_box_overlap(dc, dh, t);
}

struct Node {
	int32_t first_child = -1;   // index of 8 consecutive children, -1 for a leaf
	int32_t depth = 0;
	F3 c{ 0, 0, 0 }, h{ 0, 0, 0 };
	std::vector<int32_t> tris;  // increasing triangle index
};

// Run f(0..n-1) on `threads` threads (work handed out one index at a time).
template<class F> void parallel_for(size_t n, unsigned threads, F f)
{
	if (n == 0) return;
	threads = (unsigned)std::min<size_t>(threads, n);
	if (threads <= 1) {
		for (size_t i = 0; i < n; ++i) f(i);
		return;
	}
	std::atomic<size_t> next{ 0 };
	std::vector<std::thread> pool;
	for (unsigned t = 0; t < threads; ++t)
		pool.emplace_back([&] {
			for (size_t i; (i = next.fetch_add(1)) < n;)
				f(i);
		});
	for (auto& th : pool) th.join();
}
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

	std::vector<Tri> tris((size_t)n);
	F3 lo{ 0, 0, 0 }, hi{ 0, 0, 0 };
	for (int64_t i = 0; i < n; ++i) {
		const F3 r0{ in[i].r0[0], in[i].r0[1], in[i].r0[2] };
		const F3 e1{ in[i].e1[0], in[i].e1[1], in[i].e1[2] };
		const F3 e2{ in[i].e2[0], in[i].e2[1], in[i].e2[2] };
		Tri t{ r0, f3add(r0, e1), f3add(r0, e2) };
		tris[i] = t;
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
	size_t n_dup = 0;
	const std::vector<uint8_t> dup = duplicate_flags(tris, n_dup);
	if (n_dup)
		std::clog << "WARNING: ignored " << n_dup << " duplicate triangle(s)" << std::endl;
	const unsigned threads = std::max(1u, std::thread::hardware_concurrency());

	// The reference inserts triangles one by one and splits a leaf when it
	// holds more than split_count (octree_child::insert, :93-126); the tree it
	// ends with is the one built top-down here: a node's triangles are those
	// of its parent that overlap its inflated box (in index order), and it
	// splits when they are more than split_count below max_depth.  Nodes are
	// created level by level, children in octant order, which is the
	// breadth-first order the linearisation uses.
	std::vector<Node> nodes(1);
	nodes[0].c = center; nodes[0].h = halfsize;
	{
		// the root always splits (octree_builder.cpp:160-169, 200-208)
		std::vector<int32_t> all;
		all.reserve((size_t)n);
		std::vector<uint8_t> in_root((size_t)n, 0);
		parallel_for(((size_t)n + 65535) / 65536, threads, [&](size_t chunk) {
			const size_t a = chunk * 65536, e = std::min<size_t>((size_t)n, a + 65536);
			for (size_t ti = a; ti < e; ++ti)
				in_root[ti] = !dup[ti] && overlaps(tris[ti], center, halfsize);
		});
		for (int32_t ti = 0; ti < (int32_t)n; ++ti)
			if (in_root[ti]) all.push_back(ti);
		nodes[0].tris.swap(all);
	}
	std::vector<int32_t> level{ 0 };
	bool root = true;
	while (!level.empty()) {
		// which nodes of this level split
		std::vector<int32_t> splitting;
		for (int32_t nd : level)
			if (root || ((int)nodes[nd].tris.size() > split_count && nodes[nd].depth < max_depth))
				splitting.push_back(nd);
		root = false;
		if (splitting.empty())
			break;
		const size_t first = nodes.size();
		nodes.resize(first + 8 * splitting.size());
		for (size_t k = 0; k < splitting.size(); ++k) {
			Node& p = nodes[splitting[k]];
			p.first_child = (int32_t)(first + 8 * k);
			for (int o = 0; o < 8; ++o) {
				Node& ch = nodes[first + 8 * k + o];
				ch.depth = p.depth + 1;
				octant_box(o, p.c, p.h, ch.c, ch.h);
			}
		}
		// children's triangle lists: one task per parent for the small ones
		// (all eight children), (octant, chunk) tasks for the large ones
		const size_t chunk = 8192;
		struct Task { size_t k; int octant; size_t a, e; };
		std::vector<Task> tasks;
		std::vector<std::vector<std::vector<int32_t>>> parts(8 * splitting.size());
		for (size_t k = 0; k < splitting.size(); ++k) {
			const size_t m = nodes[splitting[k]].tris.size();
			if (m <= chunk) {
				tasks.push_back({ k, -1, 0, m });
				continue;
			}
			const size_t nch = (m + chunk - 1) / chunk;
			for (int o = 0; o < 8; ++o) {
				parts[8 * k + o].resize(nch);
				for (size_t c = 0; c < nch; ++c)
					tasks.push_back({ k, o, c * chunk, std::min(m, (c + 1) * chunk) });
			}
		}
		parallel_for(tasks.size(), threads, [&](size_t i) {
			const Task& t = tasks[i];
			const Node& p = nodes[splitting[t.k]];
			if (t.octant < 0) {
				for (int o = 0; o < 8; ++o) {
					Node& ch = nodes[first + 8 * t.k + o];
					for (int32_t ti : p.tris)
						if (overlaps(tris[ti], ch.c, ch.h))
							ch.tris.push_back(ti);
				}
				return;
			}
			const Node& ch = nodes[first + 8 * t.k + t.octant];
			std::vector<int32_t>& out = parts[8 * t.k + t.octant][t.a / chunk];
			for (size_t j = t.a; j < t.e; ++j)
				if (overlaps(tris[p.tris[j]], ch.c, ch.h))
					out.push_back(p.tris[j]);
		});
		std::vector<int32_t> next;
		next.reserve(8 * splitting.size());
		for (size_t k = 0; k < splitting.size(); ++k) {
			for (int o = 0; o < 8; ++o) {
				Node& ch = nodes[first + 8 * k + o];
				for (auto& part : parts[8 * k + o])
					ch.tris.insert(ch.tris.end(), part.begin(), part.end());
				next.push_back((int32_t)(first + 8 * k + o));
			}
		}
		parallel_for(splitting.size(), threads, [&](size_t k) {
			std::vector<int32_t>().swap(nodes[splitting[k]].tris);   // inner nodes hold none
		});
		level.swap(next);
	}
	const size_t n_nodes = nodes.size();   // creation order is breadth-first
	HostGeometry g;
	std::vector<int32_t> remap(n, -1);
	for (size_t nd = 0; nd < n_nodes; ++nd) {
		if (nodes[nd].first_child >= 0)
			continue;
		for (int32_t ti : nodes[nd].tris) {
			if (remap[ti] >= 0)
				continue;
			remap[ti] = (int32_t)g.tris.size();
			g.tris.push_back(in[ti]);
		}
	}
	// node offsets in breadth-first order (the creation order), then every
	// node writes its own words
	std::vector<int64_t> start(n_nodes + 1, 0);
	for (size_t i = 0; i < n_nodes; ++i)
		start[i + 1] = start[i] + (nodes[i].first_child < 0 ? (int64_t)nodes[i].tris.size() + 1 : 8);
	require(start[n_nodes] < (int64_t)1 << 31, "octree is too large");
	g.octree.resize((size_t)start[n_nodes]);
	parallel_for((n_nodes + 4095) / 4096, threads, [&](size_t c) {
		const size_t a = c * 4096, e = std::min(n_nodes, a + 4096);
		for (size_t nd = a; nd < e; ++nd) {
			int32_t* w = g.octree.data() + start[nd];
			if (nodes[nd].first_child < 0) {
				for (int32_t ti : nodes[nd].tris)
					*w++ = remap[ti];
				*w = -1;
			} else {
				for (int o = 0; o < 8; ++o) {
					const int32_t ch = nodes[nd].first_child + o;
					const int32_t s = (int32_t)start[ch];
					w[o] = nodes[ch].first_child < 0 ? -s : s;
				}
			}
		}
	});
	g.center[0] = center.x; g.center[1] = center.y; g.center[2] = center.z;
	g.halfsize[0] = halfsize.x; g.halfsize[1] = halfsize.y; g.halfsize[2] = halfsize.z;
	g.max_extent = max_extent_of(g.halfsize);
	return g;
}

}  // namespace nbl
