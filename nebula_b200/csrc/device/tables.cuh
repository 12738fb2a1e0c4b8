// Cross-section table lookups, bit-exact with the reference CPU build.
//
// Uniform-grid linear / bilinear / trilinear interpolation with the index
// clamped to [0, n-2] (linear extrapolation outside the grid), and the
// round-down variant clamped to [0, n-1] (reference common/util/table_1D.inl:66-81,
// table_2D.inl:73-104, table_3D.inl:79-122).  Operation order and rounding
// are the reference's, written with explicit round-to-nearest intrinsics.
//
// Tables are small (<= 1 MB per material) and read through the read-only
// path, so they stay resident in L1/L2 across the whole run.
#pragma once
#include "../nbl_device_types.h"
#include "geometry.cuh"

namespace nbl {

__device__ __forceinline__ int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

// floorr (reference common/scalar_math.h:43-55): round toward -inf to int
__device__ __forceinline__ int floor_to_int(float x) { return __float2int_rd(x); }

__device__ __forceinline__ float tab(const DevTable& t, int i, int j, int k)
{
	return __ldg(t.data + ((size_t)i * t.ny + j) * t.nz + k);
}

__device__ __forceinline__ float table1_get(const DevTable& t, float x)
{
	const float xi = fm(fs(x, t.x_min), t.x_step);
	const int lo = clampi(floor_to_int(xi), 0, t.nx - 2);
	const float a = __ldg(t.data + lo), b = __ldg(t.data + lo + 1);
	const float f = fs(xi, (float)lo);
	return fa(fm(fs(1.0f, f), a), fm(f, b));
}

__device__ __forceinline__ float table2_get(const DevTable& t, float x, float y)
{
	const float xi = fm(fs(x, t.x_min), t.x_step);
	const float yi = fm(fs(y, t.y_min), t.y_step);
	const int lx = clampi(floor_to_int(xi), 0, t.nx - 2);
	const int ly = clampi(floor_to_int(yi), 0, t.ny - 2);
	const float v00 = tab(t, lx, ly, 0), v10 = tab(t, lx + 1, ly, 0);
	const float v01 = tab(t, lx, ly + 1, 0), v11 = tab(t, lx + 1, ly + 1, 0);
	const float fx = fs(xi, (float)lx), fy = fs(yi, (float)ly);
	const float gx = fs(1.0f, fx), gy = fs(1.0f, fy);
	// ((gx*gy)*v00 + (fx*gy)*v10) + (gx*fy)*v01) + (fx*fy)*v11
	float r = fm(fm(gx, gy), v00);
	r = fa(r, fm(fm(fx, gy), v10));
	r = fa(r, fm(fm(gx, fy), v01));
	r = fa(r, fm(fm(fx, fy), v11));
	return r;
}

__device__ __forceinline__ float table2_rounddown(const DevTable& t, float x, float y)
{
	const float xi = fm(fs(x, t.x_min), t.x_step);
	const float yi = fm(fs(y, t.y_min), t.y_step);
	return tab(t, clampi(floor_to_int(xi), 0, t.nx - 1), clampi(floor_to_int(yi), 0, t.ny - 1), 0);
}

__device__ __forceinline__ float table3_get(const DevTable& t, float x, float y, float z)
{
	const float xi = fm(fs(x, t.x_min), t.x_step);
	const float yi = fm(fs(y, t.y_min), t.y_step);
	const float zi = fm(fs(z, t.z_min), t.z_step);
	const int lx = clampi(floor_to_int(xi), 0, t.nx - 2);
	const int ly = clampi(floor_to_int(yi), 0, t.ny - 2);
	const int lz = clampi(floor_to_int(zi), 0, t.nz - 2);
	const float v000 = tab(t, lx, ly, lz), v100 = tab(t, lx + 1, ly, lz);
	const float v010 = tab(t, lx, ly + 1, lz), v110 = tab(t, lx + 1, ly + 1, lz);
	const float v001 = tab(t, lx, ly, lz + 1), v101 = tab(t, lx + 1, ly, lz + 1);
	const float v011 = tab(t, lx, ly + 1, lz + 1), v111 = tab(t, lx + 1, ly + 1, lz + 1);
	const float fx = fs(xi, (float)lx), fy = fs(yi, (float)ly), fz = fs(zi, (float)lz);
	const float gx = fs(1.0f, fx), gy = fs(1.0f, fy), gz = fs(1.0f, fz);
	// each term is ((a*b)*c)*v, summed left to right (table_3D.inl:100-109)
	float r = fm(fm(fm(gx, gy), gz), v000);
	r = fa(r, fm(fm(fm(fx, gy), gz), v100));
	r = fa(r, fm(fm(fm(gx, fy), gz), v010));
	r = fa(r, fm(fm(fm(fx, fy), gz), v110));
	r = fa(r, fm(fm(fm(gx, gy), fz), v001));
	r = fa(r, fm(fm(fm(fx, gy), fz), v101));
	r = fa(r, fm(fm(fm(gx, fy), fz), v011));
	r = fa(r, fm(fm(fm(fx, fy), fz), v111));
	return r;
}

__device__ __forceinline__ float table3_rounddown(const DevTable& t, float x, float y, float z)
{
	const float xi = fm(fs(x, t.x_min), t.x_step);
	const float yi = fm(fs(y, t.y_min), t.y_step);
	const float zi = fm(fs(z, t.z_min), t.z_step);
	return tab(t, clampi(floor_to_int(xi), 0, t.nx - 1), clampi(floor_to_int(yi), 0, t.ny - 1),
		clampi(floor_to_int(zi), 0, t.nz - 1));
}

}  // namespace nbl
