// Counter-based random numbers for the transport kernels.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): a keyed bijection of a 128-bit counter, ten rounds of
// two 32x32->64 multiplies with Weyl-sequence key bumps.  Written here from
// the published description.
//
// Stream layout.  Every electron's random numbers are a pure function of
//   key     = run seed (64 bit)
//   counter = ((event << 8) | block, primary tag, lineage id lo, lineage id hi)
// so trajectories do not depend on which thread, slot or kernel ran them.
// That is what lets the batched persistent kernel reproduce the plain kernel
// exactly, and lets the adjoint replay a primary from its seed instead of
// storing event logs.  `event` counts free flights of this electron; block 0
// feeds the flight, blocks 1.. the interaction that ends it.
#pragma once
#include <stdint.h>
#include "../nbl_device_types.h"

namespace nbl {

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
	return __umulhi(a, b);
#else
	return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], PhiloxKey k)
{
	const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
	const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
	uint32_t k0 = k.k0, k1 = k.k1;
#pragma unroll
	for (int r = 0; r < 10; ++r) {
		const uint32_t hi0 = mulhi32(M0, c[0]), lo0 = M0 * c[0];
		const uint32_t hi1 = mulhi32(M1, c[2]), lo1 = M1 * c[2];
		const uint32_t n0 = hi1 ^ c[1] ^ k0;
		const uint32_t n2 = hi0 ^ c[3] ^ k1;
		c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
		k0 += W0; k1 += W1;
	}
}

// 32 random bits -> float strictly inside (0, 1): the top 24 bits plus half a
// step, so log(u) is always finite.
__host__ __device__ __forceinline__ float u01_open(uint32_t x)
{
	return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// Child lineage id from the parent's id and the parent's event counter at the
// spawning event (a parent spawns at most one secondary per event, so the
// pair is unique).  A 64-bit finaliser (splitmix64's) spreads it; the low bit
// is forced so no child id equals the primary's id 0.
__host__ __device__ __forceinline__ uint64_t child_lineage(uint64_t parent, uint32_t parent_event)
{
	uint64_t z = parent * 0x9E3779B97F4A7C15ull + ((uint64_t)parent_event << 1) + 0xD1B54A32D192ED03ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	z ^= z >> 31;
	return z | 1ull;
}

// Uniform draws for one electron within one event.
struct PhiloxStream {
	PhiloxKey key;
	uint32_t c0base, tag, lin_lo, lin_hi;
	uint32_t buf[4];
	uint32_t n;   // draws taken in this event

	__device__ __forceinline__ void init(PhiloxKey k, uint32_t event, uint32_t block0, uint32_t tag_,
		uint64_t lineage)
	{
		key = k;
		c0base = (event << 8) | block0;
		tag = tag_;
		lin_lo = (uint32_t)lineage;
		lin_hi = (uint32_t)(lineage >> 32);
		n = 0;
	}
	__device__ __forceinline__ float unit()
	{
		const uint32_t j = n & 3u;
		if (j == 0) {
			buf[0] = c0base + (n >> 2); buf[1] = tag; buf[2] = lin_lo; buf[3] = lin_hi;
			philox4x32_10(buf, key);
		}
		++n;
		return u01_open(buf[j]);
	}
};

// Uniform draws from a caller-supplied list (known-answer tests of the
// physics against the oracle with identical inputs).
struct ListStream {
	const float* u;
	uint32_t n, cap;
	__device__ __forceinline__ float unit()
	{
		const float v = n < cap ? u[n] : 0.5f;
		++n;
		return v;
	}
};

}  // namespace nbl
