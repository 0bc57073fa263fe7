// Device helpers shared by the Brownian-dynamics kernels.
//
// Arithmetic that decides a discrete outcome (Morton keys, the pairlist
// distance test, periodic wrapping) or that must reproduce the reference's
// per-pair float results uses the explicitly rounded intrinsics
// (__fadd_rn, __fmul_rn, __fdiv_rn, __fsqrt_rn, __frcp_rn). The compiler never
// contracts those into FMAs, so each operation rounds exactly as the
// reference's float code does, independent of -fmad.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mb2 {

constexpr uint32_t kInvalidCell = 0xFFFFFFFFu;  // ZOrderNeighbor.h stencil padding
// AnalyticalPairTerm bits (src/Interactions/Nonbonded/Pairwise.h:19-27).
constexpr uint32_t kTermCoulomb = 1u << 0;
constexpr uint32_t kTermDebyeHuckel = 1u << 1;
constexpr uint32_t kTermOnck = 1u << 2;
constexpr uint32_t kTermGaussian = 1u << 3;
constexpr uint32_t kTermSoftcore = 1u << 4;
constexpr uint32_t kTermTabulated = 1u << 5;    // PAIR_TERM_TABULATED (Pairwise.h:25)
constexpr uint32_t kTermAnalytical = 0x1Fu;     // every analytical bit
constexpr float kCoulomb = 332.0636f;           // constants::COULOMB (src/Constants.h:24)
constexpr uint32_t kTableShift = 8;             // kPairTableShift (Pairwise.h:30)
constexpr uint32_t kFlagRbAttached = 1u << 2;   // FLAG_RB_ATTACHED (DeviceParticle.h)
constexpr uint32_t kBdStream = 0x5324120u;      // BDIntegrate::rng_stream (BD.h:25)
constexpr uint32_t kOrientBit = 0x80000000u;    // neighbour entry: pair stored j -> i

// Orthogonal periodic box as the kernels see it.
struct Box {
	float origin[3];
	float size[3];
	float inv[3];   // RN(1/size); equals the reference's 1.0f / l
	float half[3];  // 0.5f * size (exact)
	int periodic[3];
};

// PeriodicBox::wrap_diff_scalar (src/System/PeriodicBox.h:453-461), rounded
// exactly as the reference: image = floor(x * (1/l)); x -= image * l; then
// x >= l/2 -> x - l.
__device__ __forceinline__ float wrap_diff_scalar(float x, float l, float inv, float half) {
	const float image = floorf(__fmul_rn(x, inv));
	x = __fsub_rn(x, __fmul_rn(image, l));
	return x >= half ? __fsub_rn(x, l) : x;
}

// PeriodicBox::wrap_scalar (PeriodicBox.h:445-451).
__device__ __forceinline__ float wrap_scalar(float x, float o, float l, float inv) {
	const float image = floorf(__fmul_rn(__fsub_rn(x, o), inv));
	return __fsub_rn(x, __fmul_rn(image, l));
}

__device__ __forceinline__ float3 wrap_diff(const Box& b, float dx, float dy, float dz) {
	if (b.periodic[0]) dx = wrap_diff_scalar(dx, b.size[0], b.inv[0], b.half[0]);
	if (b.periodic[1]) dy = wrap_diff_scalar(dy, b.size[1], b.inv[1], b.half[1]);
	if (b.periodic[2]) dz = wrap_diff_scalar(dz, b.size[2], b.inv[2], b.half[2]);
	return make_float3(dx, dy, dz);
}

// Correctly rounded square root by Markstein's method (P. W. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Develop. 34(1), 1990): the hardware estimate y of
// 1/sqrt(a) (PTX rsqrt.approx), g = a y, and one Newton-Raphson correction
// g + (a - g g) y / 2 whose residual a fused multiply-add computes exactly.
// Equal to __fsqrt_rn on [2^-60, FLT_MAX], every float checked on the device
// by mb2_selftest_sqrt; the pair kernel takes it only on squared distances
// inside its window (from about 1e-12 up).
__device__ __forceinline__ float sqrt_rn_nr(float a) {
	float y;
	asm("rsqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(a));
	const float g = __fmul_rn(a, y);
	const float h = __fmul_rn(0.5f, y);
	return __fmaf_rn(__fmaf_rn(-g, g, a), h, g);
}

// The reference's pair test as a window on the squared distance d2: it skips
// a pair when dist = RN(sqrt(d2)) < 1e-6 or RN(dist * dist) > cutoff_sq
// (cutoff_sq > 0). Both sides are monotone in d2, so the test is d2 < lo or
// d2 > hi exactly, with lo and hi found on the host (dist_window).
struct DistWindow {
	float lo, hi;
};
DistWindow dist_window(float cutoff_sq);

// Vector3_t::length2: x*x + y*y + z*z, left to right, no contraction.
__device__ __forceinline__ float len2(float x, float y, float z) {
	return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}

// MortonCode::splitBy3 / compactBy3 (MortonCode.h:157-182).
__host__ __device__ __forceinline__ uint32_t split_by3(uint32_t a) {
	uint32_t x = a & 1023u;
	x = (x | x << 16) & 0x30000ffu;
	x = (x | x << 8) & 0x300f00fu;
	x = (x | x << 4) & 0x30c30c3u;
	x = (x | x << 2) & 0x9249249u;
	return x;
}

__host__ __device__ __forceinline__ uint32_t compact_by3(uint32_t x) {
	x &= 0x09249249u;
	x = (x ^ (x >> 2)) & 0x030c30c3u;
	x = (x ^ (x >> 4)) & 0x0300f00fu;
	x = (x ^ (x >> 8)) & 0x030000ffu;
	x = (x ^ (x >> 16)) & 0x000003ffu;
	return x;
}

// One Morton coordinate (MortonCode.h:97-131): IEEE division by the clamped
// range, scale by 1023, clamp, truncate.
__device__ __forceinline__ uint32_t morton_coord(float p, float lo, float range) {
	const float normalized = __fdiv_rn(__fsub_rn(p, lo), range);
	const float s = fminf(fmaxf(__fmul_rn(normalized, 1023.0f), 0.0f), 1023.0f);
	return static_cast<uint32_t>(s);
}

// Tabulated potential (TabulatedPotential.h:8-14) in kernel form.
struct Table {
	const float* pot;
	float step_inv;
	uint32_t size;
	float start;
	int periodic;
};

// TabulatedPotential::compute (TabulatedPotential.h:19-52), same rounding.
// Returns (force magnitude, energy).
__device__ __forceinline__ float2 table_lookup(const float* pot, int size, float start,
											   float step_inv, int periodic, float x) {
	float w = __fmul_rn(__fsub_rn(x, start), step_inv);
	int home = static_cast<int>(floorf(w));
	w = __fsub_rn(w, static_cast<float>(home));
	if (periodic) {
		home %= size;
		if (home < 0) home += size;
	} else {
		if (home >= size - 1) return make_float2(0.0f, pot[size - 1]);
		if (home < 0) home = 0;
	}
	int home1 = periodic ? (home + 1) % size : home + 1;
	if (!periodic && home1 >= size) home1 = size - 1;
	const float u0 = pot[home];
	const float du = __fsub_rn(pot[home1], u0);
	return make_float2(__fmul_rn(-du, step_inv), __fadd_rn(__fmul_rn(du, w), u0));
}

// openrand::Philox generate/round (src/PatchOperation/Random/philox.h:97-139).
__device__ __forceinline__ uint4 philox4x32_10(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2,
											   uint32_t c3) {
	uint32_t k0 = static_cast<uint32_t>(seed >> 32), k1 = static_cast<uint32_t>(seed);
#pragma unroll
	for (int r = 0; r < 10; ++r) {
		if (r > 0) {
			k0 += 0x9E3779B9u;
			k1 += 0xBB67AE85u;
		}
		const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
		const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
		const uint32_t n0 = hi1 ^ c1 ^ k0;
		const uint32_t n2 = hi0 ^ c3 ^ k1;
		c0 = n0;
		c1 = lo1;
		c2 = n2;
		c3 = lo0;
	}
	return make_uint4(c0, c1, c2, c3);
}

// BaseRNG::u01<float, uint32_t> (base_state.h:299-305): x * 2^-32 + 2^-33.
__device__ __forceinline__ float u01(uint32_t x) {
	return __fadd_rn(__fmul_rn(__uint2float_rn(x), 2.3283064365386963e-10f), 1.1641532182693481e-10f);
}

// Vector atomic add of a float4 into global memory (sm_90+ `red.v4.f32`).
__device__ __forceinline__ void red_add_v4(float4* p, float a, float b, float c, float d) {
	asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c),
				 "f"(d)
				 : "memory");
}

__device__ __forceinline__ void red_add_v2(float2* p, float a, float b) {
	asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}

// Type id packed into the .w lane of a sorted position.
__device__ __forceinline__ int type_of(const float4& p) { return __float_as_int(p.w); }

}  // namespace mb2
