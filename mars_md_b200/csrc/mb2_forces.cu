// Tabulated pair, bond and angle forces.
//
// Pair forces replace PairNonbondedComputer's tabulated term
// (src/Interactions/Nonbonded/Pairwise.h:214-304): per pair, wrapped r_ij,
// |r_ij| by sqrt, skip |r| < 1e-6 and |r|^2 > rc^2, table lookup,
// f = r_ij / |r_ij| * F, -f on the pair's first (smaller original) index and
// +f on the second, half the energy to each. Each pair's float result is
// rounded exactly as the reference rounds it (explicit _rn intrinsics, the
// same orientation via bit 31 of the list entry); only the order in which
// the per-particle sums accumulate differs.
//
// Table lookup (TabulatedPotential::compute, TabulatedPotential.h:19-52) is
// precomputed per bin: bin_force[k] = -(U[k+1] - U[k]) * step_inv rounded as
// the reference rounds it, and 0 for the last bin (the reference's
// home >= size-1 branch); bin_energy[k] = (U[k], U[k+1] - U[k]). A lookup is
// then w = (x - start) * step_inv, home = clamp(floor(w), 0, size-1) and one
// load (through L1) -- bit-identical to the reference's branches.
//
// Layout: G lanes own one row (sorted particle i) of the sliced-ELL half list
// and H = 32 / G rows share a warp, so one warp load of entries k..k+G-1 of
// H rows is one 128-byte line. Lanes gather sorted float4 positions (type id
// in .w), accumulate -f for i in registers and scatter +f to j with one
// vector `red.global.add.v4.f32` (energy rides in .w). The row's i force is
// reduced across its G lanes with shuffles and added with one more red.
//
// FP64: total pair energy and virial are reduced in double on the device
// (per-thread double, block reduction, one double atomic per block).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "marsb200.h"
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

__device__ __forceinline__ void block_add_f64(double a, double b, double* out) {
	__shared__ double red_a[32], red_b[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
		b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
	}
	if (lane == 0) {
		red_a[warp] = a;
		red_b[warp] = b;
	}
	__syncthreads();
	if (warp == 0) {
		const int nw = blockDim.x >> 5;
		a = lane < nw ? red_a[lane] : 0.0;
		b = lane < nw ? red_b[lane] : 0.0;
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
			b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
		}
		if (lane == 0) {
			atomicAdd(out, a);
			atomicAdd(out + 1, b);
		}
	}
}

// Minimum image of one component for an all-periodic box, same rounding as
// PeriodicBox::wrap_diff_scalar.
__device__ __forceinline__ float wrap1(float x, float l, float inv, float half) {
	const float image = floorf(__fmul_rn(x, inv));
	x = __fsub_rn(x, __fmul_rn(image, l));
	return x >= half ? __fsub_rn(x, l) : x;
}

// wrap1 for a component known to lie in [-l/2, l/2] (rows inside the box,
// below): the reference's image floor(RN(x / l)) is 0 for x >= 0 and -1 for
// x < 0, so its result is x, or RN(RN(x + l) - l) (which is >= l/2 before the
// second rounding, so the reference takes that branch too), picked by the
// sign bit. -0 takes the second form: RN(RN(-0 + l) - l) = +0, as the
// reference's floor(-0) = -0 gives. (A negative x so small that x / l
// underflows, |x| < 2^-149 l, would keep x where this gives +0.)
__device__ __forceinline__ float wrap_inner(float x, float l, float negl) {
	const float w = __fadd_rn(__fadd_rn(x, l), negl);
	return __float_as_int(x) < 0 ? w : x;
}

// math::sinh_minus_x / x_cosh_minus_sinh (src/Types/Math.h:199-216): the
// reference's series below |x| = 1, the direct difference above.
__device__ __forceinline__ float sinh_minus_x(float x) {
	if (x >= 1.0f || x <= -1.0f) return __fsub_rn(sinhf(x), x);
	constexpr float c0 = static_cast<float>(1.0 / 6), c1 = static_cast<float>(1.0 / 120),
					c2 = static_cast<float>(1.0 / 5040), c3 = static_cast<float>(1.0 / 362880);
	const float w = __fmul_rn(x, x);
	return __fmul_rn(__fmul_rn(x, w),
					 __fadd_rn(c0, __fmul_rn(w, __fadd_rn(c1, __fmul_rn(w, __fadd_rn(c2, __fmul_rn(w, c3)))))));
}

__device__ __forceinline__ float x_cosh_minus_sinh(float x) {
	if (x >= 1.0f || x <= -1.0f) return __fsub_rn(__fmul_rn(x, coshf(x)), sinhf(x));
	constexpr float c0 = static_cast<float>(1.0 / 3), c1 = static_cast<float>(1.0 / 30),
					c2 = static_cast<float>(1.0 / 840), c3 = static_cast<float>(1.0 / 45360);
	const float w = __fmul_rn(x, x);
	return __fmul_rn(__fmul_rn(x, w),
					 __fadd_rn(c0, __fmul_rn(w, __fadd_rn(c1, __fmul_rn(w, __fadd_rn(c2, __fmul_rn(w, c3)))))));
}

// OnckElecPotential::dielectric and dielectric_deriv
// (src/Interactions/Nonbonded/Columb.h:68-84).
__device__ __forceinline__ float onck_dielectric(float r, const PairSolvent& s) {
	const float v = __fdiv_rn(r, s.onck_two_z);
	if (v < 1e-5f) return __fdiv_rn(__fmul_rn(__fmul_rn(s.onck_sz, v), v), 3.0f);
	const float sh = sinhf(v);
	return __fdiv_rn(__fmul_rn(__fmul_rn(s.onck_sz, sinh_minus_x(v)), __fadd_rn(sh, v)),
					 __fmul_rn(sh, sh));
}

__device__ __forceinline__ float onck_dielectric_deriv(float r, const PairSolvent& s) {
	const float v = __fdiv_rn(r, s.onck_two_z);
	if (v < 1e-5f) return __fdiv_rn(__fmul_rn(s.onck_sz, v), __fmul_rn(3.0f, s.onck_z));
	const float sh = sinhf(v);
	return __fdiv_rn(__fmul_rn(__fmul_rn(s.onck_sz, v), x_cosh_minus_sinh(v)),
					 __fmul_rn(__fmul_rn(__fmul_rn(s.onck_z, sh), sh), sh));
}

// The analytical terms of PairNonbondedComputer::operator()
// (src/Interactions/Nonbonded/Pairwise.h:246-283), added in its order into
// the pair's force magnitude (-dU/dr) and energy: Coulomb (Columb.h:11-20),
// Debye-Hueckel (Columb.h:29-42), Onck (Columb.h:86-97), Gaussian
// (Pairwise.h:55-68), softcore (Pairwise.h:82-100; its dU/dr / r becomes
// -dU/dr by -F r). d = |r|, d2v = r . r of the wrapped vector.
__device__ __forceinline__ void analytic_terms(uint32_t terms, const PairTermRef& a,
											   const PairSolvent& s, float d, float d2v,
											   float& fm, float& en) {
	if (terms & kTermCoulomb) {
		const float inv_d2 = __frcp_rn(__fmul_rn(d, d));
		const float inv_d = __frcp_rn(d);
		fm = __fadd_rn(fm, __fmul_rn(__fmul_rn(a.qq, inv_d2), kCoulomb));
		en = __fadd_rn(en, __fmul_rn(__fmul_rn(a.qq, inv_d), kCoulomb));
	}
	if (terms & kTermDebyeHuckel) {
		const float inv_r = __frcp_rn(d);
		const float screen = expf(__fdiv_rn(-d, s.dh_len));
		const float e = __fmul_rn(__fmul_rn(a.a_dh, screen), inv_r);
		fm = __fadd_rn(fm, __fmul_rn(e, __fadd_rn(inv_r, s.dh_inv_len)));
		en = __fadd_rn(en, e);
	}
	if (terms & kTermOnck) {
		const float r = d < 1e-2f ? 1e-2f : d;
		const float screen = expf(__fmul_rn(-s.onck_kappa, r));
		const float eps = onck_dielectric(r, s);
		const float er = __fmul_rn(eps, r);
		const float as = __fmul_rn(a.a_onck, screen);
		const float eps_p = onck_dielectric_deriv(r, s);
		const float t1 = __fdiv_rn(s.onck_kappa, er);
		const float t2 = __fdiv_rn(__fadd_rn(__fmul_rn(eps_p, r), eps),
								   __fmul_rn(__fmul_rn(__fmul_rn(eps, eps), r), r));
		fm = __fadd_rn(fm, __fmul_rn(as, __fadd_rn(t1, t2)));
		en = __fadd_rn(en, __fdiv_rn(as, er));
	}
	if (terms & kTermGaussian) {
		const float g2 = __fmul_rn(d, d);
		if (!(s.g_cut2 > 0.0f && g2 > s.g_cut2)) {
			const float e = __fmul_rn(s.g_amp, expf(__fmul_rn(-g2, s.g_inv_s2)));
			fm = __fadd_rn(fm, __fmul_rn(__fmul_rn(__fmul_rn(2.0f, d), e), s.g_inv_s2));
			en = __fadd_rn(en, e);
		}
	}
	if (terms & kTermSoftcore) {
		const float d6 = __fmul_rn(__fmul_rn(d2v, d2v), d2v);
		const float d6_2 = __fmul_rn(d6, d6);
		const float rad6_2 = __fmul_rn(a.rad6, a.rad6);
		const float f = __fmul_rn(__fmul_rn(-12.0f, a.eps),
								  __fsub_rn(__fdiv_rn(rad6_2, __fmul_rn(d6_2, d2v)),
											__fdiv_rn(a.rad6, __fmul_rn(d6, d2v))));
		float e = 0.0f;
		if (d6 < a.rad6)
			e = __fadd_rn(__fmul_rn(a.eps, __fsub_rn(__fdiv_rn(rad6_2, d6_2),
													 __fdiv_rn(__fmul_rn(2.0f, a.rad6), d6))),
						  a.eps);
		fm = __fadd_rn(fm, __fmul_rn(-f, d));
		en = __fadd_rn(en, e);
	}
}

// The table references of one row's type: the full 16-byte reference per j
// type, or (kUniform) the shared start / step_inv / last with a 4-byte offset
// per j type, one broadcast shared-memory word for the warp instead of a
// 128-bit load.
template <bool kUniform>
struct TableRow {
	const PairTableRef* row;
	const int* off;
	PairTableRef u;
	__device__ __forceinline__ PairTableRef operator()(int tj) const {
		if (kUniform) {
			PairTableRef t = u;
			t.offset = off[tj];
			return t;
		}
		return row[tj];
	}
};

// One pair of the half list, rounded as the reference rounds it. flip
// (bit 31 of the entry): the reference orients the pair j -> i. With kTerms,
// the analytical terms of the type pair come first, then the table.
//
// The x and y components go through sm_100's packed FP32 instructions
// (__fadd2_rn / __fmul2_rn: two IEEE round-to-nearest operations each, so
// every value is the scalar one bit for bit), z stays scalar. npi = (-pi.x,
// -pi.y); a - b is computed as a + (-b) and b * l as -(b * (-l)), both exact
// rewrites. The i-force is accumulated negated (nxy, nz): -(a - h) = (-a) + h
// in round-to-nearest, so the caller's negation at the end gives the same sum.
template <bool kEnergy, bool kAllPeriodic, bool kTerms, bool kInner, class TRow>
__device__ __forceinline__ void pair_scalar(const float4& pi, float2 npi, const float4& pj,
											uint32_t j, uint32_t flip,
											const TRow& trow, const float* bin_f,
											const float2* bin_e, const PairTermRef* arow,
											const PairSolvent& sv, const Box& box,
											const DistWindow& win, float4* force, float2& nxy, float& nz,
											float& fe, double& e_acc, double& w_acc) {
	// r = wrap_diff(pos[second] - pos[first])
	// (pi - pj is exactly -(pj - pi) in round-to-nearest, so a sign flip
	// suffices; a multiply by -1 is that flip, on the FMA pipe)
	const float sgn = __uint_as_float(flip | 0x3F800000u);  // +1, or -1 when flipped
	float2 dxy = __fmul2_rn(__fadd2_rn(make_float2(pj.x, pj.y), npi), make_float2(sgn, sgn));
	float dz = __fmul_rn(__fsub_rn(pj.z, pi.z), sgn);
	if (kInner) {
		// the row lies inside the box: |d| <= l/2 on every axis
		const float2 l = make_float2(box.size[0], box.size[1]);
		const float2 w = __fadd2_rn(__fadd2_rn(dxy, l), make_float2(-l.x, -l.y));
		dxy.x = __float_as_int(dxy.x) < 0 ? w.x : dxy.x;
		dxy.y = __float_as_int(dxy.y) < 0 ? w.y : dxy.y;
		dz = wrap_inner(dz, box.size[2], -box.size[2]);
	} else if (kAllPeriodic) {
		// wrap1 on x and y: image = floor(d / l); d -= image * l; d >= l/2 -> d - l.
		const float2 negl = make_float2(-box.size[0], -box.size[1]);
		float2 img = __fmul2_rn(dxy, make_float2(box.inv[0], box.inv[1]));
		img.x = floorf(img.x);
		img.y = floorf(img.y);
		dxy = __fadd2_rn(dxy, __fmul2_rn(img, negl));
		const float2 up = __fadd2_rn(dxy, negl);
		dxy.x = dxy.x >= box.half[0] ? up.x : dxy.x;
		dxy.y = dxy.y >= box.half[1] ? up.y : dxy.y;
		dz = wrap1(dz, box.size[2], box.inv[2], box.half[2]);
	} else {
		const float3 r = wrap_diff(box, dxy.x, dxy.y, dz);
		dxy = make_float2(r.x, r.y);
		dz = r.z;
	}
	const float dx = dxy.x, dy = dxy.y;
	const float2 sq = __fmul2_rn(dxy, dxy);
	const float d2v = __fadd_rn(__fadd_rn(sq.x, sq.y), __fmul_rn(dz, dz));
	// The reference's test (dist < 1e-6 or RN(dist^2) > cutoff_sq skips the
	// pair) taken exactly on d2v, before the root: lanes beyond the cutoff,
	// and whole warps in the rows' far ends, leave here. Inside the window the
	// root below is the correctly rounded one.
	if (d2v > win.hi || d2v < win.lo) return;
	const float dist = sqrt_rn_nr(d2v);
	const PairTableRef t = trow(type_of(pj));
	float fm = 0.0f, e = 0.0f;
	if (kTerms) {
		const PairTermRef a = arow[type_of(pj)];
		if (a.terms == 0u && t.offset < 0) return;
		analytic_terms(a.terms, a, sv, dist, d2v, fm, e);
		if (t.offset >= 0) {
			const float w = __fmul_rn(__fsub_rn(dist, t.start), t.step_inv);
			const float wf = floorf(w);
			const int home = min(max(static_cast<int>(wf), 0), t.last);
			fm = __fadd_rn(fm, bin_f[t.offset + home]);
			if (kEnergy) {
				const float2 ue = bin_e[t.offset + home];
				e = __fadd_rn(e, __fadd_rn(__fmul_rn(ue.y, __fsub_rn(w, wf)), ue.x));
			}
		}
	} else {
		if (t.offset < 0) return;
		const float w = __fmul_rn(__fsub_rn(dist, t.start), t.step_inv);
		// floor to int in one conversion (equal to int(floorf(w)) for every w)
		const int home = min(max(__float2int_rd(w), 0), t.last);
		fm = bin_f[t.offset + home];
		if (kEnergy) {
			const float2 ue = bin_e[t.offset + home];
			e = __fadd_rn(__fmul_rn(ue.y, __fsub_rn(w, floorf(w))), ue.x);
		}
	}
	const float inv = __frcp_rn(dist);
	// f = unit * F acts on the pair's second particle, -f on its first.
	const float2 gxy = __fmul2_rn(__fmul2_rn(make_float2(inv, inv), dxy), make_float2(fm, fm));
	const float gx = gxy.x, gy = gxy.y;
	const float gz = __fmul_rn(__fmul_rn(inv, dz), fm);
	float half = 0.0f;
	if (kEnergy) {
		half = __fmul_rn(e, 0.5f);
		e_acc += static_cast<double>(e);
		w_acc += static_cast<double>(gx) * dx + static_cast<double>(gy) * dy +
				 static_cast<double>(gz) * dz;
	}
	// j is the pair's second particle unless the pair is stored flipped.
	const float2 hxy = __fmul2_rn(gxy, make_float2(sgn, sgn));
	const float hz = __fmul_rn(gz, sgn);
	red_add_v4(&force[j], hxy.x, hxy.y, hz, half);
	nxy = __fadd2_rn(nxy, hxy);
	nz = __fadd_rn(nz, hz);
	fe += half;
}

// Box of a row: one box for the whole list, or the box of the row's system
// (batched replicas: system id in the top bits of the sorted key).
struct OneBox {
	Box b;
	// Displacement track (may be null) and list_rc (1 + 2^-20) + kInnerSafety.
	const unsigned int* d2max;
	float margin;
	__device__ __forceinline__ const Box& row(uint32_t) const { return b; }
};
// Added to the list radius in the inner-row test: covers kTrackBand and the
// rounding of the displacement and of the walk's radius test.
constexpr float kInnerSafety = 1.0f;
struct SystemBoxes {
	const Box* __restrict__ boxes;
	const uint32_t* __restrict__ keys;
	int sys_shift;
	__device__ __forceinline__ Box row(uint32_t i) const { return boxes[keys[i] >> sys_shift]; }
};

// Resident 256-thread blocks per SM each pair-kernel variant is compiled for.
// The force-only tabulated kernel is bound by issue and gather latency: 8
// blocks (32 registers, full occupancy) ran it 6 % faster than the 40
// registers it takes unbounded, in spite of a few bytes of spill (none in the
// uniform-table variant); the energy and analytical variants need their
// registers. The batched variant (box per row) runs best at 6 blocks (40
// registers, a few bytes of spill): 1.06 -> 1.02 ms per batched step against
// 48 registers, and 1.08 at 8 blocks, where it spills 60 bytes.
template <bool kEnergy, bool kTerms, bool kOneBox>
constexpr int pair_min_blocks() {
	return !kOneBox ? 6 : (kTerms ? 3 : (kEnergy ? 5 : 8));
}

template <int G, bool kEnergy, bool kAllPeriodic, bool kTerms, bool kUniform, class BoxSrc>
__global__ void __launch_bounds__(
	256, pair_min_blocks<kEnergy, kTerms, std::is_same<BoxSrc, OneBox>::value>()) pair_force_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ nbr,
	const uint32_t* __restrict__ row_len, uint32_t n, uint32_t cap, int T,
	const PairTableRef* __restrict__ refs_g, const int* __restrict__ offs_g, PairTableRef uref,
	const float* __restrict__ force_g,
	const float2* __restrict__ energy_g, uint32_t total_bins,
	const PairTermRef* __restrict__ terms_g, PairSolvent sv, BoxSrc boxes, DistWindow win,
	float4* force, double* __restrict__ ev) {
	constexpr int H = 32 / G;
	// The per-type-pair references (T*T, 16 B each) are staged in shared
	// memory. On the one-box path the per-bin force (and energy) tables are
	// read through L1 (a few KB, hot in every SM's L1) instead of a copy per
	// block: that leaves the L1 to the neighbour-position gathers, whose
	// latency bounds this kernel (1.63 -> 1.51 ms per 2 M-bead launch; asking
	// the driver for the largest L1 carve-out on top made it slower, 1.80 ms).
	// The batched path (many small systems, short rows, fewer resident warps)
	// is faster with the tables in shared memory.
	constexpr bool kStage = !std::is_same<BoxSrc, OneBox>::value;
	extern __shared__ float4 smem4[];
	PairTableRef* refs = reinterpret_cast<PairTableRef*>(smem4);
	int* soff = reinterpret_cast<int*>(smem4);
	for (int k = threadIdx.x; k < T * T; k += blockDim.x) {
		if (kUniform) soff[k] = offs_g[k];
		else refs[k] = refs_g[k];
	}
	const float* __restrict__ bin_f = force_g;
	const float2* __restrict__ bin_e = energy_g;
	if (kStage) {
		float* sf = reinterpret_cast<float*>(refs + T * T);
		float2* se = reinterpret_cast<float2*>(sf + ((total_bins + 1) & ~1u));
		for (uint32_t k = threadIdx.x; k < total_bins; k += blockDim.x) {
			sf[k] = force_g[k];
			if (kEnergy) se[k] = energy_g[k];
		}
		bin_f = sf;
		bin_e = se;
	}
	__syncthreads();

	const int sub = threadIdx.x & (G - 1);  // lane within the row's group
	const uint32_t i = blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
	const bool valid = i < n;
	const Box& box = boxes.row(valid ? i : 0u);
	const float4 pi = valid ? sorted_pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
	TableRow<kUniform> trow;
	trow.row = refs + (valid ? type_of(pi) : 0) * T;
	trow.off = soff + (valid ? type_of(pi) : 0) * T;
	trow.u = uref;
	const PairTermRef* arow = kTerms ? terms_g + (valid ? type_of(pi) : 0) * T : nullptr;
	const uint32_t cnt = valid ? row_len[i] : 0u;
	// Entry k of row i: ((i / H) * cap + k) * H + i % H.
	const uint32_t* col = nbr + (static_cast<size_t>(i / H) * cap) * H + (i % H);
	const float2 npi = make_float2(-pi.x, -pi.y);
	float2 nxy = make_float2(0.0f, 0.0f);  // minus the i-force, x and y
	float nz = 0.0f, fe = 0.0f;
	double e_acc = 0.0, w_acc = 0.0;
	// A row inside the box (all-periodic box, displacement tracked): every
	// neighbour's minimum image is its plain difference, |d| <= list radius +
	// twice the largest displacement since the build < l/2, so the pairs take
	// wrap_inner's shorter sequence (same result). Decided per warp.
	constexpr bool kCanInner = kAllPeriodic && std::is_same<BoxSrc, OneBox>::value;
	bool inner = false;
	if constexpr (kCanInner) {
		if (boxes.d2max != nullptr) {
			const float m = boxes.margin + 2.0f * sqrtf(__uint_as_float(__ldg(boxes.d2max)));
			const float c[3] = {pi.x, pi.y, pi.z};
			inner = true;
#pragma unroll
			for (int a = 0; a < 3; ++a)
				inner = inner && c[a] >= box.origin[a] + m &&
						c[a] <= box.origin[a] + box.size[a] - m;
			inner = inner || !valid;
		}
		inner = __all_sync(0xFFFFFFFFu, inner);
	}
	// Two entries per lane per iteration: both neighbour gathers are in flight
	// before either pair's arithmetic (the kernel is bound by gather latency).
	auto walk = [&](auto inner_tag) {
		constexpr bool kIn = decltype(inner_tag)::value;
		uint32_t t = sub;
		for (; t + G < cnt; t += 2 * G) {
			const uint32_t e0 = __ldcs(col + static_cast<size_t>(t) * H);
			const uint32_t e1 = __ldcs(col + static_cast<size_t>(t + G) * H);
			const uint32_t j0 = e0 & ~kOrientBit, j1 = e1 & ~kOrientBit;
			const float4 p0 = sorted_pos[j0];
			const float4 p1 = sorted_pos[j1];
			pair_scalar<kEnergy, kAllPeriodic, kTerms, kIn>(pi, npi, p0, j0, e0 & kOrientBit,
															trow, bin_f, bin_e, arow, sv, box,
															win, force, nxy, nz, fe, e_acc, w_acc);
			pair_scalar<kEnergy, kAllPeriodic, kTerms, kIn>(pi, npi, p1, j1, e1 & kOrientBit,
															trow, bin_f, bin_e, arow, sv, box,
															win, force, nxy, nz, fe, e_acc, w_acc);
		}
		if (t < cnt) {
			const uint32_t entry = __ldcs(col + static_cast<size_t>(t) * H);
			const uint32_t j = entry & ~kOrientBit;
			pair_scalar<kEnergy, kAllPeriodic, kTerms, kIn>(pi, npi, sorted_pos[j], j,
															entry & kOrientBit, trow, bin_f,
															bin_e, arow, sv, box, win, force, nxy,
															nz, fe, e_acc, w_acc);
		}
	};
	if constexpr (kCanInner) {
		if (inner) walk(std::true_type{});
		else walk(std::false_type{});
	} else {
		walk(std::false_type{});
	}
	// The lanes' sums of minus the i-force, then negated (exact).
	float fx = nxy.x, fy = nxy.y, fz = nz;
	if (G > 1) {
#pragma unroll
		for (int o = G / 2; o > 0; o >>= 1) {
			fx += __shfl_xor_sync(0xFFFFFFFFu, fx, o, G);
			fy += __shfl_xor_sync(0xFFFFFFFFu, fy, o, G);
			fz += __shfl_xor_sync(0xFFFFFFFFu, fz, o, G);
			if (kEnergy) fe += __shfl_xor_sync(0xFFFFFFFFu, fe, o, G);
		}
	}
	if (valid && sub == 0 && cnt != 0u) red_add_v4(&force[i], -fx, -fy, -fz, fe);
	if (kEnergy) block_add_f64(e_acc, w_acc, ev);
}

__global__ void __launch_bounds__(256) scatter_add_kernel(const float4* __restrict__ fs,
														  const uint32_t* __restrict__ s2o,
														  uint32_t n, float4* __restrict__ fe,
														  int get_energy) {
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const float4 f = fs[s];
	const uint32_t o = s2o[s];
	float4 t = fe[o];
	t.x += f.x;
	t.y += f.y;
	t.z += f.z;
	if (get_energy) t.w += f.w;
	fe[o] = t;
}

// CalcDistance::compute (src/Interactions/Interactions.h:37-51).
__device__ __forceinline__ float calc_distance(const Box& box, const float4& from,
											   const float4& to, float3& r, float3& unit) {
	r = wrap_diff(box, __fsub_rn(to.x, from.x), __fsub_rn(to.y, from.y), __fsub_rn(to.z, from.z));
	const float dist = __fsqrt_rn(len2(r.x, r.y, r.z));
	if (dist > 1e-6f) {
		const float inv = __frcp_rn(dist);
		unit = make_float3(__fmul_rn(inv, r.x), __fmul_rn(inv, r.y), __fmul_rn(inv, r.z));
	} else {
		unit = make_float3(0.0f, 0.0f, 0.0f);
	}
	return dist;
}

// TabulatedBondComputer::operator() (src/Interactions/Bonded/BondComputer.h:168-191).
// A row with table_idx < 0 has a form other than tabulated and is skipped, as
// the reference's forms[] check skips it.
__device__ __forceinline__ double bond_term(uint32_t k, const int2* __restrict__ bonds,
											const int* __restrict__ table_idx, uint32_t nb,
											const float4* __restrict__ pos, float4* fe,
											const Table* __restrict__ tables, const Box& box,
											int get_energy) {
	double e_acc = 0.0;
	if (k < nb && table_idx[k] >= 0) {
		const int2 b = bonds[k];
		float3 r, u;
		const float dist = calc_distance(box, pos[b.x], pos[b.y], r, u);
		if (dist >= 1e-6f) {
			const Table t = tables[table_idx[k]];
			const float2 fm_e =
				table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 0, dist);
			const float fx = __fmul_rn(u.x, fm_e.x), fy = __fmul_rn(u.y, fm_e.x),
						fz = __fmul_rn(u.z, fm_e.x);
			const float half = get_energy ? __fmul_rn(fm_e.y, 0.5f) : 0.0f;
			red_add_v4(&fe[b.x], -fx, -fy, -fz, half);
			red_add_v4(&fe[b.y], fx, fy, fz, half);
			e_acc = get_energy ? static_cast<double>(fm_e.y) : 0.0;
		}
	}
	return e_acc;
}

__global__ void __launch_bounds__(256) bond_kernel(const int2* __restrict__ bonds,
												   const int* __restrict__ table_idx, uint32_t nb,
												   const float4* __restrict__ pos, float4* fe,
												   const Table* __restrict__ tables, Box box,
												   int get_energy, double* energy) {
	const double e_acc = bond_term(blockIdx.x * blockDim.x + threadIdx.x, bonds, table_idx, nb,
								   pos, fe, tables, box, get_energy);
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

// TabulatedAngleComputer::operator() (BondComputer.h:236-268) with
// AngleGeometry::compute (src/Interactions/Bonded/BondGeometry.h:19-44).
// Angle tables wrap (src/Interactions/DeviceBondedInteraction.h:234).
__device__ __forceinline__ double angle_term(uint32_t k, const int4* __restrict__ angles,
											 const int* __restrict__ table_idx, uint32_t na,
											 const float4* __restrict__ pos, float4* fe,
											 const Table* __restrict__ tables, const Box& box,
											 int get_energy) {
	double e_acc = 0.0;
	if (k < na && table_idx[k] >= 0) {
		const int4 a = angles[k];
		const float4 pi = pos[a.x], pj = pos[a.y], pk = pos[a.z];
		const float3 ab = wrap_diff(box, __fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
									__fsub_rn(pj.z, pi.z));
		const float3 bc = wrap_diff(box, __fsub_rn(pk.x, pj.x), __fsub_rn(pk.y, pj.y),
									__fsub_rn(pk.z, pj.z));
		const float3 ac = wrap_diff(box, __fsub_rn(pk.x, pi.x), __fsub_rn(pk.y, pi.y),
									__fsub_rn(pk.z, pi.z));
		const float ab2 = len2(ab.x, ab.y, ab.z), bc2 = len2(bc.x, bc.y, bc.z),
					ac2 = len2(ac.x, ac.y, ac.z);
		float cs = __fdiv_rn(__fmul_rn(__fsub_rn(__fadd_rn(ab2, bc2), ac2), 0.5f),
							 __fmul_rn(__fsqrt_rn(ab2), __fsqrt_rn(bc2)));
		if (cs < -1.0f) cs = -1.0f;
		if (cs > 1.0f) cs = 1.0f;
		const float angle = acosf(cs);
		const float sn = __fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(cs, cs)));
		const Table t = tables[table_idx[k]];
		const float2 fm_e =
			table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 1, angle);
		const float sin_angle = sn > 1e-3f ? sn : 1e-3f;
		const float dudt = __fdiv_rn(-fm_e.x, sin_angle);
		const float inv_ab = __frcp_rn(__fsqrt_rn(ab2));
		const float inv_bc = __frcp_rn(__fsqrt_rn(bc2));
		const float s1 = __fmul_rn(dudt, inv_ab);
		const float c_ab = __fmul_rn(cs, inv_ab);
		const float s3 = -__fmul_rn(dudt, inv_bc);
		const float c_bc = __fmul_rn(cs, inv_bc);
		const float f1x = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.x, c_ab), __fmul_rn(bc.x, inv_bc)));
		const float f1y = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.y, c_ab), __fmul_rn(bc.y, inv_bc)));
		const float f1z = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.z, c_ab), __fmul_rn(bc.z, inv_bc)));
		const float f3x = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.x, c_bc), __fmul_rn(ab.x, inv_ab)));
		const float f3y = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.y, c_bc), __fmul_rn(ab.y, inv_ab)));
		const float f3z = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.z, c_bc), __fmul_rn(ab.z, inv_ab)));
		const float third = get_energy ? __fmul_rn(fm_e.y, 0.3333333432674408f) : 0.0f;
		red_add_v4(&fe[a.x], f1x, f1y, f1z, third);
		red_add_v4(&fe[a.y], -__fadd_rn(f1x, f3x), -__fadd_rn(f1y, f3y), -__fadd_rn(f1z, f3z),
				   third);
		red_add_v4(&fe[a.z], f3x, f3y, f3z, third);
		e_acc = get_energy ? static_cast<double>(fm_e.y) : 0.0;
	}
	return e_acc;
}

__global__ void __launch_bounds__(256) angle_kernel(const int4* __restrict__ angles,
													const int* __restrict__ table_idx, uint32_t na,
													const float4* __restrict__ pos, float4* fe,
													const Table* __restrict__ tables, Box box,
													int get_energy, double* energy) {
	const double e_acc = angle_term(blockIdx.x * blockDim.x + threadIdx.x, angles, table_idx, na,
									pos, fe, tables, box, get_energy);
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

// Bonds and angles in one launch: the first ceil(nb / 256) blocks take the
// bonds, the rest the angles (one launch fewer per step; the two kernels'
// arithmetic unchanged).
__global__ void __launch_bounds__(256) bond_angle_kernel(
	const int2* __restrict__ bonds, const int* __restrict__ bond_idx, uint32_t nb,
	const Table* __restrict__ bond_tables, const int4* __restrict__ angles,
	const int* __restrict__ angle_idx, uint32_t na, const Table* __restrict__ angle_tables,
	const float4* __restrict__ pos, float4* fe, Box box, int get_energy, double* bond_energy,
	double* angle_energy) {
	const uint32_t bond_blocks = (nb + blockDim.x - 1) / blockDim.x;
	if (blockIdx.x < bond_blocks) {
		const double e = bond_term(blockIdx.x * blockDim.x + threadIdx.x, bonds, bond_idx, nb, pos,
								   fe, bond_tables, box, get_energy);
		if (get_energy) block_add_f64(e, 0.0, bond_energy);
	} else {
		const double e = angle_term((blockIdx.x - bond_blocks) * blockDim.x + threadIdx.x, angles,
									angle_idx, na, pos, fe, angle_tables, box, get_energy);
		if (get_energy) block_add_f64(e, 0.0, angle_energy);
	}
}

__device__ __forceinline__ float3 cross3(const float3& a, const float3& b) {
	return make_float3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
					   __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
					   __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float dot3(const float3& a, const float3& b) {
	return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float len2v(const float3& a) { return len2(a.x, a.y, a.z); }
// Vector3::rLength2 (src/Types/Vector3.h:233-236).
__device__ __forceinline__ float rlen2(const float3& a) {
	const float l2 = len2v(a);
	return l2 != 0.0f ? __frcp_rn(l2) : 0.0f;
}

// TabulatedDihedralComputer::operator() (src/Interactions/Bonded/BondComputer.h:304-345)
// with DihedralGeometry::compute (src/Interactions/Bonded/BondGeometry.h:62-86):
// phi from the two plane normals, periodic table, magnitude 0 when degenerate
// and clamped to +-1000 (kMaxBondedForce), a quarter of the energy to each of
// the four particles. Rows with table_idx < 0 are skipped.
__global__ void __launch_bounds__(256) dihedral_kernel(const int4* __restrict__ dih,
													   const int* __restrict__ table_idx,
													   uint32_t nd, const float4* __restrict__ pos,
													   float4* fe, const Table* __restrict__ tables,
													   Box box, int get_energy, double* energy) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	double e_acc = 0.0;
	if (k < nd && table_idx[k] >= 0) {
		const int4 q = dih[k];
		const float4 p0 = pos[q.x], p1 = pos[q.y], p2 = pos[q.z], p3 = pos[q.w];
		const float3 ab = wrap_diff(box, __fsub_rn(p1.x, p0.x), __fsub_rn(p1.y, p0.y),
									__fsub_rn(p1.z, p0.z));
		const float3 bc = wrap_diff(box, __fsub_rn(p2.x, p1.x), __fsub_rn(p2.y, p1.y),
									__fsub_rn(p2.z, p1.z));
		const float3 cd = wrap_diff(box, __fsub_rn(p3.x, p2.x), __fsub_rn(p3.y, p2.y),
									__fsub_rn(p3.z, p2.z));
		const float3 c_abc = cross3(ab, bc), c_bcd = cross3(bc, cd), c_x = cross3(bc, c_abc);
		const float l_abc = __fsqrt_rn(len2v(c_abc)), l_bcd = __fsqrt_rn(len2v(c_bcd));
		const float cos_phi = __fdiv_rn(dot3(c_abc, c_bcd), __fmul_rn(l_abc, l_bcd));
		const float sin_phi =
			__fdiv_rn(dot3(c_x, c_bcd), __fmul_rn(__fsqrt_rn(len2v(c_x)), l_bcd));
		const float phi = atan2f(sin_phi, cos_phi);
		const float lbc = __fsqrt_rn(len2v(bc));
		const float s1 = __fmul_rn(-lbc, rlen2(c_abc));
		const float s3 = __fmul_rn(-lbc, rlen2(c_bcd));
		const float rbc = rlen2(bc);
		const float g1 = -__fmul_rn(dot3(ab, bc), rbc);
		const float g3 = __fmul_rn(dot3(bc, cd), rbc);
		const float3 f1 = make_float3(__fmul_rn(s1, c_abc.x), __fmul_rn(s1, c_abc.y),
									  __fmul_rn(s1, c_abc.z));
		const float3 f3 = make_float3(__fmul_rn(s3, c_bcd.x), __fmul_rn(s3, c_bcd.y),
									  __fmul_rn(s3, c_bcd.z));
		const float3 f2 = make_float3(__fsub_rn(__fmul_rn(g1, f1.x), __fmul_rn(g3, f3.x)),
									  __fsub_rn(__fmul_rn(g1, f1.y), __fmul_rn(g3, f3.y)),
									  __fsub_rn(__fmul_rn(g1, f1.z), __fmul_rn(g3, f3.z)));
		const bool degenerate =
			__fmul_rn(__fmul_rn(len2v(ab), len2v(bc)), rlen2(c_abc)) > 100.0f ||
			__fmul_rn(__fmul_rn(len2v(bc), len2v(cd)), rlen2(c_bcd)) > 100.0f;
		const Table t = tables[table_idx[k]];
		const float2 fm_e =
			table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 1, phi);
		float mag = degenerate ? 0.0f : fm_e.x;
		mag = mag > 1000.0f ? 1000.0f : (mag < -1000.0f ? -1000.0f : mag);
		const float3 v1 = make_float3(__fmul_rn(mag, f1.x), __fmul_rn(mag, f1.y), __fmul_rn(mag, f1.z));
		const float3 v2 = make_float3(__fmul_rn(mag, f2.x), __fmul_rn(mag, f2.y), __fmul_rn(mag, f2.z));
		const float3 v3 = make_float3(__fmul_rn(mag, f3.x), __fmul_rn(mag, f3.y), __fmul_rn(mag, f3.z));
		const float quarter = get_energy ? __fmul_rn(fm_e.y, 0.25f) : 0.0f;
		red_add_v4(&fe[q.x], v1.x, v1.y, v1.z, quarter);
		red_add_v4(&fe[q.y], __fsub_rn(v2.x, v1.x), __fsub_rn(v2.y, v1.y), __fsub_rn(v2.z, v1.z),
				   quarter);
		red_add_v4(&fe[q.z], __fsub_rn(v3.x, v2.x), __fsub_rn(v3.y, v2.y), __fsub_rn(v3.z, v2.z),
				   quarter);
		red_add_v4(&fe[q.w], -v3.x, -v3.y, -v3.z, quarter);
		e_acc = get_energy ? static_cast<double>(fm_e.y) : 0.0;
	}
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

// HarmonicRestraintComputer::operator() (src/Interactions/Bonded/BondComputer.h:110-130):
// r = wrap_diff(pos - anchor), F = unit * (-k |r|), the full energy
// 0.5 k |r|^2 to the particle; ids < 0 are skipped.
__global__ void __launch_bounds__(256) restraint_kernel(const int* __restrict__ ids,
														const float4* __restrict__ anchors,
														const float* __restrict__ k_spring,
														uint32_t nr, const float4* __restrict__ pos,
														float4* fe, Box box, int get_energy,
														double* energy) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	double e_acc = 0.0;
	if (k < nr && ids[k] >= 0) {
		const int id = ids[k];
		float3 r, u;
		const float d = calc_distance(box, anchors[k], pos[id], r, u);
		const float kk = k_spring[k];
		const float fm = __fmul_rn(-kk, d);
		const float e = __fmul_rn(__fmul_rn(__fmul_rn(0.5f, kk), d), d);
		red_add_v4(&fe[id], __fmul_rn(fm, u.x), __fmul_rn(fm, u.y), __fmul_rn(fm, u.z),
				   get_energy ? e : 0.0f);
		e_acc = get_energy ? static_cast<double>(e) : 0.0;
	}
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

template <int G, bool kEnergy, bool kAllPeriodic, bool kTerms, class BoxSrc, bool kUniform = false>
void launch_pair(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
				 uint32_t n, uint32_t cap, const PairTables& t, const BoxSrc& boxes,
				 float cutoff_sq, float4* force_sorted, double* ev, cudaStream_t st) {
	const uint32_t rows = 256 / G;
	const uint32_t blocks = (n + rows - 1) / rows;
	auto kern = pair_force_kernel<G, kEnergy, kAllPeriodic, kTerms, kUniform, BoxSrc>;
	constexpr bool kStage = !std::is_same<BoxSrc, OneBox>::value;
	const size_t smem =
		static_cast<size_t>(t.num_types * t.num_types) * sizeof(PairTableRef) +
		(kStage ? static_cast<size_t>((t.total_bins + 1) & ~1u) * 4 +
					  (kEnergy ? static_cast<size_t>(t.total_bins) * 8 : 0)
				: 0);
	if (smem > 48 * 1024)
		MB2_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  static_cast<int>(smem)));
	MB2_LAUNCH kern<<<blocks, 256, smem, st>>>(sorted_pos, nbr, row_len, n, cap, t.num_types,
											   t.refs, t.offsets, t.uniform_ref, t.bin_force,
											   t.bin_energy, t.total_bins,
											   t.terms, t.solvent, boxes, dist_window(cutoff_sq),
											   force_sorted, ev);
}

template <int G, bool kEnergy, bool kAllPeriodic, class BoxSrc>
void launch_pair_t(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
				   uint32_t n, uint32_t cap, const PairTables& t, const BoxSrc& boxes,
				   float cutoff_sq, float4* force_sorted, double* ev, cudaStream_t st) {
	// Analytical terms only on the one-box path (batched replicas are tabulated).
	if constexpr (std::is_same<BoxSrc, OneBox>::value) {
		if (t.terms) {
			launch_pair<G, kEnergy, kAllPeriodic, true>(sorted_pos, nbr, row_len, n, cap, t, boxes,
														cutoff_sq, force_sorted, ev, st);
			return;
		}
	}
	if (t.uniform && t.offsets) {
		launch_pair<G, kEnergy, kAllPeriodic, false, BoxSrc, true>(
			sorted_pos, nbr, row_len, n, cap, t, boxes, cutoff_sq, force_sorted, ev, st);
		return;
	}
	launch_pair<G, kEnergy, kAllPeriodic, false>(sorted_pos, nbr, row_len, n, cap, t, boxes,
												 cutoff_sq, force_sorted, ev, st);
}

template <int G, class BoxSrc>
void launch_pair_g(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
				   uint32_t n, uint32_t cap, const PairTables& t, const BoxSrc& boxes,
				   bool all_periodic, float cutoff_sq, int get_energy, float4* force_sorted,
				   double* ev, cudaStream_t st) {
	if (get_energy) {
		if (all_periodic) launch_pair_t<G, true, true>(sorted_pos, nbr, row_len, n, cap, t, boxes, cutoff_sq, force_sorted, ev, st);
		else launch_pair_t<G, true, false>(sorted_pos, nbr, row_len, n, cap, t, boxes, cutoff_sq, force_sorted, ev, st);
	} else {
		if (all_periodic) launch_pair_t<G, false, true>(sorted_pos, nbr, row_len, n, cap, t, boxes, cutoff_sq, force_sorted, ev, st);
		else launch_pair_t<G, false, false>(sorted_pos, nbr, row_len, n, cap, t, boxes, cutoff_sq, force_sorted, ev, st);
	}
}

template <class BoxSrc>
void launch_pair_lanes(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
					   uint32_t n, uint32_t cap, int lanes_per_row, const PairTables& t,
					   const BoxSrc& boxes, bool all_periodic, float cutoff_sq, int get_energy,
					   float4* force_sorted, double* ev, cudaStream_t st) {
	switch (lanes_per_row) {
	case 4: launch_pair_g<4>(sorted_pos, nbr, row_len, n, cap, t, boxes, all_periodic, cutoff_sq, get_energy, force_sorted, ev, st); break;
	case 8: launch_pair_g<8>(sorted_pos, nbr, row_len, n, cap, t, boxes, all_periodic, cutoff_sq, get_energy, force_sorted, ev, st); break;
	case 16: launch_pair_g<16>(sorted_pos, nbr, row_len, n, cap, t, boxes, all_periodic, cutoff_sq, get_energy, force_sorted, ev, st); break;
	default: launch_pair_g<32>(sorted_pos, nbr, row_len, n, cap, t, boxes, all_periodic, cutoff_sq, get_energy, force_sorted, ev, st); break;
	}
}

}  // namespace

namespace {

// RN(sqrt(x)) and RN(s * s) in float on the host: the double root rounded to
// float is the correctly rounded float root (53 >= 2 * 24 + 2 bits), and the
// product of two floats is exact in double.
float host_sqrt_rn(float x) { return static_cast<float>(std::sqrt(static_cast<double>(x))); }
float host_sq_rn(float s) { return static_cast<float>(static_cast<double>(s) * s); }

// Smallest non-negative float bit pattern in [lo, hi] for which pred holds
// (pred monotone false -> true over the ordered patterns), or hi + 1.
template <class P>
uint32_t first_true(uint32_t lo, uint32_t hi, P pred) {
	uint64_t a = lo, b = static_cast<uint64_t>(hi) + 1;
	while (a < b) {
		const uint64_t m = (a + b) / 2;
		float x;
		const uint32_t bits = static_cast<uint32_t>(m);
		std::memcpy(&x, &bits, 4);
		if (pred(x)) b = m;
		else a = m + 1;
	}
	return static_cast<uint32_t>(a);
}

float from_bits(uint32_t b) {
	float x;
	std::memcpy(&x, &b, 4);
	return x;
}

}  // namespace

DistWindow dist_window(float cutoff_sq) {
	constexpr uint32_t kMaxFinite = 0x7F7FFFFFu;
	DistWindow w;
	// lo: the least d2 whose root is not below 1e-6.
	w.lo = from_bits(first_true(0u, kMaxFinite, [](float x) { return host_sqrt_rn(x) >= 1e-6f; }));
	// hi: the largest d2 with RN(RN(sqrt(d2))^2) <= cutoff_sq.
	if (!(cutoff_sq > 0.0f)) {
		w.hi = INFINITY;
	} else {
		const uint32_t first_out = first_true(0u, kMaxFinite, [cutoff_sq](float x) {
			return host_sq_rn(host_sqrt_rn(x)) > cutoff_sq;
		});
		w.hi = first_out > kMaxFinite ? INFINITY : from_bits(first_out - 1u);
	}
	return w;
}

size_t pair_table_arrays(int num_types, const uint32_t* term_matrix, int num_tables,
						 const float* values, const uint32_t* sizes, const float* starts,
						 const float* step_invs, std::vector<PairTableRef>& refs,
						 std::vector<float>& bf, std::vector<float2>& be) {
	expect_arg(num_types > 0 && num_types <= 64, MB2_ERR_ARG, "pair tables: 1..64 particle types");
	expect_arg(num_tables >= 0 && term_matrix, MB2_ERR_ARG, "pair tables: bad tables");
	for (int k = 0; k < num_types * num_types; ++k) {
		const uint32_t tag = term_matrix[k];
		expect_arg(!(tag & kTermTabulated) || static_cast<int>(tag >> kTableShift) < num_tables,
				   MB2_ERR_ARG, "pair tables: a tag names a missing table");
	}
	// Per-bin force and energy, rounded exactly as TabulatedPotential::compute
	// rounds them (TabulatedPotential.h:41-51): dU = U[k+1] - U[k] and
	// F = -dU * step_inv in float; the last bin is the home >= size-1 case.
	std::vector<uint32_t> offset(num_tables);
	size_t total = 0;
	for (int k = 0; k < num_tables; ++k) {
		expect_arg(sizes[k] >= 2, MB2_ERR_ARG, "pair tables: a table needs 2 values");
		// A step of 0 (fewer than two distinct abscissae) gives an infinite
		// inverse: refused, as is a NaN or infinite start.
		expect_arg(std::isfinite(starts[k]) && std::isfinite(step_invs[k]) && step_invs[k] != 0.0f,
				   MB2_ERR_ARG, "pair tables: start and step inverse must be finite, step inverse nonzero");
		offset[k] = static_cast<uint32_t>(total);
		total += sizes[k];
	}
	bf.assign(std::max<size_t>(total, 1), 0.0f);
	be.assign(std::max<size_t>(total, 1), make_float2(0.0f, 0.0f));
	for (int k = 0; k < num_tables; ++k) {
		const float* u = values + offset[k];
		const uint32_t sz = sizes[k];
		for (uint32_t b = 0; b + 1 < sz; ++b) {
			volatile float du = u[b + 1] - u[b];
			volatile float f = -du * step_invs[k];
			bf[offset[k] + b] = f;
			be[offset[k] + b] = make_float2(u[b], du);
		}
		bf[offset[k] + sz - 1] = 0.0f;
		be[offset[k] + sz - 1] = make_float2(u[sz - 1], 0.0f);
	}
	const int tt = num_types * num_types;
	refs.assign(tt, PairTableRef{0.0f, 0.0f, 0, -1});
	for (int k = 0; k < tt; ++k) {
		const uint32_t tag = term_matrix[k];
		if (tag & kTermTabulated) {
			const int t = static_cast<int>(tag >> kTableShift);
			refs[k] = PairTableRef{starts[t], step_invs[t], static_cast<int>(sizes[t]) - 1,
								   static_cast<int>(offset[t])};
		}
	}
	return total;
}

bool uniform_tables(const std::vector<PairTableRef>& refs, std::vector<int>& offsets,
					PairTableRef& u) {
	bool uniform = false, any = false;
	u = PairTableRef{0.0f, 0.0f, 0, -1};
	offsets.assign(refs.size(), -1);
	for (size_t k = 0; k < refs.size(); ++k) {
		offsets[k] = refs[k].offset;
		if (refs[k].offset < 0) continue;
		if (!any) {
			u = refs[k];
			any = uniform = true;
		} else if (std::memcmp(&u.start, &refs[k].start, sizeof(float)) != 0 ||
				   std::memcmp(&u.step_inv, &refs[k].step_inv, sizeof(float)) != 0 ||
				   u.last != refs[k].last) {
			uniform = false;
		}
	}
	u.offset = -1;
	return uniform;
}

void pair_forces(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
				 uint32_t n, uint32_t cap, int lanes_per_row, const PairTables& t, const Box& box,
				 float cutoff_sq, int get_energy, float4* force_sorted, double* ev,
				 cudaStream_t st, const unsigned int* d2max, float list_rc) {
	if (n == 0) return;
	const bool all_periodic = box.periodic[0] && box.periodic[1] && box.periodic[2];
	const bool track = d2max != nullptr && list_rc > 0.0f && std::isfinite(list_rc);
	const OneBox one{box, track ? d2max : nullptr,
					 track ? list_rc * (1.0f + 0x1p-20f) + kInnerSafety : 0.0f};
	launch_pair_lanes(sorted_pos, nbr, row_len, n, cap, lanes_per_row, t, one, all_periodic,
					  cutoff_sq, get_energy, force_sorted, ev, st);
}

void pair_forces_systems(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
						 uint32_t n, uint32_t cap, int lanes_per_row, const PairTables& t,
						 const Box* boxes, const uint32_t* sorted_keys, int sys_shift,
						 bool all_periodic, float cutoff_sq, int get_energy, float4* force_sorted,
						 double* ev, cudaStream_t st) {
	if (n == 0) return;
	launch_pair_lanes(sorted_pos, nbr, row_len, n, cap, lanes_per_row, t,
					  SystemBoxes{boxes, sorted_keys, sys_shift}, all_periodic, cutoff_sq,
					  get_energy, force_sorted, ev, st);
}

namespace {

// Every float with bit pattern in [lo, hi]: sqrt_rn_nr against __fsqrt_rn,
// mismatches counted.
__global__ void __launch_bounds__(256) sqrt_check_kernel(uint32_t lo, uint32_t hi,
														unsigned long long* bad) {
	const uint64_t count = static_cast<uint64_t>(hi) - lo + 1;
	unsigned long long mine = 0;
	for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < count;
		 k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
		const float a = __uint_as_float(lo + static_cast<uint32_t>(k));
		mine += __float_as_uint(__fsqrt_rn(a)) != __float_as_uint(sqrt_rn_nr(a));
	}
	if (mine) atomicAdd(bad, mine);
}

}  // namespace

void selftest_sqrt(unsigned long long* bad, cudaStream_t st) {
	int sms = 148;
	int dev = 0;
	MB2_CUDA(cudaGetDevice(&dev));
	MB2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	const float lo = 0x1p-60f, hi = 3.40282347e38f;
	uint32_t b[2];
	std::memcpy(&b[0], &lo, 4);
	std::memcpy(&b[1], &hi, 4);
	MB2_LAUNCH sqrt_check_kernel<<<sms * 8, 256, 0, st>>>(b[0], b[1], bad);
}

void scatter_add_forces(const float4* force_sorted, const uint32_t* s2o, uint32_t n,
						float4* force_energy, int get_energy, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH scatter_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(force_sorted, s2o, n,
																   force_energy, get_energy);
}

void bond_forces(const int2* bonds, const int* table_idx, uint32_t nb, const float4* pos,
				 float4* fe, const Table* tables, const Box& box, int get_energy, double* energy,
				 cudaStream_t st) {
	if (nb == 0) return;
	MB2_LAUNCH bond_kernel<<<(nb + 255) / 256, 256, 0, st>>>(bonds, table_idx, nb, pos, fe, tables,
															 box, get_energy, energy);
}

void angle_forces(const int4* angles, const int* table_idx, uint32_t na, const float4* pos,
				  float4* fe, const Table* tables, const Box& box, int get_energy, double* energy,
				  cudaStream_t st) {
	if (na == 0) return;
	MB2_LAUNCH angle_kernel<<<(na + 255) / 256, 256, 0, st>>>(angles, table_idx, na, pos, fe,
															  tables, box, get_energy, energy);
}

void bond_angle_forces(const int2* bonds, const int* bond_idx, uint32_t nb, const Table* bond_tables,
					   const int4* angles, const int* angle_idx, uint32_t na,
					   const Table* angle_tables, const float4* pos, float4* fe, const Box& box,
					   int get_energy, double* bond_energy, double* angle_energy, cudaStream_t st) {
	const uint32_t blocks = (nb + 255) / 256 + (na + 255) / 256;
	if (blocks == 0) return;
	MB2_LAUNCH bond_angle_kernel<<<blocks, 256, 0, st>>>(bonds, bond_idx, nb, bond_tables, angles,
														 angle_idx, na, angle_tables, pos, fe, box,
														 get_energy, bond_energy, angle_energy);
}

void dihedral_forces(const int4* dihedrals, const int* table_idx, uint32_t nd, const float4* pos,
					 float4* fe, const Table* tables, const Box& box, int get_energy,
					 double* energy, cudaStream_t st) {
	if (nd == 0) return;
	MB2_LAUNCH dihedral_kernel<<<(nd + 255) / 256, 256, 0, st>>>(dihedrals, table_idx, nd, pos, fe,
																 tables, box, get_energy, energy);
}

void restraint_forces(const int* ids, const float4* anchors, const float* k_spring, uint32_t nr,
					  const float4* pos, float4* fe, const Box& box, int get_energy,
					  double* energy, cudaStream_t st) {
	if (nr == 0) return;
	MB2_LAUNCH restraint_kernel<<<(nr + 255) / 256, 256, 0, st>>>(ids, anchors, k_spring, nr, pos,
																  fe, box, get_energy, energy);
}

}  // namespace mb2
