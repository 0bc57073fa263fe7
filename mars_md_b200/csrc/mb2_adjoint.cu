// Adjoint of the BD step and a smoothed pair-distance histogram loss.
//
// No counterpart in the reference (it has no gradients). For one BD step
// x' = wrap(x + c F(x) + s xi) with c = D dt / kT per type and axis, the
// adjoint is lambda = lambda' + J(x)^T (c * lambda'), J = dF/dx. Every force
// on this path is minus the gradient of a potential that is piecewise linear
// in a distance or an angle (the tabulated lookup), so J is symmetric and
// J^T mu is the directional derivative of the force along mu = c * lambda':
//   * pair / bond (central) term, force F(r) u on j and -F(r) u on i with
//     u = (x_j - x_i) / r and F constant within a table bin:
//     t = F / r (dv - u (u . dv)), dv = mu_j - mu_i, added to j, subtracted from i;
//   * angle term: forward-mode (dual number) derivative of the reference's
//     AngleGeometry force formula (exact except where the sine is floored),
//     its sine taken from the cross product rather than sqrt(1 - cos^2).
// Table gradients: dF/dU[h] = +step_inv, dF/dU[h+1] = -step_inv for the bin h
// a pair falls in, so dL/dU[h] += step_inv (u . dv) and dL/dU[h+1] -= it;
// accumulated in FP64 per block in shared memory, then one atomic per bin.
//
// Histogram loss: h_b = sum over listed pairs with r < r_max of
// exp(-(r - r_b)^2 / (2 sigma^2)) for |r - r_b| <= 5 sigma, r_b = (b + 1/2) dr,
// accumulated in FP64; its gradient for a given dL/dh moves each pair's
// endpoints by dL/dr u.
#include <algorithm>
#include <cmath>

#include "marsb200.h"
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

struct Dual {
	float v, d;
};
__device__ __forceinline__ Dual dm(float v, float d) { return Dual{v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return dm(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return dm(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
	return dm(a.v * b.v, a.d * b.v + a.v * b.d);
}
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
	return dm(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v));
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
	const float r = sqrtf(a.v);
	return dm(r, r > 0.0f ? a.d / (2.0f * r) : 0.0f);
}

__device__ __forceinline__ float3 f3sub(float4 a, float4 b) {
	return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}

// Tangent accumulators hold 4 doubles per particle (x, y, z, unused): the
// per-particle sums of many float terms that largely cancel are kept in FP64,
// so a step adds no more rounding than its float terms carry.
__device__ __forceinline__ void add_d3(double* t, double x, double y, double z) {
	atomicAdd(t, x);
	atomicAdd(t + 1, y);
	atomicAdd(t + 2, z);
}

// mu = (D / kT * dt) * lambda per type and axis, in original and sorted order;
// the step's tangent accumulators cleared.
__global__ void __launch_bounds__(256) adj_mu_kernel(const float4* __restrict__ lam,
													 const int* __restrict__ type_ids,
													 const float4* __restrict__ diffusion,
													 const uint32_t* __restrict__ inv, uint32_t n,
													 float dt_over_kT, float4* __restrict__ mu,
													 float4* __restrict__ mu_sorted,
													 double4* __restrict__ tan,
													 double4* __restrict__ tan_sorted) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	// The tangent accumulators of this step start at zero.
	tan[i] = make_double4(0.0, 0.0, 0.0, 0.0);
	tan_sorted[i] = make_double4(0.0, 0.0, 0.0, 0.0);
	const float4 d = diffusion[type_ids[i]];
	const float4 l = lam[i];
	const float4 m = make_float4(d.x * dt_over_kT * l.x, d.y * dt_over_kT * l.y,
								 d.z * dt_over_kT * l.z, 0.0f);
	mu[i] = m;
	mu_sorted[inv[i]] = m;
}

// Shared FP64 accumulators for table-gradient bins, flushed once per block.
__device__ __forceinline__ void flush_bins(const double* sg, double* g, uint32_t bins) {
	__syncthreads();
	for (uint32_t k = threadIdx.x; k < bins; k += blockDim.x)
		if (sg[k] != 0.0) atomicAdd(&g[k], sg[k]);
}

// Pair term over the sliced-ELL half list (G lanes per row, rows striding
// over the grid). tan_sorted accumulates J mu in sorted order.
template <int G, bool kAllPeriodic>
__global__ void __launch_bounds__(256) adj_pair_kernel(
	const float4* __restrict__ sorted_pos, const float4* __restrict__ mu_sorted,
	const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ row_len, uint32_t n,
	uint32_t cap, int T, const PairTableRef* __restrict__ refs_g,
	const float* __restrict__ force_g, uint32_t total_bins, Box box, float cutoff_sq,
	double* tan_sorted, double* __restrict__ grad_bins) {
	constexpr int H = 32 / G;
	extern __shared__ double sg[];
	PairTableRef* refs = reinterpret_cast<PairTableRef*>(sg + total_bins);
	float* bin_f = reinterpret_cast<float*>(refs + T * T);
	for (uint32_t k = threadIdx.x; k < total_bins; k += blockDim.x) {
		sg[k] = 0.0;
		bin_f[k] = force_g[k];
	}
	for (int k = threadIdx.x; k < T * T; k += blockDim.x) refs[k] = refs_g[k];
	__syncthreads();
	const int sub = threadIdx.x & (G - 1);
	const uint32_t rows_per_block = blockDim.x / G;
	for (uint32_t row0 = blockIdx.x * rows_per_block; row0 < n; row0 += gridDim.x * rows_per_block) {
		const uint32_t i = row0 + threadIdx.x / G;
		const bool valid = i < n;
		const float4 pi = valid ? sorted_pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
		const float4 mi = valid ? mu_sorted[i] : make_float4(0.f, 0.f, 0.f, 0.f);
		const PairTableRef* trow = refs + (valid ? type_of(pi) : 0) * T;
		const uint32_t cnt = valid ? row_len[i] : 0u;
		const uint32_t* col = nbr + (static_cast<size_t>(i / H) * cap) * H + (i % H);
		double tx = 0.0, ty = 0.0, tz = 0.0;
		for (uint32_t t = sub; t < cnt; t += G) {
			const uint32_t e = __ldg(col + static_cast<size_t>(t) * H);
			const uint32_t j = e & ~kOrientBit;
			const float4 pj = sorted_pos[j];
			// Distance, cutoff test and table bin exactly as the forward pair
			// kernel decides them (the pair oriented as the reference orients
			// it, reference rounding), so the derivative is that of the map
			// the forward computed.
			const bool flip = (e & kOrientBit) != 0u;
			float3 r = flip ? make_float3(__fsub_rn(pi.x, pj.x), __fsub_rn(pi.y, pj.y),
										  __fsub_rn(pi.z, pj.z))
							: make_float3(__fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
										  __fsub_rn(pj.z, pi.z));
			r = wrap_diff(box, r.x, r.y, r.z);
			const float d = __fsqrt_rn(len2(r.x, r.y, r.z));
			if (d < 1e-6f || (cutoff_sq > 0.0f && __fmul_rn(d, d) > cutoff_sq)) continue;
			const PairTableRef tr = trow[type_of(pj)];
			if (tr.offset < 0) continue;
			const float w = __fmul_rn(__fsub_rn(d, tr.start), tr.step_inv);
			const int home = min(max(static_cast<int>(floorf(w)), 0), tr.last);
			const float F = bin_f[tr.offset + home];
			const float4 mj = mu_sorted[j];
			const float inv = flip ? -1.0f / d : 1.0f / d;  // u points from i to j
			const float ux = r.x * inv, uy = r.y * inv, uz = r.z * inv;
			const float dvx = mj.x - mi.x, dvy = mj.y - mi.y, dvz = mj.z - mi.z;
			const float ud = ux * dvx + uy * dvy + uz * dvz;
			const float k = F / d;
			const float gx = k * (dvx - ux * ud), gy = k * (dvy - uy * ud), gz = k * (dvz - uz * ud);
			add_d3(tan_sorted + 4 * static_cast<size_t>(j), gx, gy, gz);
			tx -= gx;
			ty -= gy;
			tz -= gz;
			if (home < tr.last) {
				const double gb = static_cast<double>(tr.step_inv) * ud;
				atomicAdd(&sg[tr.offset + home], gb);
				atomicAdd(&sg[tr.offset + home + 1], -gb);
			}
		}
#pragma unroll
		for (int o = G / 2; o > 0; o >>= 1) {
			tx += __shfl_xor_sync(0xFFFFFFFFu, tx, o, G);
			ty += __shfl_xor_sync(0xFFFFFFFFu, ty, o, G);
			tz += __shfl_xor_sync(0xFFFFFFFFu, tz, o, G);
		}
		if (valid && sub == 0 && cnt != 0u) add_d3(tan_sorted + 4 * static_cast<size_t>(i), tx, ty, tz);
	}
	flush_bins(sg, grad_bins, total_bins);
}

// Bond term (original order) over blocks [0, nblocks) of the launch
// (grid-stride); table bins indexed from the bonded table base, the block's
// bond-table gradient accumulated in shared memory and flushed at its end.
__device__ __forceinline__ void adj_bonds(
	uint32_t block, uint32_t nblocks, const int2* __restrict__ bonds,
	const int* __restrict__ table_idx, uint32_t nb, const float4* __restrict__ pos,
	const float4* __restrict__ mu, const Table* __restrict__ tables,
	const float* __restrict__ values_base, uint32_t total_bins, const Box& box, double* tan,
	double* __restrict__ grad_bins, double* sg) {
	for (uint32_t k = threadIdx.x; k < total_bins; k += blockDim.x) sg[k] = 0.0;
	__syncthreads();
	for (uint32_t b = block * blockDim.x + threadIdx.x; b < nb; b += nblocks * blockDim.x) {
		const int2 e = bonds[b];
		// Distance and bin as the forward bond kernel decides them.
		const float4 pa = pos[e.x], pb = pos[e.y];
		float3 r = wrap_diff(box, __fsub_rn(pb.x, pa.x), __fsub_rn(pb.y, pa.y),
							 __fsub_rn(pb.z, pa.z));
		const float d = __fsqrt_rn(len2(r.x, r.y, r.z));
		if (d < 1e-6f) continue;
		const Table t = tables[table_idx[b]];
		const int size = static_cast<int>(t.size);
		int home = static_cast<int>(floorf(__fmul_rn(__fsub_rn(d, t.start), t.step_inv)));
		if (home >= size - 1) continue;  // constant zero force: no derivative
		if (home < 0) home = 0;
		const float F = -(t.pot[home + 1] - t.pot[home]) * t.step_inv;
		const float4 mi = mu[e.x], mj = mu[e.y];
		const float inv = 1.0f / d;
		const float ux = r.x * inv, uy = r.y * inv, uz = r.z * inv;
		const float dvx = mj.x - mi.x, dvy = mj.y - mi.y, dvz = mj.z - mi.z;
		const float ud = ux * dvx + uy * dvy + uz * dvz;
		const float k = F * inv;
		const float gx = k * (dvx - ux * ud), gy = k * (dvy - uy * ud), gz = k * (dvz - uz * ud);
		add_d3(tan + 4 * static_cast<size_t>(e.y), gx, gy, gz);
		add_d3(tan + 4 * static_cast<size_t>(e.x), -gx, -gy, -gz);
		const uint32_t base = static_cast<uint32_t>(t.pot - values_base) + home;
		const double gb = static_cast<double>(t.step_inv) * ud;
		atomicAdd(&sg[base], gb);
		atomicAdd(&sg[base + 1], -gb);
	}
	flush_bins(sg, grad_bins, total_bins);
}

// Angle term: tangent of the AngleGeometry force along mu (dual numbers).
__device__ __forceinline__ void adj_angle(
	uint32_t q, const int4* __restrict__ angles, const int* __restrict__ table_idx, uint32_t na,
	const float4* __restrict__ pos, const float4* __restrict__ mu, const Table* __restrict__ tables,
	const Box& box, double* tan) {
	if (q >= na) return;
	const int4 a = angles[q];
	const float4 pi = pos[a.x], pj = pos[a.y], pk = pos[a.z];
	const float4 mi = mu[a.x], mj = mu[a.y], mk = mu[a.z];
	float3 rab = f3sub(pj, pi), rbc = f3sub(pk, pj), rac = f3sub(pk, pi);
	rab = wrap_diff(box, rab.x, rab.y, rab.z);
	rbc = wrap_diff(box, rbc.x, rbc.y, rbc.z);
	rac = wrap_diff(box, rac.x, rac.y, rac.z);
	const Dual ab[3] = {dm(rab.x, mj.x - mi.x), dm(rab.y, mj.y - mi.y), dm(rab.z, mj.z - mi.z)};
	const Dual bc[3] = {dm(rbc.x, mk.x - mj.x), dm(rbc.y, mk.y - mj.y), dm(rbc.z, mk.z - mj.z)};
	const Dual ac[3] = {dm(rac.x, mk.x - mi.x), dm(rac.y, mk.y - mi.y), dm(rac.z, mk.z - mi.z)};
	const Dual ab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
	const Dual bc2 = bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2];
	const Dual ac2 = ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2];
	const Dual lab = dsqrt(ab2), lbc = dsqrt(bc2);
	Dual cs = ((ab2 + bc2 - ac2) * dm(0.5f, 0.0f)) / (lab * lbc);
	// The angle, its table bin and the clamps as the forward angle kernel
	// decides them (reference rounding); the duals carry the derivatives.
	const float eab2 = len2(rab.x, rab.y, rab.z), ebc2 = len2(rbc.x, rbc.y, rbc.z),
				eac2 = len2(rac.x, rac.y, rac.z);
	float ecs = __fdiv_rn(__fmul_rn(__fsub_rn(__fadd_rn(eab2, ebc2), eac2), 0.5f),
						  __fmul_rn(__fsqrt_rn(eab2), __fsqrt_rn(ebc2)));
	if (ecs < -1.0f) {
		ecs = -1.0f;
		cs = dm(-1.0f, 0.0f);
	}
	if (ecs > 1.0f) {
		ecs = 1.0f;
		cs = dm(1.0f, 0.0f);
	}
	// sin(theta) = |ab x bc| / (|ab| |bc|), the same function as the forward's
	// sqrt(1 - cos^2) but without its float cancellation: near 180 degrees
	// (the harmonic angle tables' minimum) 1 - cos^2 carries a relative error
	// of about eps / sin^2, the cross product about eps / sin, and dU/dtheta =
	// -F / sin amplifies it into the tangent.
	const Dual cx = ab[1] * bc[2] - ab[2] * bc[1], cy = ab[2] * bc[0] - ab[0] * bc[2],
			   cz = ab[0] * bc[1] - ab[1] * bc[0];
	Dual sn = dsqrt(cx * cx + cy * cy + cz * cz) / (lab * lbc);
	if (__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(ecs, ecs))) <= 1e-3f) sn = dm(1e-3f, 0.0f);
	const Table t = tables[table_idx[q]];
	const float F = table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 1,
								 acosf(ecs)).x;
	const Dual dudt = dm(-F, 0.0f) / sn;
	const Dual inv_ab = dm(1.0f, 0.0f) / lab, inv_bc = dm(1.0f, 0.0f) / lbc;
	const Dual s1 = dudt * inv_ab, c_ab = cs * inv_ab;
	const Dual s3 = dm(0.0f, 0.0f) - dudt * inv_bc, c_bc = cs * inv_bc;
	float t1[3], t3[3];
#pragma unroll
	for (int c = 0; c < 3; ++c) {
		t1[c] = (s1 * (ab[c] * c_ab + bc[c] * inv_bc)).d;
		t3[c] = (s3 * (bc[c] * c_bc + ab[c] * inv_ab)).d;
	}
	add_d3(tan + 4 * static_cast<size_t>(a.x), t1[0], t1[1], t1[2]);
	add_d3(tan + 4 * static_cast<size_t>(a.y), -(t1[0] + t3[0]), -(t1[1] + t3[1]),
		   -(t1[2] + t3[2]));
	add_d3(tan + 4 * static_cast<size_t>(a.z), t3[0], t3[1], t3[2]);
}

// Bonds and angles of one adjoint step in one launch: blocks [0, bond_blocks)
// take the bonds (grid-stride, bond-table gradient through shared memory),
// the rest one angle per thread.
__global__ void __launch_bounds__(256) adj_bond_angle_kernel(
	uint32_t bond_blocks, const int2* __restrict__ bonds, const int* __restrict__ bond_idx,
	uint32_t nb, const Table* __restrict__ bond_tables, const float* __restrict__ values_base,
	uint32_t total_bins, double* __restrict__ grad_bins, const int4* __restrict__ angles,
	const int* __restrict__ angle_idx, uint32_t na, const Table* __restrict__ angle_tables,
	const float4* __restrict__ pos, const float4* __restrict__ mu, Box box, double* tan) {
	extern __shared__ double sg[];
	if (blockIdx.x < bond_blocks)
		adj_bonds(blockIdx.x, bond_blocks, bonds, bond_idx, nb, pos, mu, bond_tables, values_base,
				  total_bins, box, tan, grad_bins, sg);
	else
		adj_angle((blockIdx.x - bond_blocks) * blockDim.x + threadIdx.x, angles, angle_idx, na,
				  pos, mu, angle_tables, box, tan);
}

// lambda += tan (original order) + tan_sorted (gathered through inv).
__global__ void __launch_bounds__(256) adj_combine_kernel(float4* __restrict__ lam,
														  const double4* __restrict__ tan,
														  const double4* __restrict__ tan_sorted,
														  const uint32_t* __restrict__ inv,
														  uint32_t n) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const double4 a = tan[i], b = tan_sorted[inv[i]];
	float4 l = lam[i];
	l.x = static_cast<float>(static_cast<double>(l.x) + (a.x + b.x));
	l.y = static_cast<float>(static_cast<double>(l.y) + (a.y + b.y));
	l.z = static_cast<float>(static_cast<double>(l.z) + (a.z + b.z));
	lam[i] = l;
}

struct RdfSpec {
	uint32_t bins;
	float dr, r_max, sigma;
};

__device__ __forceinline__ void rdf_bin_range(const RdfSpec& s, float d, int& b0, int& b1) {
	b0 = max(0, static_cast<int>(ceilf((d - 5.0f * s.sigma) / s.dr - 0.5f)));
	b1 = min(static_cast<int>(s.bins) - 1, static_cast<int>(floorf((d + 5.0f * s.sigma) / s.dr - 0.5f)));
}

// kGrad = false: histogram into hist (FP64); true: gradient of sum dLdh * h
// into grad_sorted (float4, atomics).
template <int G, bool kGrad>
__global__ void __launch_bounds__(256) rdf_kernel(const float4* __restrict__ sorted_pos,
												  const uint32_t* __restrict__ nbr,
												  const uint32_t* __restrict__ row_len, uint32_t n,
												  uint32_t cap, Box box, RdfSpec spec,
												  double* __restrict__ hist,
												  const double* __restrict__ dldh,
												  float4* grad_sorted) {
	constexpr int H = 32 / G;
	extern __shared__ double sh[];
	for (uint32_t k = threadIdx.x; k < spec.bins; k += blockDim.x)
		sh[k] = kGrad ? dldh[k] : 0.0;
	__syncthreads();
	const float inv2s2 = 1.0f / (2.0f * spec.sigma * spec.sigma);
	const float invs2 = 1.0f / (spec.sigma * spec.sigma);
	const int sub = threadIdx.x & (G - 1);
	const uint32_t rows_per_block = blockDim.x / G;
	for (uint32_t row0 = blockIdx.x * rows_per_block; row0 < n; row0 += gridDim.x * rows_per_block) {
		const uint32_t i = row0 + threadIdx.x / G;
		const bool valid = i < n;
		const float4 pi = valid ? sorted_pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
		const uint32_t cnt = valid ? row_len[i] : 0u;
		const uint32_t* col = nbr + (static_cast<size_t>(i / H) * cap) * H + (i % H);
		float tx = 0.0f, ty = 0.0f, tz = 0.0f;
		for (uint32_t t = sub; t < cnt; t += G) {
			const uint32_t j = __ldg(col + static_cast<size_t>(t) * H) & ~kOrientBit;
			float3 r = f3sub(sorted_pos[j], pi);
			r = wrap_diff(box, r.x, r.y, r.z);
			const float d = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
			if (!(d < spec.r_max) || d < 1e-12f) continue;
			int b0, b1;
			rdf_bin_range(spec, d, b0, b1);
			float dldr = 0.0f;
			for (int b = b0; b <= b1; ++b) {
				const float z = d - (static_cast<float>(b) + 0.5f) * spec.dr;
				const float e = __expf(-z * z * inv2s2);
				if (kGrad) dldr += static_cast<float>(sh[b]) * e * (-z * invs2);
				else atomicAdd(&sh[b], static_cast<double>(e));
			}
			if (kGrad) {
				const float k = dldr / d;
				red_add_v4(&grad_sorted[j], k * r.x, k * r.y, k * r.z, 0.0f);
				tx -= k * r.x;
				ty -= k * r.y;
				tz -= k * r.z;
			}
		}
		if (kGrad) {
#pragma unroll
			for (int o = G / 2; o > 0; o >>= 1) {
				tx += __shfl_xor_sync(0xFFFFFFFFu, tx, o, G);
				ty += __shfl_xor_sync(0xFFFFFFFFu, ty, o, G);
				tz += __shfl_xor_sync(0xFFFFFFFFu, tz, o, G);
			}
			if (valid && sub == 0 && cnt != 0u) red_add_v4(&grad_sorted[i], tx, ty, tz, 0.0f);
		}
	}
	if (!kGrad) flush_bins(sh, hist, spec.bins);
}

// grad[o] += src_sorted[inv[o]].
__global__ void __launch_bounds__(256) gather_add_kernel(float4* __restrict__ grad,
														 const float4* __restrict__ src_sorted,
														 const uint32_t* __restrict__ inv,
														 uint32_t n) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 s = src_sorted[inv[i]];
	float4 g = grad[i];
	g.x += s.x;
	g.y += s.y;
	g.z += s.z;
	grad[i] = g;
}

constexpr uint32_t kPersistentBlocks = 148 * 4;

uint32_t grid_for_rows(uint32_t n, int lanes) {
	const uint32_t rows_per_block = 256u / static_cast<uint32_t>(lanes);
	const uint32_t blocks = (n + rows_per_block - 1) / rows_per_block;
	return blocks < kPersistentBlocks ? (blocks ? blocks : 1u) : kPersistentBlocks;
}

template <int G, bool kAllPeriodic>
void launch_adj_pair(const AdjointStepArgs& a, cudaStream_t st) {
	const size_t smem = static_cast<size_t>(a.tables.total_bins) * 8 +
						static_cast<size_t>(a.tables.num_types * a.tables.num_types) *
							sizeof(PairTableRef) +
						static_cast<size_t>(a.tables.total_bins) * 4;
	auto kern = adj_pair_kernel<G, kAllPeriodic>;
	if (smem > 48 * 1024)
		MB2_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  static_cast<int>(smem)));
	MB2_LAUNCH kern<<<grid_for_rows(a.n, G), 256, smem, st>>>(
		a.sorted_pos, a.mu_sorted, a.nbr, a.row_len, a.n, a.cap, a.tables.num_types,
		a.tables.refs, a.tables.bin_force, a.tables.total_bins, a.box, a.cutoff_sq,
		reinterpret_cast<double*>(a.tan_sorted),
		a.grad_pair);
}

template <int G>
void launch_adj_pair_g(const AdjointStepArgs& a, cudaStream_t st) {
	if (a.box.periodic[0] && a.box.periodic[1] && a.box.periodic[2]) launch_adj_pair<G, true>(a, st);
	else launch_adj_pair<G, false>(a, st);
}

template <int G>
void launch_rdf(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len, uint32_t n,
				uint32_t cap, const Box& box, const RdfSpec& spec, double* hist,
				const double* dldh, float4* grad_sorted, cudaStream_t st) {
	const size_t smem = static_cast<size_t>(spec.bins) * 8;
	if (grad_sorted)
		MB2_LAUNCH rdf_kernel<G, true><<<grid_for_rows(n, G), 256, smem, st>>>(
			sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted);
	else
		MB2_LAUNCH rdf_kernel<G, false><<<grid_for_rows(n, G), 256, smem, st>>>(
			sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted);
}

}  // namespace

void adjoint_step(const AdjointStepArgs& a, cudaStream_t st) {
	const uint32_t n = a.n;
	if (n == 0) return;
	MB2_LAUNCH adj_mu_kernel<<<(n + 255) / 256, 256, 0, st>>>(a.lam, a.type_ids, a.diffusion, a.inv,
															  n, a.dt_over_kT, a.mu, a.mu_sorted,
															  a.tan, a.tan_sorted);
	switch (a.lanes) {
	case 4: launch_adj_pair_g<4>(a, st); break;
	case 8: launch_adj_pair_g<8>(a, st); break;
	case 16: launch_adj_pair_g<16>(a, st); break;
	default: launch_adj_pair_g<32>(a, st); break;
	}
	if (a.num_bonds || a.num_angles) {
		const uint32_t bond_blocks =
			a.num_bonds ? std::min<uint32_t>((a.num_bonds + 255) / 256, kPersistentBlocks) : 0u;
		const uint32_t angle_blocks = (a.num_angles + 255) / 256;
		const size_t smem = a.num_bonds ? static_cast<size_t>(a.bond_bins) * 8 : 0;
		MB2_LAUNCH adj_bond_angle_kernel<<<bond_blocks + angle_blocks, 256, smem, st>>>(
			bond_blocks, a.bonds, a.bond_table_idx, a.num_bonds, a.bond_tables, a.bond_values_base,
			a.bond_bins, a.grad_bond, a.angles, a.angle_table_idx, a.num_angles, a.angle_tables,
			a.pos, a.mu, a.box, reinterpret_cast<double*>(a.tan));
	}
	MB2_LAUNCH adj_combine_kernel<<<(n + 255) / 256, 256, 0, st>>>(a.lam, a.tan, a.tan_sorted, a.inv,
																   n);
}

void rdf_pairs(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len, uint32_t n,
			   uint32_t cap, int lanes, const Box& box, uint32_t bins, float dr, float r_max,
			   float sigma, double* hist, const double* dldh, float4* grad_sorted,
			   cudaStream_t st) {
	if (n == 0) return;
	const RdfSpec spec{bins, dr, r_max, sigma};
	switch (lanes) {
	case 4: launch_rdf<4>(sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted, st); break;
	case 8: launch_rdf<8>(sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted, st); break;
	case 16: launch_rdf<16>(sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted, st); break;
	default: launch_rdf<32>(sorted_pos, nbr, row_len, n, cap, box, spec, hist, dldh, grad_sorted, st); break;
	}
}

void gather_add(float4* grad, const float4* src_sorted, const uint32_t* inv, uint32_t n,
				cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH gather_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(grad, src_sorted, inv, n);
}

}  // namespace mb2
