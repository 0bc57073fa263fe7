// Pairlist build over Morton-sorted particles.
//
// Replaces BuildCellRangesKernel / BuildCellNeighborsKernel /
// ZOrderCellNeighborKernel (src/PatchOperation/PairListKernels/ZOrderNeighbor.h)
// and the grow-and-retry loop of ZOrderPairlist::find_neighbors_zorder
// (src/PatchOperation/PairListKernels/ZOrderPairlist.cpp:208-366).
//
// The pair SET is the reference's: for sorted i < sorted j, keep (i, j) when
// wrap_diff(pos_j - pos_i).length2() <= rc^2 and the pair is not excluded.
// Only the search structure differs. Cells are the top 3m bits of the 30-bit
// Morton key, and the stencil is every cell whose box-to-box distance from
// the home cell can be within rc (a pruned sphere rather than the reference's
// (2r+1)^3 cube), chosen per run to minimise candidates plus per-cell cost.
//
// Storage is a CSR half list keyed by sorted i: row_start[i]..row_start[i+1]
// hold u32 sorted j. Bit 31 of an entry records the reference's pair
// orientation: set when the original index of j is smaller than that of i,
// i.e. the reference computes the pair as j -> i. Rows are filled in two
// walks (count, then exclusive scan, then fill), so the list is exact-size
// and the fill never overflows.
#include "mb2_internal.cuh"

#include <algorithm>
#include <cmath>

namespace mb2 {

CellGrid choose_cell_grid(const float* extent, const int* periodic, float rc_list, size_t n) {
	CellGrid best;
	double best_cost = -1.0;
	const double rc = static_cast<double>(rc_list);
	for (int m = 0; m <= 8; ++m) {
		const int cells = 1 << m;
		const double num_cells = std::ldexp(1.0, 3 * m);
		if (m > 0 && num_cells > 2.0 * static_cast<double>(n)) break;
		std::vector<int> off[3];
		std::vector<double> gap[3];
		for (int a = 0; a < 3; ++a) {
			if (m == 0) {
				off[a] = {0};
				gap[a] = {0.0};
				continue;
			}
			// Real-space cell widths: cell c spans Morton coordinates
			// [c 2^k, (c+1) 2^k) of the 0..1023 scale over the domain, so it is
			// extent * 2^k / 1023 wide, except the last, extent * (2^k - 1) / 1023.
			const int k = 10 - m;
			const double wmin = static_cast<double>(extent[a]) * (std::ldexp(1.0, k) - 1.0) / 1023.0 *
								(1.0 - 1e-6);
			const int r = static_cast<int>(std::floor(rc / wmin)) + 1;
			if (periodic[a] && 2 * r + 1 >= cells) {
				for (int d = 0; d < cells; ++d) {
					off[a].push_back(d);
					gap[a].push_back(0.0);
				}
			} else {
				for (int d = -r; d <= r; ++d) {
					off[a].push_back(d);
					const double g = std::max(0, std::abs(d) - 1) * wmin;
					gap[a].push_back(g);
				}
			}
		}
		std::vector<StencilEntry> st;
		const double lim = rc * rc * (1.0 + 1e-4) + 1e-6;
		for (size_t x = 0; x < off[0].size(); ++x)
			for (size_t y = 0; y < off[1].size(); ++y)
				for (size_t z = 0; z < off[2].size(); ++z) {
					const double g2 =
						gap[0][x] * gap[0][x] + gap[1][y] * gap[1][y] + gap[2][z] * gap[2][z];
					if (g2 <= lim) st.push_back(StencilEntry{off[0][x], off[1][y], off[2][z], 0});
				}
		const double per_cell = static_cast<double>(n) / num_cells;
		const double cost = static_cast<double>(st.size()) * (per_cell + 2.0);
		if (best_cost < 0.0 || cost < best_cost) {
			best_cost = cost;
			best.m = m;
			best.shift = 3 * (10 - m);
			best.num_stencil = static_cast<int>(st.size());
			best.stencil = st;
		}
	}
	return best;
}

namespace {

__global__ void __launch_bounds__(256) cell_ranges_kernel(const uint32_t* __restrict__ keys,
														  uint32_t n, int shift,
														  uint32_t* __restrict__ begin,
														  uint32_t* __restrict__ end) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t c = keys[i] >> shift;
	if (i == 0 || (keys[i - 1] >> shift) != c) begin[c] = i;
	if (i + 1 == n || (keys[i + 1] >> shift) != c) end[c] = i + 1;
}

__device__ __forceinline__ bool is_excluded(const Exclusions& ex, int a, int b, int row_b,
											int row_e, int body) {
	if (body >= 0 && ex.rigid_body_id[b] == body) return true;
	for (int e = row_b; e < row_e; ++e)
		if (ex.neighbors[e] == b) return true;
	return false;
}

template <bool kFill, bool kExcl>
__global__ void __launch_bounds__(256) walk_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ keys,
	const uint32_t* __restrict__ s2o, const uint32_t* __restrict__ begin,
	const uint32_t* __restrict__ end, const StencilEntry* __restrict__ stencil_g, int ns, int m,
	int shift, float rc2, uint32_t n, Box box, Exclusions ex, uint32_t* __restrict__ counts,
	const uint32_t* __restrict__ row_start, uint32_t* __restrict__ nbr) {
	extern __shared__ int4 stencil[];
	for (int k = threadIdx.x; k < ns; k += blockDim.x) {
		const StencilEntry e = stencil_g[k];
		stencil[k] = make_int4(e.dx, e.dy, e.dz, 0);
	}
	__syncthreads();
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 pi = sorted_pos[i];
	const uint32_t c = keys[i] >> shift;
	const int cells = 1 << m;
	const uint32_t mask = static_cast<uint32_t>(cells - 1);
	const int cx = static_cast<int>(compact_by3(c >> 2));
	const int cy = static_cast<int>(compact_by3(c >> 1));
	const int cz = static_cast<int>(compact_by3(c));
	int a = 0, row_b = 0, row_e = 0, body = -1;
	if (kFill || kExcl) a = static_cast<int>(s2o[i]);
	if (kExcl) {
		if (ex.offsets && a >= 0 && static_cast<uint32_t>(a) < ex.num_particles) {
			row_b = ex.offsets[a];
			row_e = ex.offsets[a + 1];
		}
		body = ex.rigid_body_id ? ex.rigid_body_id[a] : -1;
	}
	uint32_t count = 0;
	uint32_t out = kFill ? row_start[i] : 0u;
	for (int k = 0; k < ns; ++k) {
		const int4 s = stencil[k];
		int nx = cx + s.x, ny = cy + s.y, nz = cz + s.z;
		if (box.periodic[0]) nx = static_cast<int>(static_cast<uint32_t>(nx + cells) & mask);
		else if (nx < 0 || nx >= cells) continue;
		if (box.periodic[1]) ny = static_cast<int>(static_cast<uint32_t>(ny + cells) & mask);
		else if (ny < 0 || ny >= cells) continue;
		if (box.periodic[2]) nz = static_cast<int>(static_cast<uint32_t>(nz + cells) & mask);
		else if (nz < 0 || nz >= cells) continue;
		const uint32_t nc = (split_by3(static_cast<uint32_t>(nx)) << 2) |
							(split_by3(static_cast<uint32_t>(ny)) << 1) |
							split_by3(static_cast<uint32_t>(nz));
		const uint32_t b = begin[nc];
		const uint32_t e = end[nc];
		for (uint32_t j = b > i + 1u ? b : i + 1u; j < e; ++j) {
			const float4 pj = sorted_pos[j];
			const float3 d = wrap_diff(box, __fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
									   __fsub_rn(pj.z, pi.z));
			if (len2(d.x, d.y, d.z) <= rc2) {
				int bj = 0;
				if (kFill || kExcl) bj = static_cast<int>(s2o[j]);
				if (kExcl && is_excluded(ex, a, bj, row_b, row_e, body)) continue;
				if (kFill) nbr[out++] = j | (bj < a ? kOrientBit : 0u);
				else ++count;
			}
		}
	}
	if (!kFill) counts[i] = count;
}

__global__ void __launch_bounds__(256) export_kernel(const uint32_t* __restrict__ row_start,
													 const uint32_t* __restrict__ nbr,
													 const uint32_t* __restrict__ s2o, uint32_t n,
													 int2* __restrict__ out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int a = static_cast<int>(s2o[i]);
	for (uint32_t p = row_start[i]; p < row_start[i + 1]; ++p) {
		const int b = static_cast<int>(s2o[nbr[p] & ~kOrientBit]);
		out[p] = make_int2(a < b ? a : b, a < b ? b : a);
	}
}

// DisplacementKernel::min_image (AdaptiveKernels.h:56-65). Both inputs are
// wrapped, so one step suffices; the loops are capped so that a non-finite or
// unwrapped input can never keep a thread spinning.
__device__ __forceinline__ float min_image(float d, float l) {
	if (l <= 0.0f) return d;
	const float h = 0.5f * l;
	for (int it = 0; it < 8 && d > h; ++it) d = __fsub_rn(d, l);
	for (int it = 0; it < 8 && d < -h; ++it) d = __fadd_rn(d, l);
	return d;
}

__global__ void __launch_bounds__(256) displacement_kernel(const float4* __restrict__ cur,
														   const float4* __restrict__ prev,
														   uint32_t n, float3 len,
														   unsigned int* __restrict__ out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	float d2 = 0.0f;
	if (i < n) {
		const float4 c = cur[i], p = prev[i];
		const float dx = min_image(__fsub_rn(c.x, p.x), len.x);
		const float dy = min_image(__fsub_rn(c.y, p.y), len.y);
		const float dz = min_image(__fsub_rn(c.z, p.z), len.z);
		d2 = len2(dx, dy, dz);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xFFFFFFFFu, d2, o));
	// Non-negative floats order like their bit patterns.
	if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(d2));
}

__global__ void __launch_bounds__(256) pack_kernel(const float4* __restrict__ pos,
												   const int* __restrict__ type_ids,
												   const uint32_t* __restrict__ s2o, uint32_t n,
												   float4* __restrict__ sorted_pos) {
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const uint32_t o = s2o[s];
	float4 p = pos[o];
	p.w = __int_as_float(type_ids ? type_ids[o] : 0);
	sorted_pos[s] = p;
}

}  // namespace

void cell_ranges(const uint32_t* keys, uint32_t n, int shift, uint32_t* begin, uint32_t* end,
				 size_t num_cells, cudaStream_t st) {
	MB2_CUDA(cudaMemsetAsync(begin, 0, num_cells * sizeof(uint32_t), st));
	MB2_CUDA(cudaMemsetAsync(end, 0, num_cells * sizeof(uint32_t), st));
	if (n == 0) return;
	MB2_LAUNCH cell_ranges_kernel<<<(n + 255) / 256, 256, 0, st>>>(keys, n, shift, begin, end);
}

template <bool kFill>
static void launch_walk(const float4* sorted_pos, const uint32_t* keys, const uint32_t* s2o,
						const uint32_t* begin, const uint32_t* end, const StencilEntry* stencil,
						int ns, int m, int shift, float rc2, uint32_t n, const Box& box,
						const Exclusions& ex, uint32_t* counts, const uint32_t* row_start,
						uint32_t* nbr, cudaStream_t st) {
	if (n == 0) return;
	const size_t smem = static_cast<size_t>(ns) * sizeof(int4);
	const bool excl = ex.offsets != nullptr || ex.rigid_body_id != nullptr;
	auto kern = excl ? walk_kernel<kFill, true> : walk_kernel<kFill, false>;
	if (smem > 48 * 1024)
		MB2_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  static_cast<int>(smem)));
	MB2_LAUNCH kern<<<(n + 255) / 256, 256, smem, st>>>(sorted_pos, keys, s2o, begin, end, stencil, ns, m,
											 shift, rc2, n, box, ex, counts, row_start, nbr);
}

void neighbor_count(const float4* sorted_pos, const uint32_t* keys, const uint32_t* s2o,
					const uint32_t* begin, const uint32_t* end, const StencilEntry* stencil,
					int num_stencil, int m, int shift, float rc2, uint32_t n, const Box& box,
					const Exclusions& ex, uint32_t* counts, cudaStream_t st) {
	launch_walk<false>(sorted_pos, keys, s2o, begin, end, stencil, num_stencil, m, shift, rc2, n,
					   box, ex, counts, nullptr, nullptr, st);
}

void neighbor_fill(const float4* sorted_pos, const uint32_t* keys, const uint32_t* s2o,
				   const uint32_t* begin, const uint32_t* end, const StencilEntry* stencil,
				   int num_stencil, int m, int shift, float rc2, uint32_t n, const Box& box,
				   const Exclusions& ex, const uint32_t* row_start, uint32_t* nbr,
				   cudaStream_t st) {
	launch_walk<true>(sorted_pos, keys, s2o, begin, end, stencil, num_stencil, m, shift, rc2, n,
					  box, ex, nullptr, row_start, nbr, st);
}

void export_pairs(const uint32_t* row_start, const uint32_t* nbr, const uint32_t* s2o,
				  uint32_t n, int2* out, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH export_kernel<<<(n + 255) / 256, 256, 0, st>>>(row_start, nbr, s2o, n, out);
}

void max_displacement_sq(const float4* cur, const float4* prev, uint32_t n, const Box& box,
						 unsigned int* out_bits, cudaStream_t st) {
	MB2_CUDA(cudaMemsetAsync(out_bits, 0, sizeof(unsigned int), st));
	if (n == 0) return;
	const float3 len = make_float3(box.periodic[0] ? box.size[0] : 0.0f,
								   box.periodic[1] ? box.size[1] : 0.0f,
								   box.periodic[2] ? box.size[2] : 0.0f);
	MB2_LAUNCH displacement_kernel<<<(n + 255) / 256, 256, 0, st>>>(cur, prev, n, len, out_bits);
}

void pack_sorted_positions(const float4* pos, const int* type_ids, const uint32_t* s2o,
						   uint32_t n, float4* sorted_pos, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH pack_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, type_ids, s2o, n, sorted_pos);
}

}  // namespace mb2
