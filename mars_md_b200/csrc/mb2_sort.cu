// Z-order (Morton) sort: encode, stable LSD radix sort of (key, index),
// inverse map and gather of sorted positions.
//
// Replaces MortonEncodeKernel / InverseIndexKernel / ReorderDataKernel
// (src/PatchOperation/ZOrderKernels/ZOrderKernels.h:27-83) and the CUB call in
// device_radix_sort_pairs_cub (src/PatchOperation/ZOrderKernels/CUDASort.cu:13-98).
//
// Radix sort layout: each pass sorts on one 8-bit digit. A tile of
// kTile = kWarps * 32 * kRounds consecutive elements belongs to one CTA.
//   1. histogram: per-tile digit counts, stored digit-major [256][tiles]
//   2. scan:      exclusive prefix over that digit-major array gives each
//                 (digit, tile) its global output offset
//   3. scatter:   each CTA ranks its elements stably (rounds in order, warps
//                 in order within a round, lanes in order within a warp, via
//                 __match_any_sync) and writes them out.
// Stable per pass, so four passes equal a stable sort on the 32-bit key,
// which is the CUB SortPairs contract the reference relies on.
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

constexpr int kWarps = 8;
constexpr int kRounds = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kTile = kThreads * kRounds;  // 2048 elements per CTA

__global__ void __launch_bounds__(256) morton_encode_kernel(const float4* __restrict__ pos,
															uint32_t n, float3 lo, float3 range,
															uint32_t* __restrict__ keys,
															uint32_t* __restrict__ idx) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 p = pos[i];
	const uint32_t x = morton_coord(p.x, lo.x, range.x);
	const uint32_t y = morton_coord(p.y, lo.y, range.y);
	const uint32_t z = morton_coord(p.z, lo.z, range.z);
	keys[i] = split_by3(z) | (split_by3(y) << 1) | (split_by3(x) << 2);
	idx[i] = i;
}

__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const uint32_t* __restrict__ keys,
															  uint32_t n, int shift,
															  uint32_t num_tiles,
															  uint32_t* __restrict__ hist) {
	__shared__ uint32_t counts[256];
	counts[threadIdx.x] = 0;
	__syncthreads();
	const uint32_t base = blockIdx.x * kTile;
	for (int r = 0; r < kRounds; ++r) {
		const uint32_t i = base + r * kThreads + threadIdx.x;
		if (i < n) atomicAdd(&counts[(keys[i] >> shift) & 255u], 1u);
	}
	__syncthreads();
	hist[threadIdx.x * num_tiles + blockIdx.x] = counts[threadIdx.x];
}

__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
	const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t n,
	int shift, uint32_t num_tiles, const uint32_t* __restrict__ offsets,
	uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
	__shared__ uint32_t running[256];          // next free output slot per digit
	__shared__ uint32_t warp_counts[kWarps][256];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	running[threadIdx.x] = offsets[threadIdx.x * num_tiles + blockIdx.x];
	const uint32_t base = blockIdx.x * kTile;
	const uint32_t lanemask_lt = (1u << lane) - 1u;
	for (int r = 0; r < kRounds; ++r) {
		for (int w = 0; w < kWarps; ++w) warp_counts[w][threadIdx.x] = 0;
		__syncthreads();
		const uint32_t i = base + (r * kWarps + warp) * 32 + lane;
		const bool valid = i < n;
		const uint32_t key = valid ? keys_in[i] : 0u;
		const uint32_t val = valid ? vals_in[i] : 0u;
		// Invalid lanes take digit 256, which never matches a real digit.
		const uint32_t digit = valid ? (key >> shift) & 255u : 256u;
		const uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
		const uint32_t rank_in_warp = __popc(peers & lanemask_lt);
		const bool leader = (peers & lanemask_lt) == 0;
		if (valid && leader) warp_counts[warp][digit] = __popc(peers);
		__syncthreads();
		// One thread per digit: exclusive prefix over the warps of this round.
		{
			const int d = threadIdx.x;
			uint32_t acc = running[d];
#pragma unroll
			for (int w = 0; w < kWarps; ++w) {
				const uint32_t c = warp_counts[w][d];
				warp_counts[w][d] = acc;
				acc += c;
			}
			running[d] = acc;
		}
		__syncthreads();
		if (valid) {
			const uint32_t dst = warp_counts[warp][digit] + rank_in_warp;
			keys_out[dst] = key;
			vals_out[dst] = val;
		}
		__syncthreads();
	}
}

__global__ void __launch_bounds__(256) inverse_gather_kernel(const uint32_t* __restrict__ s2o,
															 uint32_t n,
															 const float4* __restrict__ pos,
															 uint32_t* __restrict__ inv,
															 float4* __restrict__ sorted_pos) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t o = s2o[i];
	if (inv && o < n) inv[o] = i;
	if (sorted_pos) sorted_pos[i] = pos[o];
}

// out[s] = in[s2o[s]] for 4- or 16-byte elements (DeviceParticle::permute).
template <typename T>
__global__ void __launch_bounds__(256) permute_kernel(const T* __restrict__ in,
													  const uint32_t* __restrict__ s2o, uint32_t n,
													  T* __restrict__ out) {
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) out[s] = in[s2o[s]];
}

// RemapIndicesKernel (ZOrderKernels.h:87-101): in-range indices go through inv.
__global__ void __launch_bounds__(256) remap_kernel(int* __restrict__ idx, size_t count,
													const uint32_t* __restrict__ inv, uint32_t n) {
	const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= count) return;
	const int v = idx[i];
	if (v >= 0 && static_cast<uint32_t>(v) < n) idx[i] = static_cast<int>(inv[v]);
}

}  // namespace

namespace {

// Up to this many pairs the sort runs in one CTA: the passes above take
// twenty launches, which at a few thousand elements is launch latency.
constexpr uint32_t kOneBlockSortMax = 8192;

// One-CTA sort of up to kOneBlockSortMax (key, value) pairs, stable: a
// bitonic network in shared memory over (key << 32 | position), whose
// composites are distinct, so their order is the stable order by key; each
// value then follows its position. p2: n rounded up to a power of two
// (padding sorts last).
__global__ void __launch_bounds__(1024) sort_one_block_kernel(uint32_t* __restrict__ keys,
															  uint32_t* __restrict__ vals,
															  uint32_t n, uint32_t p2) {
	extern __shared__ unsigned long long comp[];
	uint32_t* vsh = reinterpret_cast<uint32_t*>(comp + p2);
	for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) {
		comp[i] = i < n ? (static_cast<unsigned long long>(keys[i]) << 32) | i : ~0ull;
		if (i < n) vsh[i] = vals[i];
	}
	__syncthreads();
	for (uint32_t k = 2; k <= p2; k <<= 1) {
		for (uint32_t j = k >> 1; j > 0; j >>= 1) {
			for (uint32_t t = threadIdx.x; t < p2 / 2; t += blockDim.x) {
				const uint32_t lo = 2 * t - (t & (j - 1));  // bit j of lo clear
				const uint32_t hi = lo + j;
				const unsigned long long a = comp[lo], b = comp[hi];
				const bool ascending = (lo & k) == 0;
				if ((a > b) == ascending) {
					comp[lo] = b;
					comp[hi] = a;
				}
			}
			__syncthreads();
		}
	}
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
		const unsigned long long c = comp[i];
		keys[i] = static_cast<uint32_t>(c >> 32);
		vals[i] = vsh[static_cast<uint32_t>(c)];
	}
}

}  // namespace

void radix_sort_pairs(Scratch& s, uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st) {
	if (n <= 1) return;
	if (n <= kOneBlockSortMax) {
		uint32_t p2 = 2;
		while (p2 < n) p2 <<= 1;
		const size_t smem = static_cast<size_t>(p2) * (sizeof(unsigned long long) + sizeof(uint32_t));
		if (smem > 48 * 1024)
			MB2_CUDA(cudaFuncSetAttribute(sort_one_block_kernel,
										  cudaFuncAttributeMaxDynamicSharedMemorySize,
										  static_cast<int>(smem)));
		MB2_LAUNCH sort_one_block_kernel<<<1, 1024, smem, st>>>(keys, vals, n, p2);
		return;
	}
	const uint32_t tiles = (n + kTile - 1) / kTile;
	s.ensure_sort(n, tiles * 256u);
	uint32_t *ks = keys, *vs = vals, *kd = s.sort_keys_alt, *vd = s.sort_vals_alt;
	for (int pass = 0; pass < 4; ++pass) {
		const int shift = 8 * pass;
		MB2_LAUNCH radix_hist_kernel<<<tiles, kThreads, 0, st>>>(ks, n, shift, tiles, s.sort_hist);
		exclusive_scan_u32(s, s.sort_hist, s.sort_hist, tiles * 256u, nullptr, st);
		MB2_LAUNCH radix_scatter_kernel<<<tiles, kThreads, 0, st>>>(ks, vs, n, shift, tiles, s.sort_hist, kd,
														 vd);
		uint32_t* t = ks;
		ks = kd;
		kd = t;
		t = vs;
		vs = vd;
		vd = t;
	}
	// Four passes: the sorted data is back in the caller's buffers.
}

static_assert(kTile == kSortTile, "tile size shared with the scratch sizing");

void radix_sort_pairs_into(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t* keys_alt,
						   uint32_t* vals_alt, uint32_t* hist, uint32_t* block_sums,
						   cudaStream_t st) {
	if (n <= 1) return;
	const uint32_t tiles = (n + kTile - 1) / kTile;
	uint32_t *ks = keys, *vs = vals, *kd = keys_alt, *vd = vals_alt;
	for (int pass = 0; pass < 4; ++pass) {
		const int shift = 8 * pass;
		MB2_LAUNCH radix_hist_kernel<<<tiles, kThreads, 0, st>>>(ks, n, shift, tiles, hist);
		exclusive_scan_u32_into(hist, hist, static_cast<size_t>(tiles) * 256u, block_sums, st);
		MB2_LAUNCH radix_scatter_kernel<<<tiles, kThreads, 0, st>>>(ks, vs, n, shift, tiles, hist,
																	kd, vd);
		uint32_t* t = ks;
		ks = kd;
		kd = t;
		t = vs;
		vs = vd;
		vd = t;
	}
}

void morton_encode(const float4* pos, uint32_t n, const float* bmin, const float* bmax,
				   uint32_t* keys, uint32_t* idx, cudaStream_t st) {
	float3 lo = make_float3(bmin[0], bmin[1], bmin[2]);
	// range = fmaxf(box_max - box_min, 1e-6f), per axis, in float (MortonCode.h:97-109)
	float3 range = make_float3(fmaxf(bmax[0] - bmin[0], 1e-6f), fmaxf(bmax[1] - bmin[1], 1e-6f),
							   fmaxf(bmax[2] - bmin[2], 1e-6f));
	if (n == 0) return;
	MB2_LAUNCH morton_encode_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, n, lo, range, keys, idx);
}

void inverse_and_gather(const uint32_t* s2o, uint32_t n, const float4* pos, uint32_t* inv,
						float4* sorted_pos, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH inverse_gather_kernel<<<(n + 255) / 256, 256, 0, st>>>(s2o, n, pos, inv, sorted_pos);
}

void permute_gather(const void* in, const uint32_t* s2o, uint32_t n, int elem_bytes, void* out,
					cudaStream_t st) {
	if (n == 0) return;
	if (elem_bytes == 16)
		MB2_LAUNCH permute_kernel<float4><<<(n + 255) / 256, 256, 0, st>>>(
			static_cast<const float4*>(in), s2o, n, static_cast<float4*>(out));
	else
		MB2_LAUNCH permute_kernel<uint32_t><<<(n + 255) / 256, 256, 0, st>>>(
			static_cast<const uint32_t*>(in), s2o, n, static_cast<uint32_t*>(out));
}

void remap_indices(int* idx, size_t count, const uint32_t* inv, uint32_t n, cudaStream_t st) {
	if (count == 0) return;
	MB2_LAUNCH remap_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(idx, count,
																						inv, n);
}

}  // namespace mb2
