// Exclusive prefix sum of u32 values: reduce-then-scan over 1024-element
// blocks (256 threads x 4 items), a single-CTA scan of the block sums, then a
// block-local scan with the block's offset added.
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, d);
		if (lane >= d) v += t;
	}
	return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* excl) {
	__shared__ uint32_t warp_tot[kScanThreads / 32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const uint32_t inc = warp_incl_scan(v);
	if (lane == 31) warp_tot[warp] = inc;
	__syncthreads();
	if (warp == 0) {
		uint32_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
		t = warp_incl_scan(t);
		if (lane < kScanThreads / 32) warp_tot[lane] = t;
	}
	__syncthreads();
	const uint32_t warp_base = warp ? warp_tot[warp - 1] : 0u;
	*excl = warp_base + inc - v;
	const uint32_t total = warp_tot[kScanThreads / 32 - 1];
	__syncthreads();
	return total;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ in,
																   size_t n,
																   uint32_t* __restrict__ sums) {
	const size_t base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * kScanItems;
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k)
		if (base + k < n) s += in[base + k];
	uint32_t excl;
	const uint32_t total = block_excl_scan(s, &excl);
	if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One CTA scans `count` block sums in place (exclusive), carrying across chunks.
__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(uint32_t* sums, size_t count,
																 uint32_t* total) {
	uint32_t carry = 0;
	for (size_t base = 0; base < count; base += kScanThreads) {
		const size_t i = base + threadIdx.x;
		const uint32_t v = i < count ? sums[i] : 0u;
		uint32_t excl;
		const uint32_t t = block_excl_scan(v, &excl);
		if (i < count) sums[i] = carry + excl;
		carry += t;
	}
	if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t* in, size_t n,
																  const uint32_t* __restrict__ sums,
																  uint32_t* out) {
	const size_t base = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x * kScanItems;
	uint32_t v[kScanItems];
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		v[k] = base + k < n ? in[base + k] : 0u;
		s += v[k];
	}
	uint32_t excl;
	block_excl_scan(s, &excl);
	uint32_t run = sums[blockIdx.x] + excl;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		if (base + k < n) out[base + k] = run;
		run += v[k];
	}
}

}  // namespace

void exclusive_scan_u32(Scratch& s, const uint32_t* in, uint32_t* out, size_t n, uint32_t* total,
						cudaStream_t st) {
	if (n == 0) {
		if (total) MB2_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), st));
		return;
	}
	const size_t blocks = (n + kScanBlock - 1) / kScanBlock;
	s.scan_blocks.ensure(blocks);
	MB2_LAUNCH scan_reduce_kernel<<<blocks, kScanThreads, 0, st>>>(in, n, s.scan_blocks.ptr);
	MB2_LAUNCH scan_sums_kernel<<<1, kScanThreads, 0, st>>>(s.scan_blocks.ptr, blocks, total);
	MB2_LAUNCH scan_apply_kernel<<<blocks, kScanThreads, 0, st>>>(in, n, s.scan_blocks.ptr, out);
}

// Same scan with the block-sum buffer supplied by the caller: at least
// scan_blocks_needed(n) words, nothing of it read before it is written.
size_t scan_blocks_needed(size_t n) { return (n + kScanBlock - 1) / kScanBlock; }

void exclusive_scan_u32_into(const uint32_t* in, uint32_t* out, size_t n, uint32_t* block_sums,
							 cudaStream_t st) {
	if (n == 0) return;
	const size_t blocks = scan_blocks_needed(n);
	MB2_LAUNCH scan_reduce_kernel<<<blocks, kScanThreads, 0, st>>>(in, n, block_sums);
	MB2_LAUNCH scan_sums_kernel<<<1, kScanThreads, 0, st>>>(block_sums, blocks, nullptr);
	MB2_LAUNCH scan_apply_kernel<<<blocks, kScanThreads, 0, st>>>(in, n, block_sums, out);
}

}  // namespace mb2
