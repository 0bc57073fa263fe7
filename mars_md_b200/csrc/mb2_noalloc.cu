// Radix sort of (key, value) pairs over scratch that lives in this module's
// static device memory, for mb2_radix_sort_pairs_static.
//
// The context sort (mb2_radix_sort_pairs) grows its scratch with cudaMalloc
// the first time it sees a larger n, and cudaFree'ing the old buffer
// synchronises the device. Some callers cannot have either: a process whose
// memory is already handed out to another allocator (a framework's caching
// pool that holds nearly all of HBM, where a new cudaMalloc fails although the
// sort itself needs nothing new), or a latency-critical loop that must never
// stall on an implicit device-wide synchronisation. This variant uses a fixed
// array instead and so allocates nothing, at any n up to MB2_SORT_STATIC_MAX.
//
// Rules that follow from the shared array:
//  * Set-up: every call looks up the array's device address on the current
//    device (cudaGetSymbolAddress, a host-side lookup once the module is
//    loaded). With CUDA's lazy module loading the first lookup on a device
//    can itself load this module, which reserves the array's ~8.6 MB of
//    device memory then; so make one call (n = 0 is enough) at start-up,
//    before another allocator takes the device's free memory and before any
//    stream capture. After cudaDeviceReset the module is loaded anew, at a
//    possibly different address, by the next call's lookup (nothing stale is
//    kept); repeat the n = 0 call then.
//  * Every call on one device uses the same array, so calls that overlap in
//    time on one device (different streams, or host threads without ordering)
//    race and corrupt each other's results. Order them, e.g. one stream.
//  * Nothing in the array has to start at zero: each word a call reads was
//    written earlier in the same call.
#include <string>

#include "marsb200.h"
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

constexpr uint32_t kMaxPairs = MB2_SORT_STATIC_MAX;
static_assert(kMaxPairs % kSortTile == 0, "the maximum is a whole number of tiles");
constexpr size_t kAlignWords = 64;  // 256-byte sub-buffer alignment
constexpr size_t round_up(size_t w) { return (w + kAlignWords - 1) / kAlignWords * kAlignWords; }
constexpr size_t kHistWords = static_cast<size_t>(kMaxPairs / kSortTile) * 256u;
constexpr size_t kBlockSumWords = (kHistWords + 1023) / 1024;  // scan blocks of 1024 elements
constexpr size_t kKeysOff = 0;
constexpr size_t kValsOff = kKeysOff + round_up(kMaxPairs);
constexpr size_t kHistOff = kValsOff + round_up(kMaxPairs);
constexpr size_t kSumsOff = kHistOff + round_up(kHistWords);
constexpr size_t kWords = kSumsOff + round_up(kBlockSumWords);

// keys_alt | vals_alt | digit histogram | scan block sums (~8.6 MB).
static __device__ __align__(256) uint32_t g_sort_scratch[kWords];

// Device address of the array on the current device. In host code the
// array's name is only a host-side stand-in, never a device address, so the
// address is looked up (not cached: a cudaDeviceReset may move it).
uint32_t* scratch_on_current_device() {
	void* p = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
	if (e != cudaSuccess || p == nullptr)
		throw Error{MB2_ERR_CUDA, std::string("mb2_radix_sort_pairs_static: cudaGetSymbolAddress: ") +
									  cudaGetErrorString(e)};
	return static_cast<uint32_t*>(p);
}

}  // namespace

void radix_sort_pairs_static(uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st) {
	if (n > kMaxPairs)
		throw Error{MB2_ERR_CAPACITY,
					"mb2_radix_sort_pairs_static: n = " + std::to_string(n) +
						" exceeds MB2_SORT_STATIC_MAX = " + std::to_string(kMaxPairs) +
						"; use mb2_radix_sort_pairs"};
	uint32_t* base = scratch_on_current_device();
	if (n <= 1) return;
	const size_t hist_words = static_cast<size_t>((n + kSortTile - 1) / kSortTile) * 256u;
	if (hist_words > kHistWords || scan_blocks_needed(hist_words) > kBlockSumWords)
		throw Error{MB2_ERR_CAPACITY, "mb2_radix_sort_pairs_static: scratch layout too small"};
	radix_sort_pairs_into(keys, vals, n, base + kKeysOff, base + kValsOff, base + kHistOff,
						  base + kSumsOff, st);
}

}  // namespace mb2
