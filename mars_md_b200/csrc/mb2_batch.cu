// Batched replicas: many independent periodic systems of uneven size stepped
// together, one launch per stage for all of them.
//
// Layout. Systems are concatenated in the caller's arrays (system s owns
// particles [offset[s], offset[s+1])). The sort key of a particle is
// (s << 21) | (21-bit Morton code of its position in its own box), so one
// radix sort groups the systems and orders each one spatially; cells of
// system s are the top 3 m_s bits of its 21-bit code, stored after the cells
// of systems < s. The pairlist is one sliced-ELL half list over all sorted
// particles (a row's neighbours are always in its own system), walked one
// warp per row over the row's own system grid, box and stencil.
// Pair forces read each row's box from the system table; the integrator
// gathers the pair force through the inverse permutation and keys its noise
// exactly as a plain step of system s with seed (seed + s) would: Philox key
// mixed from (seed + s, patch_id, step), counter = index within the system.
//
// mb2_batch_run captures the non-rebuild step (pack, clear, pair, integrate,
// step counter) in a CUDA graph and replays it; pairlist rebuilds run eagerly
// at the rebuild period (the list is re-sized from the walk's counts).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "marsb200.h"
#include "mb2_internal.cuh"
#include "mb2_walk.cuh"

using namespace mb2;

namespace {

constexpr int kSysShift = 21;   // key = system << 21 | 21-bit Morton code
constexpr int kLocalBits = 7;   // Morton bits per axis inside a system
constexpr uint32_t kLocalMask = (1u << kSysShift) - 1u;
constexpr int kMaxLevel = kLocalBits;

// Per-system cell grid and walk parameters (device copy per system).
struct SysGrid {
	WalkGrid wg;           // wg.shift = 3 * (7 - m)
	uint32_t cell_base;    // first global cell of the system
	uint32_t stencil_off;  // the system's pruned cell stencil in the batch's array
	uint32_t stencil_n;
	uint32_t pad;
};

__device__ __forceinline__ uint32_t morton7(float x, float o, float scale) {
	const float t = __fmul_rn(__fsub_rn(x, o), scale);
	const int q = static_cast<int>(floorf(t));
	return static_cast<uint32_t>(min(max(q, 0), (1 << kLocalBits) - 1));
}

// Morton key of one particle in its own system's box.
__device__ __forceinline__ uint32_t batch_key(const float4& p, const Box& b, uint32_t s) {
	const float k = static_cast<float>(1 << kLocalBits);
	const uint32_t x = morton7(p.x, b.origin[0], __fmul_rn(k, b.inv[0]));
	const uint32_t y = morton7(p.y, b.origin[1], __fmul_rn(k, b.inv[1]));
	const uint32_t z = morton7(p.z, b.origin[2], __fmul_rn(k, b.inv[2]));
	return (s << kSysShift) | split_by3(z) | (split_by3(y) << 1) | (split_by3(x) << 2);
}

__global__ void __launch_bounds__(256) batch_encode_kernel(const float4* __restrict__ pos,
														   const uint32_t* __restrict__ sys_of,
														   const Box* __restrict__ boxes,
														   uint32_t n, uint32_t* __restrict__ keys,
														   uint32_t* __restrict__ idx) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t s = sys_of[i];
	keys[i] = batch_key(pos[i], boxes[s], s);
	idx[i] = i;
}

// A rebuild of some systems: their particles' keys, packed system after
// system (cstart[s]: the number of rebuilt particles before system s; the
// systems' particles are contiguous in the caller's order too).
__global__ void __launch_bounds__(256) batch_compact_kernel(
	const float4* __restrict__ pos, const uint32_t* __restrict__ sys_of,
	const Box* __restrict__ boxes, const uint32_t* __restrict__ offsets,
	const uint32_t* __restrict__ flags, const uint32_t* __restrict__ cstart, uint32_t n,
	uint32_t* __restrict__ ckeys, uint32_t* __restrict__ cidx) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t s = sys_of[i];
	if (!flags[s]) return;
	const uint32_t c = cstart[s] + (i - offsets[s]);
	ckeys[c] = batch_key(pos[i], boxes[s], s);
	cidx[c] = i;
}

// The rebuilt systems' sorted keys into their systems' fixed ranges of the
// sorted arrays (system s owns sorted slots [offsets[s], offsets[s + 1])).
__global__ void __launch_bounds__(256) batch_scatter_sorted_kernel(
	const uint32_t* __restrict__ ckeys, const uint32_t* __restrict__ cidx, uint32_t m,
	const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ cstart,
	uint32_t* __restrict__ keys, uint32_t* __restrict__ s2o) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= m) return;
	const uint32_t key = ckeys[k];
	const uint32_t s = key >> kSysShift;
	const uint32_t g = offsets[s] + (k - cstart[s]);
	keys[g] = key;
	s2o[g] = cidx[k];
}

// Row statistics of the whole list: stats[0] += entries, stats[1] = the
// longest row. A grid-stride loop reduced per block, one pair of atomics per
// block (per-warp atomics on the two words serialised to ~0.1 ms).
__global__ void __launch_bounds__(256) batch_row_stats_kernel(const uint32_t* __restrict__ row_len,
															  uint32_t n,
															  unsigned long long* __restrict__ stats) {
	__shared__ unsigned long long part[2][8];
	unsigned long long tot = 0, mx = 0;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const unsigned long long v = row_len[i];
		tot += v;
		mx = max(mx, v);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
		mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
	}
	const int w = threadIdx.x >> 5;
	if ((threadIdx.x & 31) == 0) {
		part[0][w] = tot;
		part[1][w] = mx;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k) {
			tot += part[0][k];
			mx = max(mx, part[1][k]);
		}
		if (tot) {
			atomicAdd(stats, tot);
			atomicMax(stats + 1, mx);
		}
	}
}

// The list-build snapshot of the rebuilt systems' positions (flags null:
// every system), from which their displacements are measured.
__global__ void __launch_bounds__(256) batch_snapshot_kernel(const float4* __restrict__ pos,
															 const uint32_t* __restrict__ sys_of,
															 const uint32_t* __restrict__ flags,
															 uint32_t n, float4* __restrict__ ref) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (flags && !flags[sys_of[i]]) return;
	ref[i] = pos[i];
}

__global__ void __launch_bounds__(256) batch_cell_ranges_kernel(const uint32_t* __restrict__ keys,
																uint32_t n,
																const SysGrid* __restrict__ grids,
																uint32_t* __restrict__ begin,
																uint32_t* __restrict__ end) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	auto cell = [&](uint32_t key) {
		const SysGrid& g = grids[key >> kSysShift];
		return g.cell_base + ((key & kLocalMask) >> g.wg.shift);
	};
	const uint32_t c = cell(keys[i]);
	if (i == 0 || cell(keys[i - 1]) != c) begin[c] = i;
	if (i + 1 == n || cell(keys[i + 1]) != c) end[c] = i + 1;
}

// One warp per particle row, the plain path's row walk (build_rows_kernel)
// with the row's own system: its cell grid, its box (periodic on every axis)
// and its pruned stencil. The lanes take the stencil's cells 32 at a time
// (cells whose Morton code precedes the particle's hold only earlier
// particles of the system and are skipped), lay their candidate ranges end to
// end by a warp scan, and test 32 consecutive candidates a round with the
// reference's exact test, each lane finding its candidate's cell by a binary
// search over the running totals held one per lane. Hits are appended in
// candidate order. Six resident blocks per SM (40 registers): 1 % faster per
// build than 48 registers at five, and than 32 at eight.
__device__ __forceinline__ uint32_t batch_row(
	uint32_t i, uint32_t lane, const float4* __restrict__ sorted_pos,
	const uint32_t* __restrict__ keys, const uint32_t* __restrict__ s2o,
	const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
	const SysGrid* __restrict__ grids, const Box* __restrict__ boxes,
	const uint4* __restrict__ stencil, uint32_t* __restrict__ nbr, uint32_t cap, int hshift) {
	const uint32_t lt = (1u << lane) - 1u;
	const uint32_t key = keys[i];
	const uint32_t sys = key >> kSysShift;
	const SysGrid* g = grids + sys;
	const int m = g->wg.m;
	const uint32_t c = (key & kLocalMask) >> g->wg.shift;
	const float rc2 = g->wg.rc2;
	const uint32_t cell_base = g->cell_base;
	const uint4* st = stencil + g->stencil_off;
	const int ns = static_cast<int>(g->stencil_n);
	const Box* bx = boxes + sys;
	const float lx = bx->size[0], ly = bx->size[1], lz = bx->size[2];
	const float ix = bx->inv[0], iy = bx->inv[1], iz = bx->inv[2];
	const float hx = bx->half[0], hy = bx->half[1], hz = bx->half[2];
	// Interleaved (Morton) cell codes: x bits at 3k + 2, y at 3k + 1, z at 3k.
	// A neighbour's code is the home code plus the stencil offset on each axis
	// in interleaved form, carried through the other axes' bits (set to one)
	// and masked, which wraps every axis modulo 2^m.
	const uint32_t lvl = (1u << (3 * m)) - 1u;
	const uint32_t mx = 0x24924924u & lvl, my = 0x12492492u & lvl, mz = 0x09249249u & lvl;
	const uint32_t cxo = c | ~mx, cyo = c | ~my, czo = c | ~mz;
	const float4 pi = sorted_pos[i];
	const int a = static_cast<int>(s2o[i]);
	const uint32_t h = 1u << hshift;
	uint32_t* base = nbr + (static_cast<size_t>(i >> hshift) * cap << hshift) + (i & (h - 1u));
	uint32_t len = 0;
	for (int k0 = 0; k0 < ns; k0 += 32) {
		uint32_t jb = 0, je = 0;
		const int k = k0 + static_cast<int>(lane);
		if (k < ns) {
			const uint4 se = st[k];  // interleaved offsets, modulo 2^m per axis
			const uint32_t nc = ((cxo + se.x) & mx) | ((cyo + se.y) & my) | ((czo + se.z) & mz);
			if (nc >= c) {
				const uint32_t b = begin[cell_base + nc];
				jb = b > i + 1u ? b : i + 1u;
				je = end[cell_base + nc];
			}
		}
		// The chunk's candidate ranges laid end to end (a scan of their
		// lengths); each round the lanes take the next 32 candidates, lane l
		// finding the cell that holds candidate t0 + l by a binary search over
		// the lanes' running totals. An empty cell (begin = end = 0) or one
		// ending at i has jb >= je.
		const uint32_t cnt = je > jb ? je - jb : 0u;
		uint32_t incl = cnt;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
			if (static_cast<int>(lane) >= o) incl += v;
		}
		const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
		const uint32_t excl = incl - cnt;
		for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
			const uint32_t t = t0 + lane;
			int owner = 0;  // first lane whose running total exceeds t
#pragma unroll
			for (int step = 16; step > 0; step >>= 1) {
				const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, owner + step - 1);
				if (v <= t) owner += step;
			}
			const uint32_t ob = __shfl_sync(0xFFFFFFFFu, jb, owner & 31);
			const uint32_t oe = __shfl_sync(0xFFFFFFFFu, excl, owner & 31);
			bool hit = false;
			uint32_t entry = 0;
			if (t < total) {
				const uint32_t j = ob + (t - oe);
				const float4 pj = sorted_pos[j];
				const float dx = wrap_diff_scalar(__fsub_rn(pj.x, pi.x), lx, ix, hx);
				const float dy = wrap_diff_scalar(__fsub_rn(pj.y, pi.y), ly, iy, hy);
				const float dz = wrap_diff_scalar(__fsub_rn(pj.z, pi.z), lz, iz, hz);
				if (len2(dx, dy, dz) <= rc2) {
					hit = true;
					entry = j | (static_cast<int>(s2o[j]) < a ? kOrientBit : 0u);
				}
			}
			const uint32_t hm = __ballot_sync(0xFFFFFFFFu, hit);
			if (hit) {
				const uint32_t p = len + static_cast<uint32_t>(__popc(hm & lt));
				if (p < cap) base[static_cast<size_t>(p) * h] = entry;
			}
			len += static_cast<uint32_t>(__popc(hm));
		}
	}
	return len;
}

// One warp per group of 32 consecutive sorted particles: a group whose
// particles all belong to one system and sit in cells within emax of each
// other walks as the plain group walk does (walk_coherent_group, over the
// system's grid and box: candidate cells pruned by their real distance from
// the group's coordinate range, candidates dropped 32 at a time by the group
// test, each survivor loaded once for all 32 lanes and decided by the cheap
// test, the exact test behind a warp vote). Any other group (at a system's
// start or end, or across a Morton discontinuity) walks its rows one at a
// time with the row walk. Same pair set; rows in candidate order.
__global__ void __launch_bounds__(256, 7) batch_group_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ keys,
	const uint32_t* __restrict__ s2o, const uint32_t* __restrict__ begin,
	const uint32_t* __restrict__ end, const SysGrid* __restrict__ grids,
	const Box* __restrict__ boxes, const uint4* __restrict__ stencil,
	const uint32_t* __restrict__ flags, uint32_t n, uint32_t* __restrict__ nbr, uint32_t cap,
	int hshift, uint32_t* __restrict__ row_len) {
	__shared__ uint32_t split_tab[1 << kLocalBits];
	__shared__ uint4 cell_buf[8 * kCellBuf];  // per warp: kept cells (jlo, end, image code, offset)
	__shared__ float4 cand_buf[8 * 32];       // per warp: candidates that pass the group test
	for (int k = threadIdx.x; k < (1 << kLocalBits); k += blockDim.x) split_tab[k] = split_by3(k);
	__syncthreads();
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t i_first = i & ~31u;
	if (i_first >= n) return;  // whole warp past the end
	const uint32_t lane = threadIdx.x & 31u;
	const bool valid = i < n;
	const uint32_t key = valid ? keys[i] : 0u;
	const uint32_t sys = key >> kSysShift;
	const uint32_t sys0 = __shfl_sync(0xFFFFFFFFu, sys, 0);
	const bool one_system = __all_sync(0xFFFFFFFFu, !valid || sys == sys0);
	// Only the rows of systems being rebuilt (flags null: all) are walked;
	// the others keep their rows.
	const bool walked = valid && (!flags || flags[sys]);
	if (!__any_sync(0xFFFFFFFFu, walked)) return;
	const SysGrid* g = grids + sys0;
	const WalkGrid& wg = g->wg;
	const uint32_t c = (key & kLocalMask) >> wg.shift;
	const int cx = static_cast<int>(compact_by3(c >> 2));
	const int cy = static_cast<int>(compact_by3(c >> 1));
	const int cz = static_cast<int>(compact_by3(c));
	const int x0 = warp_min(valid ? cx : INT_MAX), x1 = warp_max(valid ? cx : INT_MIN);
	const int y0 = warp_min(valid ? cy : INT_MAX), y1 = warp_max(valid ? cy : INT_MIN);
	const int z0 = warp_min(valid ? cz : INT_MAX), z1 = warp_max(valid ? cz : INT_MIN);
	const bool coherent = one_system && (x1 - x0) <= wg.emax && (y1 - y0) <= wg.emax &&
						  (z1 - z0) <= wg.emax;
	uint32_t len = 0;
	if (coherent) {
		const float4 pi = valid ? sorted_pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
		const int a = valid ? static_cast<int>(s2o[i]) : 0;
		const float gxlo = warp_minf(valid ? pi.x : INFINITY), gxhi = warp_maxf(valid ? pi.x : -INFINITY);
		const float gylo = warp_minf(valid ? pi.y : INFINITY), gyhi = warp_maxf(valid ? pi.y : -INFINITY);
		const float gzlo = warp_minf(valid ? pi.z : INFINITY), gzhi = warp_maxf(valid ? pi.z : -INFINITY);
		const int h = 1 << hshift;
		RowWriter row{nbr + (static_cast<size_t>(i >> hshift) * cap << hshift) + (i & (h - 1)), 0u,
					  0u, cap, h};
		const uint32_t c_first = __shfl_sync(0xFFFFFFFFu, c, 0);
		walk_coherent_group<false, true>(sorted_pos, s2o, begin + g->cell_base, end + g->cell_base,
										 split_tab, cell_buf,
										 cand_buf, wg, boxes[sys0], Exclusions{}, i, i_first,
										 valid, pi, a, 0, 0, -1, c_first, x0, x1, y0, y1, z0, z1,
										 gxlo, gxhi, gylo, gyhi, gzlo, gzhi, row);
		len = row.total();
	} else {
		uint32_t todo = __ballot_sync(0xFFFFFFFFu, walked);
		while (todo) {
			const int l = __ffs(todo) - 1;
			todo &= todo - 1u;
			const uint32_t len_l = batch_row(i_first + static_cast<uint32_t>(l), lane, sorted_pos,
											 keys, s2o, begin, end, grids, boxes, stencil, nbr,
											 cap, hshift);
			if (static_cast<int>(lane) == l) len = len_l;
		}
	}
	if (walked) row_len[i] = len;
}

// Largest squared displacement of each system's particles since their
// list-build snapshot, into out[system] (float bits; non-negative floats
// order like their bit patterns).
__global__ void __launch_bounds__(256) batch_displacement_kernel(
	const float4* __restrict__ cur, const float4* __restrict__ prev,
	const uint32_t* __restrict__ sys_of, const Box* __restrict__ boxes, uint32_t n,
	unsigned int* __restrict__ out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t i_first = i & ~31u;
	float d2 = 0.0f;
	const uint32_t s = i_first < n ? sys_of[i < n ? i : i_first] : 0u;
	if (i < n) {
		const Box& b = boxes[s];
		const float4 c = cur[i], p = prev[i];
		const float3 d = wrap_diff(b, __fsub_rn(c.x, p.x), __fsub_rn(c.y, p.y), __fsub_rn(c.z, p.z));
		d2 = len2(d.x, d.y, d.z);
	}
	// A warp of one system reduces first; the block's warps then merge runs
	// of one system, so that a system takes about one atomic per block.
	__shared__ uint32_t wsys[8];
	__shared__ float wmax[8];
	const uint32_t s0 = __shfl_sync(0xFFFFFFFFu, s, 0);
	const int w = threadIdx.x >> 5;
	if (__all_sync(0xFFFFFFFFu, s == s0)) {
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xFFFFFFFFu, d2, o));
		if ((threadIdx.x & 31) == 0) {
			wsys[w] = s0;
			wmax[w] = d2;
		}
	} else {
		if (i < n) atomicMax(&out[s], __float_as_uint(d2));
		if ((threadIdx.x & 31) == 0) wsys[w] = 0xFFFFFFFFu;  // already applied
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		const int warps = static_cast<int>(blockDim.x >> 5);
		uint32_t run = 0xFFFFFFFFu;  // system of the current run of warps
		float m = 0.0f;
		for (int k = 0; k < warps; ++k) {
			// Warps past the end of the particles hold nothing.
			if (blockIdx.x * blockDim.x + static_cast<uint32_t>(k) * 32u >= n) break;
			if (wsys[k] != run) {
				if (run != 0xFFFFFFFFu) atomicMax(&out[run], __float_as_uint(m));
				run = wsys[k];
				m = 0.0f;
			}
			if (run != 0xFFFFFFFFu) m = fmaxf(m, wmax[k]);
		}
		if (run != 0xFFFFFFFFu) atomicMax(&out[run], __float_as_uint(m));
	}
}

}  // namespace

struct mb2_batch {
	int device = 0;
	std::string last_error;
	uint32_t num_systems = 0;
	uint32_t n = 0;
	std::vector<uint32_t> offsets;  // host [S + 1]
	std::vector<Box> boxes_h;
	DevBuf<uint32_t> offsets_d, sys_of;
	DevBuf<Box> boxes;
	Scratch scratch;
	// sort / list state
	DevBuf<uint32_t> keys, s2o, inv, row_len, row_off, nbr, cell_begin, cell_end;
	DevBuf<uint32_t> ckeys, cidx, sys_flags, cstart;  // a partial rebuild's keys, flags, starts
	DevBuf<float4> sorted_pos, ref_pos, force_sorted;
	DevBuf<SysGrid> grids;
	std::vector<SysGrid> grids_h;
	DevBuf<uint4> stencil;  // every system's pruned cell stencil (interleaved offsets), concatenated
	uint32_t total_cells = 0;
	float grid_rc = -1.0f;
	int level_offset = 0;
	// Rebuild cadence in force (0: the params' rebuild_period), set by
	// mb2_batch_set_rebuild_period or chosen by mb2_batch_autotune.
	uint32_t rebuild_period = 0;
	unsigned long long rebuilds = 0;         // list builds since creation (steps with any)
	unsigned long long system_rebuilds = 0;  // systems rebuilt, summed over those builds
	DevBuf<unsigned long long> stats, step_d;
	DevBuf<unsigned int> disp;
	DevBuf<double> energy;
	unsigned long long* pinned = nullptr;
	unsigned int* pinned_sys = nullptr;  // per system: displacement readback, then rebuild flags
	unsigned int* pinned_cstart = nullptr;  // per system: rebuilt particles before it
	bool built = false;
	uint64_t num_pairs = 0;
	uint32_t cap = 0;
	int lanes = 0;
	int lanes_request = 0;
	// tables and types
	PairTables pt;
	DevBuf<PairTableRef> refs;
	DevBuf<int> table_offsets;
	DevBuf<float> bin_force;
	DevBuf<float2> bin_energy;
	TypeTable types;
	bool types_set = false;
	DevBuf<float> charge;
	DevBuf<float4> diffusion, fg_scale;
	DevBuf<int> pmf_off, pmf_cnt;
	DevBuf<int4> fg_id;
	// captured step
	cudaGraphExec_t graph = nullptr;
	std::vector<uint64_t> graph_key;
	unsigned long long launches_per_graph = 0;

	~mb2_batch() {
		if (graph) cudaGraphExecDestroy(graph);
		if (pinned) cudaFreeHost(pinned);
		if (pinned_sys) cudaFreeHost(pinned_sys);
		if (pinned_cstart) cudaFreeHost(pinned_cstart);
	}
};

namespace {

template <typename F>
int bguard(mb2_batch* b, F&& f) {
	if (!b) return MB2_ERR_ARG;
	try {
		MB2_CUDA(cudaSetDevice(b->device));
		f();
		MB2_CUDA(cudaGetLastError());
		b->last_error.clear();
		return MB2_OK;
	} catch (const Error& e) {
		b->last_error = e.msg;
		return e.code;
	} catch (const std::exception& e) {
		b->last_error = e.what();
		return MB2_ERR_CUDA;
	}
}

cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

uint64_t f2u(float f) {
	uint32_t u;
	std::memcpy(&u, &f, 4);
	return u;
}

// Per-system cell grids for list radius rc: the cost-model level (capped at
// the 7-bit Morton scale) shifted by the tuner's level offset.
void choose_grids(mb2_batch* b, float rc) {
	b->grids_h.resize(b->num_systems);
	std::vector<uint4> stencil;
	uint32_t base = 0;
	for (uint32_t s = 0; s < b->num_systems; ++s) {
		const Box& bx = b->boxes_h[s];
		const uint32_t ns = b->offsets[s + 1] - b->offsets[s];
		const CellGrid g0 = choose_cell_grid(bx.size, bx.periodic, rc, ns, 0, kMaxLevel);
		const int m = std::min(std::max(g0.m + b->level_offset, 0), kMaxLevel);
		const CellGrid g = (m == g0.m) ? g0 : choose_cell_grid(bx.size, bx.periodic, rc, ns, m, m);
		SysGrid sg{};
		WalkGrid& wg = sg.wg;
		wg.m = g.m;
		wg.shift = 3 * (kLocalBits - g.m);
		// Groups whose cells spread up to 5 apart walk together (coherent);
		// the rest walk row by row: 5.27 ms per build against 5.33 at 3 and
		// 5.75 at 7 (wider candidate boxes).
		wg.emax = 5;
		for (int a = 0; a < 3; ++a) {
			wg.radius[a] = g.radius[a];
			wg.wmin[a] = g.wmin[a];
			wg.full[a] = g.m == 0 || 2 * g.radius[a] + 1 >= (1 << g.m);
		}
		wg.lim = g.lim;
		wg.rc2 = rc * rc;
		fast_test_band(bx, rc, &wg.fast_lo, &wg.fast_hi);
		wg.split2 = INFINITY;
		// Cell c of level m spans Morton coordinates [c, c + 1) * 2^(7 - m) of
		// the 7-bit scale over the box, L / 2^m wide; the margin covers the
		// rounding of that mapping, as on the plain path.
		for (int a = 0; a < 3; ++a) {
			wg.dom_lo[a] = bx.origin[a];
			wg.cell_w[a] = static_cast<float>(static_cast<double>(bx.size[a]) / (1 << g.m));
			wg.eps[a] = static_cast<float>(
				1e-5 * (std::fabs(static_cast<double>(bx.origin[a])) + bx.size[a]) + 1e-6);
		}
		sg.cell_base = base;
		sg.stencil_off = static_cast<uint32_t>(stencil.size());
		sg.stencil_n = static_cast<uint32_t>(g.stencil.size());
		// Offsets modulo 2^m per axis (every batched box is periodic), interleaved
		// into Morton bit positions.
		const int cells = 1 << g.m;
		for (const StencilEntry& e : g.stencil) {
			auto d = [cells](int v) { return split_by3(static_cast<uint32_t>((v % cells + cells) % cells)); };
			stencil.push_back(make_uint4(d(e.dx) << 2, d(e.dy) << 1, d(e.dz), 0u));
		}
		base += 1u << (3 * g.m);
		b->grids_h[s] = sg;
	}
	b->stencil.ensure(std::max<size_t>(stencil.size(), 1));
	if (!stencil.empty())
		MB2_CUDA(cudaMemcpy(b->stencil.ptr, stencil.data(), stencil.size() * sizeof(uint4),
							cudaMemcpyHostToDevice));
	b->total_cells = base;
	b->grids.ensure(b->num_systems);
	MB2_CUDA(cudaMemcpy(b->grids.ptr, b->grids_h.data(), b->num_systems * sizeof(SysGrid),
						cudaMemcpyHostToDevice));
	b->grid_rc = rc;
}

// The list build. flags_h (pinned, one word per system; null: every system)
// names the systems to rebuild: the others keep their sort keys, sorted slots,
// rows and displacement snapshot from their own last build, as each system's
// list would if it ran alone (a patch of the reference rebuilds on its own
// skin check). A change of grid, or a row longer than the list's row
// capacity, rebuilds every system.
void batch_build(mb2_batch* b, const float4* pos, const int* type_ids, float rc, cudaStream_t st,
				 const unsigned int* flags_h = nullptr) {
	expect_arg(rc > 0.0f && std::isfinite(rc), MB2_ERR_ARG,
			   "mb2_batch_build: pairlist cutoff must be positive and finite");
	for (uint32_t s = 0; s < b->num_systems; ++s)
		for (int a = 0; a < 3; ++a)
			expect_arg(2.0f * rc < b->boxes_h[s].size[a], MB2_ERR_ARG,
					   "mb2_batch_build: every box edge must exceed twice the list radius");
	const uint32_t n = b->n;
	if (b->grid_rc != rc) {
		choose_grids(b, rc);
		flags_h = nullptr;
	}
	if (!(b->built && b->cap && b->lanes)) flags_h = nullptr;
	const uint32_t* dflags = nullptr;
	uint64_t rebuilt = b->num_systems;
	b->keys.ensure(n);
	b->s2o.ensure(n);
	b->inv.ensure(n);
	b->sorted_pos.ensure(n);
	if (flags_h) {
		// Only the rebuilt systems' particles are sorted: the others keep their
		// sorted slots (keys and order of their own last build).
		const uint32_t S = b->num_systems;
		uint32_t m = 0;
		rebuilt = 0;
		for (uint32_t s = 0; s < S; ++s) {
			b->pinned_cstart[s] = m;
			if (flags_h[s]) {
				m += b->offsets[s + 1] - b->offsets[s];
				++rebuilt;
			}
		}
		b->sys_flags.ensure(S);
		b->cstart.ensure(S);
		MB2_CUDA(cudaMemcpyAsync(b->sys_flags.ptr, flags_h, S * sizeof(unsigned int),
								 cudaMemcpyHostToDevice, st));
		MB2_CUDA(cudaMemcpyAsync(b->cstart.ptr, b->pinned_cstart, S * sizeof(unsigned int),
								 cudaMemcpyHostToDevice, st));
		dflags = b->sys_flags.ptr;
		b->ckeys.ensure(std::max<uint32_t>(m, 1));
		b->cidx.ensure(std::max<uint32_t>(m, 1));
		MB2_LAUNCH batch_compact_kernel<<<(n + 255) / 256, 256, 0, st>>>(
			pos, b->sys_of.ptr, b->boxes.ptr, b->offsets_d.ptr, dflags, b->cstart.ptr, n,
			b->ckeys.ptr, b->cidx.ptr);
		if (m) radix_sort_pairs(b->scratch, b->ckeys.ptr, b->cidx.ptr, m, st);
		if (m)
			MB2_LAUNCH batch_scatter_sorted_kernel<<<(m + 255) / 256, 256, 0, st>>>(
				b->ckeys.ptr, b->cidx.ptr, m, b->offsets_d.ptr, b->cstart.ptr, b->keys.ptr,
				b->s2o.ptr);
	} else {
		if (n)
			MB2_LAUNCH batch_encode_kernel<<<(n + 255) / 256, 256, 0, st>>>(
				pos, b->sys_of.ptr, b->boxes.ptr, n, b->keys.ptr, b->s2o.ptr);
		radix_sort_pairs(b->scratch, b->keys.ptr, b->s2o.ptr, n, st);
	}
	inverse_and_gather(b->s2o.ptr, n, pos, b->inv.ptr, nullptr, st);
	pack_sorted_positions(pos, type_ids, b->s2o.ptr, n, b->sorted_pos.ptr, st);
	b->cell_begin.ensure(b->total_cells);
	b->cell_end.ensure(b->total_cells);
	MB2_CUDA(cudaMemsetAsync(b->cell_begin.ptr, 0, b->total_cells * sizeof(uint32_t), st));
	MB2_CUDA(cudaMemsetAsync(b->cell_end.ptr, 0, b->total_cells * sizeof(uint32_t), st));
	if (n)
		MB2_LAUNCH batch_cell_ranges_kernel<<<(n + 255) / 256, 256, 0, st>>>(
			b->keys.ptr, n, b->grids.ptr, b->cell_begin.ptr, b->cell_end.ptr);
	b->row_len.ensure(n);
	b->stats.ensure(2);
	auto walk = [&](uint32_t cap, const uint32_t* fl) {
		MB2_CUDA(cudaMemsetAsync(b->stats.ptr, 0, 2 * sizeof(unsigned long long), st));
		if (n) {
			const int hshift = __builtin_ctz(32 / b->lanes);
			MB2_LAUNCH batch_group_kernel<<<(n + 255) / 256, 256, 0, st>>>(
				b->sorted_pos.ptr, b->keys.ptr, b->s2o.ptr, b->cell_begin.ptr, b->cell_end.ptr,
				b->grids.ptr, b->boxes.ptr, b->stencil.ptr, fl, n, b->nbr.ptr, cap, hshift,
				b->row_len.ptr);
			MB2_LAUNCH batch_row_stats_kernel<<<std::min<uint32_t>((n + 255) / 256, 1184), 256, 0,
												 st>>>(b->row_len.ptr, n, b->stats.ptr);
		}
		MB2_CUDA(cudaMemcpyAsync(b->pinned, b->stats.ptr, 2 * sizeof(unsigned long long),
								 cudaMemcpyDeviceToHost, st));
		MB2_CUDA(cudaStreamSynchronize(st));
		return std::make_pair(b->pinned[0], b->pinned[1]);
	};
	auto size_list = [&](uint64_t max_row) {
		const uint32_t G = static_cast<uint32_t>(b->lanes);
		uint64_t cap = max_row + max_row / 4 + G;
		cap = (cap + G - 1) / G * G;
		expect_arg(cap < 65536u, MB2_ERR_CAPACITY,
				   "mb2_batch_build: a particle has more than ~52000 list neighbours");
		b->cap = static_cast<uint32_t>(cap);
	};
	auto ensure_list = [&]() {
		const size_t hgt = static_cast<size_t>(32 / b->lanes);
		b->nbr.ensure(std::max<size_t>((n + hgt - 1) / hgt * b->cap * hgt, 1));
	};
	if (b->cap == 0 || b->lanes == 0) {
		// First build: count rows without storing (cap 0 writes nothing), to size the list.
		b->lanes = 4;
		const auto counted = walk(0u, nullptr);
		const double mean = n ? static_cast<double>(counted.first) / n : 0.0;
		b->lanes = b->lanes_request ? b->lanes_request
									: (mean >= 256.0 ? 16 : (mean >= 48.0 ? 8 : 4));
		size_list(counted.second);
	}
	ensure_list();
	auto stats = walk(b->cap, dflags);
	if (stats.second > b->cap) {
		// A longer row than the capacity: a new row stride, so every system's
		// rows are walked again.
		size_list(stats.second);
		ensure_list();
		if (dflags) {
			batch_build(b, pos, type_ids, rc, st, nullptr);
			return;
		}
		stats = walk(b->cap, nullptr);
	}
	b->ref_pos.ensure(n);
	if (n)
		MB2_LAUNCH batch_snapshot_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, b->sys_of.ptr, dflags,
																		  n, b->ref_pos.ptr);
	b->num_pairs = stats.first;
	b->built = true;
	b->system_rebuilds += rebuilt;
}

// Each system's largest displacement since its own last build, squared, into
// b->pinned_sys (float bits); synchronises. Returns the largest displacement.
float batch_sys_disp(mb2_batch* b, const float4* pos, cudaStream_t st) {
	const uint32_t S = b->num_systems;
	b->disp.ensure(S);
	MB2_CUDA(cudaMemsetAsync(b->disp.ptr, 0, S * sizeof(unsigned int), st));
	if (b->n)
		MB2_LAUNCH batch_displacement_kernel<<<(b->n + 255) / 256, 256, 0, st>>>(
			pos, b->ref_pos.ptr, b->sys_of.ptr, b->boxes.ptr, b->n, b->disp.ptr);
	MB2_CUDA(cudaMemcpyAsync(b->pinned_sys, b->disp.ptr, S * sizeof(unsigned int),
							 cudaMemcpyDeviceToHost, st));
	MB2_CUDA(cudaStreamSynchronize(st));
	float worst = 0.0f;
	for (uint32_t s = 0; s < S; ++s) {
		float d2;
		std::memcpy(&d2, &b->pinned_sys[s], 4);
		worst = std::max(worst, d2);
	}
	return std::sqrt(worst);
}

// Largest displacement (over all systems) since the last build; synchronises.
float batch_max_disp(mb2_batch* b, const float4* pos, cudaStream_t st) {
	return batch_sys_disp(b, pos, st);
}

// The per-step work after any rebuild: pack, clear, pair forces, integrate,
// advance the device step counter.
void step_body(mb2_batch* b, float4* pos, float4* fe, const int* type_ids,
			   const mb2_step_params* prm, cudaStream_t st) {
	const uint32_t n = b->n;
	if (n == 0) return;
	pack_sorted_positions(pos, type_ids, b->s2o.ptr, n, b->sorted_pos.ptr, st);
	MB2_CUDA(cudaMemsetAsync(b->force_sorted.ptr, 0, static_cast<size_t>(n) * sizeof(float4), st));
	const float cutoff_sq = prm->cutoff > 0.0f ? prm->cutoff * prm->cutoff : 0.0f;
	pair_forces_systems(b->sorted_pos.ptr, b->nbr.ptr, b->row_len.ptr, n, b->cap, b->lanes, b->pt,
						b->boxes.ptr, b->keys.ptr, kSysShift, true, cutoff_sq, 0,
						b->force_sorted.ptr, b->energy.ptr, st);
	bd_integrate_systems(pos, fe, b->force_sorted.ptr, b->inv.ptr, type_ids, b->sys_of.ptr,
						 b->offsets_d.ptr, b->boxes.ptr, n, b->types, prm->dt, prm->kT, prm->seed,
						 prm->patch_id, b->step_d.ptr, st);
	step_counter_add(b->step_d.ptr, 1, st);
}

void check_step_args(mb2_batch* b, const float* pos4, const float* fe4, const int* type_ids,
					 const mb2_step_params* prm) {
	expect_arg(prm && (b->n == 0 || (pos4 && fe4 && type_ids)), MB2_ERR_ARG,
			   "mb2_batch_step: null argument");
	expect_arg(b->types_set, MB2_ERR_STATE, "mb2_batch_step: call mb2_batch_set_particle_types");
	expect_arg(b->pt.num_types > 0, MB2_ERR_STATE,
			   "mb2_batch_step: call mb2_batch_set_pair_tables");
	expect_arg(prm->num_bonds == 0 && prm->num_angles == 0 && prm->num_dihedrals == 0 &&
				   prm->num_restraints == 0 && prm->integrator == 0,
			   MB2_ERR_ARG, "mb2_batch_step: BD without bonded terms in batched mode");
}

// The rebuild schedule of Patch.cpp:86-108 for each system, as each would
// run alone: a rebuild at the first step and at every period step, skipped
// for a system none of whose particles moved more than half the skin since
// its own last build. The period is the cadence in force: the batch's own
// (the autotuner's choice) when set, else the params'. The systems due are
// rebuilt together in one build.
void maybe_rebuild(mb2_batch* b, const float4* pos, const int* type_ids, uint64_t step,
				   const mb2_step_params* prm, cudaStream_t st) {
	const uint32_t period = b->rebuild_period ? b->rebuild_period : prm->rebuild_period;
	const bool at_period = period == 0 || (step - 1) % period == 0;
	const float skin = prm->pairlist_cutoff - prm->cutoff;
	if (!b->built || (at_period && (period == 0 || skin <= 0.0f))) {
		batch_build(b, pos, type_ids, prm->pairlist_cutoff, st);
		++b->rebuilds;
	} else if (at_period) {
		batch_sys_disp(b, pos, st);
		uint32_t due = 0;
		for (uint32_t s = 0; s < b->num_systems; ++s) {
			float d2;
			std::memcpy(&d2, &b->pinned_sys[s], 4);
			const bool r = std::sqrt(d2) > skin * 0.5f;
			b->pinned_sys[s] = r ? 1u : 0u;
			due += r ? 1u : 0u;
		}
		if (due) {
			batch_build(b, pos, type_ids, prm->pairlist_cutoff, st,
						due == b->num_systems ? nullptr : b->pinned_sys);
			++b->rebuilds;
		}
	}
	b->force_sorted.ensure(b->n);
}

void reset_tuning(mb2_batch* b, int level_offset, int lanes) {
	if (level_offset != b->level_offset) b->grid_rc = -1.0f;
	b->level_offset = level_offset;
	b->lanes_request = lanes;
	b->cap = 0;
	b->lanes = 0;
	b->built = false;
}

}  // namespace

extern "C" {

int mb2_batch_create(int device, uint32_t num_systems, const uint32_t* counts,
					 const float* box_origin3, const float* box_size3, mb2_batch** out) {
	if (!out || !counts || !box_size3 || num_systems == 0) return MB2_ERR_ARG;
	*out = nullptr;
	if (num_systems > (1u << (32 - kSysShift))) return MB2_ERR_CAPACITY;
	mb2_batch* b = new mb2_batch();
	b->device = device;
	const int rc = bguard(b, [&] {
		b->num_systems = num_systems;
		b->offsets.assign(num_systems + 1, 0);
		uint64_t total = 0;
		for (uint32_t s = 0; s < num_systems; ++s) {
			total += counts[s];
			expect_arg(total < (1ull << 31), MB2_ERR_CAPACITY,
					   "mb2_batch_create: too many particles");
			b->offsets[s + 1] = static_cast<uint32_t>(total);
		}
		b->n = static_cast<uint32_t>(total);
		b->boxes_h.resize(num_systems);
		std::vector<uint32_t> sys_of(b->n);
		for (uint32_t s = 0; s < num_systems; ++s) {
			Box& bx = b->boxes_h[s];
			for (int a = 0; a < 3; ++a) {
				const float l = box_size3[3 * s + a];
				expect_arg(l > 0.0f && std::isfinite(l), MB2_ERR_ARG,
						   "mb2_batch_create: box edges must be positive");
				bx.origin[a] = box_origin3 ? box_origin3[3 * s + a] : 0.0f;
				bx.size[a] = l;
				bx.inv[a] = 1.0f / l;
				bx.half[a] = 0.5f * l;
				bx.periodic[a] = 1;
			}
			for (uint32_t i = b->offsets[s]; i < b->offsets[s + 1]; ++i) sys_of[i] = s;
		}
		b->offsets_d.ensure(num_systems + 1);
		b->boxes.ensure(num_systems);
		b->sys_of.ensure(std::max<uint32_t>(b->n, 1));
		MB2_CUDA(cudaMemcpy(b->offsets_d.ptr, b->offsets.data(), (num_systems + 1) * 4ull,
							cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->boxes.ptr, b->boxes_h.data(), num_systems * sizeof(Box),
							cudaMemcpyHostToDevice));
		if (b->n)
			MB2_CUDA(cudaMemcpy(b->sys_of.ptr, sys_of.data(), b->n * 4ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMallocHost(&b->pinned, 64));
		MB2_CUDA(cudaMallocHost(&b->pinned_sys, num_systems * sizeof(unsigned int)));
		MB2_CUDA(cudaMallocHost(&b->pinned_cstart, num_systems * sizeof(unsigned int)));
		b->step_d.ensure(1);
		b->energy.ensure(4);
		MB2_CUDA(cudaMemset(b->energy.ptr, 0, 4 * sizeof(double)));
	});
	if (rc != MB2_OK) {
		delete b;
		return rc;
	}
	*out = b;
	return MB2_OK;
}

int mb2_batch_destroy(mb2_batch* b) {
	if (!b) return MB2_ERR_ARG;
	cudaSetDevice(b->device);
	cudaDeviceSynchronize();
	delete b;
	return MB2_OK;
}

const char* mb2_batch_last_error(const mb2_batch* b) {
	return b ? b->last_error.c_str() : "null batch";
}

int mb2_batch_set_pair_tables(mb2_batch* b, int num_types, const uint32_t* term_matrix,
							  int num_tables, const float* values, const uint32_t* sizes,
							  const float* starts, const float* step_invs) {
	return bguard(b, [&] {
		std::vector<PairTableRef> refs;
		std::vector<float> bf;
		std::vector<float2> be;
		const size_t total = pair_table_arrays(num_types, term_matrix, num_tables, values, sizes,
											   starts, step_invs, refs, bf, be);
		const int tt = num_types * num_types;
		for (int k = 0; k < tt; ++k)
			expect_arg(!(term_matrix[k] & kTermAnalytical), MB2_ERR_ARG,
					   "mb2_batch_set_pair_tables: batched mode takes tabulated pair terms only");
		expect_arg(tt * sizeof(PairTableRef) + total * 12 + 8 <= 200 * 1024, MB2_ERR_CAPACITY,
				   "mb2_batch_set_pair_tables: tables exceed the 200 KB shared-memory budget");
		b->refs.ensure(tt);
		b->bin_force.ensure(bf.size());
		b->bin_energy.ensure(be.size());
		MB2_CUDA(cudaMemcpy(b->refs.ptr, refs.data(), tt * sizeof(PairTableRef),
							cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->bin_force.ptr, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->bin_energy.ptr, be.data(), be.size() * 8, cudaMemcpyHostToDevice));
		std::vector<int> offs;
		PairTableRef u;
		const bool uniform = uniform_tables(refs, offs, u);
		b->table_offsets.ensure(tt);
		MB2_CUDA(cudaMemcpy(b->table_offsets.ptr, offs.data(), tt * sizeof(int),
							cudaMemcpyHostToDevice));
		b->pt.num_types = num_types;
		b->pt.total_bins = static_cast<uint32_t>(total);
		b->pt.refs = b->refs.ptr;
		b->pt.offsets = b->table_offsets.ptr;
		b->pt.uniform = uniform;
		b->pt.uniform_ref = u;
		b->pt.bin_force = b->bin_force.ptr;
		b->pt.bin_energy = b->bin_energy.ptr;
	});
}

int mb2_batch_set_particle_types(mb2_batch* b, int num_types, const float* charge,
								 const float* diffusion3) {
	return bguard(b, [&] {
		expect_arg(num_types > 0 && charge && diffusion3, MB2_ERR_ARG,
				   "mb2_batch_set_particle_types: bad arguments");
		std::vector<float4> dif(num_types);
		std::vector<int> zero(num_types, 0);
		std::vector<int4> fg(num_types, make_int4(-1, -1, -1, -1));
		std::vector<float4> fs(num_types, make_float4(0.f, 0.f, 0.f, 0.f));
		for (int t = 0; t < num_types; ++t)
			dif[t] = make_float4(diffusion3[3 * t], diffusion3[3 * t + 1], diffusion3[3 * t + 2],
								 0.0f);
		b->charge.ensure(num_types);
		b->diffusion.ensure(num_types);
		b->pmf_off.ensure(num_types);
		b->pmf_cnt.ensure(num_types);
		b->fg_id.ensure(num_types);
		b->fg_scale.ensure(num_types);
		MB2_CUDA(cudaMemcpy(b->charge.ptr, charge, num_types * 4ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->diffusion.ptr, dif.data(), num_types * 16ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->pmf_off.ptr, zero.data(), num_types * 4ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->pmf_cnt.ptr, zero.data(), num_types * 4ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->fg_id.ptr, fg.data(), num_types * 16ull, cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(b->fg_scale.ptr, fs.data(), num_types * 16ull, cudaMemcpyHostToDevice));
		TypeTable& ty = b->types;
		ty.num_types = num_types;
		ty.charge = b->charge.ptr;
		ty.diffusion = b->diffusion.ptr;
		ty.pmf_offset = b->pmf_off.ptr;
		ty.pmf_count = b->pmf_cnt.ptr;
		ty.terms = nullptr;
		ty.force_grid_id = b->fg_id.ptr;
		ty.force_grid_scale = b->fg_scale.ptr;
		ty.grids = nullptr;
		ty.num_grids = 0;
		b->types_set = true;
	});
}

int mb2_batch_build(mb2_batch* b, const float* pos4, const int* type_ids, float pairlist_cutoff,
					void* stream, uint64_t* num_pairs) {
	return bguard(b, [&] {
		expect_arg(b->n == 0 || (pos4 && type_ids), MB2_ERR_ARG, "mb2_batch_build: null argument");
		batch_build(b, reinterpret_cast<const float4*>(pos4), type_ids, pairlist_cutoff,
					S(stream));
		if (num_pairs) *num_pairs = b->num_pairs;
	});
}

int mb2_batch_num_pairs(const mb2_batch* b, uint64_t* num_pairs) {
	if (!b || !num_pairs) return MB2_ERR_ARG;
	*num_pairs = b->built ? b->num_pairs : 0;
	return MB2_OK;
}

int mb2_batch_export_pairs(mb2_batch* b, int* pairs2, uint64_t capacity, void* stream) {
	return bguard(b, [&] {
		expect_arg(b->built, MB2_ERR_STATE, "mb2_batch_export_pairs: no pairlist");
		expect_arg(capacity >= b->num_pairs, MB2_ERR_CAPACITY,
				   "mb2_batch_export_pairs: output smaller than the pair count");
		expect_arg(b->num_pairs == 0 || pairs2, MB2_ERR_ARG, "mb2_batch_export_pairs: null output");
		b->row_off.ensure(b->n);
		exclusive_scan_u32(b->scratch, b->row_len.ptr, b->row_off.ptr, b->n, nullptr, S(stream));
		export_pairs(b->nbr.ptr, b->row_len.ptr, b->row_off.ptr, b->s2o.ptr, b->n, b->cap,
					 __builtin_ctz(32 / b->lanes), reinterpret_cast<int2*>(pairs2), S(stream));
	});
}

int mb2_batch_step(mb2_batch* b, float* pos4, float* force_energy4, const int* type_ids,
				   uint64_t step, const mb2_step_params* prm, void* stream) {
	return bguard(b, [&] {
		check_step_args(b, pos4, force_energy4, type_ids, prm);
		const cudaStream_t st = S(stream);
		float4* pos = reinterpret_cast<float4*>(pos4);
		maybe_rebuild(b, pos, type_ids, step, prm, st);
		step_counter_set(b->step_d.ptr, step, st);
		step_body(b, pos, reinterpret_cast<float4*>(force_energy4), type_ids, prm, st);
	});
}

int mb2_batch_run(mb2_batch* b, float* pos4, float* force_energy4, const int* type_ids,
				  uint64_t first_step, uint32_t num_steps, const mb2_step_params* prm,
				  void* stream) {
	return bguard(b, [&] {
		check_step_args(b, pos4, force_energy4, type_ids, prm);
		const cudaStream_t st = S(stream);
		float4* pos = reinterpret_cast<float4*>(pos4);
		float4* fe = reinterpret_cast<float4*>(force_energy4);
		for (uint32_t k = 0; k < num_steps; ++k) {
			const uint64_t step = first_step + k;
			maybe_rebuild(b, pos, type_ids, step, prm, st);
			// The graph bakes in every pointer and size of the step body.
			const std::vector<uint64_t> key = {
				reinterpret_cast<uint64_t>(pos), reinterpret_cast<uint64_t>(fe),
				reinterpret_cast<uint64_t>(type_ids), reinterpret_cast<uint64_t>(b->nbr.ptr),
				reinterpret_cast<uint64_t>(b->force_sorted.ptr), b->cap,
				static_cast<uint64_t>(b->lanes), b->n, f2u(prm->cutoff), f2u(prm->dt),
				f2u(prm->kT), prm->seed, prm->patch_id,
				// tables and types (pointers, sizes, the uniform-table constants)
				reinterpret_cast<uint64_t>(b->pt.refs), reinterpret_cast<uint64_t>(b->pt.offsets),
				reinterpret_cast<uint64_t>(b->pt.bin_force),
				reinterpret_cast<uint64_t>(b->pt.bin_energy), b->pt.total_bins,
				static_cast<uint64_t>(b->pt.num_types), static_cast<uint64_t>(b->pt.uniform),
				f2u(b->pt.uniform_ref.start), f2u(b->pt.uniform_ref.step_inv),
				static_cast<uint64_t>(b->pt.uniform_ref.last),
				reinterpret_cast<uint64_t>(b->types.charge),
				reinterpret_cast<uint64_t>(b->types.diffusion),
				static_cast<uint64_t>(b->types.num_types)};
			if (!b->graph || key != b->graph_key) {
				if (b->graph) {
					MB2_CUDA(cudaGraphExecDestroy(b->graph));
					b->graph = nullptr;
				}
				cudaStream_t cs;
				MB2_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
				cudaGraph_t g = nullptr;
				const unsigned long long l0 = g_launches;
				MB2_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
				step_body(b, pos, fe, type_ids, prm, cs);
				const cudaError_t ec = cudaStreamEndCapture(cs, &g);
				b->launches_per_graph = g_launches - l0;
				g_launches = l0;  // counted at each replay instead
				cudaStreamDestroy(cs);
				MB2_CUDA(ec);
				const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
				cudaGraphDestroy(g);
				MB2_CUDA(ei);
				b->graph_key = key;
			}
			// Each replay advances the device step counter by one.
			if (k == 0) step_counter_set(b->step_d.ptr, step, st);
			MB2_CUDA(cudaGraphLaunch(b->graph, st));
			g_launches += b->launches_per_graph;
		}
	});
}

int mb2_batch_set_rebuild_period(mb2_batch* b, uint32_t period) {
	return bguard(b, [&] { b->rebuild_period = period; });
}

int mb2_batch_system_rebuilds(const mb2_batch* b, uint64_t* count) {
	if (!b || !count) return MB2_ERR_ARG;
	*count = b->system_rebuilds;
	return MB2_OK;
}

int mb2_batch_rebuild_schedule(const mb2_batch* b, uint32_t* period, uint64_t* rebuilds) {
	if (!b) return MB2_ERR_ARG;
	if (period) *period = b->rebuild_period;
	if (rebuilds) *rebuilds = b->rebuilds;
	return MB2_OK;
}

int mb2_batch_set_tuning(mb2_batch* b, int level_offset, int lanes) {
	return bguard(b, [&] {
		expect_arg(level_offset >= -3 && level_offset <= 3, MB2_ERR_ARG,
				   "mb2_batch_set_tuning: level offset in [-3, 3]");
		expect_arg(lanes == 0 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32,
				   MB2_ERR_ARG, "mb2_batch_set_tuning: lanes 0, 4, 8, 16 or 32");
		reset_tuning(b, level_offset, lanes);
	});
}

int mb2_batch_tuning(const mb2_batch* b, int* level_offset, int* lanes, uint32_t* total_cells) {
	if (!b) return MB2_ERR_ARG;
	if (level_offset) *level_offset = b->level_offset;
	if (lanes) *lanes = b->lanes;
	if (total_cells) *total_cells = b->total_cells;
	return MB2_OK;
}

int mb2_batch_autotune(mb2_batch* b, const float* pos4, const int* type_ids,
					   const mb2_step_params* prm, uint32_t trial_steps, void* stream,
					   mb2_batch_tuning_result* out) {
	return bguard(b, [&] {
		check_step_args(b, pos4, pos4, type_ids, prm);
		expect_arg(out != nullptr && trial_steps > 0, MB2_ERR_ARG,
				   "mb2_batch_autotune: bad arguments");
		const cudaStream_t st = S(stream);
		const uint32_t n = b->n;
		DevBuf<float4> tpos, tfe;
		tpos.ensure(std::max<uint32_t>(n, 1));
		tfe.ensure(std::max<uint32_t>(n, 1));
		cudaEvent_t e0, e1, e2;
		MB2_CUDA(cudaEventCreate(&e0));
		MB2_CUDA(cudaEventCreate(&e1));
		MB2_CUDA(cudaEventCreate(&e2));
		const uint32_t period = prm->rebuild_period ? prm->rebuild_period : 1u;
		int best_level = 0, best_lanes = 0;
		float best_cost = -1.0f, best_build = 0.0f, best_step = 0.0f;
		const int levels[3] = {-1, 0, 1};
		const int lanes_c[3] = {4, 8, 16};
		for (int li = 0; li < 3; ++li)
			for (int gi = 0; gi < 3; ++gi) {
				reset_tuning(b, levels[li], lanes_c[gi]);
				MB2_CUDA(cudaMemcpyAsync(tpos.ptr, pos4, static_cast<size_t>(n) * 16,
										 cudaMemcpyDeviceToDevice, st));
				batch_build(b, tpos.ptr, type_ids, prm->pairlist_cutoff, st);  // sizes the list
				MB2_CUDA(cudaEventRecord(e0, st));
				batch_build(b, tpos.ptr, type_ids, prm->pairlist_cutoff, st);
				MB2_CUDA(cudaEventRecord(e1, st));
				b->force_sorted.ensure(n);
				step_counter_set(b->step_d.ptr, 1, st);
				for (uint32_t k = 0; k < trial_steps; ++k)
					step_body(b, tpos.ptr, tfe.ptr, type_ids, prm, st);
				MB2_CUDA(cudaEventRecord(e2, st));
				MB2_CUDA(cudaEventSynchronize(e2));
				float tb = 0.0f, ts = 0.0f;
				MB2_CUDA(cudaEventElapsedTime(&tb, e0, e1));
				MB2_CUDA(cudaEventElapsedTime(&ts, e1, e2));
				ts /= static_cast<float>(trial_steps);
				const float cost = tb / static_cast<float>(period) + ts;
				if (best_cost < 0.0f || cost < best_cost) {
					best_cost = cost;
					best_level = levels[li];
					best_lanes = lanes_c[gi];
					best_build = tb;
					best_step = ts;
				}
			}
		// Apply the best knobs. Then the cadence: on the copy, an equilibration
		// segment of one period (rebuilt at its start), so that the overlaps of
		// a fresh start have relaxed; then two intervals of one period, each
		// from a fresh list, recording the largest displacement after every
		// step. The cadence is the largest k <= period whose displacement stayed
		// within half the skin in both: rebuilt every k steps, the list keeps
		// every pair that comes within the cutoff.
		reset_tuning(b, best_level, best_lanes);
		MB2_CUDA(cudaMemcpyAsync(tpos.ptr, pos4, static_cast<size_t>(n) * 16,
								 cudaMemcpyDeviceToDevice, st));
		b->force_sorted.ensure(n);
		step_counter_set(b->step_d.ptr, 1, st);
		batch_build(b, tpos.ptr, type_ids, prm->pairlist_cutoff, st);
		for (uint32_t k = 0; k < period; ++k) step_body(b, tpos.ptr, tfe.ptr, type_ids, prm, st);
		const float skin = prm->pairlist_cutoff - prm->cutoff;
		uint32_t cadence = period;
		float disp_at_period = 0.0f;
		for (int rep = 0; rep < 2; ++rep) {
			batch_build(b, tpos.ptr, type_ids, prm->pairlist_cutoff, st);
			bool exceeded = false;
			for (uint32_t k = 1; k <= period; ++k) {
				step_body(b, tpos.ptr, tfe.ptr, type_ids, prm, st);
				const float d = batch_max_disp(b, tpos.ptr, st);
				if (d > 0.5f * skin && !exceeded) {
					exceeded = true;
					cadence = std::min(cadence, std::max<uint32_t>(k - 1, 1u));
				}
				if (k == period) disp_at_period = std::max(disp_at_period, d);
			}
		}
		if (skin <= 0.0f) cadence = 1;
		b->rebuild_period = cadence;  // in force from the next step
		b->built = false;  // that list was built from the trial positions
		MB2_CUDA(cudaStreamSynchronize(st));
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		cudaEventDestroy(e2);
		out->level_offset = best_level;
		out->lanes = best_lanes;
		out->build_ms = best_build;
		out->step_ms = best_step;
		out->safe_rebuild_period = cadence;
		out->max_displacement_at_period = disp_at_period;
		out->total_cells = b->total_cells;
	});
}

}  // extern "C"
