// Pairlist build over Morton-sorted particles.
//
// Replaces BuildCellRangesKernel / BuildCellNeighborsKernel /
// ZOrderCellNeighborKernel (src/PatchOperation/PairListKernels/ZOrderNeighbor.h)
// and the grow-and-retry loop of ZOrderPairlist::find_neighbors_zorder
// (src/PatchOperation/PairListKernels/ZOrderPairlist.cpp:208-366).
//
// The pair SET is the reference's: for sorted i < sorted j, keep (i, j) when
// wrap_diff(pos_j - pos_i).length2() <= rc^2 (float, exactly as the reference
// rounds it) and the pair is not excluded. Only the search differs.
//
// Search. Cells are the top 3m bits of the 30-bit Morton key; a cell's
// particles are a contiguous run of the sorted array. The stencil is every
// cell whose box-to-box distance from the home cell can be within rc (a
// pruned sphere, not the reference's (2r+1)^3 cube), at the cell level chosen
// per run to minimise candidates plus per-cell cost. One warp owns one
// group of 32 consecutive sorted particles and walks, in lockstep, the cells
// within rc of the group's cell bounding box, testing one candidate per
// step against all of them. The test is a cheap minimum-image distance; only candidates
// inside a rounding band around rc (sized from the float ulp of the box)
// take the exact reference computation.
//
// Storage. A half list in sliced ELL form: rows of H consecutive particles
// form a slice; entry k of row i sits at ((i / H) * cap + k) * H + i % H, so
// that G = 32 / H lanes per row reading k..k+G-1 of H rows touch one 128-byte
// line. row_len[i] holds the row's length. Bit 31 of an entry records the
// reference's pair orientation: set when the original index of j is smaller
// than that of i (the reference computes that pair as j -> i).
#include "mb2_internal.cuh"
#include "mb2_walk.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace mb2 {

namespace {

double ulp_of(double x) {
	x = std::fabs(x);
	if (x < 1e-30) return 1e-45;
	return std::ldexp(1.0, static_cast<int>(std::floor(std::log2(x))) - 23);
}

}  // namespace

CellGrid choose_cell_grid(const float* extent, const int* periodic, float rc_list, size_t n,
						  int m_lo, int m_hi) {
	CellGrid best;
	double best_cost = -1.0;
	const double rc = static_cast<double>(rc_list);
	for (int m = m_lo; m <= m_hi; ++m) {
		const int cells = 1 << m;
		const double num_cells = std::ldexp(1.0, 3 * m);
		if (m > m_lo && num_cells > 2.0 * static_cast<double>(n)) break;
		std::vector<int> off[3];
		std::vector<double> gap[3];
		int radius[3] = {0, 0, 0};
		double wmin[3] = {0, 0, 0};
		for (int a = 0; a < 3; ++a) {
			if (m == 0) {
				off[a] = {0};
				gap[a] = {0.0};
				wmin[a] = extent[a];
				continue;
			}
			// Real-space cell widths: cell c spans Morton coordinates
			// [c 2^k, (c+1) 2^k) of the 0..1023 scale over the domain, so it is
			// extent * 2^k / 1023 wide, except the last, extent * (2^k - 1) / 1023.
			const int k = 10 - m;
			wmin[a] = static_cast<double>(extent[a]) * (std::ldexp(1.0, k) - 1.0) / 1023.0 *
					  (1.0 - 1e-6);
			const int r = static_cast<int>(std::floor(rc / wmin[a])) + 1;
			radius[a] = r;
			if (periodic[a] && 2 * r + 1 >= cells) {
				for (int d = 0; d < cells; ++d) {
					off[a].push_back(d);
					gap[a].push_back(0.0);
				}
			} else {
				for (int d = -r; d <= r; ++d) {
					off[a].push_back(d);
					gap[a].push_back(std::max(0, std::abs(d) - 1) * wmin[a]);
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
					if (g2 <= lim) {
						// pad: the offsets modulo 2^m interleaved into Morton bit
						// positions (x at 3k + 2, y at 3k + 1, z at 3k).
						const auto wrap = [cells](int v) {
							return static_cast<uint32_t>(((v % cells) + cells) % cells);
						};
						const uint32_t d = (split_by3(wrap(off[0][x])) << 2) |
										   (split_by3(wrap(off[1][y])) << 1) |
										   split_by3(wrap(off[2][z]));
						st.push_back(StencilEntry{off[0][x], off[1][y], off[2][z],
												  static_cast<int>(d)});
					}
				}
		const double per_cell = static_cast<double>(n) / num_cells;
		const double cost = static_cast<double>(st.size()) * (per_cell + 2.0);
		if (best_cost < 0.0 || cost < best_cost) {
			best_cost = cost;
			best.m = m;
			best.shift = 3 * (10 - m);
			best.num_stencil = static_cast<int>(st.size());
			best.stencil = st;
			for (int a = 0; a < 3; ++a) {
				best.radius[a] = radius[a];
				best.wmin[a] = static_cast<float>(wmin[a]);
			}
			best.lim = static_cast<float>(lim);
		}
	}
	return best;
}

void fast_test_band(const Box& box, float rc_list, float* fast_lo, float* fast_hi) {
	// Each minimum-image component differs from the reference's wrap_diff by at
	// most a few ulp of the largest coordinate magnitude; bound |d^2 - d_ref^2|.
	double mag = 0.0;
	for (int a = 0; a < 3; ++a)
		mag = std::max({mag, std::fabs(static_cast<double>(box.origin[a])),
						std::fabs(static_cast<double>(box.origin[a]) + box.size[a]),
						static_cast<double>(box.size[a])});
	const double rc = rc_list;
	const double per_axis = 4.0 * ulp_of(2.0 * mag);
	const double delta = 2.0 * rc * 3.0 * per_axis * 2.0 + rc * rc * 1e-6;
	*fast_lo = static_cast<float>(rc * rc - delta);
	*fast_hi = static_cast<float>(rc * rc + delta);
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


// One warp owns a group of 32 consecutive sorted particles, lane = particle.
// The group's cells are Morton-adjacent; the warp walks, in lockstep, every
// cell whose real extent lies within rc of the group's coordinate range (found
// by the lanes in parallel over the group's cell box widened by the stencil
// radius), loading each candidate once for all 32 lanes (a broadcast). Cells before the group's first cell in
// Morton order hold only earlier particles and are skipped without loading
// their ranges. A group whose cells straddle a Morton discontinuity (wide
// bounding box) walks each particle's own pruned stencil instead. Each row
// keeps candidate order (runs of consecutive sorted j), which keeps the force
// kernel's gathers local.
// Seven resident blocks per SM (32 registers, a little spill): the walk is
// bound by instruction issue and the latency of its dependent loads (cell
// ranges, then candidates), and more warps hide the latency. Measured on the
// 2,097,152-bead workload when the budget was set: 7.1 ms per build at 7
// blocks, 7.7 at 6 (40 registers), 7.9 at 5 (48 registers); with the group
// test and the voted exact test, 6.0 ms at 7 blocks and 6.05 at 6.
// kFull: some periodic axis is spanned whole by the group's candidate cells
// (small boxes); without it the candidate test needs no minimum-image wrap.
template <bool kExcl, bool kFull>
__global__ void __launch_bounds__(256, 7) build_walk_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ keys,
	const uint32_t* __restrict__ s2o, const uint32_t* __restrict__ begin,
	const uint32_t* __restrict__ end, const StencilEntry* __restrict__ stencil_g, int ns,
	WalkGrid wg, uint32_t n, Box box, Exclusions ex, uint32_t* __restrict__ nbr, uint32_t cap,
	int hshift, uint32_t* __restrict__ row_len, uint32_t* __restrict__ row_far,
	unsigned long long* __restrict__ stats) {
	__shared__ uint32_t split_tab[256];
	__shared__ uint4 cell_buf[8 * kCellBuf];  // per warp: kept cells (jlo, end, image code, offset)
	__shared__ float4 cand_buf[8 * 32];       // per warp: candidates that pass the group test
	const int cells = 1 << wg.m;
	for (int k = threadIdx.x; k < cells; k += blockDim.x) split_tab[k] = split_by3(k);
	__syncthreads();
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	const uint32_t i_first = i & ~31u;
	if (i_first >= n) return;  // whole warp past the end
	const bool valid = i < n;
	const int h = 1 << hshift;
	const uint32_t mask = static_cast<uint32_t>(cells - 1);
	const float4 pi = valid ? sorted_pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
	const uint32_t c = valid ? keys[i] >> wg.shift : 0u;
	const int cx = static_cast<int>(compact_by3(c >> 2));
	const int cy = static_cast<int>(compact_by3(c >> 1));
	const int cz = static_cast<int>(compact_by3(c));
	const int a = valid ? static_cast<int>(s2o[i]) : 0;
	int row_b = 0, row_e = 0, body = -1;
	if (kExcl && valid) {
		if (ex.offsets && static_cast<uint32_t>(a) < ex.num_particles) {
			row_b = ex.offsets[a];
			row_e = ex.offsets[a + 1];
		}
		body = ex.rigid_body_id ? ex.rigid_body_id[a] : -1;
	}
	RowWriter row{nbr + (static_cast<size_t>(i >> hshift) * cap << hshift) + (i & (h - 1)), 0u,
				  0u, cap, h};
	const uint32_t c_first = keys[i_first] >> wg.shift;

	// Cell bounding box of the group (valid lanes only).
	const int x0 = warp_min(valid ? cx : INT_MAX), x1 = warp_max(valid ? cx : INT_MIN);
	const int y0 = warp_min(valid ? cy : INT_MAX), y1 = warp_max(valid ? cy : INT_MIN);
	const int z0 = warp_min(valid ? cz : INT_MAX), z1 = warp_max(valid ? cz : INT_MIN);
	const bool coherent = (x1 - x0) <= wg.emax && (y1 - y0) <= wg.emax && (z1 - z0) <= wg.emax;
	// The group's coordinate range: cells are pruned by their real distance to
	// it, which is tighter than the cell-index gap.
	const float gxlo = warp_minf(valid ? pi.x : INFINITY), gxhi = warp_maxf(valid ? pi.x : -INFINITY);
	const float gylo = warp_minf(valid ? pi.y : INFINITY), gyhi = warp_maxf(valid ? pi.y : -INFINITY);
	const float gzlo = warp_minf(valid ? pi.z : INFINITY), gzhi = warp_maxf(valid ? pi.z : -INFINITY);

	if (coherent) {
		walk_coherent_group<kExcl, kFull>(sorted_pos, s2o, begin, end, split_tab, cell_buf,
										  cand_buf, wg, box, ex, i, i_first, valid, pi, a, row_b,
										  row_e, body, c_first, x0, x1, y0, y1, z0, z1, gxlo,
										  gxhi, gylo, gyhi, gzlo, gzhi, row);
	} else if (valid) {
		// Wide group: each lane walks its own pruned cell stencil, exact test.
		for (int k = 0; k < ns; ++k) {
			const StencilEntry se = stencil_g[k];
			const int4 s = make_int4(se.dx, se.dy, se.dz, 0);
			int nx = cx + s.x, ny = cy + s.y, nz = cz + s.z;
			if (box.periodic[0]) nx = static_cast<int>(static_cast<uint32_t>(nx + cells) & mask);
			else if (nx < 0 || nx >= cells) continue;
			if (box.periodic[1]) ny = static_cast<int>(static_cast<uint32_t>(ny + cells) & mask);
			else if (ny < 0 || ny >= cells) continue;
			if (box.periodic[2]) nz = static_cast<int>(static_cast<uint32_t>(nz + cells) & mask);
			else if (nz < 0 || nz >= cells) continue;
			const uint32_t nc = (split_tab[nx] << 2) | (split_tab[ny] << 1) | split_tab[nz];
			if (nc < c) continue;  // every particle there precedes i
			const uint32_t b = begin[nc], e = end[nc];
			for (uint32_t j = b > i + 1u ? b : i + 1u; j < e; ++j) {
				const float4 pj = sorted_pos[j];
				if (exact_hit(box, pi, pj, wg.rc2)) {
					const int bj = static_cast<int>(s2o[j]);
					if (kExcl && is_excluded(ex, bj, row_b, row_e, body)) continue;
					row.append(j | (bj < a ? kOrientBit : 0u));
				}
			}
		}
	}
	if (valid) {
		row_len[i] = row.total();
		row_far[i] = row.far;
	}
	// stats[0] = total pairs, stats[1] = longest row
	unsigned long long tot = valid ? row.total() : 0u;
	int mx = valid ? static_cast<int>(min(row.total(), 0x7FFFFFFFu)) : 0;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
		mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
	}
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(stats, tot);
		atomicMax(stats + 1, static_cast<unsigned long long>(mx));
	}
}

__global__ void __launch_bounds__(256) export_kernel(const uint32_t* __restrict__ nbr,
													 const uint32_t* __restrict__ row_len,
													 const uint32_t* __restrict__ row_off,
													 const uint32_t* __restrict__ s2o, uint32_t n,
													 uint32_t cap, int hshift,
													 int2* __restrict__ out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int a = static_cast<int>(s2o[i]);
	const int h = 1 << hshift;
	const uint32_t* base = nbr + (static_cast<size_t>(i >> hshift) * cap << hshift) + (i & (h - 1));
	const uint32_t len = row_len[i], off = row_off[i];
	for (uint32_t k = 0; k < len; ++k) {
		const int b = static_cast<int>(s2o[base[static_cast<size_t>(k) * h] & ~kOrientBit]);
		out[off + k] = make_int2(a < b ? a : b, a < b ? b : a);
	}
}

// Small systems: one warp per particle row. The lanes take the row's pruned
// stencil cells 32 at a time (cells whose Morton code precedes the particle's
// hold only earlier particles and are skipped). The kept cells' candidate
// ranges are laid end to end by a warp scan of their lengths, and every round
// tests 32 consecutive candidates of that stream, one per lane, with the
// reference's exact test: each lane finds the cell its candidate falls in by a
// binary search over the running totals, held one per lane and read with warp
// shuffles. A round's hits are appended with two ballots (near entries from
// the front of the row, far ones from the back, as the group walk does). The
// group walk runs one warp per 32 particles and leaves most of the GPU idle
// below some 10^5 particles; here every particle has a warp. Rows hold the
// same pairs in another order.
template <bool kExcl>
__global__ void __launch_bounds__(256) build_rows_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ keys,
	const uint32_t* __restrict__ s2o, const uint32_t* __restrict__ begin,
	const uint32_t* __restrict__ end, const StencilEntry* __restrict__ stencil_g, int ns,
	WalkGrid wg, uint32_t n, Box box, Exclusions ex, uint32_t* __restrict__ nbr, uint32_t cap,
	int hshift, uint32_t* __restrict__ row_len, uint32_t* __restrict__ row_far,
	unsigned long long* __restrict__ stats) {
	const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (i >= n) return;  // whole warp
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t lt = (1u << lane) - 1u;
	const int cells = 1 << wg.m;
	const float4 pi = sorted_pos[i];
	const uint32_t c = keys[i] >> wg.shift;
	const int cx = static_cast<int>(compact_by3(c >> 2));
	const int cy = static_cast<int>(compact_by3(c >> 1));
	const int cz = static_cast<int>(compact_by3(c));
	// A neighbour's cell code is the home code plus the stencil entry's
	// interleaved offset on each axis, carried through the other axes' bits
	// (set to one) and masked: modulo 2^m per axis, so open axes also check
	// the plain coordinate range.
	const uint32_t lvl = (1u << (3 * wg.m)) - 1u;
	const uint32_t mx = 0x24924924u & lvl, my = 0x12492492u & lvl, mz = 0x09249249u & lvl;
	const uint32_t cxo = c | ~mx, cyo = c | ~my, czo = c | ~mz;
	const int a = static_cast<int>(s2o[i]);
	int row_b = 0, row_e = 0, body = -1;
	if (kExcl) {
		if (ex.offsets && static_cast<uint32_t>(a) < ex.num_particles) {
			row_b = ex.offsets[a];
			row_e = ex.offsets[a + 1];
		}
		body = ex.rigid_body_id ? ex.rigid_body_id[a] : -1;
	}
	const uint32_t h = 1u << hshift;
	uint32_t* base = nbr + (static_cast<size_t>(i >> hshift) * cap << hshift) + (i & (h - 1u));
	uint32_t len = 0, far = 0;
	for (int k0 = 0; k0 < ns; k0 += 32) {
		uint32_t jb = 0, je = 0;
		const int k = k0 + static_cast<int>(lane);
		if (k < ns) {
			const StencilEntry se = stencil_g[k];
			bool in = true;
			if (!box.periodic[0]) in = in && static_cast<unsigned>(cx + se.dx) < static_cast<unsigned>(cells);
			if (!box.periodic[1]) in = in && static_cast<unsigned>(cy + se.dy) < static_cast<unsigned>(cells);
			if (!box.periodic[2]) in = in && static_cast<unsigned>(cz + se.dz) < static_cast<unsigned>(cells);
			if (in) {
				const uint32_t d = static_cast<uint32_t>(se.pad);
				const uint32_t nc = ((cxo + (d & mx)) & mx) | ((cyo + (d & my)) & my) |
									((czo + (d & mz)) & mz);
				if (nc >= c) {  // earlier cells hold only earlier particles
					const uint32_t b = begin[nc];
					jb = b > i + 1u ? b : i + 1u;
					je = end[nc];
				}
			}
		}
		// The batch's candidate ranges laid end to end (a scan of their
		// lengths); each round the lanes take the next 32 candidates, lane l
		// finding the cell that holds candidate t0 + l by a binary search over
		// the lanes' running totals.
		// An empty cell (begin = end = 0) or one ending at i has jb >= je.
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
			bool hit = false, near = false;
			uint32_t entry = 0;
			if (t < total) {
				const uint32_t j = ob + (t - oe);
				const float4 pj = sorted_pos[j];
				const float3 d = wrap_diff(box, __fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
										   __fsub_rn(pj.z, pi.z));
				const float d2 = len2(d.x, d.y, d.z);
				if (d2 <= wg.rc2) {
					const int bj = static_cast<int>(s2o[j]);
					if (!(kExcl && is_excluded(ex, bj, row_b, row_e, body))) {
						hit = true;
						near = d2 <= wg.split2;
						entry = j | (bj < a ? kOrientBit : 0u);
					}
				}
			}
			const uint32_t nm = __ballot_sync(0xFFFFFFFFu, hit && near);
			const uint32_t fm = __ballot_sync(0xFFFFFFFFu, hit && !near);
			if (hit) {
				// Position among all of the row's entries (for the capacity check)
				// and the slot: near entries from the front, far from the back.
				const uint32_t p = len + far + static_cast<uint32_t>(__popc((nm | fm) & lt));
				const uint32_t slot = near ? len + static_cast<uint32_t>(__popc(nm & lt))
										   : cap - 1u - (far + static_cast<uint32_t>(__popc(fm & lt)));
				if (p < cap) base[static_cast<size_t>(slot) * h] = entry;
			}
			len += static_cast<uint32_t>(__popc(nm));
			far += static_cast<uint32_t>(__popc(fm));
		}
	}
	if (lane == 0) {
		row_len[i] = len + far;
		row_far[i] = far;
		atomicAdd(stats, static_cast<unsigned long long>(len + far));
		atomicMax(stats + 1, static_cast<unsigned long long>(len + far));
	}
}

// Moves each row's far entries (stored backwards from the end of its cap
// slots) to follow its near entries, so that a row is one contiguous run:
// near entries in candidate order, then the far ones. One warp per slice of
// H rows: lane l copies entries l / H, l / H + 32 / H, ... of row l % H, so
// each load and store instruction touches neighbouring words. Destinations
// precede sources (near + far <= cap) and every batch is loaded before it is
// stored, so the in-place copy is safe.
__global__ void __launch_bounds__(256) join_far_kernel(uint32_t* __restrict__ nbr,
													   const uint32_t* __restrict__ row_len,
													   const uint32_t* __restrict__ row_far,
													   uint32_t n, uint32_t cap, int hshift) {
	const uint32_t slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t h = 1u << hshift;
	const uint32_t slices = (n + h - 1u) >> hshift;
	if (slice >= slices) return;  // whole warp
	const uint32_t r = lane & (h - 1u), kk = lane >> hshift, step = 32u >> hshift;
	const uint32_t i = (slice << hshift) + r;
	const uint32_t far = i < n ? row_far[i] : 0u;
	const uint32_t near = i < n ? row_len[i] - far : 0u;
	uint32_t most = far;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) most = max(most, __shfl_xor_sync(0xFFFFFFFFu, most, o));
	uint32_t* base = nbr + static_cast<size_t>(slice) * cap * h + r;
	for (uint32_t k0 = 0; k0 < most; k0 += step) {
		const uint32_t k = k0 + kk;
		uint32_t v = 0u;
		if (k < far) v = base[static_cast<size_t>(cap - far + k) * h];
		__syncwarp();
		if (k < far) base[static_cast<size_t>(near + k) * h] = v;
		__syncwarp();
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
	// The word so far, read before the loads so its latency overlaps theirs:
	// a warp whose maximum is not above it has nothing to raise.
	const unsigned int seen = (threadIdx.x & 31) == 0 ? *reinterpret_cast<volatile unsigned int*>(out) : 0u;
	float d2 = 0.0f;
	if (i < n) {
		const float4 c = cur[i], p = prev[i];
		const float dx = min_image(__fsub_rn(c.x, p.x), len.x);
		const float dy = min_image(__fsub_rn(c.y, p.y), len.y);
		const float dz = min_image(__fsub_rn(c.z, p.z), len.z);
		d2 = len2(dx, dy, dz);
		if (isnan(d2)) d2 = 0.0f;  // a NaN coordinate does not trip the skin check
	}
	// Non-negative floats order like their bit patterns.
	const unsigned int bits = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(d2));
	if ((threadIdx.x & 31) == 0 && bits > seen) atomicMax(out, bits);
}

__global__ void __launch_bounds__(256) pack_kernel(const float4* __restrict__ pos,
												   const int* __restrict__ type_ids,
												   const uint32_t* __restrict__ s2o, uint32_t n,
												   float4* __restrict__ sorted_pos,
												   unsigned long long* nonfinite,
												   float4* __restrict__ clear_a,
												   float4* __restrict__ clear_b,
												   DisplacementTrack track) {
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	// The tracked word so far, read before the loads (see displacement_kernel).
	const unsigned int seen = track.d2max && (threadIdx.x & 31) == 0
								  ? *reinterpret_cast<volatile unsigned int*>(track.d2max)
								  : 0u;
	float d2 = 0.0f;
	if (s < n) {
		// Accumulators of the step that follows, cleared here instead of by
		// separate memsets (one launch less each on short steps).
		if (clear_a) clear_a[s] = make_float4(0.f, 0.f, 0.f, 0.f);
		if (clear_b) clear_b[s] = make_float4(0.f, 0.f, 0.f, 0.f);
		const uint32_t o = s2o[s];
		float4 p = pos[o];
		if (nonfinite && !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z)))
			atomicAdd(nonfinite, 1ull);
		if (track.d2max) {
			const float4 r = track.ref_sorted[s];
			d2 = len2(min_image(__fsub_rn(p.x, r.x), track.len[0]),
					  min_image(__fsub_rn(p.y, r.y), track.len[1]),
					  min_image(__fsub_rn(p.z, r.z), track.len[2]));
			const float c[3] = {p.x, p.y, p.z};
			bool inside = d2 <= FLT_MAX;  // false for NaN
#pragma unroll
			for (int a = 0; a < 3; ++a)
				inside = inside && (track.len[a] == 0.0f || (c[a] >= track.lo[a] && c[a] <= track.hi[a]));
			if (!inside) d2 = INFINITY;
		}
		p.w = __int_as_float(type_ids ? type_ids[o] : 0);
		sorted_pos[s] = p;
	}
	if (track.d2max) {
		// Non-negative floats order like their bit patterns; the word only
		// grows between builds, so most warps find nothing to raise.
		const unsigned int bits = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(d2));
		if ((threadIdx.x & 31) == 0 && bits > seen) atomicMax(track.d2max, bits);
	}
}

}  // namespace

void cell_ranges(const uint32_t* keys, uint32_t n, int shift, uint32_t* begin, uint32_t* end,
				 size_t num_cells, cudaStream_t st) {
	MB2_CUDA(cudaMemsetAsync(begin, 0, num_cells * sizeof(uint32_t), st));
	MB2_CUDA(cudaMemsetAsync(end, 0, num_cells * sizeof(uint32_t), st));
	if (n == 0) return;
	MB2_LAUNCH cell_ranges_kernel<<<(n + 255) / 256, 256, 0, st>>>(keys, n, shift, begin, end);
}

void build_walk(const float4* sorted_pos, const uint32_t* keys, const uint32_t* s2o,
				const uint32_t* begin, const uint32_t* end, const StencilEntry* stencil,
				int num_stencil, const WalkGrid& wg, uint32_t n, const Box& box,
				const Exclusions& ex, uint32_t* nbr, uint32_t cap, int hshift, uint32_t* row_len,
				uint32_t* row_far, unsigned long long* stats, cudaStream_t st) {
	MB2_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), st));
	if (n == 0) return;
	const bool excl = ex.offsets != nullptr || ex.rigid_body_id != nullptr;
	// The kernel variant with the minimum-image wrap is needed when a coherent
	// group's candidate cells can span a whole periodic axis: a cell spread of
	// up to emax plus the stencil's 2 * radius + 1 reaching the cell count.
	bool full = false;
	for (int a = 0; a < 3; ++a)
		full = full || (box.periodic[a] && wg.emax + 2 * wg.radius[a] + 1 >= (1 << wg.m));
	if (n <= kRowWalkMaxN) {
		// One warp per particle (8 particles per 256-thread block).
		auto rows = excl ? build_rows_kernel<true> : build_rows_kernel<false>;
		MB2_LAUNCH rows<<<(n + 7) / 8, 256, 0, st>>>(sorted_pos, keys, s2o, begin, end, stencil,
													 num_stencil, wg, n, box, ex, nbr, cap,
													 hshift, row_len, row_far, stats);
		return;
	}
	auto kern = excl ? (full ? build_walk_kernel<true, true> : build_walk_kernel<true, false>)
					 : (full ? build_walk_kernel<false, true> : build_walk_kernel<false, false>);
	// The stencil (used by the few groups that walk per particle) is read
	// through L1, leaving shared memory to the cell buffers.
	MB2_LAUNCH kern<<<(n + 255) / 256, 256, 0, st>>>(sorted_pos, keys, s2o, begin, end,
														 stencil, num_stencil, wg, n, box, ex,
														 nbr, cap, hshift, row_len, row_far, stats);
}

void join_far(uint32_t* nbr, const uint32_t* row_len, const uint32_t* row_far, uint32_t n,
			  uint32_t cap, int hshift, cudaStream_t st) {
	if (n == 0) return;
	const uint32_t slices = (n + (1u << hshift) - 1u) >> hshift;
	const uint32_t blocks = (slices + 7u) / 8u;  // 8 warps (slices) per block
	MB2_LAUNCH join_far_kernel<<<blocks, 256, 0, st>>>(nbr, row_len, row_far, n, cap, hshift);
}

void export_pairs(const uint32_t* nbr, const uint32_t* row_len, const uint32_t* row_off,
				  const uint32_t* s2o, uint32_t n, uint32_t cap, int hshift, int2* out,
				  cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH export_kernel<<<(n + 255) / 256, 256, 0, st>>>(nbr, row_len, row_off, s2o, n, cap,
															  hshift, out);
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

DisplacementTrack displacement_track(const Box& box, const float4* ref_sorted,
									 unsigned int* d2max) {
	DisplacementTrack t;
	t.ref_sorted = ref_sorted;
	t.d2max = d2max;
	for (int a = 0; a < 3; ++a) {
		t.len[a] = box.periodic[a] ? box.size[a] : 0.0f;
		t.lo[a] = box.origin[a] - kTrackBand;
		t.hi[a] = box.origin[a] + box.size[a] + kTrackBand;
	}
	return t;
}

void pack_sorted_positions(const float4* pos, const int* type_ids, const uint32_t* s2o,
						   uint32_t n, float4* sorted_pos, cudaStream_t st,
						   unsigned long long* nonfinite, float4* clear_a, float4* clear_b,
						   const DisplacementTrack& track) {
	if (n == 0) return;
	MB2_LAUNCH pack_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, type_ids, s2o, n, sorted_pos,
															 nonfinite, clear_a, clear_b, track);
}

}  // namespace mb2
