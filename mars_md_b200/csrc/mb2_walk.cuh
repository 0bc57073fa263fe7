// Device pieces of the pairlist walks shared by the plain and the batched
// builds: the reference's exact pair test, warp reductions, the cell gap of
// the group walk, the sliced-ELL row writer and the coherent-group walk.
#pragma once

#include "mb2_internal.cuh"

namespace mb2 {

// ExclusionView::row_contains / same_body (src/Interactions/DeviceExclusions.h:22-75):
// b is excluded from the row [row_b, row_e) of the CSR or shares its rigid body.
__device__ __forceinline__ bool is_excluded(const Exclusions& ex, int b, int row_b, int row_e,
											int body) {
	if (body >= 0 && ex.rigid_body_id[b] == body) return true;
	for (int e = row_b; e < row_e; ++e)
		if (ex.neighbors[e] == b) return true;
	return false;
}

// Exact reference test: wrap_diff(pj - pi).length2() <= rc2, same rounding.
__device__ __forceinline__ bool exact_hit(const Box& box, const float4& pi, const float4& pj,
										  float rc2) {
	const float3 d = wrap_diff(box, __fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
							   __fsub_rn(pj.z, pi.z));
	return len2(d.x, d.y, d.z) <= rc2;
}

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
	return v;
}
__device__ __forceinline__ float warp_minf(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
	return v;
}
__device__ __forceinline__ float warp_maxf(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
	return v;
}

// Distance along one axis from the group's coordinate range [glo, ghi] to
// cell nx (shifted by sh, the periodic image offset): the cell's real extent
// with the Morton rounding margin; on a periodic axis the edge cells also hold
// particles that lie outside the box (their Morton coordinate clamps), so
// they extend outwards without bound.
__device__ __forceinline__ float cell_gap(const WalkGrid& wg, int ax, int nx, int cells,
										  bool periodic, float sh, float glo, float ghi) {
	float lo = wg.dom_lo[ax] + static_cast<float>(nx) * wg.cell_w[ax] + sh - wg.eps[ax];
	float hi = wg.dom_lo[ax] + static_cast<float>(nx + 1) * wg.cell_w[ax] + sh + wg.eps[ax];
	if (periodic) {
		if (nx == 0) lo = -INFINITY;
		if (nx == cells - 1) hi = INFINITY;
	}
	return fmaxf(0.0f, fmaxf(lo - ghi, glo - hi));
}

// Cells a warp buffers before walking them (32 tested at a time: at most
// 31 left over plus 32 new).
constexpr uint32_t kCellBuf = 64;

// Periodic image offset of a buffered cell on axis ax: code bits 2ax..2ax+1
// hold 1 (-size) or 2 (+size).
__device__ __forceinline__ float image_shift(uint32_t code, int ax, const Box& box) {
	const uint32_t c = (code >> (2 * ax)) & 3u;
	return c == 1u ? -box.size[ax] : (c == 2u ? box.size[ax] : 0.0f);
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
	return v;
}

// Appends one lane's row of the sliced-ELL list: near entries from the front,
// far entries (beyond the split radius) from the back of the row's cap slots;
// join_far_kernel then moves the far ones to follow the near ones. Entries
// past cap are only counted (the host then grows the list and walks again).
struct RowWriter {
	uint32_t* base;  // &nbr[entry 0 of this row]
	uint32_t len;    // near entries
	uint32_t far;    // far entries
	uint32_t cap;
	int h;           // slice height: stride between a row's entries
	__device__ __forceinline__ void append(uint32_t entry) {
		if (len + far < cap) base[static_cast<size_t>(len) * h] = entry;
		++len;
	}
	// Near entry to the front, far entry to the back, without a branch.
	__device__ __forceinline__ void put(uint32_t entry, bool near) {
		const uint32_t slot = near ? len : cap - 1u - far;
		if (len + far < cap) base[static_cast<size_t>(slot) * h] = entry;
		len += near ? 1u : 0u;
		far += near ? 0u : 1u;
	}
	__device__ __forceinline__ uint32_t total() const { return len + far; }
};

// The walk of a coherent group (its particles' cells within emax of each
// other on every axis): candidate cells are the group's cell box widened by
// the stencil radius (or every cell on an axis the stencil spans); the lanes
// test 32 of them at a time in parallel, each against the group's coordinate
// range, and append the kept ones, in box order, to the warp's buffer; the
// warp then walks the buffered cells' candidates together, each loaded once
// for all 32 lanes. begin / end index this grid's cells; c_first is the cell
// of the group's first particle, whose earlier cells hold only earlier
// particles. Shared by the plain group walk and the batched one.
template <bool kExcl, bool kFull>
__device__ __forceinline__ void walk_coherent_group(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ s2o,
	const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
	const uint32_t* split_tab, uint4* cell_buf, float4* cand_buf, const WalkGrid& wg,
	const Box& box, const Exclusions& ex, uint32_t i, uint32_t i_first, bool valid,
	const float4& pi, int a, int row_b, int row_e, int body, uint32_t c_first, int x0, int x1,
	int y0, int y1, int z0, int z1, float gxlo, float gxhi, float gylo, float gyhi, float gzlo,
	float gzhi, RowWriter& row) {
	const int cells = 1 << wg.m;
	// Candidate cells: the group's cell box widened by the stencil radius (or
	// every cell on an axis the stencil spans). The lanes test 32 of them at
	// a time in parallel, each against the group's coordinate range, and
	// append the kept ones, in box order, to the warp's buffer; the warp
	// then walks the buffered cells' candidates together.
	const int lo[3] = {x0, y0, z0}, hi[3] = {x1, y1, z1};
	const float glo[3] = {gxlo, gylo, gzlo}, ghi[3] = {gxhi, gyhi, gzhi};
	int from[3], span[3];
	bool full[3];
#pragma unroll
	for (int ax = 0; ax < 3; ++ax) {
		full[ax] = kFull && box.periodic[ax] && (hi[ax] - lo[ax] + 2 * wg.radius[ax] + 1 >= cells);
		from[ax] = full[ax] ? 0 : lo[ax] - wg.radius[ax];
		span[ax] = full[ax] ? cells : hi[ax] - lo[ax] + 2 * wg.radius[ax] + 1;
	}
	const uint32_t total = static_cast<uint32_t>(span[0] * span[1] * span[2]);
	const int lane = static_cast<int>(threadIdx.x & 31u);
	uint4* buf = cell_buf + (threadIdx.x >> 5) * kCellBuf;
	uint32_t count = 0;
	float4* cbuf = cand_buf + (threadIdx.x >> 5) * 32;
	const uint32_t lt_mask = (1u << lane) - 1u;
	// A candidate whose distance from the group's coordinate range (less
	// the Morton rounding margin) is above the fast test's upper bound gives
	// every lane d^2 > fast_hi below, so no lane keeps it; such candidates
	// are dropped 32 at a time before the lanes test the rest one by one.
	const float gate = wg.fast_hi;
	auto walk_buffered = [&](uint32_t m) {
		// Offsets of the buffered cells' candidate ranges in one stream.
		const uint32_t l0 = static_cast<uint32_t>(lane) < m ? buf[lane].y - buf[lane].x : 0u;
		const uint32_t l1 = static_cast<uint32_t>(lane) + 32u < m ? buf[lane + 32].y - buf[lane + 32].x : 0u;
		uint32_t s0 = l0, s1 = l1;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t a0 = __shfl_up_sync(0xFFFFFFFFu, s0, o);
			const uint32_t a1 = __shfl_up_sync(0xFFFFFFFFu, s1, o);
			if (lane >= o) {
				s0 += a0;
				s1 += a1;
			}
		}
		const uint32_t tot0 = __shfl_sync(0xFFFFFFFFu, s0, 31);
		const uint32_t stream = tot0 + __shfl_sync(0xFFFFFFFFu, s1, 31);
		if (static_cast<uint32_t>(lane) < m) buf[lane].w = s0 - l0;
		if (static_cast<uint32_t>(lane) + 32u < m) buf[lane + 32].w = tot0 + s1 - l1;
		__syncwarp();
		uint32_t kc = 0;  // this lane's cell in the stream (advances monotonically)
		for (uint32_t t0 = 0; t0 < stream; t0 += 32u) {
			const uint32_t t = t0 + static_cast<uint32_t>(lane);
			bool pass = false;
			float4 cand = make_float4(0.f, 0.f, 0.f, 0.f);
			if (t < stream) {
				while (kc + 1u < m && buf[kc + 1u].w <= t) ++kc;
				const uint4 cb = buf[kc];
				const uint32_t j = cb.x + (t - cb.w);
				const float4 pj = sorted_pos[j];
				// The candidate moved into the group's image.
				const float sx = pj.x + image_shift(cb.z, 0, box);
				const float sy = pj.y + image_shift(cb.z, 1, box);
				const float sz = pj.z + image_shift(cb.z, 2, box);
				const float gx = full[0] ? 0.0f : fmaxf(0.0f, fmaxf(gxlo - sx, sx - gxhi) - wg.eps[0]);
				const float gy = full[1] ? 0.0f : fmaxf(0.0f, fmaxf(gylo - sy, sy - gyhi) - wg.eps[1]);
				const float gz = full[2] ? 0.0f : fmaxf(0.0f, fmaxf(gzlo - sz, sz - gzhi) - wg.eps[2]);
				pass = gx * gx + gy * gy + gz * gz <= gate;
				cand = make_float4(sx, sy, sz, __uint_as_float(j));
			}
			const uint32_t pm = __ballot_sync(0xFFFFFFFFu, pass);
			if (pass) cbuf[__popc(pm & lt_mask)] = cand;
			__syncwarp();
			const int np = __popc(pm);
			for (int q = 0; q < np; ++q) {
				const float4 c4 = cbuf[q];
				const uint32_t j = __float_as_uint(c4.w);
				float dx = c4.x - pi.x, dy = c4.y - pi.y, dz = c4.z - pi.z;
				if (kFull) {
					if (full[0]) dx -= box.size[0] * rintf(dx * box.inv[0]);
					if (full[1]) dy -= box.size[1] * rintf(dy * box.inv[1]);
					if (full[2]) dz -= box.size[2] * rintf(dz * box.inv[2]);
				}
				const float d2 = dx * dx + dy * dy + dz * dz;
				bool hit = valid && j > i && d2 < wg.fast_lo;
				// The exact test for the few lanes within rounding of the radius,
				// behind a warp vote so that the other candidates skip it.
				const bool band = valid && j > i && !hit && d2 <= wg.fast_hi;
				if (__any_sync(0xFFFFFFFFu, band)) {
					if (band) hit = exact_hit(box, pi, sorted_pos[j], wg.rc2);
				}
				if (hit) {
					const int bj = static_cast<int>(s2o[j]);
					if (kExcl && is_excluded(ex, bj, row_b, row_e, body)) continue;
					row.put(j | (bj < a ? kOrientBit : 0u), d2 <= wg.split2);
				}
			}
			__syncwarp();
		}
	};
	for (uint32_t base = 0; base < total; base += 32u) {
		const uint32_t idx = base + static_cast<uint32_t>(lane);
		bool keep = false;
		uint4 rec = make_uint4(0u, 0u, 0u, 0u);
		if (idx < total) {
			const uint32_t iz = idx % static_cast<uint32_t>(span[2]);
			const uint32_t t = idx / static_cast<uint32_t>(span[2]);
			const int u[3] = {from[0] + static_cast<int>(t / static_cast<uint32_t>(span[1])),
							  from[1] + static_cast<int>(t % static_cast<uint32_t>(span[1])),
							  from[2] + static_cast<int>(iz)};
			bool in_range = true;
			float g2 = 0.0f;
			uint32_t code = 0, nc = 0;
#pragma unroll
			for (int ax = 0; ax < 3; ++ax) {
				int nn = u[ax];
				float sh = 0.0f;
				if (!full[ax]) {
					if (box.periodic[ax]) {
						if (nn < 0) { nn += cells; sh = -box.size[ax]; code |= 1u << (2 * ax); }
						else if (nn >= cells) { nn -= cells; sh = box.size[ax]; code |= 2u << (2 * ax); }
					} else if (nn < 0 || nn >= cells) {
						in_range = false;
						nn = 0;
					}
					const float g = cell_gap(wg, ax, nn, cells, box.periodic[ax], sh, glo[ax], ghi[ax]);
					g2 += g * g;
				}
				nc |= split_tab[nn] << (2 - ax);
			}
			if (in_range && g2 <= wg.lim && nc >= c_first) {
				const uint32_t b = begin[nc], e = end[nc];
				const uint32_t jlo = b > i_first + 1u ? b : i_first + 1u;
				if (jlo < e) {
					keep = true;
					rec = make_uint4(jlo, e, code, 0u);
				}
			}
		}
		const uint32_t kept = __ballot_sync(0xFFFFFFFFu, keep);
		if (keep) buf[count + __popc(kept & ((1u << lane) - 1u))] = rec;
		count += static_cast<uint32_t>(__popc(kept));
		__syncwarp();
		if (count >= 32u) {
			walk_buffered(count);
			count = 0;
			__syncwarp();
		}
	}
	walk_buffered(count);
}

}  // namespace mb2
