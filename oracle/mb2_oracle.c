/*
 * CPU oracle for the MARS-MD Brownian-dynamics force-and-integrate path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never part of the
 * product. Each function restates one step of the reference algorithm in
 * plain C; the reference file:line it follows is cited on every function
 * (paths are relative to the MARS-MD source tree).
 *
 * Build: gcc -std=c11 -O2 -ffp-contract=off -fno-fast-math -fPIC -shared.
 * No FMA contraction and no fast-math: float results must round exactly as
 * the reference's host-compiled functors do, which the pin tests check
 * bit-for-bit against those functors and against committed fixtures.
 */
#include "mb2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

int or_version(void) { return 1; }

/* ------------------------------------------------------------------------ */
/* Periodic box                                                             */
/* ------------------------------------------------------------------------ */

/* PeriodicBox::wrap_diff_scalar (src/System/PeriodicBox.h:453-461). */
float or_wrap_diff_scalar(float x, float l) {
	if (l <= 0.0f)
		return x;
	const float inv = 1.0f / l;
	const int image = (int)floorf(x * inv);
	x -= (float)image * l;
	if (x >= 0.5f * l)
		x -= l;
	return x;
}

/* PeriodicBox::wrap_scalar (src/System/PeriodicBox.h:445-451). */
float or_wrap_scalar(float x, float o, float l) {
	if (l <= 0.0f)
		return x;
	const float rel = x - o;
	const float inv = 1.0f / l;
	const int image = (int)floorf(rel * inv);
	return x - (float)image * l;
}

/* PeriodicBox::wrap_diff, orthogonal path (src/System/PeriodicBox.h:134-146). */
static void box_wrap_diff(const or_box* b, const float* d, float* out) {
	for (int a = 0; a < 3; ++a)
		out[a] = b->periodic[a] ? or_wrap_diff_scalar(d[a], b->size[a]) : d[a];
}

void or_wrap_diff(const or_box* b, const float* in4, float* out4, size_t n) {
	for (size_t i = 0; i < n; ++i) {
		box_wrap_diff(b, in4 + 4 * i, out4 + 4 * i);
		out4[4 * i + 3] = 0.0f;
	}
}

/* PeriodicBox::wrap, orthogonal path (src/System/PeriodicBox.h:172-184). */
void or_wrap(const or_box* b, const float* in4, float* out4, size_t n) {
	for (size_t i = 0; i < n; ++i) {
		for (int a = 0; a < 3; ++a)
			out4[4 * i + a] = b->periodic[a]
			                      ? or_wrap_scalar(in4[4 * i + a], b->origin[a], b->size[a])
			                      : in4[4 * i + a];
		out4[4 * i + 3] = 0.0f;
	}
}

/* Vector3_t::length2 (src/Types/Vector3.h): x*x + y*y + z*z, left to right. */
static float len2(const float* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }

/* ------------------------------------------------------------------------ */
/* Morton sort                                                              */
/* ------------------------------------------------------------------------ */

/* MortonCode::splitBy3 (src/PatchOperation/ZOrderKernels/MortonCode.h:157-169). */
static uint32_t split_by3(uint32_t a) {
	uint32_t x = a & 1023u;
	x = (x | x << 16) & 0x30000ffu;
	x = (x | x << 8) & 0x300f00fu;
	x = (x | x << 4) & 0x30c30c3u;
	x = (x | x << 2) & 0x9249249u;
	return x;
}

static uint32_t compact_by3(uint32_t x) {
	x &= 0x09249249u;
	x = (x ^ (x >> 2)) & 0x030c30c3u;
	x = (x ^ (x >> 4)) & 0x0300f00fu;
	x = (x ^ (x >> 8)) & 0x030000ffu;
	x = (x ^ (x >> 16)) & 0x000003ffu;
	return x;
}

/* MortonCode::encode(pos, box_min, box_max) (MortonCode.h:95-131) and
 * encode(x, y, z) (MortonCode.h:91-93): IEEE division by the clamped range,
 * scale by 1023, clamp to [0, 1023], truncate; key = z | y<<1 | x<<2. */
uint32_t or_morton_key(const float* p, const float* bmin, const float* bmax) {
	uint32_t q[3];
	for (int a = 0; a < 3; ++a) {
		float range = bmax[a] - bmin[a];
		range = fmaxf(range, 1e-6f);
		const float offset = p[a] - bmin[a];
		const float normalized = offset / range;
		q[a] = (uint32_t)fminf(fmaxf(normalized * 1023.0f, 0.0f), 1023.0f);
	}
	return split_by3(q[2]) | (split_by3(q[1]) << 1) | (split_by3(q[0]) << 2);
}

/* MortonEncodeKernel (src/PatchOperation/ZOrderKernels/ZOrderKernels.h:27-43). */
void or_morton_encode(const float* pos4, size_t n, const float* bmin, const float* bmax,
                      uint32_t* keys, uint32_t* idx) {
	for (size_t i = 0; i < n; ++i) {
		keys[i] = or_morton_key(pos4 + 4 * i, bmin, bmax);
		idx[i] = (uint32_t)i;
	}
}

/* Stable sort of (key, value) pairs by the full 32-bit key: the contract of
 * cub::DeviceRadixSort::SortPairs over bits [0, 32)
 * (src/PatchOperation/ZOrderKernels/CUDASort.cu:13-98). Restated as a
 * four-pass LSD radix sort on 8-bit digits, which is stable. */
void or_sort_pairs(uint32_t* keys, uint32_t* vals, size_t n) {
	uint32_t* k2 = (uint32_t*)malloc(n * sizeof(uint32_t) + 4);
	uint32_t* v2 = (uint32_t*)malloc(n * sizeof(uint32_t) + 4);
	uint32_t *ks = keys, *vs = vals, *kd = k2, *vd = v2;
	for (int pass = 0; pass < 4; ++pass) {
		const int shift = 8 * pass;
		size_t count[257];
		memset(count, 0, sizeof(count));
		for (size_t i = 0; i < n; ++i)
			count[((ks[i] >> shift) & 255u) + 1]++;
		for (int d = 0; d < 256; ++d)
			count[d + 1] += count[d];
		for (size_t i = 0; i < n; ++i) {
			const size_t dst = count[(ks[i] >> shift) & 255u]++;
			kd[dst] = ks[i];
			vd[dst] = vs[i];
		}
		uint32_t* t = ks; ks = kd; kd = t;
		t = vs; vs = vd; vd = t;
	}
	/* four passes: the result is back in the caller's buffers */
	free(k2);
	free(v2);
}

/* InverseIndexKernel (ZOrderKernels.h:68-83). */
void or_inverse(const uint32_t* sorted, uint32_t* inv, size_t n) {
	for (size_t i = 0; i < n; ++i)
		if (sorted[i] < n)
			inv[sorted[i]] = (uint32_t)i;
}

/* ReorderDataKernel<Vector3> (ZOrderKernels.h:48-63). */
void or_gather4(const float* in4, float* out4, const uint32_t* sorted, size_t n) {
	for (size_t i = 0; i < n; ++i)
		memcpy(out4 + 4 * i, in4 + 4 * (size_t)sorted[i], 16);
}

/* Morton domain: ZOrderPairlist::build_pairlist (src/PatchOperation/
 * PairListKernels/ZOrderPairlist.cpp:130-146) with compute_particle_extent
 * (ZOrderPairlist.cpp:368-411): open axes use the particle extent widened by
 * 1 % (and to at least 1e-4), periodic axes use the box. */
void or_morton_domain(const or_box* b, const float* pos4, size_t n, float* bmin, float* bmax) {
	for (int a = 0; a < 3; ++a) {
		float lo = 3.402823466e38f, hi = -3.402823466e38f;
		for (size_t i = 0; i < n; ++i) {
			lo = fminf(lo, pos4[4 * i + a]);
			hi = fmaxf(hi, pos4[4 * i + a]);
		}
		const float margin = (hi - lo) * 0.01f;
		lo -= margin;
		hi += margin;
		const float range = hi - lo;
		if (range < 1e-4f) {
			/* the reference mixes in double literals here */
			const float center = (float)((double)lo + (double)range * 0.5);
			lo = (float)((double)center - (double)1e-4f * 0.5);
			hi = (float)((double)center + (double)1e-4f * 0.5);
		}
		if (b->periodic[a]) {
			lo = b->origin[a];
			hi = b->origin[a] + b->size[a];
		}
		bmin[a] = lo;
		bmax[a] = hi;
	}
}

/* ------------------------------------------------------------------------ */
/* Pairlist                                                                 */
/* ------------------------------------------------------------------------ */

/* ZOrderPairlist::select_cell_grid (ZOrderPairlist.cpp:24-81): over m = 0..10
 * minimise scanned volume x slots, stopping once cells outnumber particles or
 * the cell tables outgrow the pair buffer. */
void or_select_cell_grid(const float* extent, float cutoff, size_t n, size_t max_pairs, int* m_out,
                         int* radii, int* slots_out) {
	*m_out = 0;
	radii[0] = radii[1] = radii[2] = 1;
	*slots_out = 1;
	const double ext[3] = {(double)extent[0], (double)extent[1], (double)extent[2]};
	if (cutoff <= 0.0f || ext[0] <= 0.0 || ext[1] <= 0.0 || ext[2] <= 0.0 || n == 0)
		return;
	int best_m = 0, best_r[3] = {1, 1, 1};
	long long best_slots = 1;
	double best_cost = 0.0;
	int have_best = 0;
	for (int m = 0; m <= 10; ++m) {
		const long long cells_per_axis = 1LL << m;
		const size_t num_cells = (size_t)1 << (3 * m);
		int r[3];
		long long span[3];
		double volume = 1.0;
		for (int a = 0; a < 3; ++a) {
			const double side = ext[a] / (double)cells_per_axis;
			r[a] = (int)ceil((double)cutoff / side);
			span[a] = 2LL * r[a] + 1LL;
			if (span[a] > cells_per_axis)
				span[a] = cells_per_axis;
			volume *= (double)span[a] * side;
		}
		const long long slots = span[0] * span[1] * span[2];
		if (m > 0 && num_cells > n)
			break;
		const size_t bytes = num_cells * ((size_t)slots * 4u + 8u);
		if (m > 0 && bytes > max_pairs * 8u)
			break;
		const double cost = volume * (double)slots;
		if (!have_best || cost < best_cost) {
			have_best = 1;
			best_cost = cost;
			best_m = m;
			best_r[0] = r[0];
			best_r[1] = r[1];
			best_r[2] = r[2];
			best_slots = slots;
		}
	}
	*m_out = best_m;
	radii[0] = best_r[0];
	radii[1] = best_r[1];
	radii[2] = best_r[2];
	*slots_out = (int)best_slots;
}

/* BuildCellRangesKernel (src/PatchOperation/PairListKernels/ZOrderNeighbor.h:27-43);
 * begin/end must be zero-filled by the caller. */
void or_cell_ranges(const uint32_t* keys, size_t n, int shift, uint32_t* begin, uint32_t* end) {
	for (size_t i = 0; i < n; ++i) {
		const uint32_t c = keys[i] >> shift;
		if (i == 0 || (keys[i - 1] >> shift) != c)
			begin[c] = (uint32_t)i;
		if (i + 1 == n || (keys[i + 1] >> shift) != c)
			end[c] = (uint32_t)(i + 1);
	}
}

/* BuildCellNeighborsKernel::axis_range (ZOrderNeighbor.h:83-91). */
static void axis_range(int periodic, int r, int n, int* lo, int* hi) {
	if (periodic && 2 * r + 1 >= n) {
		*lo = 0;
		*hi = n - 1;
	} else {
		*lo = -r;
		*hi = r;
	}
}

/* BuildCellNeighborsKernel (ZOrderNeighbor.h:55-139): per-cell stencil rows,
 * x outer, z inner, padded with 0xFFFFFFFF. */
void or_cell_neighbors(uint32_t* table, int m, const int* radii, int npc, const float* box_len) {
	const size_t num_cells = (size_t)1 << (3 * m);
	const int n = 1 << m;
	const uint32_t mask = (uint32_t)(n - 1);
	const int per[3] = {box_len[0] > 0.0f, box_len[1] > 0.0f, box_len[2] > 0.0f};
	int lo[3], hi[3];
	for (int a = 0; a < 3; ++a)
		axis_range(per[a], radii[a], n, &lo[a], &hi[a]);
	for (size_t c = 0; c < num_cells; ++c) {
		const uint32_t cell = (uint32_t)c;
		const int cx = (int)compact_by3(cell >> 2);
		const int cy = (int)compact_by3(cell >> 1);
		const int cz = (int)compact_by3(cell);
		uint32_t* out = table + c * (size_t)npc;
		int k = 0;
		for (int dx = lo[0]; dx <= hi[0]; ++dx) {
			int nx = cx + dx;
			if (per[0])
				nx = (int)(((uint32_t)(nx + n)) & mask);
			else if (nx < 0 || nx >= n)
				continue;
			const uint32_t mx = split_by3((uint32_t)nx) << 2;
			for (int dy = lo[1]; dy <= hi[1]; ++dy) {
				int ny = cy + dy;
				if (per[1])
					ny = (int)(((uint32_t)(ny + n)) & mask);
				else if (ny < 0 || ny >= n)
					continue;
				const uint32_t mxy = mx | (split_by3((uint32_t)ny) << 1);
				for (int dz = lo[2]; dz <= hi[2]; ++dz) {
					int nz = cz + dz;
					if (per[2])
						nz = (int)(((uint32_t)(nz + n)) & mask);
					else if (nz < 0 || nz >= n)
						continue;
					out[k++] = mxy | split_by3((uint32_t)nz);
				}
			}
		}
		for (; k < npc; ++k)
			out[k] = 0xFFFFFFFFu;
	}
}

/* ExclusionView::row_contains / same_body (src/Interactions/DeviceExclusions.h:22-75). */
static int excluded(int a, int b, const int* off, const int* nb, size_t excl_n, const int* rb) {
	if (rb && rb[a] >= 0 && rb[b] == rb[a])
		return 1;
	if (!off || a < 0 || (size_t)a >= excl_n)
		return 0;
	for (int e = off[a]; e < off[a + 1]; ++e)
		if (nb[e] == b)
			return 1;
	return 0;
}

/* ZOrderCellNeighborKernel (ZOrderNeighbor.h:155-225), one particle at a time:
 * for each stencil cell, j in [max(begin, i+1), end), keep pairs with
 * wrapped |d|^2 <= rc^2 that are not excluded, emitted as (min, max) of the
 * original indices. Returns the pair count; writes at most max_pairs. */
uint64_t or_neighbor_walk(const float* sorted_pos4, const uint32_t* keys, const uint32_t* s2o,
                          const uint32_t* begin, const uint32_t* end, const uint32_t* table,
                          int npc, int shift, float cutoff_sq, size_t n, const or_box* b,
                          const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                          const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                          uint64_t* checksum) {
	uint64_t count = 0, sum = 0;
	/* Without a pair buffer only the count and the (order-independent) hash
	 * sum are wanted, so particles may be walked in parallel. */
#pragma omp parallel for reduction(+ : count, sum) schedule(dynamic, 4096) if (pairs == NULL)
	for (size_t i = 0; i < n; ++i) {
		const float* pi = sorted_pos4 + 4 * i;
		const uint32_t cell = keys[i] >> shift;
		const uint32_t* nbrs = table + (size_t)cell * npc;
		const int a = (int)s2o[i];
		for (int k = 0; k < npc; ++k) {
			const uint32_t nc = nbrs[k];
			if (nc == 0xFFFFFFFFu)
				continue;
			const uint32_t lo = begin[nc] > (uint32_t)i + 1u ? begin[nc] : (uint32_t)i + 1u;
			for (uint32_t j = lo; j < end[nc]; ++j) {
				const float* pj = sorted_pos4 + 4 * (size_t)j;
				const float d[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
				float w[3];
				box_wrap_diff(b, d, w);
				if (len2(w) <= cutoff_sq) {
					const int bb = (int)s2o[j];
					if (excluded(a, bb, excl_offsets, excl_neighbors, excl_n, rigid_body_id))
						continue;
					if (pairs && count < max_pairs) {
						pairs[2 * count] = a < bb ? a : bb;
						pairs[2 * count + 1] = a < bb ? bb : a;
					}
					if (checksum)
						sum += or_pair_hash(a, bb);
					++count;
				}
			}
		}
	}
	if (checksum)
		*checksum = sum;
	return count;
}

/* Order-independent pair identity: splitmix64 of (min << 32 | max). */
uint64_t or_pair_hash(int a, int b) {
	uint64_t z = ((uint64_t)(uint32_t)(a < b ? a : b) << 32) | (uint32_t)(a < b ? b : a);
	z += 0x9E3779B97F4A7C15ULL;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

/* The whole build (ZOrderPairlist::build_pairlist, ZOrderPairlist.cpp:102-178;
 * find_neighbors_zorder, :208-366): domain, encode, sort, gather, grid
 * choice, ranges, stencil, walk. The pair buffer cap used by the grid choice
 * is max(max_pairs, n) pairs. Returns the pair count and, if asked, the sum
 * of or_pair_hash over all pairs (mod 2^64). */
uint64_t or_build_pairlist(const float* pos4, size_t n, const or_box* b, float rc_list,
                           const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                           const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                           uint64_t* checksum) {
	return or_build_pairlist_m(pos4, n, b, rc_list, excl_offsets, excl_neighbors, excl_n,
	                           rigid_body_id, pairs, max_pairs, checksum, -1);
}

/* As or_build_pairlist, with the cell level m forced (m_force >= 0) instead of
 * the reference's choice; the stencil radii follow the reference's rule for
 * that m (ZOrderPairlist.cpp:48-56). The pair set does not depend on m. */
uint64_t or_build_pairlist_m(const float* pos4, size_t n, const or_box* b, float rc_list,
                             const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                             const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                             uint64_t* checksum, int m_force) {
	if (n == 0) {
		if (checksum)
			*checksum = 0;
		return 0;
	}
	float bmin[3], bmax[3], extent[3], box_len[3];
	or_morton_domain(b, pos4, n, bmin, bmax);
	for (int a = 0; a < 3; ++a) {
		extent[a] = bmax[a] - bmin[a];
		box_len[a] = b->periodic[a] ? b->size[a] : 0.0f;
	}
	uint32_t* keys = (uint32_t*)malloc(n * 4);
	uint32_t* s2o = (uint32_t*)malloc(n * 4);
	float* spos = (float*)malloc(n * 16);
	or_morton_encode(pos4, n, bmin, bmax, keys, s2o);
	or_sort_pairs(keys, s2o, n);
	or_gather4(pos4, spos, s2o, n);
	const float cutoff_sq = rc_list * rc_list;
	const float cutoff = sqrtf(cutoff_sq);
	int m, radii[3], slots;
	/* The pair-buffer guard in the grid choice never binds for a grown buffer
	 * (ZOrderPairlist.h:170-177); pass an effectively unbounded capacity. */
	or_select_cell_grid(extent, cutoff, n, (size_t)1 << 40, &m, radii, &slots);
	if (m_force >= 0) {
		m = m_force;
		slots = 1;
		for (int a = 0; a < 3; ++a) {
			const long long cells = 1LL << m;
			const double side = (double)extent[a] / (double)cells;
			radii[a] = (int)ceil((double)cutoff / side);
			long long span = 2LL * radii[a] + 1LL;
			if (span > cells)
				span = cells;
			slots *= (int)span;
		}
	}
	const size_t num_cells = (size_t)1 << (3 * m);
	const int shift = 3 * (10 - m);
	uint32_t* begin = (uint32_t*)calloc(num_cells, 4);
	uint32_t* end = (uint32_t*)calloc(num_cells, 4);
	uint32_t* table = (uint32_t*)malloc(num_cells * (size_t)slots * 4);
	or_cell_ranges(keys, n, shift, begin, end);
	or_cell_neighbors(table, m, radii, slots, box_len);
	const uint64_t count =
	    or_neighbor_walk(spos, keys, s2o, begin, end, table, slots, shift, cutoff_sq, n, b,
	                     excl_offsets, excl_neighbors, excl_n, rigid_body_id, pairs, max_pairs,
	                     checksum);
	free(keys);
	free(s2o);
	free(spos);
	free(begin);
	free(end);
	free(table);
	return count;
}

/* Exclusion CSR (src/Interactions/DeviceBondedInteraction.h:112-166):
 * canonicalise each pair to (a < b), sort, count both endpoints, prefix-sum,
 * scatter partners. `offsets` holds max_index + 2 ints, `neighbors` 2 * n. */
static int cmp_pair(const void* x, const void* y) {
	const int* p = (const int*)x;
	const int* q = (const int*)y;
	if (p[0] != q[0])
		return p[0] < q[0] ? -1 : 1;
	if (p[1] != q[1])
		return p[1] < q[1] ? -1 : 1;
	return 0;
}

int or_exclusion_csr(const int* pairs, size_t n_pairs, int* offsets, int* neighbors,
                     size_t* n_excl_particles) {
	int* canon = (int*)malloc(2 * n_pairs * sizeof(int) + 8);
	int max_idx = 0;
	for (size_t i = 0; i < n_pairs; ++i) {
		int a = pairs[2 * i], b = pairs[2 * i + 1];
		if (a > b) {
			const int t = a; a = b; b = t;
		}
		canon[2 * i] = a;
		canon[2 * i + 1] = b;
		if (b > max_idx)
			max_idx = b;
	}
	qsort(canon, n_pairs, 2 * sizeof(int), cmp_pair);
	const size_t np = (size_t)max_idx + 1;
	memset(offsets, 0, (np + 1) * sizeof(int));
	for (size_t i = 0; i < n_pairs; ++i) {
		offsets[canon[2 * i] + 1]++;
		offsets[canon[2 * i + 1] + 1]++;
	}
	for (size_t p = 0; p < np; ++p)
		offsets[p + 1] += offsets[p];
	int* cursor = (int*)malloc(np * sizeof(int) + 4);
	memcpy(cursor, offsets, np * sizeof(int));
	for (size_t i = 0; i < n_pairs; ++i) {
		const int a = canon[2 * i], b = canon[2 * i + 1];
		neighbors[cursor[a]++] = b;
		neighbors[cursor[b]++] = a;
	}
	free(cursor);
	free(canon);
	*n_excl_particles = n_pairs ? np : 0;
	return 0;
}

/* DisplacementKernel::min_image + operator() (src/PatchOperation/ZOrderKernels/
 * AdaptiveKernels.h:56-81) and the sqrt of ZOrderSort::compute_max_displacement
 * (ZOrderSort.cpp:173-198). */
static float min_image(float d, float l) {
	if (l <= 0.0f)
		return d;
	while (d > 0.5f * l)
		d -= l;
	while (d < -0.5f * l)
		d += l;
	return d;
}

float or_max_displacement(const float* cur4, const float* prev4, size_t n, const float* box_len) {
	float max_sq = 0.0f;
	for (size_t i = 0; i < n; ++i) {
		float dr[3];
		for (int a = 0; a < 3; ++a)
			dr[a] = min_image(cur4[4 * i + a] - prev4[4 * i + a], box_len[a]);
		const float d2 = len2(dr);
		if (d2 > max_sq)
			max_sq = d2;
	}
	return sqrtf(max_sq);
}

/* ------------------------------------------------------------------------ */
/* Forces                                                                   */
/* ------------------------------------------------------------------------ */

/* TabulatedPotential::compute (src/Interactions/TabulatedPotential.h:19-52). */
void or_table_lookup(const or_table* t, float x, float* force, float* energy) {
	float w = (x - t->start) * t->step_inv;
	int home = (int)floorf(w);
	w = w - (float)home;
	const int size = (int)t->size;
	if (t->is_periodic) {
		home %= size;
		if (home < 0)
			home += size;
	} else {
		if (home >= size - 1) {
			*force = 0.0f;
			*energy = t->pot[size - 1];
			return;
		}
		if (home < 0)
			home = 0;
	}
	int home1 = t->is_periodic ? (home + 1) % size : home + 1;
	if (!t->is_periodic && home1 >= size)
		home1 = size - 1;
	const float u0 = t->pot[home];
	const float du = t->pot[home1] - u0;
	*force = -du * t->step_inv;
	*energy = du * w + u0;
}

/* ResolvePairTableKernel (src/Interactions/Nonbonded/Pairwise.h:104-120). */
void or_resolve_tags(const int* pairs, size_t n_pairs, const int* type_ids,
                     const uint32_t* term_matrix, int num_types, uint32_t* tags) {
	for (size_t p = 0; p < n_pairs; ++p)
		tags[p] = term_matrix[type_ids[pairs[2 * p]] * num_types + type_ids[pairs[2 * p + 1]]];
}

/* CalcDistance::compute (src/Interactions/Interactions.h:37-51): wrapped r_ij,
 * |r_ij| by sqrtf, unit = r_ij * (1/|r_ij|) when |r_ij| > 1e-6. */
static float calc_distance(const or_box* b, const float* from, const float* to, float* r,
                           float* unit) {
	const float d[3] = {to[0] - from[0], to[1] - from[1], to[2] - from[2]};
	box_wrap_diff(b, d, r);
	const float dist = sqrtf(len2(r));
	if (dist > 1e-6f) {
		const float inv = 1.0f / dist;
		unit[0] = inv * r[0];
		unit[1] = inv * r[1];
		unit[2] = inv * r[2];
	} else {
		unit[0] = unit[1] = unit[2] = 0.0f;
	}
	return dist;
}

static void accumulate(float* fe4, double* fe64, double* fabs_sum, int p, float fx, float fy,
                       float fz, float e, int get_energy) {
	if (fe4) {
		fe4[4 * p] += fx;
		fe4[4 * p + 1] += fy;
		fe4[4 * p + 2] += fz;
		if (get_energy)
			fe4[4 * p + 3] += e;
	}
	if (fe64) {
		fe64[4 * p] += fx;
		fe64[4 * p + 1] += fy;
		fe64[4 * p + 2] += fz;
		if (get_energy)
			fe64[4 * p + 3] += e;
	}
	if (fabs_sum)
		fabs_sum[p] += sqrt((double)fx * fx + (double)fy * fy + (double)fz * fz);
}

/* PairNonbondedComputer::operator() with only the tabulated term
 * (src/Interactions/Nonbonded/Pairwise.h:214-304): skip untagged pairs, pairs
 * closer than 1e-6 and pairs with d*d > rc^2; F = unit * F_table; -F to the
 * first index, +F to the second; half the energy to each. Float accumulation
 * (fe4) runs in pair order; fe64/fabs_sum receive the same per-pair float
 * contributions summed in double, plus the sum of |f| per particle. */
void or_pair_forces(const int* pairs, size_t n_pairs, const float* pos4, const uint32_t* tags,
                    const or_table* tables, const or_box* b, float cutoff_sq, int get_energy,
                    float* fe4, double* fe64, double* fabs_sum) {
	for (size_t p = 0; p < n_pairs; ++p) {
		const uint32_t tag = tags ? tags[p] : 32u;
		if (!(tag & 32u))
			continue;
		const int i = pairs[2 * p], j = pairs[2 * p + 1];
		float r[3], u[3];
		const float d = calc_distance(b, pos4 + 4 * i, pos4 + 4 * j, r, u);
		if (d < 1e-6f)
			continue;
		if (cutoff_sq > 0.0f && d * d > cutoff_sq)
			continue;
		float fm, e;
		or_table_lookup(&tables[tag >> 8], d, &fm, &e);
		const float fm_total = 0.0f + fm;
		const float e_total = 0.0f + e;
		const float f[3] = {u[0] * fm_total, u[1] * fm_total, u[2] * fm_total};
		const float half = e_total * 0.5f;
		accumulate(fe4, fe64, fabs_sum, i, -f[0], -f[1], -f[2], half, get_energy);
		accumulate(fe4, fe64, fabs_sum, j, f[0], f[1], f[2], half, get_energy);
	}
}

/* FP64 re-evaluation of the tabulated pair energy (same formulas as
 * or_pair_forces, every operation in double). */
double or_pair_energy_f64(const int* pairs, size_t n_pairs, const float* pos4,
                          const uint32_t* tags, const or_table* tables, const or_box* b,
                          float cutoff_sq) {
	double total = 0.0;
	for (size_t p = 0; p < n_pairs; ++p) {
		const uint32_t tag = tags ? tags[p] : 32u;
		if (!(tag & 32u))
			continue;
		const int i = pairs[2 * p], j = pairs[2 * p + 1];
		double r2 = 0.0;
		for (int a = 0; a < 3; ++a) {
			double x = (double)pos4[4 * j + a] - (double)pos4[4 * i + a];
			if (b->periodic[a]) {
				const double l = b->size[a];
				x -= floor(x / l) * l;
				if (x >= 0.5 * l)
					x -= l;
			}
			r2 += x * x;
		}
		const double d = sqrt(r2);
		if (d < 1e-6 || (cutoff_sq > 0.0f && d * d > (double)cutoff_sq))
			continue;
		const or_table* t = &tables[tag >> 8];
		double w = (d - (double)t->start) * (double)t->step_inv;
		int home = (int)floor(w);
		w -= home;
		double e;
		if (home >= (int)t->size - 1) {
			e = t->pot[t->size - 1];
		} else {
			if (home < 0)
				home = 0;
			const double u0 = t->pot[home];
			e = ((double)t->pot[home + 1] - u0) * w + u0;
		}
		total += e;
	}
	return total;
}

/* TabulatedBondComputer::operator() (src/Interactions/Bonded/BondComputer.h:168-191);
 * rows with table_idx < 0 (a form other than tabulated) are skipped. */
void or_bond_forces(const int* bonds, const int* table_idx, size_t nb, const float* pos4,
                    const or_table* tables, const or_box* b, int get_energy, float* fe4,
                    double* fe64, double* fabs_sum) {
	for (size_t k = 0; k < nb; ++k) {
		if (table_idx[k] < 0)
			continue;
		const int i = bonds[2 * k], j = bonds[2 * k + 1];
		float r[3], u[3];
		const float d = calc_distance(b, pos4 + 4 * i, pos4 + 4 * j, r, u);
		if (d < 1e-6f)
			continue;
		float fm, e;
		or_table_lookup(&tables[table_idx[k]], d, &fm, &e);
		const float f[3] = {u[0] * fm, u[1] * fm, u[2] * fm};
		const float half = e * 0.5f;
		accumulate(fe4, fe64, fabs_sum, i, -f[0], -f[1], -f[2], half, get_energy);
		accumulate(fe4, fe64, fabs_sum, j, f[0], f[1], f[2], half, get_energy);
	}
}

/* TabulatedAngleComputer::operator() (BondComputer.h:236-268) with
 * AngleGeometry::compute (src/Interactions/Bonded/BondGeometry.h:19-44).
 * Angle tables wrap (src/Interactions/DeviceBondedInteraction.h:234). The
 * reference's host build evaluates acos of the float cosine in double and
 * rounds to float (pinned bit-exactly against its host-compiled functor). */
void or_angle_forces(const int* angles4, const int* table_idx, size_t na, const float* pos4,
                     const or_table* tables, const or_box* b, int get_energy, float* fe4,
                     double* fe64, double* fabs_sum) {
	for (size_t k = 0; k < na; ++k) {
		if (table_idx[k] < 0)
			continue;
		const int i = angles4[4 * k], j = angles4[4 * k + 1], l = angles4[4 * k + 2];
		const float* pi = pos4 + 4 * i;
		const float* pj = pos4 + 4 * j;
		const float* pl = pos4 + 4 * l;
		float ab[3], bc[3], ac[3];
		const float dab[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
		const float dbc[3] = {pl[0] - pj[0], pl[1] - pj[1], pl[2] - pj[2]};
		const float dac[3] = {pl[0] - pi[0], pl[1] - pi[1], pl[2] - pi[2]};
		box_wrap_diff(b, dab, ab);
		box_wrap_diff(b, dbc, bc);
		box_wrap_diff(b, dac, ac);
		const float ab2 = len2(ab), bc2 = len2(bc), ac2 = len2(ac);
		float cs = (ab2 + bc2 - ac2) * 0.5f / (sqrtf(ab2) * sqrtf(bc2));
		if (cs < -1.0f)
			cs = -1.0f;
		if (cs > 1.0f)
			cs = 1.0f;
		const float angle = (float)acos((double)cs);
		const float sn = sqrtf(1.0f - cs * cs);
		float fm, e;
		or_table_lookup(&tables[table_idx[k]], angle, &fm, &e);
		const float sin_angle = sn > 1e-3f ? sn : 1e-3f;
		const float dudt = -fm / sin_angle;
		const float inv_ab = 1.0f / sqrtf(len2(ab));
		const float inv_bc = 1.0f / sqrtf(len2(bc));
		const float s1 = dudt * inv_ab;
		const float c_ab = cs * inv_ab;
		const float s3 = -(dudt * inv_bc);
		const float c_bc = cs * inv_bc;
		float f1[3], f3[3];
		for (int a = 0; a < 3; ++a) {
			f1[a] = s1 * (ab[a] * c_ab + bc[a] * inv_bc);
			f3[a] = s3 * (bc[a] * c_bc + ab[a] * inv_ab);
		}
		const float third = (float)(1.0 / 3.0);
		const float en = e * third;
		accumulate(fe4, fe64, fabs_sum, i, f1[0], f1[1], f1[2], en, get_energy);
		accumulate(fe4, fe64, fabs_sum, j, -(f1[0] + f3[0]), -(f1[1] + f3[1]), -(f1[2] + f3[2]),
		           en, get_energy);
		accumulate(fe4, fe64, fabs_sum, l, f3[0], f3[1], f3[2], en, get_energy);
	}
}

/* --- analytical pair terms ----------------------------------------------- */

#define OR_COULOMB 332.0636f /* constants::COULOMB (src/Constants.h:24) */

/* math::sinh_minus_x / x_cosh_minus_sinh (src/Types/Math.h:199-216): the
 * series below |x| = 1, the direct difference above. */
static float sinh_minus_x(float x) {
	if (x >= 1.0f || x <= -1.0f)
		return sinhf(x) - x;
	const float w = x * x;
	return x * w *
	       ((float)(1.0 / 6) +
	        w * ((float)(1.0 / 120) + w * ((float)(1.0 / 5040) + w * (float)(1.0 / 362880))));
}

static float x_cosh_minus_sinh(float x) {
	if (x >= 1.0f || x <= -1.0f)
		return x * coshf(x) - sinhf(x);
	const float w = x * x;
	return x * w *
	       ((float)(1.0 / 3) +
	        w * ((float)(1.0 / 30) + w * ((float)(1.0 / 840) + w * (float)(1.0 / 45360))));
}

/* OnckElecPotential::dielectric / dielectric_deriv (Columb.h:68-84). */
static float onck_dielectric(float r, float sz, float z) {
	const float v = r / (2.0f * z);
	if (v < 1e-5f)
		return sz * v * v / 3.0f;
	const float s = sinhf(v);
	return sz * sinh_minus_x(v) * (s + v) / (s * s);
}

static float onck_dielectric_deriv(float r, float sz, float z) {
	const float v = r / (2.0f * z);
	if (v < 1e-5f)
		return sz * v / (3.0f * z);
	const float s = sinhf(v);
	return sz * v * x_cosh_minus_sinh(v) / (z * s * s * s);
}

/* PairNonbondedComputer::operator() (src/Interactions/Nonbonded/Pairwise.h:214-304)
 * with every term: Coulomb (ColumbPotential, Columb.h:11-20), Debye-Hueckel
 * (Columb.h:29-42), Onck (Columb.h:56-97), Gaussian (Pairwise.h:50-69),
 * softcore (SoftcoreForceKernel::softcoreForce, Pairwise.h:82-100, converted
 * to -dU/dr by -F * r) and tabulated, summed in that order; F = unit * sum,
 * -F to the first index, half the energy to each. tags[p] carries the term
 * bits (bit 0..5) and the table index (>> 8). */
void or_pair_forces_terms(const int* pairs, size_t n_pairs, const float* pos4,
                          const int* type_ids, const uint32_t* tags, const or_table* tables,
                          const or_pair_terms* pt, const or_box* b, float cutoff_sq,
                          int get_energy, float* fe4, double* fe64, double* fabs_sum) {
	for (size_t p = 0; p < n_pairs; ++p) {
		const uint32_t tag = tags[p];
		const uint32_t terms = tag & pt->enabled_terms;
		if ((terms & 0xFFu) == 0)
			continue;
		const int i = pairs[2 * p], j = pairs[2 * p + 1];
		float r[3], u[3];
		const float d = calc_distance(b, pos4 + 4 * i, pos4 + 4 * j, r, u);
		if (d < 1e-6f)
			continue;
		if (cutoff_sq > 0.0f && d * d > cutoff_sq)
			continue;
		const int ti = type_ids[i], tj = type_ids[j];
		float qi = 0.0f, qj = 0.0f;
		if (terms & 7u) {
			qi = pt->charge[ti];
			qj = pt->charge[tj];
		}
		float fm = 0.0f, en = 0.0f;
		if (terms & 1u) { /* Coulomb */
			const float inv_d2 = 1.0f / (d * d);
			const float inv_d = 1.0f / d;
			fm += qi * qj * inv_d2 * OR_COULOMB;
			en += qi * qj * inv_d * OR_COULOMB;
		}
		if (terms & 2u) { /* Debye-Hueckel */
			const float inv_r = 1.0f / d;
			const float a = qi * qj * OR_COULOMB / pt->dielectric;
			const float screen = expf(-d / pt->debye_length);
			const float e = a * screen * inv_r;
			fm += e * (inv_r + 1.0f / pt->debye_length);
			en += e;
		}
		if (terms & 4u) { /* Onck */
			const float rr = d < 1e-2f ? 1e-2f : d;
			const float a = qi * qj * OR_COULOMB;
			const float screen = expf(-pt->onck_kappa * rr);
			const float eps = onck_dielectric(rr, pt->onck_sz, pt->onck_z);
			const float e = a * screen / (eps * rr);
			const float eps_p = onck_dielectric_deriv(rr, pt->onck_sz, pt->onck_z);
			fm += a * screen * (pt->onck_kappa / (eps * rr) + (eps_p * rr + eps) / (eps * eps * rr * rr));
			en += e;
		}
		if (terms & 8u) { /* Gaussian */
			const float d2 = d * d;
			if (!(pt->gaussian_cutoff_sq > 0.0f && d2 > pt->gaussian_cutoff_sq)) {
				const float inv_s2 = 1.0f / (pt->gaussian_sigma * pt->gaussian_sigma);
				const float e = pt->gaussian_amp * expf(-d2 * inv_s2);
				fm += 2.0f * d * e * inv_s2;
				en += e;
			}
		}
		if (terms & 16u) { /* softcore */
			const float rad = 0.5f * (pt->radius[ti] + pt->radius[tj]);
			const float rad2 = rad * rad;
			const float rad6 = rad2 * rad2 * rad2;
			const float eps = sqrtf(pt->eps[ti] * pt->eps[tj]);
			const float d2 = len2(r);
			const float d6 = d2 * d2 * d2;
			float f, e;
			if (d6 < rad6) {
				const float d6_2 = d6 * d6;
				const float rad6_2 = rad6 * rad6;
				e = eps * ((rad6_2 / d6_2) - (2.0f * rad6 / d6)) + eps;
				f = -12.0f * eps * (rad6_2 / (d6_2 * d2) - rad6 / (d6 * d2));
			} else {
				f = -12.0f * eps * (rad6 * rad6 / (d6 * d6 * d2) - rad6 / (d6 * d2));
				e = 0.0f;
			}
			fm += -f * d;
			en += e;
		}
		if (terms & 32u) { /* tabulated */
			float tf, te;
			or_table_lookup(&tables[tag >> 8], d, &tf, &te);
			fm += tf;
			en += te;
		}
		const float f[3] = {u[0] * fm, u[1] * fm, u[2] * fm};
		const float half = en * 0.5f;
		accumulate(fe4, fe64, fabs_sum, i, -f[0], -f[1], -f[2], half, get_energy);
		accumulate(fe4, fe64, fabs_sum, j, f[0], f[1], f[2], half, get_energy);
	}
}

/* --- dihedrals and restraints --------------------------------------------- */

static void cross3(const float* a, const float* b, float* out) {
	out[0] = a[1] * b[2] - a[2] * b[1];
	out[1] = a[2] * b[0] - a[0] * b[2];
	out[2] = a[0] * b[1] - a[1] * b[0];
}

static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static float rlen2(const float* a) {
	const float l2 = len2(a);
	return l2 != 0.0f ? 1.0f / l2 : 0.0f;
}

/* TabulatedDihedralComputer::operator() (src/Interactions/Bonded/BondComputer.h:304-345)
 * with DihedralGeometry::compute (src/Interactions/Bonded/BondGeometry.h:62-86):
 * phi = atan2(sin, cos) from the two plane normals; periodic table; force
 * magnitude 0 when degenerate, clamped to +-1000; a quarter of the energy to
 * each of the four particles. Rows of table_idx < 0 are skipped (a form other
 * than tabulated). */
void or_dihedral_forces(const int* dihedrals4, const int* table_idx, size_t nd,
                        const float* pos4, const or_table* tables, const or_box* b,
                        int get_energy, float* fe4, double* fe64, double* fabs_sum) {
	for (size_t k = 0; k < nd; ++k) {
		if (table_idx[k] < 0)
			continue;
		const int* q = dihedrals4 + 4 * k;
		float ab[3], bc[3], cd[3];
		const float* p0 = pos4 + 4 * q[0];
		const float* p1 = pos4 + 4 * q[1];
		const float* p2 = pos4 + 4 * q[2];
		const float* p3 = pos4 + 4 * q[3];
		const float d01[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
		const float d12[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
		const float d23[3] = {p3[0] - p2[0], p3[1] - p2[1], p3[2] - p2[2]};
		box_wrap_diff(b, d01, ab);
		box_wrap_diff(b, d12, bc);
		box_wrap_diff(b, d23, cd);
		float c_abc[3], c_bcd[3], c_x[3];
		cross3(ab, bc, c_abc);
		cross3(bc, cd, c_bcd);
		cross3(bc, c_abc, c_x);
		const float cos_phi = dot3(c_abc, c_bcd) / (sqrtf(len2(c_abc)) * sqrtf(len2(c_bcd)));
		const float sin_phi = dot3(c_x, c_bcd) / (sqrtf(len2(c_x)) * sqrtf(len2(c_bcd)));
		const float phi = (float)atan2((double)sin_phi, (double)cos_phi);
		const float lbc = sqrtf(len2(bc));
		const float s1 = -lbc * rlen2(c_abc);
		const float s3 = -lbc * rlen2(c_bcd);
		float f1[3], f2[3], f3[3];
		for (int a = 0; a < 3; ++a) {
			f1[a] = c_abc[a] * s1;
			f3[a] = c_bcd[a] * s3;
		}
		const float g1 = -(dot3(ab, bc) * rlen2(bc));
		const float g3 = dot3(bc, cd) * rlen2(bc);
		for (int a = 0; a < 3; ++a)
			f2[a] = f1[a] * g1 - f3[a] * g3;
		const int degenerate = (len2(ab) * len2(bc) * rlen2(c_abc) > 100.0f) ||
		                       (len2(bc) * len2(cd) * rlen2(c_bcd) > 100.0f);
		float fm, e;
		or_table_lookup(&tables[table_idx[k]], phi, &fm, &e);
		float mag = degenerate ? 0.0f : fm;
		if (mag > 1000.0f)
			mag = 1000.0f;
		else if (mag < -1000.0f)
			mag = -1000.0f;
		float v1[3], v2[3], v3[3];
		for (int a = 0; a < 3; ++a) {
			v1[a] = f1[a] * mag;
			v2[a] = f2[a] * mag;
			v3[a] = f3[a] * mag;
		}
		const float quarter = e * 0.25f;
		accumulate(fe4, fe64, fabs_sum, q[0], v1[0], v1[1], v1[2], quarter, get_energy);
		accumulate(fe4, fe64, fabs_sum, q[1], v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2], quarter,
		           get_energy);
		accumulate(fe4, fe64, fabs_sum, q[2], v3[0] - v2[0], v3[1] - v2[1], v3[2] - v2[2], quarter,
		           get_energy);
		accumulate(fe4, fe64, fabs_sum, q[3], -v3[0], -v3[1], -v3[2], quarter, get_energy);
	}
}

/* HarmonicRestraintComputer::operator() (src/Interactions/Bonded/BondComputer.h:110-130):
 * r = wrap_diff(pos - anchor), F = unit * (-k |r|), full energy 0.5 k |r|^2 to
 * the particle; ids < 0 are skipped. anchors4: x, y, z, pad per restraint. */
void or_restraint_forces(const int* ids, const float* anchors4, const float* k_spring, size_t nr,
                         const float* pos4, const or_box* b, int get_energy, float* fe4,
                         double* fe64, double* fabs_sum) {
	for (size_t k = 0; k < nr; ++k) {
		const int id = ids[k];
		if (id < 0)
			continue;
		float r[3], u[3];
		const float d = calc_distance(b, anchors4 + 4 * k, pos4 + 4 * id, r, u);
		const float kk = k_spring[k];
		const float fm = -kk * (d - 0.0f);
		const float e = 0.5f * kk * (d - 0.0f) * (d - 0.0f);
		accumulate(fe4, fe64, fabs_sum, id, fm * u[0], fm * u[1], fm * u[2], e, get_energy);
	}
}

/* ------------------------------------------------------------------------ */
/* Grid, Philox, BD                                                         */
/* ------------------------------------------------------------------------ */

/* map_grid_index + fetch_grid_value (src/Types/BaseGridDevice.h:218-250). */
static int map_index(int* j, int64_t n, int bc) {
	const int ni = (int)n;
	if (*j >= 0 && *j < ni)
		return 1;
	if (bc == 2) {
		*j = ((*j % ni) + ni) % ni;
		return 1;
	}
	if (bc == 1) {
		*j = *j < 0 ? 0 : ni - 1;
		return 1;
	}
	return 0;
}

static float fetch(const or_grid* g, int jx, int jy, int jz, int bc) {
	if (!map_index(&jx, g->dims[0], bc) || !map_index(&jy, g->dims[1], bc) ||
	    !map_index(&jz, g->dims[2], bc))
		return 0.0f;
	const size_t idx = (size_t)jz + (size_t)jy * (size_t)g->dims[2] +
	                   (size_t)jx * (size_t)g->dims[1] * (size_t)g->dims[2];
	return g->data[idx];
}

/* Matrix3::transform, column-major (src/Types/Matrix3.h:74-76). */
static void mat_transform(const float* m, const float* v, float* out) {
	for (int r = 0; r < 3; ++r)
		out[r] = v[0] * m[r] + v[1] * m[3 + r] + v[2] * m[6 + r];
}

static void grid_taps(const or_grid* g, const float* pos, int bc, float* t, float* f) {
	const float d[3] = {pos[0] - g->origin[0], pos[1] - g->origin[1], pos[2] - g->origin[2]};
	float gp[3];
	mat_transform(g->basis_inv, d, gp);
	int i0[3];
	for (int a = 0; a < 3; ++a) {
		i0[a] = (int)floorf(gp[a]);
		f[a] = gp[a] - (float)i0[a];
	}
	t[0] = fetch(g, i0[0], i0[1], i0[2], bc);
	t[1] = fetch(g, i0[0], i0[1], i0[2] + 1, bc);
	t[2] = fetch(g, i0[0], i0[1] + 1, i0[2], bc);
	t[3] = fetch(g, i0[0], i0[1] + 1, i0[2] + 1, bc);
	t[4] = fetch(g, i0[0] + 1, i0[1], i0[2], bc);
	t[5] = fetch(g, i0[0] + 1, i0[1], i0[2] + 1, bc);
	t[6] = fetch(g, i0[0] + 1, i0[1] + 1, i0[2], bc);
	t[7] = fetch(g, i0[0] + 1, i0[1] + 1, i0[2] + 1, bc);
}

/* interpolate_grid_point (BaseGridDevice.h:256-299). Taps t[] are ordered
 * v000, v001, v010, v011, v100, v101, v110, v111. */
float or_grid_value(const or_grid* g, const float* pos, int bc) {
	float t[8], f[3];
	grid_taps(g, pos, bc, t, f);
	const float fx = f[0], fy = f[1], fz = f[2];
	const float v00 = t[0] * (1.0f - fx) + t[4] * fx;
	const float v01 = t[1] * (1.0f - fx) + t[5] * fx;
	const float v10 = t[2] * (1.0f - fx) + t[6] * fx;
	const float v11 = t[3] * (1.0f - fx) + t[7] * fx;
	const float v0 = v00 * (1.0f - fy) + v10 * fy;
	const float v1 = v01 * (1.0f - fy) + v11 * fy;
	return v0 * (1.0f - fz) + v1 * fz;
}

/* compute_gradient (BaseGridDevice.h:327-365): analytic gradient of the
 * trilinear interpolant, mapped back by basis_inv^T. */
void or_grid_gradient(const or_grid* g, const float* pos, int bc, float* grad) {
	float t[8], f[3];
	grid_taps(g, pos, bc, t, f);
	const float fx = f[0], fy = f[1], fz = f[2];
	const float gx = (1.0f - fy) * (1.0f - fz) * (t[4] - t[0]) + fy * (1.0f - fz) * (t[6] - t[2]) +
	                 (1.0f - fy) * fz * (t[5] - t[1]) + fy * fz * (t[7] - t[3]);
	const float gy = (1.0f - fx) * (1.0f - fz) * (t[2] - t[0]) + fx * (1.0f - fz) * (t[6] - t[4]) +
	                 (1.0f - fx) * fz * (t[3] - t[1]) + fx * fz * (t[7] - t[5]);
	const float gz = (1.0f - fx) * (1.0f - fy) * (t[1] - t[0]) + fx * (1.0f - fy) * (t[5] - t[4]) +
	                 (1.0f - fx) * fy * (t[3] - t[2]) + fx * fy * (t[7] - t[6]);
	/* transpose(basis_inv).transform(g): row r of basis_inv dotted with g */
	const float* m = g->basis_inv;
	for (int r = 0; r < 3; ++r)
		grad[r] = gx * m[3 * r] + gy * m[3 * r + 1] + gz * m[3 * r + 2];
}

/* compute_position_dependent_force (src/Interactions/Nonbonded/Pmf.h:68-124):
 * q E, then each valid PMF term adds -scale * grad U to the force and
 * scale * U to .t; then per-axis force grids. */
void or_position_force(const float* pos, int type, const or_types* ty, const or_grid* grids,
                       const float* efield, float* force4) {
	const float q = ty->charge[type];
	force4[0] = q * efield[0];
	force4[1] = q * efield[1];
	force4[2] = q * efield[2];
	force4[3] = 0.0f;
	if (!grids)
		return;
	const int begin = ty->pmf_offset[type];
	const int end = begin + ty->pmf_count[type];
	for (int k = begin; k < end; ++k) {
		const or_grid_term term = ty->terms[k];
		if (term.grid_id < 0)
			continue;
		const or_grid* g = &grids[term.grid_id];
		if (!g->data)
			continue;
		const int bc = term.boundary_condition >= 0 ? term.boundary_condition
		                                            : g->boundary_condition;
		const float value = or_grid_value(g, pos, bc);
		float grad[3];
		or_grid_gradient(g, pos, bc, grad);
		const float s = -term.scale;
		force4[0] += grad[0] * s;
		force4[1] += grad[1] * s;
		force4[2] += grad[2] * s;
		force4[3] += term.scale * value;
	}
	for (int a = 0; a < 3; ++a) {
		const int gid = ty->force_grid_id4[4 * type + a];
		if (gid >= 0 && grids[gid].data)
			force4[a] += ty->force_grid_scale4[4 * type + a] *
			             or_grid_value(&grids[gid], pos, grids[gid].boundary_condition);
	}
}

/* openrand::Philox::generate + round (src/PatchOperation/Random/philox.h:97-139):
 * Philox4x32 with 10 rounds; key (seed_hi, seed_lo) bumped by
 * (0x9E3779B9, 0xBB67AE85) before every round after the first. */
void or_philox4x32_10(uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2,
                      uint32_t internal, uint32_t* out) {
	uint32_t k0 = (uint32_t)(seed >> 32), k1 = (uint32_t)(seed & 0xFFFFFFFFu);
	uint32_t c[4] = {ctr0, ctr1, ctr2, internal};
	for (int r = 0; r < 10; ++r) {
		if (r > 0) {
			k0 += 0x9E3779B9u;
			k1 += 0xBB67AE85u;
		}
		const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
		const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
		const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
		const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
		c[0] = hi1 ^ c[1] ^ k0;
		c[1] = lo1;
		c[2] = hi0 ^ c[3] ^ k1;
		c[3] = lo0;
	}
	memcpy(out, c, 16);
}

/* BaseRNG::u01<float, uint32_t> (src/PatchOperation/Random/base_state.h:299-305). */
float or_u01(uint32_t x) {
	const float factor = 1.0f / (4294967295.0f + 1.0f);
	const float half = 0.5f * factor;
	return (float)x * factor + half;
}

/* Patch::integrate_motion seed mixing (src/PatchOperation/Patch.cpp:252-254). */
uint64_t or_bd_seed(uint64_t seed, uint64_t patch_id, uint64_t step) {
	return (seed * 0x9E3779B97F4A7C15ULL) ^ (patch_id << 32) ^ (step * 0xBF58476D1CE4E5B9ULL);
}

/* BDIntegrate<float>::operator() (src/PatchOperation/Integrator/BD.h:44-92):
 * skip rigid-body-attached particles; add the position-dependent force (its
 * energy to .t); Philox(key, base_ctr + idx, step, 0x5324120) -> 4 uniforms
 * -> Box-Muller -> x += (D/kT) F dt + sqrt(2 D dt) xi per axis; wrap. If
 * noise4 is given, the three normals of each particle are stored there. */
void or_bd_integrate(float* pos4, float* fe4, const int* type_ids, const uint32_t* flags, size_t n,
                     const or_types* types, const or_grid* grids, const or_box* b, float dt,
                     float kT, uint64_t step, uint64_t base_seed, uint32_t base_ctr,
                     const float* efield, float* noise4) {
	for (size_t i = 0; i < n; ++i) {
		if (flags && (flags[i] & 4u))
			continue;
		float* p = pos4 + 4 * i;
		const int type = type_ids[i];
		float pmf[4];
		or_position_force(p, type, types, grids, efield, pmf);
		float force[3] = {fe4[4 * i] + pmf[0], fe4[4 * i + 1] + pmf[1], fe4[4 * i + 2] + pmf[2]};
		fe4[4 * i + 3] += pmf[3];
		const float* dif = types->diffusion4 + 4 * type;
		uint32_t u[4];
		or_philox4x32_10(base_seed, base_ctr + (uint32_t)i, 0x5324120u, (uint32_t)step, 0u, u);
		const float ux = or_u01(u[0]), uy = or_u01(u[1]), uz = or_u01(u[2]), uw = or_u01(u[3]);
		const float r1 = sqrtf(-2.0f * logf(ux));
		const float theta1 = 2.0f * 3.1415926535f * uy;
		const float r2 = sqrtf(-2.0f * logf(uz));
		const float theta2 = 2.0f * 3.1415926535f * uw;
		const float xi[3] = {r1 * cosf(theta1), r1 * sinf(theta1), r2 * cosf(theta2)};
		if (noise4) {
			noise4[4 * i] = xi[0];
			noise4[4 * i + 1] = xi[1];
			noise4[4 * i + 2] = xi[2];
			noise4[4 * i + 3] = 0.0f;
		}
		for (int a = 0; a < 3; ++a)
			p[a] += (dif[a] / kT) * force[a] * dt + sqrtf(2.0f * dif[a] * dt) * xi[a];
		for (int a = 0; a < 3; ++a)
			if (b->periodic[a])
				p[a] = or_wrap_scalar(p[a], b->origin[a], b->size[a]);
	}
}

/* FORCE_CONVERSION_FACTOR and SQRT_CAL_TO_JOULE (src/Constants.h:30,34). */
#define OR_FORCE_CONVERSION 4.18679994e4f
#define OR_SQRT_CAL_TO_JOULE 2.046167337f

static void half_kick(float* m, const float* f, float dt) {
	const float h = 0.5f * dt;
	for (int a = 0; a < 3; ++a) m[a] = m[a] + (h * f[a]) * OR_FORCE_CONVERSION;
}

void or_baoab_integrate(float* pos4, float* mom4, float* fe4, const int* type_ids,
                        const uint32_t* flags, size_t n, const or_types* types,
                        const or_grid* grids, const float* mass, const float* damping3,
                        const or_box* b, float dt, float kT, uint64_t step, uint64_t base_seed,
                        uint32_t base_ctr, const float* efield, int pending) {
	if (grids)
		for (size_t i = 0; i < n; ++i) {
			float pmf[4];
			or_position_force(pos4 + 4 * i, type_ids[i], types, grids, efield, pmf);
			for (int a = 0; a < 4; ++a) fe4[4 * i + a] += pmf[a];
		}
	for (size_t i = 0; i < n; ++i) {
		if (flags && (flags[i] & 4u))
			continue;
		float* p = pos4 + 4 * i;
		float* m = mom4 + 4 * i;
		const float* f = fe4 + 4 * i;
		const int type = type_ids[i];
		const float ms = mass[type];
		const float* g = damping3 + 3 * type;
		if (pending) half_kick(m, f, dt);
		half_kick(m, f, dt); /* B */
		const float h = 0.5f * dt;
		/* Vector3 / s multiplies by 1 / s (Vector3.h:194-197). */
		const float inv_m = 1.0f / ms;
		for (int a = 0; a < 3; ++a) p[a] = p[a] + ((h * m[a]) * inv_m) * 10000.0f; /* A */
		uint32_t u[4];
		or_philox4x32_10(base_seed, base_ctr + (uint32_t)i, 0x1356914u, (uint32_t)step, 0u, u);
		const float ux = or_u01(u[0]), uy = or_u01(u[1]), uz = or_u01(u[2]), uw = or_u01(u[3]);
		const float r1 = sqrtf(-2.0f * logf(ux));
		const float theta1 = 2.0f * 3.1415926535f * uy;
		const float r2 = sqrtf(-2.0f * logf(uz));
		const float theta2 = 2.0f * 3.1415926535f * uw;
		const float xi[3] = {r1 * cosf(theta1), r1 * sinf(theta1), r2 * cosf(theta2)};
		for (int a = 0; a < 3; ++a) { /* O */
			const float c = expf(-g[a] * dt);
			const float ns = sqrtf(kT * ms * (1.0f - c * c)) * OR_SQRT_CAL_TO_JOULE;
			m[a] = c * m[a] + ns * xi[a];
		}
		for (int a = 0; a < 3; ++a) p[a] = p[a] + ((h * m[a]) * inv_m) * 10000.0f; /* A */
		for (int a = 0; a < 3; ++a)
			if (b->periodic[a])
				p[a] = or_wrap_scalar(p[a], b->origin[a], b->size[a]);
	}
}

void or_baoab_last_update(float* mom4, const float* fe4, const uint32_t* flags, size_t n,
                          float dt) {
	for (size_t i = 0; i < n; ++i) {
		if (flags && (flags[i] & 4u))
			continue;
		half_kick(mom4 + 4 * i, fe4 + 4 * i, dt);
	}
}
