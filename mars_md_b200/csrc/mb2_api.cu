// C ABI of libmarsb200.so: context, set-up, and one entry point per
// reference interface on the Brownian-dynamics path (see include/marsb200.h).
#include "../../include/marsb200.h"
#include "mb2_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

using namespace mb2;

namespace mb2 {
unsigned long long g_launches = 0;
}

// FP64 reduction slots: pair energy, pair virial, bond, angle, dihedral and
// restraint energy.
constexpr int kEnergySlots = 6;

struct mb2_context {
	int device = 0;
	uint32_t max_particles = 0;
	std::string last_error;

	Box box{};
	bool box_set = false;
	Scratch scratch;

	// Z-order state of the last build
	DevBuf<uint32_t> keys, s2o, inv, row_len, row_off, nbr, cell_begin, cell_end, row_far;
	DevBuf<float4> sorted_pos, ref_pos, force_sorted;
	// Displacement since the last build, tracked by the step's pack (the
	// pair kernel's inner rows): the build's Z-ordered positions, the squared
	// maximum as float bits, and the build's list radius (0: not tracked).
	DevBuf<float4> ref_sorted;
	DevBuf<unsigned int> d2max;
	float track_rc = 0.0f;
	DevBuf<StencilEntry> stencil;
	DevBuf<float> bbox;  // 6 floats, ordered-int min/max
	DevBuf<unsigned int> disp;
	DevBuf<unsigned long long> stats;  // build: pairs, longest row
	DevBuf<double> energy;  // pair E, pair virial, bond E, angle E
	uint64_t* pinned = nullptr;
	CellGrid grid;
	bool grid_valid = false;
	float grid_extent[3] = {0, 0, 0};
	float grid_rc = 0.0f;
	uint32_t grid_n = 0;
	bool built = false;
	uint32_t built_n = 0;
	uint64_t num_pairs = 0;
	uint32_t cap = 0;        // entries per row of the sliced-ELL list
	int lanes = 0;           // G: lanes per row in the pair kernel (slice height 32 / G)
	uint64_t max_row = 0;
	Exclusions excl;
	int lanes_request = 0;   // 0 = choose from the mean row length
	int level_offset = 0;    // cell level relative to the cost model's choice

	// pair tables
	PairTables pt;
	DevBuf<PairTableRef> refs;
	DevBuf<int> table_offsets;  // per type pair: offset of its table's bins, -1 none
	DevBuf<float> bin_force;
	DevBuf<float2> bin_energy;

	// analytical pair terms: the tag matrix as set, per-type constants, and
	// the per-type-pair table built from both
	std::vector<uint32_t> term_matrix_h;
	bool pair_terms_set = false;
	std::vector<float> term_charge, term_radius, term_eps;
	PairSolvent solvent{};
	float term_dielectric = 80.0f;
	DevBuf<PairTermRef> term_refs;

	// bonded tables: 0 bonds, 1 angles, 2 dihedrals
	DevBuf<Table> bonded_tables[3];
	DevBuf<float> bonded_values[3];
	int bonded_count[3] = {0, 0, 0};

	// particle types and grids
	TypeTable types;
	bool types_set = false;
	DevBuf<float> charge;
	DevBuf<float4> diffusion, fg_scale;
	DevBuf<int> pmf_off, pmf_cnt;
	DevBuf<GridTermDev> terms;
	DevBuf<int4> fg_id;
	std::vector<GridView> host_grids;
	DevBuf<GridView> grids;

	uint32_t bonded_bins[3] = {0, 0, 0};  // values in the bond / angle / dihedral tables
	DevBuf<uint32_t> ro_keys, ro_s2o, ro_inv;  // canonical reorder permutation
	DevBuf<float4> ro_tmp;
	uint32_t ro_n = 0;
	DevBuf<float> mass;                // Langevin: per-type mass
	DevBuf<float4> damping;            // Langevin: per-type damping (x, y, z)
	int langevin_types = 0;

	// Adjoint window: checkpoints of the forward window and reverse-sweep buffers.
	struct Window {
		bool valid = false;
		uint32_t n = 0, num_steps = 0, every = 0;
		uint64_t first_step = 0;
		mb2_step_params prm{};
		const int* type_ids = nullptr;
	} win;
	DevBuf<float4> ckpt, states, wpos, wfe, lam, mu, mu_sorted, tan, tan_sorted;
	DevBuf<double4> adj_tan, adj_tan_sorted;  // FP64 tangent accumulators of the reverse sweep
	float4* record_states = nullptr;  // caller's buffer for the states a reverse sweep differentiates
	uint64_t record_cap = 0;          // its capacity in float4 rows
	bool rdf_built = false;  // the current list was built by mb2_rdf_histogram
	uint32_t rdf_n = 0;

	// Optional per-stage CUDA-event timing on the launching stream.
	bool profiling = false;
	// mb2_run: the replayed graph of one step body between rebuild checks, the
	// values it bakes in, its kernel launches and the device step counter.
	cudaGraphExec_t run_graph = nullptr;
	std::vector<uint64_t> run_key;
	unsigned long long run_launches = 0;
	DevBuf<unsigned long long> step_d;
	std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof[MB2_NUM_STAGES];
};

namespace {

// Brackets one stage with events when profiling is on.
struct StageScope {
	mb2_context* ctx;
	int stage;
	cudaStream_t st;
	cudaEvent_t b = nullptr, e = nullptr;
	StageScope(mb2_context* c, int s, cudaStream_t stream) : ctx(c), stage(s), st(stream) {
		if (!ctx->profiling) return;
		MB2_CUDA(cudaEventCreate(&b));
		MB2_CUDA(cudaEventCreate(&e));
		MB2_CUDA(cudaEventRecord(b, st));
	}
	~StageScope() {
		if (!b) return;
		cudaEventRecord(e, st);
		ctx->prof[stage].emplace_back(b, e);
	}
};

int fail(mb2_context* ctx, int code, const std::string& msg) {
	if (ctx) ctx->last_error = msg;
	return code;
}

template <typename F>
int guarded(mb2_context* ctx, F&& f) {
	if (!ctx) return MB2_ERR_ARG;
	try {
		MB2_CUDA(cudaSetDevice(ctx->device));
		f();
		MB2_CUDA(cudaGetLastError());
		ctx->last_error.clear();
		return MB2_OK;
	} catch (const Error& e) {
		return fail(ctx, e.code, e.msg);
	} catch (const std::exception& e) {
		return fail(ctx, MB2_ERR_CUDA, e.what());
	}
}

void require(bool cond, int code, const char* msg) {
	if (!cond) throw Error{code, msg};
}
void require(bool cond, int code, const std::string& msg) {
	if (!cond) throw Error{code, msg};
}

cudaStream_t S(void* stream) { return reinterpret_cast<cudaStream_t>(stream); }

// Ordered-int encoding so atomicMin/Max on int order floats correctly.
__device__ __forceinline__ int f2o(float f) {
	const int i = __float_as_int(f);
	return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float o2f(int i) {
	const int b = i >= 0 ? i : i ^ 0x7FFFFFFF;
	float f;
	std::memcpy(&f, &b, 4);
	return f;
}

__global__ void bbox_kernel(const float4* __restrict__ pos, uint32_t n, int* out) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
	if (i < n) {
		const float4 p = pos[i];
		lo[0] = hi[0] = f2o(p.x);
		lo[1] = hi[1] = f2o(p.y);
		lo[2] = hi[2] = f2o(p.z);
	}
#pragma unroll
	for (int a = 0; a < 3; ++a) {
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			lo[a] = min(lo[a], __shfl_xor_sync(0xFFFFFFFFu, lo[a], o));
			hi[a] = max(hi[a], __shfl_xor_sync(0xFFFFFFFFu, hi[a], o));
		}
	}
	if ((threadIdx.x & 31) == 0) {
		for (int a = 0; a < 3; ++a) {
			atomicMin(out + a, lo[a]);
			atomicMax(out + 3 + a, hi[a]);
		}
	}
}

__global__ void bbox_init_kernel(int* out) {
	if (threadIdx.x < 3) out[threadIdx.x] = INT_MAX;
	else if (threadIdx.x < 6) out[threadIdx.x] = INT_MIN;
}

// Morton domain of ZOrderPairlist::build_pairlist (ZOrderPairlist.cpp:130-146)
// and compute_particle_extent (:368-411): the box on periodic axes, the
// particle extent + 1 % (at least 1e-4 wide) on open axes.
void morton_domain(mb2_context* ctx, const float4* pos, uint32_t n, cudaStream_t st, float* bmin,
				   float* bmax) {
	const Box& b = ctx->box;
	const bool any_open = !(b.periodic[0] && b.periodic[1] && b.periodic[2]);
	float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
	if (any_open) {
		ctx->bbox.ensure(6);
		int* dev = reinterpret_cast<int*>(ctx->bbox.ptr);
		MB2_LAUNCH bbox_init_kernel<<<1, 32, 0, st>>>(dev);
		if (n) MB2_LAUNCH bbox_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, n, dev);
		int h[6];
		MB2_CUDA(cudaMemcpyAsync(h, dev, sizeof(h), cudaMemcpyDeviceToHost, st));
		MB2_CUDA(cudaStreamSynchronize(st));
		for (int a = 0; a < 3; ++a) {
			lo[a] = n ? o2f(h[a]) : std::numeric_limits<float>::max();
			hi[a] = n ? o2f(h[3 + a]) : std::numeric_limits<float>::lowest();
			// A NaN or infinite coordinate on an open axis has no Morton domain.
			require(b.periodic[a] || (std::isfinite(lo[a]) && std::isfinite(hi[a])), MB2_ERR_ARG,
					"mb2_build_pairlist: a particle has a non-finite coordinate on an open axis");
		}
	}
	for (int a = 0; a < 3; ++a) {
		if (b.periodic[a]) {
			bmin[a] = b.origin[a];
			bmax[a] = b.origin[a] + b.size[a];
			continue;
		}
		volatile float margin = (hi[a] - lo[a]) * 0.01f;
		float l = lo[a] - margin, h = hi[a] + margin;
		volatile float range = h - l;
		if (range < 1e-4f) {
			const float center = static_cast<float>(static_cast<double>(l) + static_cast<double>(range) * 0.5);
			l = static_cast<float>(static_cast<double>(center) - static_cast<double>(1e-4f) * 0.5);
			h = static_cast<float>(static_cast<double>(center) + static_cast<double>(1e-4f) * 0.5);
		}
		bmin[a] = l;
		bmax[a] = h;
	}
}

void sort_particles(mb2_context* ctx, const float4* pos, const int* type_ids, uint32_t n,
					const float* bmin, const float* bmax, cudaStream_t st,
					unsigned long long* nonfinite = nullptr) {
	ctx->keys.ensure(n);
	ctx->s2o.ensure(n);
	ctx->inv.ensure(n);
	ctx->sorted_pos.ensure(n);
	morton_encode(pos, n, bmin, bmax, ctx->keys.ptr, ctx->s2o.ptr, st);
	radix_sort_pairs(ctx->scratch, ctx->keys.ptr, ctx->s2o.ptr, n, st);
	inverse_and_gather(ctx->s2o.ptr, n, pos, ctx->inv.ptr, nullptr, st);
	pack_sorted_positions(pos, type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st, nonfinite);
}

// cutoff: the interaction cutoff the list will serve. When it lies in
// (0, rc_list), rows are split near / far (below); otherwise rows keep the
// walk's candidate order.
void build(mb2_context* ctx, const float4* pos, const int* type_ids, uint32_t n, float rc_list,
		   float cutoff, cudaStream_t st) {
	require(ctx->box_set, MB2_ERR_STATE, "mb2_build_pairlist: call mb2_set_box first");
	require(n <= ctx->max_particles, MB2_ERR_CAPACITY,
			"mb2_build_pairlist: more particles than the context was created for");
	require(rc_list > 0.0f && std::isfinite(rc_list), MB2_ERR_ARG,
			"mb2_build_pairlist: pairlist cutoff must be positive and finite");
	StageScope scope(ctx, MB2_STAGE_PAIRLIST, st);
	// A failed build leaves no list behind.
	ctx->built = false;
	float bmin[3], bmax[3], extent[3];
	morton_domain(ctx, pos, n, st, bmin, bmax);
	for (int a = 0; a < 3; ++a) extent[a] = bmax[a] - bmin[a];
	// stats: [0] pairs, [1] longest row (both set by each walk), [2] particles
	// with a non-finite coordinate (counted while packing, read with the
	// walk's statistics, so no extra synchronisation).
	ctx->stats.ensure(3);
	MB2_CUDA(cudaMemsetAsync(ctx->stats.ptr + 2, 0, sizeof(unsigned long long), st));
	sort_particles(ctx, pos, type_ids, n, bmin, bmax, st, ctx->stats.ptr + 2);

	const float rc2 = rc_list * rc_list;
	if (!ctx->grid_valid || ctx->grid_rc != rc_list || ctx->grid_n != n ||
		std::memcmp(ctx->grid_extent, extent, sizeof(extent)) != 0) {
		ctx->grid = choose_cell_grid(extent, ctx->box.periodic, std::sqrt(rc2), n);
		if (ctx->level_offset != 0) {
			const int m = std::min(8, std::max(0, ctx->grid.m + ctx->level_offset));
			ctx->grid = choose_cell_grid(extent, ctx->box.periodic, std::sqrt(rc2), n, m, m);
		}
		ctx->stencil.ensure(ctx->grid.stencil.size());
		MB2_CUDA(cudaMemcpyAsync(ctx->stencil.ptr, ctx->grid.stencil.data(),
								 ctx->grid.stencil.size() * sizeof(StencilEntry),
								 cudaMemcpyHostToDevice, st));
		ctx->grid_valid = true;
		ctx->grid_rc = rc_list;
		ctx->grid_n = n;
		std::memcpy(ctx->grid_extent, extent, sizeof(extent));
	}
	const CellGrid& g = ctx->grid;
	const size_t num_cells = static_cast<size_t>(1) << (3 * g.m);
	ctx->cell_begin.ensure(num_cells);
	ctx->cell_end.ensure(num_cells);
	cell_ranges(ctx->keys.ptr, n, g.shift, ctx->cell_begin.ptr, ctx->cell_end.ptr, num_cells, st);

	WalkGrid wg{};
	wg.m = g.m;
	wg.shift = g.shift;
	wg.emax = 3;
	for (int a = 0; a < 3; ++a) {
		wg.radius[a] = g.radius[a];
		wg.wmin[a] = g.wmin[a];
		wg.full[a] = ctx->box.periodic[a] && g.m > 0 && (2 * g.radius[a] + 1 >= (1 << g.m));
		if (g.m == 0) wg.full[a] = ctx->box.periodic[a];
	}
	wg.lim = g.lim;
	wg.rc2 = rc2;
	// Rows put the pairs that are likely to come within the interaction cutoff
	// before the next rebuild first (d <= cutoff + 25 % of the skin at build
	// time) and the rest after them: in a row's tail the whole warp's pairs are
	// beyond the cutoff for most iterations of the force kernel, which then
	// skips the force part. The split moves no pair in or out of the list.
	// Measured on the 2,097,152-bead workload (fused step, rebuild every 20
	// steps): 1.94 ms without the split; 1.87 ms at 25 % of the skin, 1.89 at
	// 10 % and at 40 %, 1.92 at 70 %.
	const float split =
		(cutoff > 0.0f && cutoff < rc_list) ? cutoff + 0.25f * (rc_list - cutoff) : 0.0f;
	wg.split2 = split > 0.0f ? split * split : INFINITY;
	for (int a = 0; a < 3; ++a) {
		// Morton coordinate q = trunc((x - bmin) / range * 1023) on 0..1023, a cell
		// of level m spanning 2^(10-m) of them; the margin covers the rounding of
		// that mapping (a few ulp of the coordinates) with room to spare.
		const double range = std::max(static_cast<double>(bmax[a]) - bmin[a], 1e-6);
		wg.dom_lo[a] = bmin[a];
		wg.cell_w[a] = static_cast<float>(std::ldexp(1.0, 10 - g.m) * range / 1023.0);
		wg.eps[a] = static_cast<float>(1e-5 * (std::fabs(static_cast<double>(bmin[a])) + range) + 1e-6);
	}
	fast_test_band(ctx->box, rc_list, &wg.fast_lo, &wg.fast_hi);
	ctx->row_len.ensure(n);
	ctx->row_far.ensure(n);
	auto walk = [&](uint32_t cap) {
		const int hshift = __builtin_ctz(32 / ctx->lanes);
		build_walk(ctx->sorted_pos.ptr, ctx->keys.ptr, ctx->s2o.ptr, ctx->cell_begin.ptr,
				   ctx->cell_end.ptr, ctx->stencil.ptr, g.num_stencil, wg, n, ctx->box, ctx->excl,
				   ctx->nbr.ptr, cap, hshift, ctx->row_len.ptr, ctx->row_far.ptr, ctx->stats.ptr,
				   st);
		MB2_CUDA(cudaMemcpyAsync(ctx->pinned, ctx->stats.ptr, 3 * sizeof(uint64_t),
								 cudaMemcpyDeviceToHost, st));
		MB2_CUDA(cudaStreamSynchronize(st));
		// The walk runs on such particles without harm (cell indices come from
		// the clamped Morton keys, and a NaN fails every distance test), but
		// the list is not the reference's meaning of one: refuse it.
		require(ctx->pinned[2] == 0, MB2_ERR_ARG,
				"mb2_build_pairlist: " + std::to_string(ctx->pinned[2]) +
					" particle(s) with a NaN or infinite coordinate");
		return std::make_pair(ctx->pinned[0], ctx->pinned[1]);
	};
	// Lanes per row of the force kernels. A system small enough for the row
	// walk leaves most of the GPU idle, so its rows get more lanes (more
	// threads, shorter per-lane chains): 16 lanes measured 5-9 % faster per
	// step than 8 or 4 at 4,096 (21.3 against 23.3 us), 32,768 (54.9 / 58.5)
	// and 65,536 beads (polymers, 52.9 / 55.5); at 2,097,152 beads 8 lanes are
	// the fastest.
	auto choose_lanes = [&](double mean) {
		if (ctx->lanes_request) return ctx->lanes_request;
		if (n <= kRowWalkMaxN) return mean >= 16.0 ? 16 : 8;
		if (mean >= 256.0) return 16;
		if (mean >= 48.0) return 8;
		return 4;
	};
	auto size_list = [&](uint64_t max_row) {
		const uint32_t G = static_cast<uint32_t>(ctx->lanes);
		uint64_t cap = max_row + max_row / 4 + G;
		cap = (cap + G - 1) / G * G;
		require(cap < 65536u, MB2_ERR_CAPACITY,
				"mb2_build_pairlist: a particle has more than ~52000 list neighbours");
		ctx->cap = static_cast<uint32_t>(cap);
		const size_t slices = (static_cast<size_t>(n) + (32 / G) - 1) / (32 / G);
		ctx->nbr.ensure(std::max<size_t>(slices * cap * (32 / G), 1));
	};
	if (ctx->cap == 0 || ctx->lanes == 0) {
		// First build: count rows without storing, to size the list.
		ctx->lanes = 4;
		const auto counted = walk(0u);
		ctx->lanes = choose_lanes(n ? static_cast<double>(counted.first) / n : 0.0);
		size_list(counted.second);
	}
	{
		const size_t h = static_cast<size_t>(32 / ctx->lanes);
		ctx->nbr.ensure(std::max<size_t>((n + h - 1) / h * ctx->cap * h, 1));
	}
	auto stats = walk(ctx->cap);
	if (stats.second > ctx->cap) {
		// Longer rows than the list was sized for: grow and walk again.
		size_list(stats.second);
		stats = walk(ctx->cap);
	}
	if (split > 0.0f)
		join_far(ctx->nbr.ptr, ctx->row_len.ptr, ctx->row_far.ptr, n, ctx->cap,
				 __builtin_ctz(32 / ctx->lanes), st);
	// Snapshot for the skin check (ZOrderPairlist.cpp:172-173).
	ctx->ref_pos.ensure(n);
	MB2_CUDA(cudaMemcpyAsync(ctx->ref_pos.ptr, pos, static_cast<size_t>(n) * sizeof(float4),
							 cudaMemcpyDeviceToDevice, st));
	// and, in Z order, the origin of the displacement the packs track. Only
	// above kRowWalkMaxN particles: the inner rows save the pair kernel
	// 2.6 % at 2,097,152 beads, while on a 65,536-bead step the pack's extra
	// read and reduction cost more (1-2 us) than they save.
	ctx->track_rc = 0.0f;
	if (n > kRowWalkMaxN) {
		ctx->ref_sorted.ensure(n);
		ctx->d2max.ensure(1);
		MB2_CUDA(cudaMemcpyAsync(ctx->ref_sorted.ptr, ctx->sorted_pos.ptr,
								 static_cast<size_t>(n) * sizeof(float4), cudaMemcpyDeviceToDevice,
								 st));
		MB2_CUDA(cudaMemsetAsync(ctx->d2max.ptr, 0, sizeof(unsigned int), st));
		ctx->track_rc = rc_list;
	}
	ctx->num_pairs = stats.first;
	ctx->max_row = stats.second;
	ctx->built = true;
	ctx->built_n = n;
	ctx->rdf_built = false;
}

bool matrix_has_analytical(const mb2_context* ctx) {
	for (uint32_t tag : ctx->term_matrix_h)
		if (tag & kTermAnalytical) return true;
	return false;
}

// The displacement track of the last build, for the step's pack (none
// before a build or after the box changed).
DisplacementTrack track_of(mb2_context* ctx) {
	if (!(ctx->track_rc > 0.0f)) return DisplacementTrack{};
	return displacement_track(ctx->box, ctx->ref_sorted.ptr, ctx->d2max.ptr);
}

// Pair kernel over the sorted positions into the zeroed sorted accumulator.
// The Z-ordered pair-force accumulator, sized for n (for a pack that clears it).
float4* sorted_forces(mb2_context* ctx, uint32_t n) {
	ctx->force_sorted.ensure(n);
	return ctx->force_sorted.ptr;
}

// cleared: the accumulator was zeroed by this step's pack.
void pair_kernel(mb2_context* ctx, uint32_t n, float cutoff, int get_energy, cudaStream_t st,
				 bool cleared = false) {
	require(ctx->built, MB2_ERR_STATE, "mb2_pair_forces: no pairlist; call mb2_build_pairlist");
	require(n == ctx->built_n, MB2_ERR_ARG,
			"mb2_pair_forces: particle count differs from the last pairlist build");
	require(ctx->pt.num_types > 0, MB2_ERR_STATE,
			"mb2_pair_forces: no pair tables; call mb2_set_pair_tables");
	require(ctx->pt.terms || !matrix_has_analytical(ctx), MB2_ERR_STATE,
			"mb2_pair_forces: the tags carry analytical terms; call mb2_set_pair_terms");
	ctx->force_sorted.ensure(n);
	if (!cleared)
		MB2_CUDA(cudaMemsetAsync(ctx->force_sorted.ptr, 0, static_cast<size_t>(n) * sizeof(float4),
								 st));
	const float cutoff_sq = cutoff > 0.0f ? cutoff * cutoff : 0.0f;
	StageScope scope(ctx, MB2_STAGE_PAIR_FORCE, st);
	// Every caller packs with track_of (or builds) just before: the track
	// covers the positions the kernel reads.
	pair_forces(ctx->sorted_pos.ptr, ctx->nbr.ptr, ctx->row_len.ptr, n, ctx->cap, ctx->lanes, ctx->pt,
				ctx->box, cutoff_sq, get_energy, ctx->force_sorted.ptr, ctx->energy.ptr, st,
				ctx->track_rc > 0.0f ? ctx->d2max.ptr : nullptr, ctx->track_rc);
}

void pair_forces_impl(mb2_context* ctx, const float4* pos, const int* type_ids, float4* fe,
					  uint32_t n, float cutoff, int get_energy, cudaStream_t st) {
	require(ctx->built, MB2_ERR_STATE, "mb2_pair_forces: no pairlist; call mb2_build_pairlist");
	if (n == 0) return;
	pack_sorted_positions(pos, type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st, nullptr,
						  sorted_forces(ctx, n), nullptr, track_of(ctx));
	pair_kernel(ctx, n, cutoff, get_energy, st, true);
	scatter_add_forces(ctx->force_sorted.ptr, ctx->s2o.ptr, n, fe, get_energy, st);
}

float max_disp(mb2_context* ctx, const float4* pos, uint32_t n, cudaStream_t st) {
	require(ctx->built && n == ctx->built_n, MB2_ERR_STATE,
			"mb2_needs_update: no pairlist for this particle count");
	ctx->disp.ensure(1);
	max_displacement_sq(pos, ctx->ref_pos.ptr, n, ctx->box, ctx->disp.ptr, st);
	MB2_CUDA(cudaMemcpyAsync(ctx->pinned, ctx->disp.ptr, sizeof(uint32_t),
							 cudaMemcpyDeviceToHost, st));
	MB2_CUDA(cudaStreamSynchronize(st));
	float d2;
	std::memcpy(&d2, ctx->pinned, 4);
	return sqrtf(d2);
}

void upload_tables(DevBuf<Table>& tbuf, DevBuf<float>& vbuf, int num_tables, const float* values,
				   const uint32_t* sizes, const float* starts, const float* step_invs,
				   int periodic, uint32_t* total_out) {
	size_t total = 0;
	for (int k = 0; k < num_tables; ++k) {
		require(sizes[k] >= 2, MB2_ERR_ARG, "table needs at least 2 values");
		require(std::isfinite(starts[k]) && std::isfinite(step_invs[k]) && step_invs[k] != 0.0f,
				MB2_ERR_ARG, "table start and step inverse must be finite, step inverse nonzero");
		total += sizes[k];
	}
	vbuf.ensure(total);
	MB2_CUDA(cudaMemcpy(vbuf.ptr, values, total * sizeof(float), cudaMemcpyHostToDevice));
	std::vector<Table> host(num_tables);
	size_t off = 0;
	for (int k = 0; k < num_tables; ++k) {
		host[k] = Table{vbuf.ptr + off, step_invs[k], sizes[k], starts[k], periodic};
		off += sizes[k];
	}
	tbuf.ensure(std::max(num_tables, 1));
	MB2_CUDA(cudaMemcpy(tbuf.ptr, host.data(), num_tables * sizeof(Table), cudaMemcpyHostToDevice));
	if (total_out) *total_out = static_cast<uint32_t>(total);
}

// Per-type-pair analytical constants from the tag matrix and the per-type
// data, each rounded as PairNonbondedComputer rounds it per pair
// (Pairwise.h:248-283, Columb.h:11-97). Leaves pt.terms null when no type
// pair has an analytical term (the tabulated-only kernel then runs).
void rebuild_pair_terms(mb2_context* ctx) {
	ctx->pt.terms = nullptr;
	if (!ctx->pair_terms_set || !matrix_has_analytical(ctx)) return;
	const int T = ctx->pt.num_types;
	require(static_cast<int>(ctx->term_charge.size()) >= T, MB2_ERR_STATE,
			"mb2_set_pair_terms: fewer types than the pair tables");
	std::vector<PairTermRef> h(static_cast<size_t>(T) * T);
	for (int a = 0; a < T; ++a)
		for (int b = 0; b < T; ++b) {
			PairTermRef& r = h[static_cast<size_t>(a) * T + b];
			r.terms = ctx->term_matrix_h[static_cast<size_t>(a) * T + b] & kTermAnalytical;
			volatile float qq = ctx->term_charge[a] * ctx->term_charge[b];
			volatile float qc = qq * kCoulomb;
			volatile float adh = qc / ctx->term_dielectric;
			volatile float rad = 0.5f * (ctx->term_radius[a] + ctx->term_radius[b]);
			volatile float rad2 = rad * rad;
			volatile float rad4 = rad2 * rad2;
			volatile float rad6 = rad4 * rad2;
			volatile float ee = ctx->term_eps[a] * ctx->term_eps[b];
			r.qq = qq;
			r.a_onck = qc;
			r.a_dh = adh;
			r.rad6 = rad6;
			r.eps = std::sqrt(static_cast<float>(ee));
			r.pad0 = r.pad1 = 0.0f;
		}
	ctx->term_refs.ensure(h.size());
	MB2_CUDA(cudaMemcpy(ctx->term_refs.ptr, h.data(), h.size() * sizeof(PairTermRef),
						cudaMemcpyHostToDevice));
	ctx->pt.terms = ctx->term_refs.ptr;
	ctx->pt.solvent = ctx->solvent;
}

// Bonded terms of one step into ForceEnergy (Patch::calculate_bonded_forces,
// Patch.cpp:180-234): bonds, angles, dihedrals, restraints.
void bonded_stage(mb2_context* ctx, const float4* pos, float4* fe, const mb2_step_params* prm,
				  int get_energy, cudaStream_t st) {
	if (prm->num_bonds || prm->num_angles)
		bond_angle_forces(reinterpret_cast<const int2*>(prm->bonds2), prm->bond_table_idx,
						  prm->num_bonds, ctx->bonded_tables[0].ptr,
						  reinterpret_cast<const int4*>(prm->angles4), prm->angle_table_idx,
						  prm->num_angles, ctx->bonded_tables[1].ptr, pos, fe, ctx->box, get_energy,
						  ctx->energy.ptr + 2, ctx->energy.ptr + 3, st);
	if (prm->num_dihedrals)
		dihedral_forces(reinterpret_cast<const int4*>(prm->dihedrals4), prm->dihedral_table_idx,
						prm->num_dihedrals, pos, fe, ctx->bonded_tables[2].ptr, ctx->box,
						get_energy, ctx->energy.ptr + 4, st);
	if (prm->num_restraints)
		restraint_forces(prm->restraint_ids, reinterpret_cast<const float4*>(prm->restraint_anchors4),
						 prm->restraint_k, prm->num_restraints, pos, fe, ctx->box, get_energy,
						 ctx->energy.ptr + 5, st);
}

bool step_has_bonded(const mb2_step_params* prm) {
	return prm->num_bonds != 0 || prm->num_angles != 0 || prm->num_dihedrals != 0 ||
		   prm->num_restraints != 0;
}

// One step of the window without the rebuild decision (the segment's list
// was built at its first step): the mb2_step sequence otherwise.
void window_step(mb2_context* ctx, float4* pos, float4* fe, const int* type_ids, uint32_t n,
				 uint64_t step, const mb2_step_params* prm, cudaStream_t st) {
	const bool bonded = prm->num_bonds != 0 || prm->num_angles != 0;
	pack_sorted_positions(pos, type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st, nullptr,
						  sorted_forces(ctx, n), bonded ? fe : nullptr, track_of(ctx));
	pair_kernel(ctx, n, prm->cutoff, 0, st, true);
	if (bonded)
		bond_angle_forces(reinterpret_cast<const int2*>(prm->bonds2), prm->bond_table_idx,
						  prm->num_bonds, ctx->bonded_tables[0].ptr,
						  reinterpret_cast<const int4*>(prm->angles4), prm->angle_table_idx,
						  prm->num_angles, ctx->bonded_tables[1].ptr, pos, fe, ctx->box, 0,
						  ctx->energy.ptr + 2, ctx->energy.ptr + 3, st);
	BdParams p{prm->dt, prm->kT, static_cast<uint32_t>(step),
			   mb2_bd_seed(prm->seed, prm->patch_id, step), 0u,
			   {prm->efield[0], prm->efield[1], prm->efield[2]}};
	bd_integrate_gather(pos, fe, ctx->force_sorted.ptr, ctx->inv.ptr, type_ids, nullptr, n,
						ctx->types, ctx->box, p, bonded ? 1 : 0, st);
}

void copy4(float4* dst, const float4* src, uint32_t n, cudaStream_t st) {
	MB2_CUDA(cudaMemcpyAsync(dst, src, static_cast<size_t>(n) * sizeof(float4),
							 cudaMemcpyDeviceToDevice, st));
}

}  // namespace

extern "C" {

int mb2_version(void) { return 100; }

int mb2_create(int device, uint32_t max_particles, mb2_context** out) {
	if (!out) return MB2_ERR_ARG;
	*out = nullptr;
	mb2_context* ctx = new (std::nothrow) mb2_context();
	if (!ctx) return MB2_ERR_CAPACITY;
	ctx->device = device;
	ctx->max_particles = max_particles;
	const int rc = guarded(ctx, [&] {
		MB2_CUDA(cudaMallocHost(&ctx->pinned, 64));
		ctx->energy.ensure(kEnergySlots);
		MB2_CUDA(cudaMemset(ctx->energy.ptr, 0, kEnergySlots * sizeof(double)));
	});
	if (rc != MB2_OK) {
		delete ctx;
		return rc;
	}
	*out = ctx;
	return MB2_OK;
}

int mb2_destroy(mb2_context* ctx) {
	if (!ctx) return MB2_ERR_ARG;
	cudaSetDevice(ctx->device);
	cudaDeviceSynchronize();
	for (auto& stage : ctx->prof)
		for (auto& be : stage) {
			cudaEventDestroy(be.first);
			cudaEventDestroy(be.second);
		}
	if (ctx->pinned) cudaFreeHost(ctx->pinned);
	if (ctx->run_graph) cudaGraphExecDestroy(ctx->run_graph);
	delete ctx;  // device buffers free themselves
	return MB2_OK;
}

const char* mb2_last_error(const mb2_context* ctx) {
	return ctx ? ctx->last_error.c_str() : "null context";
}

int mb2_set_box(mb2_context* ctx, const float origin[3], const float size[3],
				const int periodic[3]) {
	return guarded(ctx, [&] {
		require(origin && size && periodic, MB2_ERR_ARG, "mb2_set_box: null argument");
		for (int a = 0; a < 3; ++a) {
			require(size[a] > 0.0f && std::isfinite(size[a]), MB2_ERR_ARG,
					"mb2_set_box: box size must be positive (ZOrderPairlist.cpp:118-126)");
			ctx->box.origin[a] = origin[a];
			ctx->box.size[a] = size[a];
			ctx->box.inv[a] = 1.0f / size[a];
			ctx->box.half[a] = 0.5f * size[a];
			ctx->box.periodic[a] = periodic[a] ? 1 : 0;
		}
		ctx->box_set = true;
		ctx->grid_valid = false;
		ctx->track_rc = 0.0f;  // the tracked displacement belongs to the old box
	});
}

int mb2_sort_morton(mb2_context* ctx, const float* pos4, uint32_t n, const float bmin[3],
					const float bmax[3], uint32_t* keys_out, uint32_t* s2o_out,
					uint32_t* inverse_out, float* sorted_pos4_out, void* stream) {
	return guarded(ctx, [&] {
		require(n <= ctx->max_particles, MB2_ERR_CAPACITY, "mb2_sort_morton: n above capacity");
		require(n == 0 || pos4, MB2_ERR_ARG, "mb2_sort_morton: null positions");
		const cudaStream_t st = S(stream);
		const float4* pos = reinterpret_cast<const float4*>(pos4);
		ctx->keys.ensure(n);
		ctx->s2o.ensure(n);
		ctx->inv.ensure(n);
		morton_encode(pos, n, bmin, bmax, ctx->keys.ptr, ctx->s2o.ptr, st);
		radix_sort_pairs(ctx->scratch, ctx->keys.ptr, ctx->s2o.ptr, n, st);
		inverse_and_gather(ctx->s2o.ptr, n, pos, ctx->inv.ptr,
						   reinterpret_cast<float4*>(sorted_pos4_out), st);
		const size_t b = static_cast<size_t>(n) * sizeof(uint32_t);
		if (keys_out) MB2_CUDA(cudaMemcpyAsync(keys_out, ctx->keys.ptr, b, cudaMemcpyDeviceToDevice, st));
		if (s2o_out) MB2_CUDA(cudaMemcpyAsync(s2o_out, ctx->s2o.ptr, b, cudaMemcpyDeviceToDevice, st));
		if (inverse_out) MB2_CUDA(cudaMemcpyAsync(inverse_out, ctx->inv.ptr, b, cudaMemcpyDeviceToDevice, st));
		ctx->built = false;  // the sort state no longer matches a pairlist
	});
}

int mb2_radix_sort_pairs(mb2_context* ctx, uint32_t* keys, uint32_t* vals, uint32_t n,
						 void* stream) {
	return guarded(ctx, [&] {
		require(n == 0 || (keys && vals), MB2_ERR_ARG, "mb2_radix_sort_pairs: null argument");
		radix_sort_pairs(ctx->scratch, keys, vals, n, S(stream));
	});
}

int mb2_radix_sort_pairs_static(mb2_context* ctx, uint32_t* keys, uint32_t* vals, uint32_t n,
								void* stream) {
	return guarded(ctx, [&] {
		require(n == 0 || (keys && vals), MB2_ERR_ARG,
				"mb2_radix_sort_pairs_static: null argument");
		radix_sort_pairs_static(keys, vals, n, S(stream));
	});
}

int mb2_set_exclusions(mb2_context* ctx, const int* offsets, const int* neighbors,
					   uint32_t num_particles, const int* rigid_body_id) {
	return guarded(ctx, [&] {
		require(!offsets || neighbors || num_particles == 0, MB2_ERR_ARG,
				"mb2_set_exclusions: offsets without neighbors");
		ctx->excl.offsets = offsets;
		ctx->excl.neighbors = neighbors;
		ctx->excl.num_particles = offsets ? num_particles : 0;
		ctx->excl.rigid_body_id = rigid_body_id;
	});
}

int mb2_build_pairlist(mb2_context* ctx, const float* pos4, const int* type_ids, uint32_t n,
					   float pairlist_cutoff, float interaction_cutoff, void* stream,
					   uint64_t* num_pairs) {
	return guarded(ctx, [&] {
		require(n == 0 || pos4, MB2_ERR_ARG, "mb2_build_pairlist: null positions");
		require(!std::isnan(interaction_cutoff), MB2_ERR_ARG,
				"mb2_build_pairlist: interaction cutoff is NaN");
		build(ctx, reinterpret_cast<const float4*>(pos4), type_ids, n, pairlist_cutoff,
			  interaction_cutoff, S(stream));
		if (num_pairs) *num_pairs = ctx->num_pairs;
	});
}

int mb2_num_pairs(const mb2_context* ctx, uint64_t* num_pairs) {
	if (!ctx || !num_pairs) return MB2_ERR_ARG;
	*num_pairs = ctx->built ? ctx->num_pairs : 0;
	return MB2_OK;
}

int mb2_export_pairs(mb2_context* ctx, int* pairs2, uint64_t capacity, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->built, MB2_ERR_STATE, "mb2_export_pairs: no pairlist");
		require(capacity >= ctx->num_pairs, MB2_ERR_CAPACITY,
				"mb2_export_pairs: output smaller than the pair count");
		require(ctx->num_pairs == 0 || pairs2, MB2_ERR_ARG, "mb2_export_pairs: null output");
		const uint32_t n = ctx->built_n;
		ctx->row_off.ensure(n);
		exclusive_scan_u32(ctx->scratch, ctx->row_len.ptr, ctx->row_off.ptr, n, nullptr, S(stream));
		export_pairs(ctx->nbr.ptr, ctx->row_len.ptr, ctx->row_off.ptr, ctx->s2o.ptr, n, ctx->cap,
					 __builtin_ctz(32 / ctx->lanes), reinterpret_cast<int2*>(pairs2), S(stream));
	});
}

int mb2_needs_update(mb2_context* ctx, const float* pos4, uint32_t n, float skin, void* stream,
					 float* max_displacement, int* needs) {
	return guarded(ctx, [&] {
		const float d = max_disp(ctx, reinterpret_cast<const float4*>(pos4), n, S(stream));
		if (max_displacement) *max_displacement = d;
		if (needs) *needs = d > skin * 0.5f ? 1 : 0;
	});
}

int mb2_set_pair_tables(mb2_context* ctx, int num_types, const uint32_t* term_matrix,
						int num_tables, const float* values, const uint32_t* sizes,
						const float* starts, const float* step_invs) {
	return guarded(ctx, [&] {
		require(num_types > 0 && num_types <= 64, MB2_ERR_ARG,
				"mb2_set_pair_tables: 1..64 particle types");
		require(num_tables >= 0 && term_matrix, MB2_ERR_ARG, "mb2_set_pair_tables: bad tables");
		for (int k = 0; k < num_types * num_types; ++k) {
			const uint32_t tag = term_matrix[k];
			require(!(tag & kTermTabulated) || static_cast<int>(tag >> kTableShift) < num_tables,
					MB2_ERR_ARG, "mb2_set_pair_tables: tag names a missing table");
		}
		std::vector<PairTableRef> refs;
		std::vector<float> bf;
		std::vector<float2> be;
		const size_t total = pair_table_arrays(num_types, term_matrix, num_tables, values, sizes,
											   starts, step_invs, refs, bf, be);
		const int tt = num_types * num_types;
		const size_t smem = static_cast<size_t>(tt) * sizeof(PairTableRef) + total * 12 + 8;
		require(smem <= 200 * 1024, MB2_ERR_CAPACITY,
				"mb2_set_pair_tables: tables exceed the 200 KB shared-memory budget");
		ctx->refs.ensure(tt);
		ctx->bin_force.ensure(bf.size());
		ctx->bin_energy.ensure(be.size());
		MB2_CUDA(cudaMemcpy(ctx->refs.ptr, refs.data(), tt * sizeof(PairTableRef),
							cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->bin_force.ptr, bf.data(), bf.size() * sizeof(float),
							cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->bin_energy.ptr, be.data(), be.size() * sizeof(float2),
							cudaMemcpyHostToDevice));
		// Tables of one start, bin width and length for every type pair that
		// has one (compared bit for bit): the kernel reads 4-byte offsets.
		std::vector<int> offs;
		PairTableRef u;
		const bool uniform = uniform_tables(refs, offs, u);
		ctx->table_offsets.ensure(tt);
		MB2_CUDA(cudaMemcpy(ctx->table_offsets.ptr, offs.data(), tt * sizeof(int),
							cudaMemcpyHostToDevice));
		ctx->pt.num_types = num_types;
		ctx->pt.total_bins = static_cast<uint32_t>(total);
		ctx->pt.refs = ctx->refs.ptr;
		ctx->pt.offsets = ctx->table_offsets.ptr;
		ctx->pt.uniform = uniform;
		ctx->pt.uniform_ref = u;
		ctx->pt.bin_force = ctx->bin_force.ptr;
		ctx->pt.bin_energy = ctx->bin_energy.ptr;
		ctx->term_matrix_h.assign(term_matrix, term_matrix + tt);
		rebuild_pair_terms(ctx);
	});
}

int mb2_set_pair_terms(mb2_context* ctx, int num_types, const float* charge, const float* radius,
					   const float* eps, const mb2_pair_params* params) {
	return guarded(ctx, [&] {
		require(num_types > 0 && num_types <= 64 && charge && radius && eps, MB2_ERR_ARG,
				"mb2_set_pair_terms: 1..64 types with charge, radius and eps");
		mb2_pair_params p{10.0f, 80.0f, 0.1f, 80.0f, 6.86f, 1.0f, 1.0f, 0.0f};
		if (params) p = *params;
		require(p.debye_length > 0.0f && p.dielectric != 0.0f && p.onck_z > 0.0f &&
					p.gaussian_sigma != 0.0f,
				MB2_ERR_ARG, "mb2_set_pair_terms: bad solvent or Gaussian constants");
		ctx->term_charge.assign(charge, charge + num_types);
		ctx->term_radius.assign(radius, radius + num_types);
		ctx->term_eps.assign(eps, eps + num_types);
		ctx->term_dielectric = p.dielectric;
		PairSolvent& sv = ctx->solvent;
		sv.dh_len = p.debye_length;
		sv.dh_inv_len = 1.0f / p.debye_length;
		sv.onck_kappa = p.onck_kappa;
		sv.onck_sz = p.onck_sz;
		sv.onck_z = p.onck_z;
		sv.onck_two_z = 2.0f * p.onck_z;
		sv.g_amp = p.gaussian_amp;
		volatile float s2 = p.gaussian_sigma * p.gaussian_sigma;
		sv.g_inv_s2 = 1.0f / s2;
		sv.g_cut2 = p.gaussian_cutoff_sq;
		ctx->pair_terms_set = true;
		if (ctx->pt.num_types > 0) rebuild_pair_terms(ctx);
	});
}

int mb2_pair_distance_window(float cutoff, float* d2_lo, float* d2_hi) {
	if (!d2_lo || !d2_hi) return MB2_ERR_ARG;
	const DistWindow w = dist_window(cutoff > 0.0f ? cutoff * cutoff : 0.0f);
	*d2_lo = w.lo;
	*d2_hi = w.hi;
	return MB2_OK;
}

int mb2_selftest_sqrt(mb2_context* ctx, uint64_t* mismatches) {
	return guarded(ctx, [&] {
		require(mismatches, MB2_ERR_ARG, "mb2_selftest_sqrt: null output");
		DevBuf<unsigned long long> bad;
		bad.ensure(1);
		MB2_CUDA(cudaMemset(bad.ptr, 0, sizeof(unsigned long long)));
		selftest_sqrt(bad.ptr, nullptr);
		unsigned long long h = 0;
		MB2_CUDA(cudaMemcpy(&h, bad.ptr, sizeof(h), cudaMemcpyDeviceToHost));
		*mismatches = h;
	});
}

int mb2_pair_forces(mb2_context* ctx, const float* pos4, const int* type_ids,
					float* force_energy4, uint32_t n, float cutoff, int get_energy,
					void* stream) {
	return guarded(ctx, [&] {
		require(n == 0 || (pos4 && type_ids && force_energy4), MB2_ERR_ARG,
				"mb2_pair_forces: null argument");
		pair_forces_impl(ctx, reinterpret_cast<const float4*>(pos4), type_ids,
						 reinterpret_cast<float4*>(force_energy4), n, cutoff, get_energy,
						 S(stream));
	});
}

int mb2_energies(mb2_context* ctx, void* stream, double out[4]) {
	return guarded(ctx, [&] {
		require(out, MB2_ERR_ARG, "mb2_energies: null output");
		MB2_CUDA(cudaMemcpyAsync(out, ctx->energy.ptr, 4 * sizeof(double), cudaMemcpyDeviceToHost,
								 S(stream)));
		MB2_CUDA(cudaStreamSynchronize(S(stream)));
	});
}

int mb2_energy_terms(mb2_context* ctx, void* stream, double* out, int count) {
	return guarded(ctx, [&] {
		require(out && count > 0, MB2_ERR_ARG, "mb2_energy_terms: null output");
		const int c = std::min(count, kEnergySlots);
		MB2_CUDA(cudaMemcpyAsync(out, ctx->energy.ptr, c * sizeof(double), cudaMemcpyDeviceToHost,
								 S(stream)));
		MB2_CUDA(cudaStreamSynchronize(S(stream)));
	});
}

int mb2_reset_energies(mb2_context* ctx, void* stream) {
	return guarded(ctx, [&] {
		MB2_CUDA(cudaMemsetAsync(ctx->energy.ptr, 0, kEnergySlots * sizeof(double), S(stream)));
	});
}

int mb2_set_bonded_tables(mb2_context* ctx, int kind, int num_tables, const float* values,
						  const uint32_t* sizes, const float* starts, const float* step_invs) {
	return guarded(ctx, [&] {
		require(kind >= 0 && kind <= 2, MB2_ERR_ARG, "mb2_set_bonded_tables: kind is 0, 1 or 2");
		require(num_tables > 0, MB2_ERR_ARG, "mb2_set_bonded_tables: no tables");
		upload_tables(ctx->bonded_tables[kind], ctx->bonded_values[kind], num_tables, values, sizes,
					  starts, step_invs, kind >= 1 ? 1 : 0, &ctx->bonded_bins[kind]);
		ctx->bonded_count[kind] = num_tables;
	});
}

int mb2_bond_forces(mb2_context* ctx, const int* bonds2, const int* table_idx, uint32_t nb,
					const float* pos4, float* force_energy4, int get_energy, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_bond_forces: no box");
		require(nb == 0 || ctx->bonded_count[0] > 0, MB2_ERR_STATE, "mb2_bond_forces: no tables");
		bond_forces(reinterpret_cast<const int2*>(bonds2), table_idx, nb,
					reinterpret_cast<const float4*>(pos4), reinterpret_cast<float4*>(force_energy4),
					ctx->bonded_tables[0].ptr, ctx->box, get_energy, ctx->energy.ptr + 2,
					S(stream));
	});
}

int mb2_angle_forces(mb2_context* ctx, const int* angles4, const int* table_idx, uint32_t na,
					 const float* pos4, float* force_energy4, int get_energy, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_angle_forces: no box");
		require(na == 0 || ctx->bonded_count[1] > 0, MB2_ERR_STATE, "mb2_angle_forces: no tables");
		angle_forces(reinterpret_cast<const int4*>(angles4), table_idx, na,
					 reinterpret_cast<const float4*>(pos4), reinterpret_cast<float4*>(force_energy4),
					 ctx->bonded_tables[1].ptr, ctx->box, get_energy, ctx->energy.ptr + 3,
					 S(stream));
	});
}

int mb2_dihedral_forces(mb2_context* ctx, const int* dihedrals4, const int* table_idx,
						uint32_t nd, const float* pos4, float* force_energy4, int get_energy,
						void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_dihedral_forces: no box");
		require(nd == 0 || ctx->bonded_count[2] > 0, MB2_ERR_STATE,
				"mb2_dihedral_forces: no tables");
		require(nd == 0 || (dihedrals4 && table_idx && pos4 && force_energy4), MB2_ERR_ARG,
				"mb2_dihedral_forces: null argument");
		dihedral_forces(reinterpret_cast<const int4*>(dihedrals4), table_idx, nd,
						reinterpret_cast<const float4*>(pos4),
						reinterpret_cast<float4*>(force_energy4), ctx->bonded_tables[2].ptr,
						ctx->box, get_energy, ctx->energy.ptr + 4, S(stream));
	});
}

int mb2_restraint_forces(mb2_context* ctx, const int* particle_ids, const float* anchors4,
						 const float* spring_k, uint32_t nr, const float* pos4,
						 float* force_energy4, int get_energy, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_restraint_forces: no box");
		require(nr == 0 || (particle_ids && anchors4 && spring_k && pos4 && force_energy4),
				MB2_ERR_ARG, "mb2_restraint_forces: null argument");
		restraint_forces(particle_ids, reinterpret_cast<const float4*>(anchors4), spring_k, nr,
						 reinterpret_cast<const float4*>(pos4),
						 reinterpret_cast<float4*>(force_energy4), ctx->box, get_energy,
						 ctx->energy.ptr + 5, S(stream));
	});
}

int mb2_set_particle_types(mb2_context* ctx, int num_types, const float* charge,
						   const float* diffusion3, const int* pmf_offset, const int* pmf_count,
						   int n_terms, const float* terms4, const int* force_grid_id3,
						   const float* force_grid_scale3) {
	return guarded(ctx, [&] {
		require(num_types > 0 && charge && diffusion3, MB2_ERR_ARG,
				"mb2_set_particle_types: need charge and diffusion per type");
		const int T = num_types;
		std::vector<float4> dif(T), fs(T);
		std::vector<int4> fg(T);
		std::vector<int> off(T, 0), cnt(T, 0);
		for (int t = 0; t < T; ++t) {
			dif[t] = make_float4(diffusion3[3 * t], diffusion3[3 * t + 1], diffusion3[3 * t + 2], 0.f);
			fg[t] = force_grid_id3 ? make_int4(force_grid_id3[3 * t], force_grid_id3[3 * t + 1],
											   force_grid_id3[3 * t + 2], -1)
								   : make_int4(-1, -1, -1, -1);
			fs[t] = force_grid_scale3 ? make_float4(force_grid_scale3[3 * t], force_grid_scale3[3 * t + 1],
													force_grid_scale3[3 * t + 2], 0.f)
									  : make_float4(0.f, 0.f, 0.f, 0.f);
			if (pmf_offset && pmf_count) {
				off[t] = pmf_offset[t];
				cnt[t] = pmf_count[t];
				require(off[t] >= 0 && cnt[t] >= 0 && off[t] + cnt[t] <= n_terms, MB2_ERR_ARG,
						"mb2_set_particle_types: PMF term range out of bounds");
			}
		}
		std::vector<GridTermDev> tm(std::max(n_terms, 1));
		for (int k = 0; k < n_terms; ++k)
			tm[k] = GridTermDev{static_cast<int>(terms4[4 * k]), terms4[4 * k + 1],
								terms4[4 * k + 2], static_cast<int>(terms4[4 * k + 3])};
		ctx->charge.ensure(T);
		ctx->diffusion.ensure(T);
		ctx->fg_scale.ensure(T);
		ctx->fg_id.ensure(T);
		ctx->pmf_off.ensure(T);
		ctx->pmf_cnt.ensure(T);
		ctx->terms.ensure(tm.size());
		MB2_CUDA(cudaMemcpy(ctx->charge.ptr, charge, T * sizeof(float), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->diffusion.ptr, dif.data(), T * sizeof(float4), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->fg_scale.ptr, fs.data(), T * sizeof(float4), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->fg_id.ptr, fg.data(), T * sizeof(int4), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->pmf_off.ptr, off.data(), T * sizeof(int), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->pmf_cnt.ptr, cnt.data(), T * sizeof(int), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->terms.ptr, tm.data(), tm.size() * sizeof(GridTermDev),
							cudaMemcpyHostToDevice));
		ctx->types.num_types = T;
		ctx->types.charge = ctx->charge.ptr;
		ctx->types.diffusion = ctx->diffusion.ptr;
		ctx->types.pmf_offset = ctx->pmf_off.ptr;
		ctx->types.pmf_count = ctx->pmf_cnt.ptr;
		ctx->types.terms = ctx->terms.ptr;
		ctx->types.force_grid_id = ctx->fg_id.ptr;
		ctx->types.force_grid_scale = ctx->fg_scale.ptr;
		ctx->types_set = true;
	});
}

int mb2_set_grid(mb2_context* ctx, int grid_id, const float* data, const int64_t dims[3],
				 const float origin[3], const float basis_inv[9], int boundary_condition) {
	return guarded(ctx, [&] {
		require(grid_id >= 0 && grid_id < 1024, MB2_ERR_ARG, "mb2_set_grid: grid id out of range");
		require(dims && origin && basis_inv, MB2_ERR_ARG, "mb2_set_grid: null argument");
		if (static_cast<int>(ctx->host_grids.size()) <= grid_id)
			ctx->host_grids.resize(grid_id + 1, GridView{nullptr, {0, 0, 0}, {0}, {0, 0, 0}, 0});
		GridView g{};
		g.data = data;
		for (int a = 0; a < 3; ++a) {
			require(dims[a] > 0, MB2_ERR_ARG, "mb2_set_grid: dimensions must be positive");
			g.origin[a] = origin[a];
			g.dims[a] = dims[a];
		}
		for (int k = 0; k < 9; ++k) g.basis_inv[k] = basis_inv[k];
		g.boundary_condition = boundary_condition;
		ctx->host_grids[grid_id] = g;
		ctx->grids.ensure(ctx->host_grids.size());
		MB2_CUDA(cudaMemcpy(ctx->grids.ptr, ctx->host_grids.data(),
							ctx->host_grids.size() * sizeof(GridView), cudaMemcpyHostToDevice));
		ctx->types.grids = ctx->grids.ptr;
		ctx->types.num_grids = static_cast<int>(ctx->host_grids.size());
	});
}

int mb2_bd_integrate(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
					 const uint32_t* flags, uint32_t n, float dt, float kT, uint64_t step,
					 uint64_t base_seed, uint32_t base_ctr, const float efield[3],
					 void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_bd_integrate: no box");
		require(ctx->types_set, MB2_ERR_STATE, "mb2_bd_integrate: call mb2_set_particle_types");
		require(n == 0 || (pos4 && force_energy4 && type_ids), MB2_ERR_ARG,
				"mb2_bd_integrate: null argument");
		BdParams p{dt, kT, static_cast<uint32_t>(step), base_seed, base_ctr,
				   {efield ? efield[0] : 0.f, efield ? efield[1] : 0.f, efield ? efield[2] : 0.f}};
		bd_integrate(reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(force_energy4),
					 type_ids, flags, n, ctx->types, ctx->box, p, S(stream));
	});
}

int mb2_reorder_begin(mb2_context* ctx, const float* pos4, uint32_t n, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->box_set, MB2_ERR_STATE, "mb2_reorder_begin: call mb2_set_box first");
		require(n == 0 || pos4, MB2_ERR_ARG, "mb2_reorder_begin: null positions");
		require(n <= ctx->max_particles, MB2_ERR_CAPACITY,
				"mb2_reorder_begin: more particles than the context was created for");
		float bmin[3], bmax[3];
		for (int a = 0; a < 3; ++a) {
			bmin[a] = ctx->box.origin[a];
			bmax[a] = ctx->box.origin[a] + ctx->box.size[a];
			require(bmax[a] > bmin[a], MB2_ERR_ARG, "mb2_reorder_begin: degenerate Morton box");
		}
		const cudaStream_t st = S(stream);
		ctx->ro_keys.ensure(n);
		ctx->ro_s2o.ensure(n);
		ctx->ro_inv.ensure(n);
		morton_encode(reinterpret_cast<const float4*>(pos4), n, bmin, bmax, ctx->ro_keys.ptr,
					  ctx->ro_s2o.ptr, st);
		radix_sort_pairs(ctx->scratch, ctx->ro_keys.ptr, ctx->ro_s2o.ptr, n, st);
		inverse_and_gather(ctx->ro_s2o.ptr, n, reinterpret_cast<const float4*>(pos4),
						   ctx->ro_inv.ptr, nullptr, st);
		ctx->ro_n = n;
		ctx->built = false;  // every stored particle index changes: rebuild before use
		ctx->win.valid = false;
	});
}

int mb2_reorder_apply(mb2_context* ctx, void* data, uint32_t elem_bytes, uint32_t n, void* stream) {
	return guarded(ctx, [&] {
		require(n == ctx->ro_n, MB2_ERR_STATE,
				"mb2_reorder_apply: n differs from the last mb2_reorder_begin");
		require(elem_bytes == 4 || elem_bytes == 16, MB2_ERR_ARG,
				"mb2_reorder_apply: elements of 4 or 16 bytes");
		require(n == 0 || data, MB2_ERR_ARG, "mb2_reorder_apply: null data");
		if (n == 0) return;
		const cudaStream_t st = S(stream);
		ctx->ro_tmp.ensure(n);
		MB2_CUDA(cudaMemcpyAsync(ctx->ro_tmp.ptr, data, static_cast<size_t>(n) * elem_bytes,
								 cudaMemcpyDeviceToDevice, st));
		permute_gather(ctx->ro_tmp.ptr, ctx->ro_s2o.ptr, n, static_cast<int>(elem_bytes), data, st);
	});
}

int mb2_reorder_remap(mb2_context* ctx, int* indices, uint64_t count, void* stream) {
	return guarded(ctx, [&] {
		require(count == 0 || indices, MB2_ERR_ARG, "mb2_reorder_remap: null indices");
		require(ctx->ro_inv.ptr || ctx->ro_n == 0, MB2_ERR_STATE,
				"mb2_reorder_remap: call mb2_reorder_begin first");
		remap_indices(indices, count, ctx->ro_inv.ptr, ctx->ro_n, S(stream));
	});
}

int mb2_reorder_inverse(mb2_context* ctx, uint32_t* inverse_out, uint32_t n, void* stream) {
	return guarded(ctx, [&] {
		require(n == ctx->ro_n, MB2_ERR_STATE,
				"mb2_reorder_inverse: n differs from the last mb2_reorder_begin");
		require(n == 0 || inverse_out, MB2_ERR_ARG, "mb2_reorder_inverse: null output");
		if (n == 0) return;
		MB2_CUDA(cudaMemcpyAsync(inverse_out, ctx->ro_inv.ptr, static_cast<size_t>(n) * 4,
								 cudaMemcpyDeviceToDevice, S(stream)));
	});
}

int mb2_set_langevin_types(mb2_context* ctx, int num_types, const float* mass,
						   const float* damping3) {
	return guarded(ctx, [&] {
		require(num_types > 0 && mass && damping3, MB2_ERR_ARG,
				"mb2_set_langevin_types: need mass and damping per type");
		require(ctx->types_set && num_types == ctx->types.num_types, MB2_ERR_STATE,
				"mb2_set_langevin_types: call mb2_set_particle_types first, same type count");
		std::vector<float4> d(num_types);
		for (int t = 0; t < num_types; ++t) {
			require(mass[t] > 0.0f, MB2_ERR_ARG, "mb2_set_langevin_types: masses must be positive");
			d[t] = make_float4(damping3[3 * t], damping3[3 * t + 1], damping3[3 * t + 2], 0.0f);
		}
		ctx->mass.ensure(num_types);
		ctx->damping.ensure(num_types);
		MB2_CUDA(cudaMemcpy(ctx->mass.ptr, mass, num_types * sizeof(float), cudaMemcpyHostToDevice));
		MB2_CUDA(cudaMemcpy(ctx->damping.ptr, d.data(), num_types * sizeof(float4),
							cudaMemcpyHostToDevice));
		ctx->types.mass = ctx->mass.ptr;
		ctx->types.damping = ctx->damping.ptr;
		ctx->langevin_types = num_types;
	});
}

int mb2_baoab_integrate(mb2_context* ctx, float* pos4, float* mom4, float* force_energy4,
						const int* type_ids, const uint32_t* flags, uint32_t n, float dt, float kT,
						uint64_t step, uint64_t base_seed, uint32_t base_ctr, const float efield[3],
						int deferred_kick_pending, void* stream) {
	return guarded(ctx, [&] {
		require(n == 0 || (pos4 && mom4 && force_energy4 && type_ids), MB2_ERR_ARG,
				"mb2_baoab_integrate: null argument");
		require(ctx->box_set && ctx->types_set, MB2_ERR_STATE,
				"mb2_baoab_integrate: call mb2_set_box and mb2_set_particle_types");
		require(ctx->langevin_types == ctx->types.num_types, MB2_ERR_STATE,
				"mb2_baoab_integrate: call mb2_set_langevin_types");
		const float zero[3] = {0.0f, 0.0f, 0.0f};
		baoab_integrate(reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(mom4),
						reinterpret_cast<float4*>(force_energy4), type_ids, flags, n, ctx->types,
						ctx->box, dt, kT, static_cast<uint32_t>(step), base_seed, base_ctr,
						efield ? efield : zero, deferred_kick_pending, S(stream));
	});
}

int mb2_baoab_last_update(mb2_context* ctx, float* mom4, const float* force_energy4,
						  const uint32_t* flags, uint32_t n, float dt, void* stream) {
	return guarded(ctx, [&] {
		require(n == 0 || (mom4 && force_energy4), MB2_ERR_ARG,
				"mb2_baoab_last_update: null argument");
		baoab_last_update(reinterpret_cast<float4*>(mom4),
						  reinterpret_cast<const float4*>(force_energy4), flags, n, dt, S(stream));
	});
}

uint64_t mb2_bd_seed(uint64_t seed, uint64_t patch_id, uint64_t step) {
	return (seed * 0x9E3779B97F4A7C15ULL) ^ (patch_id << 32) ^ (step * 0xBF58476D1CE4E5B9ULL);
}

int mb2_philox(mb2_context* ctx, uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2,
			   uint32_t n, uint32_t* out4, float* normals4, void* stream) {
	return guarded(ctx, [&] { philox_draws(seed, ctr0, ctr1, ctr2, n, out4, normals4, S(stream)); });
}

}  // extern "C"

namespace {

void check_step(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
				uint32_t n, const mb2_step_params* prm, const char* what) {
	require(prm && (n == 0 || (pos4 && force_energy4 && type_ids)), MB2_ERR_ARG,
			std::string(what) + ": null argument");
	require(ctx->types_set, MB2_ERR_STATE, std::string(what) + ": call mb2_set_particle_types");
	require(prm->num_dihedrals == 0 || ctx->bonded_count[2] > 0, MB2_ERR_STATE,
			std::string(what) + ": dihedrals without dihedral tables");
	require(prm->integrator == 0 || prm->integrator == 1, MB2_ERR_ARG,
			std::string(what) + ": integrator is 0 (BD) or 1 (Langevin)");
	require(prm->integrator == 0 || (prm->mom4 && ctx->langevin_types > 0), MB2_ERR_STATE,
			std::string(what) + ": Langevin needs momenta and mb2_set_langevin_types");
}

// One whole step (the body of mb2_step).
void step_once(mb2_context* ctx, float4* pos, float4* fe, const int* type_ids,
			   const uint32_t* flags, uint32_t n, uint64_t step, const mb2_step_params* prm,
			   cudaStream_t st) {
	StageScope whole(ctx, MB2_STAGE_STEP, st);
	// The reference clears ForceEnergy (Patch.cpp:56) and accumulates every
	// term into it. Here pair forces stay in the Z-ordered accumulator and
	// the integrate kernel gathers them, adding what the bonded kernels
	// wrote; ForceEnergy is cleared only when those run.
	const bool bonded = step_has_bonded(prm);
	// Rebuild schedule and skin check (Patch.cpp:86-108)
	const bool at_period = prm->rebuild_period == 0 || (step - 1) % prm->rebuild_period == 0;
	bool rebuild = at_period || !ctx->built || ctx->built_n != n;
	const float skin = prm->pairlist_cutoff - prm->cutoff;
	if (rebuild && prm->rebuild_period != 0 && ctx->built && ctx->built_n == n && skin > 0.0f)
		rebuild = max_disp(ctx, pos, n, st) > skin * 0.5f;
	if (rebuild) {
		if (bonded) MB2_CUDA(cudaMemsetAsync(fe, 0, static_cast<size_t>(n) * sizeof(float4), st));
		build(ctx, pos, type_ids, n, prm->pairlist_cutoff, prm->cutoff, st);  // packs sorted_pos
	} else if (n) {
		// The pack also clears the pair-force accumulator and, when bonded
		// terms run, ForceEnergy.
		pack_sorted_positions(pos, type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st, nullptr,
							  sorted_forces(ctx, n), bonded ? fe : nullptr, track_of(ctx));
	}
	if (n == 0) return;
	pair_kernel(ctx, n, prm->cutoff, prm->get_energy, st, !rebuild);
	bonded_stage(ctx, pos, fe, prm, prm->get_energy, st);
	StageScope scope(ctx, MB2_STAGE_INTEGRATE, st);
	if (prm->integrator == 1) {
		// Patch::integrate_motion, Langevin branch (Patch.cpp:290-335).
		baoab_integrate_gather(pos, reinterpret_cast<float4*>(prm->mom4), fe,
							   ctx->force_sorted.ptr, ctx->inv.ptr, bonded ? 1 : 0, type_ids, flags,
							   n, ctx->types, ctx->box, prm->dt, prm->kT,
							   static_cast<uint32_t>(step),
							   mb2_bd_seed(prm->seed, prm->patch_id, step), 0u, prm->efield,
							   prm->deferred_kick_pending ? 1 : 0, st);
		return;
	}
	BdParams p{prm->dt, prm->kT, static_cast<uint32_t>(step),
			   mb2_bd_seed(prm->seed, prm->patch_id, step), 0u,
			   {prm->efield[0], prm->efield[1], prm->efield[2]}};
	bd_integrate_gather(pos, fe, ctx->force_sorted.ptr, ctx->inv.ptr, type_ids, flags, n,
						ctx->types, ctx->box, p, bonded ? 1 : 0, st);
}

// A BD step that is not a rebuild check, with the step number taken from
// ctx->step_d and advanced by one at the end: the body mb2_run captures.
void step_body_replayable(mb2_context* ctx, float4* pos, float4* fe, const int* type_ids,
						  const uint32_t* flags, uint32_t n, const mb2_step_params* prm,
						  cudaStream_t st) {
	const bool bonded = step_has_bonded(prm);
	pack_sorted_positions(pos, type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st, nullptr,
						  sorted_forces(ctx, n), bonded ? fe : nullptr, track_of(ctx));
	pair_kernel(ctx, n, prm->cutoff, prm->get_energy, st, true);
	bonded_stage(ctx, pos, fe, prm, prm->get_energy, st);
	BdParams p{prm->dt, prm->kT, 0u, 0u, 0u, {prm->efield[0], prm->efield[1], prm->efield[2]}};
	bd_integrate_gather(pos, fe, ctx->force_sorted.ptr, ctx->inv.ptr, type_ids, flags, n,
						ctx->types, ctx->box, p, bonded ? 1 : 0, st, ctx->step_d.ptr, prm->seed,
						prm->patch_id);
	step_counter_add(ctx->step_d.ptr, 1, st);
}

uint64_t fbits(float f) {
	uint32_t u;
	std::memcpy(&u, &f, 4);
	return u;
}

template <class T>
void push_words(std::vector<uint64_t>& k, const T& v) {
	static_assert(sizeof(T) % 4 == 0, "word-sized fields only");
	uint32_t w[sizeof(T) / 4];
	std::memcpy(w, &v, sizeof(T));
	for (uint32_t x : w) k.push_back(x);
}

// Every value the captured step body bakes into its launches.
std::vector<uint64_t> run_graph_key(const mb2_context* ctx, const float4* pos, const float4* fe,
									const int* type_ids, const uint32_t* flags, uint32_t n,
									const mb2_step_params* prm) {
	auto P = [](const void* p) { return static_cast<uint64_t>(reinterpret_cast<uintptr_t>(p)); };
	std::vector<uint64_t> k = {
		P(pos), P(fe), P(type_ids), P(flags), n, fbits(prm->cutoff), fbits(prm->dt),
		fbits(prm->kT), prm->seed, prm->patch_id, fbits(prm->efield[0]), fbits(prm->efield[1]),
		fbits(prm->efield[2]), static_cast<uint64_t>(prm->get_energy), P(prm->bonds2),
		P(prm->bond_table_idx), prm->num_bonds, P(prm->angles4), P(prm->angle_table_idx),
		prm->num_angles, P(prm->dihedrals4), P(prm->dihedral_table_idx), prm->num_dihedrals,
		P(prm->restraint_ids), P(prm->restraint_anchors4), P(prm->restraint_k),
		prm->num_restraints, P(ctx->nbr.ptr), P(ctx->row_len.ptr), ctx->cap,
		static_cast<uint64_t>(ctx->lanes), P(ctx->sorted_pos.ptr), P(ctx->s2o.ptr),
		P(ctx->inv.ptr), P(ctx->force_sorted.ptr), P(ctx->energy.ptr), P(ctx->step_d.ptr),
		P(ctx->bonded_tables[0].ptr), P(ctx->bonded_tables[1].ptr), P(ctx->bonded_tables[2].ptr),
		static_cast<uint64_t>(ctx->pt.num_types), ctx->pt.total_bins, P(ctx->pt.refs),
		P(ctx->pt.offsets), static_cast<uint64_t>(ctx->pt.uniform), fbits(ctx->pt.uniform_ref.start),
		fbits(ctx->pt.uniform_ref.step_inv), static_cast<uint64_t>(ctx->pt.uniform_ref.last),
		P(ctx->pt.bin_force), P(ctx->pt.bin_energy), P(ctx->pt.terms),
		static_cast<uint64_t>(ctx->types.num_types), P(ctx->types.charge), P(ctx->types.diffusion),
		P(ctx->types.pmf_offset), P(ctx->types.pmf_count), P(ctx->types.terms),
		P(ctx->types.force_grid_id), P(ctx->types.force_grid_scale), P(ctx->types.grids),
		static_cast<uint64_t>(ctx->types.num_grids), P(ctx->ref_sorted.ptr), P(ctx->d2max.ptr),
		fbits(ctx->track_rc)};
	push_words(k, ctx->pt.solvent);
	push_words(k, ctx->box);
	return k;
}

}  // namespace

extern "C" {

int mb2_step(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
			 const uint32_t* flags, uint32_t n, uint64_t step, const mb2_step_params* prm,
			 void* stream) {
	return guarded(ctx, [&] {
		check_step(ctx, pos4, force_energy4, type_ids, n, prm, "mb2_step");
		step_once(ctx, reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(force_energy4),
				  type_ids, flags, n, step, prm, S(stream));
	});
}

int mb2_run(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
			const uint32_t* flags, uint32_t n, uint64_t first_step, uint32_t num_steps,
			const mb2_step_params* prm, void* stream) {
	return guarded(ctx, [&] {
		check_step(ctx, pos4, force_energy4, type_ids, n, prm, "mb2_run");
		const cudaStream_t st = S(stream);
		float4* pos = reinterpret_cast<float4*>(pos4);
		float4* fe = reinterpret_cast<float4*>(force_energy4);
		// Graph replay serves BD steps that are not rebuild checks; the rest (and
		// every step while per-stage profiling is on) run as mb2_step does.
		const bool replayable = prm->integrator == 0 && prm->rebuild_period != 0 && n > 0;
		ctx->step_d.ensure(1);
		bool counter_set = false;
		for (uint32_t k = 0; k < num_steps; ++k) {
			const uint64_t step = first_step + k;
			const bool check = (step - 1) % (prm->rebuild_period ? prm->rebuild_period : 1) == 0;
			if (!replayable || check || ctx->profiling || !ctx->built || ctx->built_n != n) {
				step_once(ctx, pos, fe, type_ids, flags, n, step, prm, st);
				counter_set = false;
				continue;
			}
			ctx->force_sorted.ensure(n);  // no allocation inside the capture
			const std::vector<uint64_t> key = run_graph_key(ctx, pos, fe, type_ids, flags, n, prm);
			if (!ctx->run_graph || key != ctx->run_key) {
				if (ctx->run_graph) {
					MB2_CUDA(cudaGraphExecDestroy(ctx->run_graph));
					ctx->run_graph = nullptr;
				}
				cudaStream_t cs;
				MB2_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
				cudaGraph_t g = nullptr;
				const unsigned long long l0 = g_launches;
				MB2_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
				try {
					step_body_replayable(ctx, pos, fe, type_ids, flags, n, prm, cs);
				} catch (...) {
					cudaStreamEndCapture(cs, &g);
					if (g) cudaGraphDestroy(g);
					cudaStreamDestroy(cs);
					g_launches = l0;
					throw;
				}
				const cudaError_t ec = cudaStreamEndCapture(cs, &g);
				ctx->run_launches = g_launches - l0;
				g_launches = l0;  // counted at each replay instead
				cudaStreamDestroy(cs);
				MB2_CUDA(ec);
				const cudaError_t ei = cudaGraphInstantiate(&ctx->run_graph, g, 0);
				cudaGraphDestroy(g);
				MB2_CUDA(ei);
				ctx->run_key = key;
			}
			if (!counter_set) {
				step_counter_set(ctx->step_d.ptr, step, st);
				counter_set = true;
			}
			MB2_CUDA(cudaGraphLaunch(ctx->run_graph, st));
			g_launches += ctx->run_launches;
		}
	});
}

int mb2_window_forward(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
					   uint32_t n, uint64_t first_step, uint32_t num_steps,
					   uint32_t checkpoint_every, const mb2_step_params* prm, void* stream) {
	return guarded(ctx, [&] {
		require(prm && n > 0 && pos4 && force_energy4 && type_ids, MB2_ERR_ARG,
				"mb2_window_forward: null argument");
		require(ctx->types_set && ctx->types.num_grids == 0, MB2_ERR_STATE,
				"mb2_window_forward: particle types without grids are required");
		require(!matrix_has_analytical(ctx) && prm->num_dihedrals == 0 &&
					prm->num_restraints == 0 && prm->integrator == 0,
				MB2_ERR_STATE,
				"mb2_window_forward: BD with tabulated pair, bond and angle terms only");
		require(checkpoint_every > 0 && prm->rebuild_period > 0 &&
					prm->rebuild_period % checkpoint_every == 0 &&
					(first_step - 1) % checkpoint_every == 0,
				MB2_ERR_ARG,
				"mb2_window_forward: checkpoint_every must divide rebuild_period and the "
				"window must start on a checkpoint (first_step - 1 a multiple of it)");
		const cudaStream_t st = S(stream);
		float4* pos = reinterpret_cast<float4*>(pos4);
		float4* fe = reinterpret_cast<float4*>(force_energy4);
		const uint32_t segs = (num_steps + checkpoint_every - 1) / checkpoint_every;
		ctx->ckpt.ensure(static_cast<size_t>(std::max<uint32_t>(segs, 1)) * n);
		for (uint32_t sgi = 0; sgi < segs; ++sgi) {
			const uint32_t k0 = sgi * checkpoint_every;
			const uint32_t k1 = std::min(num_steps, k0 + checkpoint_every);
			copy4(ctx->ckpt.ptr + static_cast<size_t>(sgi) * n, pos, n, st);
			build(ctx, pos, type_ids, n, prm->pairlist_cutoff, prm->cutoff, st);
			for (uint32_t k = k0; k < k1; ++k)
				window_step(ctx, pos, fe, type_ids, n, first_step + k, prm, st);
		}
		ctx->win.valid = true;
		ctx->win.n = n;
		ctx->win.num_steps = num_steps;
		ctx->win.every = checkpoint_every;
		ctx->win.first_step = first_step;
		ctx->win.prm = *prm;
		ctx->win.type_ids = type_ids;
	});
}

int mb2_window_record_states(mb2_context* ctx, float* out4, uint64_t capacity_rows) {
	return guarded(ctx, [&] {
		ctx->record_states = reinterpret_cast<float4*>(out4);
		ctx->record_cap = out4 ? capacity_rows : 0;
	});
}

int mb2_window_checkpoints(mb2_context* ctx, float* out4, uint64_t capacity_rows, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->win.valid, MB2_ERR_STATE, "mb2_window_checkpoints: no forward window");
		const uint32_t segs = (ctx->win.num_steps + ctx->win.every - 1) / ctx->win.every;
		const uint64_t rows = static_cast<uint64_t>(segs) * ctx->win.n;
		require(capacity_rows >= rows && out4, MB2_ERR_CAPACITY,
				"mb2_window_checkpoints: output smaller than checkpoints x particles");
		MB2_CUDA(cudaMemcpyAsync(out4, ctx->ckpt.ptr, rows * sizeof(float4),
								 cudaMemcpyDeviceToDevice, S(stream)));
	});
}

int mb2_window_backward(mb2_context* ctx, const float* grad_final4, float* grad_pos0_4,
						double* grad_pair_bins, double* grad_bond_bins, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->win.valid, MB2_ERR_STATE, "mb2_window_backward: no forward window");
		require(grad_final4 && grad_pos0_4 && grad_pair_bins, MB2_ERR_ARG,
				"mb2_window_backward: null argument");
		const auto& w = ctx->win;
		const mb2_step_params* prm = &w.prm;
		require(prm->num_bonds == 0 || grad_bond_bins, MB2_ERR_ARG,
				"mb2_window_backward: bond-table gradient output needed");
		const cudaStream_t st = S(stream);
		const uint32_t n = w.n, C = w.every;
		const uint32_t segs = (w.num_steps + C - 1) / C;
		require(!ctx->record_states ||
					ctx->record_cap >= static_cast<uint64_t>(w.num_steps) * n,
				MB2_ERR_CAPACITY,
				"mb2_window_backward: the recorded-states buffer holds fewer than steps x n rows");
		ctx->states.ensure(static_cast<size_t>(C) * n);
		for (auto* b : {&ctx->wpos, &ctx->wfe, &ctx->lam, &ctx->mu, &ctx->mu_sorted})
			b->ensure(n);
		ctx->adj_tan.ensure(n);
		ctx->adj_tan_sorted.ensure(n);
		copy4(ctx->lam.ptr, reinterpret_cast<const float4*>(grad_final4), n, st);
		AdjointStepArgs a{};
		a.n = n;
		a.type_ids = w.type_ids;
		a.diffusion = ctx->types.diffusion;
		a.dt_over_kT = prm->dt / prm->kT;
		a.tables = ctx->pt;
		a.box = ctx->box;
		a.cutoff_sq = prm->cutoff > 0.0f ? prm->cutoff * prm->cutoff : 0.0f;
		a.bonds = reinterpret_cast<const int2*>(prm->bonds2);
		a.bond_table_idx = prm->bond_table_idx;
		a.num_bonds = prm->num_bonds;
		a.bond_tables = ctx->bonded_tables[0].ptr;
		a.bond_values_base = ctx->bonded_values[0].ptr;
		a.bond_bins = ctx->bonded_bins[0];
		a.angles = reinterpret_cast<const int4*>(prm->angles4);
		a.angle_table_idx = prm->angle_table_idx;
		a.num_angles = prm->num_angles;
		a.angle_tables = ctx->bonded_tables[1].ptr;
		a.lam = ctx->lam.ptr;
		a.mu = ctx->mu.ptr;
		a.mu_sorted = ctx->mu_sorted.ptr;
		a.tan = ctx->adj_tan.ptr;
		a.tan_sorted = ctx->adj_tan_sorted.ptr;
		a.grad_pair = grad_pair_bins;
		a.grad_bond = grad_bond_bins;
		for (uint32_t sgi = segs; sgi-- > 0;) {
			const uint32_t k0 = sgi * C;
			const uint32_t k1 = std::min(w.num_steps, k0 + C);
			// Recompute the segment from its checkpoint, keeping every state.
			copy4(ctx->wpos.ptr, ctx->ckpt.ptr + static_cast<size_t>(sgi) * n, n, st);
			build(ctx, ctx->wpos.ptr, w.type_ids, n, prm->pairlist_cutoff, prm->cutoff, st);
			for (uint32_t k = k0; k < k1; ++k) {
				copy4(ctx->states.ptr + static_cast<size_t>(k - k0) * n, ctx->wpos.ptr, n, st);
				if (k + 1 < k1)
					window_step(ctx, ctx->wpos.ptr, ctx->wfe.ptr, w.type_ids, n, w.first_step + k,
								prm, st);
			}
			if (ctx->record_states)
				MB2_CUDA(cudaMemcpyAsync(ctx->record_states + static_cast<size_t>(k0) * n,
										 ctx->states.ptr,
										 static_cast<size_t>(k1 - k0) * n * sizeof(float4),
										 cudaMemcpyDeviceToDevice, st));
			a.lanes = ctx->lanes;
			a.cap = ctx->cap;
			a.inv = ctx->inv.ptr;
			a.nbr = ctx->nbr.ptr;
			a.row_len = ctx->row_len.ptr;
			a.sorted_pos = ctx->sorted_pos.ptr;
			for (uint32_t k = k1; k-- > k0;) {
				const float4* xk = ctx->states.ptr + static_cast<size_t>(k - k0) * n;
				pack_sorted_positions(xk, w.type_ids, ctx->s2o.ptr, n, ctx->sorted_pos.ptr, st);
				a.pos = xk;
				adjoint_step(a, st);
			}
		}
		copy4(reinterpret_cast<float4*>(grad_pos0_4), ctx->lam.ptr, n, st);
		ctx->win.valid = true;
	});
}

int mb2_rdf_histogram(mb2_context* ctx, const float* pos4, const int* type_ids, uint32_t n,
					  uint32_t num_bins, float bin_width, float r_max, float sigma, double* hist,
					  void* stream) {
	return guarded(ctx, [&] {
		require(n > 0 && pos4 && type_ids && hist && num_bins > 0 && num_bins <= 4096 &&
					bin_width > 0.0f && sigma > 0.0f && r_max > 0.0f,
				MB2_ERR_ARG, "mb2_rdf_histogram: bad arguments");
		const cudaStream_t st = S(stream);
		build(ctx, reinterpret_cast<const float4*>(pos4), type_ids, n, r_max, 0.0f, st);
		MB2_CUDA(cudaMemsetAsync(hist, 0, num_bins * sizeof(double), st));
		rdf_pairs(ctx->sorted_pos.ptr, ctx->nbr.ptr, ctx->row_len.ptr, n, ctx->cap, ctx->lanes,
				  ctx->box, num_bins, bin_width, r_max, sigma, hist, nullptr, nullptr, st);
		ctx->rdf_built = true;
		ctx->rdf_n = n;
	});
}

int mb2_rdf_backward(mb2_context* ctx, const float* pos4, uint32_t n, uint32_t num_bins,
					 float bin_width, float r_max, float sigma, const double* dl_dhist,
					 float* grad4, void* stream) {
	return guarded(ctx, [&] {
		require(ctx->rdf_built && ctx->rdf_n == n, MB2_ERR_STATE,
				"mb2_rdf_backward: call mb2_rdf_histogram on these positions first");
		require(pos4 && dl_dhist && grad4 && num_bins > 0 && num_bins <= 4096, MB2_ERR_ARG,
				"mb2_rdf_backward: bad arguments");
		const cudaStream_t st = S(stream);
		ctx->tan_sorted.ensure(n);
		MB2_CUDA(cudaMemsetAsync(ctx->tan_sorted.ptr, 0, static_cast<size_t>(n) * sizeof(float4), st));
		rdf_pairs(ctx->sorted_pos.ptr, ctx->nbr.ptr, ctx->row_len.ptr, n, ctx->cap, ctx->lanes,
				  ctx->box, num_bins, bin_width, r_max, sigma, nullptr, dl_dhist,
				  ctx->tan_sorted.ptr, st);
		gather_add(reinterpret_cast<float4*>(grad4), ctx->tan_sorted.ptr, ctx->inv.ptr, n, st);
	});
}

uint64_t mb2_launch_count(void) { return g_launches; }

int mb2_set_profiling(mb2_context* ctx, int on) {
	return guarded(ctx, [&] { ctx->profiling = on != 0; });
}

int mb2_profile_read(mb2_context* ctx, int stage, double* total_ms, uint32_t* count) {
	return guarded(ctx, [&] {
		require(stage >= 0 && stage < MB2_NUM_STAGES && total_ms && count, MB2_ERR_ARG,
				"mb2_profile_read: bad stage or null output");
		double t = 0.0;
		for (auto& be : ctx->prof[stage]) {
			MB2_CUDA(cudaEventSynchronize(be.second));
			float ms = 0.0f;
			MB2_CUDA(cudaEventElapsedTime(&ms, be.first, be.second));
			t += ms;
			cudaEventDestroy(be.first);
			cudaEventDestroy(be.second);
		}
		*total_ms = t;
		*count = static_cast<uint32_t>(ctx->prof[stage].size());
		ctx->prof[stage].clear();
	});
}

int mb2_set_cell_level_offset(mb2_context* ctx, int offset) {
	return guarded(ctx, [&] {
		require(offset >= -2 && offset <= 2, MB2_ERR_ARG,
				"mb2_set_cell_level_offset: offset in -2..2");
		if (offset != ctx->level_offset) {
			ctx->level_offset = offset;
			ctx->grid_valid = false;
			ctx->built = false;
		}
	});
}

int mb2_cell_level(mb2_context* ctx, int* level) {
	return guarded(ctx, [&] {
		require(level != nullptr, MB2_ERR_ARG, "mb2_cell_level: null output");
		*level = ctx->grid_valid ? ctx->grid.m : -1;
	});
}

int mb2_set_lanes_per_row(mb2_context* ctx, int lanes) {
	return guarded(ctx, [&] {
		require(lanes == 0 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32, MB2_ERR_ARG,
				"mb2_set_lanes_per_row: 0, 4, 8, 16 or 32");
		if (lanes != ctx->lanes_request) {
			// The list layout depends on the lanes per row: re-size at the next build.
			ctx->lanes_request = lanes;
			ctx->cap = 0;
			ctx->lanes = 0;
			ctx->built = false;
		}
	});
}

}  // extern "C"
