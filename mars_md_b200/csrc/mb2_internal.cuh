// Internal declarations shared by the CUDA translation units of libmarsb200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "mb2_common.cuh"

namespace mb2 {

// Count of kernels this library has launched (for launch accounting).
extern unsigned long long g_launches;
#define MB2_LAUNCH ++::mb2::g_launches,

// Thrown inside the library, turned into a status code at the C boundary.
struct Error {
	int code;
	std::string msg;
};

#define MB2_CUDA(call)                                                                  \
	do {                                                                                \
		cudaError_t e_ = (call);                                                        \
		if (e_ != cudaSuccess)                                                          \
			throw ::mb2::Error{2, std::string(#call) + ": " + cudaGetErrorString(e_)};   \
	} while (0)

// Throws Error{code, msg} unless cond holds.
inline void expect_arg(bool cond, int code, const char* msg) {
	if (!cond) throw Error{code, msg};
}

// Device buffer that only grows; owned by a context.
template <typename T>
struct DevBuf {
	T* ptr = nullptr;
	size_t cap = 0;
	DevBuf() = default;
	DevBuf(const DevBuf&) = delete;
	DevBuf& operator=(const DevBuf&) = delete;
	~DevBuf() { release(); }
	void ensure(size_t n) {
		if (n <= cap) return;
		if (ptr) cudaFree(ptr);
		ptr = nullptr;
		cap = 0;
		const size_t want = n < 16 ? 16 : n;
		MB2_CUDA(cudaMalloc(&ptr, want * sizeof(T)));
		cap = want;
	}
	void release() {
		if (ptr) cudaFree(ptr);
		ptr = nullptr;
		cap = 0;
	}
};

// Context-owned scratch for sorting and scanning.
struct Scratch {
	DevBuf<uint32_t> keys_alt, vals_alt, hist, scan_blocks;
	uint32_t* sort_keys_alt = nullptr;
	uint32_t* sort_vals_alt = nullptr;
	uint32_t* sort_hist = nullptr;
	void ensure_sort(size_t n, size_t hist_n) {
		keys_alt.ensure(n);
		vals_alt.ensure(n);
		hist.ensure(hist_n);
		sort_keys_alt = keys_alt.ptr;
		sort_vals_alt = vals_alt.ptr;
		sort_hist = hist.ptr;
	}
	void release() {
		keys_alt.release();
		vals_alt.release();
		hist.release();
		scan_blocks.release();
	}
};

// One entry of the cell stencil: offsets to add to the home cell; pad holds
// the same offsets modulo 2^m interleaved into Morton bit positions.
struct StencilEntry {
	int dx, dy, dz, pad;
};

// sort.cu
void morton_encode(const float4* pos, uint32_t n, const float* bmin, const float* bmax,
				   uint32_t* keys, uint32_t* idx, cudaStream_t st);
void radix_sort_pairs(Scratch& s, uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st);
void inverse_and_gather(const uint32_t* s2o, uint32_t n, const float4* pos, uint32_t* inv,
						float4* sorted_pos, cudaStream_t st);
// out[s] = in[s2o[s]] for elements of 4 or 16 bytes.
void permute_gather(const void* in, const uint32_t* s2o, uint32_t n, int elem_bytes, void* out,
					cudaStream_t st);
// idx[i] = inv[idx[i]] where 0 <= idx[i] < n (others unchanged).
void remap_indices(int* idx, size_t count, const uint32_t* inv, uint32_t n, cudaStream_t st);
// Elements per radix-sort tile; the digit histogram holds 256 words per tile.
constexpr uint32_t kSortTile = 2048;
// Radix sort with caller-supplied scratch: keys_alt and vals_alt of n words,
// hist of 256 * ceil(n / kSortTile) words, block_sums of
// scan_blocks_needed(that) words. Nothing there needs to start at zero.
void radix_sort_pairs_into(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t* keys_alt,
						   uint32_t* vals_alt, uint32_t* hist, uint32_t* block_sums,
						   cudaStream_t st);
// noalloc.cu: the same sort over the library's static scratch (no allocation).
void radix_sort_pairs_static(uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st);

// scan.cu: exclusive prefix sum of n u32 values (in == out allowed). If
// total is non-null the grand total is stored there (device pointer).
void exclusive_scan_u32(Scratch& s, const uint32_t* in, uint32_t* out, size_t n, uint32_t* total,
						cudaStream_t st);
size_t scan_blocks_needed(size_t n);
void exclusive_scan_u32_into(const uint32_t* in, uint32_t* out, size_t n, uint32_t* block_sums,
							 cudaStream_t st);

// Exclusion view (src/Interactions/DeviceExclusions.h:22-75), device pointers.
struct Exclusions {
	const int* offsets = nullptr;
	const int* neighbors = nullptr;
	uint32_t num_particles = 0;
	const int* rigid_body_id = nullptr;
};

// pairlist.cu
struct CellGrid {
	int m = 0;                 // cells per axis = 2^m
	int shift = 30;            // 3 * (10 - m)
	int num_stencil = 0;
	std::vector<StencilEntry> stencil;  // one cell's pruned stencil
	int radius[3] = {0, 0, 0};          // stencil half-width in cells per axis
	float wmin[3] = {0, 0, 0};          // narrowest cell width per axis
	float lim = 0.0f;                   // pruning bound on the squared cell gap
};
// Up to this many particles the pairlist is walked one warp per particle
// (build_rows_kernel) instead of one warp per 32 (build_walk_kernel).
// Measured per build, group walk against row walk: 65,536-bead polymers 0.75
// vs 0.30 ms; uniform beads at 0.002 A^-3, 32,768: 0.43 vs 0.34 ms (the group
// walk's best at that size); 131,072: 1.06 vs 0.75 ms; 262,144: 1.36 vs
// 1.48 ms; 524,288: 1.74 vs 2.30 ms; 2,097,152: 5.45 vs 10.6 ms.
constexpr uint32_t kRowWalkMaxN = 131072;

// Parameters of the group walk (passed by value to the kernel).
struct WalkGrid {
	int m, shift, emax;
	int full[3];               // periodic axis whose stencil spans every cell
	int radius[3];
	float wmin[3];
	float lim;
	float rc2;                 // pairlist cutoff squared, as the reference rounds it
	float fast_lo, fast_hi;    // d^2 band that needs the exact test
	float split2;              // entries with d^2 above it go to the row's far segment
	// Real-space extent of cell c on each axis: [lo + c w - eps, lo + (c+1) w + eps)
	// (Morton domain origin, cell width, rounding margin of the Morton mapping).
	float dom_lo[3], cell_w[3], eps[3];
};
// Cell level m in [m_lo, m_hi] minimising candidates plus per-cell cost; the
// widths assume the 10-bit Morton scale (conservative for coarser scales).
CellGrid choose_cell_grid(const float* extent, const int* periodic, float rc_list, size_t n,
						  int m_lo = 0, int m_hi = 8);
void fast_test_band(const Box& box, float rc_list, float* fast_lo, float* fast_hi);
void cell_ranges(const uint32_t* keys, uint32_t n, int shift, uint32_t* begin, uint32_t* end,
				 size_t num_cells, cudaStream_t st);
// One walk over all groups: rows appended to the sliced-ELL list (entries past
// `cap` are counted, not stored); stats[0] += pairs, stats[1] = max row length.
void build_walk(const float4* sorted_pos, const uint32_t* keys, const uint32_t* s2o,
				const uint32_t* begin, const uint32_t* end, const StencilEntry* stencil,
				int num_stencil, const WalkGrid& wg, uint32_t n, const Box& box,
				const Exclusions& ex, uint32_t* nbr, uint32_t cap, int hshift, uint32_t* row_len,
				uint32_t* row_far, unsigned long long* stats, cudaStream_t st);
// After a storing walk: each row's far entries moved to follow its near ones.
void join_far(uint32_t* nbr, const uint32_t* row_len, const uint32_t* row_far, uint32_t n,
			  uint32_t cap, int hshift, cudaStream_t st);
void export_pairs(const uint32_t* nbr, const uint32_t* row_len, const uint32_t* row_off,
				  const uint32_t* s2o, uint32_t n, uint32_t cap, int hshift, int2* out,
				  cudaStream_t st);
void max_displacement_sq(const float4* cur, const float4* prev, uint32_t n, const Box& box,
						 unsigned int* out_bits, cudaStream_t st);
// The largest displacement of any particle since the last pairlist build,
// kept by the step's pack: d2max (a device word) holds its square as float
// bits, raised with atomicMax and cleared at each build; +inf when a position
// is not finite or lies outside a periodic axis of the box by more than
// kTrackBand. ref_sorted: the Z-ordered positions the list was built from.
// d2max == nullptr: not tracked.
constexpr float kTrackBand = 0.5f;
struct DisplacementTrack {
	const float4* ref_sorted = nullptr;
	unsigned int* d2max = nullptr;
	float len[3] = {0.0f, 0.0f, 0.0f};  // periodic lengths (0: open axis)
	float lo[3] = {0.0f, 0.0f, 0.0f};   // box bounds widened by kTrackBand
	float hi[3] = {0.0f, 0.0f, 0.0f};
};
DisplacementTrack displacement_track(const Box& box, const float4* ref_sorted,
									 unsigned int* d2max);
// nonfinite (optional): incremented once per particle with a NaN or infinite
// coordinate.
// clear_a / clear_b (may be null): float4[n] arrays zeroed by the same launch.
// track (optional): raises track.d2max to this step's largest displacement.
void pack_sorted_positions(const float4* pos, const int* type_ids, const uint32_t* s2o,
						   uint32_t n, float4* sorted_pos, cudaStream_t st,
						   unsigned long long* nonfinite = nullptr, float4* clear_a = nullptr,
						   float4* clear_b = nullptr,
						   const DisplacementTrack& track = DisplacementTrack{});

// forces.cu
// Per type pair: the tabulated table's lookup constants and offset into the
// per-bin arrays (offset < 0: the pair has no tabulated term).
struct PairTableRef {
	float start;
	float step_inv;
	int last;    // size - 1
	int offset;  // into bin_force / bin_energy, or -1
};
// Per type pair: the analytical terms and their per-pair constants, each
// rounded as PairNonbondedComputer rounds it per pair (Pairwise.h:248-283,
// Columb.h): qq = qi * qj, a_dh = qq * COULOMB / dielectric, a_onck =
// qq * COULOMB, rad6 = (0.5 (r_a + r_b))^6, eps = sqrt(eps_a eps_b).
struct PairTermRef {
	uint32_t terms;  // analytical bits of the type pair's tag (0: none)
	float qq, a_dh, a_onck, rad6, eps;
	float pad0, pad1;
};
// Run-wide constants of the analytical terms (SolventParams,
// NonBondedInteraction.h:123-129; GaussianPotential, Pairwise.h:50-53).
struct PairSolvent {
	float dh_len, dh_inv_len;      // Debye length and RN(1 / length)
	float onck_kappa, onck_sz, onck_z, onck_two_z;
	float g_amp, g_inv_s2, g_cut2;  // Gaussian: amp, RN(1 / sigma^2), cutoff^2 (<= 0: none)
};
struct PairTables {
	int num_types = 0;
	uint32_t total_bins = 0;
	const PairTableRef* refs = nullptr;   // device [T*T]
	const float* bin_force = nullptr;     // device: -(U[k+1]-U[k]) * step_inv, 0 at k = size-1
	const float2* bin_energy = nullptr;   // device: (U[k], U[k+1]-U[k]), (U[size-1], 0) last
	const PairTermRef* terms = nullptr;   // device [T*T], or null: tabulated terms only
	PairSolvent solvent{};
	// Every type pair with a table uses tables of one start, bin width and
	// length (uniform.start / step_inv / last): the kernel then reads only
	// each type pair's offset (device [T*T], -1: no table).
	const int* offsets = nullptr;
	bool uniform = false;
	PairTableRef uniform_ref{0.0f, 0.0f, 0, -1};
};
// d2max / list_rc (optional): the displacement track of the list's build and
// its list radius. With them, rows of an all-periodic box that lie deeper
// inside the box than list_rc + 2 * sqrt(*d2max) (plus a safety band) take a
// shorter minimum-image sequence with the same result.
void pair_forces(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
				 uint32_t n, uint32_t cap, int lanes_per_row, const PairTables& t, const Box& box,
				 float cutoff_sq, int get_energy, float4* force_sorted, double* energy_virial,
				 cudaStream_t st, const unsigned int* d2max = nullptr, float list_rc = 0.0f);
// Host: per-type-pair lookup constants and per-bin force / (U0, dU) arrays of
// a set of tabulated pair tables; returns the total number of bins.
size_t pair_table_arrays(int num_types, const uint32_t* term_matrix, int num_tables,
						 const float* values, const uint32_t* sizes, const float* starts,
						 const float* step_invs, std::vector<PairTableRef>& refs,
						 std::vector<float>& bf, std::vector<float2>& be);
// Host: per-type-pair table offsets (-1: no table) and whether every type
// pair with a table uses one start, step inverse and length (compared bit for
// bit), which *u then holds (offset -1).
bool uniform_tables(const std::vector<PairTableRef>& refs, std::vector<int>& offsets,
					PairTableRef& u);
// Batched replicas: row i's box is boxes[sorted_keys[i] >> sys_shift].
void pair_forces_systems(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len,
						 uint32_t n, uint32_t cap, int lanes_per_row, const PairTables& t,
						 const Box* boxes, const uint32_t* sorted_keys, int sys_shift,
						 bool all_periodic, float cutoff_sq, int get_energy, float4* force_sorted,
						 double* ev, cudaStream_t st);
void scatter_add_forces(const float4* force_sorted, const uint32_t* s2o, uint32_t n,
						float4* force_energy, int get_energy, cudaStream_t st);
// Exhaustive device check of sqrt_rn_nr against __fsqrt_rn on [2^-60,
// FLT_MAX]: adds the mismatch count into *bad.
void selftest_sqrt(unsigned long long* bad, cudaStream_t st);
void bond_forces(const int2* bonds, const int* table_idx, uint32_t nb, const float4* pos,
				 float4* fe, const Table* tables, const Box& box, int get_energy,
				 double* energy, cudaStream_t st);
// Bonds and angles in one launch (either count may be 0).
void bond_angle_forces(const int2* bonds, const int* bond_idx, uint32_t nb, const Table* bond_tables,
					   const int4* angles, const int* angle_idx, uint32_t na,
					   const Table* angle_tables, const float4* pos, float4* fe, const Box& box,
					   int get_energy, double* bond_energy, double* angle_energy, cudaStream_t st);
void angle_forces(const int4* angles, const int* table_idx, uint32_t na, const float4* pos,
				  float4* fe, const Table* tables, const Box& box, int get_energy, double* energy,
				  cudaStream_t st);
void dihedral_forces(const int4* dihedrals, const int* table_idx, uint32_t nd, const float4* pos,
					 float4* fe, const Table* tables, const Box& box, int get_energy,
					 double* energy, cudaStream_t st);
void restraint_forces(const int* ids, const float4* anchors, const float* k_spring, uint32_t nr,
					  const float4* pos, float4* fe, const Box& box, int get_energy,
					  double* energy, cudaStream_t st);

// bd.cu
struct GridView {
	const float* data;
	float origin[3];
	float basis_inv[9];  // column-major
	long long dims[3];
	int boundary_condition;
};
struct GridTermDev {
	int grid_id;
	float scale;
	float scale_slope;
	int boundary_condition;
};
struct TypeTable {
	int num_types = 0;
	const float* charge = nullptr;          // device [T]
	const float4* diffusion = nullptr;      // device [T]
	const int* pmf_offset = nullptr;        // device [T]
	const int* pmf_count = nullptr;         // device [T]
	const GridTermDev* terms = nullptr;     // device
	const int4* force_grid_id = nullptr;    // device [T]
	const float4* force_grid_scale = nullptr;
	const GridView* grids = nullptr;        // device
	int num_grids = 0;
	const float* mass = nullptr;            // device [T], Langevin only
	const float4* damping = nullptr;        // device [T], Langevin only (x, y, z)
};
struct BdParams {
	float dt;
	float kT;
	uint32_t step;
	uint64_t base_seed;
	uint32_t base_ctr;
	float efield[3];
};
void bd_integrate(float4* pos, float4* fe, const int* type_ids, const uint32_t* flags, uint32_t n,
				  const TypeTable& types, const Box& box, const BdParams& p, cudaStream_t st);
// The fused step's integrate: force = force_sorted[inv[i]] (+ fe[i] if read_fe).
// step_ptr non-null: the step number is read from device memory at run time
// (a replayed graph) and the Philox key mixed on the device from seed and
// patch_id; p.step and p.base_seed are then unused.
void bd_integrate_gather(float4* pos, float4* fe, const float4* force_sorted, const uint32_t* inv,
						 const int* type_ids, const uint32_t* flags, uint32_t n,
						 const TypeTable& types, const Box& box, const BdParams& p, int read_fe,
						 cudaStream_t st, const unsigned long long* step_ptr = nullptr,
						 uint64_t seed = 0, uint64_t patch_id = 0);
// Langevin BAOAB (Integrator/BAOAB.h): with grids, ForceEnergy += position
// force for every particle; `pending` applies the deferred closing half-kick
// first; then B-A-O-A and wrap. Noise key (seed, base_ctr + i, step, stream 0x1356914).
void baoab_integrate(float4* pos, float4* mom, float4* fe, const int* type_ids,
					 const uint32_t* flags, uint32_t n, const TypeTable& types, const Box& box,
					 float dt, float kT, uint32_t step, uint64_t base_seed, uint32_t base_ctr,
					 const float* efield, int pending, cudaStream_t st);
// Fused-step variant: pair force gathered from the Z-ordered accumulator
// (plus ForceEnergy when read_fe), ForceEnergy left as the reference leaves it.
void baoab_integrate_gather(float4* pos, float4* mom, float4* fe, const float4* force_sorted,
							const uint32_t* inv, int read_fe, const int* type_ids,
							const uint32_t* flags, uint32_t n, const TypeTable& types,
							const Box& box, float dt, float kT, uint32_t step, uint64_t base_seed,
							uint32_t base_ctr, const float* efield, int pending, cudaStream_t st);
// BAOAB_LastUpdate: mom += 0.5 dt F (closing half-kick) for non-frozen particles.
void baoab_last_update(float4* mom, const float4* fe, const uint32_t* flags, uint32_t n,
					   float dt, cudaStream_t st);
// Batched replicas' integrate: per-system box, seed (seed + s) mixed with
// (patch_id, *step_ptr), Philox counter = index within the system.
void bd_integrate_systems(float4* pos, float4* fe, const float4* force_sorted,
						  const uint32_t* inv, const int* type_ids, const uint32_t* sys_of,
						  const uint32_t* offsets, const Box* boxes, uint32_t n,
						  const TypeTable& types, float dt, float kT, uint64_t seed,
						  uint64_t patch_id, const unsigned long long* step_ptr, cudaStream_t st);
// adjoint.cu: one reverse BD step, lambda += J(x_k)^T (c * lambda) (J symmetric:
// the directional derivative of the force along mu = c * lambda), with table
// gradients accumulated in FP64. Positions are x_k, in both orders.
struct AdjointStepArgs {
	uint32_t n;
	int lanes;
	uint32_t cap;
	const float4* pos;         // x_k, original order
	const float4* sorted_pos;  // x_k in sorted order (type id in .w)
	const int* type_ids;
	const float4* diffusion;   // per type
	float dt_over_kT;
	const uint32_t* inv;
	const uint32_t* nbr;
	const uint32_t* row_len;
	PairTables tables;
	Box box;
	float cutoff_sq;
	const int2* bonds;
	const int* bond_table_idx;
	uint32_t num_bonds;
	const Table* bond_tables;
	const float* bond_values_base;
	uint32_t bond_bins;
	const int4* angles;
	const int* angle_table_idx;
	uint32_t num_angles;
	const Table* angle_tables;
	float4* lam;  // in: lambda_{k+1}; out: lambda_k
	float4* mu;
	float4* mu_sorted;
	double4* tan;         // FP64 tangent accumulators, original order (x, y, z, unused)
	double4* tan_sorted;  // and sorted order
	double* grad_pair;  // [total pair bins], accumulated
	double* grad_bond;  // [total bond bins], accumulated
};
void adjoint_step(const AdjointStepArgs& a, cudaStream_t st);
// Smoothed pair-distance histogram over the list (grad_sorted == nullptr:
// into hist), or the gradient of sum dldh * hist into grad_sorted.
void rdf_pairs(const float4* sorted_pos, const uint32_t* nbr, const uint32_t* row_len, uint32_t n,
			   uint32_t cap, int lanes, const Box& box, uint32_t bins, float dr, float r_max,
			   float sigma, double* hist, const double* dldh, float4* grad_sorted,
			   cudaStream_t st);
// grad[o] += src_sorted[inv[o]].
void gather_add(float4* grad, const float4* src_sorted, const uint32_t* inv, uint32_t n,
				cudaStream_t st);
// Device step counter: set to `value`, or add `value` (one-thread launches).
void step_counter_set(unsigned long long* ptr, uint64_t value, cudaStream_t st);
void step_counter_add(unsigned long long* ptr, uint64_t value, cudaStream_t st);
void philox_draws(uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2, uint32_t n,
				  uint32_t* out4, float* normals4, cudaStream_t st);

}  // namespace mb2
