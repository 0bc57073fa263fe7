// Oracle harness: the reference's own hot-path functors, run on the host.
//
// TEST INFRASTRUCTURE ONLY. This file is glue written for this project; every
// computation below is done by a functor from the reference's source tree,
// included at build time from the reference checkout (see Makefile). The
// functors are compiled for the host with the shim headers in shim/ standing
// in for the reference's Backend layer and its empty fmt submodule.
//
// Race-free functors (Morton encode, cell ranges, stencil table, pair-tag
// resolve, BD integrate) may be chunked across host threads, following the
// reference's launch_cpu_kernel policy (src/Backend/Kernels.h:204-238).
// Scatter functors (neighbour emit, pair/bond/angle forces) run on one thread:
// their host atomics are plain `+=` (src/Header.h:191, src/Types/Types.h:63-175).
// The radix sort is CUB in the reference (src/PatchOperation/ZOrderKernels/
// CUDASort.cu:13-98); CUB's LSD radix sort is stable, so std::stable_sort on
// the key gives the identical permutation.

#include "IO/DcdWriter.h"
#include "Objects/Tables.h"
#include "Interactions/Bonded/BondComputer.h"
#include "Interactions/Nonbonded/Pairwise.h"
#include "PatchOperation/Integrator/BAOAB.h"
#include "PatchOperation/Integrator/BD.h"
#include "PatchOperation/PairListKernels/ZOrderNeighbor.h"
#include "PatchOperation/ZOrderKernels/ZOrderKernels.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

using namespace MARS;

namespace {

PeriodicBox make_box(const float* origin, const float* size, const int* periodic) {
	PeriodicBox box(Vector3(size[0], size[1], size[2]), periodic[0] != 0, periodic[1] != 0,
					periodic[2] != 0);
	box.set_origin(Vector3(origin[0], origin[1], origin[2]));
	return box;
}

template <typename F>
void run_chunked(size_t n, int nthreads, const F& f) {
	if (nthreads <= 1 || n < 4096) {
		for (size_t i = 0; i < n; ++i)
			f(i);
		return;
	}
	std::vector<std::thread> pool;
	const size_t chunk = (n + nthreads - 1) / nthreads;
	for (int t = 0; t < nthreads; ++t) {
		const size_t lo = t * chunk, hi = std::min(n, lo + chunk);
		if (lo >= hi)
			break;
		pool.emplace_back([lo, hi, &f]() {
			for (size_t i = lo; i < hi; ++i)
				f(i);
		});
	}
	for (auto& th : pool)
		th.join();
}

std::vector<TabulatedPotential> make_tables(float* values, const uint32_t* offsets,
											const uint32_t* sizes, const float* starts,
											const float* step_invs, const int* periodic,
											int n_tables) {
	std::vector<TabulatedPotential> t(n_tables);
	for (int k = 0; k < n_tables; ++k) {
		t[k].pot = values + offsets[k];
		t[k].step_inv = step_invs[k];
		t[k].size = sizes[k];
		t[k].start = starts[k];
		t[k].is_periodic = periodic[k] != 0;
	}
	return t;
}

} // namespace

extern "C" {

int ref_version() { return 1; }

// MortonEncodeKernel (ZOrderKernels.h:27-43).
void ref_morton_encode(const float* pos4, size_t n, const float* bmin, const float* bmax,
					   uint32_t* keys, uint32_t* idx, int nthreads) {
	MortonEncodeKernel k{reinterpret_cast<const Vector3*>(pos4), keys, idx,
						 Vector3(bmin[0], bmin[1], bmin[2]), Vector3(bmax[0], bmax[1], bmax[2]), n};
	run_chunked(n, nthreads, [&](size_t i) { k(i); });
}

// Stable sort of (key, payload) by key: the CUB SortPairs contract.
void ref_sort_pairs(uint32_t* keys, uint32_t* vals, size_t n) {
	std::vector<uint32_t> order(n);
	std::iota(order.begin(), order.end(), 0u);
	std::stable_sort(order.begin(), order.end(),
					 [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
	std::vector<uint32_t> k2(n), v2(n);
	for (size_t i = 0; i < n; ++i) {
		k2[i] = keys[order[i]];
		v2[i] = vals[order[i]];
	}
	std::copy(k2.begin(), k2.end(), keys);
	std::copy(v2.begin(), v2.end(), vals);
}

// InverseIndexKernel (ZOrderKernels.h:68-83).
void ref_inverse(const uint32_t* sorted, uint32_t* inv, size_t n) {
	InverseIndexKernel k{sorted, inv, n};
	for (size_t i = 0; i < n; ++i)
		k(i);
}

// ReorderDataKernel<Vector3> (ZOrderKernels.h:48-63).
void ref_reorder_pos(const float* pos4, float* out4, const uint32_t* sorted, size_t n) {
	ReorderDataKernel<Vector3> k{reinterpret_cast<const Vector3*>(pos4),
								 reinterpret_cast<Vector3*>(out4), sorted, n};
	for (size_t i = 0; i < n; ++i)
		k(i);
}

// DcdWriter (src/IO/DcdWriter.h) driven as SimManager::write_dcd_frame drives
// it (SimManager.cpp:596-633): header on the first frame (N, NFILE 1,
// NPRIV = NSAVC = output period, NSTEP 0, DELTA = timestep, unit cell when any
// axis is periodic), then one writeStep per frame with the CHARMM unit cell
// (A, 0, B, 0, 0, C). frames: n_frames x n float4 rows.
int ref_dcd_write(const char* path, const float* frames4, int n_frames, int n, int nsavc,
				  float delta, int with_unitcell, const float* box) {
	try {
		DcdWriter w(path);
		for (int f = 0; f < n_frames; ++f) {
			if (f == 0) w.writeHeader(n, 1, nsavc, nsavc, 0, delta, with_unitcell != 0);
			std::vector<Vector3> frame(n);
			for (int i = 0; i < n; ++i) {
				const float* p = frames4 + (static_cast<size_t>(f) * n + i) * 4;
				frame[i] = Vector3(p[0], p[1], p[2]);
			}
			if (with_unitcell)
				w.writeStep(frame, std::vector<double>{box[0], 0.0, box[1], 0.0, 0.0, box[2]});
			else
				w.writeStep(frame);
		}
	} catch (const std::exception&) {
		return -1;
	}
	return 0;
}

// RemapIndicesKernel (ZOrderKernels.h:87-101).
void ref_remap_indices(int* indices, size_t count, const uint32_t* inv, size_t map_size) {
	RemapIndicesKernel k{indices, inv, count, map_size};
	for (size_t i = 0; i < count; ++i)
		k(i);
}

// BuildCellRangesKernel (ZOrderNeighbor.h:27-43); begin/end must be zeroed.
void ref_cell_ranges(const uint32_t* keys, size_t n, int shift, uint32_t* begin, uint32_t* end) {
	BuildCellRangesKernel k{keys, begin, end, n, shift};
	for (size_t i = 0; i < n; ++i)
		k(i);
}

// BuildCellNeighborsKernel (ZOrderNeighbor.h:55-139).
void ref_cell_neighbors(uint32_t* table, size_t num_cells, int m, const int* radii, int npc,
						const float* box_len) {
	BuildCellNeighborsKernel k{table, num_cells, m, int3(radii[0], radii[1], radii[2]), npc,
							   Vector3(box_len[0], box_len[1], box_len[2])};
	for (size_t c = 0; c < num_cells; ++c)
		k(c);
}

// ZOrderCellNeighborKernel (ZOrderNeighbor.h:155-225), run serially over all
// n * tpp work items. The host ATOMIC_ADD returns the incremented value, so
// pairs land in slots [1, count]; `pairs` must hold max_pairs + 1 int2.
// Returns the pair count.
uint32_t ref_neighbor_walk(const float* sorted_pos4, const uint32_t* keys, const uint32_t* s2o,
						   const uint32_t* cell_begin, const uint32_t* cell_end,
						   const uint32_t* table, int* pairs, size_t max_pairs, float cutoff_sq,
						   size_t n, int npc, int tpp, int shift, const float* origin,
						   const float* size, const int* periodic, const int* excl_offsets,
						   const int* excl_neighbors, size_t excl_n, const int* rigid_body_id) {
	uint32_t count = 0;
	ExclusionView ex;
	ex.offsets = excl_offsets;
	ex.excluded = excl_neighbors;
	ex.num_particles = excl_offsets ? excl_n : 0;
	ex.rigid_body_id = rigid_body_id;
	ZOrderCellNeighborKernel k{reinterpret_cast<const Vector3*>(sorted_pos4),
							   keys,
							   s2o,
							   cell_begin,
							   cell_end,
							   table,
							   reinterpret_cast<int2*>(pairs),
							   &count,
							   cutoff_sq,
							   n,
							   max_pairs + 1,
							   npc,
							   tpp,
							   shift,
							   make_box(origin, size, periodic),
							   ex};
	const size_t total = n * static_cast<size_t>(tpp);
	for (size_t t = 0; t < total; ++t)
		k(t);
	return count;
}

// The same functor run only for the listed work items (particle i with one
// thread per particle), to time a bounded sample of a large walk. Pairs are
// stored in slots [1, max_pairs] when `pairs` is given (the host ATOMIC_ADD
// returns the incremented count). Returns the number of pairs emitted.
uint64_t ref_neighbor_walk_items(const float* sorted_pos4, const uint32_t* keys,
								 const uint32_t* s2o, const uint32_t* cell_begin,
								 const uint32_t* cell_end, const uint32_t* table, float cutoff_sq,
								 size_t n, int npc, int shift, const float* origin,
								 const float* size, const int* periodic, const uint32_t* items,
								 size_t n_items, int* pairs, size_t max_pairs) {
	uint32_t count = 0;
	int2 sink[2];
	int2* out = pairs ? reinterpret_cast<int2*>(pairs) : sink;
	ExclusionView ex;
	ZOrderCellNeighborKernel k{reinterpret_cast<const Vector3*>(sorted_pos4),
							   keys,
							   s2o,
							   cell_begin,
							   cell_end,
							   table,
							   out,
							   &count,
							   cutoff_sq,
							   n,
							   pairs ? max_pairs + 1 : 0,
							   npc,
							   1,
							   shift,
							   make_box(origin, size, periodic),
							   ex};
	for (size_t t = 0; t < n_items; ++t)
		k(items[t]);
	return count;
}

// The same walk on `nthreads` host threads. The reference's host atomics are
// plain `+=`, so its functor is not run on shared outputs from several
// threads: each thread walks a contiguous range of the items into its own
// counter and buffer (the functor unchanged), and the buffers are joined in
// thread order, so the emitted order is the serial walk's. A buffer that turns
// out too small is regrown and its range walked again. Writes slots
// [1, count] of `pairs` (slot 0 unused, as the serial emit does) when the
// total fits in max_pairs.
uint64_t ref_neighbor_walk_items_mt(const float* sorted_pos4, const uint32_t* keys,
									const uint32_t* s2o, const uint32_t* cell_begin,
									const uint32_t* cell_end, const uint32_t* table,
									float cutoff_sq, size_t n, int npc, int shift,
									const float* origin, const float* size, const int* periodic,
									const uint32_t* items, size_t n_items, int* pairs,
									size_t max_pairs, int nthreads) {
	if (nthreads < 1) nthreads = 1;
	const PeriodicBox box = make_box(origin, size, periodic);
	const size_t chunk = (n_items + nthreads - 1) / nthreads;
	std::vector<std::vector<int2>> bufs(nthreads);
	std::vector<uint64_t> counts(nthreads, 0);
	auto walk = [&](int t) {
		const size_t lo = std::min(n_items, t * chunk), hi = std::min(n_items, lo + chunk);
		size_t cap = (max_pairs + 1) / std::max<size_t>(n_items, 1) * (hi - lo) + (hi - lo) / 4 + 1024;
		for (;;) {
			bufs[t].assign(cap + 1, int2{});
			uint32_t count = 0;
			ExclusionView ex;
			ZOrderCellNeighborKernel k{reinterpret_cast<const Vector3*>(sorted_pos4),
									   keys,
									   s2o,
									   cell_begin,
									   cell_end,
									   table,
									   bufs[t].data(),
									   &count,
									   cutoff_sq,
									   n,
									   cap + 1,
									   npc,
									   1,
									   shift,
									   box,
									   ex};
			for (size_t i = lo; i < hi; ++i)
				k(items[i]);
			counts[t] = count;
			if (count <= cap) return;
			cap = static_cast<size_t>(count) + count / 8 + 1024;
		}
	};
	std::vector<std::thread> pool;
	for (int t = 1; t < nthreads; ++t)
		pool.emplace_back(walk, t);
	walk(0);
	for (auto& th : pool)
		th.join();
	uint64_t total = 0;
	for (int t = 0; t < nthreads; ++t)
		total += counts[t];
	if (pairs && total <= max_pairs) {
		int2* out = reinterpret_cast<int2*>(pairs) + 1;
		for (int t = 0; t < nthreads; ++t) {
			std::memcpy(out, bufs[t].data() + 1, counts[t] * sizeof(int2));
			out += counts[t];
		}
	}
	return total;
}

// ResolvePairTableKernel (Pairwise.h:104-120).
void ref_resolve_tags(const int* pairs, size_t n_pairs, const int* type_ids,
					  const uint32_t* term_matrix, size_t num_types, uint32_t* tags, int nthreads) {
	ResolvePairTableKernel k{reinterpret_cast<const int2*>(pairs), type_ids, term_matrix,
							 num_types, tags, n_pairs};
	run_chunked(n_pairs, nthreads, [&](size_t i) { k(i); });
}

// PairNonbondedComputer (Pairwise.h:184-305), tabulated term only enabled by
// the caller through enabled_terms. Accumulates into fe4.
void ref_pair_forces(const int* pairs, size_t n_pairs, const float* pos4, int* type_ids,
					 float* fe4, const uint32_t* tags, float* table_values,
					 const uint32_t* table_offsets, const uint32_t* table_sizes,
					 const float* table_starts, const float* table_step_invs, int n_tables,
					 const float* origin, const float* size, const int* periodic, int get_energy,
					 float cutoff_sq, uint32_t enabled_terms) {
	std::vector<int> periodic_flags(n_tables, 0);
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	ParticleView pv{};
	pv.type_id = type_ids;
	pv.pos = reinterpret_cast<Vector3*>(const_cast<float*>(pos4));
	pv.ForceEnergy = reinterpret_cast<Vector3*>(fe4);
	ParticleTypeView tv{};
	const PeriodicBox box = make_box(origin, size, periodic);
	PairNonbondedComputer k(reinterpret_cast<const int2*>(pairs), pv, tags, tabs.data(), tv, &box,
							get_energy != 0, n_pairs, cutoff_sq, enabled_terms);
	for (size_t i = 0; i < n_pairs; ++i)
		k(i);
}

// The same pair forces on `nthreads` host threads: each thread runs the
// functor (unchanged) over a contiguous range of the pairs into its own
// ForceEnergy array, and the arrays are added into fe4 in thread order.
void ref_pair_forces_mt(const int* pairs, size_t n_pairs, size_t n_particles, const float* pos4,
						int* type_ids, float* fe4, const uint32_t* tags, float* table_values,
						const uint32_t* table_offsets, const uint32_t* table_sizes,
						const float* table_starts, const float* table_step_invs, int n_tables,
						const float* origin, const float* size, const int* periodic,
						int get_energy, float cutoff_sq, uint32_t enabled_terms, int nthreads) {
	if (nthreads < 1) nthreads = 1;
	std::vector<int> periodic_flags(n_tables, 0);
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	const PeriodicBox box = make_box(origin, size, periodic);
	const size_t chunk = (n_pairs + nthreads - 1) / nthreads;
	std::vector<std::vector<Vector3>> part(nthreads);
	auto run = [&](int t) {
		const size_t lo = std::min(n_pairs, t * chunk), hi = std::min(n_pairs, lo + chunk);
		part[t].assign(n_particles, Vector3());
		ParticleView pv{};
		pv.type_id = type_ids;
		pv.pos = reinterpret_cast<Vector3*>(const_cast<float*>(pos4));
		pv.ForceEnergy = part[t].data();
		ParticleTypeView tv{};
		PairNonbondedComputer k(reinterpret_cast<const int2*>(pairs), pv, tags, tabs.data(), tv,
								&box, get_energy != 0, n_pairs, cutoff_sq, enabled_terms);
		for (size_t i = lo; i < hi; ++i)
			k(i);
	};
	std::vector<std::thread> pool;
	for (int t = 1; t < nthreads; ++t)
		pool.emplace_back(run, t);
	run(0);
	for (auto& th : pool)
		th.join();
	for (int t = 0; t < nthreads; ++t)
		for (size_t i = 0; i < n_particles; ++i) {
			fe4[4 * i + 0] += part[t][i].x;
			fe4[4 * i + 1] += part[t][i].y;
			fe4[4 * i + 2] += part[t][i].z;
			fe4[4 * i + 3] += part[t][i].t;
		}
}

// PairNonbondedComputer (Pairwise.h:214-304) with every analytical term:
// per-type charge / radius / eps, the solvent constants as
// launch_pairwise_nonbonded sets them (NonBondedInteraction.h:289-293) and
// the Gaussian's constants.
void ref_pair_forces_terms(const int* pairs, size_t n_pairs, const float* pos4, int* type_ids,
						   float* fe4, const uint32_t* tags, float* table_values,
						   const uint32_t* table_offsets, const uint32_t* table_sizes,
						   const float* table_starts, const float* table_step_invs, int n_tables,
						   const float* origin, const float* size, const int* periodic,
						   int get_energy, float cutoff_sq, uint32_t enabled_terms,
						   const float* charge, const float* radius, const float* eps,
						   const float* solvent5, const float* gaussian3) {
	std::vector<int> periodic_flags(n_tables, 0);
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	ParticleView pv{};
	pv.type_id = type_ids;
	pv.pos = reinterpret_cast<Vector3*>(const_cast<float*>(pos4));
	pv.ForceEnergy = reinterpret_cast<Vector3*>(fe4);
	ParticleTypeView tv{};
	tv.charge = charge;
	tv.radius = radius;
	tv.eps = eps;
	const PeriodicBox box = make_box(origin, size, periodic);
	PairNonbondedComputer k(reinterpret_cast<const int2*>(pairs), pv, tags, tabs.data(), tv, &box,
							get_energy != 0, n_pairs, cutoff_sq, enabled_terms);
	k.debye_huckel.screen_length = solvent5[0];
	k.debye_huckel.epsilon = solvent5[1];
	k.onck.kappa = solvent5[2];
	k.onck.sz = solvent5[3];
	k.onck.z = solvent5[4];
	k.gaussian.amp = gaussian3[0];
	k.gaussian.sigma = gaussian3[1];
	k.gaussian.cutoff_squared = gaussian3[2];
	for (size_t i = 0; i < n_pairs; ++i)
		k(i);
}

// TabulatedDihedralComputer (BondComputer.h:282-346); dihedral tables wrap
// (DeviceBondedInteraction.h:250).
void ref_dihedral_forces(const int* dihedrals4, const int* table_idx, const int* forms, size_t nd,
						 const float* pos4, float* fe4, float* table_values,
						 const uint32_t* table_offsets, const uint32_t* table_sizes,
						 const float* table_starts, const float* table_step_invs, int n_tables,
						 const float* origin, const float* size, const int* periodic,
						 int get_energy) {
	std::vector<int> periodic_flags(n_tables, 1);
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	const PeriodicBox box = make_box(origin, size, periodic);
	TabulatedDihedralComputer k(reinterpret_cast<const int4*>(dihedrals4),
								reinterpret_cast<Vector3*>(const_cast<float*>(pos4)),
								reinterpret_cast<Vector3*>(fe4), tabs.data(), table_idx, forms,
								&box, get_energy != 0, nd);
	for (size_t i = 0; i < nd; ++i)
		k(i);
}

// HarmonicRestraintComputer (BondComputer.h:88-131); anchors as Vector3 rows.
void ref_restraint_forces(const int* ids, const float* anchors4, const float* k_spring, size_t nr,
						  const float* pos4, float* fe4, const float* origin, const float* size,
						  const int* periodic, int get_energy) {
	const PeriodicBox box = make_box(origin, size, periodic);
	HarmonicRestraintComputer k(ids, reinterpret_cast<Vector3*>(const_cast<float*>(pos4)),
								reinterpret_cast<Vector3*>(fe4),
								reinterpret_cast<const Vector3*>(anchors4), k_spring, &box,
								get_energy != 0, nr);
	for (size_t i = 0; i < nr; ++i)
		k(i);
}

// TabulatedBondComputer (BondComputer.h:136-192).
void ref_bond_forces(const int* bonds, const int* table_idx, const int* forms, size_t nb,
					 const float* pos4, float* fe4, float* table_values,
					 const uint32_t* table_offsets, const uint32_t* table_sizes,
					 const float* table_starts, const float* table_step_invs, int n_tables,
					 const float* origin, const float* size, const int* periodic, int get_energy) {
	std::vector<int> periodic_flags(n_tables, 0);
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	const PeriodicBox box = make_box(origin, size, periodic);
	TabulatedBondComputer k(reinterpret_cast<const int2*>(bonds),
							reinterpret_cast<Vector3*>(const_cast<float*>(pos4)),
							reinterpret_cast<Vector3*>(fe4), tabs.data(), table_idx, forms, &box,
							get_energy != 0, nb);
	for (size_t i = 0; i < nb; ++i)
		k(i);
}

// TabulatedAngleComputer (BondComputer.h:204-269); angles are int4 rows
// (i, j, k, pad) matching the reference's 16-byte int3.
void ref_angle_forces(const int* angles4, const int* table_idx, const int* forms, size_t na,
					  const float* pos4, float* fe4, float* table_values,
					  const uint32_t* table_offsets, const uint32_t* table_sizes,
					  const float* table_starts, const float* table_step_invs, int n_tables,
					  const float* origin, const float* size, const int* periodic,
					  int get_energy) {
	std::vector<int> periodic_flags(n_tables, 1); // angle tables wrap
	auto tabs = make_tables(table_values, table_offsets, table_sizes, table_starts,
							table_step_invs, periodic_flags.data(), n_tables);
	const PeriodicBox box = make_box(origin, size, periodic);
	TabulatedAngleComputer k(reinterpret_cast<const int3*>(angles4),
							 reinterpret_cast<Vector3*>(const_cast<float*>(pos4)),
							 reinterpret_cast<Vector3*>(fe4), tabs.data(), table_idx, forms, &box,
							 get_energy != 0, na);
	for (size_t i = 0; i < na; ++i)
		k(i);
}

// One dense grid as the BD functor sees it (BaseGridDevice.h GridGeometry).
struct RefGrid {
	const float* data;
	float origin[3];
	float basis[9];		// column-major: basis[3*c + r]
	float basis_inv[9]; // column-major
	int64_t dims[3];
	int boundary_condition;
};

// BDIntegrate<float> (BD.h:12-93) with the PMF grid, E field and Philox.
void ref_bd_integrate(float* pos4, float* fe4, int* type_ids, uint32_t* flags, size_t n,
					  int num_types, const float* charge, const float* diffusion4,
					  const int* pmf_offset, const int* pmf_count, const float* pmf_terms4,
					  int n_terms, const int* force_grid_id4, const float* force_grid_scale4,
					  const RefGrid* grids, int n_grids, const float* origin, const float* size,
					  const int* periodic, float dt, float kT, uint64_t step, uint64_t base_seed,
					  uint32_t base_ctr, const float* efield, int nthreads) {
	std::vector<GridTerm> terms(n_terms);
	for (int t = 0; t < n_terms; ++t) {
		terms[t].grid_id = static_cast<int>(pmf_terms4[4 * t + 0]);
		terms[t].scale = pmf_terms4[4 * t + 1];
		terms[t].scale_slope = pmf_terms4[4 * t + 2];
		terms[t].boundary_condition = static_cast<int>(pmf_terms4[4 * t + 3]);
	}
	std::vector<BaseGridView<float>> views(n_grids);
	for (int g = 0; g < n_grids; ++g) {
		auto& v = views[g];
		v.origin = Vector3(grids[g].origin[0], grids[g].origin[1], grids[g].origin[2]);
		const float* b = grids[g].basis;
		const float* bi = grids[g].basis_inv;
		v.basis = Matrix3(Vector3(b[0], b[1], b[2]), Vector3(b[3], b[4], b[5]),
						  Vector3(b[6], b[7], b[8]));
		v.basis_inv = Matrix3(Vector3(bi[0], bi[1], bi[2]), Vector3(bi[3], bi[4], bi[5]),
							  Vector3(bi[6], bi[7], bi[8]));
		v.dimensions = Vector3_t<idx_t>(grids[g].dims[0], grids[g].dims[1], grids[g].dims[2]);
		v.grid_id = g;
		v.boundary_condition = grids[g].boundary_condition;
		v.data = grids[g].data;
	}
	ParticleView pv{};
	pv.type_id = type_ids;
	pv.pos = reinterpret_cast<Vector3*>(pos4);
	pv.ForceEnergy = reinterpret_cast<Vector3*>(fe4);
	pv.flags = flags;
	ParticleTypeView tv{};
	tv.charge = charge;
	tv.diffusion = reinterpret_cast<const Vector3*>(diffusion4);
	tv.pmf_grid_offset = pmf_offset;
	tv.pmf_grid_count = pmf_count;
	tv.pmf_grid_terms = terms.data();
	tv.force_grid_id = reinterpret_cast<const int3*>(force_grid_id4);
	tv.force_grid_scale = reinterpret_cast<const Vector3*>(force_grid_scale4);
	std::vector<float> mass(num_types, 1.0f);
	tv.mass = mass.data();
	BDIntegrate<float> k(pv, tv, make_box(origin, size, periodic), dt, step, kT, n, base_seed,
						 base_ctr, n_grids > 0 ? views.data() : nullptr,
						 Vector3(efield[0], efield[1], efield[2]), InterpolationOrder::Linear);
	run_chunked(n, nthreads, [&](size_t i) { k(i); });
}

// Patch::integrate_motion's Langevin branch (Patch.cpp:290-335): ComputePMFKernel
// (Pmf.h:126-152) when grids exist, BAOAB_LastUpdate when a kick is pending,
// then BAOABIntegrate<float> (BAOAB.h:47-128).
void ref_baoab_integrate(float* pos4, float* mom4, float* fe4, int* type_ids, uint32_t* flags,
						 size_t n, int num_types, const float* charge, const float* mass,
						 const float* damping4, const int* pmf_offset, const int* pmf_count,
						 const float* pmf_terms4, int n_terms, const int* force_grid_id4,
						 const float* force_grid_scale4, const RefGrid* grids, int n_grids,
						 const float* origin, const float* size, const int* periodic, float dt,
						 float kT, uint64_t step, uint64_t base_seed, uint32_t base_ctr,
						 const float* efield, int pending) {
	std::vector<GridTerm> terms(n_terms);
	for (int t = 0; t < n_terms; ++t) {
		terms[t].grid_id = static_cast<int>(pmf_terms4[4 * t + 0]);
		terms[t].scale = pmf_terms4[4 * t + 1];
		terms[t].scale_slope = pmf_terms4[4 * t + 2];
		terms[t].boundary_condition = static_cast<int>(pmf_terms4[4 * t + 3]);
	}
	std::vector<BaseGridView<float>> views(n_grids);
	for (int g = 0; g < n_grids; ++g) {
		auto& v = views[g];
		v.origin = Vector3(grids[g].origin[0], grids[g].origin[1], grids[g].origin[2]);
		const float* b = grids[g].basis;
		const float* bi = grids[g].basis_inv;
		v.basis = Matrix3(Vector3(b[0], b[1], b[2]), Vector3(b[3], b[4], b[5]),
						  Vector3(b[6], b[7], b[8]));
		v.basis_inv = Matrix3(Vector3(bi[0], bi[1], bi[2]), Vector3(bi[3], bi[4], bi[5]),
							  Vector3(bi[6], bi[7], bi[8]));
		v.dimensions = Vector3_t<idx_t>(grids[g].dims[0], grids[g].dims[1], grids[g].dims[2]);
		v.grid_id = g;
		v.boundary_condition = grids[g].boundary_condition;
		v.data = grids[g].data;
	}
	ParticleView pv{};
	pv.type_id = type_ids;
	pv.pos = reinterpret_cast<Vector3*>(pos4);
	pv.mom = reinterpret_cast<Vector3*>(mom4);
	pv.ForceEnergy = reinterpret_cast<Vector3*>(fe4);
	pv.flags = flags;
	ParticleTypeView tv{};
	tv.charge = charge;
	tv.mass = mass;
	tv.trans_damping = reinterpret_cast<const Vector3*>(damping4);
	tv.pmf_grid_offset = pmf_offset;
	tv.pmf_grid_count = pmf_count;
	tv.pmf_grid_terms = terms.data();
	tv.force_grid_id = reinterpret_cast<const int3*>(force_grid_id4);
	tv.force_grid_scale = reinterpret_cast<const Vector3*>(force_grid_scale4);
	const BaseGridView<float>* gv = n_grids > 0 ? views.data() : nullptr;
	const Vector3 e(efield[0], efield[1], efield[2]);
	if (gv) {
		const ComputePMFKernel pmf{e, InterpolationOrder::Linear};
		for (size_t i = 0; i < n; ++i) pmf(i, pv, tv, gv, static_cast<idx_t>(n));
	}
	if (pending) {
		BAOAB_LastUpdate<float> last(pv, tv, dt, step, kT, n, base_seed, base_ctr, gv, e,
									 InterpolationOrder::Linear);
		for (size_t i = 0; i < n; ++i) last(i);
	}
	BAOABIntegrate<float> k(pv, tv, make_box(origin, size, periodic), dt, step, kT, n, base_seed,
							base_ctr, gv, e, InterpolationOrder::Linear);
	for (size_t i = 0; i < n; ++i) k(i);
}

// openrand::Philox::draw_int4 (philox.h:60-127), `ndraw` consecutive draws.
void ref_philox_int4(uint64_t seed, uint32_t ctr, uint32_t global_seed, uint32_t ctr1, int ndraw,
					 uint32_t* out) {
	openrand::Philox rng(seed, ctr, global_seed, ctr1);
	for (int d = 0; d < ndraw; ++d) {
		auto u = rng.draw_int4();
		out[4 * d + 0] = u.x;
		out[4 * d + 1] = u.y;
		out[4 * d + 2] = u.z;
		out[4 * d + 3] = u.w;
	}
}

// openrand::Philox::draw_float4 (philox.h:88-93, base_state.h:299-305).
void ref_philox_float4(uint64_t seed, uint32_t ctr, uint32_t global_seed, uint32_t ctr1, int ndraw,
					   float* out) {
	openrand::Philox rng(seed, ctr, global_seed, ctr1);
	for (int d = 0; d < ndraw; ++d) {
		auto u = rng.draw_float4();
		out[4 * d + 0] = u.x;
		out[4 * d + 1] = u.y;
		out[4 * d + 2] = u.z;
		out[4 * d + 3] = u.w;
	}
}

// DisplacementKernel (AdaptiveKernels.h:48-101) + the sqrt in
// ZOrderSort::compute_max_displacement (ZOrderSort.cpp:173-198).
float ref_max_displacement(const float* cur4, const float* prev4, size_t n, const float* box_len) {
	float max_sq = 0.0f;
	DisplacementKernel k{reinterpret_cast<const Vector3*>(cur4),
						 reinterpret_cast<const Vector3*>(prev4), &max_sq, n,
						 Vector3(box_len[0], box_len[1], box_len[2])};
	for (size_t i = 0; i < n; ++i)
		k(i);
	return sqrtf(max_sq);
}

// PeriodicBox::wrap_diff / wrap (PeriodicBox.h:134-208).
void ref_wrap_diff(const float* origin, const float* size, const int* periodic, const float* in4,
				   float* out4, size_t n) {
	const PeriodicBox box = make_box(origin, size, periodic);
	for (size_t i = 0; i < n; ++i) {
		Vector3 v(in4[4 * i], in4[4 * i + 1], in4[4 * i + 2]);
		Vector3 w = box.wrap_diff(v);
		out4[4 * i] = w.x;
		out4[4 * i + 1] = w.y;
		out4[4 * i + 2] = w.z;
		out4[4 * i + 3] = 0.0f;
	}
}

void ref_wrap(const float* origin, const float* size, const int* periodic, const float* in4,
			  float* out4, size_t n) {
	const PeriodicBox box = make_box(origin, size, periodic);
	for (size_t i = 0; i < n; ++i) {
		Vector3 v(in4[4 * i], in4[4 * i + 1], in4[4 * i + 2]);
		Vector3 w = box.wrap(v);
		out4[4 * i] = w.x;
		out4[4 * i + 1] = w.y;
		out4[4 * i + 2] = w.z;
		out4[4 * i + 3] = 0.0f;
	}
}

// Tabulated pair/bond/angle lookup (TabulatedPotential.h:19-52) for one value.
void ref_table_lookup(float x, float* values, uint32_t size, float start, float step_inv,
					  int periodic, float* out2) {
	TabulatedPotential t;
	t.pot = values;
	t.step_inv = step_inv;
	t.size = size;
	t.start = start;
	t.is_periodic = periodic != 0;
	const ScalarForceEnergy fe = TabulatedPotential::compute(x, &t);
	out2[0] = fe.force_magnitude;
	out2[1] = fe.energy;
}

// Table::read_file (src/Objects/Tables.h:61-102) of one "x y" text file, with
// the type's abscissa conversion. kind: 0 non-bonded pair, 1 bond, 2 angle,
// 3 dihedral. Writes up to cap rows of X and Y, the row count, start, step and
// whether check_same_step_size accepts the (unconverted) abscissa.
int ref_read_table(const char* path, int kind, float* x_out, float* y_out, size_t cap,
				   size_t* count, float* start, float* step, int* uniform) {
	static const TabulatedType kinds[4] = {TabulatedType::NonBondedPair, TabulatedType::Bond,
										   TabulatedType::Angle, TabulatedType::Dihedral};
	if (kind < 0 || kind > 3) return -1;
	Table t(kinds[kind]);
	t.read_file(path);
	*count = t.X.size();
	for (size_t i = 0; i < t.X.size() && i < cap; ++i) {
		x_out[i] = t.X[i];
		y_out[i] = t.Y[i];
	}
	*start = t.start;
	*step = t.step_size;
	Table raw(TabulatedType::Bond);  // same file, no conversion: the step check alone
	raw.read_file(path);
	*uniform = raw.check_same_step_size() ? 1 : 0;
	return 0;
}

} // extern "C"
