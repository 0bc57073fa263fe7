/*
 * marsb200.h -- C ABI of libmarsb200.so, the B200 (sm_100a) implementation of
 * the MARS-MD Brownian-dynamics force-and-integrate path.
 *
 * Each entry point replaces one reference interface on that path (paths are
 * relative to the MARS-MD source tree); the reference reaches them through
 * Backend/Kernels.h launch_kernel -> launch_cuda_kernel<Functor>
 * (src/Backend/Kernels.h:35-83, src/Backend/CUDA/KernelHelper.cuh:129-183),
 * which this library replaces on this path only.
 *
 * Conventions
 *   - Every function returns 0 (MB2_OK) or a positive MB2_ERR_* code; the
 *     message is available from mb2_last_error(ctx). No C++ exception crosses
 *     this boundary (the reference throws MARS::Exception instead).
 *   - Particle arrays are caller-owned DEVICE pointers in the reference's
 *     layouts: positions and ForceEnergy are float4 rows (x, y, z, w), type ids
 *     int32, flags uint32 (src/Objects/DeviceParticle.h:18-40). Vector3 is
 *     16 bytes (src/Types/Vector3.h:41). Table values, term matrices and other
 *     set-up data are HOST pointers, copied in.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream). Work is
 *     enqueued asynchronously unless a function returns a host value (noted).
 *   - Scratch (sort buffers, cell tables, the pair list) belongs to the
 *     context and grows on demand with cudaMalloc.
 */
#ifndef MARSB200_H
#define MARSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MB2_API __attribute__((visibility("default")))
#else
#define MB2_API
#endif

#define MB2_OK 0
#define MB2_ERR_ARG 1      /* invalid argument or call order */
#define MB2_ERR_CUDA 2     /* CUDA runtime error */
#define MB2_ERR_CAPACITY 3 /* more particles/pairs than the context allows */
#define MB2_ERR_STATE 4    /* required set-up missing (box, tables, pairlist) */
#define MB2_ERR_IO 5       /* file output failed */

typedef struct mb2_context mb2_context;

/* Library version (major * 100 + minor). */
MB2_API int mb2_version(void);

/* Create a context on `device` for up to `max_particles` particles.
 * Replaces the Pairlist/ZOrderPairlist/ZOrderSort constructors
 * (src/PatchOperation/Pairlist.h:66-74, PairListKernels/ZOrderPairlist.cpp:83-100,
 * ZOrderKernels/ZOrderSort.cpp:7-38). */
MB2_API int mb2_create(int device, uint32_t max_particles, mb2_context** out);
MB2_API int mb2_destroy(mb2_context* ctx);
/* Last error message of this context ("" if none). */
MB2_API const char* mb2_last_error(const mb2_context* ctx);

/* Orthogonal periodic box. Replaces Pairlist::set_periodic_box
 * (src/PatchOperation/Pairlist.h:118-120) and the PeriodicBox by-value
 * argument of launch_BD (src/PatchOperation/Integrator.h:26-54). */
MB2_API int mb2_set_box(mb2_context* ctx, const float origin[3], const float size[3],
                const int periodic[3]);

/* --- Z-order sort ---------------------------------------------------------
 * ZOrderSort::sort_particles + reorder_data (ZOrderKernels/ZOrderSort.cpp:40-70,
 * ZOrderSort.h:316-339): Morton keys against [bmin, bmax], stable sort, inverse
 * map, gathered positions. Any output pointer may be NULL. Device pointers. */
MB2_API int mb2_sort_morton(mb2_context* ctx, const float* pos4, uint32_t n, const float bmin[3],
                    const float bmax[3], uint32_t* keys_out, uint32_t* sorted_to_orig_out,
                    uint32_t* inverse_out, float* sorted_pos4_out, void* stream);

/* Stable sort of (key, value) pairs by the 32-bit key, in place. Replaces
 * device_radix_sort_pairs_cub (ZOrderKernels/CUDASort.cu:13-98). */
MB2_API int mb2_radix_sort_pairs(mb2_context* ctx, uint32_t* keys, uint32_t* vals, uint32_t n,
                         void* stream);

/* The same stable in-place sort, allocating no device memory: no counterpart
 * in the reference. mb2_radix_sort_pairs grows context scratch with cudaMalloc
 * (and frees the old buffer, which synchronises the device) whenever n grows;
 * callers that cannot allocate — a process whose HBM is already held by another
 * allocator, or a loop that must never stall on an implicit synchronisation —
 * use this one. Its scratch is a fixed array in the library's static device
 * memory (about 8.6 MB per device, held until the process exits).
 *   - n <= MB2_SORT_STATIC_MAX, else MB2_ERR_CAPACITY and nothing is touched.
 *   - Each call looks up the array's device address with the context's device
 *     current. Under CUDA's lazy module loading (the CUDA 12 default) the first
 *     call on a device may load the module and so reserve the 8.6 MB then: make
 *     one call with n = 0 at start-up, before another allocator takes the
 *     device's free memory and before any stream capture. After
 *     cudaDeviceReset, make that n = 0 call again (the module reloads, possibly
 *     at another address, which the next lookup finds).
 *   - All calls on one device share the array: calls that overlap in time on
 *     one device race. Order them (one stream, or explicit events).
 *   - ctx selects the device and receives the error message; the context's
 *     own buffers are not used. */
#define MB2_SORT_STATIC_MAX 1048576u
MB2_API int mb2_radix_sort_pairs_static(mb2_context* ctx, uint32_t* keys, uint32_t* vals,
                                uint32_t n, void* stream);

/* --- pairlist --------------------------------------------------------------
 * Exclusion CSR (device pointers, borrowed until the next build): replaces
 * Pairlist::set_exclusions with ExclusionView (Pairlist.h:125-127,
 * src/Interactions/DeviceExclusions.h:22-75). offsets has num_particles + 1
 * entries; rigid_body_id may be NULL. Pass offsets = NULL to clear. */
MB2_API int mb2_set_exclusions(mb2_context* ctx, const int* offsets, const int* neighbors,
                       uint32_t num_particles, const int* rigid_body_id);

/* Build the half pairlist within `pairlist_cutoff`. Replaces
 * ZOrderPairlist::build_pairlist (PairListKernels/ZOrderPairlist.cpp:102-178).
 * Synchronises `stream` once (to size the list); returns the pair count.
 * `interaction_cutoff` is the force cutoff the list will serve. When it lies
 * in (0, pairlist_cutoff), each row stores the pairs within
 * interaction_cutoff + 25 % of the skin first and the rest after them, so
 * the pair kernel skips whole warps in the rows' tails; otherwise (0, or not
 * below pairlist_cutoff) rows keep the walk's candidate order. The pair set
 * is the same either way; only the order in which per-particle force sums
 * accumulate differs. The result depends on the arguments alone, not on
 * earlier calls; mb2_step and mb2_run pass their params' cutoff. NaN is
 * rejected with MB2_ERR_ARG. */
MB2_API int mb2_build_pairlist(mb2_context* ctx, const float* pos4, const int* type_ids, uint32_t n,
                       float pairlist_cutoff, float interaction_cutoff, void* stream,
                       uint64_t* num_pairs);

/* Pair count of the last build (Pairlist::get_num_pairs, Pairlist.h:139-141). */
MB2_API int mb2_num_pairs(const mb2_context* ctx, uint64_t* num_pairs);

/* Write the pairs of the last build as int2 (min, max) original indices,
 * the reference's neighbor_pairs_ format (Pairlist::get_neighbor_pairs,
 * Pairlist.h:132-134). `capacity` in pairs; fails if smaller than the count. */
MB2_API int mb2_export_pairs(mb2_context* ctx, int* pairs2, uint64_t capacity, void* stream);

/* Skin check: largest minimum-image displacement since the last build; sets
 * *needs = (max > skin / 2). Replaces ZOrderPairlist::needs_update
 * (ZOrderPairlist.cpp:184-190, ZOrderSort.cpp:173-198). Synchronises. */
MB2_API int mb2_needs_update(mb2_context* ctx, const float* pos4, uint32_t n, float skin, void* stream,
                     float* max_displacement, int* needs);

/* --- pair forces -----------------------------------------------------------
 * Type-pair tag matrix and tabulated tables. Replaces
 * DevicePairNonBondedInteractions::copy_pairwise_from_host and
 * link_pairwise_tables (src/Interactions/DevicePairNonBondedInteraction.h:97-199).
 * term_matrix: host uint32 [num_types * num_types], tags as make_pair_tag
 * (bit 5 = tabulated, table index << 8; src/Interactions/Nonbonded/Pairwise.h:31-35).
 * values: host float, tables concatenated; sizes/starts/step_invs per table. */
MB2_API int mb2_set_pair_tables(mb2_context* ctx, int num_types, const uint32_t* term_matrix,
                        int num_tables, const float* values, const uint32_t* sizes,
                        const float* starts, const float* step_invs);

/* Analytical pair terms: per-type charge, softcore radius and eps
 * (ParticleTypeView::charge/radius/eps, src/Objects/DeviceParticle.h:49-53)
 * and the run-wide constants (SolventParams,
 * src/Interactions/NonBondedInteraction.h:123-129, set on the functors by
 * launch_pairwise_nonbonded, :289-293; GaussianPotential amp / sigma /
 * cutoff^2, src/Interactions/Nonbonded/Pairwise.h:50-53, which that launcher
 * leaves at 1, 1, 0). params NULL = those defaults. Tag bits of the term
 * matrix (AnalyticalPairTerm, Pairwise.h:19-27): 1 Coulomb, 2 Debye-Hueckel,
 * 4 Onck, 8 Gaussian, 16 softcore, 32 tabulated; a tag may combine them. A
 * matrix with analytical bits needs this call before mb2_pair_forces. */
typedef struct {
    float debye_length;        /* A */
    float dielectric;
    float onck_kappa;          /* 1/A */
    float onck_sz;
    float onck_z;              /* A */
    float gaussian_amp;
    float gaussian_sigma;      /* A */
    float gaussian_cutoff_sq;  /* A^2, <= 0: none */
} mb2_pair_params;
MB2_API int mb2_set_pair_terms(mb2_context* ctx, int num_types, const float* charge,
                               const float* radius, const float* eps,
                               const mb2_pair_params* params);

/* Pair forces over the last pairlist, ACCUMULATED into force_energy
 * (original order; energy halves into .w when get_energy). Replaces
 * launch_resolve_pair_tables + launch_pairwise_nonbonded
 * (src/Interactions/NonBondedInteraction.h:205-296): per pair, the terms of
 * its type pair's tag summed in PairNonbondedComputer's order (Coulomb,
 * Debye-Hueckel, Onck, Gaussian, softcore, tabulated; Pairwise.h:214-304). */
MB2_API int mb2_pair_forces(mb2_context* ctx, const float* pos4, const int* type_ids,
                    float* force_energy4, uint32_t n, float cutoff, int get_energy,
                    void* stream);

/* The pair kernels' form of the reference's pair test
 * (PairNonbondedComputer, Pairwise.h:214-304: a pair is skipped when
 * dist = sqrt(d2) < 1e-6 or dist * dist > cutoff * cutoff, in float): the
 * test is d2 < *d2_lo or d2 > *d2_hi exactly, both bounds found by bisection
 * over the floats (cutoff <= 0: no upper bound, *d2_hi = +inf). Host only. */
MB2_API int mb2_pair_distance_window(float cutoff, float* d2_lo, float* d2_hi);
/* Exhaustive device check of the pair kernels' correctly rounded square root
 * (one Newton-Raphson step on the hardware estimate) against the CUDA
 * intrinsic __fsqrt_rn on every float in [2^-60, FLT_MAX]: the mismatch count
 * (0 when the kernels' root is the IEEE one). Synchronises. */
MB2_API int mb2_selftest_sqrt(mb2_context* ctx, uint64_t* mismatches);

/* FP64 reductions of the last force calls made with get_energy: pair energy,
 * pair virial (sum of r . f), bond energy, angle energy. Synchronises.
 * New on this path: the reference sums per-particle floats on the host
 * (src/SimManager.cpp:1000-1075). */
MB2_API int mb2_energies(mb2_context* ctx, void* stream, double out[4]);
/* The same reductions with the remaining terms: out[0..count) of pair
 * energy, pair virial, bond, angle, dihedral, restraint energy (count <= 6). */
MB2_API int mb2_energy_terms(mb2_context* ctx, void* stream, double* out, int count);
MB2_API int mb2_reset_energies(mb2_context* ctx, void* stream);

/* --- bonded forces ---------------------------------------------------------
 * Tables for bonds (kind 0, non-periodic), angles (kind 1, periodic, radians)
 * or dihedrals (kind 2, periodic, radians). Replaces
 * DeviceBondedInteractions::link_tables
 * (src/Interactions/DeviceBondedInteraction.h:205-250). In every bonded call a
 * row whose table_idx is negative is skipped: it stands for a form other than
 * tabulated, which the reference's tabulated functors skip through forms[]
 * (Bonded/BondComputer.h:165-166, 233-234, 301-302). */
MB2_API int mb2_set_bonded_tables(mb2_context* ctx, int kind, int num_tables, const float* values,
                          const uint32_t* sizes, const float* starts, const float* step_invs);

/* Tabulated bond forces, accumulated. bonds: device int2 [nb]; table_idx:
 * device int [nb]. Replaces launch_tabulated_bonds
 * (DeviceBondedInteraction.h:495-521, Bonded/BondComputer.h:136-192). */
MB2_API int mb2_bond_forces(mb2_context* ctx, const int* bonds2, const int* table_idx, uint32_t nb,
                    const float* pos4, float* force_energy4, int get_energy, void* stream);

/* Tabulated angle forces, accumulated. angles: device int4 (i, j, k, pad) [na].
 * Replaces launch_tabulated_angles (DeviceBondedInteraction.h:523-549,
 * Bonded/BondComputer.h:204-269). */
MB2_API int mb2_angle_forces(mb2_context* ctx, const int* angles4, const int* table_idx, uint32_t na,
                     const float* pos4, float* force_energy4, int get_energy, void* stream);

/* Tabulated dihedral forces, accumulated. dihedrals: device int4 [nd].
 * Replaces launch_tabulated_dihedrals (DeviceBondedInteraction.h:551-578,
 * TabulatedDihedralComputer, Bonded/BondComputer.h:282-346, with
 * DihedralGeometry, Bonded/BondGeometry.h:56-87): degenerate quadruples get
 * no force, magnitudes are clamped to +-1000, energy quarters into .w. */
MB2_API int mb2_dihedral_forces(mb2_context* ctx, const int* dihedrals4, const int* table_idx,
                                uint32_t nd, const float* pos4, float* force_energy4,
                                int get_energy, void* stream);

/* Harmonic position restraints, accumulated: particle_ids device int [nr]
 * (negative = skipped), anchors4 device float4 [nr], spring_k device float
 * [nr]. Replaces launch_harmonic_restraints (DeviceBondedInteraction.h:599-620,
 * HarmonicRestraintComputer, Bonded/BondComputer.h:88-131). */
MB2_API int mb2_restraint_forces(mb2_context* ctx, const int* particle_ids, const float* anchors4,
                                 const float* spring_k, uint32_t nr, const float* pos4,
                                 float* force_energy4, int get_energy, void* stream);

/* --- integrator ------------------------------------------------------------
 * Per-type data for the BD step (ParticleTypeView, src/Objects/DeviceParticle.h:49-64).
 * Host arrays: charge[T], diffusion3[T*3], pmf_offset[T], pmf_count[T],
 * terms4[n_terms*4] as (grid_id, scale, scale_slope, boundary_condition) in
 * float, force_grid_id3[T*3] (-1 = none, may be NULL), force_grid_scale3[T*3]. */
MB2_API int mb2_set_particle_types(mb2_context* ctx, int num_types, const float* charge,
                           const float* diffusion3, const int* pmf_offset, const int* pmf_count,
                           int n_terms, const float* terms4, const int* force_grid_id3,
                           const float* force_grid_scale3);

/* Dense grid `grid_id` (BaseGridView, src/Types/BaseGridDevice.h:22-29):
 * data is a DEVICE float array [nx][ny][nz] (z fastest), borrowed;
 * basis_inv column-major; boundary_condition 0 Dirichlet, 1 Neumann, 2 Periodic. */
MB2_API int mb2_set_grid(mb2_context* ctx, int grid_id, const float* data, const int64_t dims[3],
                 const float origin[3], const float basis_inv[9], int boundary_condition);

/* One Brownian step in place. Replaces launch_BD<float> / BDIntegrate
 * (src/PatchOperation/Integrator.h:26-54, Integrator/BD.h:12-93). flags may be
 * NULL. base_seed as Patch::integrate_motion mixes it (mb2_bd_seed). */
MB2_API int mb2_bd_integrate(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
                     const uint32_t* flags, uint32_t n, float dt, float kT, uint64_t step,
                     uint64_t base_seed, uint32_t base_ctr, const float efield[3],
                     void* stream);

/* --- canonical Z-order reorder ---------------------------------------------
 * Replaces Patch::reorder_particles (src/PatchOperation/Patch.cpp:455-480):
 * Morton order of the positions over the periodic box (ZOrderSort::sort_particles
 * with origin .. origin + size as bounds), each per-particle array gathered
 * into it (DeviceParticle::permute, src/Objects/DeviceParticleManager.h:186-208,
 * ReorderDataKernel, src/PatchOperation/ZOrderKernels/ZOrderKernels.h:49-63)
 * and each stored particle index sent through the inverse map
 * (RemapIndicesKernel, ZOrderKernels.h:87-101). The host rebuilds the
 * exclusion CSR from remapped pairs as rebuild_exclusions_after_reorder does
 * (src/Interactions/DeviceBondedInteraction.h:364-430).
 *   mb2_reorder_begin: compute and keep the permutation of n positions; the
 *     context's pairlist becomes stale (the next build re-sorts). A box with
 *     a non-positive size is MB2_ERR_ARG (the reference skips the reorder).
 *   mb2_reorder_apply: permute one device array of n elements of 4 or 16 bytes
 *     in place (positions, momenta, orientations, ids, type ids, flags,
 *     rigid-body ids; force/energy is cleared each step and is not permuted);
 *     n must equal the last begin's.
 *   mb2_reorder_remap: indices[i] = inverse[indices[i]] for the `count` device
 *     ints whose value is in [0, n) (bond / angle / dihedral / restraint
 *     particle indices); others unchanged.
 *   mb2_reorder_inverse: copy the old -> new map (device uint32[n]). */
MB2_API int mb2_reorder_begin(mb2_context* ctx, const float* pos4, uint32_t n, void* stream);
MB2_API int mb2_reorder_apply(mb2_context* ctx, void* data, uint32_t elem_bytes, uint32_t n,
                              void* stream);
MB2_API int mb2_reorder_remap(mb2_context* ctx, int* indices, uint64_t count, void* stream);
MB2_API int mb2_reorder_inverse(mb2_context* ctx, uint32_t* inverse_out, uint32_t n,
                                void* stream);

/* Langevin (BAOAB) integrator. Per-type mass and translational damping
 * (ParticleTypeView::mass, trans_damping; src/Objects/DeviceParticle.h:49-64),
 * host arrays; mb2_set_particle_types must come first (same type count). */
MB2_API int mb2_set_langevin_types(mb2_context* ctx, int num_types, const float* mass,
                           const float* damping3);
/* One Langevin step of Patch::integrate_motion (Patch.cpp:290-335): with
 * grids, the position-dependent force (and energy) is accumulated into
 * force_energy for every particle (launch_PMF, Integrator.h:125-143); when
 * deferred_kick_pending, the closing half-kick of the previous step
 * (launch_BAOAB_LastUpdate, Integrator.h:98-123); then B-A-O-A and wrap
 * (launch_BAOAB, Integrator.h:56-86). mom4: caller-owned momenta (float4).
 * The caller then owes a closing kick (pass pending = 1 next step, or call
 * mb2_baoab_last_update). Noise: Philox keyed like BAOABIntegrate (stream 0x1356914). */
MB2_API int mb2_baoab_integrate(mb2_context* ctx, float* pos4, float* mom4, float* force_energy4,
                        const int* type_ids, const uint32_t* flags, uint32_t n, float dt,
                        float kT, uint64_t step, uint64_t base_seed, uint32_t base_ctr,
                        const float efield[3], int deferred_kick_pending, void* stream);
/* The closing half-kick alone (Patch::finish_deferred_kick, Patch.cpp:354-373). */
MB2_API int mb2_baoab_last_update(mb2_context* ctx, float* mom4, const float* force_energy4,
                          const uint32_t* flags, uint32_t n, float dt, void* stream);

/* Patch::integrate_motion seed mixing (src/PatchOperation/Patch.cpp:252-254). */
MB2_API uint64_t mb2_bd_seed(uint64_t seed, uint64_t patch_id, uint64_t step);

/* Philox4x32-10 draws for counters ctr0 + i (i < n), as the BD step makes them
 * (philox.h:60-139): out4 gets the raw words, normals4 the Box-Muller normals
 * (either may be NULL). Device pointers. */
MB2_API int mb2_philox(mb2_context* ctx, uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2,
               uint32_t n, uint32_t* out4, float* normals4, void* stream);

/* --- fused step ------------------------------------------------------------
 * One whole BD step as SimManager::execute_force_calculation +
 * execute_integration run it (src/SimManager.cpp:337-504) for one patch:
 * clear forces, rebuild the pairlist when (step - 1) % rebuild_period == 0
 * (unless the skin check says the list is still valid), pair forces, bonded
 * forces (bonds, angles, dihedrals, restraints where given), then the BD
 * update or, with integrator = 1, the Langevin branch of
 * Patch::integrate_motion (PMF pass, the deferred closing kick when pending,
 * B-A-O-A; the caller then owes the closing kick, as with mb2_baoab_integrate).
 * All device pointers. */
typedef struct {
    float pairlist_cutoff;
    float cutoff;
    uint32_t rebuild_period;
    float dt;
    float kT;
    uint64_t seed;       /* run seed; mixed per step as Patch::integrate_motion does */
    uint64_t patch_id;
    float efield[3];
    int get_energy;
    const int* bonds2;   /* may be NULL */
    const int* bond_table_idx;
    uint32_t num_bonds;
    const int* angles4;  /* may be NULL */
    const int* angle_table_idx;
    uint32_t num_angles;
    const int* dihedrals4;  /* may be NULL */
    const int* dihedral_table_idx;
    uint32_t num_dihedrals;
    const int* restraint_ids;  /* may be NULL */
    const float* restraint_anchors4;
    const float* restraint_k;
    uint32_t num_restraints;
    int integrator;             /* 0 Brownian (BD), 1 Langevin (BAOAB; needs mb2_set_langevin_types) */
    float* mom4;                /* Langevin: momenta (float4 [n]), updated in place */
    int deferred_kick_pending;  /* Langevin: the previous step's closing kick is owed */
} mb2_step_params;

MB2_API int mb2_step(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
             const uint32_t* flags, uint32_t n, uint64_t step, const mb2_step_params* params,
             void* stream);

/* Steps first_step .. first_step + num_steps - 1, with the results of one
 * mb2_step call per step (the loop of SimManager::run over one patch,
 * src/SimManager.cpp:337-504). The BD steps that are not rebuild checks
 * replay one CUDA graph of the step body, the step number read from a device
 * counter, so that small systems are not bound by launch overhead; the graph
 * is captured on first use and again whenever a pointer, size or parameter it
 * bakes in changes. Rebuild checks, Langevin steps and steps while per-stage
 * profiling is on run as mb2_step. */
MB2_API int mb2_run(mb2_context* ctx, float* pos4, float* force_energy4, const int* type_ids,
            const uint32_t* flags, uint32_t n, uint64_t first_step, uint32_t num_steps,
            const mb2_step_params* params, void* stream);

/* --- output ------------------------------------------------------------------
 * The output side of SimManager for one system (src/SimManager.cpp:318-330
 * initialize_output_writers, :541-575 handle_output): a DCD trajectory
 * <name>.dcd with DcdWriter's byte layout (src/IO/DcdWriter.h; header on the
 * first frame with NPRIV = NSAVC = output_period, DELTA = timestep, a CHARMM
 * unit cell (A, 0, B, 0, 0, C) per frame when any axis is periodic), with
 * momenta the Langevin momentum DCD <name>.0.momentum.dcd (:833-861);
 * <name>.energy.dat (write_energy_output, :999-1068); restart files
 * <name>.restart and <name>.0.momentum.restart, one "type x y z" line per
 * particle in shortest round-trip decimals (write_restart_files,
 * :1078-1135). An existing DCD file is renamed to <name>.dcd.BAK.
 * Rows are written in global-id order: ids (device int[n], may be NULL =
 * identity) maps each row to its place, as copy_to_host_unpermuted does
 * after a Morton reorder (src/Objects/DeviceParticleManager.h:219-260).
 * Frames and restarts are packed on the device and written by a background
 * thread: a call returns once its copy is queued; at most two are in flight
 * (a third waits). mb2_output_flush waits for them and reports a failed
 * write. Device pointers, except mass (host). */
typedef struct mb2_output mb2_output;
typedef struct {
    const char* output_name;
    uint32_t num_particles;
    int output_period;   /* DCD NSAVC (values below 1 become 1) */
    float timestep;      /* DCD DELTA */
    float box[3];        /* unit cell edges */
    int periodic[3];
    int with_momentum;   /* Langevin: momentum DCD and momentum restart */
    int device;
} mb2_output_config;
MB2_API int mb2_output_create(const mb2_output_config* cfg, mb2_output** out);
/* Waits for queued writes, closes the files. */
MB2_API int mb2_output_destroy(mb2_output* out);
MB2_API const char* mb2_output_last_error(const mb2_output* out);
/* One trajectory frame (and momentum frame). */
MB2_API int mb2_output_frame(mb2_output* out, const float* pos4, const float* mom4, const int* ids,
                             uint32_t n, void* stream);
/* Restart files (positions, type ids; momenta with with_momentum). */
MB2_API int mb2_output_restart(mb2_output* out, const float* pos4, const float* mom4,
                               const int* type_ids, const int* ids, uint32_t n, void* stream);
/* FP64 reductions on the device: potential = sum of force_energy .w (kcal/mol),
 * kinetic = sum 0.5 |p|^2 / mass[type] / SQRT_CAL_TO_JOULE^2 / kT (kT units;
 * 0 without momenta); appends both lines to <name>.energy.dat and returns
 * them in out[0] (kinetic) and out[1] (potential). Synchronises. */
MB2_API int mb2_output_energy(mb2_output* out, const float* force_energy4, const float* mom4,
                              const int* type_ids, const float* mass, int num_types, uint32_t n,
                              float kT, void* stream, double out2[2]);
MB2_API int mb2_output_flush(mb2_output* out);

/* --- tracing ---------------------------------------------------------------
 * Per-stage device timing with CUDA events on the launching stream (replaces
 * the reference's Profiler event timers, src/Backend/Profiler.h:166-205).
 * While on, the fused step and the pairlist/pair-force calls record one
 * event pair per stage; mb2_profile_read synchronises, returns the summed
 * milliseconds and launch count of a stage, and clears it. */
#define MB2_STAGE_STEP 0       /* whole mb2_step */
#define MB2_STAGE_PAIRLIST 1   /* pairlist build: sort + walks */
#define MB2_STAGE_PAIR_FORCE 2 /* the pair-force kernel alone */
#define MB2_STAGE_INTEGRATE 3  /* the BD integrate kernel */
#define MB2_NUM_STAGES 4
MB2_API int mb2_set_profiling(mb2_context* ctx, int on);
/* Number of kernels this library has launched in this process (all contexts). */
MB2_API uint64_t mb2_launch_count(void);
MB2_API int mb2_profile_read(mb2_context* ctx, int stage, double* total_ms, uint32_t* count);

/* Rows (particles) served by one group of lanes in the pair kernel: 4, 8, 16
 * or 32 lanes per row; 0 = choose from the mean row length. */
MB2_API int mb2_set_lanes_per_row(mb2_context* ctx, int lanes);

/* Cell level of the pairlist walk relative to the cost model's choice
 * (-2..2; 0 = the model's), and the level the last build used (-1 before
 * any). A tuning knob: the pair set does not depend on it. */
MB2_API int mb2_set_cell_level_offset(mb2_context* ctx, int offset);
MB2_API int mb2_cell_level(mb2_context* ctx, int* level);

/* --- adjoint of a BD window ------------------------------------------------
 * No counterpart in the reference (it computes no gradients). Gradients of a
 * loss of the final positions of a window of BD steps with fixed Philox noise,
 * with respect to the pair-table values, the bond-table values and the
 * initial positions; forward with checkpoints, reverse with recomputation.
 * Forces are minus gradients of potentials piecewise linear in a distance or
 * angle (the tabulated lookup), so one reverse step is
 *   lambda_k = lambda_{k+1} + J(x_k) (c * lambda_{k+1}),  c = D dt / kT,
 * J the (symmetric) force Jacobian; table gradients accumulate in FP64.
 * The gradient is that of the piecewise-smooth map: a pair sitting exactly on
 * a table-bin edge (or the cutoff) contributes its one-sided derivative.
 *
 * mb2_window_forward: num_steps steps from first_step (the mb2_step sequence;
 * the pairlist is rebuilt at every checkpoint), x0 in pos4 -> x_N in pos4.
 * checkpoint_every must divide params->rebuild_period, and first_step - 1 be
 * a multiple of checkpoint_every. Particle types without grids; no flags.
 * params (its bond/angle pointers) and type_ids must stay valid until the
 * backward call. */
MB2_API int mb2_window_forward(mb2_context* ctx, float* pos4, float* force_energy4,
                       const int* type_ids, uint32_t n, uint64_t first_step,
                       uint32_t num_steps, uint32_t checkpoint_every,
                       const mb2_step_params* params, void* stream);
/* The positions the last forward window stored at its checkpoints (x_0,
 * x_C, x_2C, ...; ceil(num_steps / C) blocks of n float4 rows, in order), for
 * inspecting or restarting a window; the reverse sweep recomputes each
 * segment from these. capacity_rows counts float4 rows. No counterpart in the
 * reference (it has no adjoint). */
MB2_API int mb2_window_checkpoints(mb2_context* ctx, float* out4, uint64_t capacity_rows,
                           void* stream);
/* Record the states each following mb2_window_backward differentiates: x_0 ..
 * x_{N-1} of the window (N = num_steps), n float4 rows each in step order,
 * written into out4 (device, at least N x n rows, checked at the backward
 * call) as the reverse sweep recomputes each segment from its checkpoint.
 * NULL stops recording. For checking a reverse sweep against another adjoint
 * along the very states it used. No counterpart in the reference. */
MB2_API int mb2_window_record_states(mb2_context* ctx, float* out4, uint64_t capacity_rows);
/* Reverse sweep of the last forward window: grad_final4 = dL/dx_N (float4
 * rows, .w ignored) -> grad_pos0_4 = dL/dx_0; grad_pair_bins (device double,
 * one per value of the concatenated pair tables) and grad_bond_bins (per
 * value of the concatenated bond tables; may be NULL without bonds) are
 * ACCUMULATED. Each segment is recomputed from its checkpoint. */
MB2_API int mb2_window_backward(mb2_context* ctx, const float* grad_final4, float* grad_pos0_4,
                        double* grad_pair_bins, double* grad_bond_bins, void* stream);
/* Gaussian-smoothed pair-distance histogram of non-excluded pairs with
 * r < r_max: hist[b] (device double [num_bins], overwritten) =
 * sum exp(-(r - r_b)^2 / (2 sigma^2)) over |r - r_b| <= 5 sigma, r_b = (b + 1/2) dr.
 * Builds the pairlist at r_max. */
MB2_API int mb2_rdf_histogram(mb2_context* ctx, const float* pos4, const int* type_ids, uint32_t n,
                      uint32_t num_bins, float bin_width, float r_max, float sigma,
                      double* hist, void* stream);
/* Gradient of sum_b dl_dhist[b] hist[b] with respect to the positions given
 * to the last mb2_rdf_histogram, ACCUMULATED into grad4 (float4 rows). */
MB2_API int mb2_rdf_backward(mb2_context* ctx, const float* pos4, uint32_t n, uint32_t num_bins,
                     float bin_width, float r_max, float sigma, const double* dl_dhist,
                     float* grad4, void* stream);

/* --- batched replicas ------------------------------------------------------
 * Many independent periodic systems of uneven size stepped together, one
 * launch per stage for all of them. No single counterpart in the reference:
 * each system is what one reference Patch runs (Patch.cpp:43-352) through
 * SimManager's step loop (SimManager.cpp:337-504); here all systems share
 * each launch. Systems are concatenated in the caller's arrays (system s owns
 * particles [sum(counts[<s]), sum(counts[<=s]))), each in its own periodic box
 * (origin3/size3 per system, origin NULL = 0; every edge > 2 x list radius).
 * System s steps exactly as mb2_step would with seed (params->seed + s):
 * same pair set, same Philox key and counters (index within the system).
 * Pair tables and particle types are shared by all systems; no grids, no
 * bonded terms, no exclusions in this mode. At most 2048 systems. */
typedef struct mb2_batch mb2_batch;
MB2_API int mb2_batch_create(int device, uint32_t num_systems, const uint32_t* counts,
                     const float* box_origin3, const float* box_size3, mb2_batch** out);
MB2_API int mb2_batch_destroy(mb2_batch* b);
MB2_API const char* mb2_batch_last_error(const mb2_batch* b);
MB2_API int mb2_batch_set_pair_tables(mb2_batch* b, int num_types, const uint32_t* term_matrix,
                              int num_tables, const float* values, const uint32_t* sizes,
                              const float* starts, const float* step_invs);
MB2_API int mb2_batch_set_particle_types(mb2_batch* b, int num_types, const float* charge,
                                 const float* diffusion3);
/* Pairlist of every system within pairlist_cutoff; synchronises once. */
MB2_API int mb2_batch_build(mb2_batch* b, const float* pos4, const int* type_ids,
                    float pairlist_cutoff, void* stream, uint64_t* num_pairs);
MB2_API int mb2_batch_num_pairs(const mb2_batch* b, uint64_t* num_pairs);
/* All pairs as int2(min, max) of indices into the concatenated arrays. */
MB2_API int mb2_batch_export_pairs(mb2_batch* b, int* pairs2, uint64_t capacity, void* stream);
/* One step of every system (the mb2_step sequence, rebuild schedule included:
 * at scheduled steps the lists are rebuilt when any system moved more than
 * half the skin). params->num_bonds and num_angles must be 0. */
MB2_API int mb2_batch_step(mb2_batch* b, float* pos4, float* force_energy4, const int* type_ids,
                   uint64_t step, const mb2_step_params* params, void* stream);
/* num_steps steps from first_step: rebuilds run eagerly at scheduled steps;
 * every step's force-and-integrate body is one replay of a CUDA graph
 * captured on first use (re-captured when a buffer or parameter changes). */
MB2_API int mb2_batch_run(mb2_batch* b, float* pos4, float* force_energy4, const int* type_ids,
                  uint64_t first_step, uint32_t num_steps, const mb2_step_params* params,
                  void* stream);
/* Tuning knobs: cell level relative to the cost model's choice (-3..3) and
 * lanes per pairlist row (0 = automatic, 4, 8, 16, 32). Invalidates the list. */
MB2_API int mb2_batch_set_tuning(mb2_batch* b, int level_offset, int lanes);
MB2_API int mb2_batch_tuning(const mb2_batch* b, int* level_offset, int* lanes,
                     uint32_t* total_cells);
/* Rebuild cadence: with period > 0, mb2_batch_step and mb2_batch_run check
 * every system at every period-th step instead of at params->rebuild_period
 * (0, the default, uses the params'), and rebuild the lists of the systems
 * one of whose particles moved more than half the skin since that system's
 * own last build, the rule of Patch.cpp:86-108 applied to each system as to a
 * patch; the others keep their lists. mb2_batch_autotune sets the cadence to
 * its choice. mb2_batch_rebuild_schedule reports the cadence in force and the
 * number of list builds so far (steps that rebuilt any system);
 * mb2_batch_system_rebuilds the number of system lists rebuilt, summed over
 * those builds. */
MB2_API int mb2_batch_set_rebuild_period(mb2_batch* b, uint32_t period);
MB2_API int mb2_batch_rebuild_schedule(const mb2_batch* b, uint32_t* period, uint64_t* rebuilds);
MB2_API int mb2_batch_system_rebuilds(const mb2_batch* b, uint64_t* count);
/* Autotuner: times one pairlist build and `trial_steps` steps for each cell
 * level offset in {-1, 0, +1} and lanes per row in {4, 8, 16} on a copy of
 * the positions, and keeps the pair minimising build / rebuild_period + step.
 * Then the rebuild cadence, on the copy: after an equilibration segment of
 * one params->rebuild_period (so the overlaps of a fresh start have relaxed),
 * two intervals of one period, each from a fresh list, record the largest
 * displacement after every step; the cadence is the largest k <= the period
 * whose displacement stayed within half the skin in both (at least 1). The
 * chosen knobs and cadence are put in force (mb2_batch_set_tuning,
 * mb2_batch_set_rebuild_period) and reported; max_displacement_at_period is
 * the displacement after a whole period from a fresh list. Positions are not
 * changed; the next step rebuilds the list. */
typedef struct {
    int level_offset;                  /* chosen cell level offset */
    int lanes;                         /* chosen lanes per row */
    float build_ms;                    /* pairlist build time with the choice */
    float step_ms;                     /* force-and-integrate time per step */
    uint32_t safe_rebuild_period;      /* chosen cadence, put in force */
    float max_displacement_at_period;  /* largest displacement after rebuild_period steps (A) */
    uint32_t total_cells;
} mb2_batch_tuning_result;
MB2_API int mb2_batch_autotune(mb2_batch* b, const float* pos4, const int* type_ids,
                       const mb2_step_params* params, uint32_t trial_steps, void* stream,
                       mb2_batch_tuning_result* out);

#ifdef __cplusplus
}
#endif
#endif
