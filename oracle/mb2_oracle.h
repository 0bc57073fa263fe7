/*
 * CPU oracle for the MARS-MD Brownian-dynamics force-and-integrate path.
 *
 * TEST INFRASTRUCTURE ONLY. Only the test suite, the smoke check and the
 * benchmark's CPU-baseline leg load this library, and only as the checker of
 * the CUDA path. Nothing in the product links or calls it.
 *
 * Every function restates, in plain C, one step of the reference algorithm
 * (reference file:line cited on each). Float functions follow the reference's
 * float operation order exactly; compile with -ffp-contract=off and no
 * fast-math so the results are bit-reproducible. Functions with an `_f64`
 * suffix re-evaluate the same formulas in double for energy checks.
 *
 * Vector data is float4 rows (x, y, z, w) as the reference's Vector3_t.
 */
#ifndef MB2_ORACLE_H
#define MB2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Orthogonal periodic box (src/System/PeriodicBox.h:16-461, orthogonal path). */
typedef struct {
	float origin[3];
	float size[3];
	int periodic[3];
} or_box;

/* One tabulated potential (src/Interactions/TabulatedPotential.h:8-14). */
typedef struct {
	const float* pot;
	float step_inv;
	uint32_t size;
	float start;
	int is_periodic;
} or_table;

/* One dense grid (src/Types/BaseGridDevice.h:22-29), basis column-major. */
typedef struct {
	const float* data;
	float origin[3];
	float basis[9];
	float basis_inv[9];
	int64_t dims[3];
	int boundary_condition; /* 0 Dirichlet, 1 Neumann, 2 Periodic */
} or_grid;

/* One PMF grid term (src/Types/GridTerm.h GridTerm). */
typedef struct {
	int grid_id;
	float scale;
	float scale_slope;
	int boundary_condition;
} or_grid_term;

/* Per-type data used by the BD step (src/Objects/DeviceParticle.h ParticleTypeView). */
typedef struct {
	int num_types;
	const float* charge;           /* [T] */
	const float* diffusion4;       /* [T][4] */
	const int* pmf_offset;         /* [T] */
	const int* pmf_count;          /* [T] */
	const or_grid_term* terms;     /* flat */
	const int* force_grid_id4;     /* [T][4] (x, y, z, pad); <0 = none */
	const float* force_grid_scale4;/* [T][4] */
} or_types;

int or_version(void);

/* --- periodic box ------------------------------------------------------- */
float or_wrap_diff_scalar(float x, float l);
float or_wrap_scalar(float x, float o, float l);
void or_wrap_diff(const or_box* b, const float* in4, float* out4, size_t n);
void or_wrap(const or_box* b, const float* in4, float* out4, size_t n);

/* --- Morton sort -------------------------------------------------------- */
uint32_t or_morton_key(const float* p, const float* bmin, const float* bmax);
void or_morton_encode(const float* pos4, size_t n, const float* bmin, const float* bmax,
                      uint32_t* keys, uint32_t* idx);
void or_sort_pairs(uint32_t* keys, uint32_t* vals, size_t n);
void or_inverse(const uint32_t* sorted, uint32_t* inv, size_t n);
void or_gather4(const float* in4, float* out4, const uint32_t* sorted, size_t n);
void or_morton_domain(const or_box* b, const float* pos4, size_t n, float* bmin, float* bmax);

/* --- pairlist ----------------------------------------------------------- */
void or_select_cell_grid(const float* extent, float cutoff, size_t n, size_t max_pairs, int* m,
                         int* radii, int* slots);
void or_cell_ranges(const uint32_t* keys, size_t n, int shift, uint32_t* begin, uint32_t* end);
void or_cell_neighbors(uint32_t* table, int m, const int* radii, int npc, const float* box_len);
uint64_t or_neighbor_walk(const float* sorted_pos4, const uint32_t* keys, const uint32_t* s2o,
                          const uint32_t* begin, const uint32_t* end, const uint32_t* table,
                          int npc, int shift, float cutoff_sq, size_t n, const or_box* b,
                          const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                          const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                          uint64_t* checksum);
uint64_t or_build_pairlist(const float* pos4, size_t n, const or_box* b, float rc_list,
                           const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                           const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                           uint64_t* checksum);
uint64_t or_build_pairlist_m(const float* pos4, size_t n, const or_box* b, float rc_list,
                             const int* excl_offsets, const int* excl_neighbors, size_t excl_n,
                             const int* rigid_body_id, int* pairs, uint64_t max_pairs,
                             uint64_t* checksum, int m_force);
uint64_t or_pair_hash(int a, int b);
int or_exclusion_csr(const int* pairs, size_t n_pairs, int* offsets, int* neighbors,
                     size_t* n_excl_particles);
float or_max_displacement(const float* cur4, const float* prev4, size_t n, const float* box_len);

/* --- forces ------------------------------------------------------------- */
void or_table_lookup(const or_table* t, float x, float* force, float* energy);
void or_resolve_tags(const int* pairs, size_t n_pairs, const int* type_ids,
                     const uint32_t* term_matrix, int num_types, uint32_t* tags);
void or_pair_forces(const int* pairs, size_t n_pairs, const float* pos4, const uint32_t* tags,
                    const or_table* tables, const or_box* b, float cutoff_sq, int get_energy,
                    float* fe4, double* fe64, double* fabs_sum);
void or_bond_forces(const int* bonds, const int* table_idx, size_t nb, const float* pos4,
                    const or_table* tables, const or_box* b, int get_energy, float* fe4,
                    double* fe64, double* fabs_sum);
void or_angle_forces(const int* angles4, const int* table_idx, size_t na, const float* pos4,
                     const or_table* tables, const or_box* b, int get_energy, float* fe4,
                     double* fe64, double* fabs_sum);
/* Analytical pair-term constants: per-type charge, softcore radius and eps,
 * the solvent constants (SolventParams, src/Interactions/NonBondedInteraction.h:123-129)
 * and the Gaussian's (GaussianPotential, src/Interactions/Nonbonded/Pairwise.h:50-53). */
typedef struct {
	const float* charge;
	const float* radius;
	const float* eps;
	float debye_length, dielectric, onck_kappa, onck_sz, onck_z;
	float gaussian_amp, gaussian_sigma, gaussian_cutoff_sq;
	uint32_t enabled_terms;
} or_pair_terms;
void or_pair_forces_terms(const int* pairs, size_t n_pairs, const float* pos4,
                          const int* type_ids, const uint32_t* tags, const or_table* tables,
                          const or_pair_terms* pt, const or_box* b, float cutoff_sq,
                          int get_energy, float* fe4, double* fe64, double* fabs_sum);
void or_dihedral_forces(const int* dihedrals4, const int* table_idx, size_t nd,
                        const float* pos4, const or_table* tables, const or_box* b,
                        int get_energy, float* fe4, double* fe64, double* fabs_sum);
void or_restraint_forces(const int* ids, const float* anchors4, const float* k_spring, size_t nr,
                         const float* pos4, const or_box* b, int get_energy, float* fe4,
                         double* fe64, double* fabs_sum);
double or_pair_energy_f64(const int* pairs, size_t n_pairs, const float* pos4,
                          const uint32_t* tags, const or_table* tables, const or_box* b,
                          float cutoff_sq);

/* --- grid, Philox, BD --------------------------------------------------- */
float or_grid_value(const or_grid* g, const float* pos, int bc);
void or_grid_gradient(const or_grid* g, const float* pos, int bc, float* grad);
void or_position_force(const float* pos, int type, const or_types* types, const or_grid* grids,
                       const float* efield, float* force4);
void or_philox4x32_10(uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2,
                      uint32_t internal, uint32_t* out4);
float or_u01(uint32_t x);
uint64_t or_bd_seed(uint64_t seed, uint64_t patch_id, uint64_t step);
/* Langevin BAOAB step (Integrator/BAOAB.h:47-128) with the passes that
 * Patch::integrate_motion runs before it (Patch.cpp:290-335): with grids, the
 * position-dependent force is accumulated into ForceEnergy for every particle
 * (ComputePMFKernel, Pmf.h:126-152); with a pending deferred kick, the closing
 * half-kick (BAOAB_LastUpdate, BAOAB.h:167-186) runs first. mass[T],
 * damping3[T*3]; grids may be NULL (no PMF pass). */
void or_baoab_integrate(float* pos4, float* mom4, float* fe4, const int* type_ids,
                        const uint32_t* flags, size_t n, const or_types* types,
                        const or_grid* grids, const float* mass, const float* damping3,
                        const or_box* b, float dt, float kT, uint64_t step, uint64_t base_seed,
                        uint32_t base_ctr, const float* efield, int pending);
/* BAOAB_LastUpdate alone (Patch::finish_deferred_kick, Patch.cpp:354-373). */
void or_baoab_last_update(float* mom4, const float* fe4, const uint32_t* flags, size_t n,
                          float dt);
void or_bd_integrate(float* pos4, float* fe4, const int* type_ids, const uint32_t* flags, size_t n,
                     const or_types* types, const or_grid* grids, const or_box* b, float dt,
                     float kT, uint64_t step, uint64_t base_seed, uint32_t base_ctr,
                     const float* efield, float* noise4);

#ifdef __cplusplus
}
#endif
#endif
