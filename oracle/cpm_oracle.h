/*
 * cpm_oracle.h — CPU oracle for the TreePM gravity solve.
 *
 * TEST INFRASTRUCTURE ONLY. This is a C++17 restatement of the reference Rust
 * crate's per-step TreePM path (src/mesh.rs, src/fft.rs, src/poisson.rs,
 * src/tree.rs, src/integrator.rs, src/cosmology.rs, src/ics.rs), written so
 * that every f32 expression rounds in the reference's operation order
 * (compiled with -ffp-contract=off: no FMA contraction, as in Rust).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker or the timed CPU baseline. The
 * product (libcpm_cuda.so) never links or calls it.
 *
 * Parity pins: the reference's own known-answer tests (mesh.rs:101-183,
 * poisson.rs:114-165, tree.rs:382-430, integrator.rs:368-461,
 * cosmology.rs:110-139, ics.rs:189-266) are ported in tests/test_oracle_*.py.
 * Third-party arithmetic that is not under the reference tree is restated,
 * not reproduced: rustfft 6.4.1 lines (own mixed-radix Stockham FFT here),
 * libm 0.2.16 erfcf (glibc erfcf here), and the rand 0.10.3 / rand_distr
 * 0.6.0 IC white noise (own Philox-4x32-10 + Box-Muller here). Those three
 * are therefore pinned only through the reference's tolerance tests.
 */
#ifndef CPM_ORACLE_H
#define CPM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float omega_r, omega_m, omega_l, h0; } orc_cosmology;      /* cosmology.rs:9-16 */
typedef struct { float r_split, r_cut, softening, theta; } orc_split;        /* tree.rs:21-30 */
typedef struct { float amplitude, n_s; } orc_pspec;                          /* ics.rs:21-24 */

/* Test-fixture generators of the reference's unit tests. */
void orc_scattered_mesh(size_t count, float box, float* out3);                 /* mesh.rs:90-99 */
void orc_scattered_tree(size_t count, float box, uint64_t seed, float* out3);  /* tree.rs:340-349 */

/* mesh.rs */
void orc_stencil(int n, float box, const float* x3, int64_t* idx8, float* w8);                  /* :29-59 */
void orc_deposit(int n, float box, const float* x3, size_t np, float mass, float* cells);        /* :62-69 */
void orc_deposit_f64(int n, float box, const float* x3, size_t np, float mass, double* cells);   /* exact-sum twin */
float orc_interpolate(int n, float box, const float* cells, const float* x3);                   /* :72-77 */
void orc_interpolate_many(int n, float box, const float* cells, const float* x3, size_t np, float* out);
void orc_density_contrast(int n, float box, const float* x3, size_t np, float* delta);          /* integrator.rs:117-126 */

/* fft.rs: data is n^3 interleaved (re, im) f32, indexed (ix*n+iy)*n+iz. */
void orc_fft3(int n, float* data, int inverse);                                /* :28-72 */
float orc_wavenumber(size_t i, size_t n, float box);                           /* :86-95 */
void orc_fft3_f64(int n, double* data, int inverse);                           /* FP64 twin */

/* poisson.rs */
void orc_poisson_accel(int n, float box, const float* delta, float omega_m, float a, float r_split,
                       float* gx, float* gy, float* gz);
/* orc_poisson_accel with the Green's function divided by the CIC window squared (the library's
 * CPM_SIM_DECONVOLVE; the reference has no deconvolution). */
void orc_poisson_accel_deconvolved(int n, float box, const float* delta, float omega_m, float a, float r_split,
                                   float* gx, float* gy, float* gz);                       /* :33-88 */

/* tree.rs */
orc_split orc_split_with(float box, size_t mesh_n, size_t pps, float soft_scale, float theta); /* :40-50 */
float orc_short_range_factor(float r, float r_split);                          /* :54-57 */
void orc_tree_accelerations(const float* x3, size_t n, float box, const orc_split* s, float k,
                            float* acc3);                                       /* :314-323 */
/* Diagnostic: the same walk with node centres of mass summed in FP64 (rounded once to f32). */
void orc_tree_accelerations_com64(const float* x3, size_t n, float box, const orc_split* s, float k, float* acc3);
void orc_tree_accelerations_builtin(const float* x3, size_t n, float box, const orc_split* s, float k,
                                    float* acc3);                               /* BuiltTree::accel_on :103-150 */
void orc_brute_force(const float* x3, size_t n, float box, const orc_split* s, float k, float* acc3); /* :352-370 */
/* Tree introspection: returns the node count; when the arrays are non-null they receive, per node in
 * build order, center[3], half, com[3], count, start, end, children[8], depth. `order` receives the
 * final particle order. */
size_t orc_tree_build(const float* x3, size_t n, float box, float* center3, float* half, float* com3,
                      uint32_t* count, uint32_t* start, uint32_t* end, uint32_t* children8,
                      uint32_t* depth, uint32_t* order);
/* Interaction counts of the walk (leaf pairs and accepted nodes), summed over all particles. */
void orc_tree_walk_stats(const float* x3, size_t n, float box, const orc_split* s,
                         uint64_t* leaf_pairs, uint64_t* node_accepts, uint64_t* nodes_visited);

/* Octant keys of the tree's descent: digit d (1-based) of particle i is the octant chosen at depth d-1,
 * computed with the same f32 centre arithmetic as tree.rs:186-250 (x -> bit0, y -> bit1, z -> bit2). */
void orc_octant_keys(const float* x3, size_t n, float box, int levels, uint64_t* keys);
void orc_stable_sort_perm(const uint64_t* keys, size_t n, uint32_t* perm);

/* cosmology.rs */
float orc_cosmo_e(const orc_cosmology* c, float a);                            /* :32-34 */
float orc_growth(const orc_cosmology* c, float a);                             /* :82-84 */
float orc_growth_rate(const orc_cosmology* c, float a);                        /* :87-90 */
float orc_bbks(const orc_cosmology* c, float k);                               /* :94-103 */
orc_cosmology orc_lcdm_default(void);                                          /* :21-29 */

/* integrator.rs step factors (f32, Simpson 64, 60-step bisection) */
float orc_kick_factor(const orc_cosmology* c, float a0, float a1);             /* :263-265 */
float orc_drift_factor(const orc_cosmology* c, float a0, float a1);            /* :268-270 */
float orc_midpoint(const orc_cosmology* c, float a0, float a1);                /* :273-285 */
void orc_kick(float* p3, const float* g3, size_t n, float factor);             /* :301-307 */
void orc_drift(float* x3, const float* p3, size_t n, float factor, float box);  /* :310-316 */

/* integrator.rs Simulation: split == NULL means pure PM. */
typedef struct orc_sim orc_sim;
orc_sim* orc_sim_new(const orc_cosmology* c, float box, int mesh_n, const float* x3, const float* p3,
                     size_t n, float a, const orc_split* split);              /* :54-79 */
void orc_sim_step_to(orc_sim* s, float a1);                                    /* :174-186 */
void orc_sim_get(const orc_sim* s, float* x3, float* p3, float* acc3, float* delta, float* a);
void orc_sim_accelerations(const orc_sim* s, float a, float* acc3, float* delta); /* :140-161 */
void orc_sim_free(orc_sim* s);
/* Wall-clock seconds spent in the last step's phases: kick+drift, deposit, poisson, gather, tree build, walk. */
void orc_sim_last_timings(const orc_sim* s, double* t6);

/* Timed sample of one KDK step of the reference path (integrator.rs:174-186) on the state (x3, p3, acc3)
 * at a0 -> a1, for the CPU baseline. Every phase runs on all n particles except the tree walk, which
 * runs for the m particles listed in `subset` (the caller scales it by n / m). The state is not
 * modified. t7 receives seconds for: kick+drift, deposit, Poisson, gather, tree build, walk of the
 * subset, second kick. `threads` > 0 sets the OpenMP thread count. acc_subset (may be NULL) receives
 * the force at a1 (PM + tree) of the subset; acc_subset_com64 (may be NULL) the same with the tree's
 * centres of mass summed in FP64 and rounded once (the diagnostic twin of tree_accelerations),
 * computed outside the timed phases. */
void orc_step_sample(const orc_cosmology* c, float box, int mesh_n, const float* x3, const float* p3,
                     const float* acc3, size_t n, float a0, float a1, const orc_split* split,
                     const uint32_t* subset, size_t m, int threads, double* t7,
                     float* acc_subset, float* acc_subset_com64);

/* ics.rs */
float orc_power(const orc_cosmology* c, const orc_pspec* ps, float k);           /* :27-33 */
float orc_sigma(const orc_cosmology* c, const orc_pspec* ps, float radius);      /* :36-52 */
orc_pspec orc_power_normalized(const orc_cosmology* c, float n_s, float sigma8, float radius); /* :56-63 */
/* White noise of this project (Philox-4x32-10 + Box-Muller, one N(0,1) value per cell). */
void orc_white_noise(int n, uint64_t seed, float* out);
void orc_colored_modes(int n, float box, const orc_cosmology* c, const orc_pspec* ps, uint64_t seed,
                       float* modes /* 2*n^3 */);                              /* :78-109 */
void orc_zeldovich(int n, float box, const orc_cosmology* c, const orc_pspec* ps, float a_init,
                   uint64_t seed, float* x3, float* p3);                       /* :119-182 */

/* Power spectrum of a particle set (new, not in the reference): CIC on an n^3 mesh with FP64 sums and FP64 FFT,
 * P = V |F_k|^2 / M^2 (normalisation of ics.rs:243) binned in integer shells round(|m|) (ics.rs:229-241),
 * shells 1..n_shells. Outputs per shell: mean k, mean P, mode count. */
void orc_power_spectrum(const float* x3, size_t np, float box, int n, int n_shells, double* k_mean,
                        double* p_mean, uint64_t* counts);

/* FP64 build (cpm_oracle_f64.cpp): PM (poisson.rs:33-88) plus, when split is given, the short-range
 * tree force (tree.rs:171-323, coupling k_tree) in double precision at n_sample sampled particles
 * (indices into x3); acc3 is [n_sample][3]. The precision-study reference for f32 results. */
void orc64_accelerations(const float* x3, size_t n, double box, int mesh_n, double omega_m, double a,
                         const orc_split* split, double k_tree, const uint32_t* sample, size_t n_sample,
                         double* acc3);
/* orc64_accelerations with quadrupole terms at accepted nodes when `quadrupole` (the library's
 * CPM_SIM_QUADRUPOLE; the reference's nodes are monopoles). */
void orc64_accelerations_ex(const float* x3, size_t n, double box, int mesh_n, double omega_m, double a,
                            const orc_split* split, double k_tree, const uint32_t* sample, size_t n_sample,
                            double* acc3, int quadrupole);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
