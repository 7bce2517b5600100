/*
 * cpm.h — C ABI of libcpm_cuda.so, the B200 (sm_100a) TreePM gravity solve.
 *
 * Each entry point replaces one function of the reference crate's CPU path
 * (BenSmith1202/Cosmological-Particle-Simulation, src/mesh.rs, src/fft.rs,
 * src/poisson.rs, src/tree.rs, src/integrator.rs); the comment on each
 * declaration names the reference item (file:line) it stands in for.
 *
 * Conventions
 *  - Positions, momenta and accelerations are AoS f32 triples, exactly the
 *    memory of a Rust `&[[f32; 3]]` (12-byte stride): pass `as_ptr() as *const f32`.
 *  - Meshes are n^3 f32 cells indexed (ix*n + iy)*n + iz, z fastest (mesh.rs:11).
 *  - Complex data is interleaved {re, im} f32, the layout of num_complex's
 *    `#[repr(C)] Complex<f32>`.
 *  - Every call that takes host pointers copies to the device, computes, copies
 *    back and synchronises its context's stream before returning: it behaves like
 *    the synchronous Rust function it replaces.
 *  - Every function returns CPM_OK (0) or a negative CPM_E_* code; the text of the
 *    last error of a context is available from cpm_last_error(). The reference
 *    panics where these return an error (e.g. poisson.rs:35 asserts the mesh size);
 *    a Rust shim maps a non-zero code back to panic!.
 *  - A context is not thread-safe: use one per host thread (the reference calls
 *    the path from one worker thread, runner.rs:130).
 */
#ifndef CPM_H
#define CPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define CPM_OK 0
#define CPM_E_INVALID (-1)       /* null pointer, zero or negative size, bad enum value */
#define CPM_E_MESH_MISMATCH (-2) /* mesh size differs from the context's (poisson.rs:35) */
#define CPM_E_CAPACITY (-3)      /* more particles than the context or simulation holds */
#define CPM_E_UNSUPPORTED (-4)   /* mesh size whose FFT length this build does not compile (cpm_fft_supported) */
#define CPM_E_CUDA (-5)          /* a CUDA runtime call failed */
#define CPM_E_NONFINITE (-6)     /* NaN or infinite input position */
#define CPM_E_NOMEM (-7)         /* device allocation failed */
#define CPM_E_DEVICE (-8)        /* a kernel reported an error through its status word */
#define CPM_E_NO_DEVICE (-9)     /* no CUDA device, or not an sm_100 device */

/* ------------------------------------------------------------------ plain data */
typedef struct {
  float re, im;
} cpm_cf32; /* num_complex::Complex<f32> */

typedef struct {
  float omega_r, omega_m, omega_l, h0;
} cpm_cosmology; /* cosmology.rs:9-16 `Cosmology` (pub fields) */

typedef struct {
  float r_split, r_cut, softening, theta;
} cpm_force_split; /* tree.rs:21-30 `ForceSplit` */

typedef struct cpm_ctx cpm_ctx;
typedef struct cpm_sim cpm_sim;

/* ------------------------------------------------------------------ library */
/* Version string of the library build ("cpm <semver> sm_100a"). */
const char* cpm_version(void);
/* Text of the last error recorded on `ctx` (or of the last context-free failure when ctx is NULL). */
const char* cpm_last_error(const cpm_ctx* ctx);

/* ------------------------------------------------------------------ context (fine-grained API) */
/* Creates a context for meshes of n_mesh^3 cells in a periodic box of side `box_size`, with device
 * buffers for up to `max_particles` particles (they grow on demand). Owns one CUDA stream.
 * Replaces the state that `PoissonSolver::new(n, L)` (poisson.rs:23) and `Mesh::new(n, L)`
 * (mesh.rs:16) set up. flags: 0. */
int cpm_ctx_create(int n_mesh, float box_size, size_t max_particles, uint32_t flags, cpm_ctx** out);
int cpm_ctx_destroy(cpm_ctx* ctx);

/* mesh.rs:62-69 `Mesh::deposit(&mut self, positions, mass)`: clears `cells_out` (n^3) and deposits
 * `mass` per particle with CIC weights. Accumulates in 64-bit fixed point, so the result does not
 * depend on particle order and is the exactly-rounded sum of the reference's f32 weights. */
int cpm_mesh_deposit(cpm_ctx* ctx, const float* x3, size_t n, float mass, float* cells_out);

/* No counterpart in the reference. A variant of cpm_mesh_deposit for callers that cannot let a
 * library call cudaMalloc: programs whose device memory belongs to their own allocator or pool, or
 * loops in which an allocation's implicit device synchronisation would stall other streams.
 * Positions (x3_dev, AoS [n][3]) and the output mesh (cells_dev, n_mesh^3) are device pointers; the
 * work is enqueued on `stream` (a cudaStream_t, NULL for the default stream) and the call returns
 * without waiting. The only scratch is a static device array of 64^3 u64 cells plus a status word
 * (2 MiB per GPU, kept until exit): n_mesh above 64 returns CPM_E_CAPACITY. Nothing is allocated.
 * The first call on each device looks up the arrays' addresses (cudaGetSymbolAddress); make it
 * before any stream capture. All calls on a device share the arrays (cleared by every call); calls
 * that overlap on the GPU race on them. For finite positions the result equals cpm_mesh_deposit's;
 * a NaN or infinite coordinate (which cpm_mesh_deposit reports as CPM_E_NONFINITE) sets every
 * output cell to NaN, visible once the stream has synchronised. */
int cpm_mesh_deposit_noalloc(const float* x3_dev, size_t n, int n_mesh, float box_size, float mass, float* cells_dev,
                             void* stream);

/* integrator.rs:117-126 `Simulation::density_contrast`: deposit of unit masses, then
 * delta = c / (N / n^3) - 1 in f32. */
int cpm_density_contrast(cpm_ctx* ctx, const float* x3, size_t n, float* delta_out);

/* mesh.rs:72-77 `Mesh::interpolate`, batched over n positions: out[i] = sum of the 8 CIC
 * products in the reference's stencil order (bit-identical to the reference's f32 arithmetic). */
int cpm_mesh_interpolate(cpm_ctx* ctx, const float* cells, const float* x3, size_t n, float* out);

/* integrator.rs:144-148: the three components of the PM force at n positions from the meshes
 * returned by cpm_poisson_accel, one stencil per particle; out3 is AoS [n][3]. */
int cpm_mesh_interpolate3(cpm_ctx* ctx, const float* gx, const float* gy, const float* gz, const float* x3,
                          size_t n, float* out3);

/* No counterpart in the reference (rustfft takes any length). 1 when this build compiles the n-point
 * transforms every FFT user here needs (cpm_fft3, cpm_poisson_accel, simulations, initial
 * conditions, power spectra): n in {4, 8, 16, 32, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512,
 * 1024}; else 0, and those calls return CPM_E_UNSUPPORTED. Host only. */
int cpm_fft_supported(int n);

/* fft.rs:28-33 `Fft3::forward` / `Fft3::inverse`: unnormalised in-place c2c transform of n^3
 * complex values (forward e^{-ikx}, inverse e^{+ikx}). n must equal the context's mesh size. */
int cpm_fft3(cpm_ctx* ctx, cpm_cf32* data, int n, int inverse);

/* fft.rs:86-95 `wavenumber(i, n, L)` (host function; Nyquist index of an even grid -> 0). */
float cpm_wavenumber(size_t i, size_t n, float box_size);

/* poisson.rs:33-88 `PoissonSolver::acceleration(&delta, &cosmo, a, r_split) -> [Mesh; 3]`:
 * g = -grad phi with phi_k = -(3/2) Omega_m delta_k / (a k^2) exp(-k^2 r_split^2); k = 0 dropped.
 * delta, gx, gy, gz are n^3 meshes. Returns CPM_E_MESH_MISMATCH when n differs from the context. */
int cpm_poisson_accel(cpm_ctx* ctx, const float* delta, int n, const cpm_cosmology* cosmo, float a, float r_split,
                      float* gx, float* gy, float* gz);

/* tree.rs:40-50 `ForceSplit::with(L, mesh_n, particles_per_side, softening_scale, theta)` (host). */
cpm_force_split cpm_force_split_with(float box_size, size_t mesh_n, size_t particles_per_side,
                                     float softening_scale, float theta);

/* tree.rs:54-57 `short_range_factor(r, r_split)` (host, f32). */
float cpm_short_range_factor(float r, float r_split);

/* tree.rs:314-323 `tree::accelerations(positions, L, &split, k) -> Vec<[f32; 3]>`: builds the
 * octree of tree.rs:171-250 from octant keys and walks it on the GPU with the reference's rules
 * (prune by r_cut + sqrt(3) half, direct sum when octant 0 is empty, 2 half < theta r opening). */
int cpm_tree_accel(cpm_ctx* ctx, const float* x3, size_t n, float box_size, const cpm_force_split* split, float k,
                   float* acc3);

/* The octant keys of the tree descent (tree.rs:186-250: digit d is (x>=cx)|(y>=cy)<<1|(z>=cz)<<2 at
 * depth d-1, with the same f32 centre arithmetic; `levels` <= 21 digits, first digit most
 * significant) and the stable ascending sort permutation of those keys. Either output may be NULL.
 * The reference has no such entry point: it is the sort the tree build runs on. */
int cpm_octant_keys(cpm_ctx* ctx, const float* x3, size_t n, float box_size, int levels, uint64_t* keys_out,
                    uint32_t* perm_out);

/* Tree statistics of the last cpm_tree_accel on this context: node count, leaf-pair and
 * accepted-node interaction counts, maximum depth. Any pointer may be NULL. */
int cpm_tree_stats(cpm_ctx* ctx, uint64_t* nodes, uint64_t* leaf_pairs, uint64_t* node_accepts, uint32_t* max_depth);

/* ics.rs:119-182 `zeldovich(n, L, &cosmo, &ps, a_init, seed)` with
 * ps = `PowerSpectrum::normalized(&cosmo, n_s, sigma8, 8.0)` (ics.rs:56-63): n_side^3 particles on a
 * lattice (index (ix*n+iy)*n+iz), positions and momenta AoS [n^3][3]. The white noise is this
 * library's Philox-4x32-10 (counter = cell index, key = seed) with Box-Muller, not the reference's
 * rand::StdRng stream. */
int cpm_ics_zeldovich(int n_side, float box_size, const cpm_cosmology* cosmo, float n_s, float sigma8, float a_init,
                      uint64_t seed, float* x3, float* p3);

/* No counterpart in the reference, whose only power-spectrum estimator is inside the test
 * ics.rs:213-266. The same estimator (P = V |delta_k|^2 / M^2 averaged over integer shells
 * round(|m|), ics.rs:229-243, Nyquist modes included) applied to the CIC density of n particles
 * x3 on the context's mesh (mesh.rs:29-69; delta = rho/mean - 1 as integrator.rs:117-126).
 * Shell s = 1..n_shells (1 <= n_shells <= 2048) fills k_mean[s-1] (mean of 2 pi |m| / L over its
 * modes), p_mean[s-1] (mean power) and counts[s-1] (modes; 0 leaves k_mean and p_mean 0). The
 * context's mesh must be a supported FFT size (cpm_fft_supported). Sums are FP64; their last bits
 * may vary from run to run (atomic summation order). */
int cpm_power_spectrum(cpm_ctx* ctx, const float* x3, size_t n, int n_shells, double* k_mean, double* p_mean,
                       uint64_t* counts);

/* frame.rs:30-55 `downsample_grid(delta)`: the viewer's gas texture, 1 + delta averaged over f^3
 * blocks with f = ceil(n / 128) (frame.rs:27 MAX_GRID), side m = n / f (grid_n), ordered x fastest
 * then y then z (the mesh is z fastest, so this transposes). delta is the context's n^3 mesh
 * (CPM_E_MESH_MISMATCH otherwise); grid holds m^3 floats; grid_n may be NULL. Bit-identical to the
 * reference's f32 sums. */
int cpm_density_grid(cpm_ctx* ctx, const float* delta, int n, float* grid, int* grid_n);

/* ------------------------------------------------------------------ learned short-range force */
/* No counterpart in the reference, which computes the whole short-range force with the tree walk
 * (tree.rs:264-310). A 3-layer 3x3x3 periodic convolutional net (16 channels, leaky ReLU with slope
 * 1/8 after layers 1 and 2, no biases) maps the density contrast delta of an n^3 mesh to a 3-channel
 * acceleration field F = out_scale * net(in_scale * delta), evaluated with BF16 tcgen05 tensor-core
 * kernels accumulating in FP32; a simulation gathers F to particles with the CIC stencil
 * (mesh.rs:72-77). Weights are FP32 masters W[layer][tap][out][in], 3 x 27 x 16 x 16 floats, tap
 * (dx+1)*9 + (dy+1)*3 + (dz+1), out[v] = sum_t W[t] in[v + t]; layer 1 reads input channel 0 only,
 * layer 3 writes channels 0-2 only (other entries are kept at 0). Device pointers; calls enqueue on
 * `stream` (cudaStream_t, NULL = default) and synchronise it before returning. */
typedef struct cpm_net cpm_net;
/* Number of master weights (3 * 27 * 16 * 16). */
int cpm_net_weight_count(void);
/* A net with device buffers for n_mesh^3 meshes (n_mesh a multiple of 16 in [16, 1024]); weights 0. */
int cpm_net_create(int n_mesh, cpm_net** out);
int cpm_net_destroy(cpm_net* net);
const char* cpm_net_last_error(const cpm_net* net);
/* Host arrays of cpm_net_weight_count() floats. Setting weights resets the Adam state. */
int cpm_net_set_weights(cpm_net* net, const float* w);
int cpm_net_get_weights(cpm_net* net, float* w);
/* The weight gradient of the last cpm_net_backward or cpm_net_train_step (host array). */
int cpm_net_get_grads(cpm_net* net, float* g);
/* field4_dev[(x*n + y)*n + z] = (F_x, F_y, F_z, 0) from delta_dev[n^3] (f32). */
int cpm_net_forward(cpm_net* net, const float* delta_dev, float in_scale, float out_scale, float* field4_dev,
                    void* stream);
/* Weight gradient of a loss L from dL/dF (dfield4_dev, float4 per cell) for the last forward of this
 * net with output scale out_scale. */
int cpm_net_backward(cpm_net* net, const float* dfield4_dev, float out_scale, void* stream);
/* Copies one internal BF16 tensor ([x][y][2][n+8][8], z padded by a periodic halo) to dst_dev:
 * 0 input, 1 and 2 the activations of layers 1 and 2, 3..5 the gradients of layers 3, 2, 1. */
int cpm_net_activations(cpm_net* net, int which, void* dst_dev, void* stream);
/* One training step on one mesh and its particles: F = net(in_scale * delta) (out_scale 1), the
 * loss L = inv_norm * sum_i weight_i |F(x_i) - target_i|^2 (CIC gather of F at x_i), its gradient by
 * the backward kernels, then one Adam step (b1 0.9, b2 0.999, eps 1e-8) with learning rate lr
 * (lr = 0: gradient only). loss_out (may be NULL) receives L before the update. */
int cpm_net_train_step(cpm_net* net, const float* delta_dev, float in_scale, const float* x3_dev,
                       const float* target3_dev, const float* weight_dev, size_t n_particles, float box_size,
                       float inv_norm, float lr, double* loss_out, void* stream);

/* ------------------------------------------------------------------ device-resident simulation */
/* Replaces `Simulation` (integrator.rs:34-186) under a `cuda` feature: state stays in HBM and
 * `step_to` runs one KDK step (kick, drift, deposit, FFT-Poisson, gather, tree build and walk,
 * kick) as one CUDA graph (see CPM_SIM_NO_GRAPH). */
typedef struct {
  cpm_cosmology cosmo;
  float box_size;
  int mesh_n;
  size_t n_particles;
  int use_tree;           /* 0: pure PM (split == None); 1: TreePM with `split` */
  cpm_force_split split;
  uint32_t flags;         /* CPM_SIM_* below */
} cpm_sim_params;

/* Positions as uint32 fixed point (x = q L / 2^32): the drift adds round(p d 2^32 / L) (FP64
 * product) modulo 2^32, so the periodic wrap is exact and the resolution is L / 2^32 anywhere in
 * the box (displacements per step must stay below L/2). Positions given by the caller are rounded
 * to that grid; the force kernels read the f32 value of q. Precision mode; the default f32 mode is
 * the reference's arithmetic (integrator.rs:309-316). */
#define CPM_SIM_FIXED_POINT 0x1u
/* Divide the PM Green's function by the CIC window squared (the reference does not). */
#define CPM_SIM_DECONVOLVE 0x2u
/* Record per-phase CUDA-event timings for cpm_sim_phase_times(). The step then runs uncaptured
 * (as under CPM_SIM_NO_GRAPH), with the event records between its kernels. */
#define CPM_SIM_TIMING 0x4u
/* Run the step without CUDA-graph capture (each kernel launched directly). By default the first
 * two steps run uncaptured (they allocate the sort and tree buffers) and each later step replays
 * one of two captured graphs (the sorted particle buffers alternate between them); CPM_SIM_TIMING
 * also runs every step uncaptured. */
#define CPM_SIM_NO_GRAPH 0x8u
/* Quadrupole moments in the tree (no counterpart in the reference, whose nodes are monopoles,
 * tree.rs:68-80): every node that the walk can accept carries the second moments of its particles
 * about their centre of mass, and an accepted node adds the second-order Taylor term of the
 * short-range kernel to its monopole force. Precision mode (use with CPM_SIM_FIXED_POINT); it
 * changes the forces, so plain parity with the reference holds without it. */
#define CPM_SIM_QUADRUPOLE 0x10u
/* Skip the autotuner (see cpm_sim_autotune_report) and keep the default launch choices. */
#define CPM_SIM_NO_AUTOTUNE 0x20u

/* integrator.rs:54-79 `Simulation::new`: uploads x3, p3 (AoS [n][3]) and computes the initial
 * acceleration at a0. */
int cpm_sim_create(const cpm_sim_params* params, const float* x3, const float* p3, float a0, cpm_sim** out);
/* runner.rs:209-225 `init_simulation` without the host round trip: Zel'dovich ICs of n_side^3
 * particles (ics.rs:119-182, spectrum PowerSpectrum::normalized(cosmo, n_s, sigma8, 8), ics.rs:56)
 * generated on the GPU into the simulation, then `Simulation::new` (integrator.rs:54-79) at a0.
 * params->n_particles must equal n_side^3. White noise: Philox-4x32-10 + Box-Muller (see
 * cpm_ics_zeldovich). */
int cpm_sim_create_zeldovich(const cpm_sim_params* params, int n_side, float n_s, float sigma8, float a0,
                             uint64_t seed, cpm_sim** out);
/* integrator.rs:174-186 `Simulation::step_to(a1)`. Kick and drift factors are the reference's f32
 * Simpson/bisection values (integrator.rs:263-297), computed on the host. */
int cpm_sim_step_to(cpm_sim* sim, float a1);
/* `Simulation::step_to(a1)` for a caller that owns the state on the host (the reference's pub
 * `positions` and `momenta`, integrator.rs:39-40): uploads x3 and p3 (caller order), runs one step
 * with the simulation's cached acceleration for the first half-kick (the reference's private
 * `accel`), and writes the new x3 and p3 back. Synchronous. The step runs uncaptured: the new
 * positions are copied back on a second, library-owned stream as soon as the step has sorted
 * them, overlapping the force computation; x3 must not be read or written by the caller until
 * the call returns (pinned host memory gives the fastest copies). */
int cpm_sim_step_host(cpm_sim* sim, float a1, float* x3, float* p3);
/* Reads the state in the caller's particle order. Any pointer may be NULL. delta is n^3. */
int cpm_sim_get_state(cpm_sim* sim, float* x3, float* p3, float* acc3, float* delta, float* a);
/* Number of captured step graphs (0 before the third step, under CPM_SIM_NO_GRAPH or
 * CPM_SIM_TIMING, or when capture failed and the steps run uncaptured; 2 once both buffer
 * parities are captured). */
int cpm_sim_graphs(cpm_sim* sim);
/* runner.rs:263-284 `snapshot(&sim, want_grid)` and the max speed of runner.rs:244-247, computed on
 * the device (no particle copy to the host beyond the outputs asked for). In the caller's particle
 * order: speeds[n] = |p| / a (frame.rs:9-10); densities[n] = max(1 + delta(x), 0), delta the mesh
 * of the last force evaluation interpolated by CIC (mesh.rs:72-77); rsd3[n][3] = p / (a^2 E(a))
 * (frame.rs:62-69); grid = downsample_grid(delta) as cpm_density_grid (grid_n receives its side);
 * max_speed = the largest speed. Any pointer may be NULL. Bit-identical to the reference's f32
 * arithmetic for equal state. */
int cpm_sim_snapshot(cpm_sim* sim, float* speeds, float* densities, float* rsd3, float* grid, int* grid_n,
                     float* max_speed);
/* cpm_power_spectrum of the simulation's current particles on its mesh, without copying them. */
int cpm_sim_power_spectrum(cpm_sim* sim, int n_shells, double* k_mean, double* p_mean, uint64_t* counts);
/* Overwrites positions and momenta (caller's order) and recomputes the acceleration at the current a. */
int cpm_sim_set_state(cpm_sim* sim, const float* x3, const float* p3);
/* Average device milliseconds per step of each phase since the last reset (needs CPM_SIM_TIMING):
 * [0] kick+drift, [1] keys+sort+reorder, [2] deposit, [3] FFT-Poisson, [4] gather, [5] tree build,
 * [6] tree walk, [7] whole step. Also the number of steps averaged. */
int cpm_sim_phase_times(cpm_sim* sim, double* ms8, uint64_t* steps, int reset);
/* (particle, source) pairs the last step's walk tested against r_cut inside direct-summed nodes
 * (leaf pairs are the subset within r_cut). */
int cpm_sim_walk_candidates(cpm_sim* sim, uint64_t* candidates);
/* Self-check of the walk's pair kernel (host only): largest relative error of its fitted
 * S(r) = erfc(u) + (2/sqrt(pi)) u e^{-u^2}, u = r / (2 r_split) (tree.rs:54-57), against a
 * double-precision evaluation on `samples` points of [0, r_cut]. */
int cpm_walk_kernel_fit_error(float r_split, float r_cut, int samples, double* max_rel_err);
/* Self-check of the simulation's Hilbert sort keys (host only): the keys are computed digit by
 * digit by a state machine derived from the Hilbert transform; this compares the two on `samples`
 * random integer coordinates of `levels` (21, or 19 under a batch of boxes) bits per axis and
 * reports the mismatches and the machine's number of states (0 when it could not be derived, in
 * which case the device computes the transform directly). */
int cpm_hilbert_fsm_check(int levels, uint64_t samples, uint64_t seed, uint64_t* mismatches, int* states);
/* Device-side counters of the last step: nodes, leaf pairs, accepted nodes, kernels launched per step. */
int cpm_sim_counters(cpm_sim* sim, uint64_t* nodes, uint64_t* leaf_pairs, uint64_t* node_accepts,
                     uint32_t* launches_per_step);
/* No counterpart in the reference. Attaches a learned short-range net (NULL detaches it): from the
 * next step on, the short-range force of particles whose CIC-interpolated density contrast is below
 * delta_threshold is the net's field F = K(a) (N / n^3) / h * net(in_scale * delta), gathered with
 * the CIC stencil (mesh.rs:72-77); the tree walk (tree.rs:264-310) runs only for the others. The
 * net's mesh must equal the simulation's (CPM_E_MESH_MISMATCH) and the simulation must use the tree.
 * The captured step graphs are rebuilt. The simulation does not own the net. */
int cpm_sim_set_learned(cpm_sim* sim, cpm_net* net, float delta_threshold, float in_scale);
/* The short-range tree force alone of the current state, tree::accelerations (tree.rs:314-323) on
 * the current positions with K(a) of the current a, in the caller's particle order (AoS [n][3]).
 * No counterpart as a separate call in the reference (integrator.rs:149-159 adds it to the PM
 * force); the training targets of the learned short-range net. */
int cpm_sim_short_range(cpm_sim* sim, float* sr3);
/* State file (the snapshot writer the reference planned but did not build, plan.md:160-161): the
 * positions and momenta in the caller's order, a, and every cpm_sim_params field, with a checksum of
 * the payload. cpm_sim_load creates a simulation from it (flags | extra_flags) whose next steps equal
 * those of the saved simulation; CPM_E_INVALID for a missing, foreign or corrupt file. */
int cpm_sim_save(cpm_sim* sim, const char* path);
int cpm_sim_load(const char* path, uint32_t extra_flags, cpm_sim** out);
/* The factors of one KDK step from a0 to a1: k1 = kick_factor(a0, a_mid), d = drift_factor(a0, a1),
 * k2 = kick_factor(a_mid, a1) with a_mid = midpoint(a0, a1) (integrator.rs:263-297, private there).
 * fp64 = 0: the reference's f32 Simpson/bisection on the host (what every plain simulation step
 * uses); fp64 = 1: the FP64 device computation of CPM_SIM_FIXED_POINT steps (256 Simpson
 * intervals; d is returned unrounded, k1 and k2 as the f32 values the kicks use). */
int cpm_step_factors(const cpm_cosmology* cosmo, double a0, double a1, int fp64, double* k1, double* d, double* k2);
/* No counterpart in the reference. The launch choices the autotuner made when the simulation was
 * created (each candidate timed on the simulation's own first state; cached per workload, and in the
 * file named by the environment variable CPM_TUNE_CACHE when set): the FFT plan of the Poisson passes
 * (8 or 4: shared-memory Stockham stages of largest radix 8 or 4 over the CTA; 0: one warp per
 * 256- or 512-point line with register stages, radix 8 for other lengths), the deposit tile (512,
 * 1024 or 2048 sorted particles per CTA) and the walk group (2, 4 or 8 warps of 32 particles per
 * block). ms9 (may be NULL) receives the measured ms per call: plan 8, 4, 0; tile 512, 1024, 2048;
 * warps 2, 4, 8 (0 where not timed). */
int cpm_sim_autotune_report(cpm_sim* sim, int* fft_radix, int* deposit_tile, int* walk_warps, float* ms9);
/* Overrides the autotuner's choices (FFT plan 8, 4 or 0, tile 512, 1024 or 2048, warps 2, 4 or 8); the
 * next force evaluation uses them. Deposit tile and walk group do not change any result bit; the FFT
 * plan changes FFT rounding only. */
int cpm_sim_set_tuning(cpm_sim* sim, int fft_radix, int deposit_tile, int walk_warps);
/* The last tree build's deepest split level, and the number of nodes with more than 8 particles
 * kept as leaves because their particles share every key digit (21 digits; 19 in an ensemble's
 * batch). The reference splits such nodes down to MAX_DEPTH = 40 (tree.rs:13, :211), so a non-zero
 * count marks states where the GPU's tree departs from the reference's. */
int cpm_sim_tree_depth(cpm_sim* sim, uint32_t* max_depth, uint64_t* key_depth_leaves);
/* Particles the last step walked the tree for (all of them without a net). */
int cpm_sim_learned_walked(cpm_sim* sim, uint64_t* walked);
/* The CUDA stream the simulation launches on (cudaStream_t), for callers that time with events. */
void* cpm_sim_stream(cpm_sim* sim);
int cpm_sim_destroy(cpm_sim* sim);

/* ------------------------------------------------------------------ ensembles of realisations */
/* No counterpart in the reference, which runs one realisation per run (runner.rs:228-260). An
 * ensemble holds many independent realisations of uneven sizes, grouped in classes of equal size.
 * Every box of a class shares one launch per phase (keys with the box index above the octant digits,
 * one sort, one deposit into the boxes' meshes, batched FFT passes, one gather, one tree build with a
 * root per box, one walk), and one ensemble step is one CUDA graph in which the classes run as
 * parallel branches. Each box is a Simulation of the reference's step (integrator.rs:174-186) with
 * the class's mesh and split, Zel'dovich ICs (ics.rs:119-182, as cpm_sim_create_zeldovich) from seed
 * first_seed + b, and the common box size, cosmology and schedule; steps are autotuned per class. */
typedef struct cpm_ensemble cpm_ensemble;
typedef struct {
  int n_side;           /* particles per side of every box of the class; n_side^3 a multiple of 2048 */
  int mesh_n;           /* mesh cells per side (a supported FFT length up to 512) */
  int n_boxes;          /* realisations of the class, 1..64 */
  uint64_t first_seed;  /* box b uses seed first_seed + b */
  cpm_force_split split;
} cpm_ensemble_class;
/* 1..16 classes; flags: CPM_SIM_FIXED_POINT, CPM_SIM_DECONVOLVE, CPM_SIM_NO_GRAPH, CPM_SIM_NO_AUTOTUNE. */
int cpm_ensemble_create(const cpm_cosmology* cosmo, float box_size, float n_s, float sigma8, float a0, int n_classes,
                        const cpm_ensemble_class* classes, uint32_t flags, cpm_ensemble** out);
/* One KDK step of every realisation to a1 (the third and later steps replay a captured graph). */
int cpm_ensemble_step_to(cpm_ensemble* ens, float a1);
/* Positions, momenta and accelerations (any may be NULL) of box `box` of class `cls`, in the box's
 * lattice order (AoS [n_side^3][3]). Synchronous. */
int cpm_ensemble_get_state(cpm_ensemble* ens, int cls, int box, float* x3, float* p3, float* acc3);
/* cpm_sim_power_spectrum of one box. */
int cpm_ensemble_power_spectrum(cpm_ensemble* ens, int cls, int box, int n_shells, double* k_mean, double* p_mean,
                                uint64_t* counts);
/* Captured step graphs (0, 1 or 2) and the stream the steps run on (cudaStream_t). */
int cpm_ensemble_graphs(cpm_ensemble* ens);
void* cpm_ensemble_stream(cpm_ensemble* ens);
const char* cpm_ensemble_last_error(const cpm_ensemble* ens);
int cpm_ensemble_destroy(cpm_ensemble* ens);

#ifdef __cplusplus
}
#endif
#endif /* CPM_H */
