// cpm_internal.cuh — shared device helpers and launcher declarations of libcpm_cuda.so.
//
// Arithmetic that must round exactly like the reference's Rust f32 code (CIC stencil and
// gather, density contrast, Green's function, kick/drift, the tree's accept/prune tests) is
// written with __fmul_rn/__fadd_rn/__fdiv_rn, which the compiler never contracts into FMAs.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cpm.h"

namespace cpm {

// ---------------------------------------------------------------------------------------------
// Status word written by kernels (no __trap, no device assert): the first error wins.
// ---------------------------------------------------------------------------------------------
enum DevError : int {
  DEV_OK = 0,
  DEV_NONFINITE = 1,        // NaN / Inf position
  DEV_NODE_CAPACITY = 2,    // octree needs more nodes than allocated
  DEV_STACK_OVERFLOW = 3,   // walk stack deeper than its bound
  DEV_DEPTH_LIMIT = 4,      // more than LEAF_SIZE particles share all key digits (informational)
};

struct DevStatus {
  int code;
  int detail;
};

__device__ __forceinline__ void dev_fail(DevStatus* st, int code, int detail) {
  if (atomicCAS(&st->code, 0, code) == 0) st->detail = detail;
}

// Kernels launched by this library (every launch site calls count_launch() first).
unsigned long long launch_count();
void count_launch();

// ---------------------------------------------------------------------------------------------
// Reference constants (tree.rs:12-17)
// ---------------------------------------------------------------------------------------------
constexpr int LEAF_SIZE = 8;
constexpr int MAX_DEPTH = 40;
constexpr int KEY_LEVELS = 21;  // 63-bit octant keys
constexpr float SQRT_3 = 1.7320508f;
constexpr float TWO_OVER_SQRT_PI = 1.1283792f;

// ---------------------------------------------------------------------------------------------
// mesh.rs:29-59 — CIC stencil, bit-identical to the reference's f32 arithmetic.
// ---------------------------------------------------------------------------------------------
struct CicBase {
  int b[3];    // floor(x/h - 1/2)
  float f[3];  // fractional part
};

// Cell base of one axis. The reference casts floor(s) to i64 (saturating; NaN -> 0) and wraps
// base + d with rem_euclid (mesh.rs:36-53). Positions inside [0, L] give a base in [-1, n] and are
// kept as is (the deposit's tiles rely on unwrapped neighbours being adjacent); any other value
// is reduced modulo n in 64-bit arithmetic, which selects the same cells as the reference and
// keeps every base in [-1, n], so no index or tile extent computed from it can overflow.
__device__ __forceinline__ int cic_axis_base(float i0, int n) {
  if (i0 >= -1.0f && i0 <= (float)n) return (int)i0;
  const long long b = __float2ll_rz(i0);  // i0 is integral (or +-inf / NaN): saturating conversion
  long long r = b % (long long)n;
  if (r < 0) r += n;
  return (int)r;
}

__device__ __forceinline__ void cic_base(const float x[3], float h, int n, CicBase& c) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float s = __fsub_rn(__fdiv_rn(x[k], h), 0.5f);
    const float i0 = floorf(s);
    c.b[k] = cic_axis_base(i0, n);
    c.f[k] = __fsub_rn(s, i0);
  }
}

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// mesh.rs:81-83
__device__ __forceinline__ float axis_weight(float f, int d) { return d == 0 ? __fsub_rn(1.0f, f) : f; }

// Weight of corner c (c = dx*4 + dy*2 + dz, the reference's loop order).
__device__ __forceinline__ float cic_weight(const CicBase& c, int corner) {
  const int dx = (corner >> 2) & 1, dy = (corner >> 1) & 1, dz = corner & 1;
  return __fmul_rn(__fmul_rn(axis_weight(c.f[0], dx), axis_weight(c.f[1], dy)), axis_weight(c.f[2], dz));
}

__device__ __forceinline__ size_t cic_index(const CicBase& c, int corner, int n) {
  const int dx = (corner >> 2) & 1, dy = (corner >> 1) & 1, dz = corner & 1;
  const size_t ix = (size_t)wrap_index(c.b[0] + dx, n);
  const size_t iy = (size_t)wrap_index(c.b[1] + dy, n);
  const size_t iz = (size_t)wrap_index(c.b[2] + dz, n);
  return (ix * (size_t)n + iy) * (size_t)n + iz;
}

// fft.rs:86-95 with two_pi_over_l = (2 * (f32)pi) / L precomputed on the host.
__device__ __forceinline__ float wavenumber(int i, int n, float two_pi_over_l) {
  if ((n & 1) == 0 && i == n / 2) return 0.0f;
  if (i <= n / 2) return __fmul_rn((float)i, two_pi_over_l);
  return __fmul_rn(__fsub_rn((float)i, (float)n), two_pi_over_l);
}

// f32::rem_euclid (Rust std) for the drift (integrator.rs:313).
__device__ __forceinline__ float rem_euclid_f32(float v, float rhs) {
  const float r = fmodf(v, rhs);
  return r < 0.0f ? __fadd_rn(r, fabsf(rhs)) : r;
}

// ---------------------------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

cudaError_t ensure(DevBuf& b, size_t bytes);
void release(DevBuf& b);

template <typename T>
T* as(DevBuf& b) {
  return static_cast<T*>(b.p);
}

// ---------------------------------------------------------------------------------------------
// Radix sort of (u64 key, u32 value) pairs — keys.cu / sort.cu
// ---------------------------------------------------------------------------------------------
struct SortScratch {
  DevBuf keys_alt, vals_alt, block_hist, scan_tmp;
};

// Octant keys (tree.rs descent) of positions (AoS f32 or float4), values = 0..n-1.
// With n_box > 0 (a batch of boxes of n_box particles each, in box order), the box index is placed
// above the 3 * levels octant bits. With hkeys, also the Hilbert keys of the same cubes (the same
// box bits): sorted by them, every octree node's particles stay contiguous.
void launch_octant_keys(const float* x3, size_t n, float box, int levels, uint64_t* keys, uint32_t* vals,
                        DevStatus* st, cudaStream_t s, size_t n_box = 0, uint64_t* hkeys = nullptr);
void launch_permute_u64(const uint64_t* in, const uint32_t* perm, size_t n, uint64_t* out, cudaStream_t s);
// Stable LSD sort of the low `bits` bits of keys; result in keys/vals (ping-pong handled inside).
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, size_t n, int bits, SortScratch& sc,
                             cudaStream_t s);
// Exclusive scan of u32 (in place allowed); `tmp` is grown as needed.
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, DevBuf& tmp, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Deposit — deposit.cu
// ---------------------------------------------------------------------------------------------
// Fixed-point scale exponent for masses summing to at most `total_mass`.
int fixed_point_shift(double total_mass);
// CIC deposit of `mass` per particle into the u64 fixed-point mesh (zeroed inside); tiles of
// 256 * ppt sorted particles per CTA (ppt 2, 4 or 8).
void launch_deposit_fixed(const float* x3, size_t n, float mass, int mesh_n, float h, int shift,
                          unsigned long long* mesh_fx, cudaStream_t s, int ppt = 4, size_t n_box = 0);
// cells = (float)fx * 2^-shift, or delta = cells / mean - 1 when to_delta.
void launch_fixed_to_f32(const unsigned long long* fx, size_t m, int shift, int to_delta, float mean, float* out,
                         cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// FFT / Poisson — fft.cu
// ---------------------------------------------------------------------------------------------
// Mesh sizes with compiled transforms (powers of two 4..1024 and some 2^a 3^b 5^c sizes).
bool fft_supported(int n);
bool poisson_supported(int n);
const char* fft_sizes_text();  // the list of supported sizes, for error messages
struct FftPlan {
  int n = 0;
  int max_radix = 8;  // radix plan of the Poisson passes: 8 (8.8.8 for 512) or 4 (4.4.4.4.2); autotuned
  DevBuf twiddle;  // exp(-2 pi i m / n), m < n, float2 built from double
  DevBuf deconv;   // per-axis 1 / sinc^4(pi m / n): CIC window of deposit and gather, squared
};
// Elements of one half spectrum [n][n][n/2+2] (one padding column per row).
size_t half_spectrum_elems(int n);
cudaError_t fft_plan_init(FftPlan& p, int n);
void fft_plan_free(FftPlan& p);
// In-place unnormalised c2c n^3 transform (z, then y, then x lines).
void launch_fft3_c2c(const FftPlan& p, float2* data, int inverse, cudaStream_t s);

struct PoissonParams {
  int n;
  float two_pi_over_l;
  float prefactor;  // 1.5 Omega_m / a (f32)
  float r_split;
  float scale;      // 1 / n^3 (f32)
  int deconvolve;
  const float* prefactor_dev = nullptr;  // when set, the prefactor is read from device memory
  int boxes = 1;  // a batch of meshes of the same size, one after another (meshes up to 512)
};
// Input: either f32 delta (delta != nullptr) or the u64 fixed-point mass mesh (fx != nullptr,
// converted to delta = c/mean - 1 on load). Output: three f32 meshes. spec: 3 half spectra
// of n*n*(n/2+1) float2 each; slot 0 also holds the forward spectrum.
void launch_poisson(const FftPlan& p, const PoissonParams& pp, const float* delta, const unsigned long long* fx,
                    int fx_shift, float mean, float2* spec, float* gx, float* gy, float* gz, cudaStream_t s);

// Forward R2C transform (same inputs as launch_poisson) into one padded half spectrum.
void launch_r2c3(const FftPlan& p, const float* delta, const unsigned long long* fx, int fx_shift, float mean,
                 float2* spec, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Power spectrum — pk.cu
// ---------------------------------------------------------------------------------------------
constexpr int PK_MAX_SHELLS = 2048;
struct PkSums {
  double power[PK_MAX_SHELLS + 1];  // sum over modes of |F_k|^2, shell s at index s
  double kabs[PK_MAX_SHELLS + 1];   // sum over modes of |m|
  unsigned long long count[PK_MAX_SHELLS + 1];
};
// Accumulates the half spectrum of an n^3 real field into integer shells 1..n_shells of `sums`
// (zeroed inside); modes with 0 < kz < n/2 stand for themselves and their Hermitian mirror.
void launch_pk_bin(const float2* spec, int n, int n_shells, PkSums* sums, cudaStream_t s);
// P(k) from the shell sums: k_mean = (2 pi / L) sum|m| / count, p_mean = L^3 sum|F|^2 / (M^2 count).
void pk_finish(const PkSums& sums, int n, float box, int n_shells, double* k_mean, double* p_mean, uint64_t* counts);

// ---------------------------------------------------------------------------------------------
// Gather — gather.cu
// ---------------------------------------------------------------------------------------------
void launch_interpolate(const float* cells, const float* x3, size_t n, int mesh_n, float h, float* out,
                        cudaStream_t s);
// out3[i] = (interp gx, gy, gz)[i]; when `add` != 0, out3 += that instead (f32 add in reference order).
void launch_interpolate3(const float* gx, const float* gy, const float* gz, const float* x3, size_t n, int mesh_n,
                         float h, float* out3, cudaStream_t s, size_t n_box = 0);

// ---------------------------------------------------------------------------------------------
// Tree — tree.cu
// ---------------------------------------------------------------------------------------------
struct TreeNodes {
  DevBuf geo;    // float4 centre.xyz, half
  DevBuf mass;   // float4 com.xyz, count
  DevBuf link;   // uint4 start, end, first_child, child_mask | depth << 8
  DevBuf counters;  // u32[64]: per-level allocation counts, totals
  DevBuf prefix;    // double prefix sums of sorted positions (3 per particle + 3)
  DevBuf scan_tmp;
  DevBuf x4;        // float4 copy of the sorted positions for the walk
  DevBuf quad;      // per node 2 float4: second moments about the centre of mass (quadrupole mode)
  bool has_quad = false;  // the last build computed `quad`; the walk then adds quadrupole terms
  int walk_warps = 4;     // warps (groups of 32 particles) per walk block: 2, 4 or 8 (autotuned)
  uint32_t n_box = 0;     // batch of boxes: particles per box (a multiple of 32), root of group = box
  size_t capacity = 0;
  void* walk_fit = nullptr;  // fitted pair-force coefficients of the last split (walk.cu)
};
struct TreeCounters {
  unsigned long long leaf_pairs;    // pairs within r_cut summed directly
  unsigned long long node_accepts;  // accepted centres of mass
  unsigned long long candidates;    // (particle, source) pairs tested against r_cut in direct nodes
  unsigned long long reserved;
};
// Builds the octree over sorted keys/positions (sorted x as AoS f32). Returns the node count
// through the counters buffer (read by tree_node_count). quad_half_max > 0 also computes the second
// moments of every node with half < quad_half_max (the walk then adds quadrupole terms).
// With n_box > 0 the keys hold a batch of boxes (box index above `levels` octant digits, boxes of
// n_box particles in order): one root per box (nodes 0 .. boxes - 1), and the walk starts each
// group of 32 particles at its box's root.
// sorted_keys orders the particles: octant keys, or Hilbert keys (then octant_keys gives each
// particle's octant key in the same order, from which a child's octant is read); a node's children
// are stored in the order of its sort digits.
cudaError_t tree_build(TreeNodes& t, const uint64_t* sorted_keys, const float* sorted_x3, size_t n, float box,
                       DevStatus* st, cudaStream_t s, float quad_half_max = 0.0f, int levels = KEY_LEVELS,
                       size_t n_box = 0, const uint64_t* octant_keys = nullptr);
// Half size from which a node can never be accepted by the walk (prune radius r_cut + sqrt(3) half
// from the centre, centre of mass inside the cube, 2 half < theta r): +inf when theta >= 1/sqrt(3).
float quad_half_bound(const cpm_force_split& split);
// Walks the tree for every sorted particle; acc3 (sorted order) receives g_sr, or g + g_sr
// when `accumulate` (the reference's g[c] += s[c], integrator.rs:154-158).
// The coupling k is read from *k_dev when k_dev is set. With `list`, only the sorted particles
// list[0 .. *list_n - 1] are walked (the grid is sized for n; the count is read on the device).
void launch_tree_walk(const TreeNodes& t, const float* sorted_x3, size_t n, float box, const cpm_force_split& split,
                      float k, float* acc3, int accumulate, TreeCounters* counters, DevStatus* st, cudaStream_t s,
                      const float* k_dev = nullptr, const uint32_t* list = nullptr, const uint32_t* list_n = nullptr);
// Releases the walk's per-tree state (the fitted pair-force coefficients).
void tree_walk_free(TreeNodes& t);
// ---------------------------------------------------------------------------------------------
// Particle updates — kdk.cu
// ---------------------------------------------------------------------------------------------
// The scalars of one simulation step, kept in device memory and read by its kernels, so that one
// captured CUDA graph serves every step (a one-thread kernel writes them before each launch).
struct StepScalars {
  float k1;         // first half-kick factor, kick_factor(a0, a_mid)
  float d;          // drift factor, drift_factor(a0, a1)
  float k2;         // second half-kick factor, kick_factor(a_mid, a1)
  float prefactor;  // Green's function prefactor 1.5 Omega_m / a1
  float tree_k;     // short-range coupling K(a1)
  float net_scale;  // output scale of the learned short-range field, K(a1) (N / M) / h
  float pad_;
  double d64;       // drift factor in FP64 (precision mode: the fixed-point drift uses it)
};
void launch_set_step_scalars(StepScalars* dev, const StepScalars& v, cudaStream_t s);
// Precision mode: every scalar of the step from a0 to a1 computed on the device in FP64 (kick and
// drift integrals by Simpson's rule with 256 intervals, the midpoint by 60 bisection steps, the
// Green's prefactor, the tree coupling and the net scale), rounded once to f32 (d64 kept).
// net_per_cell_h = (N / M) / h.
void launch_step_factors64(StepScalars* dev, const cpm_cosmology& c, double a0, double a1, double box,
                           double n_particles, double net_per_cell_h, cudaStream_t s);
// p += g * k (integrator.rs:301-307); k is read from *k_dev when k_dev is set.
void launch_kick(float* p3, const float* g3, size_t n, float k, cudaStream_t s, const float* k_dev = nullptr);
// Optional kick with k_prev, then kick with k1, then drift (integrator.rs:301-316); k1 and d are
// read from *sc when sc is set.
void launch_kick_kick_drift(float* x3, float* p3, const float* g3, size_t n, float k_prev, int has_prev, float k1,
                            float d, float box, cudaStream_t s, const StepScalars* sc = nullptr);
// Fixed-point positions x = q L / 2^32 (q uint32 per component). The first half-kick as
// launch_kick_kick_drift, then the drift q += round(p d 2^32 / L) (FP64 product, wrapping modulo
// 2^32, so the periodic wrap is exact for displacements below L/2), and x3 = f32 of the new q.
void launch_kick_drift_fixed(uint32_t* q3, float* x3, float* p3, const float* g3, size_t n, float box,
                             cudaStream_t s, const StepScalars* sc);
// q3 = round(x3 2^32 / L) modulo 2^32, and x3 rewritten as the f32 of q3.
void launch_to_fixed(float* x3, uint32_t* q3, size_t n, float box, cudaStream_t s);
// Gather permutation: out[i] = in[perm[i]] for AoS triples and for u32 ids.
void launch_permute3(const float* in3, const uint32_t* perm, size_t n, float* out3, cudaStream_t s);
void launch_permute_u32(const uint32_t* in, const uint32_t* perm, size_t n, uint32_t* out, cudaStream_t s);
// Scatter back to caller order: out[id[i]] = in[i].
void launch_scatter3(const float* in3, const uint32_t* id, size_t n, float* out3, cudaStream_t s);
// Flags a non-finite coordinate in the status word.
void launch_check_finite(const float* x3, size_t n, DevStatus* st, cudaStream_t s);
// id[i] = i
void launch_iota(uint32_t* id, size_t n, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Viewer snapshot — snapshot.cu (runner.rs:263-284, frame.rs)
// ---------------------------------------------------------------------------------------------
constexpr int DENSITY_GRID_MAX = 128;  // frame.rs:27 MAX_GRID
// Side m = n / ceil(n / 128) of the downsampled density grid of an n^3 mesh.
int density_grid_side(int n);
// Key-order p3 and interpolated delta in, caller-order outputs through id (any may be null);
// max_speed_bits (zeroed by the caller) receives the bits of the largest speed.
void launch_snapshot_particles(const float* p3, const float* dens_in, const uint32_t* id, size_t n, float a,
                               float rsd_scale, float* speeds, float* dens, float* rsd3, unsigned int* max_speed_bits,
                               cudaStream_t s);
// frame.rs:30-55: 1 + block means of delta, x fastest, density_grid_side(n)^3 values.
void launch_downsample_grid(const float* delta, int n, float* out, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Initial conditions — ics.cu
// ---------------------------------------------------------------------------------------------
// Zel'dovich positions and momenta (AoS f32, lattice order (ix*n + iy)*n + iz) into device memory.
cudaError_t generate_zeldovich(int n, float box, const cpm_cosmology& c, float n_s, float sigma8, float a_init,
                               uint64_t seed, float* x3_dev, float* p3_dev, DevBuf& modes, DevBuf& work,
                               FftPlan& plan, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// Learned short-range force — net.cu, learned_step.cu
// ---------------------------------------------------------------------------------------------
// The net's field F = out_scale * net(in_scale * delta) (float4 per cell, in the net's own buffer,
// returned) from the u64 fixed-point mass mesh; the scale is read from *out_scale_dev when set.
float4* net_field_from_mesh(cpm_net* net, const unsigned long long* fx, int fx_shift, float mean, float in_scale,
                            float out_scale, const float* out_scale_dev, cudaStream_t s);
int net_mesh(const cpm_net* net);
int* net_status_word(cpm_net* net);
// acc = g_pm + F (delta_i < threshold) or g_pm with flag_i = 1 (delta_i >= threshold), one stencil.
void launch_learned_gather(const float* gx, const float* gy, const float* gz, const unsigned long long* fx, int shift,
                           float mean, const float4* field, const float* x3, size_t n, int mesh_n, float h,
                           float threshold, float* out3, uint32_t* flag, cudaStream_t s);
// list = indices i with flag_i = 1 in increasing order, *count = their number (offset: scratch).
cudaError_t launch_compact(const uint32_t* flag, uint32_t* offset, size_t n, uint32_t* list, uint32_t* count,
                           DevBuf& scan_tmp, cudaStream_t s);

}  // namespace cpm
