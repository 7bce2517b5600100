// kdk.cu — kick and drift (integrator.rs:301-316), permutations of the particle arrays.
//
// The reference's `p += g * k` and `x = (x + p * d).rem_euclid(L)` are written with separately
// rounded f32 operations (no FMA), so the update is bit-identical to the reference.
#include "cpm_internal.cuh"

namespace cpm {

__global__ void k_kick(float* __restrict__ p3, const float* __restrict__ g3, size_t n3, float k,
                       const float* __restrict__ k_dev) {
  if (k_dev) k = *k_dev;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
    p3[i] = __fadd_rn(p3[i], __fmul_rn(g3[i], k));
}

// Second half-kick of the previous step (when has_prev), first half-kick of this step, drift.
__global__ void k_kick_kick_drift(float* __restrict__ x3, float* __restrict__ p3, const float* __restrict__ g3,
                                  size_t n3, float k_prev, int has_prev, float k1, float d, float box,
                                  const StepScalars* __restrict__ sc) {
  if (sc) {
    k1 = sc->k1;
    d = sc->d;
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const float g = g3[i];
    float p = p3[i];
    if (has_prev) p = __fadd_rn(p, __fmul_rn(g, k_prev));
    p = __fadd_rn(p, __fmul_rn(g, k1));
    p3[i] = p;
    x3[i] = rem_euclid_f32(__fadd_rn(x3[i], __fmul_rn(p, d)), box);
  }
}

__device__ __forceinline__ float fixed_to_x(uint32_t q, double unit) { return (float)((double)q * unit); }

__global__ void k_kick_drift_fixed(uint32_t* __restrict__ q3, float* __restrict__ x3, float* __restrict__ p3,
                                   const float* __restrict__ g3, size_t n3, float box,
                                   const StepScalars* __restrict__ sc) {
  const float k1 = sc->k1;
  const double d = sc->d64;
  const double per_length = 4294967296.0 / (double)box, unit = (double)box / 4294967296.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const float p = __fadd_rn(p3[i], __fmul_rn(g3[i], k1));
    p3[i] = p;
    const long long dq = __double2ll_rn((double)p * d * per_length);
    const uint32_t q = q3[i] + (uint32_t)(unsigned long long)dq;  // modulo 2^32: the periodic wrap
    q3[i] = q;
    x3[i] = fixed_to_x(q, unit);
  }
}

__global__ void k_to_fixed(float* __restrict__ x3, uint32_t* __restrict__ q3, size_t n3, float box) {
  const double per_length = 4294967296.0 / (double)box, unit = (double)box / 4294967296.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const long long qq = __double2ll_rn((double)x3[i] * per_length);
    const uint32_t q = (uint32_t)(unsigned long long)qq;
    q3[i] = q;
    x3[i] = fixed_to_x(q, unit);
  }
}

__global__ void k_permute3(const float* __restrict__ in3, const uint32_t* __restrict__ perm, size_t n,
                           float* __restrict__ out3) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = perm[i];
  out3[3 * i] = in3[3 * j];
  out3[3 * i + 1] = in3[3 * j + 1];
  out3[3 * i + 2] = in3[3 * j + 2];
}

__global__ void k_permute_u32(const uint32_t* __restrict__ in, const uint32_t* __restrict__ perm, size_t n,
                              uint32_t* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[perm[i]];
}

__global__ void k_scatter3(const float* __restrict__ in3, const uint32_t* __restrict__ id, size_t n,
                           float* __restrict__ out3) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = id[i];
  out3[3 * j] = in3[3 * i];
  out3[3 * j + 1] = in3[3 * i + 1];
  out3[3 * j + 2] = in3[3 * i + 2];
}

__global__ void k_check_finite(const float* __restrict__ x3, size_t n3, DevStatus* st) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(x3[i])) dev_fail(st, DEV_NONFINITE, (int)(i / 3));
}

__global__ void k_iota(uint32_t* __restrict__ id, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    id[i] = (uint32_t)i;
}

static unsigned grid_for(size_t work) {
  size_t b = (work + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b ? b : 1);
}

__global__ void k_set_step_scalars(StepScalars* dev, StepScalars v) { *dev = v; }

// cosmology.rs:32-34 in FP64.
__device__ __forceinline__ double cosmo_e64(const cpm_cosmology& c, double a) {
  const double a2 = a * a;
  return sqrt((double)c.omega_r / (a2 * a2) + (double)c.omega_m / (a2 * a) + (double)c.omega_l);
}

// Simpson's rule (integrator.rs:288-297) with 256 intervals in FP64, summed by one warp:
// kind 0: 1 / (a E(a)) (kick, integrator.rs:263-265); kind 1: 1 / (a^3 E(a)) (drift, :268-270).
__device__ double simpson_warp64(const cpm_cosmology& c, double lo, double hi, int kind) {
  constexpr int N = 256;
  const int lane = threadIdx.x & 31;
  const double h = (hi - lo) / N;
  double sum = 0.0;
  for (int i = lane; i <= N; i += 32) {
    const double a = lo + i * h;
    const double f = kind == 0 ? 1.0 / (a * cosmo_e64(c, a)) : 1.0 / (a * a * a * cosmo_e64(c, a));
    const double w = (i == 0 || i == N) ? 1.0 : ((i & 1) ? 4.0 : 2.0);
    sum += w * f;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  return sum * h / 3.0;
}

__global__ void k_step_factors64(StepScalars* dev, cpm_cosmology c, double a0, double a1, double box, double n_part,
                                 double net_per_cell_h) {
  // integrator.rs:273-285: the scale factor where the kick integral is half its total
  const double half = 0.5 * simpson_warp64(c, a0, a1, 0);
  double lo = a0, hi = a1;
  for (int it = 0; it < 60; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (simpson_warp64(c, a0, mid, 0) < half)
      lo = mid;
    else
      hi = mid;
  }
  const double am = 0.5 * (lo + hi);
  const double k1 = simpson_warp64(c, a0, am, 0), k2 = simpson_warp64(c, am, a1, 0);
  const double d = simpson_warp64(c, a0, a1, 1);
  if ((threadIdx.x & 31) == 0) {
    const double pi = 3.14159265358979323846;
    const double tree_k = 1.5 * (double)c.omega_m * box * box * box / (4.0 * pi * a1 * n_part);  // integrator.rs:152
    StepScalars v;
    v.k1 = (float)k1;
    v.d = (float)d;
    v.k2 = (float)k2;
    v.prefactor = (float)(1.5 * (double)c.omega_m / a1);  // poisson.rs:46
    v.tree_k = (float)tree_k;
    v.net_scale = (float)(tree_k * net_per_cell_h);
    v.pad_ = 0.0f;
    v.d64 = d;
    *dev = v;
  }
}

void launch_step_factors64(StepScalars* dev, const cpm_cosmology& c, double a0, double a1, double box,
                           double n_particles, double net_per_cell_h, cudaStream_t s) {
  count_launch();
  k_step_factors64<<<1, 32, 0, s>>>(dev, c, a0, a1, box, n_particles, net_per_cell_h);
}

void launch_set_step_scalars(StepScalars* dev, const StepScalars& v, cudaStream_t s) {
  count_launch();
  k_set_step_scalars<<<1, 1, 0, s>>>(dev, v);
}

void launch_kick(float* p3, const float* g3, size_t n, float k, cudaStream_t s, const float* k_dev) {
  if (n == 0) return;
  count_launch();
  k_kick<<<grid_for(3 * n), 256, 0, s>>>(p3, g3, 3 * n, k, k_dev);
}

void launch_kick_kick_drift(float* x3, float* p3, const float* g3, size_t n, float k_prev, int has_prev, float k1,
                            float d, float box, cudaStream_t s, const StepScalars* sc) {
  if (n == 0) return;
  count_launch();
  k_kick_kick_drift<<<grid_for(3 * n), 256, 0, s>>>(x3, p3, g3, 3 * n, k_prev, has_prev, k1, d, box, sc);
}

void launch_kick_drift_fixed(uint32_t* q3, float* x3, float* p3, const float* g3, size_t n, float box,
                             cudaStream_t s, const StepScalars* sc) {
  if (n == 0) return;
  count_launch();
  k_kick_drift_fixed<<<grid_for(3 * n), 256, 0, s>>>(q3, x3, p3, g3, 3 * n, box, sc);
}

void launch_to_fixed(float* x3, uint32_t* q3, size_t n, float box, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_to_fixed<<<grid_for(3 * n), 256, 0, s>>>(x3, q3, 3 * n, box);
}

void launch_permute3(const float* in3, const uint32_t* perm, size_t n, float* out3, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_permute3<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in3, perm, n, out3);
}

void launch_permute_u32(const uint32_t* in, const uint32_t* perm, size_t n, uint32_t* out, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_permute_u32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, perm, n, out);
}

void launch_scatter3(const float* in3, const uint32_t* id, size_t n, float* out3, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_scatter3<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in3, id, n, out3);
}

void launch_iota(uint32_t* id, size_t n, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_iota<<<grid_for(n), 256, 0, s>>>(id, n);
}

void launch_check_finite(const float* x3, size_t n, DevStatus* st, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_check_finite<<<grid_for(3 * n), 256, 0, s>>>(x3, 3 * n, st);
}

}  // namespace cpm
