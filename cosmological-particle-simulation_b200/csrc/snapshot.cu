// snapshot.cu — the per-step frame of the reference's viewer thread (runner.rs:263-284
// `snapshot`, frame.rs:1-70) computed on the device, so that a caller needs no copy of the
// particles to build it: peculiar speeds |p|/a, densities max(1 + delta(x), 0) from the mesh of the
// last force evaluation, redshift-space shifts p / (a^2 E), the downsampled 1 + delta texture grid
// and the largest speed (runner.rs:244-247). Every value uses the reference's f32 operations in its
// order, so the results are bit-identical to it for equal inputs.
#include <algorithm>

#include "cpm_internal.cuh"

namespace cpm {

// Per particle (key order in, caller order out through id): speed, density, rsd shift; and the
// largest speed as the bits of a non-negative float (ordered like the float).
__global__ void k_snapshot_particles(const float* __restrict__ p3, const float* __restrict__ dens_in,
                                     const uint32_t* __restrict__ id, size_t n, float a, float rsd_scale,
                                     float* __restrict__ speeds, float* __restrict__ dens, float* __restrict__ rsd3,
                                     unsigned int* __restrict__ max_speed_bits) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float v = 0.0f;
  if (i < n) {
    const float p0 = p3[3 * i], p1 = p3[3 * i + 1], p2 = p3[3 * i + 2];
    // frame.rs / runner.rs: (p0 p0 + p1 p1 + p2 p2).sqrt() / a
    v = __fdiv_rn(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(p0, p0), __fmul_rn(p1, p1)), __fmul_rn(p2, p2))), a);
    const size_t j = id[i];
    if (speeds) speeds[j] = v;
    if (dens) dens[j] = fmaxf(__fadd_rn(1.0f, dens_in[i]), 0.0f);  // (1 + delta.interpolate(x)).max(0)
    if (rsd3) {  // frame.rs:65-69: p * (1 / (a^2 E))
      rsd3[3 * j] = __fmul_rn(p0, rsd_scale);
      rsd3[3 * j + 1] = __fmul_rn(p1, rsd_scale);
      rsd3[3 * j + 2] = __fmul_rn(p2, rsd_scale);
    }
  }
  if (max_speed_bits) {
    unsigned int b = (i < n && v >= 0.0f) ? __float_as_uint(v) : 0u;  // NaN speeds do not count
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0 && b) atomicMax(max_speed_bits, b);
  }
}

// frame.rs:30-55 `downsample_grid`: texel (x, y, z) of the m^3 grid, x fastest, is 1 + the mean of
// the f^3 block of delta cells starting at (x f, y f, z f), summed in the reference's loop order.
__global__ void k_downsample_grid(const float* __restrict__ delta, int n, int f, int m, float norm,
                                  float* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t mm = (size_t)m * m * m;
  if (t >= mm) return;
  const int x = (int)(t % m), y = (int)((t / m) % m), z = (int)(t / ((size_t)m * m));
  float sum = 0.0f;
  for (int dx = 0; dx < f; ++dx)
    for (int dy = 0; dy < f; ++dy)
      for (int dz = 0; dz < f; ++dz) {
        const size_t ix = (size_t)(x * f + dx), iy = (size_t)(y * f + dy), iz = (size_t)(z * f + dz);
        sum = __fadd_rn(sum, delta[(ix * n + iy) * n + iz]);
      }
  out[t] = __fadd_rn(1.0f, __fmul_rn(sum, norm));
}

int density_grid_side(int n) { return n / std::max(1, (n + DENSITY_GRID_MAX - 1) / DENSITY_GRID_MAX); }

void launch_snapshot_particles(const float* p3, const float* dens_in, const uint32_t* id, size_t n, float a,
                               float rsd_scale, float* speeds, float* dens, float* rsd3, unsigned int* max_speed_bits,
                               cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_snapshot_particles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p3, dens_in, id, n, a, rsd_scale, speeds, dens,
                                                                   rsd3, max_speed_bits);
}

void launch_downsample_grid(const float* delta, int n, float* out, cudaStream_t s) {
  const int f = std::max(1, (n + DENSITY_GRID_MAX - 1) / DENSITY_GRID_MAX);  // n.div_ceil(MAX_GRID).max(1)
  const int m = n / f;
  const float norm = 1.0f / (float)(f * f * f);
  const size_t mm = (size_t)m * m * m;
  if (mm == 0) return;
  count_launch();
  k_downsample_grid<<<(unsigned)((mm + 255) / 256), 256, 0, s>>>(delta, n, f, m, norm, out);
}

}  // namespace cpm
