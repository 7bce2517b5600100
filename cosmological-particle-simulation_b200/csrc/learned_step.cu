// learned_step.cu — the force assembly of a simulation step with the learned short-range force.
//
// The reference adds the tree's short-range force to the PM force of every particle
// (integrator.rs:144-159). With a net attached to the simulation, the step instead
//   1. gathers, per particle, with one CIC stencil (mesh.rs:29-77): the three PM force components
//      (bit-identical to the plain gather), the density contrast delta_i from the fixed-point mass
//      mesh (delta = c / mean - 1 per cell as in integrator.rs:117-126, with the division by the mean
//      taken as a product with its reciprocal: delta_i only selects the force model) and the net's
//      field F;
//      acc = g_pm + F where delta_i < threshold, acc = g_pm and flag_i = 1 elsewhere;
//   2. compacts the flagged (dense) particles into a list that keeps the sorted order (a Hilbert
//      order in a simulation);
//   3. walks the tree (tree.rs:264-310 rules, unchanged) for the listed particles only, adding
//      their short-range force to acc.
#include "cpm_internal.cuh"

namespace cpm {

__global__ void k_learned_gather(const float* __restrict__ gx, const float* __restrict__ gy,
                                 const float* __restrict__ gz, const unsigned long long* __restrict__ fx, float inv_fx,
                                 float mean, const float4* __restrict__ field, const float* __restrict__ x3, size_t n,
                                 int mesh_n, float h, float threshold, float* __restrict__ out3,
                                 uint32_t* __restrict__ flag) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x[3] = {x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]};
  CicBase c;
  cic_base(x, h, mesh_n, c);
  const float inv_mean = 1.0f / mean;
  float sx = -0.0f, sy = -0.0f, sz = -0.0f, d = 0.0f;
  float fx0 = 0.0f, fy0 = 0.0f, fz0 = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const size_t idx = cic_index(c, k, mesh_n);
    const float w = cic_weight(c, k);
    sx = __fadd_rn(sx, __fmul_rn(__ldg(gx + idx), w));
    sy = __fadd_rn(sy, __fmul_rn(__ldg(gy + idx), w));
    sz = __fadd_rn(sz, __fmul_rn(__ldg(gz + idx), w));
    // the cell's density contrast for the threshold test only (not a force term): c * (1 / mean) - 1
    const float cell = __fmul_rn(__ull2float_rn(__ldg(fx + idx)), inv_fx) * inv_mean - 1.0f;
    d += w * cell;
    const float4 f = __ldg(field + idx);
    fx0 += w * f.x;
    fy0 += w * f.y;
    fz0 += w * f.z;
  }
  const bool dense = !(d < threshold);
  if (!dense) {
    sx += fx0;
    sy += fy0;
    sz += fz0;
  }
  out3[3 * i] = sx;
  out3[3 * i + 1] = sy;
  out3[3 * i + 2] = sz;
  flag[i] = dense ? 1u : 0u;
}

__global__ void k_compact(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ offset, size_t n,
                          uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flag[i]) list[offset[i]] = (uint32_t)i;
  if (i == n - 1) *count = offset[i] + flag[i];
}

void launch_learned_gather(const float* gx, const float* gy, const float* gz, const unsigned long long* fx, int shift,
                           float mean, const float4* field, const float* x3, size_t n, int mesh_n, float h,
                           float threshold, float* out3, uint32_t* flag, cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_learned_gather<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gx, gy, gz, fx, ldexpf(1.0f, -shift), mean, field, x3,
                                                               n, mesh_n, h, threshold, out3, flag);
}

cudaError_t launch_compact(const uint32_t* flag, uint32_t* offset, size_t n, uint32_t* list, uint32_t* count,
                           DevBuf& scan_tmp, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = exclusive_scan_u32(flag, offset, n, scan_tmp, s);
  if (e != cudaSuccess) return e;
  count_launch();
  k_compact<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(flag, offset, n, list, count);
  return cudaGetLastError();
}

}  // namespace cpm
