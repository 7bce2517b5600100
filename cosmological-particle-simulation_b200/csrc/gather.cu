// gather.cu — CIC interpolation (mesh.rs:72-77) and the PM force gather (integrator.rs:144-148).
//
// One stencil per particle serves all three force components. The 8 products are summed in
// the reference's corner order with separately rounded f32 operations, so the result is
// bit-identical to the reference's `interpolate` given the same mesh values.
#include "cpm_internal.cuh"

namespace cpm {

__global__ void k_interpolate(const float* __restrict__ cells, const float* __restrict__ x3, size_t n, int mesh_n,
                              float h, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x[3] = {x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]};
  CicBase c;
  cic_base(x, h, mesh_n, c);
  float sum = -0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) sum = __fadd_rn(sum, __fmul_rn(__ldg(cells + cic_index(c, k, mesh_n)), cic_weight(c, k)));
  out[i] = sum;
}

// n_box > 0: a batch of boxes (box i / n_box reads its own meshes, mesh_n^3 cells each, in order).
__global__ void k_interpolate3(const float* __restrict__ gx, const float* __restrict__ gy,
                               const float* __restrict__ gz, const float* __restrict__ x3, size_t n, int mesh_n,
                               float h, float* __restrict__ out3, size_t n_box) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (n_box) {
    const size_t off = (i / n_box) * ((size_t)mesh_n * mesh_n * mesh_n);
    gx += off;
    gy += off;
    gz += off;
  }
  const float x[3] = {x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]};
  CicBase c;
  cic_base(x, h, mesh_n, c);
  float sx = -0.0f, sy = -0.0f, sz = -0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const size_t idx = cic_index(c, k, mesh_n);
    const float w = cic_weight(c, k);
    sx = __fadd_rn(sx, __fmul_rn(__ldg(gx + idx), w));
    sy = __fadd_rn(sy, __fmul_rn(__ldg(gy + idx), w));
    sz = __fadd_rn(sz, __fmul_rn(__ldg(gz + idx), w));
  }
  out3[3 * i] = sx;
  out3[3 * i + 1] = sy;
  out3[3 * i + 2] = sz;
}

void launch_interpolate(const float* cells, const float* x3, size_t n, int mesh_n, float h, float* out,
                        cudaStream_t s) {
  if (n == 0) return;
  count_launch();
  k_interpolate<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cells, x3, n, mesh_n, h, out);
}

void launch_interpolate3(const float* gx, const float* gy, const float* gz, const float* x3, size_t n, int mesh_n,
                         float h, float* out3, cudaStream_t s, size_t n_box) {
  if (n == 0) return;
  count_launch();
  k_interpolate3<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gx, gy, gz, x3, n, mesh_n, h, out3, n_box);
}

}  // namespace cpm
