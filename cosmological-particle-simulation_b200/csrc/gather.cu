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

// The PM force gather for sorted particles. A CTA takes a chunk of GAT_CHUNK consecutive particles
// (spatially compact in key order), loads the box of cells their stencils cover from the three force
// meshes into shared memory with row-contiguous loads, and gathers from there: the scattered
// 4-byte loads of the stencils (24 per particle) no longer go through L1, which they saturated. A
// chunk whose box exceeds the shared-memory tile (unsorted input, or a chunk across two boxes of a
// batch) gathers from global memory. Either way each particle's sums are the same f32 operations
// on the same values.
// n_box > 0: a batch of boxes (box i / n_box reads its own meshes, mesh_n^3 cells each, in order).
constexpr int GAT_THREADS = 256;
constexpr int GAT_PPT = 2;
constexpr int GAT_CHUNK = GAT_THREADS * GAT_PPT;
constexpr int GAT_CELLS = 6144;  // 3 x 24 KB of f32 per CTA

__global__ void __launch_bounds__(GAT_THREADS) k_interpolate3(const float* __restrict__ gx, const float* __restrict__ gy,
                                                              const float* __restrict__ gz, const float* __restrict__ x3,
                                                              size_t n, int mesh_n, float h, float* __restrict__ out3,
                                                              size_t n_box) {
  extern __shared__ float sg[];  // [3][GAT_CELLS]
  __shared__ int bb[6];
  if (threadIdx.x < 3) bb[threadIdx.x] = 0x7fffffff;
  else if (threadIdx.x < 6) bb[threadIdx.x] = -0x7fffffff;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * GAT_CHUNK;
  const size_t cells_per_box = (size_t)mesh_n * mesh_n * mesh_n;
  bool one_box = true;
  size_t box_off = 0;
  if (n_box) {
    const size_t last = min(base + GAT_CHUNK, n) - 1;
    one_box = base / n_box == last / n_box;
    box_off = (base / n_box) * cells_per_box;
  }
  CicBase cb[GAT_PPT];
  bool valid[GAT_PPT];
  int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
#pragma unroll
  for (int q = 0; q < GAT_PPT; ++q) {
    const size_t i = base + (size_t)q * GAT_THREADS + threadIdx.x;
    valid[q] = i < n;
    if (valid[q]) {
      const float x[3] = {x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]};
      cic_base(x, h, mesh_n, cb[q]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = min(lo[k], cb[q].b[k]);
        hi[k] = max(hi[k], cb[q].b[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(&bb[k], lo[k]);
      atomicMax(&bb[3 + k], hi[k]);
    }
  }
  __syncthreads();
  if (bb[0] > bb[3]) return;  // empty chunk
  const int e0 = bb[3] - bb[0] + 2, e1 = bb[4] - bb[1] + 2, e2 = bb[5] - bb[2] + 2;
  const long long cells = (long long)e0 * e1 * e2;
  const bool tiled = one_box && cells <= GAT_CELLS;
  if (tiled) {
    const float* mx = gx + box_off;
    const float* my = gy + box_off;
    const float* mz = gz + box_off;
    // t -> (lx, ly, lz), z fastest: floor(t / e) as floor((t + 1/2) * fl(1/e)), exact for t < 2^15
    const float inv_e2 = 1.0f / (float)e2, inv_e1 = 1.0f / (float)e1;
    for (int t = threadIdx.x; t < (int)cells; t += GAT_THREADS) {
      const int row = (int)(((float)t + 0.5f) * inv_e2);
      const int lx = (int)(((float)row + 0.5f) * inv_e1);
      const int lz = t - row * e2, ly = row - lx * e1;
      const size_t idx = ((size_t)wrap_index(bb[0] + lx, mesh_n) * mesh_n + (size_t)wrap_index(bb[1] + ly, mesh_n)) *
                             mesh_n +
                         (size_t)wrap_index(bb[2] + lz, mesh_n);
      sg[t] = __ldg(mx + idx);
      sg[GAT_CELLS + t] = __ldg(my + idx);
      sg[2 * GAT_CELLS + t] = __ldg(mz + idx);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < GAT_PPT; ++q) {
    if (!valid[q]) continue;
    const size_t i = base + (size_t)q * GAT_THREADS + threadIdx.x;
    float sx = -0.0f, sy = -0.0f, sz = -0.0f;
    if (tiled) {
      const int lx = cb[q].b[0] - bb[0], ly = cb[q].b[1] - bb[1], lz = cb[q].b[2] - bb[2];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int dx = (k >> 2) & 1, dy = (k >> 1) & 1, dz = k & 1;
        const int li = ((lx + dx) * e1 + (ly + dy)) * e2 + (lz + dz);
        const float w = cic_weight(cb[q], k);
        sx = __fadd_rn(sx, __fmul_rn(sg[li], w));
        sy = __fadd_rn(sy, __fmul_rn(sg[GAT_CELLS + li], w));
        sz = __fadd_rn(sz, __fmul_rn(sg[2 * GAT_CELLS + li], w));
      }
    } else {
      const size_t off = n_box ? (i / n_box) * cells_per_box : 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const size_t idx = off + cic_index(cb[q], k, mesh_n);
        const float w = cic_weight(cb[q], k);
        sx = __fadd_rn(sx, __fmul_rn(__ldg(gx + idx), w));
        sy = __fadd_rn(sy, __fmul_rn(__ldg(gy + idx), w));
        sz = __fadd_rn(sz, __fmul_rn(__ldg(gz + idx), w));
      }
    }
    out3[3 * i] = sx;
    out3[3 * i + 1] = sy;
    out3[3 * i + 2] = sz;
  }
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
  constexpr int smem = 3 * GAT_CELLS * (int)sizeof(float);
  cudaFuncSetAttribute(k_interpolate3, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  count_launch();
  k_interpolate3<<<(unsigned)((n + GAT_CHUNK - 1) / GAT_CHUNK), GAT_THREADS, smem, s>>>(gx, gy, gz, x3, n, mesh_n, h,
                                                                                       out3, n_box);
}

}  // namespace cpm
