// deposit.cu — CIC mass deposit (mesh.rs:62-69) into a 64-bit fixed-point mesh.
//
// Particles arrive sorted by octant key, so a chunk of consecutive particles covers a compact
// box of cells. Each CTA accumulates its chunk into that box in shared memory with 64-bit
// integer atomics, then adds the box to the global mesh: one bulk reduction (TMA unit,
// cp.reduce.async.bulk .add.u64) per row of the box along z, split at the periodic boundary, so
// whole rows leave shared memory in 16-byte multiples instead of one L2 atomic per cell (the box
// starts at an even z and has an even length for that alignment). Integer addition is
// associative, so the mesh does not depend on particle order or scheduling (bit-reproducible),
// and it holds the exactly rounded sum of the reference's f32 weights `mass * w`. Chunks whose box
// does not fit in shared memory fall back to direct global atomics (same integers, same result),
// and odd meshes flush the box cell by cell with atomics.
#include <algorithm>
#include <cmath>

#include "cpm_internal.cuh"

namespace cpm {

constexpr int DEP_THREADS = 256;
// Particles per thread PPT (tile of 256 * PPT consecutive sorted particles per CTA): 2, 4 or 8,
// picked per workload by the autotuner (4 by default). The shared-memory box grows with the tile:
// 48 KB (four CTAs per SM), 96 KB (two) or 192 KB (one) of u64 cells.
template <int PPT>
__host__ __device__ constexpr int dep_smem_cells() {
  return PPT <= 2 ? 6144 : (PPT <= 4 ? 12288 : 24576);
}

int fixed_point_shift(double total_mass) {
  // Largest k with total_mass * 2^k < 2^62, clamped so a unit weight keeps >= 24 fractional bits.
  const double m = total_mass > 1e-30 ? total_mass : 1e-30;
  int k = 62 - (int)std::ceil(std::log2(m));
  if (k > 60) k = 60;
  if (k < 24) k = 24;
  return k;
}

// dst[i] += src[i] for size / 8 u64 elements, element-wise atomic in L2 (bulk-async group of the
// calling thread); both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_reduce_add_u64(unsigned long long* dst, const unsigned long long* src,
                                                    uint32_t bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(src);
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u64 [%0], [%1], %2;" ::"l"(dst), "r"(s),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ unsigned long long to_fixed(float mass, float w, float scale) {
  // mass * w is the reference's f32 product; scaling by 2^k is exact.
  return __float2ull_rn(__fmul_rn(__fmul_rn(mass, w), scale));
}

// With n_box > 0 the particles form a batch of boxes (box i / n_box, each with its own mesh of
// mesh_n^3 cells, one after another); a tile that spans two boxes takes the global-atomic path.
template <int DEP_PPT>
__global__ void __launch_bounds__(DEP_THREADS) k_deposit_fixed(const float* __restrict__ x3, size_t n, float mass,
                                                               int mesh_n, float h, float scale,
                                                               unsigned long long* __restrict__ mesh, size_t n_box) {
  extern __shared__ __align__(16) unsigned long long sm_cells[];
  __shared__ int bb[6];  // min x,y,z then max x,y,z of the stencil base
  if (threadIdx.x < 3) bb[threadIdx.x] = 0x7fffffff;
  else if (threadIdx.x < 6) bb[threadIdx.x] = -0x7fffffff;
  __syncthreads();

  constexpr int DEP_CHUNK = DEP_THREADS * DEP_PPT;
  const size_t base = (size_t)blockIdx.x * DEP_CHUNK;
  const size_t cells_per_box = (size_t)mesh_n * mesh_n * mesh_n;
  bool one_box = true;
  if (n_box) {
    const size_t last = min(base + DEP_CHUNK, n) - 1;
    one_box = base / n_box == last / n_box;
    mesh += (base / n_box) * cells_per_box;  // the tile's box (the global path re-bases per particle)
  }
  CicBase cb[DEP_PPT];
  bool valid[DEP_PPT];
  int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
#pragma unroll
  for (int q = 0; q < DEP_PPT; ++q) {
    const size_t i = base + (size_t)q * DEP_THREADS + threadIdx.x;
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
  // box: x, y from the lowest base; z from the even cell at or below it, an even number of cells
  const int z0 = bb[2] & ~1;
  const int e0 = bb[3] - bb[0] + 2, e1 = bb[4] - bb[1] + 2, e2 = (bb[5] + 2 - z0 + 1) & ~1;
  const long long cells = (long long)e0 * e1 * e2;

  if (one_box && cells <= dep_smem_cells<DEP_PPT>() && e0 > 0 && e1 > 0 && e2 > 0) {
    for (int t = threadIdx.x; t < (int)cells; t += DEP_THREADS) sm_cells[t] = 0ull;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < DEP_PPT; ++q) {
      if (!valid[q]) continue;
      const int lx = cb[q].b[0] - bb[0], ly = cb[q].b[1] - bb[1], lz = cb[q].b[2] - z0;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
        const int li = ((lx + dx) * e1 + (ly + dy)) * e2 + (lz + dz);
        atomicAdd(&sm_cells[li], to_fixed(mass, cic_weight(cb[q], c), scale));
      }
    }
    __syncthreads();
    if ((mesh_n & 1) == 0 && e2 <= mesh_n) {
      // the atomics' results become visible to the bulk-copy (async) proxy, then each thread
      // reduces whole box rows into the mesh
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      const int zw = wrap_index(z0, mesh_n);
      const int len1 = min(e2, mesh_n - zw), len2 = e2 - len1;
      for (int r = threadIdx.x; r < e0 * e1; r += DEP_THREADS) {
        const int lx = r / e1, ly = r - lx * e1;
        const size_t gx = (size_t)wrap_index(bb[0] + lx, mesh_n);
        const size_t gy = (size_t)wrap_index(bb[1] + ly, mesh_n);
        unsigned long long* grow = mesh + (gx * mesh_n + gy) * mesh_n;
        const unsigned long long* srow = sm_cells + (size_t)r * e2;
        bulk_reduce_add_u64(grow + zw, srow, (uint32_t)len1 * 8u);
        if (len2 > 0) bulk_reduce_add_u64(grow, srow + len1, (uint32_t)len2 * 8u);
      }
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      return;
    }
    // floor(t / e) as floor((t + 1/2) * fl(1/e)): (t + 1/2) / e lies at least 1/(2e) from an
    // integer, and for t < 2^15 the two f32 roundings move it by less than 2^-7 / e.
    const float inv_e2 = 1.0f / (float)e2, inv_e1 = 1.0f / (float)e1;
    for (int t = threadIdx.x; t < (int)cells; t += DEP_THREADS) {
      const unsigned long long v = sm_cells[t];
      if (v == 0ull) continue;
      const int row = (int)(((float)t + 0.5f) * inv_e2);
      const int lx = (int)(((float)row + 0.5f) * inv_e1);
      const int lz = t - row * e2, ly = row - lx * e1;
      const size_t gx = (size_t)wrap_index(bb[0] + lx, mesh_n);
      const size_t gy = (size_t)wrap_index(bb[1] + ly, mesh_n);
      const size_t gz = (size_t)wrap_index(z0 + lz, mesh_n);
      atomicAdd(&mesh[(gx * mesh_n + gy) * mesh_n + gz], v);
    }
  } else {
#pragma unroll
    for (int q = 0; q < DEP_PPT; ++q) {
      if (!valid[q]) continue;
      unsigned long long* m = mesh;
      if (n_box && !one_box) {
        const size_t i = base + (size_t)q * DEP_THREADS + threadIdx.x;
        m = mesh + ((i / n_box) - (base / n_box)) * cells_per_box;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c)
        atomicAdd(&m[cic_index(cb[q], c, mesh_n)], to_fixed(mass, cic_weight(cb[q], c), scale));
    }
  }
}

template <int PPT>
static void deposit_ppt(const float* x3, size_t n, float mass, int mesh_n, float h, float scale,
                        unsigned long long* mesh_fx, cudaStream_t s, size_t n_box) {
  // Per device (a cheap host call, so made on every launch): a failure shows up as the launch's error.
  constexpr int smem = dep_smem_cells<PPT>() * (int)sizeof(unsigned long long);
  cudaFuncSetAttribute(k_deposit_fixed<PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  constexpr size_t chunk = (size_t)DEP_THREADS * PPT;
  const unsigned blocks = (unsigned)((n + chunk - 1) / chunk);
  count_launch();
  k_deposit_fixed<PPT><<<blocks, DEP_THREADS, smem, s>>>(x3, n, mass, mesh_n, h, scale, mesh_fx, n_box);
}

void launch_deposit_fixed(const float* x3, size_t n, float mass, int mesh_n, float h, int shift,
                          unsigned long long* mesh_fx, cudaStream_t s, int ppt, size_t n_box) {
  const size_t boxes = n_box ? (n + n_box - 1) / n_box : 1;
  const size_t m = (size_t)mesh_n * mesh_n * mesh_n * boxes;
  cudaMemsetAsync(mesh_fx, 0, m * sizeof(unsigned long long), s);
  if (n == 0) return;
  const float scale = std::ldexp(1.0f, shift);
  if (ppt == 2)
    deposit_ppt<2>(x3, n, mass, mesh_n, h, scale, mesh_fx, s, n_box);
  else if (ppt == 8)
    deposit_ppt<8>(x3, n, mass, mesh_n, h, scale, mesh_fx, s, n_box);
  else
    deposit_ppt<4>(x3, n, mass, mesh_n, h, scale, mesh_fx, s, n_box);
}

// integrator.rs:117-126: cell mass c = fixed * 2^-k rounded once to f32; delta = c / mean - 1.
__global__ void k_fixed_to_f32(const unsigned long long* __restrict__ fx, size_t m, float inv_scale, int to_delta,
                               float mean, float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const float c = __fmul_rn(__ull2float_rn(fx[i]), inv_scale);
    out[i] = to_delta ? __fsub_rn(__fdiv_rn(c, mean), 1.0f) : c;
  }
}

void launch_fixed_to_f32(const unsigned long long* fx, size_t m, int shift, int to_delta, float mean, float* out,
                         cudaStream_t s) {
  if (m == 0) return;
  const float inv_scale = std::ldexp(1.0f, -shift);
  const size_t blocks = std::min<size_t>((m + 255) / 256, 148 * 32);
  count_launch();
  k_fixed_to_f32<<<(unsigned)blocks, 256, 0, s>>>(fx, m, inv_scale, to_delta, mean, out);
}

}  // namespace cpm
