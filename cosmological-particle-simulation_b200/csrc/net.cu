// net.cu — the learned short-range force: a 3-layer convolutional net on the CIC density mesh,
// with hand-written BF16 tcgen05 implicit-GEMM kernels for inference and training.
//
// The reference computes the short-range force with a Barnes-Hut walk (tree.rs:264-310); it has no
// learned component. Here a net maps the density contrast delta on the PM mesh to a 3-channel
// short-range acceleration field, which the simulation gathers to particles with the CIC stencil
// (mesh.rs:72-77) wherever the particle's density contrast is below a threshold; the tree walk
// stays for the particles above it.
//
// Network: three 3x3x3 periodic convolutions without biases, 16 channels, leaky ReLU (slope 1/8)
// after the first two:   y = W3 * lrelu(W2 * lrelu(W1 * (s_in delta))),   F = s_out y.
// Without biases and with a positively homogeneous activation the net is homogeneous of degree one
// (F(lambda delta) = lambda F(delta) for lambda > 0, F(0) = 0), like the linear map from density to
// force it approximates. Convolution here is out[v] = sum_t W[t] in[v + t], t in {-1,0,1}^3,
// tap index t = (dx+1)*9 + (dy+1)*3 + (dz+1).
//
// Layout of every activation tensor (BF16): [x][y][chunk 2][ZP][8], ZP = n + 8. Voxel z of row
// (x, y) sits at padded index z + 1; index 0 holds a copy of z = n - 1 and index n + 1 a copy of
// z = 0 (periodic halo), so one TMA box of a row covers the tile and its z neighbours. Channels
// 0-7 form chunk 0, 8-15 chunk 1, each chunk a contiguous plane of 16-byte voxels. In shared memory
// a row box lands as [chunk][136 voxels][8 channels]: the K-major canonical layout of an MMA A
// operand (core matrix = 8 voxels x 8 channels, SBO = 128 B, LBO = one chunk plane), and a shift
// of the tile by one voxel along z is a shift of the descriptor's start address by 16 bytes. So a
// 3^3 convolution over a row of 128 voxels is 9 row loads and 27 MMAs of 128 x 16 x 16 (implicit
// GEMM: no im2col copy); the forward kernel groups them per input row (below).
//
// Kernels (warp-specialised, persistent over tiles of 128-voxel rows):
//   k_conv3       forward convolution (also the data gradient, with transposed and flipped weights):
//                 warp 0 = TMA producer, warp 1 = MMA issuer (one thread), warps 2-5 = epilogue
//                 (TMEM -> registers, leaky ReLU or the activation-derivative gate, BF16 or FP32 out).
//                 A tile is 16 output rows (consecutive y) of 128 voxels; each input row is loaded
//                 once per tile and feeds the (up to) three output rows it touches through one MMA
//                 of N = 48 whose weight operand stacks the three dy taps: 9 MMAs per input row
//                 instead of 27 per output row, so each 4 KB activation operand read from shared
//                 memory serves three times the arithmetic.
//   k_conv3_wgrad weight gradient dW[t][co][ci] = sum_v dOut[v][co] In[v + t][ci]: 9 gradient rows
//                 (x - dx, y - dy) and one input row per tile, both MN-major operands; M = 128 =
//                 8 rows x 16 output channels, N = 32 = 4 z shifts x 8 input channels, K = voxels;
//                 accumulated in TMEM over all tiles of the CTA, reduced with atomics at the end
// plus elementwise kernels (input conversion, field gather and loss gradient, Adam).
#include <cuda.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cpm_host.h"
#include "cpm_internal.cuh"
#include "umma.cuh"

namespace cpm {

constexpr int NET_C = 16;
constexpr int NET_TAPS = 27;
constexpr int NET_LAYERS = 3;
constexpr int NET_OUT = 3;
constexpr float NET_SLOPE = 0.125f;
constexpr int NET_WEIGHTS = NET_LAYERS * NET_TAPS * NET_C * NET_C;  // master weights [3][27][16][16]

constexpr int TILE_M = 128;                     // voxels per tile
constexpr int ROW_BOX = 136;                    // voxels per input row load (tile, halo, rounding)
constexpr int PLANE_BYTES = ROW_BOX * 16;       // one 8-channel chunk plane of a loaded row
constexpr int ROW_BYTES = 2 * PLANE_BYTES;      // 4352
constexpr int GRAD_PLANE = TILE_M * 16;         // a gradient row (weight-gradient kernel): 128 voxels
constexpr int GRAD_ROW = 2 * GRAD_PLANE;        // 4096
constexpr int W_TAP_BYTES = 2 * NET_C * 16;     // [chunk][cout 16][8 cin] bf16 = 512
constexpr int W_BYTES = NET_TAPS * W_TAP_BYTES;  // 13824
constexpr int CONV_THREADS = 192;               // 6 warps (weight-gradient kernel)
constexpr int FWD_THREADS = 320;                // 10 warps (forward kernel: 8 epilogue warps)
constexpr int CONV_ROWS = 16;                   // output rows (consecutive y) per forward tile
constexpr int CONV_SLOTS = 12;                  // input row triplets in flight (forward kernel)
constexpr int SLOT_BYTES = 3 * ROW_BYTES;       // rows x-1, x, x+1 at one y
constexpr int WS_BYTES = 2 * 3 * NET_C * 16;    // stacked weights of one (dx, dz): [chunk][48][8 cin] bf16
constexpr int WG_STAGES = 2;
constexpr long long WAIT_BUDGET = 1ll << 32;    // clock cycles (about 2 s) before a wait gives up

enum NetError : int { NET_OK = 0, NET_TIMEOUT = 7 };

// ---------------------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float lrelu(float v) { return v > 0.0f ? v : NET_SLOPE * v; }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpack_bf16x2(uint32_t v) {
  __nv_bfloat162 h;
  *reinterpret_cast<uint32_t*>(&h) = v;
  return __bfloat1622float2(h);
}

struct TensorGeo {
  int n;
  int zp;  // n + 8
  // element offset of (x, y, chunk, padded z, 0)
  __host__ __device__ size_t at(int x, int y, int c, int pz) const {
    return ((((size_t)x * n + y) * 2 + c) * (size_t)zp + pz) * 8;
  }
};

// Stores 16 channels of voxel z (0..n-1) of row (x, y) and, for z = 0 and z = n - 1, its halo copy.
__device__ __forceinline__ void store_voxel16(__nv_bfloat16* t, const TensorGeo& g, int x, int y, int z,
                                              const uint4& c0, const uint4& c1) {
  *reinterpret_cast<uint4*>(t + g.at(x, y, 0, z + 1)) = c0;
  *reinterpret_cast<uint4*>(t + g.at(x, y, 1, z + 1)) = c1;
  if (z == 0) {
    *reinterpret_cast<uint4*>(t + g.at(x, y, 0, g.n + 1)) = c0;
    *reinterpret_cast<uint4*>(t + g.at(x, y, 1, g.n + 1)) = c1;
  }
  if (z == g.n - 1) {
    *reinterpret_cast<uint4*>(t + g.at(x, y, 0, 0)) = c0;
    *reinterpret_cast<uint4*>(t + g.at(x, y, 1, 0)) = c1;
  }
}

struct ConvArgs {
  TensorGeo g;
  int tiles_z;
  long long tiles;
  const __nv_bfloat16* w;     // packed weights [27][2][16][8]
  __nv_bfloat16* out16;       // BF16 tensor output, or null
  float4* out_f4;             // FP32 field output [n^3] (x, y, z, 0), or null
  const __nv_bfloat16* gate;  // multiply channel c by lrelu'(gate[v][c]) (backward), or null
  int act;                    // apply lrelu to the output
  float out_scale;
  const float* out_scale_dev;  // when set, the scale is read from device memory
  int* status;
};

// ---------------------------------------------------------------------------------------------
// Forward convolution
// ---------------------------------------------------------------------------------------------
// FOLD: the first layer on the folded input (channel 3 (dy+1) + (dz+1) holds delta at (y+dy, z+dz),
// written by k_net_input_fold): the y and z taps are input channels, so an output row takes the
// three x rows at its own y, one MMA of 128 x 16 x 16 each (K = 9 live channels), instead of 27 taps
// over a single live channel.
template <int NSLOT, bool FOLD>
__global__ void __launch_bounds__(FWD_THREADS, 1) k_conv3(const __grid_constant__ CUtensorMap in_map, ConvArgs a) {
  constexpr int R = CONV_ROWS;            // output rows (consecutive y) per tile
  constexpr int NY = FOLD ? R : R + 2;    // input row triplets per tile: y0-1 .. y0+R (folded: y0 .. y0+R-1)
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* slots = smem;                               // [NSLOT][3 rows x-1, x, x+1][ROW_BYTES]
  uint8_t* wsm = smem + NSLOT * SLOT_BYTES;            // weights stacked over dy, [dx][dz][chunk][48][8]
  uint64_t* bars = reinterpret_cast<uint64_t*>(wsm + W_BYTES);
  uint64_t* full = bars;                  // [NSLOT] triplet loaded
  uint64_t* empty = bars + NSLOT;         // [NSLOT] triplet consumed by the MMAs
  uint64_t* acc_full = bars + 2 * NSLOT;      // [2] accumulators ready
  uint64_t* acc_empty = bars + 2 * NSLOT + 2;  // [2] accumulators read by the epilogue
  uint64_t* done = bars + 2 * NSLOT + 4;
  uint32_t* tmem_sh = reinterpret_cast<uint32_t*>(bars + 2 * NSLOT + 5);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = a.g.n;
  const int yq_count = n / R;
  // Restack the weights [tap][chunk][cout][8 cin] as, per (dx, dz), one N = 48 operand whose rows
  // are (dy = +1, 0, -1) x cout: the output rows fed by one input row, in increasing y.
  if constexpr (FOLD) {
    // per dx: [chunk 2][co 16][8 channels], channel c = 3 dyi + dzi < 9 from input channel 0 of tap
    // (dx, dyi - 1, dzi - 1)
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    __nv_bfloat16* wf = reinterpret_cast<__nv_bfloat16*>(wsm);
    for (int i = threadIdx.x; i < 3 * 2 * NET_C * 8; i += FWD_THREADS) {
      const int k = i % 8, co = (i / 8) % NET_C, ch = (i / (8 * NET_C)) % 2, dxi = i / (16 * NET_C);
      const int c = ch * 8 + k;
      wf[i] = c < 9 ? a.w[(((dxi * 3 + c / 3) * 3 + c % 3) * 2 * NET_C + co) * 8] : zero;
    }
  } else {
    for (int i = threadIdx.x; i < W_BYTES / 16; i += FWD_THREADS) {
      const int co = i % 48, blk = i / 48;  // blk = (dxi * 3 + dz) * 2 + chunk
      const int ch = blk & 1, dxz = blk >> 1, dxi = dxz / 3, dz = dxz % 3;
      const int dyi = 2 - co / 16, c = co % 16;
      const int tap = (dxi * 3 + dyi) * 3 + dz;
      reinterpret_cast<uint4*>(wsm)[i] = __ldg(reinterpret_cast<const uint4*>(a.w) + (tap * 2 + ch) * 16 + c);
    }
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < NSLOT; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      umma::mbar_init(&acc_full[b], 1);
      umma::mbar_init(&acc_empty[b], 256);
    }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tmem_sh, 2 * R * NET_C);
    umma::tmem_relinquish();
  }
  umma::fence_proxy_async();
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tmem_sh;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer: triplets (x-1..x+1, y) for y = y0-1 .. y0+R of each tile
      umma::tma_prefetch_map(&in_map);
      int s = 0;
      uint32_t ph = 0;
      long long issued = 0;
      bool ok = true;
      for (long long t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
        const int zt = (int)(t % a.tiles_z);
        const long long xy = t / a.tiles_z;
        const int y0 = (int)(xy % yq_count) * R, x = (int)(xy / yq_count);
        for (int yi = 0; yi < NY; ++yi) {
          if (!umma::mbar_wait(&empty[s], ph ^ 1, WAIT_BUDGET)) {
            atomicCAS(a.status, 0, NET_TIMEOUT);
            ok = false;
            break;
          }
          const int ys = (y0 + yi - (FOLD ? 0 : 1) + n) % n;
          umma::mbar_arrive_expect_tx(&full[s], 3 * ROW_BYTES);
          for (int r = 0; r < 3; ++r) {
            const int xs = (x + r - 1 + n) % n;
            umma::tma_load_5d(slots + (size_t)(s * 3 + r) * ROW_BYTES, &in_map, &full[s], 0, zt * (TILE_M / 8), 0, ys,
                              xs);
          }
          ++issued;
          if (++s == NSLOT) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      // drain: wait until the loads still in flight have landed (they complete without a consumer)
      for (int k = 0; k < NSLOT && issued > 0; ++k, --issued) {
        s = s == 0 ? NSLOT - 1 : s - 1;
        if (s == NSLOT - 1) ph ^= 1;
        umma::mbar_wait(&full[s], ph, WAIT_BUDGET);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer. Input row (x + dx, y) feeds output rows y - dy, dy in {+1, 0, -1}, of the tile:
      // one MMA of N = 16 x (rows in the tile) per (dx, dz) with the stacked weights, written to
      // those rows' adjacent accumulators. An output row's accumulator starts on the first MMA of
      // the triplet y = row - 1 (dx = -1, dz = -1), which is split so that the new row is
      // written without accumulation.
      // Descriptors as 64-bit words, moved by adding (bytes >> 4) to the start-address field (shared
      // addresses stay below 256 KB, so the 14-bit field never carries): A of slot 0, row x-1, no z
      // shift; B of the (dx, dz) = (-1, -1) stack. N = 16 x rows is bits 17.. of the instruction word.
      const uint64_t a0 = umma::sdesc(umma::smem_u32(slots), PLANE_BYTES, 128);
      const uint64_t b0 = umma::sdesc(umma::smem_u32(wsm), WS_BYTES / 2, 128);
      constexpr uint32_t ID0 = umma::idesc_bf16(TILE_M, 0, false, false);
      int s = 0, ab = 0;
      uint32_t ph = 0, aph = 0;
      bool ok = true;
      for (long long t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
        if (!umma::mbar_wait(&acc_empty[ab], aph ^ 1, WAIT_BUDGET)) {
          atomicCAS(a.status, 0, NET_TIMEOUT);
          break;
        }
        const uint32_t dbase = tmem + (uint32_t)(ab * R * NET_C);
        for (int yi = 0; yi < NY; ++yi) {
          if (!umma::mbar_wait(&full[s], ph, WAIT_BUDGET)) {
            atomicCAS(a.status, 0, NET_TIMEOUT);
            ok = false;
            break;
          }
          umma::tc_fence_after();
          const uint64_t as = a0 + (uint64_t)(s * (SLOT_BYTES >> 4));
          if constexpr (FOLD) {  // output row yi from the rows x-1, x, x+1 at its y, z shift 0
            const uint64_t bf = umma::sdesc(umma::smem_u32(wsm), 256, 128);
            const uint32_t d = dbase + (uint32_t)(yi * NET_C);
#pragma unroll
            for (int dxi = 0; dxi < 3; ++dxi)
              umma::mma_bf16(d, as + (uint64_t)(dxi * (ROW_BYTES >> 4) + 1), bf + (uint64_t)(dxi * 32),
                             ID0 | (1u << 18), dxi ? 1u : 0u);
            umma::mma_commit(&empty[s]);
            if (++s == NSLOT) {
              s = 0;
              ph ^= 1;
            }
            continue;
          }
          const int a_lo = yi - 2 > 0 ? yi - 2 : 0, a_hi = yi < R - 1 ? yi : R - 1;
          const int j = a_lo - (yi - 2);  // first stacked block used
          const uint64_t bj = b0 + (uint64_t)(j * 16);
          const uint32_t d = dbase + (uint32_t)(a_lo * NET_C);
          const uint32_t idn = ID0 | ((uint32_t)(a_hi - a_lo + 1) << 18);
          if (yi < R) {  // (dx, dz) = (-1, -1): rows a_lo .. yi-1 accumulate, row yi starts here
            const int old = yi - a_lo;
            if (old > 0) umma::mma_bf16(d, as, bj, ID0 | ((uint32_t)old << 18), 1u);
            umma::mma_bf16(d + (uint32_t)(old * NET_C), as, bj + (uint64_t)(old * 16), ID0 | (1u << 18), 0u);
          } else {
            umma::mma_bf16(d, as, bj, idn, 1u);
          }
#pragma unroll
          for (int k = 1; k < 9; ++k) {  // k = (dx + 1) * 3 + (dz + 1)
            const uint32_t aoff = (uint32_t)((k / 3) * (ROW_BYTES >> 4) + (k % 3));
            umma::mma_bf16(d, as + aoff, bj + (uint64_t)(k * (WS_BYTES >> 4)), idn, 1u);
          }
          umma::mma_commit(&empty[s]);
          if (++s == NSLOT) {
            s = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        umma::mma_commit(&acc_full[ab]);
        if (++ab == 2) {
          ab = 0;
          aph ^= 1;
        }
      }
      umma::mma_commit(done);
      umma::mbar_wait(done, 0, WAIT_BUDGET);
    }
  } else {
    // epilogue: warps 2..9. Warp w reads TMEM lane quarter w % 4 (its voxels); warps 2-5 take
    // output rows 0-7 of the tile, warps 6-9 rows 8-15, four rows per TMEM round trip.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int m = q * 32 + lane;
    int ab = 0;
    uint32_t aph = 0;
    const float scale = a.out_scale_dev ? *a.out_scale_dev : a.out_scale;
    constexpr int HR = R / 2, GR = 4;
    for (long long t = blockIdx.x; t < a.tiles; t += gridDim.x) {
      if (!umma::mbar_wait(&acc_full[ab], aph, WAIT_BUDGET)) {
        atomicCAS(a.status, 0, NET_TIMEOUT);
        break;
      }
      umma::tc_fence_after();
      const int zt = (int)(t % a.tiles_z);
      const long long xy = t / a.tiles_z;
      const int y0 = (int)(xy % yq_count) * R, x = (int)(xy / yq_count);
      const int z = zt * TILE_M + m;
      for (int g = 0; g < HR; g += GR) {
        uint32_t r4[GR][16];
#pragma unroll
        for (int j = 0; j < GR; ++j)
          umma::tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((ab * R + half * HR + g + j) * NET_C), r4[j]);
        umma::tmem_wait_ld();
        if (g + GR == HR) {  // every accumulator of this warp is in registers: release them
          umma::tc_fence_before();
          umma::mbar_arrive(&acc_empty[ab]);
        }
        if (z >= n) continue;
#pragma unroll
        for (int j = 0; j < GR; ++j) {
          const int y = y0 + half * HR + g + j;
          float v[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r4[j][c]);
          if (a.out_f4) {
            a.out_f4[((size_t)x * n + y) * n + z] = make_float4(v[0] * scale, v[1] * scale, v[2] * scale, 0.0f);
            continue;
          }
          if (a.act) {
#pragma unroll
            for (int c = 0; c < 16; ++c) v[c] = lrelu(v[c]);
          }
          if (a.gate) {
            const uint4 g0 = *reinterpret_cast<const uint4*>(a.gate + a.g.at(x, y, 0, z + 1));
            const uint4 g1 = *reinterpret_cast<const uint4*>(a.gate + a.g.at(x, y, 1, z + 1));
            const uint32_t gw[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const float2 gv = unpack_bf16x2(gw[k]);
              v[2 * k] *= gv.x > 0.0f ? 1.0f : NET_SLOPE;
              v[2 * k + 1] *= gv.y > 0.0f ? 1.0f : NET_SLOPE;
            }
          }
          const uint4 c0 = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                      pack_bf16x2(v[6], v[7]));
          const uint4 c1 = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
                                      pack_bf16x2(v[14], v[15]));
          store_voxel16(a.out16, a.g, x, y, z, c0, c1);
        }
      }
      if (++ab == 2) {
        ab = 0;
        aph ^= 1;
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  if (warp == 0) umma::tmem_dealloc(tmem, 2 * R * NET_C);
}

// ---------------------------------------------------------------------------------------------
// Weight gradient
// ---------------------------------------------------------------------------------------------
struct WgradArgs {
  TensorGeo g;
  int tiles_z;
  long long tiles;
  float* dw;  // [27][16 co][16 ci] FP32, accumulated with atomics
  int* status;
};

template <int NSTAGE>
__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv3_wgrad(const __grid_constant__ CUtensorMap grad_map, const __grid_constant__ CUtensorMap in_map,
                  WgradArgs a) {
  constexpr int STAGE_BYTES = 9 * GRAD_ROW + ROW_BYTES;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NSTAGE * STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + NSTAGE;
  uint64_t* done = bars + 2 * NSTAGE;
  uint32_t* tmem_sh = reinterpret_cast<uint32_t*>(bars + 2 * NSTAGE + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = a.g.n;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) {
    umma::tmem_alloc(tmem_sh, 128);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tmem_sh;
  bool mma_started = false;

  if (warp == 0) {
    if (lane == 0) {  // producer: gradient rows j -> (x - dx, y - dy), input row (x, y)
      umma::tma_prefetch_map(&grad_map);
      umma::tma_prefetch_map(&in_map);
      int s = 0;
      uint32_t ph = 0;
      long long issued = 0;
      for (long long t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        if (!umma::mbar_wait(&empty[s], ph ^ 1, WAIT_BUDGET)) {
          atomicCAS(a.status, 0, NET_TIMEOUT);
          break;
        }
        const int zt = (int)(t % a.tiles_z);
        const long long xy = t / a.tiles_z;
        const int y = (int)(xy % n), x = (int)(xy / n);
        uint8_t* st = smem + (size_t)s * STAGE_BYTES;
        umma::mbar_arrive_expect_tx(&full[s], 9 * GRAD_ROW + ROW_BYTES);
        for (int j = 0; j < 9; ++j) {
          const int xs = (x - (j / 3 - 1) + n) % n, ys = (y - (j % 3 - 1) + n) % n;
          umma::tma_load_5d(st + (size_t)j * GRAD_ROW, &grad_map, &full[s], 0, zt * TILE_M + 1, 0, ys, xs);
        }
        umma::tma_load_5d(st + 9 * GRAD_ROW, &in_map, &full[s], 0, zt * (TILE_M / 8), 0, y, x);
        ++issued;
        if (++s == NSTAGE) {
          s = 0;
          ph ^= 1;
        }
      }
      for (int k = 0; k < NSTAGE && issued > 0; ++k, --issued) {
        s = s == 0 ? NSTAGE - 1 : s - 1;
        if (s == NSTAGE - 1) ph ^= 1;
        umma::mbar_wait(&full[s], ph, WAIT_BUDGET);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t IDESC = umma::idesc_bf16(TILE_M, 32, true, true);
      int s = 0;
      uint32_t ph = 0;
      for (long long t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        if (!umma::mbar_wait(&full[s], ph, WAIT_BUDGET)) {
          atomicCAS(a.status, 0, NET_TIMEOUT);
          break;
        }
        umma::tc_fence_after();
        const int zt = (int)(t % a.tiles_z);
        const int ksteps = min(TILE_M, n - zt * TILE_M) / 16;
        const uint32_t gbase = umma::smem_u32(smem + (size_t)s * STAGE_BYTES);
        const uint32_t ibase = gbase + 9 * GRAD_ROW;
        for (int k = 0; k < ksteps; ++k)
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            // A: rows j = mt .. mt+7, MN-major: 8 output channels per core matrix, groups (j, chunk)
            // 2048 B apart, 8-voxel K groups 128 B apart
            const uint64_t ad = umma::sdesc(gbase + (uint32_t)(mt * GRAD_ROW + k * 256), 128, GRAD_PLANE);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              // B: input chunk c; N groups = z shifts s = 0..3 (16 B apart, overlapping), K groups 128 B
              const uint64_t bd = umma::sdesc(ibase + (uint32_t)(c * PLANE_BYTES + k * 256), 128, 16);
              umma::mma_bf16(tmem + (uint32_t)((mt * 2 + c) * 32), ad, bd, IDESC, mma_started ? 1u : 0u);
            }
            if (mt == 1) mma_started = true;
          }
        umma::mma_commit(&empty[s]);
        if (++s == NSTAGE) {
          s = 0;
          ph ^= 1;
        }
      }
      umma::mma_commit(done);
    }
  } else {  // epilogue: after every MMA of the CTA, reduce the accumulators into dW
    if (!umma::mbar_wait(done, 0, WAIT_BUDGET)) atomicCAS(a.status, 0, NET_TIMEOUT);
    umma::tc_fence_after();
    const int q = warp & 3;
    const int m = q * 32 + lane;
    const bool any = blockIdx.x < a.tiles;  // every CTA of the grid owns at least one tile of >= 16 voxels
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll 1
      for (int c = 0; c < 2; ++c) {
        uint32_t r0[16], r1[16];
        const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((mt * 2 + c) * 32);
        umma::tmem_ld16(ta, r0);
        umma::tmem_ld16(ta + 16, r1);
        umma::tmem_wait_ld();
        const int j = mt + m / 16, co = m % 16;
        if (!any || (mt == 1 && j != 8)) continue;
#pragma unroll
        for (int nn = 0; nn < 24; ++nn) {
          const float v = __uint_as_float(nn < 16 ? r0[nn] : r1[nn - 16]);
          const int sft = nn / 8, ci = c * 8 + (nn % 8);
          atomicAdd(&a.dw[((j * 3 + sft) * NET_C + co) * NET_C + ci], v);
        }
      }
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// ---------------------------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------------------------
// Input tensor: channel 0 = in_scale * delta, other channels 0. delta from an f32 mesh or from the
// u64 fixed-point mass mesh (delta = c / mean - 1, integrator.rs:117-126).
__global__ void k_net_input(const float* __restrict__ delta, const unsigned long long* __restrict__ fx, float inv_fx,
                            float mean, float in_scale, TensorGeo g, __nv_bfloat16* __restrict__ out) {
  const size_t m = (size_t)g.n * g.n * g.n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % g.n);
    const size_t xy = i / g.n;
    const int y = (int)(xy % g.n), x = (int)(xy / g.n);
    float d;
    if (delta) {
      d = delta[i];
    } else {
      const float c = __fmul_rn(__ull2float_rn(fx[i]), inv_fx);
      d = __fsub_rn(__fdiv_rn(c, mean), 1.0f);
    }
    const uint4 c0 = make_uint4(pack_bf16x2(d * in_scale, 0.0f), 0u, 0u, 0u);
    store_voxel16(out, g, x, y, z, c0, make_uint4(0u, 0u, 0u, 0u));
  }
}

// The first layer's input with its y and z taps folded into channels: channel 3 dyi + dzi of voxel
// (x, y, z) holds s_in delta at (x, y + dyi - 1, z + dzi - 1) (periodic), channels 9-15 are 0 — the
// same BF16 values as k_net_input's channel 0, nine times. A CTA covers 8 y by 32 z of one x plane
// and stages the 10 x 34 neighbourhood in shared memory. delta as in k_net_input.
__global__ void __launch_bounds__(256) k_net_input_fold(const unsigned long long* __restrict__ fx, float inv_fx,
                                                        float mean, float in_scale, TensorGeo g,
                                                        __nv_bfloat16* __restrict__ out) {
  __shared__ float sd[10][34];
  const int n = g.n;
  const int z0 = blockIdx.x * 32, y0 = blockIdx.y * 8, x = blockIdx.z;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  for (int k = tid; k < 10 * 34; k += 256) {
    const int yy = k / 34, zz = k % 34;
    const int y = (y0 - 1 + yy + n) % n, z = (z0 - 1 + zz + n) % n;
    const float c = __fmul_rn(__ull2float_rn(fx[((size_t)x * n + y) * n + z]), inv_fx);
    sd[yy][zz] = __fsub_rn(__fdiv_rn(c, mean), 1.0f) * in_scale;
  }
  __syncthreads();
  const int z = z0 + threadIdx.x, y = y0 + threadIdx.y;
  if (z >= n || y >= n) return;
  float v[10];
#pragma unroll
  for (int c = 0; c < 9; ++c) v[c] = sd[threadIdx.y + c / 3][threadIdx.x + c % 3];
  v[9] = 0.0f;
  const uint4 c0 = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                              pack_bf16x2(v[6], v[7]));
  const uint4 c1 = make_uint4(pack_bf16x2(v[8], v[9]), 0u, 0u, 0u);
  store_voxel16(out, g, x, y, z, c0, c1);
}

// Gradient of the loss with respect to the field, as a BF16 tensor: channels 0-2 = s * dF, rest 0.
__global__ void k_net_grad_input(const float4* __restrict__ df, float s, TensorGeo g, __nv_bfloat16* __restrict__ out) {
  const size_t m = (size_t)g.n * g.n * g.n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % g.n);
    const size_t xy = i / g.n;
    const int y = (int)(xy % g.n), x = (int)(xy / g.n);
    const float4 v = df[i];
    const uint4 c0 = make_uint4(pack_bf16x2(v.x * s, v.y * s), pack_bf16x2(v.z * s, 0.0f), 0u, 0u);
    store_voxel16(out, g, x, y, z, c0, make_uint4(0u, 0u, 0u, 0u));
  }
}

// Packs master weights W[t][co][ci] (FP32) into the B-operand layout [t][chunk][co][8] (BF16):
// forward, and (transpose) the data-gradient operand W'[t][ci][co] = W[26 - t][co][ci].
__global__ void k_net_pack(const float* __restrict__ w, int transpose, __nv_bfloat16* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NET_TAPS * NET_C * NET_C) return;
  const int k = i % 8, o = (i / 8) % NET_C, c = (i / (8 * NET_C)) % 2, t = i / (16 * NET_C);
  const int inner = c * 8 + k;  // K index (input channel of this operand)
  const float v = transpose ? w[((NET_TAPS - 1 - t) * NET_C + inner) * NET_C + o] : w[(t * NET_C + o) * NET_C + inner];
  out[i] = __float2bfloat16_rn(v);
}

// Which master weights exist: layer 0 reads channel 0 only; layer 2 writes channels 0-2 only.
__device__ __forceinline__ bool net_weight_live(int idx) {
  const int layer = idx / (NET_TAPS * NET_C * NET_C);
  const int ci = idx % NET_C, co = (idx / NET_C) % NET_C;
  if (layer == 0 && ci != 0) return false;
  if (layer == NET_LAYERS - 1 && co >= NET_OUT) return false;
  return true;
}

__global__ void k_net_mask(float* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NET_WEIGHTS && !net_weight_live(i)) w[i] = 0.0f;
}

// Adam (Kingma & Ba 2015) on the live master weights; bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t.
__global__ void k_net_adam(float* __restrict__ w, float* __restrict__ m1, float* __restrict__ m2,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NET_WEIGHTS || !net_weight_live(i)) return;
  const float gi = grad[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// Loss of one training sample and its gradient with respect to the field F (float4 mesh):
// pred_i = CIC gather of F at x_i (mesh.rs:72-77 stencil); for particles with weight_i > 0,
// L = sum_i weight_i |pred_i - target_i|^2 * inv_norm; dF += CIC scatter of dL/dpred_i.
__global__ void k_net_loss_grad(const float4* __restrict__ f, const float* __restrict__ x3,
                                const float* __restrict__ target3, const float* __restrict__ weight, size_t np,
                                int n, float h, float inv_norm, float4* __restrict__ df, double* __restrict__ sums) {
  double l_acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    const float wi = weight[i];
    if (!(wi > 0.0f)) continue;
    const float x[3] = {x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]};
    CicBase cb;
    cic_base(x, h, n, cb);
    float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
    size_t idx[8];
    float w8[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      idx[c] = cic_index(cb, c, n);
      w8[c] = cic_weight(cb, c);
      const float4 v = __ldg(f + idx[c]);
      p0 += w8[c] * v.x;
      p1 += w8[c] * v.y;
      p2 += w8[c] * v.z;
    }
    const float d0 = p0 - target3[3 * i], d1 = p1 - target3[3 * i + 1], d2 = p2 - target3[3 * i + 2];
    l_acc += (double)(wi * (d0 * d0 + d1 * d1 + d2 * d2));
    const float gs = 2.0f * wi * inv_norm;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float* dst = reinterpret_cast<float*>(df + idx[c]);
      atomicAdd(dst, gs * d0 * w8[c]);
      atomicAdd(dst + 1, gs * d1 * w8[c]);
      atomicAdd(dst + 2, gs * d2 * w8[c]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l_acc += __shfl_xor_sync(0xffffffffu, l_acc, o);
  if ((threadIdx.x & 31) == 0 && l_acc != 0.0) atomicAdd(&sums[0], l_acc * (double)inv_norm);
}

// ---------------------------------------------------------------------------------------------
// Host side: tensor maps, buffers, launches
// ---------------------------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn(std::string* err) {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  if (!fn && err) *err = "cuTensorMapEncodeTiled is not available from the driver";
  return fn;
}

// Tensor maps over a BF16 activation tensor [x][y][chunk 2][n + 8][8].
// Row map (forward and weight-gradient input rows, loaded at z offsets that are multiples of 8
// voxels): viewed as 5-D (64 = 8 voxels x 8 channels, (n + 8) / 8, chunk, y, x), box (64, box_z / 8,
// 2, 1, 1), so the box's innermost extent is 128 contiguous bytes and the TMA unit requests whole
// 128-byte lines. With a 16-byte innermost extent (8 channels of one voxel) it read every 32-byte
// sector twice: 3.85 GB from L2 for the 1.93 GB of rows a forward layer at 256^3 loads.
// Gradient-row map (weight gradient, loaded at z + 1): (8 channels, n + 8, chunk, y, x), box
// (8, box_z, 2, 1, 1) — its z offset is not a multiple of 8.
static bool make_row_map(CUtensorMap* map, const __nv_bfloat16* t, int n, int box_z, bool grouped, std::string* err) {
  EncodeTiledFn fn = encode_fn(err);
  if (!fn) return false;
  const cuuint64_t zp = (cuuint64_t)n + 8;
  const cuuint64_t dims_g[5] = {64, zp / 8, 2, (cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides_g[4] = {128, zp * 16, 2 * zp * 16, (cuuint64_t)n * 2 * zp * 16};
  const cuuint32_t box_g[5] = {64, (cuuint32_t)box_z / 8, 2, 1, 1};
  const cuuint64_t dims_v[5] = {8, zp, 2, (cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides_v[4] = {16, zp * 16, 2 * zp * 16, (cuuint64_t)n * 2 * zp * 16};
  const cuuint32_t box_v[5] = {8, (cuuint32_t)box_z, 2, 1, 1};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(t),
                        grouped ? dims_g : dims_v, grouped ? strides_g : strides_v, grouped ? box_g : box_v, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS && err) *err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
  return r == CUDA_SUCCESS;
}

constexpr size_t conv_smem_bytes(int slots) {
  return (size_t)slots * SLOT_BYTES + W_BYTES + 8 * (2 * slots + 5) + 16;
}
constexpr size_t wgrad_smem_bytes(int stages) {
  return (size_t)stages * (9 * GRAD_ROW + ROW_BYTES) + 8 * (2 * stages + 1) + 16;
}

static int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached = v > 0 ? v : 148;
  }
  return cached;
}

}  // namespace cpm

using namespace cpm;

struct cpm_net {
  int n = 0;
  TensorGeo g{};
  std::string err;
  cudaStream_t own = nullptr;
  DevBuf t_in, t_a1, t_a2, t_g3, t_g2, t_g1;  // BF16 tensors
  DevBuf w, m1, m2, grad;                     // FP32 master weights, Adam moments, gradient
  DevBuf wf, wb;                              // packed BF16 operands: forward, data gradient (3 layers each)
  DevBuf field, dfield;                       // float4 meshes
  DevBuf scratch;                             // status word, loss sums
  CUtensorMap map_in, map_a1, map_a2;         // row maps of the inputs of the three layers
  CUtensorMap map_g3, map_g2;                 // row maps of the gradient tensors (data gradient input)
  CUtensorMap gmap_g3, gmap_g2, gmap_g1;      // gradient-row maps of the weight-gradient kernel
  long long adam_t = 0;
  bool train_ready = false;
};

namespace {

#define NET_CU(net, call)                                                                                    \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess)                                                                                   \
      return set_error(&(net)->err, e_ == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,              \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                                  \
  } while (0)

int* net_status(cpm_net* net) { return static_cast<int*>(net->scratch.p); }
double* net_sums(cpm_net* net) { return reinterpret_cast<double*>(static_cast<char*>(net->scratch.p) + 16); }

size_t tensor_bytes(int n) { return (size_t)n * n * 2 * ((size_t)n + 8) * 8 * sizeof(__nv_bfloat16); }

void launch_conv(cpm_net* net, const CUtensorMap& in_map, int layer, bool transpose, __nv_bfloat16* out16,
                 float4* out_f4, const __nv_bfloat16* gate, int act, float out_scale, const float* out_scale_dev,
                 cudaStream_t s, bool fold = false) {
  ConvArgs a;
  a.g = net->g;
  a.tiles_z = (net->n + TILE_M - 1) / TILE_M;
  a.tiles = (long long)net->n * (net->n / CONV_ROWS) * a.tiles_z;  // n is a multiple of 16
  a.w = static_cast<const __nv_bfloat16*>(transpose ? net->wb.p : net->wf.p) + (size_t)layer * NET_TAPS * NET_C * NET_C;
  a.out16 = out16;
  a.out_f4 = out_f4;
  a.gate = gate;
  a.act = act;
  a.out_scale = out_scale;
  a.out_scale_dev = out_scale_dev;
  a.status = net_status(net);
  const size_t smem = conv_smem_bytes(CONV_SLOTS);
  const long long grid = std::min<long long>(a.tiles, sm_count());
  count_launch();
  if (fold) {
    cudaFuncSetAttribute(k_conv3<CONV_SLOTS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_conv3<CONV_SLOTS, true><<<(unsigned)grid, FWD_THREADS, smem, s>>>(in_map, a);
  } else {
    cudaFuncSetAttribute(k_conv3<CONV_SLOTS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_conv3<CONV_SLOTS, false><<<(unsigned)grid, FWD_THREADS, smem, s>>>(in_map, a);
  }
}

void launch_wgrad(cpm_net* net, const CUtensorMap& grad_map, const CUtensorMap& in_map, int layer, cudaStream_t s) {
  WgradArgs a;
  a.g = net->g;
  a.tiles_z = (net->n + TILE_M - 1) / TILE_M;
  a.tiles = (long long)net->n * net->n * a.tiles_z;
  a.dw = static_cast<float*>(net->grad.p) + (size_t)layer * NET_TAPS * NET_C * NET_C;
  a.status = net_status(net);
  const size_t smem = wgrad_smem_bytes(WG_STAGES);
  cudaFuncSetAttribute(k_conv3_wgrad<WG_STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long grid = std::min<long long>(a.tiles, sm_count());
  count_launch();
  k_conv3_wgrad<WG_STAGES><<<(unsigned)grid, CONV_THREADS, smem, s>>>(grad_map, in_map, a);
}

unsigned grid_1d(size_t work) {
  size_t b = (work + 255) / 256;
  if (b > (size_t)sm_count() * 16) b = (size_t)sm_count() * 16;
  return (unsigned)(b ? b : 1);
}

void pack_weights(cpm_net* net, cudaStream_t s) {
  const int per = NET_TAPS * NET_C * NET_C;
  for (int l = 0; l < NET_LAYERS; ++l) {
    const float* w = static_cast<const float*>(net->w.p) + (size_t)l * per;
    count_launch();
    k_net_pack<<<(per + 255) / 256, 256, 0, s>>>(w, 0, static_cast<__nv_bfloat16*>(net->wf.p) + (size_t)l * per);
    count_launch();
    k_net_pack<<<(per + 255) / 256, 256, 0, s>>>(w, 1, static_cast<__nv_bfloat16*>(net->wb.p) + (size_t)l * per);
  }
}

int net_check(cpm_net* net, cudaStream_t s) {
  NET_CU(net, cudaStreamSynchronize(s));
  NET_CU(net, cudaGetLastError());
  int st = 0;
  NET_CU(net, cudaMemcpy(&st, net->scratch.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != NET_OK) {
    cudaMemset(net->scratch.p, 0, sizeof(int));
    return set_error(&net->err, CPM_E_DEVICE, "net kernel reported status " + std::to_string(st) + " (a wait timed out)");
  }
  return CPM_OK;
}

int ensure_train(cpm_net* net) {
  if (net->train_ready) return CPM_OK;
  const size_t tb = tensor_bytes(net->n);
  for (DevBuf* b : {&net->t_g3, &net->t_g2, &net->t_g1}) NET_CU(net, ensure(*b, tb));
  NET_CU(net, ensure(net->dfield, (size_t)net->n * net->n * net->n * sizeof(float4)));
  NET_CU(net, cudaMemset(net->t_g3.p, 0, tb));
  NET_CU(net, cudaMemset(net->t_g2.p, 0, tb));
  NET_CU(net, cudaMemset(net->t_g1.p, 0, tb));
  const __nv_bfloat16* g3 = static_cast<const __nv_bfloat16*>(net->t_g3.p);
  const __nv_bfloat16* g2 = static_cast<const __nv_bfloat16*>(net->t_g2.p);
  const __nv_bfloat16* g1 = static_cast<const __nv_bfloat16*>(net->t_g1.p);
  if (!make_row_map(&net->map_g3, g3, net->n, ROW_BOX, true, &net->err) ||
      !make_row_map(&net->map_g2, g2, net->n, ROW_BOX, true, &net->err) ||
      !make_row_map(&net->gmap_g3, g3, net->n, TILE_M, false, &net->err) ||
      !make_row_map(&net->gmap_g2, g2, net->n, TILE_M, false, &net->err) ||
      !make_row_map(&net->gmap_g1, g1, net->n, TILE_M, false, &net->err))
    return set_error(&net->err, CPM_E_CUDA, net->err);
  net->train_ready = true;
  return CPM_OK;
}

// Input tensor from delta (f32 mesh) or the fixed-point mass mesh, then the three layers into `field`.
// fold (inference from the mass mesh): the first layer on the folded input; the training path keeps
// the single-channel input, whose tensor the first layer's weight gradient reads.
void net_forward_launch(cpm_net* net, const float* delta, const unsigned long long* fx, int fx_shift, float mean,
                        float in_scale, float out_scale, const float* out_scale_dev, float4* field, cudaStream_t s,
                        bool fold = false) {
  const size_t m = (size_t)net->n * net->n * net->n;
  const int n = net->n;
  count_launch();
  if (fold && fx) {
    k_net_input_fold<<<dim3((unsigned)((n + 31) / 32), (unsigned)((n + 7) / 8), (unsigned)n), dim3(32, 8), 0, s>>>(
        fx, std::ldexp(1.0f, -fx_shift), mean, in_scale, net->g, static_cast<__nv_bfloat16*>(net->t_in.p));
  } else {
    fold = false;
    k_net_input<<<grid_1d(m), 256, 0, s>>>(delta, fx, std::ldexp(1.0f, -fx_shift), mean, in_scale, net->g,
                                           static_cast<__nv_bfloat16*>(net->t_in.p));
  }
  launch_conv(net, net->map_in, 0, false, static_cast<__nv_bfloat16*>(net->t_a1.p), nullptr, nullptr, 1, 1.0f, nullptr, s,
              fold);
  launch_conv(net, net->map_a1, 1, false, static_cast<__nv_bfloat16*>(net->t_a2.p), nullptr, nullptr, 1, 1.0f, nullptr, s);
  launch_conv(net, net->map_a2, 2, false, nullptr, field, nullptr, 0, out_scale, out_scale_dev, s);
}

// Backward from dL/dF (float4 mesh `dfield`, F = out_scale * y) into the weight gradient (zeroed first).
void net_backward_launch(cpm_net* net, float out_scale, cudaStream_t s) {
  const size_t m = (size_t)net->n * net->n * net->n;
  cudaMemsetAsync(net->grad.p, 0, NET_WEIGHTS * sizeof(float), s);
  __nv_bfloat16* g3 = static_cast<__nv_bfloat16*>(net->t_g3.p);
  __nv_bfloat16* g2 = static_cast<__nv_bfloat16*>(net->t_g2.p);
  __nv_bfloat16* g1 = static_cast<__nv_bfloat16*>(net->t_g1.p);
  count_launch();
  k_net_grad_input<<<grid_1d(m), 256, 0, s>>>(static_cast<const float4*>(net->dfield.p), out_scale, net->g, g3);
  launch_wgrad(net, net->gmap_g3, net->map_a2, 2, s);
  launch_conv(net, net->map_g3, 2, true, g2, nullptr, static_cast<const __nv_bfloat16*>(net->t_a2.p), 0, 1.0f,
              nullptr, s);
  launch_wgrad(net, net->gmap_g2, net->map_a1, 1, s);
  launch_conv(net, net->map_g2, 1, true, g1, nullptr, static_cast<const __nv_bfloat16*>(net->t_a1.p), 0, 1.0f,
              nullptr, s);
  launch_wgrad(net, net->gmap_g1, net->map_in, 0, s);
}

}  // namespace

namespace cpm {
// Simulation hook (sim.cu): the field of the learned short-range force from the fixed-point mesh.
float4* net_field_from_mesh(cpm_net* net, const unsigned long long* fx, int fx_shift, float mean, float in_scale,
                            float out_scale, const float* out_scale_dev, cudaStream_t s) {
  float4* field = static_cast<float4*>(net->field.p);
  net_forward_launch(net, nullptr, fx, fx_shift, mean, in_scale, out_scale, out_scale_dev, field, s, true);
  return field;
}
int net_mesh(const cpm_net* net) { return net ? net->n : 0; }
int* net_status_word(cpm_net* net) { return net_status(net); }
}  // namespace cpm

extern "C" {

int cpm_net_create(int n_mesh, cpm_net** out) {
  if (!out) return set_error(nullptr, CPM_E_INVALID, "cpm_net_create: out is NULL");
  *out = nullptr;
  if (n_mesh < 16 || n_mesh > 1024 || n_mesh % 16 != 0)
    return set_error(nullptr, CPM_E_INVALID, "cpm_net_create: n_mesh must be a multiple of 16 in [16, 1024]");
  int rc = check_device_once(nullptr);
  if (rc) return rc;
  cpm_net* net = new cpm_net();
  net->n = n_mesh;
  net->g = TensorGeo{n_mesh, n_mesh + 8};
  auto fail = [&](int code) {
    g_last_error = net->err;
    cpm_net_destroy(net);
    return code;
  };
  const size_t tb = tensor_bytes(n_mesh);
  bool ok = true;
  for (DevBuf* b : {&net->t_in, &net->t_a1, &net->t_a2}) ok = ok && ensure(*b, tb) == cudaSuccess;
  for (DevBuf* b : {&net->w, &net->m1, &net->m2, &net->grad}) ok = ok && ensure(*b, NET_WEIGHTS * sizeof(float)) == cudaSuccess;
  for (DevBuf* b : {&net->wf, &net->wb}) ok = ok && ensure(*b, NET_WEIGHTS * sizeof(__nv_bfloat16)) == cudaSuccess;
  ok = ok && ensure(net->field, (size_t)n_mesh * n_mesh * n_mesh * sizeof(float4)) == cudaSuccess;
  ok = ok && ensure(net->scratch, 64) == cudaSuccess;
  if (!ok) {
    net->err = "cpm_net_create: device allocation failed";
    return fail(CPM_E_NOMEM);
  }
  for (DevBuf* b : {&net->t_in, &net->t_a1, &net->t_a2}) cudaMemset(b->p, 0, tb);
  for (DevBuf* b : {&net->w, &net->m1, &net->m2, &net->grad}) cudaMemset(b->p, 0, NET_WEIGHTS * sizeof(float));
  cudaMemset(net->scratch.p, 0, 64);
  if (!make_row_map(&net->map_in, static_cast<const __nv_bfloat16*>(net->t_in.p), n_mesh, ROW_BOX, true, &net->err) ||
      !make_row_map(&net->map_a1, static_cast<const __nv_bfloat16*>(net->t_a1.p), n_mesh, ROW_BOX, true, &net->err) ||
      !make_row_map(&net->map_a2, static_cast<const __nv_bfloat16*>(net->t_a2.p), n_mesh, ROW_BOX, true, &net->err))
    return fail(set_error(&net->err, CPM_E_CUDA, net->err));
  pack_weights(net, nullptr);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    net->err = "cpm_net_create: initialisation failed";
    return fail(CPM_E_CUDA);
  }
  *out = net;
  return CPM_OK;
}

int cpm_net_destroy(cpm_net* net) {
  if (!net) return CPM_OK;
  cudaDeviceSynchronize();
  for (DevBuf* b : {&net->t_in, &net->t_a1, &net->t_a2, &net->t_g3, &net->t_g2, &net->t_g1, &net->w, &net->m1,
                    &net->m2, &net->grad, &net->wf, &net->wb, &net->field, &net->dfield, &net->scratch})
    release(*b);
  delete net;
  return CPM_OK;
}

const char* cpm_net_last_error(const cpm_net* net) { return net ? net->err.c_str() : g_last_error.c_str(); }

int cpm_net_weight_count(void) { return NET_WEIGHTS; }

int cpm_net_set_weights(cpm_net* net, const float* w) {
  if (!net || !w) return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_set_weights: null pointer");
  NET_CU(net, cudaMemcpy(net->w.p, w, NET_WEIGHTS * sizeof(float), cudaMemcpyHostToDevice));
  count_launch();
  k_net_mask<<<(NET_WEIGHTS + 255) / 256, 256>>>(static_cast<float*>(net->w.p));
  NET_CU(net, cudaMemset(net->m1.p, 0, NET_WEIGHTS * sizeof(float)));
  NET_CU(net, cudaMemset(net->m2.p, 0, NET_WEIGHTS * sizeof(float)));
  net->adam_t = 0;
  pack_weights(net, nullptr);
  return net_check(net, nullptr);
}

int cpm_net_get_weights(cpm_net* net, float* w) {
  if (!net || !w) return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_get_weights: null pointer");
  NET_CU(net, cudaMemcpy(w, net->w.p, NET_WEIGHTS * sizeof(float), cudaMemcpyDeviceToHost));
  return CPM_OK;
}

int cpm_net_get_grads(cpm_net* net, float* g) {
  if (!net || !g) return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_get_grads: null pointer");
  NET_CU(net, cudaDeviceSynchronize());
  NET_CU(net, cudaMemcpy(g, net->grad.p, NET_WEIGHTS * sizeof(float), cudaMemcpyDeviceToHost));
  return CPM_OK;
}

int cpm_net_forward(cpm_net* net, const float* delta_dev, float in_scale, float out_scale, float* field4_dev,
                    void* stream) {
  if (!net || !delta_dev || !field4_dev)
    return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_forward: null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  net_forward_launch(net, delta_dev, nullptr, 0, 1.0f, in_scale, out_scale, nullptr,
                     reinterpret_cast<float4*>(field4_dev), s);
  return net_check(net, s);
}

int cpm_net_backward(cpm_net* net, const float* dfield4_dev, float out_scale, void* stream) {
  if (!net || !dfield4_dev) return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_backward: null pointer");
  int rc = ensure_train(net);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NET_CU(net, cudaMemcpyAsync(net->dfield.p, dfield4_dev, (size_t)net->n * net->n * net->n * sizeof(float4),
                              cudaMemcpyDeviceToDevice, s));
  net_backward_launch(net, out_scale, s);
  return net_check(net, s);
}

int cpm_net_activations(cpm_net* net, int which, void* dst_dev, void* stream) {
  if (!net || !dst_dev || which < 0 || which > 5)
    return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_activations: bad arguments");
  const DevBuf* src[6] = {&net->t_in, &net->t_a1, &net->t_a2, &net->t_g3, &net->t_g2, &net->t_g1};
  if (!src[which]->p) return set_error(&net->err, CPM_E_INVALID, "cpm_net_activations: tensor not allocated yet");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NET_CU(net, cudaMemcpyAsync(dst_dev, src[which]->p, tensor_bytes(net->n), cudaMemcpyDeviceToDevice, s));
  return net_check(net, s);
}

int cpm_net_train_step(cpm_net* net, const float* delta_dev, float in_scale, const float* x3_dev,
                       const float* target3_dev, const float* weight_dev, size_t n_particles, float box_size,
                       float inv_norm, float lr, double* loss_out, void* stream) {
  if (!net || !delta_dev || !x3_dev || !target3_dev || !weight_dev)
    return set_error(net ? &net->err : nullptr, CPM_E_INVALID, "cpm_net_train_step: null pointer");
  if (!(box_size > 0.0f) || !(lr >= 0.0f))
    return set_error(&net->err, CPM_E_INVALID, "cpm_net_train_step: box_size must be > 0 and lr >= 0");
  int rc = ensure_train(net);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t m = (size_t)net->n * net->n * net->n;
  float4* field = static_cast<float4*>(net->field.p);
  net_forward_launch(net, delta_dev, nullptr, 0, 1.0f, in_scale, 1.0f, nullptr, field, s);
  NET_CU(net, cudaMemsetAsync(net->dfield.p, 0, m * sizeof(float4), s));
  NET_CU(net, cudaMemsetAsync(net_sums(net), 0, 2 * sizeof(double), s));
  if (n_particles) {
    count_launch();
    k_net_loss_grad<<<grid_1d(n_particles), 256, 0, s>>>(field, x3_dev, target3_dev, weight_dev, n_particles, net->n,
                                                         box_size / (float)net->n, inv_norm,
                                                         static_cast<float4*>(net->dfield.p), net_sums(net));
  }
  net_backward_launch(net, 1.0f, s);
  if (lr > 0.0f) {
    net->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)net->adam_t), c2 = 1.0f - std::pow(b2, (float)net->adam_t);
    count_launch();
    k_net_adam<<<(NET_WEIGHTS + 255) / 256, 256, 0, s>>>(static_cast<float*>(net->w.p), static_cast<float*>(net->m1.p),
                                                         static_cast<float*>(net->m2.p),
                                                         static_cast<const float*>(net->grad.p), lr, b1, b2, 1e-8f, c1,
                                                         c2);
    pack_weights(net, s);
  }
  double sums[2] = {0.0, 0.0};
  NET_CU(net, cudaMemcpyAsync(sums, net_sums(net), sizeof(sums), cudaMemcpyDeviceToHost, s));
  rc = net_check(net, s);
  if (rc) return rc;
  if (loss_out) *loss_out = sums[0];
  return CPM_OK;
}

}  // extern "C"
