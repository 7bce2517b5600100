// fft.cu — shared-memory Stockham FFTs and the PM Poisson solve (fft.rs:40-95, poisson.rs:33-88).
//
// Layouts
//   real mesh      f32  [n][n][n]          (ix*n + iy)*n + iz, z fastest (mesh.rs:11)
//   half spectrum  c32  [n][n][n/2+1]      kz in [0, n/2]; the rest follows from Hermitian symmetry
//
// Every pass moves a tile of lines between HBM and shared memory once: lines along the
// contiguous z axis are loaded as rows; lines along y or x are loaded as W adjacent columns, so
// each row segment of the tile is a contiguous W*8-byte run. Inside shared memory the lines are
// transformed by radix-8/4/2 Stockham stages (in place: each stage reads its butterflies into
// registers, synchronises, then writes them to their autosorted positions). Twiddles come from a
// table exp(-2 pi i m / n) built in double precision on the host.
//
// The Poisson solve runs as
//   1. z pass: R2C of each z row (the input is either f32 delta or the u64 fixed-point mass mesh,
//      converted to delta = c/mean - 1 on load, integrator.rs:117-126);
//   2. y pass: forward c2c along y;
//   3. x pass: forward c2c along x, then the Green's function (poisson.rs:52-74, same f32
//      operation order) applied once, then for each force component the gradient factor -i k_a
//      and the inverse c2c along x — three half spectra written;
//   4. y pass: inverse c2c along y of the three spectra;
//   5. z pass: C2R of each row, scaled by 1/n^3 (poisson.rs:77-87), into three f32 meshes.
#include <cmath>
#include <vector>

#include "cpm_internal.cuh"

namespace cpm {

// ---------------------------------------------------------------------------------------------
// Complex helpers and small DFTs
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by exp(sign i pi/2): -i for the forward transform, +i for the inverse
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
  const float2 a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  const float2 a = cadd(v0, v2), b = csub(v0, v2), c = cadd(v1, v3), d = rot90<INV>(csub(v1, v3));
  v0 = cadd(a, c);
  v1 = cadd(b, d);
  v2 = csub(a, c);
  v3 = csub(b, d);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
  // even/odd split: E = DFT4(v0,v2,v4,v6), O = DFT4(v1,v3,v5,v7); y_m = E_m + w^m O_m, y_{m+4} = E_m - w^m O_m
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  const float r = 0.70710678118654752440f;
  // w = exp(sign i pi / 4)
  const float2 t1 = INV ? make_float2(r * (o1.x - o1.y), r * (o1.x + o1.y)) : make_float2(r * (o1.x + o1.y), r * (o1.y - o1.x));
  const float2 t2 = rot90<INV>(o2);
  const float2 t3 = INV ? make_float2(-r * (o3.x + o3.y), r * (o3.x - o3.y)) : make_float2(r * (o3.y - o3.x), -r * (o3.x + o3.y));
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else dft8<INV>(v);
}

// Shared-memory leading dimension of a line (odd float2 stride spreads columns over banks).
template <int N>
__host__ __device__ constexpr int line_ld() {
  return N + 1;
}

// One Stockham stage of radix R on W lines of length N held in shared memory.
template <int N, int R, int NS, int W, int THREADS, bool INV>
__device__ __forceinline__ void stockham_stage(float2* sm, const float2* __restrict__ tw) {
  constexpr int NB = N / R;
  constexpr int TOTAL = W * NB;
  constexpr int BPT = (TOTAL + THREADS - 1) / THREADS;
  constexpr int LD = line_ld<N>();
  float2 v[BPT][R];
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * THREADS;
    if (TOTAL % THREADS == 0 || b < TOTAL) {
      const int l = b / NB, j = b % NB;
      const float2* line = sm + l * LD;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = line[j + r * NB];
      if constexpr (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = __ldg(tw + r * k * (N / (NS * R)));
          if (INV) w.y = -w.y;
          v[q][r] = cmul(v[q][r], w);
        }
      }
      dft<R, INV>(v[q]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * THREADS;
    if (TOTAL % THREADS == 0 || b < TOTAL) {
      const int l = b / NB, j = b % NB;
      const int k = j % NS;
      float2* line = sm + l * LD;
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) line[base + r * NS] = v[q][r];
    }
  }
  __syncthreads();
}

// Full length-N transform of W lines: radix-8 stages, then a final radix-4 or radix-2 stage.
template <int N, int W, int THREADS, bool INV>
__device__ __forceinline__ void fft_lines(float2* sm, const float2* __restrict__ tw) {
  static_assert((N & (N - 1)) == 0 && N >= 2 && N <= 1024, "power-of-two lengths 2..1024");
  if constexpr (N == 2) {
    stockham_stage<N, 2, 1, W, THREADS, INV>(sm, tw);
  } else if constexpr (N == 4) {
    stockham_stage<N, 4, 1, W, THREADS, INV>(sm, tw);
  } else {
    stockham_stage<N, 8, 1, W, THREADS, INV>(sm, tw);
    if constexpr (N == 16) stockham_stage<N, 2, 8, W, THREADS, INV>(sm, tw);
    if constexpr (N == 32) stockham_stage<N, 4, 8, W, THREADS, INV>(sm, tw);
    if constexpr (N >= 64) stockham_stage<N, 8, 8, W, THREADS, INV>(sm, tw);
    if constexpr (N == 128) stockham_stage<N, 2, 64, W, THREADS, INV>(sm, tw);
    if constexpr (N == 256) stockham_stage<N, 4, 64, W, THREADS, INV>(sm, tw);
    if constexpr (N >= 512) stockham_stage<N, 8, 64, W, THREADS, INV>(sm, tw);
    if constexpr (N == 1024) stockham_stage<N, 2, 512, W, THREADS, INV>(sm, tw);
  }
}

// ---------------------------------------------------------------------------------------------
// Tile geometry: element t of line l of tile (o, c) is at
//   base = o * outer_stride + (c * W + l) * line_stride + t * elem_stride.
// With line_stride == 1 the W lines are adjacent columns (coalesced rows of W elements); with
// elem_stride == 1 each line is a contiguous row.
// ---------------------------------------------------------------------------------------------
struct TileGeo {
  long long outer_stride;
  long long line_stride;
  long long elem_stride;
  int lines;  // number of lines along the tiled direction
};

template <int N, int W, int THREADS>
__device__ __forceinline__ void load_tile(float2* sm, const float2* __restrict__ src, const TileGeo& g, int valid) {
  constexpr int LD = line_ld<N>();
  const long long base = (long long)blockIdx.x * g.outer_stride + (long long)blockIdx.y * W * g.line_stride;
  for (int q = threadIdx.x; q < N * W; q += THREADS) {
    int t, l;
    if (g.line_stride == 1) {
      l = q % W;
      t = q / W;
    } else {
      t = q % N;
      l = q / N;
    }
    if (l < valid) sm[l * LD + t] = src[base + (long long)l * g.line_stride + (long long)t * g.elem_stride];
  }
}

template <int N, int W, int THREADS>
__device__ __forceinline__ void store_tile(const float2* sm, float2* __restrict__ dst, const TileGeo& g, int valid) {
  constexpr int LD = line_ld<N>();
  const long long base = (long long)blockIdx.x * g.outer_stride + (long long)blockIdx.y * W * g.line_stride;
  for (int q = threadIdx.x; q < N * W; q += THREADS) {
    int t, l;
    if (g.line_stride == 1) {
      l = q % W;
      t = q / W;
    } else {
      t = q % N;
      l = q / N;
    }
    if (l < valid) dst[base + (long long)l * g.line_stride + (long long)t * g.elem_stride] = sm[l * LD + t];
  }
}

// Generic c2c pass over one axis (gridDim.z selects one of up to 3 arrays spaced by comp_stride).
template <int N, int W, int THREADS, bool INV>
__global__ void __launch_bounds__(THREADS) k_fft_pass(float2* data, long long comp_stride, TileGeo g,
                                                      const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  float2* d = data + (long long)blockIdx.z * comp_stride;
  const int valid = min(W, g.lines - (int)blockIdx.y * W);
  load_tile<N, W, THREADS>(sm, d, g, valid);
  __syncthreads();
  fft_lines<N, W, THREADS, INV>(sm, tw);
  store_tile<N, W, THREADS>(sm, d, g, valid);
}

// z pass, forward: W real rows of length N -> N/2+1 complex each. Input is either f32 delta or
// the u64 fixed-point mass mesh (cell mass c = fx * 2^-k in f32, delta = c / mean - 1).
template <int N, int W, int THREADS>
__global__ void __launch_bounds__(THREADS) k_r2c_z(const float* __restrict__ delta,
                                                   const unsigned long long* __restrict__ fx, float inv_scale,
                                                   float mean, float2* __restrict__ spec, int rows,
                                                   const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int LD = line_ld<N>();
  constexpr int NH = N / 2 + 1;
  const int row0 = blockIdx.x * W;
  const int valid = min(W, rows - row0);
  for (int q = threadIdx.x; q < N * W; q += THREADS) {
    const int l = q / N, t = q % N;
    if (l < valid) {
      const size_t gi = (size_t)(row0 + l) * N + t;
      float v;
      if (fx) {
        const float c = __fmul_rn(__ull2float_rn(fx[gi]), inv_scale);
        v = __fsub_rn(__fdiv_rn(c, mean), 1.0f);
      } else {
        v = delta[gi];
      }
      sm[l * LD + t] = make_float2(v, 0.0f);
    }
  }
  __syncthreads();
  fft_lines<N, W, THREADS, false>(sm, tw);
  for (int q = threadIdx.x; q < NH * W; q += THREADS) {
    const int l = q / NH, t = q % NH;
    if (l < valid) spec[(size_t)(row0 + l) * NH + t] = sm[l * LD + t];
  }
}

// z pass, inverse: N/2+1 complex per row -> N real values (Hermitian extension), times scale.
template <int N, int W, int THREADS>
__global__ void __launch_bounds__(THREADS) k_c2r_z(const float2* __restrict__ spec, long long comp_stride,
                                                   float* __restrict__ out0, float* __restrict__ out1,
                                                   float* __restrict__ out2, float scale, int rows,
                                                   const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int LD = line_ld<N>();
  constexpr int NH = N / 2 + 1;
  const float2* sp = spec + (long long)blockIdx.z * comp_stride;
  float* out = blockIdx.z == 0 ? out0 : (blockIdx.z == 1 ? out1 : out2);
  const int row0 = blockIdx.x * W;
  const int valid = min(W, rows - row0);
  for (int q = threadIdx.x; q < NH * W; q += THREADS) {
    const int l = q / NH, t = q % NH;
    if (l < valid) {
      const float2 v = sp[(size_t)(row0 + l) * NH + t];
      sm[l * LD + t] = v;
      if (t > 0 && t < N / 2) sm[l * LD + (N - t)] = make_float2(v.x, -v.y);
    }
  }
  __syncthreads();
  fft_lines<N, W, THREADS, true>(sm, tw);
  for (int q = threadIdx.x; q < N * W; q += THREADS) {
    const int l = q / N, t = q % N;
    if (l < valid) out[(size_t)(row0 + l) * N + t] = __fmul_rn(sm[l * LD + t].x, scale);
  }
}

// x pass of the Poisson solve: forward c2c along x of W kz-columns at fixed ky, the Green's
// function of poisson.rs:52-74, then per component the factor -i k_a and the inverse c2c along x.
// blockIdx.x = iy, blockIdx.y = kz tile. spec_in: forward half spectrum after the y pass.
// spec_out: 3 half spectra (component stride comp_stride).
template <int N, int W, int THREADS>
__global__ void __launch_bounds__(THREADS) k_poisson_x(const float2* __restrict__ spec_in, float2* spec_out,
                                                       long long comp_stride, TileGeo g, PoissonParams pp,
                                                       const float* __restrict__ deconv,
                                                       const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int LD = line_ld<N>();
  float2* phi = sm;
  float2* work = sm + W * LD;
  const int valid = min(W, g.lines - (int)blockIdx.y * W);
  load_tile<N, W, THREADS>(phi, spec_in, g, valid);
  __syncthreads();
  fft_lines<N, W, THREADS, false>(phi, tw);

  const int iy = blockIdx.x;
  const int z0 = blockIdx.y * W;
  const float ky = wavenumber(iy, N, pp.two_pi_over_l);
  // phi_k = delta_k * (-prefactor / k^2 * exp(-k^2 r_s^2)), k = 0 skipped (left zero).
  for (int q = threadIdx.x; q < N * W; q += THREADS) {
    const int l = q / N, t = q % N;
    if (l >= valid) continue;
    const float kx = wavenumber(t, N, pp.two_pi_over_l);
    const float kz = wavenumber(z0 + l, N, pp.two_pi_over_l);
    float k2 = -0.0f;
    k2 = __fadd_rn(k2, __fmul_rn(kx, kx));
    k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
    k2 = __fadd_rn(k2, __fmul_rn(kz, kz));
    float2 v = phi[l * LD + t];
    if (k2 == 0.0f) {
      v = make_float2(0.0f, 0.0f);
    } else {
      const float filter = expf(__fmul_rn(__fmul_rn(-k2, pp.r_split), pp.r_split));
      float sc = __fmul_rn(__fdiv_rn(-pp.prefactor, k2), filter);
      if (deconv) sc = __fmul_rn(sc, __fmul_rn(__fmul_rn(deconv[t], deconv[iy]), deconv[z0 + l]));
      v = make_float2(__fmul_rn(v.x, sc), __fmul_rn(v.y, sc));
    }
    phi[l * LD + t] = v;
  }
  __syncthreads();
  for (int comp = 0; comp < 3; ++comp) {
    // g_k = phi_k * (0 - i k_a): re = phi.re*0 - phi.im*(-k_a), im = phi.re*(-k_a) + phi.im*0
    for (int q = threadIdx.x; q < N * W; q += THREADS) {
      const int l = q / N, t = q % N;
      if (l >= valid) continue;
      float ka;
      if (comp == 0) ka = wavenumber(t, N, pp.two_pi_over_l);
      else if (comp == 1) ka = ky;
      else ka = wavenumber(z0 + l, N, pp.two_pi_over_l);
      const float2 p = phi[l * LD + t];
      const float nk = -ka;
      work[l * LD + t] = make_float2(__fsub_rn(__fmul_rn(p.x, 0.0f), __fmul_rn(p.y, nk)),
                                     __fadd_rn(__fmul_rn(p.x, nk), __fmul_rn(p.y, 0.0f)));
    }
    __syncthreads();
    fft_lines<N, W, THREADS, true>(work, tw);
    store_tile<N, W, THREADS>(work, spec_out + (long long)comp * comp_stride, g, valid);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
bool fft_supported(int n) { return n >= 4 && n <= 1024 && (n & (n - 1)) == 0; }

cudaError_t fft_plan_init(FftPlan& p, int n) {
  if (p.n == n && p.twiddle.p) return cudaSuccess;
  p.n = n;
  std::vector<float2> tw(n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < n; ++m) {
    const double a = -two_pi * (double)m / (double)n;
    tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  cudaError_t e = ensure(p.twiddle, n * sizeof(float2));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(p.twiddle.p, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
}

void fft_plan_free(FftPlan& p) {
  release(p.twiddle);
  p.n = 0;
}

constexpr int FFT_THREADS = 256;
constexpr int W_COL = 16;  // columns per tile for y/x passes
constexpr int W_ROW = 8;   // rows per tile for z passes
constexpr int W_PX = 8;    // columns per tile for the fused Poisson x pass

template <typename K>
static void set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N>
static void c2c_pass(float2* data, long long comp_stride, int ncomp, TileGeo g, int outer, int inverse,
                     const float2* tw, cudaStream_t s) {
  const size_t smem = (size_t)W_COL * line_ld<N>() * sizeof(float2);
  dim3 grid(outer, (g.lines + W_COL - 1) / W_COL, ncomp);
  if (inverse) {
    auto k = k_fft_pass<N, W_COL, FFT_THREADS, true>;
    set_smem(k, smem);
    count_launch();
    k<<<grid, FFT_THREADS, smem, s>>>(data, comp_stride, g, tw);
  } else {
    auto k = k_fft_pass<N, W_COL, FFT_THREADS, false>;
    set_smem(k, smem);
    count_launch();
    k<<<grid, FFT_THREADS, smem, s>>>(data, comp_stride, g, tw);
  }
}

template <int N>
static void fft3_c2c_n(float2* data, int inverse, const float2* tw, cudaStream_t s) {
  const long long n = N;
  // z lines: contiguous rows; tile = W_COL rows of one x-plane
  c2c_pass<N>(data, 0, 1, TileGeo{n * n, n, 1, N}, N, inverse, tw, s);
  // y lines: elements n apart, columns along z adjacent
  c2c_pass<N>(data, 0, 1, TileGeo{n * n, 1, n, N}, N, inverse, tw, s);
  // x lines: elements n*n apart; outer index = y
  c2c_pass<N>(data, 0, 1, TileGeo{n, 1, n * n, N}, N, inverse, tw, s);
}

void launch_fft3_c2c(const FftPlan& p, float2* data, int inverse, cudaStream_t s) {
  const float2* tw = static_cast<const float2*>(p.twiddle.p);
  switch (p.n) {
    case 4: fft3_c2c_n<4>(data, inverse, tw, s); break;
    case 8: fft3_c2c_n<8>(data, inverse, tw, s); break;
    case 16: fft3_c2c_n<16>(data, inverse, tw, s); break;
    case 32: fft3_c2c_n<32>(data, inverse, tw, s); break;
    case 64: fft3_c2c_n<64>(data, inverse, tw, s); break;
    case 128: fft3_c2c_n<128>(data, inverse, tw, s); break;
    case 256: fft3_c2c_n<256>(data, inverse, tw, s); break;
    case 512: fft3_c2c_n<512>(data, inverse, tw, s); break;
    case 1024: fft3_c2c_n<1024>(data, inverse, tw, s); break;
    default: break;
  }
}

template <int N>
static void poisson_n(const FftPlan& p, const PoissonParams& pp, const float* delta, const unsigned long long* fx,
                      int fx_shift, float mean, float2* spec, float* gx, float* gy, float* gz,
                      const float* deconv, cudaStream_t s) {
  const float2* tw = static_cast<const float2*>(p.twiddle.p);
  constexpr int NH = N / 2 + 1;
  const long long n = N;
  const long long comp = n * n * NH;  // elements per half spectrum
  const int rows = N * N;
  // Slot 0 holds the forward spectrum; the x pass reads each tile of it before writing the
  // same tile of slots 0..2, and tiles are disjoint, so the update in place is safe.
  float2* s0 = spec;
  // 1. z: R2C into slot 0
  {
    const size_t smem = (size_t)W_ROW * line_ld<N>() * sizeof(float2);
    auto k = k_r2c_z<N, W_ROW, FFT_THREADS>;
    set_smem(k, smem);
    count_launch();
    k<<<(rows + W_ROW - 1) / W_ROW, FFT_THREADS, smem, s>>>(delta, fx, std::ldexp(1.0f, -fx_shift), mean, s0, rows,
                                                            tw);
  }
  // 2. y forward on slot 0: lines along y (stride NH), columns along kz adjacent, outer = x
  c2c_pass<N>(s0, 0, 1, TileGeo{n * NH, 1, NH, NH}, N, 0, tw, s);
  // 3. x forward + Green + gradient + x inverse -> slots 0..2; outer = y
  {
    const size_t smem = (size_t)2 * W_PX * line_ld<N>() * sizeof(float2);
    auto k = k_poisson_x<N, W_PX, FFT_THREADS>;
    set_smem(k, smem);
    dim3 grid(N, (NH + W_PX - 1) / W_PX, 1);
    count_launch();
    k<<<grid, FFT_THREADS, smem, s>>>(s0, spec, comp, TileGeo{NH, 1, n * NH, NH}, pp, deconv, tw);
  }
  // 4. y inverse on the three component spectra
  c2c_pass<N>(spec, comp, 3, TileGeo{n * NH, 1, NH, NH}, N, 1, tw, s);
  // 5. z: C2R with 1/n^3
  {
    const size_t smem = (size_t)W_ROW * line_ld<N>() * sizeof(float2);
    auto k = k_c2r_z<N, W_ROW, FFT_THREADS>;
    set_smem(k, smem);
    dim3 grid((rows + W_ROW - 1) / W_ROW, 1, 3);
    count_launch();
    k<<<grid, FFT_THREADS, smem, s>>>(spec, comp, gx, gy, gz, pp.scale, rows, tw);
  }
}

void launch_poisson(const FftPlan& p, const PoissonParams& pp, const float* delta, const unsigned long long* fx,
                    int fx_shift, float mean, float2* spec, float* gx, float* gy, float* gz, cudaStream_t s) {
  const float* deconv = nullptr;
  switch (p.n) {
    case 4: poisson_n<4>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 8: poisson_n<8>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 16: poisson_n<16>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 32: poisson_n<32>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 64: poisson_n<64>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 128: poisson_n<128>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 256: poisson_n<256>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 512: poisson_n<512>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    case 1024: poisson_n<1024>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, deconv, s); break;
    default: break;
  }
}

}  // namespace cpm
