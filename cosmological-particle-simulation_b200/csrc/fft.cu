// fft.cu — shared-memory Stockham FFTs and the PM Poisson solve (fft.rs:40-95, poisson.rs:33-88).
//
// Layouts in HBM
//   real mesh      f32  [n][n][n]            (ix*n + iy)*n + iz, z fastest (mesh.rs:11)
//   half spectrum  c32  [n][n][n/2+2]        kz in [0, n/2]; one padding column keeps rows 16-byte
//                                            aligned; the rest of kz follows from Hermitian symmetry
//
// Every pass moves tiles of W = 16 lines between HBM and shared memory once. In shared memory
// element t of line l sits at t*(W+1) + l ("transposed", line index fastest):
//   - FFT stages give the line index to consecutive lanes, so each half-warp touches 16
//     consecutive elements (one 128-byte row) whatever the stage's stride: no bank conflicts;
//   - transfers of contiguous z rows give t to consecutive lanes; the odd stride W+1 spreads those
//     16 elements over all banks, again without conflicts;
//   - transfers of strided y/x lines give the line (the contiguous kz column) to consecutive
//     lanes, so global accesses are 128-byte rows.
// Each pass is a persistent kernel that walks its tiles with two shared-memory buffers: while one
// tile is transformed, the next one streams in with cp.async, so HBM stays busy during the
// shared-memory work. Lines are transformed by radix-8/4/2 Stockham stages in place (each stage
// reads its butterflies into registers, synchronises, writes them to their autosorted positions).
// Twiddles come from a table exp(-2 pi i m / n) built in double precision on the host.
//
// Real z lines use the half-length complex transform: z[m] = x[2m] + i x[2m+1] is transformed
// with n/2 points and split into the n/2+1 outputs with the twiddles of length n (and the
// reverse for C2R), which halves the arithmetic and shared memory of the z passes.
//
// The Poisson solve runs as
//   1. z pass: R2C of each z row; the input is the f32 delta or the u64 fixed-point mass mesh,
//      converted on load to delta = c/mean - 1 (integrator.rs:117-126);
//   2. y pass: forward c2c along y;
//   3. x pass: forward c2c along x, the Green's function of poisson.rs:52-74 in the reference's f32
//      operation order (optionally divided by the CIC window squared), then two inverse x
//      transforms: of -i k_x phi (x component) and of phi — two half spectra written;
//   4. y pass: inverse c2c along y of the x component; and, reading the x-transformed phi once,
//      of -i k_y phi and -i k_z phi (k_y and k_z are constant along an x line, so the factors
//      commute with the x transform), written as the y and z components;
//   5. z pass: C2R of each row, scaled by 1/n^3 (poisson.rs:77-87), into three f32 meshes.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cpm_internal.cuh"

namespace cpm {

constexpr int TW = 16;       // lines per tile
constexpr int TLD = TW + 1;  // shared-memory row pitch (elements)
constexpr size_t SMEM_LIMIT = 227 * 1024;

template <int L, int MR = 8>
constexpr int threads_for();

// ---------------------------------------------------------------------------------------------
// Complex helpers and small DFTs
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
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

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
  // y1,2 = x0 - (x1 + x2)/2 -/+ i (sqrt(3)/2)(x1 - x2) (signs of i flipped for the inverse)
  const float h = 0.86602540378443864676f;
  const float2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
  const float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
  const float2 r = rot90<INV>(make_float2(h * t2.x, h * t2.y));
  v[0] = cadd(v[0], t1);
  v[1] = cadd(m, r);
  v[2] = csub(m, r);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2* v) {
  // t1 = x1 + x4, t2 = x2 + x3, t3 = x1 - x4, t4 = x2 - x3;
  // y1,4 = x0 + c1 t1 + c2 t2 -/+ i (s1 t3 + s2 t4), y2,3 = x0 + c2 t1 + c1 t2 -/+ i (s2 t3 - s1 t4)
  const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
  const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
  const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  const float2 m1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  const float2 m2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  const float2 n1 = rot90<INV>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
  const float2 n2 = rot90<INV>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
  v[0] = cadd(v[0], cadd(t1, t2));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 3) dft3<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 5) dft5<INV>(v);
  else dft8<INV>(v);
}

// One Stockham stage of radix R on the TW lines of a tile (element t of line l at t*TLD + l),
// T threads. Twiddle exp(-2 pi i m / N) is tw[m * TS] (TS = 2 when the table is for length 2N).
// NT = 2 transforms a second tile (sm1) in the same stage: one pair of barriers and one set of
// twiddle loads serve both.
template <int N, int R, int NS, bool INV, int T, int TS, int NT = 1>
__device__ __forceinline__ void stockham_stage(float2* sm0, float2* sm1, const float2* __restrict__ tw) {
  constexpr int NB = N / R;
  constexpr int TOTAL = TW * NB;
  constexpr int BPT = (TOTAL + T - 1) / T;
  float2 v[NT][BPT][R];
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * T;
    if (TOTAL % T == 0 || b < TOTAL) {
      const int l = b % TW, j = b / TW;
#pragma unroll
      for (int p = 0; p < NT; ++p) {
        const float2* sm = p ? sm1 : sm0;
#pragma unroll
        for (int r = 0; r < R; ++r) v[p][q][r] = sm[(j + r * NB) * TLD + l];
      }
      if constexpr (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = __ldg(tw + r * k * (N / (NS * R)) * TS);
          if (INV) w.y = -w.y;
#pragma unroll
          for (int p = 0; p < NT; ++p) v[p][q][r] = cmul(v[p][q][r], w);
        }
      }
#pragma unroll
      for (int p = 0; p < NT; ++p) dft<R, INV>(v[p][q]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int b = threadIdx.x + q * T;
    if (TOTAL % T == 0 || b < TOTAL) {
      const int l = b % TW, j = b / TW;
      const int k = j % NS;
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int p = 0; p < NT; ++p) {
        float2* sm = p ? sm1 : sm0;
#pragma unroll
        for (int r = 0; r < R; ++r) sm[(base + r * NS) * TLD + l] = v[p][q][r];
      }
    }
  }
  __syncthreads();
}

// Radix of the next Stockham stage for a remaining length L = 2^a 3^b 5^c under a plan whose
// largest radix is MR: MR = 8 takes 8 while it divides, then 4 or 2, then 3s, then 5s (512 = 8.8.8);
// MR = 4 takes 4 while it divides, then 2, 3s, 5s (512 = 4.4.4.4.2). The autotuner picks the plan.
template <int L, int MR>
constexpr int next_radix() {
  if constexpr (MR >= 8)
    return L % 8 == 0 ? 8 : (L % 4 == 0 ? 4 : (L % 2 == 0 ? 2 : (L % 3 == 0 ? 3 : 5)));
  else
    return L % 4 == 0 ? 4 : (L % 2 == 0 ? 2 : (L % 3 == 0 ? 3 : 5));
}
constexpr bool smooth235(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  while (n % 5 == 0) n /= 5;
  return n == 1;
}

template <int N, int NS, bool INV, int T, int TS, int MR, int NT = 1>
__device__ __forceinline__ void fft_stages(float2* sm0, float2* sm1, const float2* __restrict__ tw) {
  if constexpr (NS < N) {
    constexpr int R = next_radix<N / NS, MR>();
    stockham_stage<N, R, NS, INV, T, TS, NT>(sm0, sm1, tw);
    fft_stages<N, NS * R, INV, T, TS, MR, NT>(sm0, sm1, tw);
  }
}

// ---------------------------------------------------------------------------------------------
// Warp-per-line plan (MR = 0) for N = 256 and 512: warp w transforms line w of the tile by itself,
// with three register stages of radix R1, R2, R3 (N = R1 R2 R3; 8.8.8 and 4.8.8) and two exchanges
// through the line's own shared-memory elements, synchronised with __syncwarp only. With
// n = s + S1 r (S1 = N / R1), s = sa + R3 sb, k = k1 + R1 (k2 + R2 k3):
//   A: Y[s][k1]   = w_N^(s k1)     sum_r  x[s + S1 r] w_R1^(r k1)        stored at s + S1 k1
//   B: Z[sa][k2]  = w_S1^(sa k2)   sum_sb Y[sa + R3 sb][k1] w_R2^(sb k2)  stored at sa + R3 k2 + S1 k1
//   C: X[k]       =                sum_sa Z[sa][k2] w_R3^(sa k3)         stored at k (natural order)
// Element t of the line sits in bank pair (t + l) mod 16 (pitch TW + 1 = 17 float2), so an access is
// conflict-free when the 16 lanes of each half-warp hold distinct t mod 16. The lanes of stages B
// and C take their inputs in an order rotated per lane so that this holds (B: by k1 mod 2; C: by
// k1 + 4 ((k2 / 2) mod 2), mod 8), and put the values back in place with register selects.
template <int N>
struct WarpPlan {
  static constexpr bool ok = false;
};
template <>
struct WarpPlan<512> {
  static constexpr bool ok = true;
  static constexpr int R1 = 8, R2 = 8, R3 = 8;
};
template <>
struct WarpPlan<256> {
  static constexpr bool ok = true;
  static constexpr int R1 = 4, R2 = 8, R3 = 8;
};

// Threads of a CTA that transforms TW lines of length L: one warp per line for the warp plan, else
// about one radix-8 butterfly each, a multiple of 32 in 256..1024.
template <int L, int MR>
constexpr int threads_for() {
  if constexpr (MR == 0 && WarpPlan<L>::ok) {
    return 32 * TW;
  } else {
    constexpr int t = (TW * L / 8 + 31) / 32 * 32;
    return t < 256 ? 256 : (t > 1024 ? 1024 : t);
  }
}

template <bool INV>
__device__ __forceinline__ float2 twiddle(const float2* __restrict__ tw, int idx) {
  float2 w = __ldg(tw + idx);
  if (INV) w.y = -w.y;
  return w;
}

// v[j] = u[(j - k) mod R] when `on` (a rotation of the array by k places), else unchanged
template <int R, int K>
__device__ __forceinline__ void rotate_if(float2 (&v)[R], bool on) {
  float2 u[R];
#pragma unroll
  for (int j = 0; j < R; ++j) u[j] = v[j];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const float2 a = u[(j - K + R) % R];
    v[j].x = on ? a.x : u[j].x;
    v[j].y = on ? a.y : u[j].y;
  }
}

template <int N, bool INV, int TS>
__device__ __forceinline__ void warp_fft_line(float2* sm, int l, const float2* __restrict__ tw) {
  using P = WarpPlan<N>;
  constexpr int R1 = P::R1, R2 = P::R2, R3 = P::R3, S1 = N / R1;
  static_assert(R2 == 8 && R3 == 8 && S1 == 64, "plans with S1 = 64 = 8 x 8");
  const int lane = threadIdx.x & 31;
  float2* line = sm + l;
  // A: columns s = lane + 32 q
  {
    constexpr int QA = S1 / 32;
    float2 v[QA][R1];
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int s = lane + 32 * q;
#pragma unroll
      for (int r = 0; r < R1; ++r) v[q][r] = line[(s + S1 * r) * TLD];
      dft<R1, INV>(v[q]);
#pragma unroll
      for (int k1 = 1; k1 < R1; ++k1) v[q][k1] = cmul(v[q][k1], twiddle<INV>(tw, s * k1 * TS));
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int s = lane + 32 * q;
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) line[(s + S1 * k1) * TLD] = v[q][k1];
    }
    __syncwarp();
  }
  // B: pairs p = lane + 32 q -> (sa = p % R3, k1 = p / R3); lanes with odd k1 rotate sb by one
  {
    constexpr int QB = R3 * R1 / 32;
    float2 v[QB][R2];
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int p = lane + 32 * q, sa = p % R3, k1 = p / R3, rho = k1 & 1;
#pragma unroll
      for (int i = 0; i < R2; ++i) v[q][i] = line[(sa + R3 * ((i + rho) % R2) + S1 * k1) * TLD];
      rotate_if<R2, 1>(v[q], rho);  // v[sb]
      dft<R2, INV>(v[q]);
#pragma unroll
      for (int k2 = 1; k2 < R2; ++k2) v[q][k2] = cmul(v[q][k2], twiddle<INV>(tw, R1 * sa * k2 * TS));
      rotate_if<R2, R2 - 1>(v[q], rho);  // v[i] = Z[(i + rho) % R2]
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int p = lane + 32 * q, sa = p % R3, k1 = p / R3, rho = k1 & 1;
#pragma unroll
      for (int i = 0; i < R2; ++i) line[(sa + R3 * ((i + rho) % R2) + S1 * k1) * TLD] = v[q][i];
    }
    __syncwarp();
  }
  // C: pairs p = lane + 32 q -> (k1 = p % R1, k2 = p / R1); lane rotation rho of sa
  {
    constexpr int QC = R1 * R2 / 32;
    float2 v[QC][R3];
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const int p = lane + 32 * q, k1 = p % R1, k2 = p / R1, rho = (k1 + 4 * ((k2 >> 1) & 1)) & 7;
#pragma unroll
      for (int i = 0; i < R3; ++i) v[q][i] = line[(((i + rho) & 7) + R3 * k2 + S1 * k1) * TLD];
      rotate_if<R3, 1>(v[q], rho & 1);
      rotate_if<R3, 2>(v[q], rho & 2);
      rotate_if<R3, 4>(v[q], rho & 4);  // v[sa]
      dft<R3, INV>(v[q]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const int p = lane + 32 * q, k1 = p % R1, k2 = p / R1;
#pragma unroll
      for (int k3 = 0; k3 < R3; ++k3) line[(k1 + R1 * k2 + R1 * R2 * k3) * TLD] = v[q][k3];
    }
  }
}

// Full length-N transform of the tile (N = 2^a 3^b 5^c) with the radix plan MR (MR = 0: the
// warp-per-line plan where it exists, else the radix-8 Stockham plan).
template <int N, bool INV, int T, int TS = 1, int MR = 8>
__device__ __forceinline__ void fft_lines(float2* sm, const float2* __restrict__ tw) {
  static_assert(N >= 2 && N <= 1024 && smooth235(N), "lengths 2..1024 with prime factors 2, 3, 5");
  if constexpr (MR == 0 && WarpPlan<N>::ok) {
    static_assert(T == 32 * TW, "one warp per line");
    warp_fft_line<N, INV, TS>(sm, threadIdx.x >> 5, tw);
    __syncthreads();
  } else {
    fft_stages<N, 1, INV, T, TS, (MR == 0 ? 8 : MR)>(sm, sm, tw);
  }
}

// Two independent tiles transformed together (the same length and direction).
template <int N, bool INV, int T, int TS = 1, int MR = 8>
__device__ __forceinline__ void fft_lines2(float2* a, float2* b, const float2* __restrict__ tw) {
  if constexpr (MR == 0 && WarpPlan<N>::ok) {
    static_assert(T == 32 * TW, "one warp per line");
    warp_fft_line<N, INV, TS>(a, threadIdx.x >> 5, tw);
    warp_fft_line<N, INV, TS>(b, threadIdx.x >> 5, tw);
    __syncthreads();
  } else {
    fft_stages<N, 1, INV, T, TS, (MR == 0 ? 8 : MR), 2>(a, b, tw);
  }
}

// ---------------------------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, completion tracked per thread by groups)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// ---------------------------------------------------------------------------------------------
// Tile geometry. Strided passes: element t of column c of tile (o, ct) is at
//   o * outer_stride + (ct * TW + c) + t * elem_stride   (columns contiguous in memory).
// Row passes: tile r covers rows r*TW .. r*TW + TW - 1, each contiguous.
// ---------------------------------------------------------------------------------------------
struct ColGeo {
  long long outer_stride;
  long long elem_stride;
  int cols;       // valid columns along the contiguous axis
  int col_tiles;  // ceil(cols / TW)
  int outer;      // number of outer indices (over every box of a batch)
  int per_box = 0;            // outer indices per box when a batch's boxes are not one linear run
  long long box_stride = 0;   // elements between the boxes of such a batch
  __host__ __device__ long long offset(int o) const {
    return per_box ? (long long)(o / per_box) * box_stride + (long long)(o % per_box) * outer_stride
                   : (long long)o * outer_stride;
  }
  __host__ __device__ int in_box(int o) const { return per_box ? o % per_box : o; }
};

// Row transfers: chunks of TT = min(L, 16) consecutive t go to consecutive lanes, chunk-major
// over the TW rows: work item q -> (t, l) with t < L, l < TW.
template <int L>
__device__ __forceinline__ int row_t(int q) {
  constexpr int TT = L < 16 ? L : 16;
  return (q % TT) + TT * (q / (TT * TW));
}
template <int L>
__device__ __forceinline__ int row_l(int q) {
  constexpr int TT = L < 16 ? L : 16;
  return (q / TT) % TW;
}
// Work items that cover t < count on every row.
template <int L>
__device__ __forceinline__ int row_span(int count) {
  constexpr int TT = L < 16 ? L : 16;
  return TT * TW * ((count + TT - 1) / TT);
}

// Column transfers: thread tid moves column l = tid % TW of rows t = tid / TW, tid / TW + T / TW, ...;
// its global address advances by a fixed (T / TW) rows per step (T is a multiple of TW).
template <int N, int T>
__device__ __forceinline__ void async_load_cols(float2* buf, const float2* src, long long base, long long es,
                                                int valid) {
  static_assert(T % TW == 0, "whole rows per step");
  constexpr int RS = T / TW;
  const int l = threadIdx.x % TW;
  if (l >= valid) return;
  const float2* g = src + base + l + (long long)(threadIdx.x / TW) * es;
  const long long step = (long long)RS * es;
#pragma unroll 2
  for (int t = threadIdx.x / TW; t < N; t += RS, g += step) cp_async8(buf + t * TLD + l, g);
}

template <int N, int T>
__device__ __forceinline__ void store_cols(const float2* buf, float2* dst, long long base, long long es, int valid) {
  static_assert(T % TW == 0, "whole rows per step");
  constexpr int RS = T / TW;
  const int l = threadIdx.x % TW;
  if (l >= valid) return;
  float2* g = dst + base + l + (long long)(threadIdx.x / TW) * es;
  const long long step = (long long)RS * es;
#pragma unroll 2
  for (int t = threadIdx.x / TW; t < N; t += RS, g += step) *g = buf[t * TLD + l];
}

// Persistent pipeline: each CTA walks tiles blockIdx.x, +gridDim.x, ...; with NBUF = 2 the next
// tile's copies are in flight while the current one is processed. `tile_elems` is the size of one
// buffer in float2 units.
template <int NBUF, typename Load, typename Work>
__device__ __forceinline__ void pipeline(float2* smem, int tile_elems, int total, Load load, Work work) {
  int k = 0;
  int tile = blockIdx.x;
  if (tile < total) load(smem, tile);
  cp_async_commit();
  for (; tile < total; tile += gridDim.x, ++k) {
    const int next = tile + gridDim.x;
    float2* cur = smem + (NBUF == 2 ? (k & 1) * tile_elems : 0);
    if constexpr (NBUF == 2) {
      if (next < total) load(smem + ((k + 1) & 1) * tile_elems, next);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    work(cur, tile);
    __syncthreads();
    if constexpr (NBUF == 1) {
      if (next < total) load(cur, next);
      cp_async_commit();
    }
  }
  cp_async_wait<0>();
}

// c2c pass over a strided axis; tile -> (comp, outer, column tile).
template <int N, bool INV, int NBUF, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_fft_cols(float2* data, long long comp_stride, ColGeo g, int ncomp,
                                                const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int per_comp = g.outer * g.col_tiles;
  auto locate = [&](int tile, long long& base, int& valid, float2*& d) {
    const int comp = tile / per_comp, rest = tile % per_comp;
    const int o = rest / g.col_tiles, ct = rest % g.col_tiles;
    d = data + (long long)comp * comp_stride;
    base = g.offset(o) + (long long)ct * TW;
    valid = min(TW, g.cols - ct * TW);
  };
  pipeline<NBUF>(
      smem, N * TLD, ncomp * per_comp,
      [&](float2* buf, int tile) {
        long long base;
        int valid;
        float2* d;
        locate(tile, base, valid, d);
        async_load_cols<N, T>(buf, d, base, g.elem_stride, valid);
      },
      [&](float2* cur, int tile) {
        long long base;
        int valid;
        float2* d;
        locate(tile, base, valid, d);
        fft_lines<N, INV, T, 1, MR>(cur, tw);
        store_cols<N, T>(cur, d, base, g.elem_stride, valid);
      });
}

// c2c pass over contiguous rows (the z lines of a full complex n^3 array).
template <int N, bool INV, int NBUF, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_fft_rows(float2* data, int rows, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  pipeline<NBUF>(
      smem, N * TLD, (rows + TW - 1) / TW,
      [&](float2* buf, int tile) {
        const int row0 = tile * TW, valid = min(TW, rows - row0);
        for (int q = threadIdx.x; q < row_span<N>(N); q += T) {
          const int t = row_t<N>(q), l = row_l<N>(q);
          if (l < valid && t < N) cp_async8(buf + t * TLD + l, data + (size_t)(row0 + l) * N + t);
        }
      },
      [&](float2* cur, int tile) {
        const int row0 = tile * TW, valid = min(TW, rows - row0);
        fft_lines<N, INV, T, 1, MR>(cur, tw);
#pragma unroll 4
        for (int q = threadIdx.x; q < row_span<N>(N); q += T) {
          const int t = row_t<N>(q), l = row_l<N>(q);
          if (l < valid && t < N) data[(size_t)(row0 + l) * N + t] = cur[t * TLD + l];
        }
      });
}

// z pass, forward: TW real rows of length N -> N/2+1 complex each (rows of the padded half
// spectrum), as an N/2-point complex transform of z[m] = x[2m] + i x[2m+1]. Input: f32 delta, or
// the u64 fixed-point mass mesh (c = fx * 2^-k in f32, delta = c / mean - 1). Each thread loads its
// input pairs straight into registers (16-byte loads of two u64 cells, all of a tile's loads issued
// before any is used), converts them and writes the complex tile: shared memory holds only that
// tile, so several CTAs per SM keep the loads of their tiles in flight.
template <int N, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_r2c_z(const float* __restrict__ delta,
                                             const unsigned long long* __restrict__ fx, float inv_scale, float mean,
                                             float2* __restrict__ spec, int rows, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  constexpr int M = N / 2, NH = N / 2 + 1, NHP = N / 2 + 2;
  constexpr int SPAN = TW * ((M + 15) / 16) * 16;  // row_span<M>(M)
  constexpr int PER = (SPAN + T - 1) / T;
  float2* cplx = smem;
  const int tiles = (rows + TW - 1) / TW;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int row0 = tile * TW, valid = min(TW, rows - row0);
    float2 v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int q = threadIdx.x + k * T;
      const int m = row_t<M>(q), l = row_l<M>(q);
      v[k] = make_float2(0.0f, 0.0f);
      if (q < SPAN && l < valid && m < M) {
        const size_t gi = (size_t)(row0 + l) * N + 2 * m;
        if (fx) {
          const ulonglong2 u = __ldg(reinterpret_cast<const ulonglong2*>(fx + gi));
          const float c0 = __fmul_rn(__ull2float_rn(u.x), inv_scale);
          const float c1 = __fmul_rn(__ull2float_rn(u.y), inv_scale);
          v[k] = make_float2(__fsub_rn(__fdiv_rn(c0, mean), 1.0f), __fsub_rn(__fdiv_rn(c1, mean), 1.0f));
        } else {
          v[k] = __ldg(reinterpret_cast<const float2*>(delta + gi));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int q = threadIdx.x + k * T;
      const int m = row_t<M>(q), l = row_l<M>(q);
      if (q < SPAN && m < M) cplx[m * TLD + l] = v[k];
    }
    __syncthreads();
    fft_lines<M, false, T, 2, MR>(cplx, tw);
    // X[k] = (Z[k] + conj(Z[M-k]))/2 + w^k (Z[k] - conj(Z[M-k]))/(2i), w = exp(-2 pi i / N)
    for (int q = threadIdx.x; q < row_span<M>(NH); q += T) {
      const int k = row_t<M>(q), l = row_l<M>(q);
      if (l >= valid || k >= NH) continue;
      // Z is M-periodic: Z[M] = Z[0] (k runs over 0..M)
      const float2 zk = cplx[(k == M ? 0 : k) * TLD + l];
      const float2 zm = cplx[(k == 0 ? 0 : M - k) * TLD + l];
      const float2 fe = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      const float2 fo = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      spec[(size_t)(row0 + l) * NHP + k] = cadd(fe, cmul(__ldg(tw + k), fo));
    }
    __syncthreads();  // the next tile overwrites the complex tile
  }
}

// z pass, inverse: N/2+1 complex per row -> N real values times scale, as an N/2-point complex
// inverse transform of Z'[k] = (X[k] + conj(X[M-k])) + i (X[k] - conj(X[M-k])) conj(w^k), whose
// output is x[2m] + i x[2m+1]. tile -> (comp, row tile). Shared memory: NBUF tiles of (M+1)*TLD.
template <int N, int NBUF, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_c2r_z(const float2* __restrict__ spec, long long comp_stride,
                                             float* __restrict__ out0, float* __restrict__ out1,
                                             float* __restrict__ out2, float scale, int rows,
                                             const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  constexpr int M = N / 2, NH = N / 2 + 1, NHP = N / 2 + 2;
  const int row_tiles = (rows + TW - 1) / TW;
  pipeline<NBUF>(
      smem, (M + 1) * TLD, 3 * row_tiles,
      [&](float2* buf, int tile) {
        const int comp = tile / row_tiles, row0 = (tile % row_tiles) * TW, valid = min(TW, rows - row0);
        const float2* sp = spec + (long long)comp * comp_stride;
        for (int q = threadIdx.x; q < row_span<M>(NH); q += T) {
          const int t = row_t<M>(q), l = row_l<M>(q);
          if (l < valid && t < NH) cp_async8(buf + t * TLD + l, sp + (size_t)(row0 + l) * NHP + t);
        }
      },
      [&](float2* cur, int tile) {
        const int comp = tile / row_tiles, row0 = (tile % row_tiles) * TW, valid = min(TW, rows - row0);
        float* out = comp == 0 ? out0 : (comp == 1 ? out1 : out2);
        for (int q = threadIdx.x; q < (M / 2 + 1) * TW; q += T) {
          const int l = q % TW, k = q / TW;
          float2 xk = cur[k * TLD + l], xm = cur[(M - k) * TLD + l];
          // X[0] and X[M] enter the real output through their real parts only (as in Re of a
          // full complex inverse); their imaginary parts are round-off of the Hermitian planes.
          if (k == 0) xk.y = xm.y = 0.0f;
          const float2 wk = __ldg(tw + k);
          // Z'[k] and, for 0 < k < M/2, Z'[M-k] (w^(M-k) = -conj(w^k))
          const float2 a = cadd(xk, conjf2(xm)), b = csub(xk, conjf2(xm));
          const float2 bw = cmul(b, conjf2(wk));
          cur[k * TLD + l] = make_float2(a.x - bw.y, a.y + bw.x);
          if (k > 0 && 2 * k < M) {
            const float2 a2 = cadd(xm, conjf2(xk)), b2 = csub(xm, conjf2(xk));
            const float2 bw2 = cmul(b2, make_float2(-wk.x, -wk.y));
            cur[(M - k) * TLD + l] = make_float2(a2.x - bw2.y, a2.y + bw2.x);
          }
        }
        __syncthreads();
        fft_lines<M, true, T, 2, MR>(cur, tw);
#pragma unroll 4
        for (int q = threadIdx.x; q < row_span<M>(M); q += T) {
          const int m = row_t<M>(q), l = row_l<M>(q);
          if (l < valid && m < M) {
            const float2 v = cur[m * TLD + l];
            reinterpret_cast<float2*>(out + (size_t)(row0 + l) * N)[m] =
                make_float2(__fmul_rn(v.x, scale), __fmul_rn(v.y, scale));
          }
        }
      });
}

// x pass of the Poisson solve for TW kz columns at fixed ky (tile -> (iy, column tile)): forward
// c2c along x, the Green's function of poisson.rs:52-74, then
//   x component: inverse x transform of -i k_x phi;
//   y, z components: -i k_y and -i k_z times the inverse x transform of phi (k_y, k_z constant
//   along the line, so the factor commutes with the transform), applied by k_grad_yz.
// The gradient factor is the reference's (phi * (0 - i k_a), poisson.rs:70); for y and z it
// multiplies the transformed phi instead, which differs only in round-off.
// Shared memory: NBUF input tiles, then one work tile for -i k_x phi.
template <int N, int NBUF, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_poisson_x(const float2* __restrict__ spec_in, float2* spec_out,
                                                 long long comp_stride, ColGeo g, PoissonParams pp,
                                                 const float* __restrict__ deconv, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  float2* gxb = smem + NBUF * N * TLD;
  pipeline<NBUF>(
      smem, N * TLD, g.outer * g.col_tiles,
      [&](float2* buf, int tile) {
        const int iy = tile / g.col_tiles, ct = tile % g.col_tiles;
        const long long base = g.offset(iy) + (long long)ct * TW;
        async_load_cols<N, T>(buf, spec_in, base, g.elem_stride, min(TW, g.cols - ct * TW));
      },
      [&](float2* phi, int tile) {
        const int iy = tile / g.col_tiles, ct = tile % g.col_tiles;
        const int valid = min(TW, g.cols - ct * TW);
        const long long base = g.offset(iy) + (long long)ct * TW;
        const int z0 = ct * TW;
        const float prefactor = pp.prefactor_dev ? *pp.prefactor_dev : pp.prefactor;
        fft_lines<N, false, T, 1, MR>(phi, tw);
        const float ky = wavenumber(g.in_box(iy), N, pp.two_pi_over_l);
        for (int q = threadIdx.x; q < N * TW; q += T) {
          const int l = q % TW, t = q / TW;
          const float kx = wavenumber(t, N, pp.two_pi_over_l);
          const float kz = wavenumber(min(z0 + l, N / 2), N, pp.two_pi_over_l);
          float k2 = -0.0f;
          k2 = __fadd_rn(k2, __fmul_rn(kx, kx));
          k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
          k2 = __fadd_rn(k2, __fmul_rn(kz, kz));
          float2 v = phi[t * TLD + l];
          if (k2 == 0.0f || l >= valid) {
            v = make_float2(0.0f, 0.0f);
          } else {
            // phi_k = delta_k * (-prefactor / k^2 * exp(-k^2 r_s^2)), k = 0 skipped (left zero)
            const float filter = expf(__fmul_rn(__fmul_rn(-k2, pp.r_split), pp.r_split));
            float sc = __fmul_rn(__fdiv_rn(-prefactor, k2), filter);
            if (deconv) sc = __fmul_rn(sc, __fmul_rn(__fmul_rn(deconv[t], deconv[g.in_box(iy)]), deconv[z0 + l]));
            v = make_float2(__fmul_rn(v.x, sc), __fmul_rn(v.y, sc));
          }
          phi[t * TLD + l] = v;
          // -i k_x phi: re = phi.re*0 - phi.im*(-k_x), im = phi.re*(-k_x) + phi.im*0
          const float nk = -kx;
          gxb[t * TLD + l] = make_float2(__fsub_rn(__fmul_rn(v.x, 0.0f), __fmul_rn(v.y, nk)),
                                         __fadd_rn(__fmul_rn(v.x, nk), __fmul_rn(v.y, 0.0f)));
        }
        __syncthreads();
        fft_lines2<N, true, T, 1, MR>(gxb, phi, tw);
        // -i k_x phi to slot 0; the x-transformed phi to slot 1, from which the y pass forms the
        // y and z components (k_y and k_z are constant along an x line)
        store_cols<N, T>(gxb, spec_out, base, g.elem_stride, valid);
        store_cols<N, T>(phi, spec_out + comp_stride, base, g.elem_stride, valid);
      });
}

// Inverse y pass of the y and z gradient components: reads the x-transformed potential of slot 1
// once, forms -i k_y phi and -i k_z phi (the f32 operations of k_green_grad) and writes their
// inverse y transforms to slots 1 and 2; tile -> (x, column tile), lines along y.
template <int N, int NBUF, int T, int MR = 8>
__global__ void __launch_bounds__(T) k_grad_yz(float2* spec, long long comp_stride, ColGeo g, PoissonParams pp,
                                               const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  float2* gzb = smem + NBUF * N * TLD;
  float2* phi_slot = spec + comp_stride;
  pipeline<NBUF>(
      smem, N * TLD, g.outer * g.col_tiles,
      [&](float2* buf, int tile) {
        const int o = tile / g.col_tiles, ct = tile % g.col_tiles;
        const long long base = g.offset(o) + (long long)ct * TW;
        async_load_cols<N, T>(buf, phi_slot, base, g.elem_stride, min(TW, g.cols - ct * TW));
      },
      [&](float2* cur, int tile) {
        const int o = tile / g.col_tiles, ct = tile % g.col_tiles;
        const int valid = min(TW, g.cols - ct * TW);
        const long long base = g.offset(o) + (long long)ct * TW;
        const int z0 = ct * TW;
        for (int q = threadIdx.x; q < N * TW; q += T) {
          const int l = q % TW, t = q / TW;
          const float2 p = cur[t * TLD + l];
          const float nky = -wavenumber(t, N, pp.two_pi_over_l);
          const float nkz = -wavenumber(z0 + l, N, pp.two_pi_over_l);
          cur[t * TLD + l] = make_float2(__fsub_rn(__fmul_rn(p.x, 0.0f), __fmul_rn(p.y, nky)),
                                         __fadd_rn(__fmul_rn(p.x, nky), __fmul_rn(p.y, 0.0f)));
          gzb[t * TLD + l] = make_float2(__fsub_rn(__fmul_rn(p.x, 0.0f), __fmul_rn(p.y, nkz)),
                                         __fadd_rn(__fmul_rn(p.x, nkz), __fmul_rn(p.y, 0.0f)));
        }
        __syncthreads();
        fft_lines2<N, true, T, 1, MR>(cur, gzb, tw);
        store_cols<N, T>(cur, phi_slot, base, g.elem_stride, valid);
        store_cols<N, T>(gzb, spec + 2 * comp_stride, base, g.elem_stride, valid);
      });
}

// Green's function and gradient of poisson.rs:52-74 applied elementwise to the half spectrum in
// slot 0, writing -i k_a phi to slots 0..2 (the same f32 operations as k_poisson_x). Used where
// the fused x pass does not fit in shared memory.
__global__ void k_green_grad(float2* spec, long long comp, int n, PoissonParams pp, const float* __restrict__ deconv) {
  const int nh = n / 2 + 1, nhp = n / 2 + 2;
  const long long total = (long long)n * n * nh;
  const float prefactor = pp.prefactor_dev ? *pp.prefactor_dev : pp.prefactor;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int kz = (int)(e % nh);
    const long long line = e / nh;
    const int iy = (int)(line % n), ix = (int)(line / n);
    const long long gi = line * nhp + kz;
    const float kx = wavenumber(ix, n, pp.two_pi_over_l), ky = wavenumber(iy, n, pp.two_pi_over_l);
    const float kzv = wavenumber(kz, n, pp.two_pi_over_l);
    float k2 = -0.0f;
    k2 = __fadd_rn(k2, __fmul_rn(kx, kx));
    k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
    k2 = __fadd_rn(k2, __fmul_rn(kzv, kzv));
    float2 v = spec[gi];
    if (k2 == 0.0f) {
      v = make_float2(0.0f, 0.0f);
    } else {
      const float filter = expf(__fmul_rn(__fmul_rn(-k2, pp.r_split), pp.r_split));
      float sc = __fmul_rn(__fdiv_rn(-prefactor, k2), filter);
      if (deconv) sc = __fmul_rn(sc, __fmul_rn(__fmul_rn(deconv[ix], deconv[iy]), deconv[kz]));
      v = make_float2(__fmul_rn(v.x, sc), __fmul_rn(v.y, sc));
    }
    const float nk[3] = {-kx, -ky, -kzv};
#pragma unroll
    for (int a = 0; a < 3; ++a)
      spec[a * comp + gi] = make_float2(__fsub_rn(__fmul_rn(v.x, 0.0f), __fmul_rn(v.y, nk[a])),
                                        __fadd_rn(__fmul_rn(v.x, nk[a]), __fmul_rn(v.y, 0.0f)));
  }
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
// Mesh sizes with compiled transforms: powers of two 4..1024 and the 2^a 3^b 5^c sizes below.
#define CPM_FFT_SIZES(X) \
  X(4) X(8) X(16) X(32) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(256) X(320) X(384) X(512) X(1024)

bool fft_supported(int n) {
  switch (n) {
#define CPM_CASE(N) case N:
    CPM_FFT_SIZES(CPM_CASE)
#undef CPM_CASE
    return true;
    default:
      return false;
  }
}
bool poisson_supported(int n) { return fft_supported(n); }

const char* fft_sizes_text() {
  return "4, 8, 16, 32, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512 or 1024";
}

size_t half_spectrum_elems(int n) { return (size_t)n * n * (size_t)(n / 2 + 2); }

cudaError_t fft_plan_init(FftPlan& p, int n) {
  if (p.n == n && p.twiddle.p && p.deconv.p) return cudaSuccess;
  p.n = n;
  std::vector<float2> tw(n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < n; ++m) {
    const double a = -two_pi * (double)m / (double)n;
    tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  // CIC deconvolution per axis: 1 / W(k)^2 with W = sinc^2(pi m / n) (deposit and gather)
  std::vector<float> dc(n);
  for (int i = 0; i < n; ++i) {
    const int m = i <= n / 2 ? i : i - n;
    const double x = 3.14159265358979323846 * (double)m / (double)n;
    const double s = m == 0 ? 1.0 : std::sin(x) / x;
    dc[i] = (float)(1.0 / (s * s * s * s));
  }
  cudaError_t e = ensure(p.twiddle, n * sizeof(float2));
  if (e == cudaSuccess) e = ensure(p.deconv, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(p.twiddle.p, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p.deconv.p, dc.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  return e;
}

void fft_plan_free(FftPlan& p) {
  release(p.twiddle);
  release(p.deconv);
  p.n = 0;
}

static int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// Persistent launch: as many CTAs as fit on all SMs at once, at most one per tile.
template <typename K, typename... Args>
static void launch_persistent(K kernel, int threads, size_t smem, int total, cudaStream_t s, Args... args) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int grid = std::max(1, std::min(total, per_sm * num_sms()));
  count_launch();
  kernel<<<grid, threads, smem, s>>>(args...);
}

constexpr size_t c_tile(int rows_of_tile) { return (size_t)rows_of_tile * TLD * sizeof(float2); }

template <int N, int MR = 8>
static void cols_pass(float2* data, long long comp_stride, int ncomp, ColGeo g, int inverse, const float2* tw,
                      cudaStream_t s) {
  constexpr int T = threads_for<N, MR>();
  constexpr int NB = 2 * c_tile(N) <= SMEM_LIMIT ? 2 : 1;
  const size_t smem = NB * c_tile(N);
  g.col_tiles = (g.cols + TW - 1) / TW;
  const int total = ncomp * g.outer * g.col_tiles;
  if (inverse)
    launch_persistent(k_fft_cols<N, true, NB, T, MR>, T, smem, total, s, data, comp_stride, g, ncomp, tw);
  else
    launch_persistent(k_fft_cols<N, false, NB, T, MR>, T, smem, total, s, data, comp_stride, g, ncomp, tw);
}

template <int N>
static void fft3_c2c_n(float2* data, int inverse, const float2* tw, cudaStream_t s) {
  constexpr int T = threads_for<N>();
  constexpr int NB = 2 * c_tile(N) <= SMEM_LIMIT ? 2 : 1;
  const size_t smem = NB * c_tile(N);
  const long long n = N;
  const int rows = N * N;
  const int total = (rows + TW - 1) / TW;
  if (inverse)
    launch_persistent(k_fft_rows<N, true, NB, T>, T, smem, total, s, data, rows, tw);
  else
    launch_persistent(k_fft_rows<N, false, NB, T>, T, smem, total, s, data, rows, tw);
  // y lines: elements n apart, columns along z adjacent, outer = x
  cols_pass<N>(data, 0, 1, ColGeo{n * n, n, N, 0, N}, inverse, tw, s);
  // x lines: elements n*n apart, outer = y
  cols_pass<N>(data, 0, 1, ColGeo{n, n * n, N, 0, N}, inverse, tw, s);
}

void launch_fft3_c2c(const FftPlan& p, float2* data, int inverse, cudaStream_t s) {
  const float2* tw = static_cast<const float2*>(p.twiddle.p);
  switch (p.n) {
#define CPM_CASE(N) \
  case N: fft3_c2c_n<N>(data, inverse, tw, s); break;
    CPM_FFT_SIZES(CPM_CASE)
#undef CPM_CASE
    default: break;
  }
}

// Forward R2C n^3 transform of delta (f32, or the u64 fixed-point mass mesh converted to
// delta = c/mean - 1 on load) into the padded half spectrum: z, then y, then x lines.
template <int N>
static void r2c3_n(const FftPlan& p, const float* delta, const unsigned long long* fx, int fx_shift, float mean,
                   float2* spec, cudaStream_t s) {
  const float2* tw = static_cast<const float2*>(p.twiddle.p);
  constexpr int M = N / 2, NH = N / 2 + 1, NHP = N / 2 + 2;
  const long long n = N;
  const int rows = N * N;
  {
    constexpr int T = threads_for<M>();
    launch_persistent(k_r2c_z<N, T>, T, c_tile(M), (rows + TW - 1) / TW, s, delta, fx, std::ldexp(1.0f, -fx_shift),
                      mean, spec, rows, tw);
  }
  cols_pass<N>(spec, 0, 1, ColGeo{n * NHP, NHP, NH, 0, N}, 0, tw, s);  // y lines, outer = x
  cols_pass<N>(spec, 0, 1, ColGeo{NHP, n * NHP, NH, 0, N}, 0, tw, s);  // x lines, outer = y
}

template <int N, int MR>
static void poisson_n(const FftPlan& p, const PoissonParams& pp, const float* delta, const unsigned long long* fx,
                      int fx_shift, float mean, float2* spec, float* gx, float* gy, float* gz, cudaStream_t s) {
  const float2* tw = static_cast<const float2*>(p.twiddle.p);
  const float* deconv = pp.deconvolve ? static_cast<const float*>(p.deconv.p) : nullptr;
  constexpr int M = N / 2, NH = N / 2 + 1, NHP = N / 2 + 2;
  const long long n = N;
  const int nb = pp.boxes > 1 ? pp.boxes : 1;  // a batch of nb meshes, one after another
  const long long comp = nb * n * n * NHP;     // elements per half spectrum (every box)
  const int rows = nb * N * N;
  const int row_tiles = (rows + TW - 1) / TW;
  if constexpr (2 * c_tile(N) > SMEM_LIMIT) {
    // The fused x pass needs two N-point tiles: not on one SM at this size. Forward R2C, the
    // Green's function and gradient elementwise, then inverse x and y passes on three spectra.
    r2c3_n<N>(p, delta, fx, fx_shift, mean, spec, s);
    const long long total = n * n * NH;
    const int grid = (int)std::min<long long>((total + 255) / 256, 16LL * num_sms());
    count_launch();
    k_green_grad<<<grid, 256, 0, s>>>(spec, comp, N, pp, deconv);
    cols_pass<N, MR>(spec, comp, 3, ColGeo{NHP, n * NHP, NH, 0, N}, 1, tw, s);  // x lines, outer = y
  } else {
    // Slot 0 holds the forward spectrum; the x pass reads each tile of it before writing the
    // same tile of slots 0..2, and tiles are disjoint, so the update in place is safe.
    float2* s0 = spec;
    {  // 1. z: R2C into slot 0 (one complex tile in shared memory per CTA)
      constexpr int T = threads_for<M, MR>();
      launch_persistent(k_r2c_z<N, T, MR>, T, c_tile(M), row_tiles, s, delta, fx, std::ldexp(1.0f, -fx_shift), mean, s0,
                        rows, tw);
    }
    // 2. y forward on slot 0: lines along y (stride NHP), columns along kz adjacent, outer = x
    //    (the x planes of a batch's boxes form one run)
    cols_pass<N, MR>(s0, 0, 1, ColGeo{n * NHP, NHP, NH, 0, nb * N}, 0, tw, s);
    {  // 3. x forward + Green + gradient + x inverse -> slots 0 (-i k_x phi) and 1 (phi); outer = y
      constexpr int T = threads_for<N, MR>();
      constexpr int NBX = 3 * c_tile(N) <= SMEM_LIMIT ? 2 : 1;
      const size_t smem = (NBX + 1) * c_tile(N);
      ColGeo g{NHP, n * NHP, NH, (NH + TW - 1) / TW, nb * N, nb > 1 ? N : 0, n * n * NHP};
      launch_persistent(k_poisson_x<N, NBX, T, MR>, T, smem, g.outer * g.col_tiles, s, s0, spec, comp, g, pp, deconv, tw);
    }
    // 4. y inverse: slot 0 (x component), then slots 1, 2 (y, z components) from the potential
    cols_pass<N, MR>(spec, comp, 1, ColGeo{n * NHP, NHP, NH, 0, nb * N}, 1, tw, s);
    {
      constexpr int T = threads_for<N, MR>();
      constexpr int NBY = 3 * c_tile(N) <= SMEM_LIMIT ? 2 : 1;
      const size_t smem = (NBY + 1) * c_tile(N);
      ColGeo g{n * NHP, NHP, NH, (NH + TW - 1) / TW, nb * N};
      launch_persistent(k_grad_yz<N, NBY, T, MR>, T, smem, g.outer * g.col_tiles, s, spec, comp, g, pp, tw);
    }
  }
  if constexpr (2 * c_tile(N) > SMEM_LIMIT) {
    // 4. y inverse on the three component spectra
    cols_pass<N, MR>(spec, comp, 3, ColGeo{n * NHP, NHP, NH, 0, N}, 1, tw, s);
  }
  {  // 5. z: C2R with 1/n^3
    constexpr int T = threads_for<M, MR>();
    constexpr int NB = 2 * c_tile(M + 1) <= SMEM_LIMIT ? 2 : 1;
    const size_t smem = NB * c_tile(M + 1);
    launch_persistent(k_c2r_z<N, NB, T, MR>, T, smem, 3 * row_tiles, s, spec, comp, gx, gy, gz, pp.scale, rows, tw);
  }
}

void launch_r2c3(const FftPlan& p, const float* delta, const unsigned long long* fx, int fx_shift, float mean,
                 float2* spec, cudaStream_t s) {
  switch (p.n) {
#define CPM_CASE(N) \
  case N: r2c3_n<N>(p, delta, fx, fx_shift, mean, spec, s); break;
    CPM_FFT_SIZES(CPM_CASE)
#undef CPM_CASE
    default: break;
  }
}

void launch_poisson(const FftPlan& p, const PoissonParams& pp, const float* delta, const unsigned long long* fx,
                    int fx_shift, float mean, float2* spec, float* gx, float* gy, float* gz, cudaStream_t s) {
  switch (p.n) {
#define CPM_CASE(N)                                                          \
  case N:                                                                    \
    if (p.max_radix == 4)                                                    \
      poisson_n<N, 4>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, s); \
    else if (p.max_radix == 0)                                               \
      poisson_n<N, 0>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, s); \
    else                                                                     \
      poisson_n<N, 8>(p, pp, delta, fx, fx_shift, mean, spec, gx, gy, gz, s); \
    break;
    CPM_FFT_SIZES(CPM_CASE)
#undef CPM_CASE
    default: break;
  }
}

}  // namespace cpm
