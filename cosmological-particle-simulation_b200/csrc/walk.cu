// walk.cu — the short-range tree walk (tree.rs:264-323) and its pair kernel (tree.rs:54-66).
//
// Traversal. One warp walks for 32 consecutive sorted particles (one per lane) with one shared
// LIFO stack of (node, lane mask) entries. A lane is in a node's mask exactly when its own
// reference walk (tree.rs:264-310) would pop that node; each lane applies the reference's tests
// for itself: prune when |min_image(centre - x)| > r_cut + sqrt(3) half; direct sum over the
// node's particles when its octant-0 child is missing (`children[0] == NO_CHILD`, which includes
// leaves); else accept the centre of mass when 2 half < theta |min_image(com - x)|, or push the
// children 0..7 for the lanes that opened it (they pop 7..0, as in the reference, so each lane
// adds its contributions in the reference's node order). Every decision (prune, accept, cutoff,
// self) is computed with separately rounded f32 operations and an exact minimum image, so it
// matches the reference for equal inputs; where a faster form is used (the square root of the
// opening test) it is checked against the exact one whenever the two could disagree.
//
// Direct sums run lane-per-particle over the node's sources, staged as float4 in shared memory.
// A lane whose particle is far enough from the box faces (|centre - x| + half < 0.49 L on every
// axis) cannot need a periodic image for any source of the node, and skips the image test.
//
// Pair force. f = -K m S(r) / (r^2 + eps^2)^{3/2}, S(r) = erfc(u) + (2/sqrt(pi)) u e^{-u^2},
// u = r / (2 r_s). S is evaluated as e^{-u^2} R(u) with R(u) = erfcx(u) + 2u/sqrt(pi), a smooth
// function fitted on the host for each split: Chebyshev interpolation in double precision
// (erfc from the C library), converted to a degree-12 polynomial in x in [-1, 1] and evaluated
// by f32 Horner — about 2e-7 relative over the range of the leaf pairs (checked by
// cpm_walk_kernel_fit_error). e^{-u^2} uses exp2f with the FMA-exact residual of u*u; r and
// (r^2 + eps^2)^{-3/2} come from rsqrtf. Against the reference's erfcf-based S the pair force
// differs by a few 1e-7 relative; the 1e-5 RMS parity tests cover the sum.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cpm_host.h"
#include "cpm_internal.cuh"

namespace cpm {

constexpr int WALK_WARPS = 4;
constexpr int WALK_THREADS = WALK_WARPS * 32;
constexpr int STACK_CAP = 8 * (KEY_LEVELS + 2);
constexpr int FIT_DEG = 12;
constexpr int FAR_PIECES_MAX = 8;
constexpr double U_NEGLIGIBLE = 9.0;  // S(9) ~ 1e-34: contributions beyond are below f32 resolution

struct SFit {
  float scale0, offset0, umax0;  // piece 0: x = u * scale0 + offset0 for u <= umax0
  float c0[FIT_DEG + 1];
  float far_lo, far_w, far_inv_w, far_hi;  // pieces of width far_w covering [far_lo, far_hi]
  int far_n;
};

struct WalkParams {
  float box;
  float guard;  // |x| below this: round(x / L) == 0 exactly
  float r_cut;
  float cut2;   // r_cut * r_cut
  float theta;
  float inv_two_rs;
  float eps2;   // softening^2
  float k;      // Newtonian coupling
  SFit fit;
};

// ------------------------------------------------------------------ host: the fit of R(u)

static double r_exact(double u) { return std::exp(u * u) * std::erfc(u) + 2.0 * u / std::sqrt(M_PI); }

// Degree-D interpolant of R on [lo, hi] at Chebyshev nodes, as monomial coefficients in x in [-1, 1].
static void fit_piece(double lo, double hi, float* coef) {
  const int D = FIT_DEG, M = D + 1;
  std::vector<double> fx(M), c(M, 0.0);
  for (int k = 0; k < M; ++k) {
    const double x = std::cos(M_PI * (k + 0.5) / M);
    fx[k] = r_exact(lo + (x + 1.0) * 0.5 * (hi - lo));
  }
  for (int j = 0; j < M; ++j) {
    double s = 0.0;
    for (int k = 0; k < M; ++k) s += fx[k] * std::cos(M_PI * j * (k + 0.5) / M);
    c[j] = (j == 0 ? 1.0 : 2.0) * s / M;
  }
  // Chebyshev -> monomial: T_0 = 1, T_1 = x, T_{j+1} = 2x T_j - T_{j-1}
  std::vector<std::vector<double>> T(M, std::vector<double>(M, 0.0));
  T[0][0] = 1.0;
  if (M > 1) T[1][1] = 1.0;
  for (int j = 1; j + 1 < M; ++j)
    for (int p = 0; p < M; ++p) T[j + 1][p] = (p ? 2.0 * T[j][p - 1] : 0.0) - T[j - 1][p];
  for (int p = 0; p < M; ++p) {
    double s = 0.0;
    for (int j = 0; j < M; ++j) s += c[j] * T[j][p];
    coef[p] = (float)s;
  }
}

static float horner_host(const float* c, float x) {
  float acc = c[FIT_DEG];
  for (int j = FIT_DEG - 1; j >= 0; --j) acc = std::fma(acc, x, c[j]);
  return acc;
}

// Piece 0 covers the leaf pairs (u <= r_cut / (2 r_s), at most 2.5 so that degree 12 keeps ~2e-7);
// further pieces of width <= 2.25 reach u = 9.
static SFit make_fit(float r_split, float r_cut, std::vector<float>& far) {
  SFit f{};
  const double u0 = std::min(2.5, std::max(0.25, (double)r_cut / (2.0 * (double)r_split) * 1.0001));
  fit_piece(0.0, u0, f.c0);
  f.umax0 = (float)u0;
  f.scale0 = (float)(2.0 / u0);
  f.offset0 = -1.0f;
  const double rest = U_NEGLIGIBLE - u0;
  f.far_n = rest > 0 ? std::min(FAR_PIECES_MAX, (int)std::ceil(rest / 2.25)) : 0;
  f.far_lo = (float)u0;
  f.far_hi = (float)U_NEGLIGIBLE;
  const double w = f.far_n ? rest / f.far_n : 1.0;
  f.far_w = (float)w;
  f.far_inv_w = (float)(1.0 / w);
  far.assign((size_t)std::max(f.far_n, 1) * (FIT_DEG + 1), 0.0f);
  for (int p = 0; p < f.far_n; ++p) fit_piece(u0 + p * w, u0 + (p + 1) * w, far.data() + (size_t)p * (FIT_DEG + 1));
  return f;
}

// Host twin of the device evaluation of R (same coefficients, same f32 Horner) for the self-check.
static float r_fit_host(const SFit& f, const std::vector<float>& far, float u) {
  if (u <= f.umax0) return horner_host(f.c0, std::fma(u, f.scale0, f.offset0));
  if (u >= f.far_hi || f.far_n == 0) return 0.0f;
  const int p = std::min((int)((u - f.far_lo) * f.far_inv_w), f.far_n - 1);
  const float lo = f.far_lo + (float)p * f.far_w;
  const float x = (u - lo) * (2.0f * f.far_inv_w) - 1.0f;
  return horner_host(far.data() + (size_t)p * (FIT_DEG + 1), x);
}

// ------------------------------------------------------------------ device

__device__ __forceinline__ float horner_dev(const float* c, float x) {
  float acc = c[FIT_DEG];
#pragma unroll
  for (int j = FIT_DEG - 1; j >= 0; --j) acc = fmaf(acc, x, c[j]);
  return acc;
}

__device__ __forceinline__ float horner_far(const float* __restrict__ c, float x) {
  float acc = __ldg(c + FIT_DEG);
#pragma unroll
  for (int j = FIT_DEG - 1; j >= 0; --j) acc = fmaf(acc, x, __ldg(c + j));
  return acc;
}

// S(u) = e^{-u^2} R(u)
__device__ __forceinline__ float short_range_S(float u, const SFit& f, const float* __restrict__ far) {
  float R;
  if (u <= f.umax0) {
    R = horner_dev(f.c0, fmaf(u, f.scale0, f.offset0));
  } else if (u < f.far_hi) {
    const int p = min((int)((u - f.far_lo) * f.far_inv_w), f.far_n - 1);
    const float lo = fmaf((float)p, f.far_w, f.far_lo);
    R = horner_far(far + p * (FIT_DEG + 1), fmaf(u - lo, 2.0f * f.far_inv_w, -1.0f));
  } else {
    return 0.0f;
  }
  const float uu = u * u;
  const float err = fmaf(u, u, -uu);  // u*u = uu + err exactly
  const float e = exp2f(-uu * 1.44269504f);
  return fmaf(-e, err, e) * R;
}

// tree.rs:61-66 without the division and square roots: f = -K m S(r) (r^2 + eps^2)^{-3/2}
__device__ __forceinline__ float pair_factor(float r2, float neg_km, const WalkParams& w,
                                             const float* __restrict__ far) {
  const float r = r2 > 0.0f ? r2 * rsqrtf(r2) : 0.0f;
  const float S = short_range_S(r * w.inv_two_rs, w.fit, far);
  const float rs = rsqrtf(r2 + w.eps2);
  return neg_km * S * (rs * rs * rs);
}

// tree.rs:253-261: d = x - L round(x / L), x = a - b, exact. |x| < 0.49 L gives a zero quotient
// whatever its last bit; the rest divides with IEEE division.
__device__ __forceinline__ float min_image_slow(float x, const WalkParams& w) {
  if (fabsf(x) < w.guard) return x;
  const float q = roundf(__fdiv_rn(x, w.box));
  return __fsub_rn(x, __fmul_rn(w.box, q));
}

// Minimum image of the three components of a - b (raw differences already formed).
__device__ __forceinline__ void min_image3(float& d0, float& d1, float& d2, const WalkParams& w) {
  if (fmaxf(fabsf(d0), fmaxf(fabsf(d1), fabsf(d2))) >= w.guard) {
    d0 = min_image_slow(d0, w);
    d1 = min_image_slow(d1, w);
    d2 = min_image_slow(d2, w);
  }
}

__device__ __forceinline__ float norm2(float a, float b, float c) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

// The reference's opening test `2 half < theta * sqrt(r2)` (tree.rs:297) with IEEE sqrt, evaluated
// with rsqrtf and settled exactly only when the two sides are within a few ulps.
__device__ __forceinline__ bool accept_node(float half, float theta, float r2) {
  const float lhs = __fmul_rn(2.0f, half);
  const float ra = r2 > 0.0f ? r2 * rsqrtf(r2) : 0.0f;
  const float rhs_a = theta * ra;
  if (fabsf(rhs_a - lhs) > 1e-6f * lhs) return lhs < rhs_a;
  return lhs < __fmul_rn(theta, sqrtf(r2));
}

__global__ void __launch_bounds__(WALK_THREADS) k_tree_walk(const uint4* __restrict__ link,
                                                            const float4* __restrict__ geo,
                                                            const float4* __restrict__ mass,
                                                            const float4* __restrict__ x4, size_t n, WalkParams w,
                                                            const float* __restrict__ far, float* __restrict__ acc3,
                                                            int accumulate, unsigned long long* counters,
                                                            DevStatus* st) {
  __shared__ uint2 stack[WALK_WARPS][STACK_CAP];
  __shared__ float4 src[WALK_WARPS][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t gb = ((size_t)blockIdx.x * WALK_WARPS + warp) * 32;
  const size_t i = gb + lane;
  const bool valid = i < n;
  const unsigned group = __ballot_sync(0xffffffffu, valid);
  if (group == 0) return;
  const float4 xi = valid ? __ldg(x4 + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float x0 = xi.x, x1 = xi.y, x2 = xi.z;
  const float neg_k = -w.k;
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
  unsigned long long n_pairs = 0, n_accepts = 0, n_cand = 0;
  uint2* stk = stack[warp];
  float4* sw = src[warp];
  int sp = 0;
  if (lane == 0) stk[0] = make_uint2(0u, group);
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    --sp;
    const uint2 top = stk[sp];
    __syncwarp();
    const uint32_t node = top.x;
    const bool act = (top.y >> lane) & 1u;
    const float4 G = __ldg(geo + node);
    bool live = false, nowrap = false;
    if (act) {
      float t0 = __fsub_rn(G.x, x0), t1 = __fsub_rn(G.y, x1), t2 = __fsub_rn(G.z, x2);
      // every source y of the node lies in [centre - half, centre + half]
      nowrap = fmaxf(fabsf(t0), fmaxf(fabsf(t1), fabsf(t2))) + G.w < w.guard;
      min_image3(t0, t1, t2, w);
      const float max_r = __fadd_rn(w.r_cut, __fmul_rn(SQRT_3, G.w));
      live = !(norm2(t0, t1, t2) > __fmul_rn(max_r, max_r));
    }
    const unsigned live_mask = __ballot_sync(0xffffffffu, live);
    if (live_mask == 0) continue;
    const uint4 L = __ldg(link + node);
    if ((L.w & 1u) == 0u) {
      // children[0] == NO_CHILD: direct sum over the node's particles (tree.rs:286-298)
      if (live) n_cand += L.y - L.x;
      for (uint32_t b0 = L.x; b0 < L.y; b0 += 32) {
        const uint32_t j = b0 + lane;
        if (j < L.y) sw[lane] = __ldg(x4 + j);
        __syncwarp();
        if (live) {
          const int cnt = (int)min(32u, L.y - b0);
          const int self = (gb == b0) ? lane : ((size_t)b0 <= i && i < (size_t)b0 + 32 ? (int)(i - b0) : -1);
          if (nowrap) {
#pragma unroll 4
            for (int t = 0; t < cnt; ++t) {
              const float4 y = sw[t];
              const float d0 = __fsub_rn(x0, y.x), d1 = __fsub_rn(x1, y.y), d2 = __fsub_rn(x2, y.z);
              const float r2 = norm2(d0, d1, d2);
              if (!(r2 > w.cut2) && t != self) {
                const float f = pair_factor(r2, neg_k, w, far);
                a0 = fmaf(d0, f, a0);
                a1 = fmaf(d1, f, a1);
                a2 = fmaf(d2, f, a2);
                ++n_pairs;
              }
            }
          } else {
            for (int t = 0; t < cnt; ++t) {
              const float4 y = sw[t];
              float d0 = __fsub_rn(x0, y.x), d1 = __fsub_rn(x1, y.y), d2 = __fsub_rn(x2, y.z);
              min_image3(d0, d1, d2, w);
              const float r2 = norm2(d0, d1, d2);
              if (!(r2 > w.cut2) && t != self) {
                const float f = pair_factor(r2, neg_k, w, far);
                a0 = fmaf(d0, f, a0);
                a1 = fmaf(d1, f, a1);
                a2 = fmaf(d2, f, a2);
                ++n_pairs;
              }
            }
          }
        }
        __syncwarp();
      }
    } else {
      bool open = false;
      if (live) {
        const float4 M = __ldg(mass + node);
        float t0 = __fsub_rn(M.x, x0), t1 = __fsub_rn(M.y, x1), t2 = __fsub_rn(M.z, x2);
        min_image3(t0, t1, t2, w);
        const float r2 = norm2(t0, t1, t2);
        if (accept_node(G.w, w.theta, r2)) {
          const float f = pair_factor(r2, neg_k * M.w, w, far);
          a0 = fmaf(-t0, f, a0);
          a1 = fmaf(-t1, f, a1);
          a2 = fmaf(-t2, f, a2);
          ++n_accepts;
        } else {
          open = true;
        }
      }
      const unsigned open_mask = __ballot_sync(0xffffffffu, open);
      if (open_mask) {
        const uint32_t cmask = L.w & 0xFFu;
        const int nch = __popc(cmask);
        if (sp + nch > STACK_CAP) {
          if (lane == 0) dev_fail(st, DEV_STACK_OVERFLOW, (int)node);
          break;
        }
        if (lane < nch) stk[sp + lane] = make_uint2(L.z + (uint32_t)lane, open_mask);
        sp += nch;
        __syncwarp();
      }
    }
  }
  if (valid) {
    if (accumulate) {
      acc3[3 * i] = __fadd_rn(acc3[3 * i], a0);
      acc3[3 * i + 1] = __fadd_rn(acc3[3 * i + 1], a1);
      acc3[3 * i + 2] = __fadd_rn(acc3[3 * i + 2], a2);
    } else {
      acc3[3 * i] = a0;
      acc3[3 * i + 1] = a1;
      acc3[3 * i + 2] = a2;
    }
  }
  if (counters) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      n_pairs += __shfl_xor_sync(0xffffffffu, n_pairs, o);
      n_accepts += __shfl_xor_sync(0xffffffffu, n_accepts, o);
      n_cand += __shfl_xor_sync(0xffffffffu, n_cand, o);
    }
    if (lane == 0) {
      atomicAdd(&counters[0], n_pairs);
      atomicAdd(&counters[1], n_accepts);
      atomicAdd(&counters[2], n_cand);
    }
  }
}

// Packs AoS positions into float4 (x, y, z, 0) for 16-byte loads.
__global__ void k_pack4(const float* __restrict__ x3, size_t n, float4* __restrict__ x4) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x4[i] = make_float4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], 0.0f);
}

// ------------------------------------------------------------------ host launch

struct FitCache {
  float r_split = -1.0f, r_cut = -1.0f;
  SFit fit{};
  std::vector<float> far;
  DevBuf far_dev;
};

static FitCache& fit_cache() {
  static thread_local FitCache c;
  return c;
}

void launch_tree_walk(const TreeNodes& t, const float* sorted_x3, size_t n, float box, const cpm_force_split& split,
                      float k, float* acc3, int accumulate, TreeCounters* counters, DevStatus* st, cudaStream_t s) {
  if (n == 0) return;
  FitCache& fc = fit_cache();
  if (fc.r_split != split.r_split || fc.r_cut != split.r_cut || !fc.far_dev.p) {
    fc.fit = make_fit(split.r_split, split.r_cut, fc.far);
    if (ensure(fc.far_dev, fc.far.size() * sizeof(float)) != cudaSuccess) return;
    cudaMemcpy(fc.far_dev.p, fc.far.data(), fc.far.size() * sizeof(float), cudaMemcpyHostToDevice);
    fc.r_split = split.r_split;
    fc.r_cut = split.r_cut;
  }
  TreeNodes& tm = const_cast<TreeNodes&>(t);
  if (ensure(tm.x4, n * sizeof(float4)) != cudaSuccess) return;
  const unsigned pb = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
  count_launch();
  k_pack4<<<pb, 256, 0, s>>>(sorted_x3, n, as<float4>(tm.x4));

  WalkParams w;
  w.box = box;
  w.guard = 0.49f * box;
  w.r_cut = split.r_cut;
  w.cut2 = split.r_cut * split.r_cut;
  w.theta = split.theta;
  w.inv_two_rs = (float)(1.0 / (2.0 * (double)split.r_split));
  w.eps2 = split.softening * split.softening;
  w.k = k;
  w.fit = fc.fit;
  const size_t groups = (n + 31) / 32;
  const unsigned blocks = (unsigned)((groups + WALK_WARPS - 1) / WALK_WARPS);
  count_launch();
  k_tree_walk<<<blocks, WALK_THREADS, 0, s>>>(static_cast<const uint4*>(t.link.p), static_cast<const float4*>(t.geo.p),
                                              static_cast<const float4*>(t.mass.p), as<float4>(tm.x4), n, w,
                                              static_cast<const float*>(fc.far_dev.p), acc3, accumulate,
                                              reinterpret_cast<unsigned long long*>(counters), st);
}

}  // namespace cpm

using namespace cpm;

// Self-check of the fitted pair kernel: max relative error of e^{-u^2} R_fit(u) (f32 Horner, host)
// against the double-precision S(u) over u in [0, u_max], u_max = r_cut / (2 r_split), on `samples`
// points. Host only; no device is needed.
extern "C" int cpm_walk_kernel_fit_error(float r_split, float r_cut, int samples, double* max_rel_err) {
  if (!(r_split > 0.0f) || !(r_cut > 0.0f) || samples < 2 || !max_rel_err)
    return set_error(nullptr, CPM_E_INVALID, "cpm_walk_kernel_fit_error: bad arguments");
  std::vector<float> far;
  const SFit f = make_fit(r_split, r_cut, far);
  const double umax = std::min(U_NEGLIGIBLE, (double)r_cut / (2.0 * (double)r_split));
  double worst = 0.0;
  for (int q = 0; q < samples; ++q) {
    const float u = (float)(umax * q / (samples - 1));
    const double ud = (double)u;
    const double exact = std::erfc(ud) + 2.0 * ud / std::sqrt(M_PI) * std::exp(-ud * ud);
    const double got = std::exp(-ud * ud) * (double)r_fit_host(f, far, u);
    worst = std::max(worst, std::fabs(got - exact) / exact);
  }
  *max_rel_err = worst;
  return CPM_OK;
}
