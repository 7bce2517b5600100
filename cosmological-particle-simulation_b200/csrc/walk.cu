// walk.cu — the short-range tree walk (tree.rs:264-323) and its pair kernel (tree.rs:54-66).
//
// Traversal. One warp walks for 32 consecutive sorted particles (one per lane). The stack holds
// batches: the children of one opened node (contiguous in the node arrays), with the mask of the
// lanes that opened it. The unit of work is a step of up to 32 nodes, one per lane: the top batch
// and, while the stack is shallow (which bounds its depth), the batches below it as long as they
// fit. Lane c copies node c's three 16-byte records (centre and half, centre of mass and mass,
// link) into shared memory with cp.async, double-buffered: the next step's copies are in flight
// while the current step is summed. Lane c also derives the node's constants once for the warp
// (prune radius squared, (2 half)^2), and a test against the bounding box of the warp's particles
// drops nodes that every lane would prune. Every lane then applies the reference's tests
// (tree.rs:264-310), for itself, to each remaining node of the batches it opened: prune when
// |min_image(centre - x)| > r_cut + sqrt(3) half; direct sum over the node's particles when its
// octant-0 child is missing (`children[0] == NO_CHILD`, which includes leaves); else accept the
// centre of mass when 2 half < theta |min_image(com - x)|, or open the node, which becomes a new
// batch on the stack tagged with the lanes that opened it. A lane's set of interactions is
// exactly the one its own reference walk visits: every decision uses separately rounded f32
// operations and an exact minimum image (skipped for steps whose nodes are all far from the
// box faces, where it is the identity), and the opening test, evaluated on squares, falls back to
// the reference's square-root form whenever the two sides are within 1e-5; only the order in
// which a lane adds its interactions differs.
//
// Direct sums concatenate the sources of all direct nodes of a step into chunks of 32 (negated
// positions, one array per axis, in shared memory); lane q finds the node of source base + q by a
// binary search over the nodes' prefix sums. Per chunk a lane first marks the sources
// within r_cut of it (bit mask; differences and squares two sources per f32x2 instruction, the
// sums scalar so that r^2 rounds like the reference's), then evaluates the pair force only for
// the marked ones, two per iteration in f32x2, so lanes do not idle on sources outside the cutoff
// of other lanes. A lane whose direct nodes all lie far enough from the box faces
// (|centre - x| + half < 0.49 L on every axis) cannot need a periodic image, and skips the image
// test.
//
// Pair force. f = -K m S(r) / (r^2 + eps^2)^{3/2}, S(r) = erfc(u) + (2/sqrt(pi)) u e^{-u^2},
// u = r / (2 r_s). S is evaluated as e^{-u^2} R(u) with R(u) = erfcx(u) + 2u/sqrt(pi), a smooth
// function fitted on the host for each split: Chebyshev interpolation in double precision
// (erfc from the C library), converted to a degree-12 polynomial in x in [-1, 1] and evaluated
// by f32 Horner — about 2e-7 relative over the range of the leaf pairs (checked by
// cpm_walk_kernel_fit_error). e^{-u^2} takes the FMA-exact residual of u*u; for the direct pairs
// e^{-u^2}, r and (r^2 + eps^2)^{-3/2} come from the hardware approximations (ex2, rsqrt; about
// 2^-22 relative), for accepted nodes from exp2f and rsqrtf. The coupling K multiplies each
// particle's sum once at the end. Against the reference's erfcf-based S the pair force differs
// by a few 1e-7 relative; the 1e-5 RMS parity tests cover the sum.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cpm_host.h"
#include "cpm_internal.cuh"

namespace cpm {

constexpr int SLOTS = 32;     // nodes per step of a warp's walk (one per lane)
constexpr int MERGE_SP = 96;  // stack entries are merged into one step only while the stack is this shallow
// Stack bound: a merging step starts at depth <= MERGE_SP and pushes at most SLOTS entries; from
// there single-entry steps (depth first) keep at most 7 unvisited sibling entries per tree level
// below, plus the 8 just pushed.
constexpr int STACK_CAP = MERGE_SP + SLOTS + 7 * KEY_LEVELS + 8;
constexpr uint32_t FIRST_BITS = 29;  // a stack entry: first node (29 bits) | (count - 1) << 29
constexpr int FIT_DEG = 12;
constexpr int FAR_PIECES_MAX = 8;
constexpr double U_NEGLIGIBLE = 9.0;  // S(9) ~ 1e-34: contributions beyond are below f32 resolution

struct SFit {
  float scale0, offset0, umax0;  // piece 0: x = u * scale0 + offset0 for u <= umax0
  float c0[FIT_DEG + 1];
  float far_lo, far_w, far_inv_w, far_hi;  // pieces of width far_w covering [far_lo, far_hi]
  int far_n;
};

// The constants of the direct-sum pair force, duplicated for the packed (two pairs per
// instruction) evaluation.
struct PairConst2 {
  float2 tiny;        // added to r^2 under the reciprocal square root, so that r = 0 stays 0
  float2 inv_two_rs;  // 1 / (2 r_s)
  float2 scale0, offset0;
  float2 c0[FIT_DEG + 1];
  float2 neg_log2e;   // -log2(e)
  float2 eps2;        // softening^2
  float2 neg_m;       // -m (the coupling K multiplies the sum at the end)
};

struct WalkParams {
  float box;
  float guard;  // |x| below this: round(x / L) == 0 exactly
  float r_cut;
  float cut2;   // r_cut * r_cut
  float theta;
  float theta2;  // theta * theta (f32), for the squared form of the opening test
  float inv_two_rs;
  float eps2;   // softening^2
  float k;      // Newtonian coupling
  uint32_t n_box;  // batch of boxes: particles per box (multiple of 32); a warp starts at root i / n_box
  SFit fit;
  PairConst2 p2;
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

// Hardware approximations (MUFU): relative error about 2^-22, no special handling of
// denormal inputs (the arguments here are r^2 + tiny, r^2 + eps^2 and -u^2 log2(e)).
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float exp2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// pair_factor for two pairs at once (f32x2 arithmetic), coupling -K m of a particle.
__device__ __forceinline__ float2 pair_factor2(float2 r2, const WalkParams& w, const float* __restrict__ far) {
  const PairConst2& c = w.p2;
  const float2 rr = __fadd2_rn(r2, c.tiny);
  const float2 r = __fmul2_rn(r2, make_float2(rsqrt_approx(rr.x), rsqrt_approx(rr.y)));
  const float2 u = __fmul2_rn(r, c.inv_two_rs);
  float2 S;
  if (fmaxf(u.x, u.y) <= w.fit.umax0) {
    const float2 x = __ffma2_rn(u, c.scale0, c.offset0);
    float2 R = c.c0[FIT_DEG];
#pragma unroll
    for (int j = FIT_DEG - 1; j >= 0; --j) R = __ffma2_rn(R, x, c.c0[j]);
    // e^{-u^2} = 2^{-uu log2 e} (1 - err) with uu + err = u*u exactly
    const float2 uu = __fmul2_rn(u, u);
    const float2 nerr = __ffma2_rn(__fmul2_rn(u, make_float2(-1.0f, -1.0f)), u, uu);
    const float2 ea = __fmul2_rn(uu, c.neg_log2e);
    const float2 e = make_float2(exp2_approx(ea.x), exp2_approx(ea.y));
    S = __fmul2_rn(__ffma2_rn(e, nerr, e), R);
  } else {
    S = make_float2(short_range_S(u.x, w.fit, far), short_range_S(u.y, w.fit, far));
  }
  const float2 q = __fadd2_rn(r2, c.eps2);
  const float2 rs = make_float2(rsqrt_approx(q.x), rsqrt_approx(q.y));
  return __fmul2_rn(__fmul2_rn(c.neg_m, S), __fmul2_rn(__fmul2_rn(rs, rs), rs));
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

// The reference's opening test `2 half < theta * sqrt(r2)` (tree.rs:297), from per-node
// constants: lhs = 2 half, L2 = lhs^2, tol = 1e-5 L2. theta^2 r2 and
// L2 carry at most ~7e-7 relative rounding against the exact squares of both sides, so outside
// the 1e-5 band the squared comparison decides like the reference's; inside it the reference's
// expression is evaluated (IEEE square root).
__device__ __forceinline__ bool accept_node_sq(float r2, const float4& pre, const WalkParams& w) {
  const float diff = __fsub_rn(__fmul_rn(w.theta2, r2), pre.y);
  if (fabsf(diff) > pre.z) return diff > 0.0f;
  return pre.w < __fmul_rn(w.theta, __fsqrt_rn(r2));
}

// Per-warp shared state of the walk.
struct WalkShared {
  uint2 stack[STACK_CAP];          // (first node | (count - 1) << 29, lane mask): a batch of siblings
  float4 geo[2][SLOTS];            // the current and the next step's nodes: centre, half
  float4 mass[2][SLOTS];           //                                        centre of mass, count
  uint4 link[2][SLOTS];            //                                        start, end, first child, child mask
  float4 pre[SLOTS];               // per node of the current step: prune radius^2, (2 half)^2,
                                   // 1e-5 (2 half)^2, 2 half
  uint32_t dbeg[SLOTS], dend[SLOTS], dsrc[SLOTS];  // direct sums: node c's sources are positions
                                                   // dbeg .. dend - 1 of the concatenation,
                                                   // particles dsrc + (position - dbeg)
  float nx[32], ny[32], nz[32];    // a chunk of direct-sum sources, negated: -x, -y, -z
  float4 box_c, box_h;             // the warp's bounding box: centre, half extent (+ tolerance)
};

// 16-byte asynchronous copy global -> shared (completion awaited with cp.async.wait_all).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
// Bits lo .. lo + len - 1 (len in 1..32).
__device__ __forceinline__ uint32_t bit_span(uint32_t lo, uint32_t len) {
  return (len >= 32u ? 0xffffffffu : ((1u << len) - 1u)) << lo;
}

// Direct-sum phase 1 for one chunk: bit t set when source t lies within r_cut of the lane's
// particle (tree.rs:286-298); the caller keeps the bits of the sources it sums directly. The
// difference and its squared norm round exactly like the reference's separate f32 operations;
// without periodic images the differences and squares of two sources are formed per instruction
// (f32x2, each element rounded like the scalar operation) and the sums are scalar.
template <bool WRAP>
__device__ __forceinline__ uint32_t chunk_candidates(const WalkShared& sh, int cnt, float x0, float x1, float x2,
                                                     const WalkParams& w) {
  uint32_t pm = 0;
  if (!WRAP) {
    const float2 X0 = make_float2(x0, x0), X1 = make_float2(x1, x1), X2 = make_float2(x2, x2);
#pragma unroll 4
    for (int t = 0; t < cnt; t += 2) {
      const float2 d0 = __fadd2_rn(X0, *reinterpret_cast<const float2*>(sh.nx + t));
      const float2 d1 = __fadd2_rn(X1, *reinterpret_cast<const float2*>(sh.ny + t));
      const float2 d2 = __fadd2_rn(X2, *reinterpret_cast<const float2*>(sh.nz + t));
      // The squares are packed, the sums scalar: a packed multiply feeding a packed add can be
      // contracted into one FMA, which would round differently from the reference's f32 ops.
      const float2 q0 = __fmul2_rn(d0, d0), q1 = __fmul2_rn(d1, d1), q2 = __fmul2_rn(d2, d2);
      const float r2a = __fadd_rn(__fadd_rn(q0.x, q1.x), q2.x), r2b = __fadd_rn(__fadd_rn(q0.y, q1.y), q2.y);
      pm |= ((uint32_t)!(r2a > w.cut2) | ((uint32_t)!(r2b > w.cut2) << 1)) << t;
    }
  } else {
    for (int t = 0; t < cnt; ++t) {
      float d0 = __fadd_rn(x0, sh.nx[t]), d1 = __fadd_rn(x1, sh.ny[t]), d2 = __fadd_rn(x2, sh.nz[t]);
      min_image3(d0, d1, d2, w);
      pm |= (uint32_t)!(norm2(d0, d1, d2) > w.cut2) << t;
    }
  }
  return pm;
}

// Direct-sum phase 2: the pair forces of the sources in pm, two per iteration, added to the
// packed accumulators (even and odd pairs).
template <bool WRAP>
__device__ __forceinline__ void chunk_forces(const WalkShared& sh, uint32_t pm, float x0, float x1, float x2,
                                             const WalkParams& w, const float* __restrict__ far, float2& A0,
                                             float2& A1, float2& A2) {
  const float2 X0 = make_float2(x0, x0), X1 = make_float2(x1, x1), X2 = make_float2(x2, x2);
  while (pm) {
    const int t1 = __ffs(pm) - 1;
    pm &= pm - 1;
    int t2 = t1;
    float keep = 0.0f;  // a lone last pair is evaluated twice and its copy weighted by 0
    if (pm) {
      t2 = __ffs(pm) - 1;
      pm &= pm - 1;
      keep = 1.0f;
    }
    float2 d0 = __fadd2_rn(X0, make_float2(sh.nx[t1], sh.nx[t2]));
    float2 d1 = __fadd2_rn(X1, make_float2(sh.ny[t1], sh.ny[t2]));
    float2 d2 = __fadd2_rn(X2, make_float2(sh.nz[t1], sh.nz[t2]));
    if (WRAP) {
      min_image3(d0.x, d1.x, d2.x, w);
      min_image3(d0.y, d1.y, d2.y, w);
    }
    const float2 r2 = __ffma2_rn(d2, d2, __ffma2_rn(d1, d1, __fmul2_rn(d0, d0)));
    const float2 f = __fmul2_rn(pair_factor2(r2, w, far), make_float2(1.0f, keep));
    A0 = __ffma2_rn(d0, f, A0);
    A1 = __ffma2_rn(d1, f, A1);
    A2 = __ffma2_rn(d2, f, A2);
  }
}

// Quadrupole term of an accepted node (no counterpart in the reference, whose nodes are monopoles,
// tree.rs:68-80): the second-order Taylor term of a = sum_j g(|d_j|) d_j about the centre of mass,
// d_j = D + e_j with sum_j e_j = 0, T = sum_j e_j e_j^T, g(r) = S(r / 2 r_s) (r^2 + eps^2)^(-3/2):
//   da = (1/2) [ h (D.T.D) D + (g'/r) (tr(T) D + 2 T D) ],   h = (g'' - g'/r) / r^2,
// with S' = -(2/sqrt(pi)) u^2 e^{-u^2} / r_s and S'' = -(2/sqrt(pi)) u (1 - u^2) e^{-u^2} / r_s^2
// (u = r / 2 r_s). Unit coupling, like the walk's sums; precision mode only (CUDA's erfcf / expf).
__device__ __forceinline__ void quad_term(float d0, float d1, float d2, const float4& Q0, const float4& Q1,
                                          const WalkParams& w, float2& A0, float2& A1, float2& A2) {
  const float r2 = d0 * d0 + d1 * d1 + d2 * d2;
  if (!(r2 > 0.0f)) return;
  const float r = sqrtf(r2), inv_r = 1.0f / r;
  const float rs = 0.5f / w.inv_two_rs;
  const float u = r * w.inv_two_rs, e = expf(-u * u);
  const float S = erfcf(u) + TWO_OVER_SQRT_PI * u * e;
  const float S1 = -TWO_OVER_SQRT_PI * u * u * e / rs;
  const float S2 = -TWO_OVER_SQRT_PI * u * (1.0f - u * u) * e / (rs * rs);
  const float q = r2 + w.eps2, iq = 1.0f / q, rq = rsqrtf(q);
  const float P = rq * iq, P1 = -3.0f * r * P * iq, P2 = -3.0f * P * iq + 15.0f * r2 * P * iq * iq;
  const float g1 = S1 * P + S * P1;
  const float g2 = S2 * P + 2.0f * S1 * P1 + S * P2;
  const float h = (g2 - g1 * inv_r) / r2;
  const float td0 = Q0.x * d0 + Q0.w * d1 + Q1.x * d2;
  const float td1 = Q0.w * d0 + Q0.y * d1 + Q1.y * d2;
  const float td2 = Q1.x * d0 + Q1.y * d1 + Q0.z * d2;
  const float dtd = d0 * td0 + d1 * td1 + d2 * td2, tr = Q0.x + Q0.y + Q0.z;
  const float a = 0.5f * h * dtd, b = 0.5f * g1 * inv_r;
  A0.y += a * d0 + b * (tr * d0 + 2.0f * td0);
  A1.y += a * d1 + b * (tr * d1 + 2.0f * td1);
  A2.y += a * d2 + b * (tr * d2 + 2.0f * td2);
}

template <bool QUAD, bool LIST, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_tree_walk(const uint4* __restrict__ link,
                                                            const float4* __restrict__ geo,
                                                            const float4* __restrict__ mass,
                                                            const float4* __restrict__ x4, size_t n, WalkParams w,
                                                            const float* __restrict__ far, float* __restrict__ acc3,
                                                            int accumulate, unsigned long long* counters,
                                                            DevStatus* st, const float* __restrict__ k_dev,
                                                            const uint32_t* __restrict__ list,
                                                            const uint32_t* __restrict__ list_n,
                                                            const float4* __restrict__ quad) {
  // Dynamic shared memory: WARPS WalkShared records, then (quadrupoles) the node index of each slot.
  extern __shared__ __align__(16) unsigned char walk_smem[];
  WalkShared* shared = reinterpret_cast<WalkShared*>(walk_smem);
  uint32_t(*node_ids)[2][SLOTS] = reinterpret_cast<uint32_t(*)[2][SLOTS]>(walk_smem + WARPS * sizeof(WalkShared));
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Lane t of the grid walks for sorted particle t, or, with a list, for particle list[t] (t below
  // *list_n): the list keeps the sorted order, so a warp's particles stay spatially coherent.
  const size_t t = ((size_t)blockIdx.x * WARPS + warp) * 32 + lane;
  const bool valid = LIST ? t < (size_t)*list_n : t < n;
  const size_t i = LIST ? (valid ? (size_t)list[t] : 0) : t;
  const unsigned group = __ballot_sync(FULL, valid);
  if (group == 0) return;
  WalkShared& sh = shared[warp];
  const float4 xi = valid ? __ldg(x4 + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float x0 = xi.x, x1 = xi.y, x2 = xi.z;
  const uint32_t self = (uint32_t)i;

  // Bounding box of the warp's particles (centre cg, half extent hg), for a conservative
  // warp-level prune test: a node farther than r_cut + sqrt(3) half from the whole box is pruned
  // by every lane, whose own test is then skipped.
  float lo0 = valid ? x0 : INFINITY, lo1 = valid ? x1 : INFINITY, lo2 = valid ? x2 : INFINITY;
  float hi0 = valid ? x0 : -INFINITY, hi1 = valid ? x1 : -INFINITY, hi2 = valid ? x2 : -INFINITY;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo0 = fminf(lo0, __shfl_xor_sync(FULL, lo0, o));
    lo1 = fminf(lo1, __shfl_xor_sync(FULL, lo1, o));
    lo2 = fminf(lo2, __shfl_xor_sync(FULL, lo2, o));
    hi0 = fmaxf(hi0, __shfl_xor_sync(FULL, hi0, o));
    hi1 = fmaxf(hi1, __shfl_xor_sync(FULL, hi1, o));
    hi2 = fmaxf(hi2, __shfl_xor_sync(FULL, hi2, o));
  }
  if (lane == 0) {
    const float tol = 1e-5f * w.box;  // far above the rounding of positions and differences
    sh.box_c = make_float4(0.5f * (lo0 + hi0), 0.5f * (lo1 + hi1), 0.5f * (lo2 + hi2), 0.0f);
    sh.box_h = make_float4(0.5f * (hi0 - lo0) + tol, 0.5f * (hi1 - lo1) + tol, 0.5f * (hi2 - lo2) + tol, 0.0f);
  }
  // Accumulators of the even and odd pairs (x: even pairs and accepted nodes).
  float2 A0 = make_float2(0.0f, 0.0f), A1 = A0, A2 = A0;
  uint32_t n_pairs = 0, n_accepts = 0, n_cand = 0;

  // A step of the walk handles up to SLOTS nodes, one per lane: one or more stack entries (each the
  // children of an opened node, with the mask of the lanes that opened it) placed in consecutive
  // slots. `mine` holds the slots this lane walks. Lane c copies slot c's three records into shared
  // buffer `cur` asynchronously; the next step's copies are in flight while the current step is
  // summed. The walk starts at the root: node 0, or in a batch of boxes the root of the warp's box
  // (nodes 0 .. boxes - 1; a box's particles fill whole warps, and a list keeps each box's
  // particles in whole warps, so the first valid lane's box is the warp's).
  const uint32_t root = w.n_box ? __shfl_sync(FULL, (uint32_t)(i / w.n_box), __ffs(group) - 1) : 0u;
  uint32_t b_count = 1, mine = (group >> lane) & 1u;
  int cur = 0;
  if (lane == 0) {
    cp_async16(&sh.geo[0][0], geo + root);
    cp_async16(&sh.mass[0][0], mass + root);
    cp_async16(&sh.link[0][0], link + root);
    if constexpr (QUAD) node_ids[warp][0][0] = root;
  }
  int sp = 0;
  for (;;) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    const float4* bgeo = sh.geo[cur];
    const float4* bmass = sh.mass[cur];
    const uint4* blink = sh.link[cur];

    // Warp-level prune test, lane c for node c. It applies where no lane can need a periodic
    // image (|centre - x| < 0.49 L on every axis for the whole box), so that the lanes' own
    // distances are the raw differences; it keeps a node unless even the box's nearest point is
    // beyond r_cut + sqrt(3) half by a relative margin of 1e-5.
    bool keep = false, far_edge = false, direct = false;
    if ((uint32_t)lane < b_count) {
      const float4 bc = sh.box_c, bh = sh.box_h, pg = bgeo[lane];
      const float e0 = fabsf(pg.x - bc.x), e1 = fabsf(pg.y - bc.y), e2 = fabsf(pg.z - bc.z);
      const float mr = __fadd_rn(w.r_cut, __fmul_rn(SQRT_3, pg.w));
      const float lhs = __fmul_rn(2.0f, pg.w), l2 = __fmul_rn(lhs, lhs);
      sh.pre[lane] = make_float4(__fmul_rn(mr, mr), l2, 1e-5f * l2, lhs);
      direct = (blink[lane].w & 1u) == 0u;
      keep = true;
      const float emax = fmaxf(e0 + bh.x, fmaxf(e1 + bh.y, e2 + bh.z));
      if (emax < w.guard) {
        const float g0 = fmaxf(e0 - bh.x, 0.0f), g1 = fmaxf(e1 - bh.y, 0.0f), g2 = fmaxf(e2 - bh.z, 0.0f);
        keep = !(g0 * g0 + g1 * g1 + g2 * g2 > mr * mr * 1.00001f);
      }
      // No lane needs a periodic image for this node: every difference between a lane's
      // particle and the node's centre, centre of mass or particles (all inside the cube) is
      // below 0.49 L on every axis.
      far_edge = emax + pg.w < w.guard;
    }
    const uint32_t cand = __ballot_sync(FULL, keep);
    const uint32_t nwall = __ballot_sync(FULL, far_edge);
    const uint32_t dbits = __ballot_sync(FULL, direct);
    __syncwarp();

    // Classify every remaining node of this lane for its particle: prune, direct sum, accept or open.
    uint32_t dmask = 0, nwmask = 0, amask = 0, omask = 0;
    const uint32_t todo = cand & mine;
    if ((todo & ~nwall) == 0u) {
      // No node of the step involves a periodic image: raw differences.
      for (uint32_t rem = todo; rem; rem &= rem - 1) {
        const uint32_t c = __ffs(rem) - 1;
        const float4 G = bgeo[c], P = sh.pre[c];
        const float t0 = __fsub_rn(G.x, x0), t1 = __fsub_rn(G.y, x1), t2 = __fsub_rn(G.z, x2);
        if (norm2(t0, t1, t2) > P.x) continue;
        if ((dbits >> c) & 1u) {
          dmask |= 1u << c;
          continue;
        }
        const float4 M = bmass[c];
        const float s0 = __fsub_rn(M.x, x0), s1 = __fsub_rn(M.y, x1), s2 = __fsub_rn(M.z, x2);
        if (accept_node_sq(norm2(s0, s1, s2), P, w))
          amask |= 1u << c;
        else
          omask |= 1u << c;
      }
      nwmask = dmask;
    } else {
      for (uint32_t rem = todo; rem; rem &= rem - 1) {
        const uint32_t c = __ffs(rem) - 1;
        const float4 G = bgeo[c], P = sh.pre[c];
        float t0 = __fsub_rn(G.x, x0), t1 = __fsub_rn(G.y, x1), t2 = __fsub_rn(G.z, x2);
        // every source y of the node lies in [centre - half, centre + half]
        const bool nowrap = fmaxf(fabsf(t0), fmaxf(fabsf(t1), fabsf(t2))) + G.w < w.guard;
        min_image3(t0, t1, t2, w);
        if (norm2(t0, t1, t2) > P.x) continue;
        if ((dbits >> c) & 1u) {
          // children[0] == NO_CHILD: direct sum over the node's particles (tree.rs:286-298)
          dmask |= 1u << c;
          nwmask |= (uint32_t)nowrap << c;
          continue;
        }
        const float4 M = bmass[c];
        float s0 = __fsub_rn(M.x, x0), s1 = __fsub_rn(M.y, x1), s2 = __fsub_rn(M.z, x2);
        min_image3(s0, s1, s2, w);
        if (accept_node_sq(norm2(s0, s1, s2), P, w))
          amask |= 1u << c;
        else
          omask |= 1u << c;
      }
    }

    // Push the opened nodes' children as new stack entries (any order gives each lane the same
    // set of interactions; only the order of its sums differs). Higher slots go deeper into the
    // stack, so that the entries popped first, which fill the lowest slots, have their children
    // popped first again.
    const uint32_t ouni = __reduce_or_sync(FULL, omask);
    if (ouni) {
      uint32_t opened_by = 0;
      for (uint32_t rem = ouni; rem; rem &= rem - 1) {
        const int c = __ffs(rem) - 1;
        const uint32_t b = __ballot_sync(FULL, (omask >> c) & 1u);
        if (lane == c) opened_by = b;
      }
      const int npush = __popc(ouni);
      // (node indices above 29 bits, trees of more than 2^28 particles, do not fit an entry)
      const bool wide = __any_sync(FULL, ((ouni >> lane) & 1u) && (blink[lane].z >> FIRST_BITS) != 0u);
      if (sp + npush > STACK_CAP || wide) {
        if (lane == 0) dev_fail(st, DEV_STACK_OVERFLOW, sp);
        break;
      }
      if ((ouni >> lane) & 1u) {
        const uint4 L = blink[lane];
        const int slot = sp + __popc(ouni >> lane) - 1;
        sh.stack[slot] = make_uint2(L.z | ((uint32_t)(__popc(L.w & 0xFFu) - 1) << FIRST_BITS), opened_by);
      }
      sp += npush;
      __syncwarp();
    }

    // Pop the next step: the top entry, and while the stack is shallow, further entries as long as
    // they fit in the slots. Its copies complete during the work below.
    uint32_t nx_count = 0, nx_mine = 0;
    if (sp > 0) {
      const bool merge = sp <= MERGE_SP;
      for (;;) {
        const uint2 e = sh.stack[--sp];
        const uint32_t first = e.x & ((1u << FIRST_BITS) - 1u), cnt = (e.x >> FIRST_BITS) + 1u;
        if ((uint32_t)lane >= nx_count && (uint32_t)lane < nx_count + cnt) {
          const uint32_t node = first + ((uint32_t)lane - nx_count);
          cp_async16(&sh.geo[cur ^ 1][lane], geo + node);
          cp_async16(&sh.mass[cur ^ 1][lane], mass + node);
          cp_async16(&sh.link[cur ^ 1][lane], link + node);
          if constexpr (QUAD) node_ids[warp][cur ^ 1][lane] = node;
        }
        if ((e.y >> lane) & 1u) nx_mine |= bit_span(nx_count, cnt);
        nx_count += cnt;
        if (!merge || sp == 0 || nx_count + (sh.stack[sp - 1].x >> FIRST_BITS) + 1u > (uint32_t)SLOTS) break;
      }
    }

    // Accepted centres of mass (tree.rs:299-305).
    for (; amask; amask &= amask - 1) {
      const int c = __ffs(amask) - 1;
      const float4 M = bmass[c];
      float s0 = __fsub_rn(M.x, x0), s1 = __fsub_rn(M.y, x1), s2 = __fsub_rn(M.z, x2);
      min_image3(s0, s1, s2, w);
      const float f = pair_factor(norm2(s0, s1, s2), -M.w, w, far);
      A0.x = fmaf(-s0, f, A0.x);
      A1.x = fmaf(-s1, f, A1.x);
      A2.x = fmaf(-s2, f, A2.x);
      if constexpr (QUAD) {
        const size_t node = node_ids[warp][cur][c];
        quad_term(s0, s1, s2, __ldg(quad + 2 * node), __ldg(quad + 2 * node + 1), w, A0, A1, A2);
      }
      ++n_accepts;
    }

    // Direct sums: the sources of all direct nodes of the step, concatenated in slot order, in
    // chunks of 32.
    const uint32_t dset = __reduce_or_sync(FULL, dmask);
    if (dset) {
      uint32_t cnt = 0, first = 0;
      if ((dset >> lane) & 1u) {
        const uint4 L = blink[lane];
        cnt = L.y - L.x;
        first = L.x;
      }
      uint32_t end = cnt;  // inclusive prefix sum over the slots
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, end, o);
        if (lane >= o) end += v;
      }
      sh.dbeg[lane] = end - cnt;
      sh.dend[lane] = end;
      sh.dsrc[lane] = first;
      const uint32_t total = __shfl_sync(FULL, end, 31);
      __syncwarp();
      // This lane's candidates, and its own particle's position in the concatenation (j != i).
      uint32_t selfpos = 0xffffffffu;
      for (uint32_t rem = dmask; rem; rem &= rem - 1) {
        const int c = __ffs(rem) - 1;
        const uint32_t b0 = sh.dbeg[c], e0 = sh.dend[c], f0 = sh.dsrc[c];
        n_cand += e0 - b0;
        if (self - f0 < e0 - b0) selfpos = b0 + (self - f0);
      }
      const bool wrap = (dmask & ~nwmask) != 0u;
      uint32_t open_d = dmask;  // this lane's direct nodes not yet wholly behind the current chunk
      for (uint32_t base = 0; base < total; base += 32) {
        // Lane q loads source base + q: node c, the last with dbeg <= base + q (binary search).
        const uint32_t g = base + (uint32_t)lane;
        if (g < total) {
          int c = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1)
            if (sh.dend[c + step - 1] <= g) c += step;
          const float4 y = __ldg(x4 + sh.dsrc[c] + (g - sh.dbeg[c]));
          sh.nx[lane] = -y.x;
          sh.ny[lane] = -y.y;
          sh.nz[lane] = -y.z;
        }
        // `live`: the chunk positions of this lane's direct nodes, without its own particle.
        const uint32_t top = base + 32u;
        uint32_t live = 0;
        while (open_d) {
          const int c = __ffs(open_d) - 1;
          const uint32_t b0 = sh.dbeg[c], e0 = sh.dend[c];
          if (b0 >= top) break;
          const uint32_t lo = max(b0, base), hi = min(e0, top);
          live |= bit_span(lo - base, hi - lo);
          if (e0 > top) break;
          open_d &= open_d - 1;
        }
        if (selfpos - base < 32u) live &= ~(1u << (selfpos - base));
        __syncwarp();
        if (live) {
          const int cnt_chunk = (int)min(32u, total - base);
          if (wrap) {
            const uint32_t pairs = chunk_candidates<true>(sh, cnt_chunk, x0, x1, x2, w) & live;
            n_pairs += __popc(pairs);
            chunk_forces<true>(sh, pairs, x0, x1, x2, w, far, A0, A1, A2);
          } else {
            const uint32_t pairs = chunk_candidates<false>(sh, cnt_chunk, x0, x1, x2, w) & live;
            n_pairs += __popc(pairs);
            chunk_forces<false>(sh, pairs, x0, x1, x2, w, far, A0, A1, A2);
          }
        }
        __syncwarp();
      }
    }
    if (nx_count == 0) break;
    b_count = nx_count;
    mine = nx_mine;
    cur ^= 1;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  // tree.rs:61-66 multiplies every pair by the coupling K; here the unit-coupling sum is scaled once
  const float kk = k_dev ? *k_dev : w.k;
  const float a0 = kk * (A0.x + A0.y), a1 = kk * (A1.x + A1.y), a2 = kk * (A2.x + A2.y);
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
    unsigned long long p = n_pairs, a = n_accepts, c = n_cand;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      p += __shfl_xor_sync(FULL, p, o);
      a += __shfl_xor_sync(FULL, a, o);
      c += __shfl_xor_sync(FULL, c, o);
    }
    if (lane == 0) {
      atomicAdd(&counters[0], p);
      atomicAdd(&counters[1], a);
      atomicAdd(&counters[2], c);
    }
  }
}

// Packs AoS positions into float4 (x, y, z, 0) for 16-byte loads.
__global__ void k_pack4(const float* __restrict__ x3, size_t n, float4* __restrict__ x4) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x4[i] = make_float4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], 0.0f);
}

// ------------------------------------------------------------------ host launch

// Fitted pair-force coefficients of one tree's last split (refitted when the split changes; a
// simulation's split is fixed, so its first step uploads them and later steps, captured graphs
// included, only read them).
struct FitCache {
  float r_split = -1.0f, r_cut = -1.0f;
  SFit fit{};
  std::vector<float> far;
  DevBuf far_dev;
};

void tree_walk_free(TreeNodes& t) {
  FitCache* fc = static_cast<FitCache*>(t.walk_fit);
  if (fc) {
    release(fc->far_dev);
    delete fc;
  }
  t.walk_fit = nullptr;
}

void launch_tree_walk(const TreeNodes& t, const float* sorted_x3, size_t n, float box, const cpm_force_split& split,
                      float k, float* acc3, int accumulate, TreeCounters* counters, DevStatus* st, cudaStream_t s,
                      const float* k_dev, const uint32_t* list, const uint32_t* list_n) {
  if (n == 0) return;
  TreeNodes& tm = const_cast<TreeNodes&>(t);
  if (!tm.walk_fit) tm.walk_fit = new FitCache();
  FitCache& fc = *static_cast<FitCache*>(tm.walk_fit);
  if (fc.r_split != split.r_split || fc.r_cut != split.r_cut || !fc.far_dev.p) {
    fc.fit = make_fit(split.r_split, split.r_cut, fc.far);
    if (ensure(fc.far_dev, fc.far.size() * sizeof(float)) != cudaSuccess) return;
    cudaMemcpy(fc.far_dev.p, fc.far.data(), fc.far.size() * sizeof(float), cudaMemcpyHostToDevice);
    fc.r_split = split.r_split;
    fc.r_cut = split.r_cut;
  }
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
  w.theta2 = split.theta * split.theta;
  w.inv_two_rs = (float)(1.0 / (2.0 * (double)split.r_split));
  w.eps2 = split.softening * split.softening;
  w.k = k;
  w.n_box = t.n_box;
  w.fit = fc.fit;
  auto dup = [](float v) { return make_float2(v, v); };
  w.p2.tiny = dup(1e-30f);
  w.p2.inv_two_rs = dup(w.inv_two_rs);
  w.p2.scale0 = dup(fc.fit.scale0);
  w.p2.offset0 = dup(fc.fit.offset0);
  for (int j = 0; j <= FIT_DEG; ++j) w.p2.c0[j] = dup(fc.fit.c0[j]);
  w.p2.neg_log2e = dup(-1.44269504f);
  w.p2.eps2 = dup(w.eps2);
  w.p2.neg_m = dup(-1.0f);
  const size_t groups = (n + 31) / 32;
  // warps per block: the autotuned group count for the plain and list walks; 4 with quadrupoles
  const int warps = t.has_quad ? 4 : (t.walk_warps == 2 || t.walk_warps == 8 ? t.walk_warps : 4);
  const unsigned blocks = (unsigned)((groups + warps - 1) / warps);
  count_launch();
  auto kernel = t.has_quad ? (list ? k_tree_walk<true, true, 4> : k_tree_walk<true, false, 4>)
              : warps == 2 ? (list ? k_tree_walk<false, true, 2> : k_tree_walk<false, false, 2>)
              : warps == 8 ? (list ? k_tree_walk<false, true, 8> : k_tree_walk<false, false, 8>)
                           : (list ? k_tree_walk<false, true, 4> : k_tree_walk<false, false, 4>);
  const size_t smem = (size_t)warps * (sizeof(WalkShared) + (t.has_quad ? 2 * SLOTS * sizeof(uint32_t) : 0));
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kernel<<<blocks, warps * 32, smem, s>>>(static_cast<const uint4*>(t.link.p), static_cast<const float4*>(t.geo.p),
                                         static_cast<const float4*>(t.mass.p), as<float4>(tm.x4), n, w,
                                         static_cast<const float*>(fc.far_dev.p), acc3, accumulate,
                                         reinterpret_cast<unsigned long long*>(counters), st, k_dev, list, list_n,
                                         t.has_quad ? static_cast<const float4*>(t.quad.p) : nullptr);
}

float quad_half_bound(const cpm_force_split& split) {
  const double th = split.theta;
  const double den = 2.0 - 2.0 * std::sqrt(3.0) * th;
  if (!(den > 0.0)) return INFINITY;
  return (float)(1.01 * th * (double)split.r_cut / den);
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
