// cpm_oracle.cpp — CPU oracle for the TreePM gravity solve (test infrastructure only).
//
// A C++17 restatement of the reference Rust crate's per-step TreePM path. Every function cites
// the reference file:line it follows. f32 expressions keep the reference's operation order; the
// file is compiled with -ffp-contract=off, so no multiply-add is fused (Rust does not fuse either).
// Parallel loops use OpenMP exactly where the reference uses rayon; loops the reference runs
// serially stay serial, so the timed CPU baseline has the reference's structure.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.

#include "cpm_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------------------------

template <typename T>
struct cpx {
  T re, im;
};

// num_complex's Mul: (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re).
template <typename T>
inline cpx<T> cmul(cpx<T> a, cpx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
inline cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
inline cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.re - b.re, a.im - b.im}; }

// i64::rem_euclid for a positive modulus.
inline int64_t rem_euclid_i64(int64_t a, int64_t n) {
  int64_t r = a % n;
  return r < 0 ? r + n : r;
}

// f32::rem_euclid (Rust std): r = self % rhs; if r < 0 { r + |rhs| } else { r }.
inline float rem_euclid_f32(float v, float rhs) {
  float r = std::fmod(v, rhs);
  return r < 0.0f ? r + std::fabs(rhs) : r;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------------------------
// mesh.rs
// ---------------------------------------------------------------------------------------------

// mesh.rs:81-83
inline float axis_weight(float f, int d) { return d == 0 ? 1.0f - f : f; }

struct Stencil {
  int64_t idx[8];
  float w[8];
};

// mesh.rs:29-59. h = L / n in f32, s = x/h - 0.5, i0 = floor(s), f = s - i0, periodic wrap of
// i0 and i0 + 1, weights multiplied x-then-y-then-z, corners ordered dx, dy, dz.
inline void stencil(int64_t n, float box, const float* x, Stencil& st) {
  const float h = box / (float)n;
  int64_t base[3];
  float frac[3];
  for (int k = 0; k < 3; ++k) {
    const float s = x[k] / h - 0.5f;
    const float i0 = std::floor(s);
    base[k] = (int64_t)i0;
    frac[k] = s - i0;
  }
  int c = 0;
  for (int dx = 0; dx < 2; ++dx)
    for (int dy = 0; dy < 2; ++dy)
      for (int dz = 0; dz < 2; ++dz) {
        const float w = axis_weight(frac[0], dx) * axis_weight(frac[1], dy) * axis_weight(frac[2], dz);
        const int64_t ix = rem_euclid_i64(base[0] + dx, n);
        const int64_t iy = rem_euclid_i64(base[1] + dy, n);
        const int64_t iz = rem_euclid_i64(base[2] + dz, n);
        st.idx[c] = (ix * n + iy) * n + iz;
        st.w[c] = w;
        ++c;
      }
}

// mesh.rs:72-77: the 8 products summed in stencil order (Rust's f32 Sum folds from -0.0).
inline float interpolate(int64_t n, float box, const float* cells, const float* x) {
  Stencil st;
  stencil(n, box, x, st);
  float sum = -0.0f;
  for (int c = 0; c < 8; ++c) sum += cells[st.idx[c]] * st.w[c];
  return sum;
}

// ---------------------------------------------------------------------------------------------
// fft.rs: unnormalised c2c transforms. The 1D lines are this project's mixed-radix Stockham FFT
// (the reference calls rustfft 6.4.1 here; its lines are not reproduced bit for bit).
// ---------------------------------------------------------------------------------------------

template <typename T>
struct LinePlan {
  int n = 0;
  int sign = -1;
  std::vector<int> radix;
  std::vector<std::vector<cpx<T>>> tw;     // per stage: tw[k*R + r] = exp(sign 2 pi i r k / (Ns R))
  std::vector<std::vector<cpx<T>>> roots;  // per stage: exp(sign 2 pi i m / R), m < R
};

template <typename T>
LinePlan<T> make_plan(int n, int sign) {
  LinePlan<T> p;
  p.n = n;
  p.sign = sign;
  int m = n;
  while (m % 4 == 0 && m > 4 && (m / 4) % 2 == 0) { p.radix.push_back(4); m /= 4; }
  for (int r : {4, 2, 3, 5, 7}) {
    while (m % r == 0) { p.radix.push_back(r); m /= r; }
  }
  for (int r = 11; m > 1; r += 2) {
    while (m % r == 0) { p.radix.push_back(r); m /= r; }
  }
  const double two_pi = 6.283185307179586476925286766559;
  int ns = 1;
  for (int R : p.radix) {
    std::vector<cpx<T>> tw((size_t)ns * R);
    for (int k = 0; k < ns; ++k)
      for (int r = 0; r < R; ++r) {
        const double ang = sign * two_pi * (double)r * (double)k / (double)(ns * R);
        tw[(size_t)k * R + r] = {(T)std::cos(ang), (T)std::sin(ang)};
      }
    std::vector<cpx<T>> rt(R);
    for (int q = 0; q < R; ++q) {
      const double ang = sign * two_pi * (double)q / (double)R;
      rt[q] = {(T)std::cos(ang), (T)std::sin(ang)};
    }
    p.tw.push_back(std::move(tw));
    p.roots.push_back(std::move(rt));
    ns *= R;
  }
  return p;
}

template <typename T>
void run_line(const LinePlan<T>& p, cpx<T>* data, cpx<T>* scratch) {
  const int n = p.n;
  if (n <= 1) return;
  cpx<T>* src = data;
  cpx<T>* dst = scratch;
  int ns = 1;
  cpx<T> v[64];
  cpx<T> y[64];
  for (size_t s = 0; s < p.radix.size(); ++s) {
    const int R = p.radix[s];
    const int m = n / R;
    const cpx<T>* tw = p.tw[s].data();
    const cpx<T>* rt = p.roots[s].data();
    for (int j = 0; j < m; ++j) {
      const int k = j % ns;
      for (int r = 0; r < R; ++r) v[r] = src[j + r * m];
      if (ns > 1)
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[(size_t)k * R + r]);
      if (R == 2) {
        y[0] = cadd(v[0], v[1]);
        y[1] = csub(v[0], v[1]);
      } else if (R == 4) {
        const cpx<T> a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const cpx<T> c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        // w d with w = exp(sign i pi / 2) = sign * i
        const cpx<T> wd = p.sign < 0 ? cpx<T>{d.im, -d.re} : cpx<T>{-d.im, d.re};
        y[0] = cadd(a, c);
        y[1] = cadd(b, wd);
        y[2] = csub(a, c);
        y[3] = csub(b, wd);
      } else {
        for (int q = 0; q < R; ++q) {
          cpx<T> acc = v[0];
          for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], rt[(r * q) % R]));
          y[q] = acc;
        }
      }
      const int base = (j / ns) * ns * R + k;
      for (int r = 0; r < R; ++r) dst[base + r * ns] = y[r];
    }
    std::swap(src, dst);
    ns *= R;
  }
  if (src != data) std::memcpy(data, src, sizeof(cpx<T>) * (size_t)n);
}

// fft.rs:76-82
inline size_t flat_index(size_t n, int axis, size_t a, size_t b, size_t t) {
  switch (axis) {
    case 0: return (t * n + a) * n + b;
    case 1: return (a * n + t) * n + b;
    default: return (a * n + b) * n + t;
  }
}

// fft.rs:40-72: z lines in place (parallel); then for axis y and x: gather lines (parallel),
// transform (parallel), scatter back (serial, as in the reference).
template <typename T>
void fft3(int n_, cpx<T>* data, int inverse) {
  const size_t n = (size_t)n_;
  const LinePlan<T> plan = make_plan<T>(n_, inverse ? 1 : -1);
#pragma omp parallel
  {
    std::vector<cpx<T>> scratch(n);
#pragma omp for schedule(static)
    for (long long l = 0; l < (long long)(n * n); ++l) run_line(plan, data + (size_t)l * n, scratch.data());
  }
  std::vector<cpx<T>> lines(n * n * n);
  for (int axis : {1, 0}) {
#pragma omp parallel
    {
      std::vector<cpx<T>> scratch(n);
#pragma omp for schedule(static)
      for (long long ab = 0; ab < (long long)(n * n); ++ab) {
        const size_t a = (size_t)ab / n, b = (size_t)ab % n;
        cpx<T>* line = lines.data() + (size_t)ab * n;
        for (size_t t = 0; t < n; ++t) line[t] = data[flat_index(n, axis, a, b, t)];
        run_line(plan, line, scratch.data());
      }
    }
    for (size_t ab = 0; ab < n * n; ++ab) {
      const size_t a = ab / n, b = ab % n;
      for (size_t t = 0; t < n; ++t) data[flat_index(n, axis, a, b, t)] = lines[ab * n + t];
    }
  }
}

// fft.rs:86-95. 2 pi / L with pi rounded to f32 first; the Nyquist index of an even grid is 0.
inline float wavenumber(size_t i, size_t n, float box) {
  const float two_pi_over_l = 2.0f * (float)3.14159265358979323846 / box;
  if (n % 2 == 0 && i == n / 2) return 0.0f;
  if (i <= n / 2) return (float)i * two_pi_over_l;
  return ((float)i - (float)n) * two_pi_over_l;
}

// ---------------------------------------------------------------------------------------------
// tree.rs
// ---------------------------------------------------------------------------------------------

constexpr size_t LEAF_SIZE = 8;          // tree.rs:12
constexpr uint32_t MAX_DEPTH = 40;       // tree.rs:13
constexpr uint32_t NO_CHILD = 0xFFFFFFFFu;
constexpr float SQRT_3 = 1.7320508f;     // tree.rs:15
constexpr float TWO_OVER_SQRT_PI = 1.1283792f;  // tree.rs:17

// tree.rs:54-57
inline float short_range_factor(float r, float r_split) {
  const float u = r / (2.0f * r_split);
  return erfcf(u) + TWO_OVER_SQRT_PI * u * std::exp(-u * u);
}

inline float norm2(const float* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }

// tree.rs:61-66
inline void pair(const float* d, float mass, float k, const orc_split& s, float* out) {
  const float r2 = norm2(d);
  const float sf = r2 + s.softening * s.softening;
  const float f = -k * mass * short_range_factor(std::sqrt(r2), s.r_split) / (sf * std::sqrt(sf));
  out[0] = d[0] * f;
  out[1] = d[1] * f;
  out[2] = d[2] * f;
}

inline void add_to(float* acc, const float* v) {
  acc[0] += v[0];
  acc[1] += v[1];
  acc[2] += v[2];
}

struct Node {  // tree.rs:68-80
  float center[3];
  float half;
  float com[3];
  uint32_t count;
  uint32_t children[8];
  uint32_t start, end;
  uint32_t depth;  // recorded for introspection only
};

struct Tree {
  const float* pos;  // AoS [n][3]
  float box;
  int com_f64 = 0;   // 0: f32 sequential sum (tree.rs:190-200); 1: FP64 sum rounded once (diagnostic)
  std::vector<uint32_t> order;
  std::vector<Node> nodes;

  // tree.rs:171-183
  void build(const float* positions, size_t n, float box_size) {
    pos = positions;
    box = box_size;
    order.resize(n);
    std::iota(order.begin(), order.end(), 0u);
    nodes.clear();
    nodes.reserve(2 * n / LEAF_SIZE + 1);
    const float half = box_size / 2.0f;
    const float c[3] = {half, half, half};
    build_node(0, n, c, half, 0);
  }

  // tree.rs:186-250
  uint32_t build_node(size_t start, size_t end, const float* center, float half, uint32_t depth) {
    const uint32_t idx = (uint32_t)nodes.size();
    float com[3] = {0.0f, 0.0f, 0.0f};
    if (com_f64) {
      double sd[3] = {0.0, 0.0, 0.0};
      for (size_t t = start; t < end; ++t) {
        const float* p = pos + 3 * (size_t)order[t];
        for (int k = 0; k < 3; ++k) sd[k] += (double)p[k];
      }
      for (int k = 0; k < 3; ++k) com[k] = (float)(sd[k] / (double)(end - start));
    } else {
      for (size_t t = start; t < end; ++t) {
        const float* p = pos + 3 * (size_t)order[t];
        for (int k = 0; k < 3; ++k) com[k] += p[k];
      }
      const float count = (float)(end - start);
      for (int k = 0; k < 3; ++k) com[k] /= count;
    }
    Node nd;
    for (int k = 0; k < 3; ++k) {
      nd.center[k] = center[k];
      nd.com[k] = com[k];
    }
    nd.half = half;
    nd.count = (uint32_t)(end - start);
    for (int o = 0; o < 8; ++o) nd.children[o] = NO_CHILD;
    nd.start = (uint32_t)start;
    nd.end = (uint32_t)end;
    nd.depth = depth;
    nodes.push_back(nd);

    if (end - start <= LEAF_SIZE || depth >= MAX_DEPTH) return idx;

    auto octant = [&](const float* p) {
      return (size_t)(p[0] >= center[0]) | ((size_t)(p[1] >= center[1]) << 1) |
             ((size_t)(p[2] >= center[2]) << 2);
    };
    size_t counts[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t t = start; t < end; ++t) counts[octant(pos + 3 * (size_t)order[t])] += 1;
    size_t offsets[8];
    size_t running = start;
    for (int o = 0; o < 8; ++o) {
      offsets[o] = running;
      running += counts[o];
    }
    size_t next[8];
    std::memcpy(next, offsets, sizeof(next));
    std::vector<uint32_t> sorted(end - start);
    for (size_t t = start; t < end; ++t) {
      const uint32_t j = order[t];
      const size_t o = octant(pos + 3 * (size_t)j);
      sorted[next[o] - start] = j;
      next[o] += 1;
    }
    std::copy(sorted.begin(), sorted.end(), order.begin() + (long)start);

    const float quarter = half / 2.0f;
    for (int o = 0; o < 8; ++o) {
      if (counts[o] == 0) continue;
      float cc[3];
      for (int k = 0; k < 3; ++k) cc[k] = center[k] + (((o >> k) & 1) == 1 ? quarter : -quarter);
      const uint32_t child = build_node(offsets[o], offsets[o] + counts[o], cc, quarter, depth + 1);
      nodes[idx].children[o] = child;
    }
    return idx;
  }

  // tree.rs:253-261 (Tree::min_image divides by L)
  inline void min_image(const float* a, const float* b, float* d) const {
    const float l = box;
    for (int k = 0; k < 3; ++k) {
      const float x = a[k] - b[k];
      d[k] = x - l * std::round(x / l);
    }
  }

  // tree.rs:264-310 (Tree::accel_on: opening test 2 half < theta r)
  void accel_on(size_t i, const orc_split& s, float k, std::vector<uint32_t>& stack, float* acc,
                uint64_t* stats) const {
    const float* xi = pos + 3 * i;
    const float cut2 = s.r_cut * s.r_cut;
    acc[0] = acc[1] = acc[2] = 0.0f;
    stack.clear();
    stack.push_back(0);
    while (!stack.empty()) {
      const uint32_t n = stack.back();
      stack.pop_back();
      const Node& node = nodes[n];
      if (stats) stats[2] += 1;
      float to_centre[3];
      min_image(node.center, xi, to_centre);
      const float max_r = s.r_cut + SQRT_3 * node.half;
      if (norm2(to_centre) > max_r * max_r) continue;
      if (node.children[0] == NO_CHILD) {
        for (uint32_t t = node.start; t < node.end; ++t) {
          const size_t j = order[t];
          if (j == i) continue;
          float d[3];
          min_image(xi, pos + 3 * j, d);
          if (norm2(d) > cut2) continue;
          float v[3];
          pair(d, 1.0f, k, s, v);
          add_to(acc, v);
          if (stats) stats[0] += 1;
        }
      } else {
        float to_com[3];
        min_image(node.com, xi, to_com);
        const float r = std::sqrt(norm2(to_com));
        if (2.0f * node.half < s.theta * r) {
          const float d[3] = {-to_com[0], -to_com[1], -to_com[2]};
          float v[3];
          pair(d, (float)node.count, k, s, v);
          add_to(acc, v);
          if (stats) stats[1] += 1;
        } else {
          for (int o = 0; o < 8; ++o)
            if (node.children[o] != NO_CHILD) stack.push_back(node.children[o]);
        }
      }
    }
  }

  // tree.rs:103-150 (BuiltTree::accel_on: multiplies by 1/L, opening test 4 half^2 < theta^2 r^2)
  void accel_on_built(size_t i, const orc_split& s, float k, std::vector<uint32_t>& stack,
                      float* acc) const {
    const float* xi = pos + 3 * i;
    const float inv_l = 1.0f / box;
    auto mi = [&](const float* a, const float* b, float* d) {
      for (int q = 0; q < 3; ++q) {
        const float x = a[q] - b[q];
        d[q] = x - box * std::round(x * inv_l);
      }
    };
    const float cut2 = s.r_cut * s.r_cut;
    const float theta2 = s.theta * s.theta;
    acc[0] = acc[1] = acc[2] = 0.0f;
    stack.clear();
    stack.push_back(0);
    while (!stack.empty()) {
      const uint32_t n = stack.back();
      stack.pop_back();
      const Node& node = nodes[n];
      float to_centre[3];
      mi(node.center, xi, to_centre);
      const float max_r = s.r_cut + SQRT_3 * node.half;
      if (norm2(to_centre) > max_r * max_r) continue;
      if (node.children[0] == NO_CHILD) {
        for (uint32_t t = node.start; t < node.end; ++t) {
          const size_t j = order[t];
          if (j == i) continue;
          float d[3];
          mi(xi, pos + 3 * j, d);
          if (norm2(d) > cut2) continue;
          float v[3];
          pair(d, 1.0f, k, s, v);
          add_to(acc, v);
        }
      } else {
        float to_com[3];
        mi(node.com, xi, to_com);
        const float r2 = norm2(to_com);
        if (4.0f * node.half * node.half < theta2 * r2) {
          const float d[3] = {-to_com[0], -to_com[1], -to_com[2]};
          float v[3];
          pair(d, (float)node.count, k, s, v);
          add_to(acc, v);
        } else {
          for (int o = 0; o < 8; ++o)
            if (node.children[o] != NO_CHILD) stack.push_back(node.children[o]);
        }
      }
    }
  }
};

// tree.rs:314-323: build (serial), then a parallel walk per particle.
void tree_accelerations(const float* x3, size_t n, float box, const orc_split& s, float k, float* acc3,
                        double* t_build, double* t_walk) {
  const double t0 = now_s();
  Tree tree;
  tree.build(x3, n, box);
  const double t1 = now_s();
#pragma omp parallel
  {
    std::vector<uint32_t> stack;
    stack.reserve(64);
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i) tree.accel_on((size_t)i, s, k, stack, acc3 + 3 * (size_t)i, nullptr);
  }
  const double t2 = now_s();
  if (t_build) *t_build = t1 - t0;
  if (t_walk) *t_walk = t2 - t1;
}

// ---------------------------------------------------------------------------------------------
// cosmology.rs
// ---------------------------------------------------------------------------------------------

constexpr int GROWTH_STEPS = 4000;  // cosmology.rs:7

// cosmology.rs:32-34
inline float cosmo_e(const orc_cosmology& c, float a) {
  return std::sqrt(c.omega_r / (a * a * a * a) + c.omega_m / (a * a * a) + c.omega_l);
}

// cosmology.rs:47-79: f32 RK4 in ln a from a = 1e-3 with the Meszaros start.
void growth_state(const orc_cosmology& c, float a_end, float* d_out, float* dl_out) {
  const float a_start = 1e-3f;
  float d, dl;
  if (c.omega_r > 0.0f) {
    const float y = a_start * c.omega_m / c.omega_r;
    d = 1.0f + 1.5f * y;
    dl = 1.5f * y;
  } else {
    d = a_start;
    dl = a_start;
  }
  auto rhs = [&](float la, float dd, float dll, float* o0, float* o1) {
    const float a = std::exp(la);
    const float e2 = c.omega_r / (a * a * a * a) + c.omega_m / (a * a * a) + c.omega_l;
    const float dln_e = 0.5f * (-4.0f * c.omega_r / (a * a * a * a) - 3.0f * c.omega_m / (a * a * a)) / e2;
    const float source = 1.5f * c.omega_m / (a * a * a * e2) * dd;
    *o0 = dll;
    *o1 = -(2.0f + dln_e) * dll + source;
  };
  const float la0 = std::log(a_start);
  const float h = (std::log(a_end) - la0) / (float)GROWTH_STEPS;
  for (int step = 0; step < GROWTH_STEPS; ++step) {
    const float la = la0 + (float)step * h;
    float k1d, k1l, k2d, k2l, k3d, k3l, k4d, k4l;
    rhs(la, d, dl, &k1d, &k1l);
    rhs(la + 0.5f * h, d + 0.5f * h * k1d, dl + 0.5f * h * k1l, &k2d, &k2l);
    rhs(la + 0.5f * h, d + 0.5f * h * k2d, dl + 0.5f * h * k2l, &k3d, &k3l);
    rhs(la + h, d + h * k3d, dl + h * k3l, &k4d, &k4l);
    d += h / 6.0f * (k1d + 2.0f * k2d + 2.0f * k3d + k4d);
    dl += h / 6.0f * (k1l + 2.0f * k2l + 2.0f * k3l + k4l);
  }
  *d_out = d;
  *dl_out = dl;
}

// ---------------------------------------------------------------------------------------------
// integrator.rs step factors
// ---------------------------------------------------------------------------------------------

constexpr int STEP_INTEGRAL_STEPS = 64;   // integrator.rs:19
constexpr int MIDPOINT_ITERATIONS = 60;   // integrator.rs:21

// integrator.rs:288-297
template <typename F>
float simpson(float lo, float hi, F f) {
  const int n = STEP_INTEGRAL_STEPS;
  const float h = (hi - lo) / (float)n;
  float sum = f(lo) + f(hi);
  for (int i = 1; i < n; ++i) {
    const float weight = (i % 2 == 1) ? 4.0f : 2.0f;
    sum += weight * f(lo + (float)i * h);
  }
  return sum * h / 3.0f;
}

float kick_factor(const orc_cosmology& c, float a0, float a1) {  // :263-265
  return simpson(a0, a1, [&](float a) { return 1.0f / (a * cosmo_e(c, a)); });
}
float drift_factor(const orc_cosmology& c, float a0, float a1) {  // :268-270
  return simpson(a0, a1, [&](float a) { return 1.0f / (a * a * a * cosmo_e(c, a)); });
}
float midpoint(const orc_cosmology& c, float a0, float a1) {  // :273-285
  const float half = kick_factor(c, a0, a1) / 2.0f;
  float lo = a0, hi = a1;
  for (int it = 0; it < MIDPOINT_ITERATIONS; ++it) {
    const float mid = 0.5f * (lo + hi);
    if (kick_factor(c, a0, mid) < half)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5f * (lo + hi);
}

// integrator.rs:301-307 (serial)
void kick(float* p3, const float* g3, size_t n, float factor) {
  for (size_t i = 0; i < 3 * n; ++i) p3[i] += g3[i] * factor;
}
// integrator.rs:310-316 (serial)
void drift(float* x3, const float* p3, size_t n, float factor, float box) {
  for (size_t i = 0; i < 3 * n; ++i) x3[i] = rem_euclid_f32(x3[i] + p3[i] * factor, box);
}

// ---------------------------------------------------------------------------------------------
// poisson.rs:33-88
// ---------------------------------------------------------------------------------------------

// Per-axis 1 / sinc^4(pi m / n) (the CIC window of deposit and gather, squared), built in double and
// rounded to f32. No counterpart in the reference, which does not deconvolve (poisson.rs:52-74); this
// is the factor of the library's optional deconvolved Green's function.
std::vector<float> cic_deconvolution_table(int n) {
  std::vector<float> dc((size_t)n);
  for (int i = 0; i < n; ++i) {
    const int m = i <= n / 2 ? i : i - n;
    const double x = 3.14159265358979323846 * (double)m / (double)n;
    const double s = m == 0 ? 1.0 : std::sin(x) / x;
    dc[(size_t)i] = (float)(1.0 / (s * s * s * s));
  }
  return dc;
}

// poisson.rs:33-88; with `deconvolve`, the Green's function of each mode is multiplied by
// (d[ix] * d[iy]) * d[iz] from cic_deconvolution_table (f32 products in that order).
void poisson_accel(int n_, float box, const float* delta, float omega_m, float a, float r_split, float* gx,
                   float* gy, float* gz, int deconvolve = 0) {
  const size_t n = (size_t)n_;
  const size_t n3 = n * n * n;
  std::vector<cpx<float>> delta_k(n3);
  for (size_t i = 0; i < n3; ++i) delta_k[i] = {delta[i], 0.0f};
  fft3<float>(n_, delta_k.data(), 0);

  const float prefactor = 1.5f * omega_m / a;
  const std::vector<float> dc = deconvolve ? cic_deconvolution_table(n_) : std::vector<float>();
  std::vector<cpx<float>> accel_k[3];
  for (int ax = 0; ax < 3; ++ax) accel_k[ax].assign(n3, cpx<float>{0.0f, 0.0f});
  for (size_t ix = 0; ix < n; ++ix)
    for (size_t iy = 0; iy < n; ++iy)
      for (size_t iz = 0; iz < n; ++iz) {
        const size_t idx = (ix * n + iy) * n + iz;
        const float k[3] = {wavenumber(ix, n, box), wavenumber(iy, n, box), wavenumber(iz, n, box)};
        float k2 = -0.0f;
        for (int q = 0; q < 3; ++q) k2 += k[q] * k[q];
        if (k2 == 0.0f) continue;
        const float filter = std::exp(-k2 * r_split * r_split);
        float sc = -prefactor / k2 * filter;
        if (deconvolve) sc = sc * ((dc[ix] * dc[iy]) * dc[iz]);
        const cpx<float> phi = {delta_k[idx].re * sc, delta_k[idx].im * sc};
        for (int ax = 0; ax < 3; ++ax) accel_k[ax][idx] = cmul(phi, cpx<float>{0.0f, -k[ax]});
      }
  const float scale = 1.0f / (float)(n * n * n);
  float* outs[3] = {gx, gy, gz};
  for (int ax = 0; ax < 3; ++ax) {
    fft3<float>(n_, accel_k[ax].data(), 1);
    for (size_t i = 0; i < n3; ++i) outs[ax][i] = accel_k[ax][i].re * scale;
  }
}

// ---------------------------------------------------------------------------------------------
// ics.rs
// ---------------------------------------------------------------------------------------------

float bbks(const orc_cosmology& c, float k) {  // cosmology.rs:94-103
  const float h = c.h0 / 100.0f;
  const float q = k / (c.omega_m * h);
  if (q == 0.0f) return 1.0f;
  const float x2 = 16.1f * q, x3 = 5.46f * q, x4 = 6.71f * q;
  const float p2 = x2 * x2;
  const float p3 = x3 * (x3 * x3);
  const float x4s = x4 * x4;
  const float p4 = x4s * x4s;
  const float poly = 1.0f + 3.89f * q + p2 + p3 + p4;
  return std::log1p(2.34f * q) / (2.34f * q) * std::pow(poly, -0.25f);
}

float power(const orc_cosmology& c, const orc_pspec& ps, float k) {  // ics.rs:27-33
  if (k == 0.0f) return 0.0f;
  const float t = bbks(c, k);
  return ps.amplitude * std::pow(k, ps.n_s) * t * t;
}

float tophat(float x) {  // ics.rs:68-73
  if (x < 1e-4f) return 1.0f;
  return 3.0f * (std::sin(x) - x * std::cos(x)) / (x * x * x);
}

float sigma(const orc_cosmology& c, const orc_pspec& ps, float radius) {  // ics.rs:36-52
  const int steps = 8192;
  const float ln_lo = std::log(1e-4f), ln_hi = std::log(1e3f);
  const float h = (ln_hi - ln_lo) / (float)steps;
  auto integrand = [&](float ln_k) {
    const float k = std::exp(ln_k);
    const float w = tophat(k * radius);
    const float k3 = k * (k * k);
    return k3 * power(c, ps, k) * w * w;
  };
  float sum = integrand(ln_lo) + integrand(ln_hi);
  for (int i = 1; i < steps; ++i) {
    const float weight = (i % 2 == 1) ? 4.0f : 2.0f;
    sum += weight * integrand(ln_lo + (float)i * h);
  }
  const float integral = sum * h / 3.0f;
  const double pi = 3.14159265358979323846;
  return std::sqrt(integral / (2.0f * (float)(pi * pi)));
}

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter = (cell, 0, 0, 0), key = seed.
inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// One N(0,1) value per cell: Box-Muller on the first two Philox words, in double, rounded to f32.
inline float white_noise_cell(uint64_t cell, uint64_t seed) {
  uint32_t c[4] = {(uint32_t)cell, (uint32_t)(cell >> 32), 0u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u1 = ((double)c[0] + 1.0) * (1.0 / 4294967296.0);  // (0, 1]
  const double u2 = (double)c[1] * (1.0 / 4294967296.0);          // [0, 1)
  return (float)(std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925286766559 * u2));
}

// ics.rs:78-109
void colored_modes(int n_, float box, const orc_cosmology& c, const orc_pspec& ps, uint64_t seed,
                   cpx<float>* modes) {
  const size_t n = (size_t)n_;
  const size_t n3 = n * n * n;
  const float volume = box * box * box;
  for (size_t i = 0; i < n3; ++i) modes[i] = {white_noise_cell(i, seed), 0.0f};
  fft3<float>(n_, modes, 0);
  for (size_t ix = 0; ix < n; ++ix)
    for (size_t iy = 0; iy < n; ++iy)
      for (size_t iz = 0; iz < n; ++iz) {
        const size_t idx = (ix * n + iy) * n + iz;
        const float k[3] = {wavenumber(ix, n, box), wavenumber(iy, n, box), wavenumber(iz, n, box)};
        float ksq = -0.0f;
        for (int q = 0; q < 3; ++q) ksq += k[q] * k[q];
        const float k_mag = std::sqrt(ksq);
        if (k_mag == 0.0f) {
          modes[idx] = {0.0f, 0.0f};
        } else {
          const float sc = std::sqrt((float)n3 * power(c, ps, k_mag) / volume);
          modes[idx] = {modes[idx].re * sc, modes[idx].im * sc};
        }
      }
}

}  // namespace

// =============================================================================================
// Exported C ABI
// =============================================================================================

extern "C" {

// mesh.rs:90-99
void orc_scattered_mesh(size_t count, float box, float* out3) {
  uint64_t state = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < 3 * count; ++i) {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    out3[i] = (float)(state >> 11) / (float)(1ull << 53) * box;
  }
}

// tree.rs:340-349
void orc_scattered_tree(size_t count, float box, uint64_t seed, float* out3) {
  uint64_t state = seed;
  for (size_t i = 0; i < 3 * count; ++i) {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    out3[i] = (float)(state >> 40) / (float)(1ull << 24) * box;
  }
}

void orc_stencil(int n, float box, const float* x3, int64_t* idx8, float* w8) {
  Stencil st;
  stencil(n, box, x3, st);
  for (int c = 0; c < 8; ++c) {
    idx8[c] = st.idx[c];
    w8[c] = st.w[c];
  }
}

// mesh.rs:62-69 (serial)
void orc_deposit(int n, float box, const float* x3, size_t np, float mass, float* cells) {
  const size_t m = (size_t)n * n * n;
  std::fill(cells, cells + m, 0.0f);
  Stencil st;
  for (size_t i = 0; i < np; ++i) {
    stencil(n, box, x3 + 3 * i, st);
    for (int c = 0; c < 8; ++c) cells[st.idx[c]] += mass * st.w[c];
  }
}

void orc_deposit_f64(int n, float box, const float* x3, size_t np, float mass, double* cells) {
  const size_t m = (size_t)n * n * n;
  std::fill(cells, cells + m, 0.0);
  Stencil st;
  for (size_t i = 0; i < np; ++i) {
    stencil(n, box, x3 + 3 * i, st);
    for (int c = 0; c < 8; ++c) cells[st.idx[c]] += (double)(mass * st.w[c]);
  }
}

float orc_interpolate(int n, float box, const float* cells, const float* x3) {
  return interpolate(n, box, cells, x3);
}

void orc_interpolate_many(int n, float box, const float* cells, const float* x3, size_t np, float* out) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)np; ++i) out[i] = interpolate(n, box, cells, x3 + 3 * (size_t)i);
}

// integrator.rs:117-126
void orc_density_contrast(int n, float box, const float* x3, size_t np, float* delta) {
  orc_deposit(n, box, x3, np, 1.0f, delta);
  const size_t m = (size_t)n * n * n;
  const float cells = (float)m;
  const float mean = (float)np / cells;
  for (size_t i = 0; i < m; ++i) delta[i] = delta[i] / mean - 1.0f;
}

void orc_fft3(int n, float* data, int inverse) { fft3<float>(n, reinterpret_cast<cpx<float>*>(data), inverse); }
void orc_fft3_f64(int n, double* data, int inverse) {
  fft3<double>(n, reinterpret_cast<cpx<double>*>(data), inverse);
}
float orc_wavenumber(size_t i, size_t n, float box) { return wavenumber(i, n, box); }

void orc_poisson_accel(int n, float box, const float* delta, float omega_m, float a, float r_split, float* gx,
                       float* gy, float* gz) {
  poisson_accel(n, box, delta, omega_m, a, r_split, gx, gy, gz);
}

void orc_poisson_accel_deconvolved(int n, float box, const float* delta, float omega_m, float a, float r_split,
                                   float* gx, float* gy, float* gz) {
  poisson_accel(n, box, delta, omega_m, a, r_split, gx, gy, gz, 1);
}

// tree.rs:40-50
orc_split orc_split_with(float box, size_t mesh_n, size_t pps, float soft_scale, float theta) {
  const float cell = box / (float)mesh_n;
  const float r_split = 1.25f * cell;
  const float spacing = box / (float)pps;
  orc_split s;
  s.r_split = r_split;
  s.r_cut = 4.5f * r_split;
  s.softening = soft_scale * spacing;
  s.theta = theta;
  return s;
}

float orc_short_range_factor(float r, float r_split) { return short_range_factor(r, r_split); }

void orc_tree_accelerations(const float* x3, size_t n, float box, const orc_split* s, float k, float* acc3) {
  tree_accelerations(x3, n, box, *s, k, acc3, nullptr, nullptr);
}

// Diagnostic twin of orc_tree_accelerations with the centre of mass summed in FP64.
void orc_tree_accelerations_com64(const float* x3, size_t n, float box, const orc_split* s, float k, float* acc3) {
  Tree tree;
  tree.com_f64 = 1;
  tree.build(x3, n, box);
#pragma omp parallel
  {
    std::vector<uint32_t> stack;
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i) tree.accel_on((size_t)i, *s, k, stack, acc3 + 3 * (size_t)i, nullptr);
  }
}

void orc_tree_accelerations_builtin(const float* x3, size_t n, float box, const orc_split* s, float k,
                                    float* acc3) {
  Tree tree;
  tree.build(x3, n, box);
#pragma omp parallel
  {
    std::vector<uint32_t> stack;
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i) tree.accel_on_built((size_t)i, *s, k, stack, acc3 + 3 * (size_t)i);
  }
}

// tree.rs:352-370
void orc_brute_force(const float* x3, size_t n, float box, const orc_split* s, float k, float* acc3) {
  Tree tree;
  tree.pos = x3;
  tree.box = box;
  const float cut2 = s->r_cut * s->r_cut;
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)n; ++ii) {
    const size_t i = (size_t)ii;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      float d[3];
      tree.min_image(x3 + 3 * i, x3 + 3 * j, d);
      if (norm2(d) > cut2) continue;
      float v[3];
      pair(d, 1.0f, k, *s, v);
      add_to(acc, v);
    }
    for (int q = 0; q < 3; ++q) acc3[3 * i + q] = acc[q];
  }
}

size_t orc_tree_build(const float* x3, size_t n, float box, float* center3, float* half, float* com3,
                      uint32_t* count, uint32_t* start, uint32_t* end, uint32_t* children8, uint32_t* depth,
                      uint32_t* order) {
  Tree tree;
  tree.build(x3, n, box);
  const size_t nn = tree.nodes.size();
  for (size_t i = 0; i < nn; ++i) {
    const Node& d = tree.nodes[i];
    if (center3)
      for (int k = 0; k < 3; ++k) center3[3 * i + k] = d.center[k];
    if (half) half[i] = d.half;
    if (com3)
      for (int k = 0; k < 3; ++k) com3[3 * i + k] = d.com[k];
    if (count) count[i] = d.count;
    if (start) start[i] = d.start;
    if (end) end[i] = d.end;
    if (children8)
      for (int o = 0; o < 8; ++o) children8[8 * i + o] = d.children[o];
    if (depth) depth[i] = d.depth;
  }
  if (order) std::copy(tree.order.begin(), tree.order.end(), order);
  return nn;
}

void orc_tree_walk_stats(const float* x3, size_t n, float box, const orc_split* s, uint64_t* leaf_pairs,
                         uint64_t* node_accepts, uint64_t* nodes_visited) {
  Tree tree;
  tree.build(x3, n, box);
  uint64_t a = 0, b = 0, c = 0;
#pragma omp parallel reduction(+ : a, b, c)
  {
    std::vector<uint32_t> stack;
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i) {
      uint64_t st[3] = {0, 0, 0};
      float acc[3];
      tree.accel_on((size_t)i, *s, 1.0f, stack, acc, st);
      a += st[0];
      b += st[1];
      c += st[2];
    }
  }
  *leaf_pairs = a;
  *node_accepts = b;
  *nodes_visited = c;
}

// Octant digits along the descent of tree.rs:186-250: at each depth, octant = (x >= cx) | (y >= cy) << 1 |
// (z >= cz) << 2 against the node centre; the child centre is centre +- half/2 in f32.
void orc_octant_keys(const float* x3, size_t n, float box, int levels, uint64_t* keys) {
#pragma omp parallel for schedule(static)
  for (long long ii = 0; ii < (long long)n; ++ii) {
    const float* p = x3 + 3 * (size_t)ii;
    float half = box / 2.0f;
    float c[3] = {half, half, half};
    uint64_t key = 0;
    for (int d = 0; d < levels; ++d) {
      const uint32_t o = (uint32_t)(p[0] >= c[0]) | ((uint32_t)(p[1] >= c[1]) << 1) | ((uint32_t)(p[2] >= c[2]) << 2);
      key = (key << 3) | o;
      const float quarter = half / 2.0f;
      for (int k = 0; k < 3; ++k) c[k] = c[k] + (((o >> k) & 1) ? quarter : -quarter);
      half = quarter;
    }
    keys[ii] = key;
  }
}

void orc_stable_sort_perm(const uint64_t* keys, size_t n, uint32_t* perm) {
  std::vector<uint32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
  std::copy(idx.begin(), idx.end(), perm);
}

float orc_cosmo_e(const orc_cosmology* c, float a) { return cosmo_e(*c, a); }
float orc_growth(const orc_cosmology* c, float a) {
  float d, dl, d1, dl1;
  growth_state(*c, a, &d, &dl);
  growth_state(*c, 1.0f, &d1, &dl1);
  return d / d1;
}
float orc_growth_rate(const orc_cosmology* c, float a) {
  float d, dl;
  growth_state(*c, a, &d, &dl);
  return dl / d;
}
float orc_bbks(const orc_cosmology* c, float k) { return bbks(*c, k); }
orc_cosmology orc_lcdm_default(void) {  // cosmology.rs:21-29
  const float omega_r = 9.14e-5f;
  orc_cosmology c;
  c.omega_r = omega_r;
  c.omega_m = 0.315f;
  c.omega_l = 1.0f - 0.315f - omega_r;
  c.h0 = 67.4f;
  return c;
}

float orc_kick_factor(const orc_cosmology* c, float a0, float a1) { return kick_factor(*c, a0, a1); }
float orc_drift_factor(const orc_cosmology* c, float a0, float a1) { return drift_factor(*c, a0, a1); }
float orc_midpoint(const orc_cosmology* c, float a0, float a1) { return midpoint(*c, a0, a1); }
void orc_kick(float* p3, const float* g3, size_t n, float factor) { kick(p3, g3, n, factor); }
void orc_drift(float* x3, const float* p3, size_t n, float factor, float box) { drift(x3, p3, n, factor, box); }

// integrator.rs:34-51
struct orc_sim {
  orc_cosmology cosmo;
  float box;
  int mesh_n;
  std::vector<float> x, p, acc, delta;
  float a;
  bool has_split;
  orc_split split;
  double t[6];
};

// integrator.rs:140-161
static void sim_accelerations(const orc_sim* s, float a, float* acc, float* delta, double* t) {
  const size_t np = s->x.size() / 3;
  const int n = s->mesh_n;
  const size_t m = (size_t)n * n * n;
  const double t0 = now_s();
  orc_density_contrast(n, s->box, s->x.data(), np, delta);
  const double t1 = now_s();
  const float r_split = s->has_split ? s->split.r_split : 0.0f;
  std::vector<float> g(3 * m);
  poisson_accel(n, s->box, delta, s->cosmo.omega_m, a, r_split, g.data(), g.data() + m, g.data() + 2 * m);
  const double t2 = now_s();
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)np; ++i) {
    const float* xi = s->x.data() + 3 * (size_t)i;
    for (int q = 0; q < 3; ++q) acc[3 * (size_t)i + q] = interpolate(n, s->box, g.data() + (size_t)q * m, xi);
  }
  const double t3 = now_s();
  double tb = 0.0, tw = 0.0;
  if (s->has_split) {
    const float nf = (float)np;
    const float L = s->box;
    const float k = 1.5f * s->cosmo.omega_m * (L * L * L) / (4.0f * (float)3.14159265358979323846 * a * nf);
    std::vector<float> sr(3 * np);
    tree_accelerations(s->x.data(), np, s->box, s->split, k, sr.data(), &tb, &tw);
    for (size_t i = 0; i < 3 * np; ++i) acc[i] += sr[i];
  }
  if (t) {
    t[1] = t1 - t0;
    t[2] = t2 - t1;
    t[3] = t3 - t2;
    t[4] = tb;
    t[5] = tw;
  }
}

orc_sim* orc_sim_new(const orc_cosmology* c, float box, int mesh_n, const float* x3, const float* p3, size_t n,
                     float a, const orc_split* split) {
  orc_sim* s = new orc_sim();
  s->cosmo = *c;
  s->box = box;
  s->mesh_n = mesh_n;
  s->x.assign(x3, x3 + 3 * n);
  s->p.assign(p3, p3 + 3 * n);
  s->acc.assign(3 * n, 0.0f);
  s->delta.assign((size_t)mesh_n * mesh_n * mesh_n, 0.0f);
  s->a = a;
  s->has_split = split != nullptr;
  if (split) s->split = *split;
  for (double& v : s->t) v = 0.0;
  sim_accelerations(s, a, s->acc.data(), s->delta.data(), nullptr);
  return s;
}

// integrator.rs:174-186
void orc_sim_step_to(orc_sim* s, float a1) {
  const size_t np = s->x.size() / 3;
  const double t0 = now_s();
  const float a0 = s->a;
  const float am = midpoint(s->cosmo, a0, a1);
  const float k1 = kick_factor(s->cosmo, a0, am);
  kick(s->p.data(), s->acc.data(), np, k1);
  const float d = drift_factor(s->cosmo, a0, a1);
  drift(s->x.data(), s->p.data(), np, d, s->box);
  const double t1 = now_s();
  sim_accelerations(s, a1, s->acc.data(), s->delta.data(), s->t);
  const double t2 = now_s();
  const float k2 = kick_factor(s->cosmo, am, a1);
  kick(s->p.data(), s->acc.data(), np, k2);
  s->a = a1;
  const double t3 = now_s();
  s->t[0] = (t1 - t0) + (t3 - t2);
}

void orc_sim_get(const orc_sim* s, float* x3, float* p3, float* acc3, float* delta, float* a) {
  if (x3) std::copy(s->x.begin(), s->x.end(), x3);
  if (p3) std::copy(s->p.begin(), s->p.end(), p3);
  if (acc3) std::copy(s->acc.begin(), s->acc.end(), acc3);
  if (delta) std::copy(s->delta.begin(), s->delta.end(), delta);
  if (a) *a = s->a;
}

void orc_sim_accelerations(const orc_sim* s, float a, float* acc3, float* delta) {
  std::vector<float> dtmp;
  if (!delta) {
    dtmp.resize((size_t)s->mesh_n * s->mesh_n * s->mesh_n);
    delta = dtmp.data();
  }
  sim_accelerations(s, a, acc3, delta, nullptr);
}

void orc_sim_free(orc_sim* s) { delete s; }

void orc_sim_last_timings(const orc_sim* s, double* t6) {
  for (int i = 0; i < 6; ++i) t6[i] = s->t[i];
}

void orc_step_sample(const orc_cosmology* c, float box, int mesh_n, const float* x3, const float* p3,
                     const float* acc3, size_t n, float a0, float a1, const orc_split* split,
                     const uint32_t* subset, size_t m, int threads, double* t7, float* acc_subset,
                     float* acc_subset_com64) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  std::vector<float> x(x3, x3 + 3 * n), p(p3, p3 + 3 * n);
  const size_t mm = (size_t)mesh_n * mesh_n * mesh_n;
  std::vector<float> delta(mm), g(3 * mm), acc(3 * n);
  const double t0 = now_s();
  const float am = midpoint(*c, a0, a1);
  const float k1 = kick_factor(*c, a0, am);
  kick(p.data(), acc3, n, k1);
  const float d = drift_factor(*c, a0, a1);
  drift(x.data(), p.data(), n, d, box);
  const double t1 = now_s();
  orc_density_contrast(mesh_n, box, x.data(), n, delta.data());
  const double t2 = now_s();
  poisson_accel(mesh_n, box, delta.data(), c->omega_m, a1, split ? split->r_split : 0.0f, g.data(), g.data() + mm,
                g.data() + 2 * mm);
  const double t3 = now_s();
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n; ++i)
    for (int q = 0; q < 3; ++q)
      acc[3 * (size_t)i + q] = interpolate(mesh_n, box, g.data() + (size_t)q * mm, x.data() + 3 * (size_t)i);
  const double t4 = now_s();
  double t5 = t4, t6 = t4;
  if (split) {
    Tree tree;
    tree.build(x.data(), n, box);
    t5 = now_s();
    const float L = box;
    const float kc = 1.5f * c->omega_m * (L * L * L) / (4.0f * (float)3.14159265358979323846 * a1 * (float)n);
#pragma omp parallel
    {
      std::vector<uint32_t> stack;
#pragma omp for schedule(dynamic, 64)
      for (long long t = 0; t < (long long)m; ++t) {
        float sr[3];
        const size_t i = subset[t];
        tree.accel_on(i, *split, kc, stack, sr, nullptr);
        for (int q = 0; q < 3; ++q) acc[3 * i + q] += sr[q];
      }
    }
    t6 = now_s();
  }
  if (acc_subset)  // the force evaluated at a1 for the sampled particles (outside the timed phases)
    for (size_t t = 0; t < m; ++t)
      for (int q = 0; q < 3; ++q) acc_subset[3 * t + q] = acc[3 * (size_t)subset[t] + q];

  const float k2 = kick_factor(*c, am, a1);
  kick(p.data(), acc.data(), n, k2);
  const double t7e = now_s();
  t7[0] = t1 - t0;
  t7[1] = t2 - t1;
  t7[2] = t3 - t2;
  t7[3] = t4 - t3;
  t7[4] = t5 - t4;
  t7[5] = t6 - t5;
  t7[6] = t7e - t6;
  if (acc_subset_com64 && split) {  // the same force with FP64 centre-of-mass sums (after the timing)
    Tree tree64;
    tree64.com_f64 = 1;
    tree64.build(x.data(), n, box);
    const float L = box;
    const float kc = 1.5f * c->omega_m * (L * L * L) / (4.0f * (float)3.14159265358979323846 * a1 * (float)n);
#pragma omp parallel
    {
      std::vector<uint32_t> stack;
#pragma omp for schedule(dynamic, 64)
      for (long long t = 0; t < (long long)m; ++t) {
        float sr[3];
        const size_t i = subset[t];
        tree64.accel_on(i, *split, kc, stack, sr, nullptr);
        for (int q = 0; q < 3; ++q)  // the PM part of acc[i] (same f32 value), then the tree force
          acc_subset_com64[3 * (size_t)t + q] = interpolate(mesh_n, box, g.data() + (size_t)q * mm, x.data() + 3 * i) + sr[q];
      }
    }
  }
}

float orc_power(const orc_cosmology* c, const orc_pspec* ps, float k) { return power(*c, *ps, k); }
float orc_sigma(const orc_cosmology* c, const orc_pspec* ps, float radius) { return sigma(*c, *ps, radius); }
orc_pspec orc_power_normalized(const orc_cosmology* c, float n_s, float sigma8, float radius) {  // ics.rs:56-63
  orc_pspec unit;
  unit.amplitude = 1.0f;
  unit.n_s = n_s;
  const float su = sigma(*c, unit, radius);
  const float r = sigma8 / su;
  orc_pspec out;
  out.amplitude = r * r;
  out.n_s = n_s;
  return out;
}

void orc_white_noise(int n, uint64_t seed, float* out) {
  const size_t n3 = (size_t)n * n * n;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)n3; ++i) out[i] = white_noise_cell((uint64_t)i, seed);
}

void orc_colored_modes(int n, float box, const orc_cosmology* c, const orc_pspec* ps, uint64_t seed, float* modes) {
  colored_modes(n, box, *c, *ps, seed, reinterpret_cast<cpx<float>*>(modes));
}

// ics.rs:119-182
void orc_zeldovich(int n_, float box, const orc_cosmology* c, const orc_pspec* ps, float a_init, uint64_t seed,
                   float* x3, float* p3) {
  const size_t n = (size_t)n_;
  const size_t n3 = n * n * n;
  const float h = box / (float)n;
  std::vector<cpx<float>> modes(n3);
  colored_modes(n_, box, *c, *ps, seed, modes.data());
  std::vector<float> psi[3];
  std::vector<cpx<float>> psi_k(n3);
  for (int axis = 0; axis < 3; ++axis) {
    std::fill(psi_k.begin(), psi_k.end(), cpx<float>{0.0f, 0.0f});
    for (size_t ix = 0; ix < n; ++ix)
      for (size_t iy = 0; iy < n; ++iy)
        for (size_t iz = 0; iz < n; ++iz) {
          const size_t idx = (ix * n + iy) * n + iz;
          const float k[3] = {wavenumber(ix, n, box), wavenumber(iy, n, box), wavenumber(iz, n, box)};
          float k2 = -0.0f;
          for (int q = 0; q < 3; ++q) k2 += k[q] * k[q];
          if (k2 > 0.0f) {
            const cpx<float> t = cmul(modes[idx], cpx<float>{0.0f, k[axis]});
            psi_k[idx] = {t.re / k2, t.im / k2};
          }
        }
    fft3<float>(n_, psi_k.data(), 1);
    psi[axis].resize(n3);
    for (size_t i = 0; i < n3; ++i) psi[axis][i] = psi_k[i].re / (float)n3;
  }
  const float d = orc_growth(c, a_init);
  const float f = orc_growth_rate(c, a_init);
  const float e = cosmo_e(*c, a_init);
  const float momentum_scale = a_init * a_init * f * e * d;
  for (size_t ix = 0; ix < n; ++ix)
    for (size_t iy = 0; iy < n; ++iy)
      for (size_t iz = 0; iz < n; ++iz) {
        const size_t idx = (ix * n + iy) * n + iz;
        const float q[3] = {(float)ix * h, (float)iy * h, (float)iz * h};
        for (int axis = 0; axis < 3; ++axis) {
          x3[3 * idx + axis] = rem_euclid_f32(q[axis] + d * psi[axis][idx], box);
          p3[3 * idx + axis] = momentum_scale * psi[axis][idx];
        }
      }
}

void orc_power_spectrum(const float* x3, size_t np, float box, int n_, int n_shells, double* k_mean, double* p_mean,
                        uint64_t* counts) {
  const size_t n = (size_t)n_;
  const size_t m = n * n * n;
  std::vector<double> rho(m);
  orc_deposit_f64(n_, box, x3, np, 1.0f, rho.data());
  const double mean = (double)np / (double)m;
  std::vector<cpx<double>> f(m);
  for (size_t i = 0; i < m; ++i) f[i] = {rho[i] / mean - 1.0, 0.0};
  fft3<double>(n_, f.data(), 0);
  const double volume = (double)box * box * box;
  const double kf = 6.283185307179586476925286766559 / (double)box;
  std::vector<double> ks(n_shells + 1, 0.0), ps(n_shells + 1, 0.0);
  std::vector<uint64_t> cs(n_shells + 1, 0);
  auto sgn = [&](size_t i) { return i <= n / 2 ? (long long)i : (long long)i - (long long)n; };
  for (size_t ix = 0; ix < n; ++ix)
    for (size_t iy = 0; iy < n; ++iy)
      for (size_t iz = 0; iz < n; ++iz) {
        const long long mx = sgn(ix), my = sgn(iy), mz = sgn(iz);
        const long long m2 = mx * mx + my * my + mz * mz;
        const long long shell = (long long)std::llround(std::sqrt((double)m2));
        if (shell < 1 || shell > n_shells) continue;
        const size_t idx = (ix * n + iy) * n + iz;
        const double pw = volume * (f[idx].re * f[idx].re + f[idx].im * f[idx].im) / ((double)m * (double)m);
        ks[shell] += kf * std::sqrt((double)m2);
        ps[shell] += pw;
        cs[shell] += 1;
      }
  for (int s = 1; s <= n_shells; ++s) {
    k_mean[s - 1] = cs[s] ? ks[s] / (double)cs[s] : 0.0;
    p_mean[s - 1] = cs[s] ? ps[s] / (double)cs[s] : 0.0;
    counts[s - 1] = cs[s];
  }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
