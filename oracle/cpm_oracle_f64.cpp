// cpm_oracle_f64.cpp — the FP64 build of the oracle for precision studies (test infrastructure).
//
// The same TreePM force as cpm_oracle.cpp (poisson.rs:33-88 for the PM part, tree.rs:171-323 for the
// short-range part) with every operation in double precision: CIC weights, deposit, delta, the FFT,
// the Green's function, the gradient, the gather, the octree (centres, halves, centres of mass),
// the opening and cutoff tests and the pair force with the C library's double erfc and exp. The
// reference's rules are kept: Nyquist wavenumbers are 0, k = 0 is dropped, a node whose octant-0
// child is missing is summed directly, leaves hold at most 8 particles, depth stops at 40. Forces
// are evaluated only at sampled particles (the PM meshes are full size, the tree walk runs for the
// samples), which makes a check of 10^5 particles of a 512^3-particle, 1024^3-mesh run feasible on
// the host. Only tests/ and bench.py's precision leg load this library.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "cpm_oracle.h"

namespace {

constexpr double PI = 3.14159265358979323846;

struct Stencil64 {
  size_t idx[8];
  double w[8];
};

// mesh.rs:29-59 in double.
void stencil64(size_t n, double box, const double* x, Stencil64& st) {
  const double h = box / (double)n;
  int64_t b[3];
  double f[3];
  for (int k = 0; k < 3; ++k) {
    const double s = x[k] / h - 0.5;
    const double i0 = std::floor(s);
    b[k] = (int64_t)i0;
    f[k] = s - i0;
  }
  auto wrap = [&](int64_t i) { int64_t r = i % (int64_t)n; return (size_t)(r < 0 ? r + (int64_t)n : r); };
  int c = 0;
  for (int dx = 0; dx < 2; ++dx)
    for (int dy = 0; dy < 2; ++dy)
      for (int dz = 0; dz < 2; ++dz, ++c) {
        st.idx[c] = (wrap(b[0] + dx) * n + wrap(b[1] + dy)) * n + wrap(b[2] + dz);
        st.w[c] = (dx ? f[0] : 1.0 - f[0]) * (dy ? f[1] : 1.0 - f[1]) * (dz ? f[2] : 1.0 - f[2]);
      }
}

// fft.rs:86-95 in double: the Nyquist index of an even grid gives 0.
double wavenumber64(size_t i, size_t n, double box) {
  if (n % 2 == 0 && i == n / 2) return 0.0;
  const double m = i <= n / 2 ? (double)i : (double)i - (double)n;
  return m * 2.0 * PI / box;
}

struct Node64 {
  double center[3], half, com[3];
  double quad[6];  // second moments about com: xx, yy, zz, xy, xz, yz (library quadrupole mode)
  uint32_t count, start, end;
  uint32_t children[8];
};
constexpr uint32_t NONE = 0xFFFFFFFFu;

struct Tree64 {
  const double* pos = nullptr;
  double box = 0.0;
  std::vector<uint32_t> order;
  std::vector<Node64> nodes;

  void build(const double* p, size_t n, double b) {
    pos = p;
    box = b;
    order.resize(n);
    std::iota(order.begin(), order.end(), 0u);
    nodes.clear();
    nodes.reserve(n / 3 + 16);
    const double c[3] = {b / 2, b / 2, b / 2};
    build_node(0, n, c, b / 2, 0);
  }

  // tree.rs:186-250 in double; centres of mass summed in double.
  uint32_t build_node(size_t start, size_t end, const double* center, double half, uint32_t depth) {
    const uint32_t idx = (uint32_t)nodes.size();
    Node64 nd;
    double com[3] = {0, 0, 0};
    for (size_t t = start; t < end; ++t)
      for (int k = 0; k < 3; ++k) com[k] += pos[3 * (size_t)order[t] + k];
    for (int k = 0; k < 3; ++k) {
      nd.center[k] = center[k];
      nd.com[k] = com[k] / (double)(end - start);
    }
    for (double& q : nd.quad) q = 0.0;
    for (size_t t = start; t < end; ++t) {
      const double* p = pos + 3 * (size_t)order[t];
      const double e0 = p[0] - nd.com[0], e1 = p[1] - nd.com[1], e2 = p[2] - nd.com[2];
      nd.quad[0] += e0 * e0;
      nd.quad[1] += e1 * e1;
      nd.quad[2] += e2 * e2;
      nd.quad[3] += e0 * e1;
      nd.quad[4] += e0 * e2;
      nd.quad[5] += e1 * e2;
    }
    nd.half = half;
    nd.count = (uint32_t)(end - start);
    nd.start = (uint32_t)start;
    nd.end = (uint32_t)end;
    for (auto& ch : nd.children) ch = NONE;
    nodes.push_back(nd);
    if (end - start <= 8 || depth >= 40) return idx;
    auto octant = [&](uint32_t j) {
      const double* p = pos + 3 * (size_t)j;
      return (size_t)(p[0] >= center[0]) | ((size_t)(p[1] >= center[1]) << 1) | ((size_t)(p[2] >= center[2]) << 2);
    };
    size_t counts[8] = {0};
    for (size_t t = start; t < end; ++t) counts[octant(order[t])] += 1;
    size_t offsets[8], next[8], run = start;
    for (int o = 0; o < 8; ++o) {
      offsets[o] = next[o] = run;
      run += counts[o];
    }
    std::vector<uint32_t> sorted(end - start);
    for (size_t t = start; t < end; ++t) {
      const uint32_t j = order[t];
      const size_t o = octant(j);
      sorted[next[o]++ - start] = j;
    }
    std::copy(sorted.begin(), sorted.end(), order.begin() + (long)start);
    const double q = half / 2.0;
    for (int o = 0; o < 8; ++o) {
      if (!counts[o]) continue;
      double cc[3];
      for (int k = 0; k < 3; ++k) cc[k] = center[k] + (((o >> k) & 1) ? q : -q);
      const uint32_t child = build_node(offsets[o], offsets[o] + counts[o], cc, q, depth + 1);
      nodes[idx].children[o] = child;
    }
    return idx;
  }

  void min_image(const double* a, const double* b, double* d) const {
    for (int k = 0; k < 3; ++k) {
      const double x = a[k] - b[k];
      d[k] = x - box * std::round(x / box);
    }
  }

  // tree.rs:264-310 in double (opening test 2 half < theta r). With `quad`, an accepted node also
  // adds the second-order Taylor term of sum_j g(|d_j|) d_j about its centre of mass (the library's
  // CPM_SIM_QUADRUPOLE): (1/2)[h (D.T.D) D + (g'/r)(tr T D + 2 T D)], h = (g'' - g'/r) / r^2.
  void accel_on(size_t i, const orc_split& s, double kk, std::vector<uint32_t>& stack, double* acc,
                bool quad = false) const {
    const double* xi = pos + 3 * i;
    const double rs = s.r_split, rc = s.r_cut, eps2 = (double)s.softening * s.softening, theta = s.theta;
    auto pair = [&](const double* d, double mass) {
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const double r = std::sqrt(r2), u = r / (2.0 * rs);
      const double sr = std::erfc(u) + 2.0 / std::sqrt(PI) * u * std::exp(-u * u);
      const double q = r2 + eps2;
      const double f = -kk * mass * sr / (q * std::sqrt(q));
      for (int k = 0; k < 3; ++k) acc[k] += d[k] * f;
    };
    acc[0] = acc[1] = acc[2] = 0.0;
    stack.assign(1, 0u);
    while (!stack.empty()) {
      const Node64& nd = nodes[stack.back()];
      stack.pop_back();
      double tc[3];
      min_image(nd.center, xi, tc);
      const double max_r = rc + std::sqrt(3.0) * nd.half;
      if (tc[0] * tc[0] + tc[1] * tc[1] + tc[2] * tc[2] > max_r * max_r) continue;
      if (nd.children[0] == NONE) {
        for (uint32_t t = nd.start; t < nd.end; ++t) {
          const size_t j = order[t];
          if (j == i) continue;
          double d[3];
          min_image(xi, pos + 3 * j, d);
          if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > rc * rc) continue;
          pair(d, 1.0);
        }
      } else {
        double to[3];
        min_image(nd.com, xi, to);
        const double r = std::sqrt(to[0] * to[0] + to[1] * to[1] + to[2] * to[2]);
        if (2.0 * nd.half < theta * r) {
          const double d[3] = {-to[0], -to[1], -to[2]};
          pair(d, (double)nd.count);
          if (quad && r > 0.0) {
            const double D[3] = {to[0], to[1], to[2]};  // from the particle to the centre of mass
            const double r2 = r * r, u = r / (2.0 * rs), e = std::exp(-u * u), c = 2.0 / std::sqrt(PI);
            const double S = std::erfc(u) + c * u * e, S1 = -c * u * u * e / rs, S2 = -c * u * (1 - u * u) * e / (rs * rs);
            const double q = r2 + eps2, P = 1.0 / (q * std::sqrt(q)), P1 = -3.0 * r * P / q;
            const double P2 = -3.0 * P / q + 15.0 * r2 * P / (q * q);
            const double g1 = S1 * P + S * P1, g2 = S2 * P + 2.0 * S1 * P1 + S * P2, h = (g2 - g1 / r) / r2;
            const double* T = nd.quad;
            const double td[3] = {T[0] * D[0] + T[3] * D[1] + T[4] * D[2], T[3] * D[0] + T[1] * D[1] + T[5] * D[2],
                                  T[4] * D[0] + T[5] * D[1] + T[2] * D[2]};
            const double dtd = D[0] * td[0] + D[1] * td[1] + D[2] * td[2], tr = T[0] + T[1] + T[2];
            for (int k = 0; k < 3; ++k) acc[k] += kk * 0.5 * (h * dtd * D[k] + g1 / r * (tr * D[k] + 2.0 * td[k]));
          }
        } else {
          for (int o = 0; o < 8; ++o)
            if (nd.children[o] != NONE) stack.push_back(nd.children[o]);
        }
      }
    }
  }
};

}  // namespace

extern "C" {

void orc64_accelerations_ex(const float* x3, size_t n, double box, int mesh_n, double omega_m, double a,
                            const orc_split* split, double k_tree, const uint32_t* sample, size_t n_sample,
                            double* acc3, int quadrupole);

void orc64_accelerations(const float* x3, size_t n, double box, int mesh_n, double omega_m, double a,
                         const orc_split* split, double k_tree, const uint32_t* sample, size_t n_sample,
                         double* acc3) {
  orc64_accelerations_ex(x3, n, box, mesh_n, omega_m, a, split, k_tree, sample, n_sample, acc3, 0);
}

void orc64_accelerations_ex(const float* x3, size_t n, double box, int mesh_n, double omega_m, double a,
                            const orc_split* split, double k_tree, const uint32_t* sample, size_t n_sample,
                            double* acc3, int quadrupole) {
  const size_t mn = (size_t)mesh_n;
  const size_t m = mn * mn * mn;
  std::vector<double> x(3 * n);
  for (size_t i = 0; i < 3 * n; ++i) x[i] = (double)x3[i];
  std::fill(acc3, acc3 + 3 * n_sample, 0.0);

  // PM part (poisson.rs:33-88, integrator.rs:117-126 and 144-148) in double.
  {
    std::vector<double> rho(m, 0.0);
    Stencil64 st;
    for (size_t i = 0; i < n; ++i) {
      stencil64(mn, box, &x[3 * i], st);
      for (int c = 0; c < 8; ++c) rho[st.idx[c]] += st.w[c];
    }
    const double mean = (double)n / (double)m;
    std::vector<double> f(2 * m);
    for (size_t i = 0; i < m; ++i) {
      f[2 * i] = rho[i] / mean - 1.0;
      f[2 * i + 1] = 0.0;
    }
    std::vector<double>().swap(rho);
    orc_fft3_f64(mesh_n, f.data(), 0);
    const double r_split = split ? (double)split->r_split : 0.0;
    const double pref = 1.5 * omega_m / a;
#pragma omp parallel for schedule(static)
    for (size_t ix = 0; ix < mn; ++ix)
      for (size_t iy = 0; iy < mn; ++iy)
        for (size_t iz = 0; iz < mn; ++iz) {
          const double kx = wavenumber64(ix, mn, box), ky = wavenumber64(iy, mn, box), kz = wavenumber64(iz, mn, box);
          const double k2 = kx * kx + ky * ky + kz * kz;
          const size_t idx = (ix * mn + iy) * mn + iz;
          const double g = k2 == 0.0 ? 0.0 : -pref / k2 * std::exp(-k2 * r_split * r_split);
          f[2 * idx] *= g;
          f[2 * idx + 1] *= g;
        }
    std::vector<double> g(2 * m);
    for (int axis = 0; axis < 3; ++axis) {
#pragma omp parallel for schedule(static)
      for (size_t ix = 0; ix < mn; ++ix)
        for (size_t iy = 0; iy < mn; ++iy)
          for (size_t iz = 0; iz < mn; ++iz) {
            const size_t idx = (ix * mn + iy) * mn + iz;
            const size_t ia = axis == 0 ? ix : (axis == 1 ? iy : iz);
            const double nk = -wavenumber64(ia, mn, box);
            // phi * (0 - i k): (re, im) -> (-im * (-k), re * (-k))
            g[2 * idx] = -f[2 * idx + 1] * nk;
            g[2 * idx + 1] = f[2 * idx] * nk;
          }
      orc_fft3_f64(mesh_n, g.data(), 1);
      const double scale = 1.0 / (double)m;
      for (size_t s = 0; s < n_sample; ++s) {
        stencil64(mn, box, &x[3 * (size_t)sample[s]], st);
        double v = 0.0;
        for (int c = 0; c < 8; ++c) v += g[2 * st.idx[c]] * scale * st.w[c];
        acc3[3 * s + axis] += v;
      }
    }
  }

  // Short-range part (tree.rs:314-323) in double.
  if (split) {
    Tree64 tree;
    tree.build(x.data(), n, box);
#pragma omp parallel
    {
      std::vector<uint32_t> stack;
      double a3[3];
#pragma omp for schedule(dynamic, 64)
      for (long long s = 0; s < (long long)n_sample; ++s) {
        tree.accel_on(sample[s], *split, k_tree, stack, a3, quadrupole != 0);
        for (int k = 0; k < 3; ++k) acc3[3 * s + k] += a3[k];
      }
    }
  }
}

}  // extern "C"
