// cpm_host.h — host-side helpers shared by the C-ABI translation units: error slots, the f32
// scalars of the Poisson solve, and the reference's f32 step factors (integrator.rs:263-297,
// cosmology.rs:32-34). Host code is compiled with -ffp-contract=off, so these scalars round
// exactly as the reference's Rust f32 code does.
#pragma once

#include <cmath>
#include <string>

#include "cpm_internal.cuh"

namespace cpm {

extern thread_local std::string g_last_error;
int set_error(std::string* slot, int code, const std::string& msg);
int check_device_once(std::string* err);

inline PoissonParams make_poisson_params(int n, float box, float omega_m, float a, float r_split, int deconvolve) {
  PoissonParams pp;
  pp.n = n;
  pp.two_pi_over_l = 2.0f * (float)3.14159265358979323846 / box;  // fft.rs:87
  pp.prefactor = 1.5f * omega_m / a;                              // poisson.rs:46
  pp.r_split = r_split;
  const size_t n3 = (size_t)n * n * n;
  pp.scale = 1.0f / (float)n3;  // poisson.rs:77
  pp.deconvolve = deconvolve;
  return pp;
}

// cosmology.rs:32-34
inline float cosmo_e(const cpm_cosmology& c, float a) {
  return std::sqrt(c.omega_r / (a * a * a * a) + c.omega_m / (a * a * a) + c.omega_l);
}

// integrator.rs:288-297 (Simpson, 64 intervals)
template <typename F>
inline float simpson64(float lo, float hi, F f) {
  const int n = 64;
  const float h = (hi - lo) / (float)n;
  float sum = f(lo) + f(hi);
  for (int i = 1; i < n; ++i) {
    const float weight = (i % 2 == 1) ? 4.0f : 2.0f;
    sum += weight * f(lo + (float)i * h);
  }
  return sum * h / 3.0f;
}

// integrator.rs:263-265
inline float kick_factor(const cpm_cosmology& c, float a0, float a1) {
  return simpson64(a0, a1, [&](float a) { return 1.0f / (a * cosmo_e(c, a)); });
}
// integrator.rs:268-270
inline float drift_factor(const cpm_cosmology& c, float a0, float a1) {
  return simpson64(a0, a1, [&](float a) { return 1.0f / (a * a * a * cosmo_e(c, a)); });
}
// integrator.rs:273-285 (60 bisection steps)
inline float midpoint(const cpm_cosmology& c, float a0, float a1) {
  const float half = kick_factor(c, a0, a1) / 2.0f;
  float lo = a0, hi = a1;
  for (int it = 0; it < 60; ++it) {
    const float mid = 0.5f * (lo + hi);
    if (kick_factor(c, a0, mid) < half)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5f * (lo + hi);
}

// cosmology.rs:47-79: f32 RK4 in ln a (4000 steps) from a = 1e-3 with the Meszaros start.
inline void growth_state(const cpm_cosmology& c, float a_end, float* d_out, float* dl_out) {
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
  const float h = (std::log(a_end) - la0) / 4000.0f;
  for (int step = 0; step < 4000; ++step) {
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

// cosmology.rs:82-90
inline float growth(const cpm_cosmology& c, float a) {
  float d, dl, d1, dl1;
  growth_state(c, a, &d, &dl);
  growth_state(c, 1.0f, &d1, &dl1);
  return d / d1;
}
inline float growth_rate(const cpm_cosmology& c, float a) {
  float d, dl;
  growth_state(c, a, &d, &dl);
  return dl / d;
}

// cosmology.rs:94-103 (BBKS, powi expanded as the compiler does: x*x, x*(x*x), (x*x)*(x*x))
inline float bbks(const cpm_cosmology& c, float k) {
  const float h = c.h0 / 100.0f;
  const float q = k / (c.omega_m * h);
  if (q == 0.0f) return 1.0f;
  const float x2 = 16.1f * q, x3 = 5.46f * q, x4 = 6.71f * q;
  const float x4s = x4 * x4;
  const float poly = 1.0f + 3.89f * q + x2 * x2 + x3 * (x3 * x3) + x4s * x4s;
  return std::log1p(2.34f * q) / (2.34f * q) * std::pow(poly, -0.25f);
}

// ics.rs:27-33
inline float power_spectrum(const cpm_cosmology& c, float amplitude, float n_s, float k) {
  if (k == 0.0f) return 0.0f;
  const float t = bbks(c, k);
  return amplitude * std::pow(k, n_s) * t * t;
}

// ics.rs:36-63: sigma(R) by Simpson (8192 intervals in ln k), amplitude = (sigma8 / sigma_unit)^2.
inline float power_amplitude(const cpm_cosmology& c, float n_s, float sigma8, float radius) {
  const int steps = 8192;
  const float ln_lo = std::log(1e-4f), ln_hi = std::log(1e3f);
  const float h = (ln_hi - ln_lo) / (float)steps;
  auto tophat = [](float x) { return x < 1e-4f ? 1.0f : 3.0f * (std::sin(x) - x * std::cos(x)) / (x * x * x); };
  auto integrand = [&](float ln_k) {
    const float k = std::exp(ln_k);
    const float w = tophat(k * radius);
    return k * (k * k) * power_spectrum(c, 1.0f, n_s, k) * w * w;
  };
  float sum = integrand(ln_lo) + integrand(ln_hi);
  for (int i = 1; i < steps; ++i) sum += ((i % 2 == 1) ? 4.0f : 2.0f) * integrand(ln_lo + (float)i * h);
  const float integral = sum * h / 3.0f;
  const double pi = 3.14159265358979323846;
  const float sigma_unit = std::sqrt(integral / (2.0f * (float)(pi * pi)));
  const float r = sigma8 / sigma_unit;
  return r * r;
}

// integrator.rs:150-152: K = (3/2) Omega_m L^3 / (4 pi a N), L^3 as L*(L*L) (powi(3)).
inline float tree_coupling(float omega_m, float box, float a, size_t n) {
  const float nf = (float)n;
  const float l3 = box * (box * box);
  return 1.5f * omega_m * l3 / (4.0f * (float)3.14159265358979323846 * a * nf);
}

}  // namespace cpm
