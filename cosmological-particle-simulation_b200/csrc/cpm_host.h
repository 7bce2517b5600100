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

// integrator.rs:150-152: K = (3/2) Omega_m L^3 / (4 pi a N), L^3 as L*(L*L) (powi(3)).
inline float tree_coupling(float omega_m, float box, float a, size_t n) {
  const float nf = (float)n;
  const float l3 = box * (box * box);
  return 1.5f * omega_m * l3 / (4.0f * (float)3.14159265358979323846 * a * nf);
}

}  // namespace cpm
