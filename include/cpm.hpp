// cpm.hpp — header-only C++ mirror of the reference crate's TreePM interface over the C ABI of
// libcpm_cuda.so (cpm.h). Names and argument meaning follow the Rust items they stand in for;
// where the reference panics, these throw cpm::Error (status code + library message).
//
//   Mesh          mesh.rs:6-78        new, deposit, interpolate
//   Fft3          fft.rs:11-72        new, forward, inverse;  wavenumber  fft.rs:86-95
//   PoissonSolver poisson.rs:14-88    new, acceleration
//   ForceSplit    tree.rs:20-51       with;  short_range_factor  tree.rs:54-57
//   tree::accelerations               tree.rs:314-323
//   Simulation    integrator.rs:34-186 new, step_to, positions/momenta, delta
#pragma once

#include <algorithm>
#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cpm.h"

namespace cpm {

using Real = float;  // real.rs:2
using Vec3 = std::array<Real, 3>;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const cpm_ctx* ctx = nullptr) {
  if (rc != CPM_OK) throw Error(rc, cpm_last_error(ctx));
}

// One context per (mesh size, box); not thread-safe, like the reference's single worker thread.
class Context {
 public:
  Context(int n, Real box) {
    cpm_ctx* c = nullptr;
    check(cpm_ctx_create(n, box, 0, 0, &c));
    ctx_.reset(c);
  }
  cpm_ctx* get() const { return ctx_.get(); }

 private:
  struct Del {
    void operator()(cpm_ctx* c) const { cpm_ctx_destroy(c); }
  };
  std::unique_ptr<cpm_ctx, Del> ctx_;
};

struct Cosmology {  // cosmology.rs:9-29
  Real omega_r, omega_m, omega_l, h0;
  static Cosmology lcdm_default() {
    const Real omega_r = 9.14e-5f;
    return Cosmology{omega_r, 0.315f, 1.0f - 0.315f - omega_r, 67.4f};
  }
  cpm_cosmology c() const { return cpm_cosmology{omega_r, omega_m, omega_l, h0}; }
};

class Mesh {  // mesh.rs:6-78
 public:
  std::size_t n;
  Real box_size;
  std::vector<Real> cells;

  Mesh(std::size_t n_, Real box) : n(n_), box_size(box), cells(n_ * n_ * n_, 0.0f) {}
  static Mesh make(std::size_t n_, Real box) { return Mesh(n_, box); }

  void deposit(const std::vector<Vec3>& positions, Real mass) {  // mesh.rs:62-69
    Context& c = ctx();
    check(cpm_mesh_deposit(c.get(), positions.empty() ? nullptr : positions[0].data(), positions.size(), mass,
                           cells.data()),
          c.get());
  }
  Real interpolate(const Vec3& x) const {  // mesh.rs:72-77
    Real out = 0.0f;
    Context& c = ctx();
    check(cpm_mesh_interpolate(c.get(), cells.data(), x.data(), 1, &out), c.get());
    return out;
  }

 private:
  Context& ctx() const {
    if (!ctx_) ctx_ = std::make_shared<Context>((int)n, box_size);
    return *ctx_;
  }
  mutable std::shared_ptr<Context> ctx_;
};

inline Real wavenumber(std::size_t i, std::size_t n, Real box) { return cpm_wavenumber(i, n, box); }

class Fft3 {  // fft.rs:11-72
 public:
  explicit Fft3(std::size_t n) : n_(n), ctx_((int)n, 1.0f) {}
  void forward(std::vector<std::complex<Real>>& data) { run(data, 0); }
  void inverse(std::vector<std::complex<Real>>& data) { run(data, 1); }

 private:
  void run(std::vector<std::complex<Real>>& data, int inv) {
    if (data.size() != n_ * n_ * n_) throw Error(CPM_E_INVALID, "Fft3: data must hold n^3 values");
    check(cpm_fft3(ctx_.get(), reinterpret_cast<cpm_cf32*>(data.data()), (int)n_, inv), ctx_.get());
  }
  std::size_t n_;
  Context ctx_;
};

class PoissonSolver {  // poisson.rs:14-88
 public:
  PoissonSolver(std::size_t n, Real box) : n_(n), box_(box), ctx_((int)n, box) {}
  std::array<Mesh, 3> acceleration(const Mesh& delta, const Cosmology& cosmo, Real a, Real r_split) {
    std::array<Mesh, 3> g{Mesh(n_, box_), Mesh(n_, box_), Mesh(n_, box_)};
    const cpm_cosmology c = cosmo.c();
    check(cpm_poisson_accel(ctx_.get(), delta.cells.data(), (int)delta.n, &c, a, r_split, g[0].cells.data(),
                            g[1].cells.data(), g[2].cells.data()),
          ctx_.get());
    return g;
  }

 private:
  std::size_t n_;
  Real box_;
  Context ctx_;
};

struct ForceSplit {  // tree.rs:20-51
  Real r_split, r_cut, softening, theta;
  static ForceSplit with(Real box, std::size_t mesh_n, std::size_t pps, Real softening_scale, Real theta) {
    const cpm_force_split s = cpm_force_split_with(box, mesh_n, pps, softening_scale, theta);
    return ForceSplit{s.r_split, s.r_cut, s.softening, s.theta};
  }
  cpm_force_split c() const { return cpm_force_split{r_split, r_cut, softening, theta}; }
};

inline Real short_range_factor(Real r, Real r_split) { return cpm_short_range_factor(r, r_split); }

namespace tree {
// tree.rs:314-323
inline std::vector<Vec3> accelerations(const std::vector<Vec3>& positions, Real box, const ForceSplit& split, Real k) {
  std::vector<Vec3> out(positions.size());
  if (positions.empty()) return out;
  Context c(1, box);
  const cpm_force_split s = split.c();
  check(cpm_tree_accel(c.get(), positions[0].data(), positions.size(), box, &s, k, out[0].data()), c.get());
  return out;
}
}  // namespace tree

class Simulation {  // integrator.rs:34-186
 public:
  // `split` null means pure PM (the reference's Option<ForceSplit>).
  Simulation(const Cosmology& cosmo, Real box, std::size_t mesh_n, std::vector<Vec3> positions_,
             std::vector<Vec3> momenta_, Real a_, const ForceSplit* split)
      : positions(std::move(positions_)), momenta(std::move(momenta_)), a(a_), mesh_n_(mesh_n), box_(box) {
    if (positions.size() != momenta.size() || positions.empty())
      throw Error(CPM_E_INVALID, "Simulation: positions and momenta must be non-empty and of equal length");
    cpm_sim_params p{};
    p.cosmo = cosmo.c();
    p.box_size = box;
    p.mesh_n = (int)mesh_n;
    p.n_particles = positions.size();
    p.use_tree = split ? 1 : 0;
    if (split) p.split = split->c();
    cpm_sim* s = nullptr;
    check(cpm_sim_create(&p, positions[0].data(), momenta[0].data(), a, &s));
    sim_.reset(s);
  }

  // integrator.rs:174-186: the pub `positions` and `momenta` are the caller's, stepped in place.
  void step_to(Real a1) {
    check(cpm_sim_step_host(sim_.get(), a1, positions[0].data(), momenta[0].data()));
    a = a1;
  }

  Mesh delta() const {  // integrator.rs:128-131
    Mesh m(mesh_n_, box_);
    check(cpm_sim_get_state(sim_.get(), nullptr, nullptr, nullptr, m.cells.data(), nullptr));
    return m;
  }

  // runner.rs:263-284 `snapshot`, reduced on the device (frame.rs:1-70): speeds |p|/a,
  // densities max(1 + delta(x), 0), rsd shifts p / (a^2 E), the density grid when asked, max speed.
  struct Frame {
    Real redshift;
    std::vector<Real> speeds, densities;
    std::vector<Vec3> rsd;
    std::size_t grid_n = 0;
    std::vector<Real> grid;  // grid_n^3, x fastest
    Real max_speed;
  };
  Frame snapshot(bool want_grid) const {
    Frame f;
    const std::size_t n = positions.size();
    f.redshift = 1.0f / a - 1.0f;
    f.speeds.resize(n);
    f.densities.resize(n);
    f.rsd.resize(n);
    if (want_grid) {
      const std::size_t fac = std::max<std::size_t>(1, (mesh_n_ + 127) / 128);
      const std::size_t m = mesh_n_ / fac;
      f.grid.resize(m * m * m);
    }
    int gn = 0;
    check(cpm_sim_snapshot(sim_.get(), f.speeds.data(), f.densities.data(), f.rsd[0].data(),
                           want_grid ? f.grid.data() : nullptr, &gn, &f.max_speed));
    f.grid_n = want_grid ? (std::size_t)gn : 0;
    return f;
  }

  // Shell-averaged P(k) of the current particles (the estimator of ics.rs:213-266), on the device.
  struct PowerSpectrum {
    std::vector<double> k_mean, p_mean;
    std::vector<std::uint64_t> counts;
  };
  PowerSpectrum power_spectrum(int n_shells) const {
    PowerSpectrum ps;
    ps.k_mean.resize(n_shells);
    ps.p_mean.resize(n_shells);
    ps.counts.resize(n_shells);
    check(cpm_sim_power_spectrum(sim_.get(), n_shells, ps.k_mean.data(), ps.p_mean.data(), ps.counts.data()));
    return ps;
  }

  std::vector<Vec3> positions;
  std::vector<Vec3> momenta;
  Real a;

 private:
  struct Del {
    void operator()(cpm_sim* s) const { cpm_sim_destroy(s); }
  };
  std::unique_ptr<cpm_sim, Del> sim_;
  std::size_t mesh_n_;
  Real box_;
};

}  // namespace cpm
