// Exercises the C++ mirror (include/cpm.hpp) the way integrator.rs and the reference's tests call
// the Rust path: prints "ok <name>" per check and exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "cpm.hpp"

using cpm::Real;
using cpm::Vec3;

#define CHECK(name, cond)                                  \
  do {                                                     \
    if (!(cond)) {                                         \
      std::printf("FAIL %s\n", name);                      \
      return 1;                                            \
    }                                                      \
    std::printf("ok %s\n", name);                          \
  } while (0)

int main() {
  // mesh.rs:151-162 — a particle on x = L splits between the last and the first cell.
  {
    cpm::Mesh m(4, 1.0f);
    const Real h = 1.0f / 4.0f;
    m.deposit({Vec3{1.0f, 0.5f * h, 0.5f * h}}, 1.0f);
    CHECK("deposit_wraps", std::fabs(m.cells[((3 * 4) + 0) * 4 + 0] - 0.5f) < 1e-5f && std::fabs(m.cells[0] - 0.5f) < 1e-5f);
    cpm::Mesh c(8, 1.0f);
    for (auto& v : c.cells) v = 2.5f;
    CHECK("interpolate_constant", std::fabs(c.interpolate(Vec3{0.3f, 0.7f, 0.1f}) - 2.5f) < 1e-5f);
  }
  // poisson.rs:114-139 — plane wave.
  {
    const int n = 16;
    const Real a = 0.5f, k0 = 2.0f * (Real)M_PI;
    const auto cosmo = cpm::Cosmology::lcdm_default();
    const Real cc = 1.5f * cosmo.omega_m / a;
    cpm::Mesh delta(n, 1.0f);
    const Real h = 1.0f / n;
    for (int ix = 0; ix < n; ++ix)
      for (int j = 0; j < n * n; ++j) delta.cells[ix * n * n + j] = std::cos(k0 * (ix + 0.5f) * h);
    cpm::PoissonSolver solver(n, 1.0f);
    auto g = solver.acceleration(delta, cosmo, a, 0.0f);
    Real err = 0.0f;
    for (int ix = 0; ix < n; ++ix)
      for (int j = 0; j < n * n; ++j)
        err = std::fmax(err, std::fabs(g[0].cells[ix * n * n + j] + (cc / k0) * std::sin(k0 * (ix + 0.5f) * h)));
    CHECK("plane_wave", err < 1e-5f * (cc / k0));
    bool threw = false;
    try {
      cpm::Mesh wrong(8, 1.0f);
      solver.acceleration(wrong, cosmo, a, 0.0f);
    } catch (const cpm::Error& e) {
      threw = e.code == CPM_E_MESH_MISMATCH;
    }
    CHECK("mesh_mismatch_throws", threw);
  }
  // tree.rs:420-430 — minimum image across the boundary.
  {
    const cpm::ForceSplit s{0.5f, 2.0f, 0.05f, 0.5f};
    auto acc = cpm::tree::accelerations({Vec3{0.1f, 5.0f, 5.0f}, Vec3{9.9f, 5.0f, 5.0f}}, 10.0f, s, 1.0f);
    CHECK("periodic_pair", acc[0][0] < 0.0f && acc[1][0] > 0.0f);
  }
  // integrator.rs:437-461 — TreePM pair force vs Newton, then a few steps.
  {
    const auto cosmo = cpm::Cosmology::lcdm_default();
    cpm::ForceSplit split = cpm::ForceSplit::with(100.0f, 64, 2, 0.05f, 0.5f);
    split.softening = 0.01f;
    cpm::Simulation sim(cosmo, 100.0f, 64, {Vec3{50.0f, 50.0f, 50.0f}, Vec3{53.0f, 50.0f, 50.0f}},
                        {Vec3{0, 0, 0}, Vec3{0, 0, 0}}, 1.0f, &split);
    const Real before = sim.positions[1][0] - sim.positions[0][0];
    sim.step_to(1.0002f);
    sim.step_to(1.0004f);
    const Real after = sim.positions[1][0] - sim.positions[0][0];
    CHECK("pair_attracts", after < before && after > 0.0f && sim.a == 1.0004f);
    // runner.rs:263-284 snapshot on the device: both particles move, the grid is 64^3 of 1 + delta
    const auto frame = sim.snapshot(true);
    CHECK("snapshot", frame.speeds.size() == 2 && frame.speeds[0] > 0.0f && frame.max_speed >= frame.speeds[1] &&
                          frame.grid_n == 64 && frame.grid.size() == 64u * 64u * 64u && frame.densities[0] >= 0.0f);
    const auto ps = sim.power_spectrum(8);
    CHECK("power_spectrum", ps.counts.size() == 8 && ps.counts[0] > 0 && ps.p_mean[0] > 0.0);
  }
  std::printf("all ok\n");
  return 0;
}
