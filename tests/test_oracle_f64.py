"""The FP64 build of the oracle (the precision-study reference) against the f32-faithful oracle:
the same TreePM force, so they agree to f32 rounding."""
import numpy as np


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def test_fp64_oracle_matches_f32_oracle_treepm(orc):
    box, mesh, nside = 32.0, 32, 16
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    ps = orc.power_normalized(c, 0.96, 0.8, 8.0)
    x, p = orc.zeldovich(nside, box, c, ps, 0.2, 21)
    split = orc.split_with(box, mesh, nside, 1.0 / 30.0, 0.5)
    sim = orc.Simulation(c, box, mesh, x, p, 0.2, split)
    acc32 = sim.state()["acc"]
    sample = np.random.default_rng(0).choice(len(x), 500, replace=False)
    acc64 = orc.accelerations_f64(x, box, mesh, c.omega_m, 0.2, split, sample)
    assert _rel_rms(acc32[sample], acc64) < 1e-5


def test_fp64_oracle_pm_only_matches_f32_oracle(orc):
    box, mesh = 16.0, 16
    x = orc.scattered_mesh(3000, box)
    c = orc.lcdm_default()
    delta = orc.density_contrast(mesh, box, x)
    gx, gy, gz = orc.poisson_accel(mesh, box, delta, c.omega_m, 0.7, 0.0)
    g32 = np.stack([orc.interpolate_many(mesh, box, g, x) for g in (gx, gy, gz)], 1)
    sample = np.arange(0, len(x), 7)
    g64 = orc.accelerations_f64(x, box, mesh, c.omega_m, 0.7, None, sample)
    assert _rel_rms(g32[sample], g64) < 1e-5
