"""GPU power spectrum (the estimator of ics.rs:213-266 applied to particles) against the oracle's
FP64 version: CIC density, delta = rho/mean - 1, FFT, V |delta_k|^2 / M^2 in integer shells."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Relative tolerance of the shell powers for k <= k_Nyquist / 2 (f32 FFT against FP64).
PK_RTOL = 1e-3


def _ics(orc, n, box, a_init, seed):
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    ps = orc.power_normalized(c, 0.96, 0.8, 8.0)
    x, p = orc.zeldovich(n, box, c, ps, a_init, seed)
    return c, x, p


def _clustered(n_particles, box, seed):
    """Particles in Gaussian blobs plus a uniform background: power over many decades."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, box, (40, 3))
    member = rng.integers(0, 40, n_particles)
    x = centres[member] + rng.normal(0.0, 0.03 * box, (n_particles, 3))
    bg = n_particles // 4
    x[:bg] = rng.uniform(0.0, box, (bg, 3))
    return np.mod(x, box).astype(np.float32)


def _compare(k_g, p_g, c_g, k_o, p_o, c_o, n):
    np.testing.assert_array_equal(c_g, c_o)
    nz = c_o > 0
    np.testing.assert_allclose(k_g[nz], k_o[nz], rtol=1e-12)
    low = np.arange(1, len(p_o) + 1) <= n // 4
    sel = nz & low
    rel = np.abs(p_g[sel] - p_o[sel]) / p_o[sel]
    assert rel.max() < PK_RTOL, (rel.max(), int(np.argmax(rel)) + 1)


@pytest.mark.parametrize("n_side,mesh,box,seed", [(16, 32, 64.0, 42), (32, 64, 100.0, 7)])
def test_power_spectrum_of_ics_matches_oracle(cpm, orc, n_side, mesh, box, seed):
    _, x, _ = _ics(orc, n_side, box, 0.02, seed)
    shells = mesh // 2
    k_o, p_o, c_o = orc.power_spectrum(x, box, mesh, shells)
    k_g, p_g, c_g = cpm.power_spectrum(x, box, mesh, shells)
    _compare(k_g, p_g, c_g, k_o, p_o, c_o, mesh)


@pytest.mark.parametrize("mesh", [16, 64])
def test_power_spectrum_of_clustered_particles_matches_oracle(cpm, orc, mesh):
    box = 50.0
    x = _clustered(60_000, box, 3)
    shells = int(math.ceil(math.sqrt(3.0) * mesh / 2))  # every shell of the spectrum
    k_o, p_o, c_o = orc.power_spectrum(x, box, mesh, shells)
    k_g, p_g, c_g = cpm.power_spectrum(x, box, mesh, shells)
    _compare(k_g, p_g, c_g, k_o, p_o, c_o, mesh)
    # every mode of the n^3 spectrum but k = 0 falls in some shell 1..ceil(sqrt(3) n / 2)
    assert int(c_g.sum()) == mesh ** 3 - 1


def test_sim_power_spectrum_equals_particle_estimate(cpm, orc):
    c, x, p = _ics(orc, 16, 64.0, 0.02, 5)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    split = cpm.ForceSplit.with_(64.0, 32, 16, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation(cc, 64.0, 32, x, p, 0.02, split)
    for a1 in cpm.ln_a_schedule(0.02, 0.05, 2):
        sim.step_to(a1)
    k_s, p_s, c_s = sim.power_spectrum(16)
    k_g, p_g, c_g = cpm.power_spectrum(sim.positions, 64.0, 32, 16)
    np.testing.assert_array_equal(c_s, c_g)
    np.testing.assert_allclose(k_s, k_g, rtol=1e-12)
    np.testing.assert_allclose(p_s, p_g, rtol=1e-9)


def test_power_spectrum_rejects_bad_arguments(cpm):
    x = np.zeros((8, 3), np.float32)
    for shells in (0, 2049):
        with pytest.raises(cpm.CpmError):
            cpm.power_spectrum(x, 10.0, 16, shells)
    with pytest.raises(cpm.CpmError):
        cpm.power_spectrum(np.zeros((0, 3), np.float32), 10.0, 16, 4)
    with pytest.raises(cpm.CpmError):
        cpm.power_spectrum(x, 10.0, 100, 4)  # no compiled transform for n = 100
