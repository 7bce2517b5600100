"""Pins the CPU oracle to the reference crate's own known-answer tests.

Each test restates one `#[test]` of the reference (file:line in its docstring) with the same
inputs and tolerance, run against the oracle. These are the oracle's pins: the reference cannot
be compiled here (no Rust toolchain), so its own tests are the golden vectors.
"""
import math

import numpy as np
import pytest


# ------------------------------------------------------------------ mesh.rs

def test_deposit_conserves_total_mass(orc):
    """mesh.rs:101-109"""
    pos = orc.scattered_mesh(5000, 1.0)
    cells = orc.deposit(16, 1.0, pos, 0.25)
    total = np.float32(0.0)
    for v in cells:  # f32 sequential sum, as `cells.iter().sum()`
        total = np.float32(total + v)
    assert abs(total - 0.25 * 5000.0) < 1e-5 * 0.25 * 5000.0


def test_particle_at_cell_centre_fills_one_cell(orc):
    """mesh.rs:111-124"""
    n, box = 8, 1.0
    h = np.float32(box) / np.float32(n)
    p = np.array([np.float32(2.5) * h, np.float32(3.5) * h, np.float32(4.5) * h], np.float32)
    cells = orc.deposit(n, box, p[None, :], 1.0)
    assert abs(cells[(2 * n + 3) * n + 4] - 1.0) < 1e-5
    assert abs(cells.sum(dtype=np.float64) - 1.0) < 1e-5
    assert int((cells > 1e-12).sum()) == 1


def test_lattice_deposits_uniform_grid(orc):
    """mesh.rs:126-149"""
    n, box = 8, 2.0
    h = np.float32(box) / np.float32(n)
    g = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * h
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    cells = orc.deposit(n, box, pos, 3.0)
    assert np.all(np.abs(cells - 3.0) < 1e-5)


def test_particle_on_boundary_wraps_to_opposite_face(orc):
    """mesh.rs:151-162"""
    n, box = 4, 1.0
    h = np.float32(box) / np.float32(n)
    p = np.array([[box, np.float32(0.5) * h, np.float32(0.5) * h]], np.float32)
    cells = orc.deposit(n, box, p, 1.0)
    assert abs(cells[((n - 1) * n + 0) * n + 0] - 0.5) < 1e-5
    assert abs(cells[0] - 0.5) < 1e-5


def test_interpolating_constant_field_returns_constant(orc):
    """mesh.rs:164-171"""
    cells = np.full(8 ** 3, 2.5, np.float32)
    vals = orc.interpolate_many(8, 1.0, cells, orc.scattered_mesh(200, 1.0))
    assert np.all(np.abs(vals - 2.5) < 1e-5)


def test_interpolation_reproduces_cell_value_at_centre(orc):
    """mesh.rs:173-183"""
    n = 8
    h = np.float32(1.0) / np.float32(n)
    cells = np.zeros(n ** 3, np.float32)
    cells[(5 * n + 1) * n + 6] = 7.0
    v = orc.interpolate(n, 1.0, cells, np.array([5.5 * h, 1.5 * h, 6.5 * h], np.float32))
    assert abs(v - 7.0) < 1e-5


# ------------------------------------------------------------------ poisson.rs

def _mesh_from_fn(n, box, f):
    h = np.float32(box) / np.float32(n)
    x = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * h
    vals = f(x).astype(np.float32)
    return np.broadcast_to(vals[:, None, None], (n, n, n)).ravel().copy()


def test_plane_wave_force_matches_analytic(orc):
    """poisson.rs:114-139"""
    n, box, a = 16, 1.0, 0.5
    cosmo = orc.lcdm_default()
    k0 = np.float32(2.0 * np.float32(np.pi))
    c = np.float32(np.float32(1.5) * np.float32(cosmo.omega_m)) / np.float32(a)
    delta = _mesh_from_fn(n, box, lambda x: np.cos(k0 * x))
    gx, gy, gz = orc.poisson_accel(n, box, delta, cosmo.omega_m, a, 0.0)
    expected = _mesh_from_fn(n, box, lambda x: -(c / k0) * np.sin(k0 * x))
    amplitude = c / k0
    assert np.max(np.abs(gx - expected)) < 1e-5 * amplitude
    assert np.max(np.abs(gy)) < 1e-5 * amplitude
    assert np.max(np.abs(gz)) < 1e-5 * amplitude


def test_uniform_density_contrast_gives_no_force(orc):
    """poisson.rs:141-152"""
    cosmo = orc.lcdm_default()
    delta = np.ones(8 ** 3, np.float32)
    for g in orc.poisson_accel(8, 1.0, delta, cosmo.omega_m, 1.0, 0.0):
        assert np.max(np.abs(g)) < 1e-5


def test_force_scales_inversely_with_scale_factor(orc):
    """poisson.rs:154-165"""
    cosmo = orc.lcdm_default()
    delta = _mesh_from_fn(16, 1.0, lambda x: np.cos(np.float32(2.0 * np.pi) * x))
    g_early = orc.poisson_accel(16, 1.0, delta, cosmo.omega_m, 0.5, 0.0)[0]
    g_late = orc.poisson_accel(16, 1.0, delta, cosmo.omega_m, 1.0, 0.0)[0]
    ratio = np.max(np.abs(g_early)) / np.max(np.abs(g_late))
    assert abs(ratio - 2.0) < 1e-4


# ------------------------------------------------------------------ tree.rs

def test_short_range_factor_limits(orc):
    """tree.rs:382-394"""
    assert abs(orc.short_range_factor(0.0, 1.0) - 1.0) < 1e-6
    assert orc.short_range_factor(10.0, 1.0) < 1e-6
    prev = 1.0
    for step in range(1, 51):
        s = orc.short_range_factor(float(np.float32(step) * np.float32(0.1)), 1.0)
        assert s <= prev + 1e-7
        prev = s


def _max_norm(v):
    return float(np.max(np.sqrt((v.astype(np.float64) ** 2).sum(1))))


def _max_diff(a, b):
    return float(np.max(np.sqrt(((a.astype(np.float64) - b) ** 2).sum(1))))


def test_tree_with_theta_zero_matches_brute_force(orc):
    """tree.rs:396-406"""
    split = orc.Split(0.5, 2.0, 0.05, 0.0)
    pos = orc.scattered_tree(400, 10.0, 7)
    fast = orc.tree_accelerations(pos, 10.0, split, 1.0)
    slow = orc.brute_force(pos, 10.0, split, 1.0)
    assert _max_diff(fast, slow) / _max_norm(slow) < 1e-5


def test_tree_with_theta_half_is_close_to_brute_force(orc):
    """tree.rs:408-418"""
    split = orc.Split(0.5, 2.5, 0.05, 0.5)
    pos = orc.scattered_tree(3000, 10.0, 11)
    fast = orc.tree_accelerations(pos, 10.0, split, 1.0)
    slow = orc.brute_force(pos, 10.0, split, 1.0)
    assert _max_diff(fast, slow) / _max_norm(slow) < 0.02


def test_periodic_pair_interacts_across_the_boundary(orc):
    """tree.rs:420-430"""
    split = orc.Split(0.5, 2.0, 0.05, 0.5)
    pos = np.array([[0.1, 5.0, 5.0], [9.9, 5.0, 5.0]], np.float32)
    acc = orc.tree_accelerations(pos, 10.0, split, 1.0)
    assert acc[0, 0] < 0.0
    assert acc[1, 0] > 0.0


def test_builtin_walk_agrees_with_tree_walk(orc):
    """tree.rs:103-150 vs :264-310: the two walk variants differ only in rounding of the tests."""
    split = orc.Split(0.5, 2.5, 0.05, 0.5)
    pos = orc.scattered_tree(3000, 10.0, 11)
    a = orc.tree_accelerations(pos, 10.0, split, 1.0)
    b = orc.tree_accelerations_builtin(pos, 10.0, split, 1.0)
    rms = np.sqrt(((a.astype(np.float64) - b) ** 2).sum() / (a.astype(np.float64) ** 2).sum())
    assert rms < 1e-4


# ------------------------------------------------------------------ cosmology.rs

def test_expansion_rate_is_one_today(orc):
    """cosmology.rs:110-115"""
    c = orc.lcdm_default()
    assert abs(orc.cosmo_e(c, 1.0) - 1.0) < 1e-5


def test_growth_is_one_today(orc):
    """cosmology.rs:117-121"""
    assert abs(orc.growth(orc.lcdm_default(), 1.0) - 1.0) < 1e-5


def test_growth_scales_as_a_early(orc):
    """cosmology.rs:123-131"""
    d = orc.lcdm_default()
    c = orc.cosmology(0.0, d.omega_m, d.omega_l, d.h0)
    r1 = orc.growth(c, 1e-3) / 1e-3
    r2 = orc.growth(c, 2e-3) / 2e-3
    assert abs(r1 - r2) / r1 < 1e-4


def test_growth_matches_reference_at_half(orc):
    """cosmology.rs:133-139: golden value D(0.5) = 0.6068044."""
    assert abs(orc.growth(orc.lcdm_default(), 0.5) - 0.6068044) < 1e-4


# ------------------------------------------------------------------ ics.rs

N_S, SIGMA8, SIGMA8_RADIUS = 0.965, 0.811, 8.0  # ics.rs:15-18


def test_bbks_transfer_is_one_at_large_scales(orc):
    """ics.rs:189-193"""
    assert abs(orc.bbks(orc.lcdm_default(), 1e-6) - 1.0) < 1e-3


def test_normalized_spectrum_gives_sigma8(orc):
    """ics.rs:195-202"""
    c = orc.lcdm_default()
    ps = orc.power_normalized(c, N_S, SIGMA8, SIGMA8_RADIUS)
    s8 = orc.sigma(c, ps, SIGMA8_RADIUS)
    assert abs(s8 - SIGMA8) / SIGMA8 < 1e-6


def test_growth_rate_matches_omega_m_approximation_today(orc):
    """ics.rs:204-210"""
    c = orc.lcdm_default()
    assert abs(orc.growth_rate(c, 1.0) - c.omega_m ** 0.55) < 0.01


def test_measured_power_matches_input(orc):
    """ics.rs:212-266 (shell-binned power of the coloured modes within 3 sigma)."""
    n, box = 32, 100.0
    c = orc.lcdm_default()
    ps = orc.power_normalized(c, N_S, SIGMA8, SIGMA8_RADIUS)
    modes = orc.colored_modes(n, box, c, ps, 42).reshape(n, n, n)
    n3 = float(n ** 3)
    volume = box ** 3
    kf = 2.0 * math.pi / box
    m = np.arange(n)
    m = np.where(m <= n // 2, m, m - n)
    mx, my, mz = np.meshgrid(m, m, m, indexing="ij")
    keep = ~((np.abs(mx) == n // 2) | (np.abs(my) == n // 2) | (np.abs(mz) == n // 2))
    m2 = mx ** 2 + my ** 2 + mz ** 2
    shell = np.rint(np.sqrt(m2)).astype(int)
    keep &= (shell > 0) & (shell < n)
    p_meas = volume * np.abs(modes.astype(np.complex128)) ** 2 / (n3 * n3)
    checked = 0
    for s in range(1, n):
        sel = keep & (shell == s)
        cnt = int(sel.sum())
        if cnt < 200:
            continue
        meas = p_meas[sel].mean()
        exp = np.mean([orc.power(c, ps, float(kf * math.sqrt(v))) for v in m2[sel]])
        tol = 3.0 * math.sqrt(2.0 / cnt)
        assert abs(meas - exp) / exp < tol, (s, meas, exp)
        checked += 1
    assert checked >= 3


# ------------------------------------------------------------------ integrator.rs

def _plane_wave(orc, n, box, amp, cosmo, a_init):
    """integrator.rs:326-348 in f32."""
    f32 = np.float32
    k = f32(f32(2.0) * f32(np.pi)) / f32(box)
    h = f32(box) / f32(n)
    d = f32(orc.growth(cosmo, a_init))
    f = f32(orc.growth_rate(cosmo, a_init))
    e = f32(orc.cosmo_e(cosmo, a_init))
    a = f32(a_init)
    i = np.arange(n, dtype=np.float32) * h
    qx, qy, qz = np.meshgrid(i, i, i, indexing="ij")
    qx, qy, qz = qx.ravel(), qy.ravel(), qz.ravel()
    psi_x = (-(f32(amp) / k) * np.sin(k * qx).astype(np.float32)).astype(np.float32)
    x = np.mod(qx + d * psi_x, f32(box)).astype(np.float32)
    pos = np.stack([x, qy, qz], 1).astype(np.float32)
    mom = np.zeros_like(pos)
    mom[:, 0] = (a * a * f * e * d) * psi_x
    return pos, mom


def _mode_amplitude(orc, x, n, box):
    """integrator.rs:351-366"""
    delta = orc.density_contrast(n, box, x).reshape(n, n, n).astype(np.float64)
    h = box / n
    k = 2.0 * np.pi / box
    cx = np.cos((np.arange(n) + 0.5) * h * k)
    return 2.0 * float((delta * cx[:, None, None]).sum()) / n ** 3


def _run(orc, sim, a_start, a_end, steps):
    for a1 in orc.ln_a_schedule(a_start, a_end, steps):
        sim.step_to(a1)


def test_linear_growth_matches_growth_factor(orc):
    """integrator.rs:368-388"""
    box, cosmo = 1.0, orc.lcdm_default()
    a_init, a_final, amp = 0.02, 0.1, 0.5
    x, p = _plane_wave(orc, 32, box, amp, cosmo, a_init)
    sim = orc.Simulation(cosmo, box, 32, x, p, a_init, None)
    before = _mode_amplitude(orc, x, 32, box)
    _run(orc, sim, a_init, a_final, 40)
    after = _mode_amplitude(orc, sim.state()["x"], 32, box)
    expected = orc.growth(cosmo, a_final) / orc.growth(cosmo, a_init)
    assert abs(after / before - expected) / expected < 0.01


def test_steps_converge(orc):
    """integrator.rs:390-415"""
    box, cosmo = 1.0, orc.lcdm_default()

    def run(steps):
        x, p = _plane_wave(orc, 16, box, 0.5, cosmo, 0.02)
        sim = orc.Simulation(cosmo, box, 32, x, p, 0.02, None)
        _run(orc, sim, 0.02, 0.1, steps)
        return sim.state()["x"]

    d = np.abs(run(10).astype(np.float64) - run(40))
    d = np.minimum(d, box - d)
    assert d.max() < 1e-3 * box


def test_total_momentum_stays_near_zero(orc):
    """integrator.rs:417-435"""
    box, cosmo = 1.0, orc.lcdm_default()
    x, p = _plane_wave(orc, 16, box, 0.5, cosmo, 0.02)
    sim = orc.Simulation(cosmo, box, 32, x, p, 0.02, None)
    _run(orc, sim, 0.02, 0.1, 20)
    mom = sim.state()["p"].astype(np.float64)
    scale = np.abs(mom[:, 0]).sum()
    assert np.all(np.abs(mom.sum(0)) < 1e-3 * scale)


def test_treepm_pair_force_matches_newton(orc):
    """integrator.rs:437-461"""
    box, mesh_n = 100.0, 64
    cosmo = orc.lcdm_default()
    a, n = 1.0, 2.0
    std = orc.split_with(box, mesh_n, 2, 0.05, 0.5)
    split = orc.Split(std.r_split, std.r_cut, 0.01, std.theta)
    pos = np.array([[50.0, 50.0, 50.0], [53.0, 50.0, 50.0]], np.float32)
    sim = orc.Simulation(cosmo, box, mesh_n, pos, np.zeros_like(pos), a, split)
    acc = sim.accelerations(a)
    f32 = np.float32
    k = f32(1.5) * f32(cosmo.omega_m) * f32(box) ** 3 / (f32(4.0) * f32(np.pi) * f32(a) * f32(n))
    newton = float(k / f32(9.0))
    assert acc[0, 0] > 0.0 and acc[1, 0] < 0.0
    assert abs(acc[0, 0] - newton) / newton < 0.05
    assert abs(acc[1, 0] + newton) / newton < 0.05
