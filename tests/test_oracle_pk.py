"""The oracle's particle power spectrum (the checker of the GPU estimator) pinned against the
reference's estimator of ics.rs:213-266 written out in numpy, and against the linear power it must
recover from Zel'dovich initial conditions."""
import math

import numpy as np

N_S, SIGMA8, SIGMA8_RADIUS = 0.96, 0.8, 8.0


def _reference_estimator(delta, box, n_shells):
    """ics.rs:229-243: V |F|^2 / M^2 binned in shells round(|m|), here over every mode (the
    reference's test also drops Nyquist-containing modes, which its coloured modes leave zero)."""
    n = delta.shape[0]
    f = np.fft.fftn(delta)
    m = np.arange(n)
    m = np.where(m <= n // 2, m, m - n)
    mx, my, mz = np.meshgrid(m, m, m, indexing="ij")
    m2 = mx ** 2 + my ** 2 + mz ** 2
    shell = np.rint(np.sqrt(m2)).astype(int)
    pw = box ** 3 * np.abs(f) ** 2 / float(n ** 3) ** 2
    kf = 2.0 * math.pi / box
    k_mean, p_mean, counts = np.zeros(n_shells), np.zeros(n_shells), np.zeros(n_shells, np.uint64)
    for s in range(1, n_shells + 1):
        sel = shell == s
        c = int(sel.sum())
        counts[s - 1] = c
        if c:
            k_mean[s - 1] = kf * np.sqrt(m2[sel]).mean()
            p_mean[s - 1] = pw[sel].mean()
    return k_mean, p_mean, counts


def test_oracle_power_spectrum_is_the_reference_estimator(orc):
    rng = np.random.default_rng(11)
    box, n = 10.0, 16
    x = rng.uniform(0.0, box, (3000, 3)).astype(np.float32)
    rho = orc.deposit_f64(n, box, x, 1.0).reshape(n, n, n)
    delta = rho / (len(x) / n ** 3) - 1.0
    k_r, p_r, c_r = _reference_estimator(delta, box, 14)
    k_o, p_o, c_o = orc.power_spectrum(x, box, n, 14)
    np.testing.assert_array_equal(c_o, c_r)
    np.testing.assert_allclose(k_o, k_r, rtol=1e-12)
    np.testing.assert_allclose(p_o, p_r, rtol=1e-9)


def test_oracle_power_spectrum_of_ics_recovers_linear_power(orc):
    """Zel'dovich ICs at a = 0.02: shell power = D(a)^2 P_lin(k) times the CIC window squared,
    within 3 sigma of sampling (sqrt(2 / N_modes)) plus 3 % for the window's shell average."""
    n, box, a = 32, 200.0, 0.02
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    ps = orc.power_normalized(c, N_S, SIGMA8, SIGMA8_RADIUS)
    x, _ = orc.zeldovich(n, box, c, ps, a, 42)
    k_o, p_o, c_o = orc.power_spectrum(x, box, n, n // 4)
    d2 = orc.growth(c, a) ** 2
    m = np.arange(n)
    m = np.where(m <= n // 2, m, m - n)
    mx, my, mz = np.meshgrid(m, m, m, indexing="ij")
    m2 = mx ** 2 + my ** 2 + mz ** 2
    shell = np.rint(np.sqrt(m2)).astype(int)
    win = (np.sinc(mx / n) * np.sinc(my / n) * np.sinc(mz / n)) ** 4  # (CIC window)^2, np.sinc = sin(pi t)/(pi t)
    kf = 2.0 * math.pi / box
    checked = 0
    for s in range(2, n // 4 + 1):
        sel = shell == s
        cnt = int(sel.sum())
        assert cnt == int(c_o[s - 1])
        exp = np.mean([d2 * orc.power(c, ps, float(kf * math.sqrt(v))) * w for v, w in zip(m2[sel], win[sel])])
        tol = 3.0 * math.sqrt(2.0 / cnt) + 0.03
        assert abs(p_o[s - 1] - exp) / exp < tol, (s, p_o[s - 1], exp)
        checked += 1
    assert checked >= 5
