"""The net oracle (oracle/net_oracle.py) against finite differences and its own identities, on the
CPU: the backward pass it uses to check the GPU's gradients is the exact gradient of its forward."""
import numpy as np

import net_oracle as no


def _setup(n=8, seed=0):
    rng = np.random.default_rng(seed)
    w = no.random_weights(seed, scale=0.8).astype(np.float64)
    delta = rng.standard_normal(n ** 3)
    r = rng.standard_normal((n ** 3, 3))
    return w, delta, r


def _loss(w, delta, r, n):
    st = no.forward64(delta, w, 0.7, 1.3, n)
    return float((st["field"] * r).sum())


def test_backward64_matches_finite_differences():
    n = 8
    w, delta, r = _setup(n)
    st = no.forward64(delta, w, 0.7, 1.3, n)
    grad = no.backward64(st, w, r, 1.3, n)
    live = np.argwhere(no.live_mask())
    rng = np.random.default_rng(5)
    for k in rng.choice(len(live), 24, replace=False):
        idx = tuple(live[k])
        eps = 1e-6 * max(1.0, abs(w[idx]))
        wp, wm = w.copy(), w.copy()
        wp[idx] += eps
        wm[idx] -= eps
        fd = (_loss(wp, delta, r, n) - _loss(wm, delta, r, n)) / (2 * eps)
        assert abs(fd - grad[idx]) <= 1e-5 * max(1.0, abs(fd)), (idx, fd, grad[idx])


def test_conv_t_is_the_adjoint_of_conv():
    rng = np.random.default_rng(1)
    n = 6
    w = rng.standard_normal((27, 16, 16))
    a = rng.standard_normal((16, n, n, n))
    b = rng.standard_normal((16, n, n, n))
    assert abs((no.conv(a, w) * b).sum() - (a * no.conv_t(b, w)).sum()) < 1e-9 * np.abs(a).sum() * np.abs(b).sum()


def test_net_is_positively_homogeneous():
    n = 8
    w, delta, _ = _setup(n, 3)
    f1 = no.forward64(delta, w, 1.0, 1.0, n)["field"]
    f2 = no.forward64(2.5 * delta, w, 1.0, 1.0, n)["field"]
    assert np.allclose(f2, 2.5 * f1, rtol=1e-12, atol=1e-12)
    assert np.abs(no.forward64(np.zeros(n ** 3), w, 1.0, 1.0, n)["field"]).max() == 0.0


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-39], np.float32)
    got = no.bf16(x)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == np.float32(1.0 + 4 * 2 ** -8)
    assert got[3] == 1.0 and got[4] == -2.5


def test_cic_scatter_is_the_adjoint_of_gather():
    rng = np.random.default_rng(2)
    n, box = 8, 4.0
    x = rng.uniform(0, box, (300, 3))
    f = rng.standard_normal((n ** 3, 3))
    v = rng.standard_normal((300, 3))
    assert abs((no.cic_gather(f, x, box, n) * v).sum() - (f * no.cic_scatter(v, x, box, n)).sum()) < 1e-9
