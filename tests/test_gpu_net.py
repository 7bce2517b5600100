"""The learned short-range net's tcgen05 kernels (through the C ABI) against the numpy oracle
(oracle/net_oracle.py), which rounds to BF16 exactly where the kernels do and sums in FP64.

Bars: stored BF16 activations equal the oracle's except for rare one-ulp flips (FP32 accumulation
order against FP64), field within 2e-4 relative RMS, weight gradients within 2e-3 relative RMS per
layer; exact positive homogeneity (scaling by 2 is exact in every operation); a training run on a
teacher net's field reduces the loss.
"""
import numpy as np
import pytest

import net_oracle as no

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def _delta(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(n ** 3).astype(np.float32)
    d[rng.integers(0, n ** 3, n ** 3 // 50)] *= np.float32(20.0)  # a few dense cells
    return d


def _unpad(t, n):
    """(n, n, 2, n+8, 8) padded tensor -> (16, n, n, n) interior, plus its two halo planes."""
    a = t.reshape(n, n, 2, n + 8, 8)
    interior = a[:, :, :, 1:n + 1, :].transpose(2, 4, 0, 1, 3).reshape(16, n, n, n)
    lo = a[:, :, :, 0, :].transpose(2, 3, 0, 1).reshape(16, n, n)
    hi = a[:, :, :, n + 1, :].transpose(2, 3, 0, 1).reshape(16, n, n)
    return interior, lo, hi


@pytest.mark.parametrize("n", [32, 48, 144])
def test_net_forward_matches_oracle(cpm, n):
    import torch
    from importlib import import_module

    learned = import_module("cosmological-particle-simulation_b200.learned")
    w = no.random_weights(n)
    delta = _delta(n, n)
    net = cpm.ShortRangeNet(n, w)
    out = net.forward(torch.from_numpy(delta).cuda(), in_scale=0.5, out_scale=3.0)
    torch.cuda.synchronize()
    ref = no.forward_bf16(delta, w, 0.5, 3.0, n)
    # the stored activations of layer 1, interior and periodic halo
    a1, lo, hi = _unpad(learned.bf16_to_f32(net.tensor(1)), n)
    flips = np.mean(a1 != ref["a1"])
    assert flips < 1e-3, flips
    assert rel_rms(a1, ref["a1"]) < 1e-4
    assert np.array_equal(lo, a1[:, :, :, n - 1]) and np.array_equal(hi, a1[:, :, :, 0])
    got = out.cpu().numpy()
    assert np.all(got[:, 3] == 0.0)
    assert rel_rms(got[:, :3], ref["field"]) < 2e-4
    net.close()


@pytest.mark.parametrize("n", [32, 48])
def test_net_weight_gradient_matches_oracle(cpm, n):
    import torch

    w = no.random_weights(n + 1)
    delta = _delta(n, n + 1)
    net = cpm.ShortRangeNet(n, w)
    net.forward(torch.from_numpy(delta).cuda(), in_scale=0.5, out_scale=2.0)
    rng = np.random.default_rng(n)
    dfield = np.zeros((n ** 3, 4), np.float32)
    dfield[:, :3] = rng.standard_normal((n ** 3, 3)).astype(np.float32)
    grad = net.backward(torch.from_numpy(dfield).cuda(), out_scale=2.0)
    ref_state = no.forward_bf16(delta, w, 0.5, 2.0, n)
    ref = no.backward_bf16(ref_state, dfield[:, :3], 2.0, n)
    for layer in range(3):
        assert rel_rms(grad[layer], ref[layer]) < 2e-3, (layer, rel_rms(grad[layer], ref[layer]))
    assert np.all(grad[~no.live_mask()] == 0.0)
    net.close()


def test_net_is_exactly_homogeneous(cpm):
    import torch

    n = 32
    net = cpm.ShortRangeNet(n, no.random_weights(7))
    d = torch.from_numpy(_delta(n, 7)).cuda()
    f1 = net.forward(d).cpu().numpy()
    f2 = net.forward(2.0 * d).cpu().numpy()
    f0 = net.forward(torch.zeros_like(d)).cpu().numpy()
    assert np.array_equal(f2, 2.0 * f1)
    assert np.all(f0 == 0.0)
    net.close()


def test_net_training_reduces_the_loss_on_a_teacher_field(cpm):
    """Particles sample a teacher net's field; a student net trained by cpm_net_train_step (forward,
    CIC gather and loss, tcgen05 backward, Adam) fits it."""
    import torch

    n, box, npart = 32, 32.0, 40000
    rng = np.random.default_rng(11)
    teacher = no.random_weights(101, scale=0.6)
    delta = _delta(n, 12)
    x = rng.uniform(0.0, box, (npart, 3)).astype(np.float32)
    tf = no.forward_bf16(delta, teacher, 1.0, 1.0, n)["field"]
    target = no.cic_gather(tf.astype(np.float64), x, box, n).astype(np.float32)
    inv_norm = 1.0 / float((target.astype(np.float64) ** 2).sum())
    net = cpm.ShortRangeNet(n, no.random_weights(202, scale=0.6))
    dd = torch.from_numpy(delta).cuda()
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(target).cuda()
    wd = torch.ones(npart, dtype=torch.float32, device="cuda")
    losses = [net.train_step(dd, xd, td, wd, box, inv_norm, 3e-3) for _ in range(300)]
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])
    # the loss reported by the kernel is the oracle's loss of the same weights
    w_now = net.weights
    field = no.forward_bf16(delta, w_now, 1.0, 1.0, n)["field"].astype(np.float64)
    pred = no.cic_gather(field, x, box, n)
    want = float(((pred - target) ** 2).sum() * inv_norm)
    got = net.train_step(dd, xd, td, wd, box, inv_norm, 0.0)
    assert abs(got - want) < 1e-3 * want + 1e-7, (got, want)
    net.close()
