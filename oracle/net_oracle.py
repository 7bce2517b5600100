"""CPU oracle of the learned short-range net (test infrastructure only: imported by tests/, never by
the library). The reference has no learned component; this is a numpy restatement of the math the
library's tensor-core kernels implement, so that their forward pass and gradients can be checked.

Net: three 3x3x3 periodic convolutions without biases, 16 channels, leaky ReLU (slope 1/8) after the
first two: y = W3 * lrelu(W2 * lrelu(W1 * x)), x = in_scale * delta in channel 0, F = out_scale * y
(channels 0-2). Convolution: out[v] = sum_t W[t] in[v + t], t = (dx, dy, dz) in {-1,0,1}^3, tap
index (dx+1)*9 + (dy+1)*3 + (dz+1); W[layer][tap][out][in].

`forward_bf16` / `backward_bf16` round exactly where the kernels round (inputs, weights and stored
activations and gradients to BF16, round to nearest even) and sum in FP64, so they differ from the
kernels only by the FP32 accumulation order. `forward64` / `backward64` are the same math in FP64
without rounding, checked against finite differences (tests/test_net_oracle.py).
"""
from __future__ import annotations

import numpy as np

SLOPE = 0.125
C = 16
TAPS = [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)]


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    out = ((u + r) & 0xFFFF0000).astype(np.uint32)
    return out.view(np.float32).reshape(a.shape)


def live_mask() -> np.ndarray:
    """Master weights that exist: layer 1 reads input channel 0 only, layer 3 writes channels 0-2."""
    m = np.ones((3, 27, C, C), bool)
    m[0, :, :, 1:] = False
    m[2, :, 3:, :] = False
    return m


def random_weights(seed: int, scale: float = 0.3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((3, 27, C, C)).astype(np.float32)
    w *= np.float32(scale) / np.sqrt(np.array([27.0, 27.0 * C, 27.0 * C], np.float32))[:, None, None, None]
    return (w * live_mask()).astype(np.float32)


def conv(inp: np.ndarray, w: np.ndarray) -> np.ndarray:
    """out[o, v] = sum_t sum_i w[t, o, i] inp[i, v + t] (periodic); inp (C, n, n, n), FP64."""
    out = np.zeros((w.shape[1],) + inp.shape[1:], np.float64)
    for t, (dx, dy, dz) in enumerate(TAPS):
        shifted = np.roll(inp, shift=(-dx, -dy, -dz), axis=(1, 2, 3))
        out += np.tensordot(w[t].astype(np.float64), shifted, axes=([1], [0]))
    return out


def conv_t(grad: np.ndarray, w: np.ndarray) -> np.ndarray:
    """The adjoint of conv: din[i, v] = sum_t sum_o w[t, o, i] grad[o, v - t]."""
    out = np.zeros((w.shape[2],) + grad.shape[1:], np.float64)
    for t, (dx, dy, dz) in enumerate(TAPS):
        shifted = np.roll(grad, shift=(dx, dy, dz), axis=(1, 2, 3))
        out += np.tensordot(w[t].astype(np.float64).T, shifted, axes=([1], [0]))
    return out


def wgrad(grad: np.ndarray, inp: np.ndarray) -> np.ndarray:
    """dW[t, o, i] = sum_v grad[o, v] inp[i, v + t]."""
    out = np.zeros((27, grad.shape[0], inp.shape[0]), np.float64)
    g2 = grad.reshape(grad.shape[0], -1).astype(np.float64)
    for t, (dx, dy, dz) in enumerate(TAPS):
        shifted = np.roll(inp, shift=(-dx, -dy, -dz), axis=(1, 2, 3)).reshape(inp.shape[0], -1)
        out[t] = g2 @ shifted.astype(np.float64).T
    return out


def lrelu(z):
    return np.where(z > 0, z, SLOPE * z)


def _input(delta: np.ndarray, in_scale: float, n: int) -> np.ndarray:
    x = np.zeros((C, n, n, n), np.float32)
    x[0] = (delta.reshape(n, n, n).astype(np.float32) * np.float32(in_scale)).astype(np.float32)
    return x


def forward_bf16(delta: np.ndarray, w: np.ndarray, in_scale: float, out_scale: float, n: int) -> dict:
    """Forward pass with the kernels' roundings; returns the field (n^3, 3) and the stored tensors."""
    wb = bf16(w)
    x0 = bf16(_input(delta, in_scale, n))
    a1 = bf16(lrelu(conv(x0, wb[0]).astype(np.float32)))
    a2 = bf16(lrelu(conv(a1, wb[1]).astype(np.float32)))
    y = conv(a2, wb[2]).astype(np.float32)
    field = (y[:3].reshape(3, -1).T * np.float32(out_scale)).astype(np.float32)
    return {"x0": x0, "a1": a1, "a2": a2, "y": y, "field": field, "wb": wb}


def backward_bf16(state: dict, dfield: np.ndarray, out_scale: float, n: int) -> np.ndarray:
    """Weight gradient (3, 27, 16, 16) from dL/dF (n^3, 3) with the kernels' roundings."""
    wb = state["wb"]
    g3 = np.zeros((C, n, n, n), np.float32)
    g3[:3] = (dfield[:, :3].T.reshape(3, n, n, n) * np.float32(out_scale)).astype(np.float32)
    g3 = bf16(g3)
    dw = np.zeros((3, 27, C, C), np.float64)
    dw[2] = wgrad(g3, state["a2"])
    gate2 = np.where(state["a2"] > 0, np.float32(1.0), np.float32(SLOPE))
    g2 = bf16(conv_t(g3, wb[2]).astype(np.float32) * gate2)
    dw[1] = wgrad(g2, state["a1"])
    gate1 = np.where(state["a1"] > 0, np.float32(1.0), np.float32(SLOPE))
    g1 = bf16(conv_t(g2, wb[1]).astype(np.float32) * gate1)
    dw[0] = wgrad(g1, state["x0"])
    return dw * live_mask()


def forward64(delta: np.ndarray, w: np.ndarray, in_scale: float, out_scale: float, n: int) -> dict:
    x0 = np.zeros((C, n, n, n))
    x0[0] = delta.reshape(n, n, n) * in_scale
    z1 = conv(x0, w[0])
    a1 = lrelu(z1)
    z2 = conv(a1, w[1])
    a2 = lrelu(z2)
    y = conv(a2, w[2])
    return {"x0": x0, "z1": z1, "a1": a1, "z2": z2, "a2": a2, "field": y[:3].reshape(3, -1).T * out_scale}


def backward64(state: dict, w: np.ndarray, dfield: np.ndarray, out_scale: float, n: int) -> np.ndarray:
    g3 = np.zeros((C, n, n, n))
    g3[:3] = dfield[:, :3].T.reshape(3, n, n, n) * out_scale
    dw = np.zeros((3, 27, C, C))
    dw[2] = wgrad(g3, state["a2"])
    g2 = conv_t(g3, w[2]) * np.where(state["z2"] > 0, 1.0, SLOPE)
    dw[1] = wgrad(g2, state["a1"])
    g1 = conv_t(g2, w[1]) * np.where(state["z1"] > 0, 1.0, SLOPE)
    dw[0] = wgrad(g1, state["x0"])
    return dw * live_mask()


def cic_gather(field: np.ndarray, x: np.ndarray, box: float, n: int) -> np.ndarray:
    """CIC interpolation (mesh.rs:29-77 stencil, FP64 sums) of an (n^3, k) field at positions x."""
    h = box / n
    s = x.astype(np.float64) / h - 0.5
    i0 = np.floor(s).astype(np.int64)
    f = s - i0
    out = np.zeros((len(x), field.shape[1]))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (np.where(dx, f[:, 0], 1 - f[:, 0]) * np.where(dy, f[:, 1], 1 - f[:, 1])
                     * np.where(dz, f[:, 2], 1 - f[:, 2]))
                idx = (((i0[:, 0] + dx) % n) * n + (i0[:, 1] + dy) % n) * n + (i0[:, 2] + dz) % n
                out += w[:, None] * field[idx]
    return out


def cic_scatter(values: np.ndarray, x: np.ndarray, box: float, n: int) -> np.ndarray:
    """The adjoint of cic_gather: an (n^3, k) field."""
    h = box / n
    s = x.astype(np.float64) / h - 0.5
    i0 = np.floor(s).astype(np.int64)
    f = s - i0
    out = np.zeros((n ** 3, values.shape[1]))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (np.where(dx, f[:, 0], 1 - f[:, 0]) * np.where(dy, f[:, 1], 1 - f[:, 1])
                     * np.where(dz, f[:, 2], 1 - f[:, 2]))
                idx = (((i0[:, 0] + dx) % n) * n + (i0[:, 1] + dy) % n) * n + (i0[:, 2] + dz) % n
                np.add.at(out, idx, w[:, None] * values)
    return out
