"""Python front end of the learned short-range force (cpm_net_* in include/cpm.h).

The reference has no learned component: its short-range force is the tree walk of tree.rs:264-310.
`ShortRangeNet` owns a cpm_net (BF16 tcgen05 convolution kernels with FP32 master weights and
Adam state on the device). Device arrays are torch CUDA tensors, used here only as device memory;
every computation runs in libcpm_cuda.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import CpmError

WEIGHT_SHAPE = (3, 27, 16, 16)


def _check(rc: int, handle) -> None:
    if rc != nat.CPM_OK:
        msg = nat.lib().cpm_net_last_error(handle)
        raise CpmError(rc, msg.decode() if msg else "")


def _dev_ptr(t, dtype_name: str, numel: int):
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
        raise CpmError(-1, "expected a contiguous CUDA tensor")
    if str(t.dtype) != dtype_name or t.numel() != numel:
        raise CpmError(-1, f"expected {numel} elements of {dtype_name}, got {t.numel()} of {t.dtype}")
    return C.c_void_p(t.data_ptr())


class ShortRangeNet:
    """A 3-layer 3x3x3 convolutional net on an n^3 mesh: F = out_scale * net(in_scale * delta)."""

    def __init__(self, n_mesh: int, weights: np.ndarray | None = None):
        h = C.c_void_p()
        rc = nat.lib().cpm_net_create(int(n_mesh), C.byref(h))
        if rc != nat.CPM_OK:
            raise CpmError(rc, nat.last_error(None))
        self.h = h
        self.n = int(n_mesh)
        if weights is not None:
            self.weights = weights

    @property
    def weights(self) -> np.ndarray:
        w = np.empty(WEIGHT_SHAPE, np.float32)
        _check(nat.lib().cpm_net_get_weights(self.h, nat.ptr(w)), self.h)
        return w

    @weights.setter
    def weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32).reshape(WEIGHT_SHAPE)
        _check(nat.lib().cpm_net_set_weights(self.h, nat.ptr(w)), self.h)

    def grads(self) -> np.ndarray:
        g = np.empty(WEIGHT_SHAPE, np.float32)
        _check(nat.lib().cpm_net_get_grads(self.h, nat.ptr(g)), self.h)
        return g

    def forward(self, delta, in_scale: float = 1.0, out_scale: float = 1.0, out=None, stream=None):
        """delta: CUDA float32 tensor of n^3 cells; returns (or fills) an (n^3, 4) float32 CUDA tensor."""
        import torch

        m = self.n ** 3
        if out is None:
            out = torch.empty((m, 4), dtype=torch.float32, device=delta.device)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _check(nat.lib().cpm_net_forward(self.h, _dev_ptr(delta, "torch.float32", m), float(in_scale),
                                         float(out_scale), _dev_ptr(out, "torch.float32", 4 * m), C.c_void_p(s)),
               self.h)
        return out

    def backward(self, dfield, out_scale: float = 1.0, stream=None) -> np.ndarray:
        """Weight gradient for dL/dF = dfield ((n^3, 4) CUDA float32) after the last forward."""
        import torch

        m = self.n ** 3
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _check(nat.lib().cpm_net_backward(self.h, _dev_ptr(dfield, "torch.float32", 4 * m), float(out_scale),
                                          C.c_void_p(s)), self.h)
        return self.grads()

    def tensor(self, which: int):
        """Internal BF16 tensor (0 input, 1-2 activations, 3-5 gradients of layers 3, 2, 1) as a
        uint16 CUDA tensor shaped (n, n, 2, n + 8, 8)."""
        import torch

        n = self.n
        out = torch.empty((n, n, 2, n + 8, 8), dtype=torch.int16, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        _check(nat.lib().cpm_net_activations(self.h, int(which), C.c_void_p(out.data_ptr()), C.c_void_p(s)), self.h)
        return out

    def train_step(self, delta, x3, target3, weight, box_size: float, inv_norm: float, lr: float,
                   in_scale: float = 1.0, stream=None) -> float:
        """One Adam step on one mesh and its particles; returns the loss before the update."""
        import torch

        m = self.n ** 3
        npart = int(x3.numel() // 3)
        loss = C.c_double(0.0)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _check(nat.lib().cpm_net_train_step(self.h, _dev_ptr(delta, "torch.float32", m), float(in_scale),
                                            _dev_ptr(x3, "torch.float32", 3 * npart),
                                            _dev_ptr(target3, "torch.float32", 3 * npart),
                                            _dev_ptr(weight, "torch.float32", npart), npart, float(box_size),
                                            float(inv_norm), float(lr), C.byref(loss), C.c_void_p(s)), self.h)
        return float(loss.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            nat.lib().cpm_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bf16_to_f32(t) -> np.ndarray:
    """uint16/int16 bfloat16 bits (any shape, host or device) as float32 numpy."""
    a = t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)
    return (a.astype(np.uint16).astype(np.uint32) << 16).view(np.float32)
