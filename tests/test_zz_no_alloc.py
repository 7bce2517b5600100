"""The allocation-free CIC deposit (cpm_mesh_deposit_noalloc), called through the C ABI.

It exists for callers that cannot call cudaMalloc (code running during CUDA-graph stream capture,
or programs whose device memory belongs to their own allocator): positions and the output mesh
are the caller's device buffers and the only scratch is a static device array. Its output must
equal the allocating entry point's (cpm_mesh_deposit) — both sum the same 64-bit fixed-point
weights, so the test asks for equality, inside the 1e-6 relative bar of the deposit tests — on
consecutive calls that share the static array. The file name sorts last so a run that stops at
the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn(cpm):
    f = cpm.lib().cpm_mesh_deposit_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
    return f


def test_noalloc_deposit_matches_allocating_deposit(cpm, orc):
    import torch

    fn = _fn(cpm)
    cases = [(20000, 32, 1.0, 0.5), (50000, 64, 64.0, 1.0), (20000, 32, 1.0, 0.5)]
    stream = torch.cuda.current_stream()
    for n, mesh, box, mass in cases:
        x = orc.scattered_mesh(n, box)
        ref = cpm.Mesh(mesh, box)
        ref.deposit(x, mass)
        xd = torch.from_numpy(x).to("cuda")
        out = torch.full((mesh ** 3,), float("nan"), dtype=torch.float32, device="cuda")
        rc = fn(xd.data_ptr(), n, mesh, box, mass, out.data_ptr(), stream.cuda_stream)
        assert rc == 0, cpm._native.last_error()
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, ref.cells)
        exact = orc.deposit_f64(mesh, box, x, mass)
        assert np.max(np.abs(got - exact) / np.maximum(np.abs(exact), 1e-30)) < 1e-6


def test_noalloc_deposit_rejects_meshes_above_its_limit(cpm):
    import torch

    fn = _fn(cpm)
    xd = torch.zeros((10, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros(65 ** 3, dtype=torch.float32, device="cuda")
    rc = fn(xd.data_ptr(), 10, 65, 1.0, 1.0, out.data_ptr(), None)
    assert rc == -3  # CPM_E_CAPACITY
    assert "64^3" in cpm._native.last_error()
