"""The allocation-free CIC deposit (cpm_mesh_deposit_noalloc), called through the C ABI.

It exists for programs that cannot let a library call cudaMalloc (their device memory belongs to
their own allocator or pool, or an allocation's implicit synchronisation would stall their other
streams): positions and the output mesh are the caller's device buffers and the only scratch is a
static device array. Its output must equal the allocating entry point's (cpm_mesh_deposit) — both
sum the same 64-bit fixed-point weights, so the test asks for equality, inside the 1e-6 relative
bar of the deposit tests — on consecutive calls that share the static array. The cases cover
unsorted input (the kernel's global-atomic branch), spatially sorted and clustered input (its
shared-memory tile branch), positions far outside the box, and a non-finite position, which
this entry point reports by filling the output with NaN. The file name sorts last so a run that
stops at the first failure has run every other test first.
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


def _morton_sorted(x: np.ndarray, mesh: int, box: float) -> np.ndarray:
    """Positions ordered by the Morton code of their cell, so consecutive chunks cover compact boxes."""
    cell = np.clip((x / np.float32(box / mesh)).astype(np.int64), 0, mesh - 1)
    code = np.zeros(len(x), np.int64)
    for bit in range(int(mesh).bit_length()):
        for k in range(3):
            code |= ((cell[:, k] >> bit) & 1) << (3 * bit + k)
    return np.ascontiguousarray(x[np.argsort(code, kind="stable")])


def _clustered(n: int, box: float, mesh: int, seed: int) -> np.ndarray:
    """n positions inside a 10-cell cube: every 1024-particle chunk's stencil box fits in shared memory."""
    rng = np.random.default_rng(seed)
    h = box / mesh
    x = (np.float32(5 * h) + rng.random((n, 3), dtype=np.float32) * np.float32(10 * h)).astype(np.float32)
    return _morton_sorted(x, mesh, box)


def _run(cpm, fn, x, mesh, box, mass, stream):
    import torch

    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to("cuda")
    out = torch.full((mesh ** 3,), float("nan"), dtype=torch.float32, device="cuda")
    rc = fn(xd.data_ptr(), len(x), mesh, box, mass, out.data_ptr(), stream.cuda_stream)
    assert rc == 0, cpm._native.last_error()
    stream.synchronize()
    return out.cpu().numpy()


def test_noalloc_deposit_matches_allocating_deposit(cpm, orc):
    import torch

    fn = _fn(cpm)
    stream = torch.cuda.current_stream()
    scattered = orc.scattered_mesh(50000, 64.0)
    cases = [
        ("unsorted", orc.scattered_mesh(20000, 1.0), 32, 1.0, 0.5),
        ("unsorted", scattered, 64, 64.0, 1.0),
        ("clustered, sorted", _clustered(20000, 64.0, 64, 3), 64, 64.0, 1.0),
        ("sorted", _morton_sorted(scattered, 64, 64.0), 64, 64.0, 0.25),
        ("unsorted again", orc.scattered_mesh(20000, 1.0), 32, 1.0, 0.5),
        ("clustered again", _clustered(30000, 32.0, 32, 4), 32, 32.0, 2.0),
    ]
    for name, x, mesh, box, mass in cases:
        ref = cpm.Mesh(mesh, box)
        ref.deposit(x, mass)
        got = _run(cpm, fn, x, mesh, box, mass, stream)
        assert np.array_equal(got, ref.cells), name
        exact = orc.deposit_f64(mesh, box, x, mass)
        assert np.max(np.abs(got - exact) / np.maximum(np.abs(exact), 1e-30)) < 1e-6, name


def test_noalloc_deposit_far_positions_wrap_like_the_reference(cpm, orc):
    """Finite positions many boxes away wrap by rem_euclid of the i64 cell index (mesh.rs:36-53)."""
    import torch

    fn = _fn(cpm)
    rng = np.random.default_rng(11)
    x = orc.scattered_mesh(4000, 16.0)
    far = np.array([1e12, -3.7e9, 5.0e15, -2.5e11, 16.0, -16.5, 123456.789, -0.0], np.float32)
    x.reshape(-1)[:3 * len(far)] = np.resize(far, 3 * len(far))
    x[rng.integers(0, len(x), 64)] *= np.float32(-1e7)
    got = _run(cpm, fn, x, 16, 16.0, 1.0, torch.cuda.current_stream())
    exact = orc.deposit_f64(16, 16.0, x, 1.0)
    assert np.max(np.abs(got - exact) / np.maximum(np.abs(exact), 1e-30)) < 1e-6


def test_noalloc_deposit_marks_non_finite_positions(cpm, orc):
    import torch

    fn = _fn(cpm)
    stream = torch.cuda.current_stream()
    x = orc.scattered_mesh(5000, 1.0)
    x[1234, 1] = np.nan
    got = _run(cpm, fn, x, 16, 1.0, 1.0, stream)
    assert np.isnan(got).all()
    x[1234, 1] = np.inf
    assert np.isnan(_run(cpm, fn, x, 16, 1.0, 1.0, stream)).all()
    # the status word is cleared by the next call
    x[1234, 1] = 0.5
    got = _run(cpm, fn, x, 16, 1.0, 1.0, stream)
    ref = cpm.Mesh(16, 1.0)
    ref.deposit(x, 1.0)
    assert np.array_equal(got, ref.cells)


def test_noalloc_deposit_rejects_meshes_above_its_limit(cpm):
    import torch

    fn = _fn(cpm)
    xd = torch.zeros((10, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros(65 ** 3, dtype=torch.float32, device="cuda")
    rc = fn(xd.data_ptr(), 10, 65, 1.0, 1.0, out.data_ptr(), None)
    assert rc == -3  # CPM_E_CAPACITY
    assert "64^3" in cpm._native.last_error()
