"""GPU parity: libcpm_cuda.so (through its C ABI) against the CPU oracle on the same inputs.

Bars (stated per test): bit-exact for octant keys, sort permutations, the CIC stencil gather and
kick/drift; deposited mass within 1e-6 relative of the FP64-summed oracle; FFT and PM forces
within 1e-5 relative RMS; tree and TreePM accelerations within 1e-5 relative RMS of the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


# ------------------------------------------------------------------ keys and sort (bit-exact)

@pytest.mark.parametrize("n,box,levels", [(5000, 1.0, 21), (20000, 64.0, 21), (3000, 10.0, 7)])
def test_octant_keys_and_permutation_bit_exact(cpm, orc, n, box, levels):
    x = orc.scattered_mesh(n, box)
    x[:7] = np.array([0.0, box, box / 2], np.float32)  # boundary values: 0, L, exact centres
    keys, perm = cpm.octant_keys(x, box, levels)
    ok = orc.octant_keys(x, box, levels)
    assert np.array_equal(keys, ok)
    assert np.array_equal(perm, orc.stable_sort_perm(ok))


def test_sort_is_stable_with_many_equal_keys(cpm, orc):
    rng = np.random.default_rng(3)
    x = (rng.integers(0, 4, size=(50000, 3)) * 0.25 + 0.125).astype(np.float32)  # 64 distinct cells
    keys, perm = cpm.octant_keys(x, 1.0, 21)
    assert np.array_equal(perm, orc.stable_sort_perm(orc.octant_keys(x, 1.0, 21)))


# ------------------------------------------------------------------ deposit / interpolate

def test_deposit_matches_fp64_oracle(cpm, orc):
    x = orc.scattered_mesh(5000, 1.0)
    m = cpm.Mesh(16, 1.0)
    m.deposit(x, 0.25)
    ref = orc.deposit_f64(16, 1.0, x, 0.25)
    assert np.max(np.abs(m.cells - ref) / np.maximum(np.abs(ref), 1e-30)) < 1e-6
    # mesh.rs:101-109 on the GPU result
    assert abs(m.cells.sum(dtype=np.float64) - 1250.0) < 1e-5 * 1250.0


def test_deposit_reference_cases(cpm, orc):
    """mesh.rs:111-162 on the GPU."""
    n, box = 8, 1.0
    h = np.float32(box) / np.float32(n)
    m = cpm.Mesh(n, box)
    m.deposit(np.array([[2.5 * h, 3.5 * h, 4.5 * h]], np.float32), 1.0)
    assert abs(m.cells[(2 * n + 3) * n + 4] - 1.0) < 1e-5 and int((m.cells > 1e-12).sum()) == 1
    n, box = 8, 2.0
    h = np.float32(box) / np.float32(n)
    g = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * h
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    m = cpm.Mesh(n, box)
    m.deposit(lat, 3.0)
    assert np.all(np.abs(m.cells - 3.0) < 1e-5)
    n, box = 4, 1.0
    h = np.float32(box) / np.float32(n)
    m = cpm.Mesh(n, box)
    m.deposit(np.array([[box, 0.5 * h, 0.5 * h]], np.float32), 1.0)
    assert abs(m.cells[((n - 1) * n) * n] - 0.5) < 1e-5 and abs(m.cells[0] - 0.5) < 1e-5


def test_deposit_is_order_independent_and_deterministic(cpm, orc):
    x = orc.scattered_mesh(40000, 1.0)
    a = cpm.Mesh(32, 1.0)
    a.deposit(x, 1.0)
    b = cpm.Mesh(32, 1.0)
    b.deposit(x[np.random.default_rng(0).permutation(len(x))], 1.0)
    assert np.array_equal(a.cells, b.cells)


def test_density_contrast_matches_oracle(cpm, orc):
    x = orc.scattered_mesh(20000, 2.0)
    d = cpm.density_contrast(x, 16, 2.0).cells
    ref = orc.deposit_f64(16, 2.0, x, 1.0)
    mean = np.float32(20000) / np.float32(16 ** 3)
    # delta = c/mean - 1 from the exactly rounded cell mass
    expect = (ref.astype(np.float32) / mean - np.float32(1.0)).astype(np.float32)
    assert np.max(np.abs(d - expect)) <= 4e-7 * np.max(np.abs(expect) + 1)


def test_interpolate_bit_exact(cpm, orc):
    rng = np.random.default_rng(1)
    cells = rng.standard_normal(16 ** 3).astype(np.float32)
    x = orc.scattered_mesh(3000, 1.0)
    x[:3] = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 1.0, 0.0]], np.float32)
    got = cpm.Mesh(16, 1.0, cells).interpolate_many(x)
    assert np.array_equal(got, orc.interpolate_many(16, 1.0, cells, x))


def test_far_positions_wrap_like_the_reference(cpm, orc):
    """Finite positions many boxes outside [0, L) (the reference accepts any finite position: floor
    cast to i64, then rem_euclid, mesh.rs:36-53) in the deposit and the gather, including +-inf-free
    values beyond 2^31 cells of opposite sign in one 1024-particle chunk."""
    x = orc.scattered_mesh(6000, 16.0)
    far = np.array([1e12, -3.7e9, 5.0e15, -2.5e11, 16.0, -16.5, 123456.789, -0.0, 2.2e9, -2.2e9], np.float32)
    x.reshape(-1)[:3 * len(far)] = np.resize(far, 3 * len(far))
    x[np.random.default_rng(5).integers(0, len(x), 64)] *= np.float32(-1e7)
    m = cpm.Mesh(16, 16.0)
    m.deposit(x, 1.0)
    ref = orc.deposit_f64(16, 16.0, x, 1.0)
    assert np.max(np.abs(m.cells - ref) / np.maximum(np.abs(ref), 1e-30)) < 1e-6
    cells = np.random.default_rng(2).standard_normal(16 ** 3).astype(np.float32)
    got = cpm.Mesh(16, 16.0, cells).interpolate_many(x)
    assert np.array_equal(got, orc.interpolate_many(16, 16.0, cells, x))


def test_interpolate_reference_cases(cpm):
    """mesh.rs:164-183 on the GPU."""
    from oracle import scattered_mesh
    m = cpm.Mesh(8, 1.0, np.full(8 ** 3, 2.5, np.float32))
    assert np.all(np.abs(m.interpolate_many(scattered_mesh(200, 1.0)) - 2.5) < 1e-5)
    h = np.float32(1.0) / np.float32(8)
    cells = np.zeros(8 ** 3, np.float32)
    cells[(5 * 8 + 1) * 8 + 6] = 7.0
    assert abs(cpm.Mesh(8, 1.0, cells).interpolate([5.5 * h, 1.5 * h, 6.5 * h]) - 7.0) < 1e-5


# ------------------------------------------------------------------ FFT / Poisson

@pytest.mark.parametrize("n", [4, 8, 16, 32, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft3_matches_oracle(cpm, orc, n, inverse):
    """Every compiled length up to the 512-point transform of the 512^3 headline mesh (1024-thread
    CTAs) against the oracle's FFT (fft.rs:40-72); numpy's FP64 FFT as a second reference to 256."""
    rng = np.random.default_rng(n)
    data = (rng.standard_normal(n ** 3) + 1j * rng.standard_normal(n ** 3)).astype(np.complex64)
    ref = orc.fft3(data.copy(), inverse)
    got = data.copy()
    f = cpm.Fft3(n)
    (f.inverse if inverse else f.forward)(got)
    assert rel_rms(got.view(np.float32), ref.view(np.float32)) < 1e-5
    del ref
    if n <= 256:
        exact = (np.fft.ifftn(data.reshape(n, n, n).astype(np.complex128)) * n ** 3 if inverse
                 else np.fft.fftn(data.reshape(n, n, n).astype(np.complex128))).ravel()
        assert rel_rms(got.view(np.float32), exact.astype(np.complex64).view(np.float32)) < 1e-5


def _dft_mode(field: np.ndarray, k: tuple) -> complex:
    """One output mode of the unnormalised forward 3D DFT, summed in FP64 axis by axis."""
    n = field.shape[0]
    e = [np.exp(-2j * np.pi * ki * np.arange(n) / n) for ki in k]
    total = 0j
    for x0 in range(0, n, 32):  # x slabs keep the FP64 temporaries at 0.5 GB
        s = field[x0:x0 + 32].astype(np.complex128) @ e[2]
        total += complex((s @ e[1]) @ e[0][x0:x0 + 32])
    return total


def test_fft3_random_field_at_1024(cpm):
    """A random complex field on the 1024^3 mesh (8 GB): forward then inverse returns n^3 times
    the input, the forward obeys Parseval, and five modes equal their FP64 DFT sums."""
    n = 1024
    rng = np.random.default_rng(1024)
    data = np.empty(n ** 3, np.complex64)
    step = n ** 3 // 16
    for i in range(16):
        blk = slice(i * step, (i + 1) * step)
        data.real[blk] = rng.standard_normal(step, dtype=np.float32)
        data.imag[blk] = rng.standard_normal(step, dtype=np.float32)
    f = cpm.Fft3(n)
    spec = data.copy()
    f.forward(spec)
    e_x = float(np.vdot(data, data).real)
    e_k = float(np.vdot(spec, spec).real)
    assert abs(e_k / (e_x * n ** 3) - 1.0) < 1e-5
    cube = data.reshape(n, n, n)
    for k in [(0, 0, 0), (1, 0, 0), (3, 511, 7), (512, 512, 512), (1000, 17, 600)]:
        want = _dft_mode(cube, k)
        got = complex(spec[(k[0] * n + k[1]) * n + k[2]])
        assert abs(got - want) < 1e-5 * np.sqrt(e_k / n ** 3) * 10 + 1e-5 * abs(want), k
    f.inverse(spec)
    spec /= np.float32(n ** 3)
    assert rel_rms(spec.view(np.float32), data.view(np.float32)) < 1e-5


def test_fft3_rejects_mesh_mismatch(cpm):
    f = cpm.Fft3(16)
    with pytest.raises(cpm.CpmError) as e:
        cpm.Context(8, 1.0)  # creating a context is fine
        data = np.zeros(12 ** 3, np.complex64)
        cpm.Fft3(12).forward(data)
    assert e.value.code == -4  # CPM_E_UNSUPPORTED
    del f


@pytest.mark.parametrize("n,box,a,r_split", [(16, 1.0, 0.5, 0.0), (32, 64.0, 0.3, 1.25), (64, 64.0, 1.0, 1.25),
                                             (48, 50.0, 0.7, 1.25), (96, 100.0, 1.0, 1.25),
                                             (192, 128.0, 0.6, 0.625), (256, 128.0, 1.0, 0.625),
                                             (320, 128.0, 0.8, 0.5), (512, 256.0, 1.0, 0.625)])
def test_poisson_matches_oracle(cpm, orc, n, box, a, r_split):
    x = orc.scattered_mesh(4 * n ** 3 // 8, box)
    delta = orc.density_contrast(n, box, x)
    cosmo = orc.lcdm_default()
    ref = orc.poisson_accel(n, box, delta, cosmo.omega_m, a, r_split)
    got = cpm.PoissonSolver(n, box).acceleration(cpm.Mesh(n, box, delta), cpm.Cosmology.lcdm_default(), a, r_split)
    for g, r in zip(got, ref):
        assert rel_rms(g.cells, r) < 1e-5


def test_plane_wave_force_matches_analytic(cpm):
    """poisson.rs:114-139 on the GPU."""
    n, box, a = 16, 1.0, 0.5
    cosmo = cpm.Cosmology.lcdm_default()
    k0 = np.float32(2.0 * np.float32(np.pi))
    c = np.float32(np.float32(1.5) * np.float32(cosmo.omega_m)) / np.float32(a)
    h = np.float32(box) / np.float32(n)
    xs = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * h
    field = lambda v: np.broadcast_to(v.astype(np.float32)[:, None, None], (n, n, n)).ravel().copy()
    delta = cpm.Mesh(n, box, field(np.cos(k0 * xs)))
    gx, gy, gz = cpm.PoissonSolver(n, box).acceleration(delta, cosmo, a, 0.0)
    amp = c / k0
    assert np.max(np.abs(gx.cells - field(-(c / k0) * np.sin(k0 * xs)))) < 1e-5 * amp
    assert np.max(np.abs(gy.cells)) < 1e-5 * amp and np.max(np.abs(gz.cells)) < 1e-5 * amp


def test_plane_wave_force_at_1024(cpm):
    """poisson.rs:114-139 at n = 1024, where the Green's function runs as its own k-space pass (the
    fused x pass needs more shared memory than one SM has): a wave along z of wavenumber 3."""
    n, box, a, m = 1024, 512.0, 1.0, 3
    cosmo = cpm.Cosmology.lcdm_default()
    k0 = np.float32(2.0 * np.pi * m / box)
    c = np.float32(np.float32(1.5) * np.float32(cosmo.omega_m)) / np.float32(a)
    zs = (np.arange(n, dtype=np.float64) + 0.5) * (box / n)
    delta = cpm.Mesh(n, box, np.broadcast_to(np.cos(k0 * zs).astype(np.float32), (n * n, n)).ravel().copy())
    gx, gy, gz = cpm.PoissonSolver(n, box).acceleration(delta, cosmo, a, 0.0)
    del delta
    amp = c / k0
    want = -(c / k0) * np.sin(k0 * zs)
    assert np.max(np.abs(gx.cells)) < 1e-5 * amp and np.max(np.abs(gy.cells)) < 1e-5 * amp
    assert np.max(np.abs(gz.cells.reshape(n * n, n) - want.astype(np.float32))) < 1e-5 * amp


def test_poisson_mesh_mismatch_raises(cpm):
    with pytest.raises(cpm.CpmError) as e:
        cpm.PoissonSolver(16, 1.0).acceleration(cpm.Mesh(8, 1.0), cpm.Cosmology.lcdm_default(), 1.0, 0.0)
    assert e.value.code == -2


# ------------------------------------------------------------------ tree

def test_tree_theta_zero_matches_brute_force(cpm, orc):
    """tree.rs:396-406 on the GPU."""
    split = cpm.ForceSplit(0.5, 2.0, 0.05, 0.0)
    x = orc.scattered_tree(400, 10.0, 7)
    fast = cpm.tree_accelerations(x, 10.0, split, 1.0)
    slow = orc.brute_force(x, 10.0, orc.Split(0.5, 2.0, 0.05, 0.0), 1.0)
    d = np.sqrt(((fast.astype(np.float64) - slow) ** 2).sum(1)).max()
    assert d / np.sqrt((slow.astype(np.float64) ** 2).sum(1)).max() < 1e-5


@pytest.mark.parametrize("n,seed,theta,r_cut", [(3000, 11, 0.5, 2.5), (20000, 5, 0.5, 1.0), (20000, 3, 0.5, 1.5)])
def test_tree_matches_oracle(cpm, orc, n, seed, theta, r_cut):
    """tree.rs:314-323 parity at the reference's theta = 0.5: within 1e-5 relative RMS."""
    x = orc.scattered_tree(n, 10.0, seed)
    got = cpm.tree_accelerations(x, 10.0, cpm.ForceSplit(0.5, r_cut, 0.05, theta), 1.0)
    ref = orc.tree_accelerations(x, 10.0, orc.Split(0.5, r_cut, 0.05, theta), 1.0)
    assert rel_rms(got, ref) < 1e-5


@pytest.mark.parametrize("n,seed,theta,r_cut", [(3000, 11, 0.5, 2.5), (20000, 9, 0.8, 1.5), (20000, 2, 1.0, 1.2)])
def test_tree_walk_matches_fp64_com_oracle(cpm, orc, n, seed, theta, r_cut):
    """The walk itself, any theta: against the oracle whose node centres of mass are FP64 sums
    rounded once (as on the GPU), within 1e-6 relative RMS. The reference sums them in f32; at
    large theta that rounding flips opening decisions (about 1.6e-4 RMS at theta = 0.8)."""
    x = orc.scattered_tree(n, 10.0, seed)
    got = cpm.tree_accelerations(x, 10.0, cpm.ForceSplit(0.5, r_cut, 0.05, theta), 1.0)
    ref = orc.tree_accelerations_com64(x, 10.0, orc.Split(0.5, r_cut, 0.05, theta), 1.0)
    assert rel_rms(got, ref) < 1e-6


def test_tree_clustered_matches_oracle(cpm, orc):
    rng = np.random.default_rng(4)
    centres = rng.uniform(0, 20, size=(12, 3))
    x = (centres[rng.integers(0, 12, 30000)] + rng.standard_normal((30000, 3)) * 0.3) % 20.0
    x = x.astype(np.float32)
    got = cpm.tree_accelerations(x, 20.0, cpm.ForceSplit(0.4, 1.8, 0.02, 0.5), 0.7)
    ref = orc.tree_accelerations(x, 20.0, orc.Split(0.4, 1.8, 0.02, 0.5), 0.7)
    assert rel_rms(got, ref) < 1e-5


def test_tree_interaction_counts_match_oracle(cpm, orc):
    x = orc.scattered_tree(20000, 10.0, 5)
    stats = {}
    cpm.tree_accelerations(x, 10.0, cpm.ForceSplit(0.5, 1.0, 0.05, 0.5), 1.0, stats=stats)
    lp, na, _ = orc.tree_walk_stats(x, 10.0, orc.Split(0.5, 1.0, 0.05, 0.5))
    assert abs(stats["leaf_pairs"] - lp) <= 1e-4 * lp
    assert abs(stats["node_accepts"] - na) <= 1e-3 * max(na, 1)
    assert stats["nodes"] == len(orc.tree_build(x, 10.0)["count"])


@pytest.mark.parametrize("n,box,r_cut", [(300_000, 40.0, 1.2), (200_000, 20.0, 0.9)])
def test_cutoff_decisions_exact_at_scale(cpm, orc, n, box, r_cut):
    """theta = 0 accepts no node, so the pair count depends only on the node centres (bit-exact)
    and the reference's f32 cutoff test r^2 > r_cut^2: the count must equal the oracle's exactly,
    over ~1e8 candidate pairs, many of them within an ulp of the cutoff."""
    x = orc.scattered_tree(n, box, 17)
    stats = {}
    cpm.tree_accelerations(x, box, cpm.ForceSplit(0.5, r_cut, 0.05, 0.0), 1.0, stats=stats)
    lp, na, _ = orc.tree_walk_stats(x, box, orc.Split(0.5, r_cut, 0.05, 0.0))
    assert na == 0 and stats["node_accepts"] == 0
    assert stats["leaf_pairs"] == lp


def test_periodic_pair_interacts_across_the_boundary(cpm):
    """tree.rs:420-430 on the GPU."""
    acc = cpm.tree_accelerations(np.array([[0.1, 5.0, 5.0], [9.9, 5.0, 5.0]], np.float32), 10.0,
                                 cpm.ForceSplit(0.5, 2.0, 0.05, 0.5), 1.0)
    assert acc[0, 0] < 0.0 and acc[1, 0] > 0.0


def test_nonfinite_position_is_reported(cpm):
    x = np.zeros((100, 3), np.float32)
    x[17, 1] = np.nan
    with pytest.raises(cpm.CpmError) as e:
        cpm.tree_accelerations(x, 1.0, cpm.ForceSplit(0.1, 0.3, 0.01, 0.5), 1.0)
    assert e.value.code == -6


def test_tree_coincident_particles_match_oracle(cpm, orc):
    """More than LEAF_SIZE particles at one exact position share all 21 key digits, so their node
    at the key depth stays a leaf; the reference keeps splitting that one-child chain (to depth 40)
    and sums the particles directly at its first node without an octant-0 child. The
    accelerations agree all the same, and coincident pairs (r = 0) add nothing."""
    x = orc.scattered_tree(5000, 10.0, 8)
    x[:20] = x[0]
    x[20:32] = x[100]
    split = (0.5, 1.5, 0.05, 0.5)
    got = cpm.tree_accelerations(x, 10.0, cpm.ForceSplit(*split), 1.0)
    ref = orc.tree_accelerations(x, 10.0, orc.Split(*split), 1.0)
    assert np.all(np.isfinite(got))
    assert rel_rms(got, ref) < 1e-5
