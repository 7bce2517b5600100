"""CPU-only checks of the C ABI: the library builds, loads, exports every symbol include/cpm.h
declares, and its host-only functions agree bit for bit with the oracle. No GPU compute here."""
import ctypes as C
import subprocess

import numpy as np
import pytest


@pytest.fixture(scope="module")
def native(cpm):
    from importlib import import_module
    nat = import_module("cosmological-particle-simulation_b200._native")
    if not nat.LIB_PATH.exists():
        import_module("cosmological-particle-simulation_b200.build").build()
    return nat


def test_library_exports_every_declared_symbol(native):
    names = native.exported_symbols()
    assert len(names) >= 20
    raw = C.CDLL(str(native.LIB_PATH))
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(native.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported


def test_library_targets_sm100a(native):
    out = subprocess.run(["cuobjdump", "--list-elf", str(native.LIB_PATH)], capture_output=True, text=True)
    assert out.returncode == 0 and "sm_100a" in out.stdout


def test_version_string(native):
    assert native.lib().cpm_version().decode().startswith("cpm ")


def test_fft_size_set(native):
    """Sizes with compiled transforms: powers of two 4..1024 and the listed 2^a 3^b 5^c sizes."""
    L = native.lib()
    supported = {n for n in range(1, 2049) if L.cpm_fft_supported(n)}
    assert supported == {4, 8, 16, 32, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512, 1024}


def test_host_wavenumber_bit_exact(native, orc):
    for n in (4, 7, 16, 64, 512):
        for i in range(n):
            assert native.lib().cpm_wavenumber(i, n, 64.0) == orc.wavenumber(i, n, 64.0)


def test_host_force_split_bit_exact(native, orc):
    for args in [(64.0, 64, 32, 1 / 30, 0.5), (256.0, 512, 256, 1 / 30, 0.5), (100.0, 80, 40, 0.05, 0.5)]:
        a = native.lib().cpm_force_split_with(*args)
        b = orc.split_with(*args)
        assert (a.r_split, a.r_cut, a.softening, a.theta) == (b.r_split, b.r_cut, b.softening, b.theta)


def test_host_short_range_factor_bit_exact(native, orc):
    for r in np.linspace(0.0, 6.0, 301, dtype=np.float32):
        assert native.lib().cpm_short_range_factor(float(r), 0.7) == orc.short_range_factor(float(r), 0.7)


def test_invalid_arguments_fail_without_a_device(native):
    h = C.c_void_p()
    rc = native.lib().cpm_ctx_create(0, 1.0, 0, 0, C.byref(h))
    assert rc == -1 and h.value is None
    assert "n_mesh" in native.last_error()
    assert native.lib().cpm_ctx_create(8, 1.0, 0, 0, None) == -1
    assert native.lib().cpm_mesh_deposit(None, None, 0, 1.0, None) == -1


def _compile_mirror(native, out_dir):
    root = native.HERE.parent
    exe = out_dir / "mirror_check"
    cmd = ["g++", "-std=c++17", "-O1", "-I", str(root / "include"), str(root / "tests" / "cpp" / "mirror_check.cpp"),
           "-o", str(exe), "-L", str(native.HERE), "-lcpm_cuda", f"-Wl,-rpath,{native.HERE}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_mirror_compiles_and_links(native, tmp_path):
    """include/cpm.hpp (the C++ mirror of the reference interface) builds against the library."""
    assert _compile_mirror(native, tmp_path).exists()


@pytest.mark.parametrize("r_split,r_cut", [(0.625, 2.8125), (0.5, 2.0), (0.5, 2.5), (0.4, 1.8), (1.0, 9.0)])
def test_walk_pair_kernel_fit_is_accurate(native, r_split, r_cut):
    """The walk's fitted S(r) (tree.rs:54-57) stays within 5e-7 relative of double precision."""
    err = C.c_double()
    assert native.lib().cpm_walk_kernel_fit_error(r_split, r_cut, 20001, C.byref(err)) == 0
    assert err.value < 5e-7, err.value


def test_reference_step_factors_on_the_host(cpm, orc):
    """cpm_step_factors(fp64 = 0) is host code: the reference's f32 kick/drift/midpoint
    (integrator.rs:263-297), equal to the oracle's restatement bit for bit."""
    import ctypes as C

    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    for a0, a1 in [(0.02, 0.0206), (0.5, 0.52), (0.97, 1.0)]:
        k1, d, k2 = C.c_double(), C.c_double(), C.c_double()
        assert cpm.lib().cpm_step_factors(C.byref(cc), a0, a1, 0, C.byref(k1), C.byref(d), C.byref(k2)) == 0
        am = orc.midpoint(c, a0, a1)
        assert (k1.value, d.value, k2.value) == (orc.kick_factor(c, a0, am), orc.drift_factor(c, a0, a1),
                                                 orc.kick_factor(c, am, a1))
