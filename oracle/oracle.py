"""ctypes front end of the CPU oracle (liboracle.so) — test infrastructure only.

The oracle restates the reference crate's TreePM path on the CPU (see cpm_oracle.h for the
file:line map). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class Cosmology(C.Structure):
    """cosmology.rs:9-16"""
    _fields_ = [("omega_r", C.c_float), ("omega_m", C.c_float), ("omega_l", C.c_float), ("h0", C.c_float)]


class Split(C.Structure):
    """tree.rs:21-30"""
    _fields_ = [("r_split", C.c_float), ("r_cut", C.c_float), ("softening", C.c_float), ("theta", C.c_float)]


class PSpec(C.Structure):
    """ics.rs:21-24"""
    _fields_ = [("amplitude", C.c_float), ("n_s", C.c_float)]


def build() -> Path:
    """Compile liboracle.so with the Makefile beside this file (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "cpm_oracle.cpp").stat().st_mtime:
        build()
    L = C.CDLL(str(LIB_PATH))
    sz, fl, i = C.c_size_t, C.c_float, C.c_int
    sig = {
        "orc_scattered_mesh": (None, [sz, fl, f32p]),
        "orc_scattered_tree": (None, [sz, fl, C.c_uint64, f32p]),
        "orc_stencil": (None, [i, fl, f32p, i64p, f32p]),
        "orc_deposit": (None, [i, fl, f32p, sz, fl, f32p]),
        "orc_deposit_f64": (None, [i, fl, f32p, sz, fl, f64p]),
        "orc_interpolate": (fl, [i, fl, f32p, f32p]),
        "orc_interpolate_many": (None, [i, fl, f32p, f32p, sz, f32p]),
        "orc_density_contrast": (None, [i, fl, f32p, sz, f32p]),
        "orc_fft3": (None, [i, f32p, i]),
        "orc_fft3_f64": (None, [i, f64p, i]),
        "orc_wavenumber": (fl, [sz, sz, fl]),
        "orc_poisson_accel": (None, [i, fl, f32p, fl, fl, fl, f32p, f32p, f32p]),
        "orc_poisson_accel_deconvolved": (None, [i, fl, f32p, fl, fl, fl, f32p, f32p, f32p]),
        "orc_split_with": (Split, [fl, sz, sz, fl, fl]),
        "orc_short_range_factor": (fl, [fl, fl]),
        "orc_tree_accelerations": (None, [f32p, sz, fl, C.POINTER(Split), fl, f32p]),
        "orc_tree_accelerations_builtin": (None, [f32p, sz, fl, C.POINTER(Split), fl, f32p]),
        "orc_tree_accelerations_com64": (None, [f32p, sz, fl, C.POINTER(Split), fl, f32p]),
        "orc_brute_force": (None, [f32p, sz, fl, C.POINTER(Split), fl, f32p]),
        "orc_tree_build": (sz, [f32p, sz, fl] + [C.c_void_p] * 9),
        "orc_tree_walk_stats": (None, [f32p, sz, fl, C.POINTER(Split), C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "orc_octant_keys": (None, [f32p, sz, fl, i, u64p]),
        "orc_stable_sort_perm": (None, [u64p, sz, u32p]),
        "orc_cosmo_e": (fl, [C.POINTER(Cosmology), fl]),
        "orc_growth": (fl, [C.POINTER(Cosmology), fl]),
        "orc_growth_rate": (fl, [C.POINTER(Cosmology), fl]),
        "orc_bbks": (fl, [C.POINTER(Cosmology), fl]),
        "orc_lcdm_default": (Cosmology, []),
        "orc_kick_factor": (fl, [C.POINTER(Cosmology), fl, fl]),
        "orc_drift_factor": (fl, [C.POINTER(Cosmology), fl, fl]),
        "orc_midpoint": (fl, [C.POINTER(Cosmology), fl, fl]),
        "orc_kick": (None, [f32p, f32p, sz, fl]),
        "orc_drift": (None, [f32p, f32p, sz, fl, fl]),
        "orc_sim_new": (C.c_void_p, [C.POINTER(Cosmology), fl, i, f32p, f32p, sz, fl, C.c_void_p]),
        "orc_sim_step_to": (None, [C.c_void_p, fl]),
        "orc_sim_get": (None, [C.c_void_p] + [C.c_void_p] * 5),
        "orc_sim_accelerations": (None, [C.c_void_p, fl, f32p, C.c_void_p]),
        "orc_sim_free": (None, [C.c_void_p]),
        "orc_sim_last_timings": (None, [C.c_void_p, f64p]),
        "orc_power": (fl, [C.POINTER(Cosmology), C.POINTER(PSpec), fl]),
        "orc_sigma": (fl, [C.POINTER(Cosmology), C.POINTER(PSpec), fl]),
        "orc_power_normalized": (PSpec, [C.POINTER(Cosmology), fl, fl, fl]),
        "orc_white_noise": (None, [i, C.c_uint64, f32p]),
        "orc_colored_modes": (None, [i, fl, C.POINTER(Cosmology), C.POINTER(PSpec), C.c_uint64, f32p]),
        "orc_zeldovich": (None, [i, fl, C.POINTER(Cosmology), C.POINTER(PSpec), fl, C.c_uint64, f32p, f32p]),
        "orc_power_spectrum": (None, [f32p, sz, fl, i, i, f64p, f64p, u64p]),
        "orc_num_threads": (i, []),
        "orc64_accelerations": (None, [f32p, sz, C.c_double, i, C.c_double, C.c_double, C.c_void_p, C.c_double,
                                       u32p, sz, f64p]),
        "orc64_accelerations_ex": (None, [f32p, sz, C.c_double, i, C.c_double, C.c_double, C.c_void_p, C.c_double,
                                          u32p, sz, f64p, i]),
        "orc_step_sample": (None, [C.POINTER(Cosmology), fl, i, f32p, f32p, f32p, sz, fl, fl, C.c_void_p, u32p, sz,
                                   i, f64p, C.c_void_p, C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ fixtures of the reference tests

def scattered_mesh(count: int, box: float) -> np.ndarray:
    """mesh.rs:90-99 (xorshift seed 0x9E3779B97F4A7C15, 53-bit mantissa)."""
    out = np.empty((count, 3), np.float32)
    lib().orc_scattered_mesh(count, box, out)
    return out


def scattered_tree(count: int, box: float, seed: int) -> np.ndarray:
    """tree.rs:340-349 (xorshift, 24-bit mantissa)."""
    out = np.empty((count, 3), np.float32)
    lib().orc_scattered_tree(count, box, seed, out)
    return out


# ------------------------------------------------------------------ mesh.rs

def stencil(n: int, box: float, x) -> tuple[np.ndarray, np.ndarray]:
    idx = np.empty(8, np.int64)
    w = np.empty(8, np.float32)
    lib().orc_stencil(n, box, _f32(x), idx, w)
    return idx, w


def deposit(n: int, box: float, x, mass: float) -> np.ndarray:
    x = _f32(x)
    cells = np.empty(n ** 3, np.float32)
    lib().orc_deposit(n, box, x, len(x), mass, cells)
    return cells


def deposit_f64(n: int, box: float, x, mass: float) -> np.ndarray:
    x = _f32(x)
    cells = np.empty(n ** 3, np.float64)
    lib().orc_deposit_f64(n, box, x, len(x), mass, cells)
    return cells


def interpolate(n: int, box: float, cells, x) -> float:
    return lib().orc_interpolate(n, box, _f32(cells), _f32(x))


def interpolate_many(n: int, box: float, cells, x) -> np.ndarray:
    x = _f32(x)
    out = np.empty(len(x), np.float32)
    lib().orc_interpolate_many(n, box, _f32(cells), x, len(x), out)
    return out


def density_contrast(n: int, box: float, x) -> np.ndarray:
    x = _f32(x)
    out = np.empty(n ** 3, np.float32)
    lib().orc_density_contrast(n, box, x, len(x), out)
    return out


# ------------------------------------------------------------------ fft.rs / poisson.rs

def fft3(data: np.ndarray, inverse: bool = False) -> np.ndarray:
    """Unnormalised c2c transform of an n^3 complex64 array (fft.rs:28-72)."""
    n = round(data.size ** (1 / 3))
    buf = np.ascontiguousarray(data, dtype=np.complex64).view(np.float32).ravel().copy()
    lib().orc_fft3(n, buf, int(inverse))
    return buf.view(np.complex64).reshape(data.shape)


def wavenumber(i: int, n: int, box: float) -> float:
    return lib().orc_wavenumber(i, n, box)


def poisson_accel(n: int, box: float, delta, omega_m: float, a: float, r_split: float, deconvolve: bool = False):
    """poisson.rs:33-88; `deconvolve` divides the Green's function by the CIC window squared (no
    counterpart in the reference: the library's CPM_SIM_DECONVOLVE)."""
    d = _f32(delta).ravel()
    g = [np.empty(n ** 3, np.float32) for _ in range(3)]
    fn = lib().orc_poisson_accel_deconvolved if deconvolve else lib().orc_poisson_accel
    fn(n, box, d, omega_m, a, r_split, g[0], g[1], g[2])
    return g


# ------------------------------------------------------------------ tree.rs

def split_with(box: float, mesh_n: int, pps: int, soft_scale: float, theta: float) -> Split:
    return lib().orc_split_with(box, mesh_n, pps, soft_scale, theta)


def short_range_factor(r: float, r_split: float) -> float:
    return lib().orc_short_range_factor(r, r_split)


def tree_accelerations(x, box: float, split: Split, k: float) -> np.ndarray:
    x = _f32(x)
    out = np.empty((len(x), 3), np.float32)
    lib().orc_tree_accelerations(x, len(x), box, C.byref(split), k, out)
    return out


def tree_accelerations_com64(x, box: float, split: Split, k: float) -> np.ndarray:
    """Diagnostic twin of tree_accelerations with FP64 centre-of-mass sums."""
    x = _f32(x)
    out = np.empty((len(x), 3), np.float32)
    lib().orc_tree_accelerations_com64(x, len(x), box, C.byref(split), k, out)
    return out


def tree_accelerations_builtin(x, box: float, split: Split, k: float) -> np.ndarray:
    x = _f32(x)
    out = np.empty((len(x), 3), np.float32)
    lib().orc_tree_accelerations_builtin(x, len(x), box, C.byref(split), k, out)
    return out


def brute_force(x, box: float, split: Split, k: float) -> np.ndarray:
    x = _f32(x)
    out = np.empty((len(x), 3), np.float32)
    lib().orc_brute_force(x, len(x), box, C.byref(split), k, out)
    return out


def tree_build(x, box: float) -> dict:
    """Nodes of Tree::build (tree.rs:171-250) in build order, plus the final particle order."""
    x = _f32(x)
    nn = lib().orc_tree_build(x, len(x), box, *([None] * 9))
    out = dict(center=np.empty((nn, 3), np.float32), half=np.empty(nn, np.float32),
               com=np.empty((nn, 3), np.float32), count=np.empty(nn, np.uint32),
               start=np.empty(nn, np.uint32), end=np.empty(nn, np.uint32),
               children=np.empty((nn, 8), np.uint32), depth=np.empty(nn, np.uint32),
               order=np.empty(len(x), np.uint32))
    keys = ["center", "half", "com", "count", "start", "end", "children", "depth", "order"]
    lib().orc_tree_build(x, len(x), box, *[_ptr(out[k]) for k in keys])
    return out


def tree_walk_stats(x, box: float, split: Split) -> tuple[int, int, int]:
    x = _f32(x)
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    lib().orc_tree_walk_stats(x, len(x), box, C.byref(split), C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def octant_keys(x, box: float, levels: int = 21) -> np.ndarray:
    x = _f32(x)
    out = np.empty(len(x), np.uint64)
    lib().orc_octant_keys(x, len(x), box, levels, out)
    return out


def stable_sort_perm(keys) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.empty(len(keys), np.uint32)
    lib().orc_stable_sort_perm(keys, len(keys), out)
    return out


# ------------------------------------------------------------------ cosmology.rs / integrator.rs

def lcdm_default() -> Cosmology:
    return lib().orc_lcdm_default()


def cosmology(omega_r: float, omega_m: float, omega_l: float, h0: float) -> Cosmology:
    return Cosmology(omega_r, omega_m, omega_l, h0)


def cosmo_e(c: Cosmology, a: float) -> float:
    return lib().orc_cosmo_e(C.byref(c), a)


def growth(c: Cosmology, a: float) -> float:
    return lib().orc_growth(C.byref(c), a)


def growth_rate(c: Cosmology, a: float) -> float:
    return lib().orc_growth_rate(C.byref(c), a)


def bbks(c: Cosmology, k: float) -> float:
    return lib().orc_bbks(C.byref(c), k)


def kick_factor(c: Cosmology, a0: float, a1: float) -> float:
    return lib().orc_kick_factor(C.byref(c), a0, a1)


def drift_factor(c: Cosmology, a0: float, a1: float) -> float:
    return lib().orc_drift_factor(C.byref(c), a0, a1)


def midpoint(c: Cosmology, a0: float, a1: float) -> float:
    return lib().orc_midpoint(C.byref(c), a0, a1)


class Simulation:
    """integrator.rs:34-186 Simulation (f32, reference-faithful)."""

    def __init__(self, cosmo: Cosmology, box: float, mesh_n: int, x, p, a: float, split: Split | None):
        self.x_in = _f32(x)
        self.p_in = _f32(p)
        self.n = len(self.x_in)
        self.mesh_n = mesh_n
        self.cosmo = cosmo
        self._split = split
        self.h = lib().orc_sim_new(C.byref(cosmo), box, mesh_n, self.x_in, self.p_in, self.n, a,
                                   C.cast(C.pointer(split), C.c_void_p) if split is not None else None)

    def step_to(self, a1: float) -> None:
        lib().orc_sim_step_to(self.h, a1)

    def state(self, want_delta: bool = False) -> dict:
        x = np.empty((self.n, 3), np.float32)
        p = np.empty((self.n, 3), np.float32)
        acc = np.empty((self.n, 3), np.float32)
        delta = np.empty(self.mesh_n ** 3, np.float32) if want_delta else None
        a = C.c_float()
        lib().orc_sim_get(self.h, _ptr(x), _ptr(p), _ptr(acc), _ptr(delta), C.cast(C.byref(a), C.c_void_p))
        return dict(x=x, p=p, acc=acc, delta=delta, a=a.value)

    def accelerations(self, a: float) -> np.ndarray:
        acc = np.empty((self.n, 3), np.float32)
        lib().orc_sim_accelerations(self.h, a, acc, None)
        return acc

    def last_timings(self) -> np.ndarray:
        t = np.empty(6, np.float64)
        lib().orc_sim_last_timings(self.h, t)
        return t

    def close(self) -> None:
        if self.h:
            lib().orc_sim_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ln_a_schedule(a_start: float, a_end: float, steps: int) -> list[float]:
    """runner.rs:240 / integrator.rs:168: a1 = a0 (a_end/a0)^(i/steps), evaluated in f32."""
    a0 = np.float32(a_start)
    ratio = np.float32(np.float32(a_end) / a0)
    out = []
    for i in range(1, steps + 1):
        e = np.float32(np.float32(i) / np.float32(steps))
        out.append(float(np.float32(a0 * np.float32(np.power(ratio, e, dtype=np.float32)))))
    return out


# ------------------------------------------------------------------ ics.rs

def power_normalized(c: Cosmology, n_s: float, sigma8: float, radius: float) -> PSpec:
    return lib().orc_power_normalized(C.byref(c), n_s, sigma8, radius)


def power(c: Cosmology, ps: PSpec, k: float) -> float:
    return lib().orc_power(C.byref(c), C.byref(ps), k)


def sigma(c: Cosmology, ps: PSpec, radius: float) -> float:
    return lib().orc_sigma(C.byref(c), C.byref(ps), radius)


def white_noise(n: int, seed: int) -> np.ndarray:
    out = np.empty(n ** 3, np.float32)
    lib().orc_white_noise(n, seed, out)
    return out


def colored_modes(n: int, box: float, c: Cosmology, ps: PSpec, seed: int) -> np.ndarray:
    out = np.empty(2 * n ** 3, np.float32)
    lib().orc_colored_modes(n, box, C.byref(c), C.byref(ps), seed, out)
    return out.view(np.complex64)


def zeldovich(n: int, box: float, c: Cosmology, ps: PSpec, a_init: float, seed: int):
    x = np.empty((n ** 3, 3), np.float32)
    p = np.empty((n ** 3, 3), np.float32)
    lib().orc_zeldovich(n, box, C.byref(c), C.byref(ps), a_init, seed, x, p)
    return x, p


def power_spectrum(x, box: float, n: int, n_shells: int):
    x = _f32(x)
    k = np.empty(n_shells, np.float64)
    p = np.empty(n_shells, np.float64)
    c = np.empty(n_shells, np.uint64)
    lib().orc_power_spectrum(x, len(x), box, n, n_shells, k, p, c)
    return k, p, c


def tree_coupling64(omega_m: float, box: float, a: float, n: int) -> float:
    """integrator.rs:150-152 in double: K = (3/2) Omega_m L^3 / (4 pi a N)."""
    return 1.5 * omega_m * box ** 3 / (4.0 * np.pi * a * n)


def accelerations_f64(x, box: float, mesh_n: int, omega_m: float, a: float, split: Split | None,
                      sample, quadrupole: bool = False) -> np.ndarray:
    """FP64 build: PM + short-range tree force (coupling tree_coupling64) at the sampled particles,
    everything in double precision; `quadrupole` adds the quadrupole terms of accepted nodes (the
    library's CPM_SIM_QUADRUPOLE). Returns (len(sample), 3) float64."""
    x = _f32(x)
    sample = np.ascontiguousarray(sample, np.uint32)
    out = np.empty((len(sample), 3), np.float64)
    k = tree_coupling64(omega_m, box, a, len(x))
    sp = C.cast(C.pointer(split), C.c_void_p) if split is not None else None
    lib().orc64_accelerations_ex(x, len(x), float(box), int(mesh_n), float(omega_m), float(a), sp, k, sample,
                                 len(sample), out, 1 if quadrupole else 0)
    return out


def num_threads() -> int:
    return lib().orc_num_threads()


def step_sample(c: Cosmology, box: float, mesh_n: int, x, p, acc, a0: float, a1: float, split: Split | None,
                subset, threads: int = 0, want_acc: bool = False, want_com64: bool = False):
    """Seconds of each phase of one reference KDK step on (x, p, acc); the walk runs for `subset` only.
    Returns [kick+drift, deposit, poisson, gather, tree build, walk(subset), second kick], and with
    `want_acc` also the force at a1 (PM + tree) of the subset particles, shape (len(subset), 3);
    with `want_com64` as well the same force with FP64 centre-of-mass sums (untimed)."""
    x, p, acc = _f32(x), _f32(p), _f32(acc)
    sub = np.ascontiguousarray(subset, dtype=np.uint32)
    t = np.zeros(7, np.float64)
    out = np.empty((len(sub), 3), np.float32) if want_acc else None
    out64 = np.empty((len(sub), 3), np.float32) if want_com64 else None
    lib().orc_step_sample(C.byref(c), box, mesh_n, x, p, acc, len(x), a0, a1,
                          C.cast(C.pointer(split), C.c_void_p) if split is not None else None, sub, len(sub),
                          threads, t, out.ctypes.data if want_acc else None,
                          out64.ctypes.data if want_com64 else None)
    if want_com64:
        return t, out, out64
    return (t, out) if want_acc else t


os.environ.setdefault("OMP_PROC_BIND", "false")
