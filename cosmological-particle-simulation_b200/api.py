"""Host-side mirror of the reference crate's TreePM interface, backed by libcpm_cuda.so.

Names, argument meaning and error behaviour follow the Rust items they stand in for
(mesh.rs, fft.rs, poisson.rs, tree.rs, integrator.rs, cosmology.rs); where the reference
panics (a mesh-size mismatch, poisson.rs:35) these raise CpmError. Positions and momenta are
(N, 3) float32 arrays, the memory of a Rust `Vec<[f32; 3]>`; meshes are n^3 float32 cells
indexed (ix*n + iy)*n + iz.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import CpmError, Cosmology, check, f32c, ptr

__all__ = ["Context", "Mesh", "Fft3", "wavenumber", "PoissonSolver", "ForceSplit", "short_range_factor",
           "tree_accelerations", "octant_keys", "Simulation", "Cosmology", "CpmError", "ln_a_schedule"]


class Context:
    """A cpm_ctx: one CUDA stream and device buffers for meshes of n^3 cells in a box of side L."""

    def __init__(self, n: int, box_size: float, max_particles: int = 0):
        h = C.c_void_p()
        check(nat.lib().cpm_ctx_create(int(n), float(box_size), int(max_particles), 0, C.byref(h)))
        self.h = h
        self.n = int(n)
        self.box_size = float(box_size)

    def close(self):
        if getattr(self, "h", None):
            nat.lib().cpm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self.h)


_contexts: dict[tuple[int, float], Context] = {}


def _ctx(n: int, box: float) -> Context:
    key = (int(n), float(np.float32(box)))
    c = _contexts.get(key)
    if c is None:
        c = _contexts[key] = Context(n, box)
    return c


class Mesh:
    """mesh.rs:6-78 `Mesh { n, box_size, cells }`."""

    def __init__(self, n: int, box_size: float, cells: np.ndarray | None = None):
        self.n = int(n)
        self.box_size = float(np.float32(box_size))
        self.cells = np.zeros(self.n ** 3, np.float32) if cells is None else f32c(cells).reshape(-1)
        if self.cells.size != self.n ** 3:
            raise CpmError(-1, "cells must hold n^3 values")

    @staticmethod
    def new(n: int, box_size: float) -> "Mesh":
        return Mesh(n, box_size)

    def deposit(self, positions, mass: float) -> None:
        """mesh.rs:62-69: clears the grid, then deposits `mass` per particle with CIC weights."""
        x = f32c(positions).reshape(-1, 3)
        c = _ctx(self.n, self.box_size)
        c._check(nat.lib().cpm_mesh_deposit(c.h, ptr(x), len(x), float(mass), ptr(self.cells)))

    def interpolate(self, x) -> float:
        """mesh.rs:72-77 for one position."""
        return float(self.interpolate_many(np.asarray(x, np.float32).reshape(1, 3))[0])

    def interpolate_many(self, positions) -> np.ndarray:
        x = f32c(positions).reshape(-1, 3)
        out = np.empty(len(x), np.float32)
        c = _ctx(self.n, self.box_size)
        c._check(nat.lib().cpm_mesh_interpolate(c.h, ptr(self.cells), ptr(x), len(x), ptr(out)))
        return out


def density_contrast(positions, mesh_n: int, box_size: float) -> Mesh:
    """integrator.rs:117-126 `Simulation::density_contrast`."""
    x = f32c(positions).reshape(-1, 3)
    m = Mesh(mesh_n, box_size)
    c = _ctx(mesh_n, box_size)
    c._check(nat.lib().cpm_density_contrast(c.h, ptr(x), len(x), ptr(m.cells)))
    return m


def interpolate3(gx: Mesh, gy: Mesh, gz: Mesh, positions) -> np.ndarray:
    """integrator.rs:144-148: the PM force at each position, (N, 3)."""
    x = f32c(positions).reshape(-1, 3)
    out = np.empty((len(x), 3), np.float32)
    c = _ctx(gx.n, gx.box_size)
    c._check(nat.lib().cpm_mesh_interpolate3(c.h, ptr(gx.cells), ptr(gy.cells), ptr(gz.cells), ptr(x), len(x),
                                             ptr(out)))
    return out


class Fft3:
    """fft.rs:11-72 `Fft3`: unnormalised in-place c2c transforms of n^3 complex64 values."""

    def __init__(self, n: int):
        self.n = int(n)

    @staticmethod
    def new(n: int) -> "Fft3":
        return Fft3(n)

    def _run(self, data: np.ndarray, inverse: int) -> None:
        if data.dtype != np.complex64 or not data.flags.c_contiguous or data.size != self.n ** 3:
            raise CpmError(-1, "data must be a C-contiguous complex64 array of n^3 values")
        c = _ctx(self.n, 1.0)
        c._check(nat.lib().cpm_fft3(c.h, ptr(data), self.n, inverse))

    def forward(self, data: np.ndarray) -> None:
        self._run(data, 0)

    def inverse(self, data: np.ndarray) -> None:
        self._run(data, 1)


def wavenumber(i: int, n: int, box_size: float) -> float:
    """fft.rs:86-95."""
    return nat.lib().cpm_wavenumber(int(i), int(n), float(box_size))


class PoissonSolver:
    """poisson.rs:14-88 `PoissonSolver`."""

    def __init__(self, n: int, box_size: float):
        self.n = int(n)
        self.box_size = float(np.float32(box_size))

    @staticmethod
    def new(n: int, box_size: float) -> "PoissonSolver":
        return PoissonSolver(n, box_size)

    def acceleration(self, delta: Mesh, cosmo: Cosmology, a: float, r_split: float) -> list[Mesh]:
        """poisson.rs:33-88: [gx, gy, gz] on the mesh; raises on a mesh-size mismatch (poisson.rs:35)."""
        out = [Mesh(self.n, self.box_size) for _ in range(3)]
        c = _ctx(self.n, self.box_size)
        c._check(nat.lib().cpm_poisson_accel(c.h, ptr(delta.cells), int(delta.n), C.byref(cosmo), float(a),
                                             float(r_split), ptr(out[0].cells), ptr(out[1].cells),
                                             ptr(out[2].cells)))
        return out


class ForceSplit:
    """tree.rs:20-51 `ForceSplit`."""

    def __init__(self, r_split: float, r_cut: float, softening: float, theta: float):
        self.r_split, self.r_cut, self.softening, self.theta = (float(np.float32(v)) for v in
                                                                (r_split, r_cut, softening, theta))

    @staticmethod
    def with_(box_size: float, mesh_n: int, particles_per_side: int, softening_scale: float,
              theta: float) -> "ForceSplit":
        s = nat.lib().cpm_force_split_with(float(box_size), int(mesh_n), int(particles_per_side),
                                           float(softening_scale), float(theta))
        return ForceSplit(s.r_split, s.r_cut, s.softening, s.theta)

    def as_c(self) -> nat.ForceSplitC:
        return nat.ForceSplitC(self.r_split, self.r_cut, self.softening, self.theta)

    def __repr__(self):
        return (f"ForceSplit(r_split={self.r_split}, r_cut={self.r_cut}, softening={self.softening}, "
                f"theta={self.theta})")


def short_range_factor(r: float, r_split: float) -> float:
    """tree.rs:54-57."""
    return nat.lib().cpm_short_range_factor(float(r), float(r_split))


def tree_accelerations(positions, box_size: float, split: ForceSplit, k: float, stats: dict | None = None) -> np.ndarray:
    """tree.rs:314-323 `tree::accelerations`: short-range acceleration of every particle, (N, 3)."""
    x = f32c(positions).reshape(-1, 3)
    out = np.empty_like(x)
    c = _ctx(1, box_size)
    sc = split.as_c()
    c._check(nat.lib().cpm_tree_accel(c.h, ptr(x), len(x), float(box_size), C.byref(sc), float(k), ptr(out)))
    if stats is not None:
        nn, lp, na, md = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        c._check(nat.lib().cpm_tree_stats(c.h, C.byref(nn), C.byref(lp), C.byref(na), C.byref(md)))
        stats.update(nodes=nn.value, leaf_pairs=lp.value, node_accepts=na.value, max_depth=md.value)
    return out


def octant_keys(positions, box_size: float, levels: int = 21) -> tuple[np.ndarray, np.ndarray]:
    """Octant keys of the tree descent (tree.rs:186-250) and their stable sort permutation."""
    x = f32c(positions).reshape(-1, 3)
    keys = np.empty(len(x), np.uint64)
    perm = np.empty(len(x), np.uint32)
    c = _ctx(1, box_size)
    c._check(nat.lib().cpm_octant_keys(c.h, ptr(x), len(x), float(box_size), int(levels), ptr(keys), ptr(perm)))
    return keys, perm


def power_spectrum(positions, box_size: float, mesh_n: int, n_shells: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Shell-averaged matter power spectrum of the particles' CIC density on an n^3 mesh: the
    estimator of ics.rs:213-266 (V |delta_k|^2 / M^2 in shells round(|m|) = 1..n_shells).
    Returns (k_mean, p_mean, counts)."""
    x = f32c(positions).reshape(-1, 3)
    k = np.zeros(n_shells, np.float64)
    p = np.zeros(n_shells, np.float64)
    cnt = np.zeros(n_shells, np.uint64)
    c = _ctx(int(mesh_n), box_size)
    c._check(nat.lib().cpm_power_spectrum(c.h, ptr(x), len(x), int(n_shells), ptr(k), ptr(p), ptr(cnt)))
    return k, p, cnt


def density_grid(delta: "Mesh") -> np.ndarray:
    """frame.rs:30-55 `downsample_grid`: the (m, m, m) texture, index [z, y, x], of 1 + block means."""
    n = delta.n
    gm = n // max(1, -(-n // 128))
    out = np.empty(gm ** 3, np.float32)
    side = C.c_int()
    c = _ctx(n, delta.box_size)
    c._check(nat.lib().cpm_density_grid(c.h, ptr(f32c(delta.cells)), int(n), ptr(out), C.byref(side)))
    return out.reshape(side.value, side.value, side.value)


def ln_a_schedule(a_start: float, a_end: float, steps: int) -> list[float]:
    """runner.rs:240 / integrator.rs:168: a_i = a0 (a_end / a0)^(i / steps) in f32, i = 1..steps."""
    a0 = np.float32(a_start)
    ratio = np.float32(np.float32(a_end) / a0)
    return [float(np.float32(a0 * np.float32(np.power(ratio, np.float32(np.float32(i) / np.float32(steps)),
                                                      dtype=np.float32))))
            for i in range(1, steps + 1)]


def zeldovich(n: int, box_size: float, cosmo: Cosmology, n_s: float, sigma8: float, a_init: float,
              seed: int) -> tuple[np.ndarray, np.ndarray]:
    """ics.rs:119-182 `zeldovich` with `PowerSpectrum::normalized(cosmo, n_s, sigma8, 8)`, on the GPU.
    Returns positions and momenta, (n^3, 3) each, in lattice order."""
    x = np.empty((n ** 3, 3), np.float32)
    p = np.empty((n ** 3, 3), np.float32)
    check(nat.lib().cpm_ics_zeldovich(int(n), float(box_size), C.byref(cosmo), float(n_s), float(sigma8),
                                      float(a_init), int(seed), ptr(x), ptr(p)), sim=True)
    return x, p


def _sim_params(cosmo, box_size, mesh_n, n_particles, split, flags) -> nat.SimParams:
    prm = nat.SimParams()
    prm.cosmo = cosmo
    prm.box_size = float(box_size)
    prm.mesh_n = int(mesh_n)
    prm.n_particles = int(n_particles)
    prm.use_tree = 1 if split is not None else 0
    if split is not None:
        prm.split = split.as_c()
    prm.flags = int(flags)
    return prm


class Simulation:
    """integrator.rs:34-186 `Simulation`, with the state resident on the GPU.

    `split=None` means pure PM (the reference's `Option<ForceSplit>`).
    """

    def __init__(self, cosmo: Cosmology, box_size: float, mesh_n: int, positions, momenta, a: float,
                 split: ForceSplit | None, flags: int = 0, _handle=None, _n: int = 0):
        if _handle is None:
            x = f32c(positions).reshape(-1, 3)
            p = f32c(momenta).reshape(-1, 3)
            if x.shape != p.shape:
                raise CpmError(-1, "positions and momenta must have the same shape")
            prm = _sim_params(cosmo, box_size, mesh_n, len(x), split, flags)
            h = C.c_void_p()
            check(nat.lib().cpm_sim_create(C.byref(prm), ptr(x), ptr(p), float(a), C.byref(h)), sim=True)
            _n = len(x)
        else:
            h = _handle
        self.h = h
        self.n = int(_n)
        self.mesh_n = int(mesh_n)
        self.box_size = float(box_size)
        self.cosmo = cosmo
        self.split = split

    @staticmethod
    def from_zeldovich(cosmo: Cosmology, box_size: float, mesh_n: int, n_side: int, n_s: float, sigma8: float,
                       a_init: float, seed: int, split: ForceSplit | None, flags: int = 0) -> "Simulation":
        """runner.rs:209-225 `init_simulation` with the ICs generated on the GPU (no host round trip)."""
        prm = _sim_params(cosmo, box_size, mesh_n, n_side ** 3, split, flags)
        h = C.c_void_p()
        check(nat.lib().cpm_sim_create_zeldovich(C.byref(prm), int(n_side), float(n_s), float(sigma8),
                                                 float(a_init), int(seed), C.byref(h)), sim=True)
        return Simulation(cosmo, box_size, mesh_n, None, None, a_init, split, flags, _handle=h, _n=n_side ** 3)

    def step_to(self, a1: float) -> None:
        """integrator.rs:174-186."""
        check(nat.lib().cpm_sim_step_to(self.h, float(a1)), sim=True)

    def step_host(self, a1: float, positions: np.ndarray, momenta: np.ndarray) -> None:
        """`step_to` for host-owned state: positions and momenta (float32 (N, 3), C order) are
        uploaded, stepped with the cached acceleration, and overwritten with the new state."""
        for arr in (positions, momenta):
            if arr.dtype != np.float32 or not arr.flags.c_contiguous or arr.size != 3 * self.n:
                raise CpmError(-1, "step_host needs C-contiguous float32 arrays of shape (N, 3)")
        check(nat.lib().cpm_sim_step_host(self.h, float(a1), ptr(positions), ptr(momenta)), sim=True)

    def run(self, a_end: float, steps: int) -> None:
        """integrator.rs:165-171."""
        for a1 in ln_a_schedule(self.a, a_end, steps):
            self.step_to(a1)

    def state(self, want_delta: bool = False) -> dict:
        x = np.empty((self.n, 3), np.float32)
        p = np.empty((self.n, 3), np.float32)
        acc = np.empty((self.n, 3), np.float32)
        delta = np.empty(self.mesh_n ** 3, np.float32) if want_delta else None
        a = C.c_float()
        check(nat.lib().cpm_sim_get_state(self.h, ptr(x), ptr(p), ptr(acc), ptr(delta), C.byref(a)), sim=True)
        return dict(x=x, p=p, acc=acc, delta=delta, a=a.value)

    def set_state(self, positions, momenta) -> None:
        x = f32c(positions).reshape(-1, 3)
        p = f32c(momenta).reshape(-1, 3)
        check(nat.lib().cpm_sim_set_state(self.h, ptr(x), ptr(p)), sim=True)

    @property
    def positions(self) -> np.ndarray:
        return self.state()["x"]

    @property
    def momenta(self) -> np.ndarray:
        return self.state()["p"]

    @property
    def a(self) -> float:
        a = C.c_float()
        check(nat.lib().cpm_sim_get_state(self.h, None, None, None, None, C.byref(a)), sim=True)
        return a.value

    def delta(self) -> Mesh:
        """integrator.rs:128-131: density contrast of the last force calculation."""
        return Mesh(self.mesh_n, self.box_size, self.state(want_delta=True)["delta"])

    def power_spectrum(self, n_shells: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """power_spectrum() of the current particles, computed on the device."""
        k = np.zeros(n_shells, np.float64)
        p = np.zeros(n_shells, np.float64)
        cnt = np.zeros(n_shells, np.uint64)
        check(nat.lib().cpm_sim_power_spectrum(self.h, int(n_shells), ptr(k), ptr(p), ptr(cnt)), sim=True)
        return k, p, cnt

    def phase_times(self, reset: bool = False) -> tuple[np.ndarray, int]:
        ms = np.zeros(8, np.float64)
        steps = C.c_uint64()
        check(nat.lib().cpm_sim_phase_times(self.h, ptr(ms), C.byref(steps), int(reset)), sim=True)
        return ms, steps.value

    def counters(self) -> dict:
        nn, lp, na, ln = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        check(nat.lib().cpm_sim_counters(self.h, C.byref(nn), C.byref(lp), C.byref(na), C.byref(ln)), sim=True)
        cand = C.c_uint64()
        check(nat.lib().cpm_sim_walk_candidates(self.h, C.byref(cand)), sim=True)
        return dict(nodes=nn.value, leaf_pairs=lp.value, node_accepts=na.value, launches_per_step=ln.value,
                    candidates=cand.value)

    def snapshot(self, want_grid: bool = False) -> dict:
        """runner.rs:263-284 `snapshot`: redshift, positions, speeds, densities, rsd shifts, the
        optional density grid and the max speed, with the reductions done on the device."""
        n = self.n
        speeds = np.empty(n, np.float32)
        dens = np.empty(n, np.float32)
        rsd = np.empty((n, 3), np.float32)
        gside = C.c_int()
        gm = self.mesh_n // max(1, -(-self.mesh_n // 128))
        grid = np.empty(gm ** 3, np.float32) if want_grid else None
        vmax = C.c_float()
        check(nat.lib().cpm_sim_snapshot(self.h, ptr(speeds), ptr(dens), ptr(rsd), ptr(grid), C.byref(gside),
                                         C.byref(vmax)), sim=True)
        st = self.state()
        return dict(redshift=np.float32(1.0) / np.float32(st["a"]) - np.float32(1.0), positions=st["x"], speeds=speeds, densities=dens,
                    rsd=rsd, grid=grid.reshape(gside.value, gside.value, gside.value) if want_grid else None,
                    max_speed=vmax.value)

    def graphs(self) -> int:
        """Captured step graphs: 2 once both sorted-buffer parities replay a graph."""
        return int(nat.lib().cpm_sim_graphs(self.h))

    def save(self, path) -> None:
        """Writes the state file (positions, momenta, a and every parameter; cpm_sim_save)."""
        check(nat.lib().cpm_sim_save(self.h, str(path).encode()), sim=True)

    @staticmethod
    def load(path, extra_flags: int = 0) -> "Simulation":
        """A simulation created from a state file written by `save` (cpm_sim_load)."""
        h = C.c_void_p()
        check(nat.lib().cpm_sim_load(str(path).encode(), int(extra_flags), C.byref(h)), sim=True)
        with open(path, "rb") as f:
            hdr = f.read(128)
        n = int(np.frombuffer(hdr[16:24], np.uint64)[0])
        box = float(np.frombuffer(hdr[28:32], np.float32)[0])
        mesh = int(np.frombuffer(hdr[32:36], np.int32)[0])
        use_tree = int(np.frombuffer(hdr[36:40], np.int32)[0])
        cf = np.frombuffer(hdr[40:56], np.float32)
        sp = np.frombuffer(hdr[56:72], np.float32)
        cosmo = Cosmology(*(float(v) for v in cf))
        split = ForceSplit(*(float(v) for v in sp)) if use_tree else None
        a = float(np.frombuffer(hdr[24:28], np.float32)[0])
        return Simulation(cosmo, box, mesh, None, None, a, split, extra_flags, _handle=h, _n=n)

    def set_learned(self, net, delta_threshold: float = 50.0, in_scale: float = 1.0) -> None:
        """Attach a learned short-range net (a `ShortRangeNet` on this mesh; None detaches): particles
        below `delta_threshold` take the net's field, the others keep the tree walk. The simulation
        keeps a reference to the net."""
        check(nat.lib().cpm_sim_set_learned(self.h, net.h if net is not None else None, float(delta_threshold),
                                            float(in_scale)), sim=True)
        self._net = net

    def short_range(self) -> np.ndarray:
        """tree::accelerations (tree.rs:314-323) alone on the current state, caller order."""
        out = np.empty((self.n, 3), np.float32)
        check(nat.lib().cpm_sim_short_range(self.h, ptr(out)), sim=True)
        return out

    def tuning(self) -> dict:
        """The autotuner's choices and the measured ms of every candidate (cpm_sim_autotune_report)."""
        r, t, wp = C.c_int(), C.c_int(), C.c_int()
        ms = np.zeros(9, np.float32)
        check(nat.lib().cpm_sim_autotune_report(self.h, C.byref(r), C.byref(t), C.byref(wp), ptr(ms)), sim=True)
        names = ["fft_radix8", "fft_radix4", "fft_warp", "deposit_tile512", "deposit_tile1024", "deposit_tile2048",
                 "walk_warps2", "walk_warps4", "walk_warps8"]
        return {"fft_radix": r.value, "deposit_tile": t.value, "walk_warps": wp.value,
                "ms": {k: round(float(v), 4) for k, v in zip(names, ms)}}

    def set_tuning(self, fft_radix: int, deposit_tile: int, walk_warps: int) -> None:
        check(nat.lib().cpm_sim_set_tuning(self.h, int(fft_radix), int(deposit_tile), int(walk_warps)), sim=True)

    def tree_depth(self) -> dict:
        """The last tree build's deepest split level and the nodes kept as leaves at the key depth
        (the reference keeps splitting those to depth 40, tree.rs:13)."""
        d, k = C.c_uint32(), C.c_uint64()
        check(nat.lib().cpm_sim_tree_depth(self.h, C.byref(d), C.byref(k)), sim=True)
        return {"max_depth": int(d.value), "key_depth_leaves": int(k.value)}

    def walked(self) -> int:
        """Particles the last step walked the tree for."""
        v = C.c_uint64()
        check(nat.lib().cpm_sim_learned_walked(self.h, C.byref(v)), sim=True)
        return int(v.value)

    def stream(self) -> int:
        return nat.lib().cpm_sim_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None):
            nat.lib().cpm_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EnsembleClass(C.Structure):
    _fields_ = [("n_side", C.c_int), ("mesh_n", C.c_int), ("n_boxes", C.c_int), ("first_seed", C.c_uint64),
                ("split", nat.ForceSplitC)]


class Ensemble:
    """Many independent realisations of uneven sizes (cpm_ensemble_*): classes of equal-size boxes,
    every box a Simulation of integrator.rs:174-186 from Zel'dovich ICs (ics.rs:119-182) with seed
    first_seed + b; every box of a class shares each launch, and one step of the ensemble is one CUDA
    graph with a branch per class. `classes` is a list of (n_side, mesh_n, n_boxes, first_seed, split)."""

    def __init__(self, cosmo: Cosmology, box_size: float, n_s: float, sigma8: float, a_init: float, classes,
                 flags: int = 0):
        arr = (EnsembleClass * len(classes))()
        for i, (n_side, mesh_n, n_boxes, first_seed, split) in enumerate(classes):
            arr[i] = EnsembleClass(int(n_side), int(mesh_n), int(n_boxes), int(first_seed), split.as_c())
        h = C.c_void_p()
        rc = nat.lib().cpm_ensemble_create(C.byref(cosmo), float(box_size), float(n_s), float(sigma8), float(a_init),
                                           len(classes), arr, int(flags), C.byref(h))
        check(rc, sim=True)
        self.h = h
        self.classes = [tuple(c) for c in classes]
        self.a = float(a_init)

    def _check(self, rc):
        if rc != nat.CPM_OK:
            msg = nat.lib().cpm_ensemble_last_error(self.h)
            raise CpmError(rc, msg.decode() if msg else "")

    def step_to(self, a1: float) -> None:
        self._check(nat.lib().cpm_ensemble_step_to(self.h, float(a1)))
        self.a = float(a1)

    def state(self, cls: int, box: int) -> dict:
        n = int(self.classes[cls][0]) ** 3
        x = np.empty((n, 3), np.float32)
        p = np.empty((n, 3), np.float32)
        acc = np.empty((n, 3), np.float32)
        self._check(nat.lib().cpm_ensemble_get_state(self.h, int(cls), int(box), ptr(x), ptr(p), ptr(acc)))
        return dict(x=x, p=p, acc=acc, a=self.a)

    def power_spectrum(self, cls: int, box: int, n_shells: int):
        k = np.empty(n_shells, np.float64)
        pk = np.empty(n_shells, np.float64)
        cnt = np.empty(n_shells, np.uint64)
        self._check(nat.lib().cpm_ensemble_power_spectrum(self.h, int(cls), int(box), int(n_shells), ptr(k), ptr(pk),
                                                          ptr(cnt)))
        return k, pk, cnt

    def graphs(self) -> int:
        return int(nat.lib().cpm_ensemble_graphs(self.h))

    def stream(self) -> int:
        return nat.lib().cpm_ensemble_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None):
            nat.lib().cpm_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
