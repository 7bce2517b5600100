#!/usr/bin/env python
"""Throughput of the TreePM step in particle-steps/s on B200s (one JSON line on rank 0).

Workload (default): 256^3 = 16,777,216 particles in a periodic 256 Mpc/h box with a 512^3 PM
mesh; Zel'dovich ICs at z = 49 (a = 0.02) from a seed-7 Gaussian field with a BBKS spectrum
(Omega_m 0.3, Omega_L 0.7, h 0.7, sigma8 0.8, n_s 0.96); r_s = 1.25 cells, r_cut = 4.5 r_s,
theta = 0.5, Plummer softening 1/30 of the mean spacing; KDK steps on the 128-step schedule
uniform in ln a to z = 0. A "step" is one KDK step of that schedule: the first W are warm-up, the
next K are timed. Inputs are generated on the GPU (synthetic, no dataset).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device time (CUDA events on the simulation's stream, max over ranks) with the state
resident in HBM; `e2e` is the same metric through the host-buffer C-ABI step (cpm_sim_step_host:
positions and momenta copied host->device and back every step). `--impl reference` times the
CPU restatement of the reference path (oracle/) on this host's cores.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
PKG = "cosmological-particle-simulation_b200"

WORKLOADS = {
    # the headline workload: 256^3 particles, 512^3 mesh, 256 Mpc/h, seed 7, 128 steps to z = 0.
    "treepm-256": dict(n_side=256, mesh=512, box=256.0, seed=7, steps_total=128),
    # the reference's CPU-runnable case: 32^3 particles, 64^3 mesh, 64 Mpc/h, seed 42, 64 steps.
    "treepm-32": dict(n_side=32, mesh=64, box=64.0, seed=42, steps_total=64),
    # profiling case: same physics at 128^3 particles (a few GB on the device).
    "treepm-128": dict(n_side=128, mesh=256, box=128.0, seed=7, steps_total=128),
    # profiling case for the PM traffic: the headline's 1/8 particle per cell at 192^3 / 384^3 (meshes
    # and positions larger than L2, about 3 GB on the device); per-step bytes scale by (256/192)^3.
    "treepm-192": dict(n_side=192, mesh=384, box=192.0, seed=7, steps_total=128),
    # profiling case for the PM kernels: full-size 512^3 mesh, 128^3 particles.
    "pm512-128": dict(n_side=128, mesh=512, box=128.0, seed=7, steps_total=128),
    # the headline workload with the learned short-range force (trained weights, tree walk kept for
    # particles in cells with density contrast >= the trained threshold)
    "learned-256": dict(n_side=256, mesh=512, box=256.0, seed=7, steps_total=128, learned=True),
    "learned-128": dict(n_side=128, mesh=256, box=128.0, seed=7, steps_total=128, learned=True),
}
NET_WEIGHTS = ROOT / PKG / "weights" / "short_range_net.npz"
# the batched ensemble: 64 realisations (seeds 0-63), 16 each at 64^3 / 96^3 / 128^3 / 160^3 particles
# on 128 / 192 / 256 / 320 meshes, 128 Mpc/h boxes, 64 ln-a steps from z = 49
ENSEMBLE = dict(box=128.0, steps_total=64, classes=[(64, 128, 16, 0), (96, 192, 16, 16), (128, 256, 16, 32),
                                                    (160, 320, 16, 48)])
COSMO = dict(omega_r=0.0, omega_m=0.3, omega_l=0.7, h0=70.0)
N_S, SIGMA8, A_INIT, A_END, THETA, SOFT = 0.96, 0.8, 0.02, 1.0, 0.5, 1.0 / 30.0


def pm_bytes_per_step(n: int, mesh: int) -> int:
    """Algorithmic HBM bytes of the PM kernels per step: deposit 12N + 4M, R2C 4M + 4M, k-space
    4M + 12M, 3 C2R 12M + 12M, gather 12M + 24N  =>  36N + 64M."""
    m = mesh ** 3
    return 36 * n + 64 * m


def schedule(steps_total: int, count: int) -> list[float]:
    """runner.rs:240: a_i = a0 (a_end / a0)^(i / steps), i = 1..count (continues past a_end if asked)."""
    a0, ratio = np.float32(A_INIT), np.float32(np.float32(A_END) / np.float32(A_INIT))
    return [float(np.float32(a0 * np.float32(np.power(ratio, np.float32(np.float32(i) / np.float32(steps_total)),
                                                      dtype=np.float32))))
            for i in range(1, count + 1)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def ncu_traffic() -> dict | None:
    """Per-launch DRAM bytes of the PM kernels from the committed ncu summary, when present."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return None
    return None


# ------------------------------------------------------------------------------------------ ours

def replica_seed(base: int, rank: int) -> int:
    """The replicas of a multi-GPU run differ only in the seed of their initial conditions."""
    return base + rank


def max_over_ranks(ms: float, dist, device) -> float:
    """The job's time: the slowest rank's device time. Every rank calls it, in the same order."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(n: int, world: int, steps: int, ms: float) -> float:
    """Whole-job throughput: each of `world` ranks advances its own n particles by `steps` steps."""
    return n * world * steps / (ms / 1e3)


def run_ours(args, rank: int, world: int, dist) -> dict | None:
    import torch

    cpm = importlib.import_module(PKG)
    wl = WORKLOADS[args.workload]
    n_side, mesh, box = wl["n_side"], wl["mesh"], wl["box"]
    n = n_side ** 3
    cosmo = cpm.Cosmology(**COSMO)
    split = cpm.ForceSplit.with_(box, mesh, n_side, SOFT, THETA)
    sched = schedule(wl["steps_total"], args.warmup + args.steps)
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)

    if args.load_state:
        # continue the schedule from a saved state file (cpm_sim_save; profiling of a given epoch, e.g. z = 0)
        loaded = cpm.Simulation.load(args.load_state)
        st0 = loaded.state()
        loaded.close()
        a_saved = float(st0["a"])
        full = schedule(wl["steps_total"], wl["steps_total"] + args.warmup + args.steps + 1)
        i0 = int(np.searchsorted(np.asarray(full, np.float32), np.float32(a_saved), side="right"))
        sched = full[i0:i0 + args.warmup + args.steps]

    net, net_threshold, net_in_scale = None, None, 1.0
    if wl.get("learned"):
        z = np.load(NET_WEIGHTS)
        net = cpm.ShortRangeNet(mesh, z["weights"])
        net_threshold = float(z["threshold"])
        net_in_scale = float(z["in_scale"]) if "in_scale" in z else 1.0

    def make_sim(flags: int, learned: bool = bool(wl.get("learned"))):
        if args.no_autotune:
            flags |= cpm._native.SIM_NO_AUTOTUNE
        if args.load_state:
            sim_ = cpm.Simulation(cosmo, box, mesh, st0["x"], st0["p"], a_saved, split, flags=flags)
        else:
            sim_ = cpm.Simulation.from_zeldovich(cosmo, box, mesh, n_side, N_S, SIGMA8, A_INIT,
                                                 replica_seed(wl["seed"], rank), split, flags=flags)
        if learned:
            sim_.set_learned(net, net_threshold, net_in_scale)
        return sim_

    # The timed run replays the step's captured CUDA graphs (no per-phase events).
    sim = make_sim(0)
    stream = torch.cuda.ExternalStream(sim.stream())
    for a1 in sched[:args.warmup]:
        sim.step_to(a1)
    snapshots = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        st = sim.state()
        snapshots["start"] = (st["x"], st["p"], st["acc"], sched[args.warmup - 1] if args.warmup else A_INIT)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for a1 in sched[args.warmup:]:
        sim.step_to(a1)
    t_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_local = t_start.elapsed_time(t_end)
    if dist:
        dist.barrier()
    ms = max_over_ranks(ms_local, dist, dev)
    counters = sim.counters()
    graphs = sim.graphs()
    walked = sim.walked()
    tuning = sim.tuning()
    depth = sim.tree_depth()
    if args.save_state and rank == 0:
        sim.save(args.save_state)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        st = sim.state()
        snapshots["end"] = (st["x"], st["p"], st["acc"], sched[-1])

    sim.close()

    # Phase breakdown: the same window again with per-phase CUDA events (uncaptured steps).
    phases, nsteps = np.zeros(8), 0
    walk = None
    if not args.no_phases:
        simp = make_sim(cpm._native.SIM_TIMING)
        for a1 in sched[:args.warmup]:
            simp.step_to(a1)
        simp.phase_times(reset=True)
        for a1 in sched[args.warmup:]:
            simp.step_to(a1)
        phases, nsteps = simp.phase_times(reset=True)
        # one more step from the end state (the most clustered): interactions per second of the walk
        simp.step_to(float(np.float32(sched[-1] * sched[-1] / sched[-2])))
        ph1, _ = simp.phase_times()
        c1 = simp.counters()
        inter = c1["leaf_pairs"] + c1["node_accepts"]
        walk = {"interactions": inter, "leaf_pairs": c1["leaf_pairs"], "node_accepts": c1["node_accepts"],
                "candidates": c1["candidates"], "walk_ms": round(float(ph1[6]), 4),
                "interactions_per_s": inter / (float(ph1[6]) / 1e3) if ph1[6] > 0 else None,
                "note": "one step after the timed window (a beyond the last timed a), walk + second kick timed"}
        simp.close()

    # End to end through the host-buffer C-ABI step, same schedule window, on a fresh simulation.
    e2e = None
    if not args.no_e2e:
        sim2 = make_sim(0)
        for a1 in sched[:args.warmup]:
            sim2.step_to(a1)
        xs = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        ps = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        st = sim2.state()
        xs.numpy()[:] = st["x"]
        ps.numpy()[:] = st["p"]
        xh, ph = xs.numpy(), ps.numpy()
        e2e_steps = sched[args.warmup:args.warmup + args.e2e_steps] if args.e2e_steps else sched[args.warmup:]
        s2 = torch.cuda.ExternalStream(sim2.stream())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s2)
        for a1 in e2e_steps:
            sim2.step_host(a1, xh, ph)
        e1.record(s2)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        sim2.close()
        e2e = {"value": job_rate(n, world, len(e2e_steps), ems), "unit": "particle-steps/s",
               "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n, "steps": len(e2e_steps),
               "api": "cpm_sim_step_host (pinned host x, p in/out each step)"}

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    pm_ms = phases[2] + phases[3] + phases[4]  # deposit, FFT-Poisson, gather
    pm_b = pm_bytes_per_step(n, mesh)
    achieved = pm_b / (pm_ms / 1e3) / 1e9 if pm_ms > 0 else 0.0
    traffic = ncu_traffic()
    phase_names = ["kick_drift", "keys_sort_reorder", "deposit", "fft_poisson", "gather", "tree_build",
                   "tree_walk_kick2", "step"]
    line = {
        "metric": "particle-steps/s", "value": job_rate(n, world, args.steps, ms), "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (Zel'dovich ICs generated on the GPU, Philox white noise)",
        "config": {"workload": f"TreePM {n_side}^3 particles, {mesh}^3 mesh, L={box:g} Mpc/h, seed {wl['seed']}"
                               f"{'+rank' if world > 1 else ''}, theta={THETA}, a={A_INIT}->{A_END} in "
                               f"{wl['steps_total']} ln-a steps; timed steps {args.warmup + 1}..{args.warmup + args.steps}"
                               f" (a={sched[args.warmup]:.4f}..{sched[-1]:.4f})",
                   "particles_per_gpu": n, "mesh": mesh, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (positions 201 MB, meshes 537 MB each)"},
        "roofline": {"bound": "hbm", "kernels": "PM: deposit + FFT-Poisson + gather",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "peak_kind": peak_kind, "algorithmic_bytes_per_step": pm_b,
                     "traffic": traffic.get("pm_bytes_per_step")
                     if traffic and traffic.get("workload") == args.workload else None},
        "phase_ms": {k: round(float(v), 4) for k, v in zip(phase_names, phases)} if nsteps else None,
        "phase_steps": nsteps,
        "phase_note": "per-phase CUDA events on a second run of the same window (uncaptured steps)",
        "step_graphs": graphs,
        "tree": {"nodes_last_step": counters["nodes"], "leaf_pairs_last_step": counters["leaf_pairs"],
                 "node_accepts_last_step": counters["node_accepts"],
                 "candidates_last_step": counters["candidates"]},
        "tree_walk_end_state": walk,
        "walked_last_step": walked,
        "autotune": tuning,
        "tree_depth_last_step": depth,
        "learned": ({"net": "3-layer 3^3 conv, 16 channels, BF16 tcgen05 kernels", "weights": str(NET_WEIGHTS.name),
                     "delta_threshold": net_threshold,
                     "note": "phase gather_ms includes the net inference; walk only for particles at or above "
                             "the threshold"} if net is not None else None),
        "gpu_launches": counters["launches_per_step"] * args.steps,
        "launches_per_step": counters["launches_per_step"],
        "clocks": clk,
        "e2e": e2e,
    }
    if snapshots:
        line["cpu_baseline"], line["parity"] = cpu_baseline(args, snapshots, wl, n)
    return line


def cpu_baseline(args, snapshots: dict, wl: dict, n: int) -> tuple[dict, dict]:
    """The oracle (CPU restatement of the reference path, OpenMP on all host cores) timed on one
    sampled KDK step at the start and at the end of the timed window, from the GPU run's state:
    every phase on all particles, the tree walk on a random subset scaled to all particles. The
    sampled step has zero length (a1 = a0: kick and drift factors 0, the same work), so its force
    evaluation is on the GPU state's own positions at the GPU state's a; the oracle's PM + tree force
    on the sampled particles is then compared with the GPU's (relative RMS), which is the parity
    number of the headline workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    cores = os.cpu_count() or 1
    c = orc.cosmology(COSMO["omega_r"], COSMO["omega_m"], COSMO["omega_l"], COSMO["h0"])
    split = orc.split_with(wl["box"], wl["mesh"], wl["n_side"], SOFT, THETA)
    frac = args.cpu_walk_fraction
    rng = np.random.default_rng(0)
    m = max(1024, int(n * frac))
    subset = np.sort(rng.choice(n, size=min(m, n), replace=False)).astype(np.uint32)
    per_step, detail, parity = [], {}, {}
    for name, (x, p, acc, a0) in snapshots.items():
        t, acc_cpu, acc_64 = orc.step_sample(c, wl["box"], wl["mesh"], x, p, acc, a0, a0, split, subset,
                                             threads=cores, want_acc=True, want_com64=True)
        est = float(t[:5].sum() + t[5] * (n / len(subset)) + t[6])
        per_step.append(est)
        detail[name] = {"a": a0, "s_per_step_est": round(est, 3), "phases_s": [round(float(v), 3) for v in t]}
        g = acc[subset].astype(np.float64)
        for key, ref in (("", acc_cpu), ("com64_", acc_64)):
            r = ref.astype(np.float64)
            err = np.sqrt(((g - r) ** 2).sum(1)) / np.maximum(np.sqrt((r ** 2).sum(1)), 1e-30)
            parity[f"acc_{key}rel_rms_{name}"] = float(np.sqrt(((g - r) ** 2).sum() / (r ** 2).sum()))
            parity[f"acc_{key}rel_p99_{name}"] = float(np.percentile(err, 99))
        parity[f"a_{name}"] = a0
    mean_step = sum(per_step) / len(per_step)
    parity.update({"particles": len(subset), "bar": 1e-5,
                   "what": "PM + tree acceleration of a random subset of particles, GPU vs the oracle on the "
                           "same positions: relative RMS over the subset and 99th percentile of the per-particle "
                           "relative error; acc_ against the reference's arithmetic (f32 centre-of-mass sums), "
                           "acc_com64_ against the oracle's twin with FP64 centre-of-mass sums rounded once, as on "
                           "the GPU (where f32 sums round a node's centre differently, an opening decision at its "
                           "boundary can flip)"})
    return ({"value": n / mean_step, "unit": "particle-steps/s", "cores": cores, "kind": "port",
             "sample": (f"one oracle KDK step of zero length (a1 = a0, the work of a full step) at the start "
                        f"(a={snapshots['start'][3]:.4f}) and end (a={snapshots['end'][3]:.4f}) of the timed window, "
                        f"from the GPU state; all phases on all {n} particles except the tree walk, run for a random "
                        f"{len(subset)} ({frac:.4g}) and scaled; value = N / mean estimated step time"),
             "detail": detail}, parity)


def run_ensemble(args, rank: int, world: int, dist) -> dict | None:
    """The batched ensemble (each rank its own copy, seeds offset by 64 * rank): one ensemble step of
    all realisations per timed step, replayed from its captured CUDA graph."""
    import torch

    cpm = importlib.import_module(PKG)
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    cosmo = cpm.Cosmology(**COSMO)
    box = ENSEMBLE["box"]
    classes = [(n_side, mesh, boxes, seed + 64 * rank, cpm.ForceSplit.with_(box, mesh, n_side, SOFT, THETA))
               for n_side, mesh, boxes, seed in ENSEMBLE["classes"]]
    n = sum(c[0] ** 3 * c[2] for c in classes)
    sched = schedule(ENSEMBLE["steps_total"], args.warmup + args.steps)
    ens = cpm.Ensemble(cosmo, box, N_S, SIGMA8, A_INIT, classes)
    stream = torch.cuda.ExternalStream(ens.stream())
    for a1 in sched[:args.warmup]:
        ens.step_to(a1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for a1 in sched[args.warmup:]:
        ens.step_to(a1)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(t0.elapsed_time(t1), dist, dev)
    graphs = ens.graphs()
    ens.close()
    if rank != 0:
        return None
    return {
        "metric": "particle-steps/s", "value": job_rate(n, world, args.steps, ms), "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (Zel'dovich ICs generated on the GPU, Philox white noise, seed per realisation)",
        "config": {"workload": "batched ensemble: 64 realisations, 16 each at 64^3/96^3/128^3/160^3 particles on "
                               "128/192/256/320 meshes, L=128 Mpc/h, 64 ln-a steps from z=49; timed steps "
                               f"{args.warmup + 1}..{args.warmup + args.steps}",
                   "particles_per_gpu": n, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2"},
        "step_graphs": graphs, "clocks": clk, "e2e": None,
        "e2e_note": "device-resident ensemble; the host-buffer end-to-end path is measured on the headline workload",
    }


# ------------------------------------------------------------------------------------- reference

def run_reference(args, rank: int, world: int) -> dict | None:
    """The CPU restatement of the reference path (oracle/, OpenMP on all cores), full KDK steps on
    the same workload from its Zel'dovich ICs (oracle IC generator, same spectrum and seed), timed
    by wall clock; steps stop once the time budget is spent (at least one)."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    if args.workload == "ensemble":  # the oracle steps one realisation: time its largest class
        args.workload = "treepm-128"
    wl = WORKLOADS[args.workload]
    n_side, mesh, box = wl["n_side"], wl["mesh"], wl["box"]
    n = n_side ** 3
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    c = orc.cosmology(COSMO["omega_r"], COSMO["omega_m"], COSMO["omega_l"], COSMO["h0"])
    ps = orc.power_normalized(c, N_S, SIGMA8, 8.0)
    x, p = orc.zeldovich(n_side, box, c, ps, A_INIT, wl["seed"])
    split = orc.split_with(box, mesh, n_side, SOFT, THETA)
    sim = orc.Simulation(c, box, mesh, x, p, A_INIT, split)
    sched = schedule(wl["steps_total"], max(args.steps, 1) + 1)
    t0 = time.perf_counter()
    done = 0
    for a1 in sched[:args.steps]:
        sim.step_to(a1)
        done += 1
        if time.perf_counter() - t0 > args.ref_budget_s:
            break
    wall = time.perf_counter() - t0
    sim.close()
    value = n * done / wall
    sample = (f"{done} full oracle KDK steps (of {args.steps} requested; time budget {args.ref_budget_s:.0f} s) "
              f"from the z=49 ICs, all {n} particles, {cores} OpenMP threads")
    return {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": done,
        "warmup": 0, "ms_per_step": wall * 1e3 / done, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (Zel'dovich ICs from the oracle IC generator)",
        "config": {"workload": f"TreePM {n_side}^3 particles, {mesh}^3 mesh, L={box:g} Mpc/h, seed {wl['seed']}, "
                               f"theta={THETA}; steps from a={A_INIT}"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=125)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["ensemble"], default="treepm-256")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps in the end-to-end run (0 = same as --steps)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-phases", action="store_true", help="skip the second, per-phase timed run")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch parameters (FFT radix 8, deposit tile 1024, walk group 4 warps), no timing "
                         "of alternatives: a fixed launch sequence for profiling")
    ap.add_argument("--cpu-walk-fraction", type=float, default=1.0 / 64.0)
    ap.add_argument("--ref-budget-s", type=float, default=120.0)
    ap.add_argument("--save-state", default="", help="write the state file (cpm_sim_save) after the timed steps")
    ap.add_argument("--load-state", default="", help="start from a state file (cpm_sim_save) and continue its schedule")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    # The timed steps end at z = 0: a workload's schedule has steps_total steps (warm-up included).
    total = ENSEMBLE["steps_total"] if args.workload == "ensemble" else WORKLOADS[args.workload]["steps_total"]
    if args.impl == "ours" and not args.load_state and args.warmup + args.steps > total:
        args.steps = max(1, total - args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        if world > 1:
            import torch
            import torch.distributed as tdist
            from datetime import timedelta
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
            dist = tdist
        line = run_ensemble(args, rank, world, dist) if args.workload == "ensemble" else run_ours(args, rank, world, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
