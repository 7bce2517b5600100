"""Precision study: GPU (f32 arithmetic, uint32 fixed-point positions) against the FP64 build of the
oracle on sampled particles — force error and P(k) error stated per result.

test_precision_small runs always (64^3 particles, 128^3 mesh). test_precision_config3 is the full
study (512^3 particles, 512 Mpc/h, 1024^3 mesh, seed 11, 128 steps to z = 0, checks at the start
and the end on 10^5 particles); its FP64 checks take minutes and ~60 GB of host memory, so it runs
only when CPM_PRECISION_CONFIG3=1, and prints one JSON line with the results."""
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COSMO = (0.0, 0.3, 0.7, 70.0)


def _check(cpm, orc, sim, box, mesh, n, n_sample, seed, quad=False):
    st = sim.state()
    a = float(st["a"])
    sample = np.sort(np.random.default_rng(seed).choice(n, size=min(n_sample, n), replace=False))
    split = orc.split_with(box, mesh, round(n ** (1 / 3)), 1.0 / 30.0, 0.5)
    t0 = time.time()
    ref = orc.accelerations_f64(st["x"], box, mesh, COSMO[1], a, split, sample, quadrupole=quad)
    t_acc = time.time() - t0
    got = st["acc"][sample].astype(np.float64)
    err = np.linalg.norm(got - ref, axis=1)
    mag = np.linalg.norm(ref, axis=1)
    shells = mesh // 4  # k <= k_Nyquist / 2
    t0 = time.time()
    k_o, p_o, c_o = orc.power_spectrum(st["x"], box, mesh, shells)
    t_pk = time.time() - t0
    k_g, p_g, c_g = sim.power_spectrum(shells)
    ok = c_o > 0
    return {
        "a": a, "sampled": int(len(sample)),
        "acc_rel_rms": float(np.sqrt((err ** 2).sum() / (mag ** 2).sum())),
        "acc_rel_median": float(np.median(err / mag)), "acc_rel_p99": float(np.percentile(err / mag, 99)),
        "pk_max_rel": float(np.max(np.abs(p_g[ok] / p_o[ok] - 1.0))),
        "pk_counts_equal": bool(np.array_equal(c_g, c_o)),
        "oracle_s": {"forces": round(t_acc, 1), "pk": round(t_pk, 1)},
    }


def _run(cpm, orc, n_side, mesh, box, seed, steps, n_sample, check_start, quad=False):
    cc = cpm.Cosmology(*COSMO)
    split = cpm.ForceSplit.with_(box, mesh, n_side, 1.0 / 30.0, 0.5)
    flags = cpm._native.SIM_FIXED_POINT | (cpm._native.SIM_QUADRUPOLE if quad else 0)
    sim = cpm.Simulation.from_zeldovich(cc, box, mesh, n_side, 0.96, 0.8, 0.02, seed, split, flags=flags)
    n = n_side ** 3
    out = {"quadrupole": quad}
    if check_start:
        out["start"] = _check(cpm, orc, sim, box, mesh, n, n_sample, 1, quad)
    t0 = time.time()
    for a1 in cpm.ln_a_schedule(0.02, 1.0, steps):
        sim.step_to(a1)
    sim.state()
    out["gpu_run_s"] = round(time.time() - t0, 1)
    out["end"] = _check(cpm, orc, sim, box, mesh, n, n_sample, 2, quad)
    sim.close()
    return out


def test_precision_small(cpm, orc):
    res = _run(cpm, orc, 64, 128, 64.0, 11, 32, 20000, True)
    print(json.dumps({"precision_small": res}))
    for key in ("start", "end"):
        r = res[key]
        assert r["acc_rel_rms"] < 1e-4 and r["acc_rel_median"] < 1e-5, r
        assert r["pk_counts_equal"] and r["pk_max_rel"] < 1e-3, r


@pytest.mark.skipif(os.environ.get("CPM_PRECISION_CONFIG3") != "1", reason="full precision study on request only")
@pytest.mark.parametrize("quad", [False, True])
def test_precision_config3(cpm, orc, quad):
    """The precision mode as a whole: uint32 positions, FP64 kick/drift factors on the device and,
    with quad, quadrupole moments of accepted nodes (checked against the FP64 oracle with the same
    quadrupole terms)."""
    res = _run(cpm, orc, 512, 1024, 512.0, 11, 128, 100000, True, quad)
    print(json.dumps({"precision_config3": res}))
    for key in ("start", "end"):
        r = res[key]
        assert r["acc_rel_rms"] < 1e-3 and r["pk_counts_equal"] and r["pk_max_rel"] < 1e-3, r


def test_quadrupole_forces_match_fp64_oracle_and_beat_monopoles(cpm, orc):
    """CPM_SIM_QUADRUPOLE (no counterpart in the reference): the GPU's quadrupole tree force equals the
    FP64 oracle's quadrupole force to 1e-5 relative RMS of the total, and its short-range error
    against the exact pair sum (the FP64 oracle at theta = 0) is at most a third of the monopole's."""
    rng = np.random.default_rng(4)
    box, mesh, n_side = 32.0, 32, 27
    centres = rng.uniform(0.0, box, (20, 3))
    x = np.mod(centres[rng.integers(0, 20, n_side ** 3)] + rng.normal(0.0, 1.0, (n_side ** 3, 3)),
               box).astype(np.float32)
    p = np.zeros_like(x)
    split = orc.split_with(box, mesh, n_side, 1.0 / 30.0, 0.5)
    exact_split = orc.split_with(box, mesh, n_side, 1.0 / 30.0, 0.0)
    cc = cpm.Cosmology(*COSMO)
    cs = cpm.ForceSplit(split.r_split, split.r_cut, split.softening, split.theta)
    a = 1.0
    nat = cpm._native
    quad = cpm.Simulation(cc, box, mesh, x, p, a, cs, flags=nat.SIM_QUADRUPOLE).state()["acc"]
    mono = cpm.Simulation(cc, box, mesh, x, p, a, cs).state()["acc"]
    sample = np.arange(0, len(x), 29).astype(np.uint32)
    ref_q = orc.accelerations_f64(x, box, mesh, COSMO[1], a, split, sample, quadrupole=True)
    exact = orc.accelerations_f64(x, box, mesh, COSMO[1], a, exact_split, sample)
    pm = orc.accelerations_f64(x, box, mesh, COSMO[1], a, None, sample)

    def rel(u, v):
        return float(np.sqrt(((u - v) ** 2).sum() / (v ** 2).sum()))

    gq = quad[sample].astype(np.float64)
    gm = mono[sample].astype(np.float64)
    assert rel(gq, ref_q) < 1e-5
    err_q = rel(gq - pm, exact - pm)
    err_m = rel(gm - pm, exact - pm)
    print(f"short-range force error vs exact: monopole {err_m:.3e}, quadrupole {err_q:.3e}")
    assert err_q < err_m / 3.0
