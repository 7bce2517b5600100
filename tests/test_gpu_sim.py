"""GPU parity of the device-resident simulation (integrator.rs:34-186) against the oracle, and the
reference's integrator tests (integrator.rs:368-461) run on the GPU path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def periodic_max_diff(a, b, box):
    d = np.abs(a.astype(np.float64) - b)
    return float(np.minimum(d, box - d).max())


def _plane_wave(orc, n, box, amp, cosmo, a_init):
    f32 = np.float32
    k = f32(f32(2.0) * f32(np.pi)) / f32(box)
    h = f32(box) / f32(n)
    d = f32(orc.growth(cosmo, a_init))
    f = f32(orc.growth_rate(cosmo, a_init))
    e = f32(orc.cosmo_e(cosmo, a_init))
    a = f32(a_init)
    i = np.arange(n, dtype=np.float32) * h
    qx, qy, qz = (v.ravel() for v in np.meshgrid(i, i, i, indexing="ij"))
    psi_x = (-(f32(amp) / k) * np.sin(k * qx).astype(np.float32)).astype(np.float32)
    x = np.mod(qx + d * psi_x, f32(box)).astype(np.float32)
    pos = np.stack([x, qy, qz], 1).astype(np.float32)
    mom = np.zeros_like(pos)
    mom[:, 0] = (a * a * f * e * d) * psi_x
    return pos, mom


def _ics(orc, n, box, a_init, seed):
    """Zel'dovich ICs of the config cosmology (Omega_m 0.3, h 0.7, sigma8 0.8, n_s 0.96)."""
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    ps = orc.power_normalized(c, 0.96, 0.8, 8.0)
    x, p = orc.zeldovich(n, box, c, ps, a_init, seed)
    return c, x, p


def test_pm_step_matches_oracle_bit_for_bit_kick_drift(cpm, orc):
    """PM only: the initial force within 1e-5 RMS, and after 3 steps positions within 1e-5 L."""
    c, x, p = _ics(orc, 16, 64.0, 0.02, 42)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    gpu = cpm.Simulation(cc, 64.0, 32, x, p, 0.02, None)
    ref = orc.Simulation(c, 64.0, 32, x, p, 0.02, None)
    assert rel_rms(gpu.state()["acc"], ref.state()["acc"]) < 1e-5
    for a1 in cpm.ln_a_schedule(0.02, 0.05, 3):
        gpu.step_to(a1)
        ref.step_to(a1)
    g, r = gpu.state(), ref.state()
    assert g["a"] == r["a"]
    assert periodic_max_diff(g["x"], r["x"], 64.0) < 1e-5 * 64.0
    assert rel_rms(g["acc"], r["acc"]) < 1e-5


@pytest.mark.parametrize("mesh", [32, 48])
def test_deconvolved_pm_forces_match_oracle(cpm, orc, mesh):
    """CPM_SIM_DECONVOLVE (no counterpart in the reference): the PM force with the Green's function
    divided by the CIC window squared, against the oracle's poisson.rs:33-88 with the same factor,
    gathered with mesh.rs:72-77; the factor itself changes the force well beyond that bar."""
    rng = np.random.default_rng(mesh)
    box = 64.0
    centres = rng.uniform(0.0, box, (12, 3))
    x = np.mod(centres[rng.integers(0, 12, 20000)] + rng.normal(0.0, 2.0, (20000, 3)), box).astype(np.float32)
    p = np.zeros_like(x)
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    a = 0.5
    acc = cpm.Simulation(cc, box, mesh, x, p, a, None, flags=cpm._native.SIM_DECONVOLVE).state()["acc"]
    delta = orc.density_contrast(mesh, box, x)
    ref = np.stack([orc.interpolate_many(mesh, box, g, x)
                    for g in orc.poisson_accel(mesh, box, delta, c.omega_m, a, 0.0, deconvolve=True)], 1)
    plain = np.stack([orc.interpolate_many(mesh, box, g, x)
                      for g in orc.poisson_accel(mesh, box, delta, c.omega_m, a, 0.0)], 1)
    assert rel_rms(acc, ref) < 1e-5
    assert rel_rms(plain, ref) > 1e-3


def test_pm_step_on_a_mixed_radix_mesh(cpm, orc):
    """PM steps on a 48^3 mesh (radix 2 and 3) with 20^3 particles: force and positions as the oracle."""
    c, x, p = _ics(orc, 20, 60.0, 0.02, 8)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    gpu = cpm.Simulation(cc, 60.0, 48, x, p, 0.02, None)
    ref = orc.Simulation(c, 60.0, 48, x, p, 0.02, None)
    assert rel_rms(gpu.state()["acc"], ref.state()["acc"]) < 1e-5
    for a1 in cpm.ln_a_schedule(0.02, 0.04, 2):
        gpu.step_to(a1)
        ref.step_to(a1)
    g, r = gpu.state(), ref.state()
    assert periodic_max_diff(g["x"], r["x"], 60.0) < 1e-5 * 60.0
    assert rel_rms(g["acc"], r["acc"]) < 1e-5


def test_treepm_accelerations_match_oracle(cpm, orc):
    """TreePM force at the ICs and after 2 steps: within 1e-5 relative RMS (config-1 cosmology)."""
    n, box, mesh = 16, 32.0, 32
    c, x, p = _ics(orc, n, box, 0.02, 42)
    split = orc.split_with(box, mesh, n, 1.0 / 30.0, 0.5)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    cs = cpm.ForceSplit(split.r_split, split.r_cut, split.softening, split.theta)
    gpu = cpm.Simulation(cc, box, mesh, x, p, 0.02, cs)
    ref = orc.Simulation(c, box, mesh, x, p, 0.02, split)
    assert rel_rms(gpu.state()["acc"], ref.state()["acc"]) < 1e-5
    for a1 in cpm.ln_a_schedule(0.02, 0.2, 8)[:2]:
        gpu.step_to(a1)
        ref.step_to(a1)
    g, r = gpu.state(want_delta=True), ref.state(want_delta=True)
    assert periodic_max_diff(g["x"], r["x"], box) < 1e-5 * box
    assert rel_rms(g["acc"], r["acc"]) < 1e-5
    assert rel_rms(g["delta"] + 1.0, r["delta"] + 1.0) < 1e-6


def test_linear_growth_matches_growth_factor(cpm, orc):
    """integrator.rs:368-388 on the GPU."""
    box, cosmo = 1.0, orc.lcdm_default()
    a_init, a_final = 0.02, 0.1
    x, p = _plane_wave(orc, 32, box, 0.5, cosmo, a_init)
    sim = cpm.Simulation(cpm.Cosmology.lcdm_default(), box, 32, x, p, a_init, None)

    def mode(xs):
        d = orc.density_contrast(32, box, xs).reshape(32, 32, 32).astype(np.float64)
        cx = np.cos((np.arange(32) + 0.5) * (box / 32) * 2 * np.pi / box)
        return 2.0 * float((d * cx[:, None, None]).sum()) / 32 ** 3

    before = mode(x)
    for a1 in cpm.ln_a_schedule(a_init, a_final, 40):
        sim.step_to(a1)
    after = mode(sim.positions)
    expected = orc.growth(cosmo, a_final) / orc.growth(cosmo, a_init)
    assert abs(after / before - expected) / expected < 0.01


def test_total_momentum_stays_near_zero(cpm, orc):
    """integrator.rs:417-435 on the GPU."""
    x, p = _plane_wave(orc, 16, 1.0, 0.5, orc.lcdm_default(), 0.02)
    sim = cpm.Simulation(cpm.Cosmology.lcdm_default(), 1.0, 32, x, p, 0.02, None)
    for a1 in cpm.ln_a_schedule(0.02, 0.1, 20):
        sim.step_to(a1)
    mom = sim.momenta.astype(np.float64)
    assert np.all(np.abs(mom.sum(0)) < 1e-3 * np.abs(mom[:, 0]).sum())


def test_treepm_pair_force_matches_newton(cpm, orc):
    """integrator.rs:437-461 on the GPU."""
    box, mesh_n = 100.0, 64
    std = cpm.ForceSplit.with_(box, mesh_n, 2, 0.05, 0.5)
    split = cpm.ForceSplit(std.r_split, std.r_cut, 0.01, std.theta)
    pos = np.array([[50.0, 50.0, 50.0], [53.0, 50.0, 50.0]], np.float32)
    cosmo = cpm.Cosmology.lcdm_default()
    sim = cpm.Simulation(cosmo, box, mesh_n, pos, np.zeros_like(pos), 1.0, split)
    acc = sim.state()["acc"]
    f32 = np.float32
    k = f32(1.5) * f32(cosmo.omega_m) * f32(box) ** 3 / (f32(4.0) * f32(np.pi) * f32(1.0) * f32(2.0))
    newton = float(k / f32(9.0))
    assert acc[0, 0] > 0.0 and acc[1, 0] < 0.0
    assert abs(acc[0, 0] - newton) / newton < 0.05 and abs(acc[1, 0] + newton) / newton < 0.05


@pytest.mark.parametrize("n,box,seed", [(16, 64.0, 42), (32, 128.0, 7), (48, 96.0, 3)])
def test_zeldovich_ics_match_oracle(cpm, orc, n, box, seed):
    """ics.rs:78-182 on the GPU vs the oracle: same Philox noise, same f32 scalars; FFT round-off only."""
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    ps = orc.power_normalized(c, 0.96, 0.8, 8.0)
    xr, pr = orc.zeldovich(n, box, c, ps, 0.02, seed)
    xg, pg = cpm.zeldovich(n, box, cpm.Cosmology(0.0, 0.3, 0.7, 70.0), 0.96, 0.8, 0.02, seed)
    assert periodic_max_diff(xg, xr, box) < 1e-5 * box
    assert rel_rms(pg, pr) < 1e-5


def test_sim_from_device_ics_equals_host_ics(cpm, orc):
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(32.0, 32, 16, 1.0 / 30.0, 0.5)
    x, p = cpm.zeldovich(16, 32.0, cc, 0.96, 0.8, 0.02, 5)
    a = cpm.Simulation(cc, 32.0, 32, x, p, 0.02, split)
    b = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 5, split)
    sa, sb = a.state(), b.state()
    assert np.array_equal(sa["x"], sb["x"]) and np.array_equal(sa["p"], sb["p"])
    assert np.array_equal(sa["acc"], sb["acc"])


def test_step_host_equals_step_to(cpm):
    """cpm_sim_step_host (host-owned state; positions copied out on a second stream while the
    forces run) gives bit-identical results to the resident step, graph-replayed steps included,
    and resident steps may follow host steps."""
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(32.0, 32, 16, 1.0 / 30.0, 0.5)
    a = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 9, split)
    b = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 9, split)
    st = b.state()
    xh, ph = st["x"].copy(), st["p"].copy()
    sched = cpm.ln_a_schedule(0.02, 0.3, 8)
    for a1 in sched[:6]:
        a.step_to(a1)
        b.step_host(a1, xh, ph)
        sa = a.state()
        assert np.array_equal(sa["x"], xh) and np.array_equal(sa["p"], ph)
    for a1 in sched[6:]:
        a.step_to(a1)
        b.step_to(a1)
    sa, sb = a.state(), b.state()
    assert np.array_equal(sa["x"], sb["x"]) and np.array_equal(sa["p"], sb["p"])


def test_graph_replay_equals_direct_launches(cpm):
    """Steps replayed from the captured CUDA graphs give bit-identical states to steps launched
    kernel by kernel (CPM_SIM_NO_GRAPH); both parities get a graph after four steps."""
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(32.0, 32, 16, 1.0 / 30.0, 0.5)
    g = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 4, split)
    d = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 4, split, flags=cpm._native.SIM_NO_GRAPH)
    for i, a1 in enumerate(cpm.ln_a_schedule(0.02, 0.5, 8)):
        g.step_to(a1)
        d.step_to(a1)
        if i == 1:
            assert g.graphs() == 0  # the first step of each parity runs uncaptured
    assert g.graphs() == 2 and d.graphs() == 0
    sg, sd = g.state(), d.state()
    for key in ("x", "p", "acc"):
        assert np.array_equal(sg[key], sd[key]), key
    assert g.counters()["leaf_pairs"] == d.counters()["leaf_pairs"]


def test_fixed_point_mode_tracks_f32_mode(cpm):
    """CPM_SIM_FIXED_POINT (uint32 positions) follows the f32 trajectory from the same ICs."""
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(32.0, 32, 16, 1.0 / 30.0, 0.5)
    f = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 5, split)
    q = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 5, split, flags=cpm._native.SIM_FIXED_POINT)
    for a1 in cpm.ln_a_schedule(0.02, 0.3, 6):
        f.step_to(a1)
        q.step_to(a1)
    sf, sq = f.state(), q.state()
    assert periodic_max_diff(sq["x"], sf["x"], 32.0) < 1e-4 * 32.0
    assert rel_rms(sq["p"], sf["p"]) < 1e-3
    assert sq["x"].min() >= 0.0 and sq["x"].max() <= 32.0


def test_fixed_point_drift_wraps_exactly(cpm, orc):
    """A force-free lattice streaming across the periodic boundary several times ends where the
    summed drift factors put it, to f32 resolution (the uint32 wrap loses nothing)."""
    box = 32.0
    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    g = np.array([4.0, 20.0], np.float32)
    x0 = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    sched = cpm.ln_a_schedule(0.5, 1.0, 5)
    a_prev, dsum = 0.5, 0.0
    for a1 in sched:
        dsum += orc.drift_factor(c, a_prev, a1)
        a_prev = a1
    v = np.float32(3.3 * box / dsum)  # 3.3 box lengths along x over the run
    p0 = np.zeros_like(x0)
    p0[:, 0] = v
    split = cpm.ForceSplit.with_(box, 32, 2, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation(cc, box, 32, x0, p0, 0.5, split, flags=cpm._native.SIM_FIXED_POINT)
    for a1 in sched:
        sim.step_to(a1)
    st = sim.state()
    assert np.max(np.abs(st["p"] - p0)) < 1e-5 * v  # the lattice feels no net force
    want = np.mod(x0[:, 0].astype(np.float64) + float(v) * dsum, box)
    assert periodic_max_diff(st["x"][:, 0], want, box) < 2e-5 * box
    assert np.max(np.abs(st["x"][:, 1:] - x0[:, 1:])) < 1e-5


def test_phase_timing_and_counters(cpm):
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(32.0, 32, 16, 1.0 / 30.0, 0.5)
    s = cpm.Simulation.from_zeldovich(cc, 32.0, 32, 16, 0.96, 0.8, 0.02, 9, split, flags=cpm._native.SIM_TIMING)
    for a1 in cpm.ln_a_schedule(0.02, 0.3, 6):
        s.step_to(a1)
    ms, steps = s.phase_times()
    assert s.graphs() == 0  # phase timing records events between kernels: no capture
    assert steps == 6 and np.all(ms >= 0) and ms[7] > 0
    assert abs(ms[:7].sum() - ms[7]) < 0.05 * ms[7] + 1e-3
    c = s.counters()
    assert c["nodes"] > 0 and c["leaf_pairs"] > 0 and c["launches_per_step"] > 10


def test_sim_rejects_bad_arguments(cpm):
    x = np.zeros((8, 3), np.float32)
    with pytest.raises(cpm.CpmError) as e:
        cpm.Simulation(cpm.Cosmology.lcdm_default(), 1.0, 12, x, x, 0.1, None)
    assert e.value.code == -4
    x[3, 0] = np.inf
    with pytest.raises(cpm.CpmError) as e:
        cpm.Simulation(cpm.Cosmology.lcdm_default(), 1.0, 8, x, np.zeros_like(x), 0.1, None)
    assert e.value.code == -6


def test_state_file_round_trip(cpm, tmp_path):
    """cpm_sim_save / cpm_sim_load: the loaded simulation holds the same x, p and a, and steps on
    exactly like the saved one; a corrupted file is rejected."""
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(64.0, 64, 32, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation.from_zeldovich(cc, 64.0, 64, 32, 0.96, 0.8, 0.02, 42, split)
    sched = cpm.ln_a_schedule(0.02, 1.0, 64)
    for a1 in sched[:20]:
        sim.step_to(a1)
    path = tmp_path / "state.cpm"
    sim.save(path)
    other = cpm.Simulation.load(path)
    s0, s1 = sim.state(), other.state()
    assert np.array_equal(s0["x"], s1["x"]) and np.array_equal(s0["p"], s1["p"]) and s0["a"] == s1["a"]
    assert rel_rms(s1["acc"], s0["acc"]) < 1e-6
    for a1 in sched[20:24]:
        sim.step_to(a1)
        other.step_to(a1)
    s0, s1 = sim.state(), other.state()
    assert periodic_max_diff(s1["x"], s0["x"], 64.0) < 1e-5
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0xFF
    bad = tmp_path / "bad.cpm"
    bad.write_bytes(bytes(raw))
    with pytest.raises(cpm.CpmError) as e:
        cpm.Simulation.load(bad)
    assert e.value.code == -1
    sim.close()
    other.close()


def test_step_factors_fp64_and_reference(cpm, orc):
    """cpm_step_factors: the f32 path equals the oracle's restatement of integrator.rs:263-297 bit for
    bit; the FP64 device path (precision mode) agrees with a 4096-interval Simpson and bisection in
    double to 1e-12 relative (d) and to f32 rounding (k1, k2)."""
    import ctypes as C
    import math

    c = orc.cosmology(0.0, 0.3, 0.7, 70.0)
    cc = cpm.Cosmology(c.omega_r, c.omega_m, c.omega_l, c.h0)
    L = cpm.lib()

    def factors(a0, a1, fp64):
        k1, d, k2 = C.c_double(), C.c_double(), C.c_double()
        assert L.cpm_step_factors(C.byref(cc), a0, a1, fp64, C.byref(k1), C.byref(d), C.byref(k2)) == 0
        return k1.value, d.value, k2.value

    om, ol = float(np.float32(0.3)), float(np.float32(0.7))  # the cosmology's f32 fields, widened

    def e64(a):
        return math.sqrt(om / a ** 3 + ol)

    def simpson(f, lo, hi, m=4096):
        h = (hi - lo) / m
        return (f(lo) + f(hi) + sum((4 if i % 2 else 2) * f(lo + i * h) for i in range(1, m))) * h / 3

    kick = lambda a: 1.0 / (a * e64(a))
    drift = lambda a: 1.0 / (a ** 3 * e64(a))
    for a0, a1 in [(0.02, 0.0206), (0.3, 0.31), (0.95, 1.0)]:
        r = factors(a0, a1, 0)
        am = orc.midpoint(c, a0, a1)
        assert r == (orc.kick_factor(c, a0, am), orc.drift_factor(c, a0, a1), orc.kick_factor(c, am, a1))
        half = simpson(kick, a0, a1) / 2
        lo, hi = a0, a1
        for _ in range(60):
            mid = 0.5 * (lo + hi)
            lo, hi = (mid, hi) if simpson(kick, a0, mid, 512) < half else (lo, mid)
        am64 = 0.5 * (lo + hi)
        k1, d, k2 = factors(a0, a1, 1)
        assert abs(d / simpson(drift, a0, a1) - 1.0) < 1e-12
        assert abs(k1 / simpson(kick, a0, am64) - 1.0) < 2e-7
        assert abs(k2 / simpson(kick, am64, a1) - 1.0) < 2e-7


def test_autotuned_variants_give_the_same_forces(cpm):
    """The autotuner's alternatives: every deposit tile and walk group gives bit-identical forces;
    the radix-4 plan of the Poisson FFT agrees with the radix-8 plan to FFT rounding."""
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(64.0, 64, 32, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation.from_zeldovich(cc, 64.0, 64, 32, 0.96, 0.8, 0.02, 5, split)
    for a1 in cpm.ln_a_schedule(0.02, 1.0, 64)[:48]:
        sim.step_to(a1)
    t = sim.tuning()
    assert t["fft_radix"] in (0, 4, 8) and t["deposit_tile"] in (512, 1024, 2048) and t["walk_warps"] in (2, 4, 8)
    assert all(v > 0.0 for v in t["ms"].values())
    st = sim.state()
    accs = {}
    for radix in (8, 4, 0):
        for tile in (512, 1024, 2048):
            for warps in (2, 4, 8):
                sim.set_tuning(radix, tile, warps)
                sim.set_state(st["x"], st["p"])
                accs[(radix, tile, warps)] = sim.state()["acc"]
    for key, acc in accs.items():
        same_radix = accs[(key[0], 1024, 4)]
        assert np.array_equal(acc, same_radix), key
    assert rel_rms(accs[(4, 1024, 4)], accs[(8, 1024, 4)]) < 1e-6
    assert np.array_equal(accs[(0, 1024, 4)], accs[(8, 1024, 4)])  # no warp plan for 64- and 32-point lines
    sim.close()


@pytest.mark.parametrize("mesh", [256, 512])
def test_warp_fft_plan_matches_stockham_plan(cpm, mesh):
    """FFT plan 0 (one warp per 256- or 512-point line, register stages) against the radix-8 Stockham
    plan, whose Poisson solve is checked against the oracle at these sizes: the PM forces of the
    same state agree to FFT rounding (the plans add in different orders; f32 FFT round-off grows
    with log n, about 1e-6 relative at these sizes). Mesh 512 runs every pass on the warp plan
    (512-point x and y lines, 256-point half-length z lines); mesh 256 its x and y passes."""
    n_side = mesh // 4
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(float(mesh), mesh, n_side, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation.from_zeldovich(cc, float(mesh), mesh, n_side, 0.96, 0.8, 0.02, 11, split,
                                        flags=cpm._native.SIM_NO_AUTOTUNE)
    st = sim.state()
    accs = {}
    for plan in (8, 0):
        sim.set_tuning(plan, 1024, 4)
        sim.set_state(st["x"], st["p"])
        accs[plan] = sim.state()["acc"]
    assert rel_rms(accs[0], accs[8]) < 4e-6
    sim.close()
