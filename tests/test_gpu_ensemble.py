"""The ensemble of realisations (cpm_ensemble_*) through the C ABI: every box of a mixed batch
against its own single-box simulation (cpm_sim_create_zeldovich with the same seed), after steps
that replay the ensemble's captured graph.

A batch's particles share one sort (the box index above 19 octant digits instead of 21), one tree
(a root per box) and FP64 prefix sums over the whole batch for the centres of mass, whose last f32
bit can round differently from a single box's; deposit, FFT, gather and kick/drift are per box the
same arithmetic. So the initial conditions must be equal, the initial forces within 1e-6 relative RMS; after 40 steps
(the last ones replayed from the ensemble's graph, where the chaotic growth of last-bit differences
shows) positions within 1e-5 L, forces within 1e-4 relative RMS and the boxes' P(k) within 1e-4.
Both sides keep the default launch choices (no autotuning): the autotuner picks an FFT plan per
workload by timing, and two plans round differently, which the 40 chaotic steps would amplify."""
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


def test_every_box_of_a_mixed_ensemble_equals_its_single_run(cpm):
    box = 64.0
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    classes = []
    for n_side, mesh, boxes, seed in [(16, 32, 3, 100), (32, 64, 2, 200), (48, 96, 2, 300)]:
        split = cpm.ForceSplit.with_(box, mesh, n_side, 1.0 / 30.0, 0.5)
        classes.append((n_side, mesh, boxes, seed, split))
    fixed = cpm._native.SIM_NO_AUTOTUNE
    ens = cpm.Ensemble(cc, box, 0.96, 0.8, 0.02, classes, flags=fixed)
    # the forces of the initial conditions: every box against its own single-box simulation
    for ci, (n_side, mesh, boxes, seed, split) in enumerate(classes):
        for b in range(boxes):
            single = cpm.Simulation.from_zeldovich(cc, box, mesh, n_side, 0.96, 0.8, 0.02, seed + b, split,
                                                    flags=fixed)
            s, e = single.state(), ens.state(ci, b)
            assert np.array_equal(e["x"], s["x"]) and np.array_equal(e["p"], s["p"]), (ci, b)
            assert rel_rms(e["acc"], s["acc"]) < 1e-6, (ci, b)
            single.close()
    sched = cpm.ln_a_schedule(0.02, 1.0, 64)[:40]
    for a1 in sched:
        ens.step_to(a1)
    assert ens.graphs() == 2
    for ci, (n_side, mesh, boxes, seed, split) in enumerate(classes):
        for b in range(boxes):
            single = cpm.Simulation.from_zeldovich(cc, box, mesh, n_side, 0.96, 0.8, 0.02, seed + b, split,
                                                    flags=fixed)
            for a1 in sched:
                single.step_to(a1)
            s, e = single.state(), ens.state(ci, b)
            assert periodic_max_diff(e["x"], s["x"], box) < 1e-5 * box, (ci, b)
            assert rel_rms(e["acc"], s["acc"]) < 1e-4, (ci, b)
            _, p_s, c_s = single.power_spectrum(mesh // 4)
            _, p_e, c_e = ens.power_spectrum(ci, b, mesh // 4)
            np.testing.assert_array_equal(c_s, c_e)
            assert np.max(np.abs(p_e / p_s - 1.0)) < 1e-4, (ci, b)
            single.close()
    ens.close()


def test_ensemble_rejects_bad_classes(cpm):
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    split = cpm.ForceSplit.with_(64.0, 32, 12, 1.0 / 30.0, 0.5)
    with pytest.raises(cpm.CpmError) as e:
        cpm.Ensemble(cc, 64.0, 0.96, 0.8, 0.02, [(12, 32, 2, 0, split)])  # 12^3 not a multiple of 2048
    assert e.value.code == -1
