"""The viewer snapshot (runner.rs:263-284, frame.rs) on the device: the reference's frame.rs tests
and bit-exact agreement with its f32 arithmetic on a simulation's state."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_small_grids_keep_every_cell_and_transpose(cpm):
    """frame.rs:75-81"""
    mesh = cpm.Mesh(4, 10.0)
    mesh.cells[(1 * 4 + 2) * 4 + 3] = 5.0
    g = cpm.density_grid(mesh)
    assert g.shape == (4, 4, 4)
    assert g[3, 2, 1] == 6.0  # texture order: x = 1, y = 2, z = 3
    assert int((g == 1.0).sum()) == 63


def test_large_grids_average_blocks(cpm):
    """frame.rs:84-93"""
    mesh = cpm.Mesh(200, 100.0)
    mesh.cells[0] = 8.0
    g = cpm.density_grid(mesh)
    assert g.shape == (100, 100, 100)
    assert abs(g[0, 0, 0] - 2.0) < 1e-6
    assert abs(g[0, 0, 1] - 1.0) < 1e-6


def test_rsd_shift_is_velocity_over_a_h(cpm):
    """frame.rs:95-100 through a simulation: a = 0.5 and E = 2 (Omega_m = 0.5, nothing else), p = (1, 0, 0)."""
    cc = cpm.Cosmology(0.0, 0.5, 0.0, 70.0)
    x = np.array([[5.0, 5.0, 5.0]], np.float32)
    p = np.array([[1.0, 0.0, 0.0]], np.float32)
    sim = cpm.Simulation(cc, 10.0, 4, x, p, 0.5, None)
    snap = sim.snapshot()
    assert abs(snap["rsd"][0, 0] - 2.0) < 1e-6 and snap["rsd"][0, 1] == 0.0 and snap["rsd"][0, 2] == 0.0
    assert snap["speeds"][0] == np.float32(2.0) and snap["max_speed"] == np.float32(2.0)


def _downsample_f32(delta, n):
    """frame.rs:35-55 with f32 sums in the reference's loop order."""
    f = max(1, -(-n // 128))
    m = n // f
    cells = delta.reshape(n, n, n)
    s = np.zeros((m, m, m), np.float32)  # indexed [x, y, z]
    for dx in range(f):
        for dy in range(f):
            for dz in range(f):
                s = (s + cells[dx:m * f:f, dy:m * f:f, dz:m * f:f]).astype(np.float32)
    norm = np.float32(1.0) / np.float32(f * f * f)
    return (np.float32(1.0) + s * norm).astype(np.float32).transpose(2, 1, 0)  # -> [z, y, x]


@pytest.mark.parametrize("mesh", [32, 256])
def test_snapshot_matches_reference_arithmetic(cpm, orc, mesh):
    cc = cpm.Cosmology(0.0, 0.3, 0.7, 70.0)
    box = 32.0
    split = cpm.ForceSplit.with_(box, mesh, 16, 1.0 / 30.0, 0.5)
    sim = cpm.Simulation.from_zeldovich(cc, box, mesh, 16, 0.96, 0.8, 0.02, 3, split)
    for a1 in cpm.ln_a_schedule(0.02, 0.2, 5):
        sim.step_to(a1)
    snap = sim.snapshot(want_grid=True)
    st = sim.state(want_delta=True)
    a = np.float32(st["a"])
    p = st["p"]
    speeds = (np.sqrt((p[:, 0] * p[:, 0] + p[:, 1] * p[:, 1]) + p[:, 2] * p[:, 2]) / a).astype(np.float32)
    assert np.array_equal(snap["speeds"], speeds)
    assert snap["max_speed"] == speeds.max()
    e = np.float32(orc.cosmo_e(orc.cosmology(0.0, 0.3, 0.7, 70.0), float(a)))
    s = np.float32(1.0) / (a * a * e)
    assert np.array_equal(snap["rsd"], (p * s).astype(np.float32))
    dens = np.maximum(np.float32(1.0) + orc.interpolate_many(mesh, box, st["delta"], st["x"]).astype(np.float32),
                      np.float32(0.0))
    assert np.array_equal(snap["densities"], dens)
    assert np.array_equal(snap["grid"], _downsample_f32(st["delta"], mesh))
    assert snap["redshift"] == np.float32(1.0) / a - np.float32(1.0)
