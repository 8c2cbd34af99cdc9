"""Seeded initial conditions (src/physics/InitialConditions.js algorithm)."""
import numpy as np

from galaxy_sim_b200 import initial_conditions as ic


def test_disk16k_reproducible_and_shaped():
    a, b = ic.disk_16k(), ic.disk_16k()
    assert np.array_equal(a.particles, b.particles) and np.array_equal(a.stellar, b.stellar)
    P = a.particles
    assert P.shape == (16384, 8) and P.dtype == np.float32
    assert abs(P[:, 3].astype(np.float64).sum() - 1.0) < 1e-5      # masses rescaled to 1
    r = np.hypot(P[:, 0], P[:, 1])
    assert r.max() <= 6.0 + 1e-5                                   # truncated at 6 Rd
    assert np.all(P[:, 7] == 0)                                    # no gas
    assert abs(a.halo_mass - 5 * 0.85) < 0.05                      # halo = 5 x disk mass
    assert np.all(np.isfinite(P))


def test_disk512k_gas_fraction():
    g = ic.disk_512k(N=65536)
    gas = g.particles[:, 7] < -0.5
    disk = np.arange(g.N) >= int(g.N * 0.15)
    frac = gas[disk].mean()
    assert 0.27 < frac < 0.33
    assert np.all(g.stellar[gas, 0] == -1)


def test_collision_two_black_holes():
    g = ic.two_galaxy_collision(8192, 3)
    assert g.central == (0, 4096)
    assert abs(g.particles[0, 3] - 0.01) < 1e-7 and abs(g.particles[4096, 3] - 0.01) < 1e-7
    sep = np.linalg.norm(g.particles[4096, :3] - g.particles[0, :3])
    assert abs(sep - 30.0) < 0.5
    assert len(g.halo_centers) == 2


def test_sphere():
    g = ic.hernquist_sphere(4096, 5)
    assert np.all(g.particles[:, 4:7] == 0)
    assert np.linalg.norm(g.particles[:, :3], axis=1).max() <= 20.0 + 1e-4
