"""Batches: many galaxies stepped by one set of launches (segmented sort, build,
walk) must give every galaxy exactly its solo result.

Each galaxy of the pool sits at its own particle offset with its own Params,
Morton frame, tree, clock and tracked centres; the kernels see tiles and walk
groups that never cross galaxies, so positions, velocities, stellar records,
trees and FP64 diagnostics are bit-identical to a solo context's. Galaxies are
admitted into holes left by released ones (continuous batching) with the same
guarantee.
"""
import numpy as np
import pytest

from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.pool import GalaxyPool, pool_bytes
from galaxy_sim_b200.simulation import Physics, params_dict

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    g = ic.galaxy_disk(5000, 11, Q=1.2, arms=4, gas_frac=0.3)
    g.sf_density *= 0.2
    out.append((g, Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.5)))
    out.append((ic.galaxy_disk(16384, 12, Q=1.5, arms=2), Physics(0.05, 0.7, 0.0025)))
    out.append((ic.hernquist_sphere(33, 13), Physics(0.05, 0.5, 0.005)))
    out.append((ic.two_galaxy_collision(4000, 14, Q=1.5, arms=2), Physics(0.02, 0.5, 0.005)))
    out.append((ic.galaxy_disk(1, 15), Physics(0.02, 0.5, 0.005)))
    return out


def _tracking(g):
    c1, c2 = g.central
    if c1 < 0 and c2 < 0:
        return None
    hc = g.halo_centers
    return (c1, c2, hc[0] if len(hc) > 0 else None, hc[1] if len(hc) > 1 else None)


def _solo(g, ph, steps, sf, walk_group=32, walk_split=1):
    sim = NBodyGPU(0, g.particles, g.stellar, walkGroup=walk_group, walkSplit=walk_split)  # the pool's setting
    sim.updateParams(**params_dict(g, ph))
    t = _tracking(g)
    if t is not None:
        sim.setTracking(*t)
    sim.run(steps, sf)
    P, S = sim.readState()
    e = sim.energy()
    tr = sim.getTracking()
    sim.destroy()
    return P, S, e, tr


def _check_same(pool, slot, solo):
    P, S = pool.read_state(slot)
    SP, SS, se, st = solo
    assert np.array_equal(P.view(np.uint32), SP.view(np.uint32))
    assert np.array_equal(S.view(np.uint32), SS.view(np.uint32))
    e = pool.energy(slot)
    assert e["e_diag"] == se["e_diag"] and e["e_true"] == se["e_true"]
    assert e["momentum"] == se["momentum"] and e["mass"] == se["mass"]
    tr = pool.get_tracking(slot)
    assert tr[0] == st[0] and tr[1] == st[1]
    assert np.array_equal(tr[2], st[2]) and np.array_equal(tr[3], st[3])
    assert pool.device_errors(slot) == 0


def test_batch_equals_solo_runs(gpu_lib):
    cases = _cases()
    steps = 3
    solos = [_solo(g, ph, steps, True) for g, ph in cases]
    cap = sum(g.N + 256 for g, _ in cases) + 4096
    pool = GalaxyPool(cap, 8)
    slots = [pool.add(g.particles, g.stellar, params_dict(g, ph), _tracking(g)) for g, ph in cases]
    assert None not in slots
    pool.run(steps, True)
    for s, solo in zip(slots, solos):
        _check_same(pool, s, solo)
    E = pool.energies()
    for s, solo in zip(slots, solos):
        assert E[s, 0] == solo[2]["e_diag"]
    pool.close()


def test_batch_equals_solo_with_walk_groups_by_size(gpu_lib):
    """With the walk group chosen by each galaxy's size (8, 16 or 32 particles
    per warp, one walk launch per size class in the pool), every galaxy still
    equals its solo run with the same setting, bit for bit."""
    from galaxy_sim_b200 import _lib

    cases = _cases() + [(ic.galaxy_disk(90000, 16, gas_frac=0.3), Physics(0.02, 0.5, 0.005, gas_drag=0.25,
                                                                        sf_eff=0.02)),
                        (ic.galaxy_disk(160000, 17), Physics(0.02, 0.7, 0.005))]
    steps = 2
    solos = [_solo(g, ph, steps, True, walk_group=0) for g, ph in cases]
    pool = GalaxyPool(sum(g.N + 256 for g, _ in cases) + 4096, 8)
    _lib.check(_lib.lib().gs_set_tuning(pool._ctx, _lib.TUNE_WALK_GROUP, 0), pool._ctx)
    slots = [pool.add(g.particles, g.stellar, params_dict(g, ph), _tracking(g)) for g, ph in cases]
    pool.run(steps, True)
    for s, solo in zip(slots, solos):
        _check_same(pool, s, solo)
    pool.close()


def test_walk_split_applies_to_a_lone_galaxy_only(gpu_lib):
    """The split knob splits the walk of a pool holding one galaxy (the same bits
    as a solo run with that split); a pool of several galaxies walks unsplit
    whatever the knob says (the same bits as unsplit solo runs)."""
    from galaxy_sim_b200 import _lib

    cases = _cases()[:2]
    steps = 2
    pool = GalaxyPool(sum(g.N + 256 for g, _ in cases) + 4096, 4)
    _lib.check(_lib.lib().gs_set_tuning(pool._ctx, _lib.TUNE_WALK_GROUP, 8), pool._ctx)
    _lib.check(_lib.lib().gs_set_tuning(pool._ctx, _lib.TUNE_WALK_SPLIT, 4), pool._ctx)
    g, ph = cases[1]
    s1 = pool.add(g.particles, g.stellar, params_dict(g, ph), _tracking(g))
    pool.run(steps, True)
    split = _solo(g, ph, steps, True, walk_group=8, walk_split=4)
    unsplit = _solo(g, ph, steps, True, walk_group=8, walk_split=1)
    assert not np.array_equal(split[0].view(np.uint32), unsplit[0].view(np.uint32))  # the split was taken
    _check_same(pool, s1, split)
    pool.remove(s1)
    slots = [pool.add(g.particles, g.stellar, params_dict(g, ph), _tracking(g)) for g, ph in cases]
    pool.run(steps, True)
    for s, (g, ph) in zip(slots, cases):
        _check_same(pool, s, _solo(g, ph, steps, True, walk_group=8, walk_split=1))
    pool.close()


def test_admission_into_holes_keeps_results(gpu_lib):
    """Release a galaxy mid-run, admit a new one into its hole: the others
    continue exactly as alone, and the newcomer runs exactly as alone."""
    cases = _cases()
    (g0, p0), (g1, p1), (g2, p2), (g3, p3), _ = cases
    k1, k2 = 2, 3
    cap = g0.N + g1.N + g2.N + 3 * 256 + 256
    pool = GalaxyPool(cap, 4)
    s0 = pool.add(g0.particles, g0.stellar, params_dict(g0, p0))
    s1 = pool.add(g1.particles, g1.stellar, params_dict(g1, p1))
    s2 = pool.add(g2.particles, g2.stellar, params_dict(g2, p2))
    # the pool is full for the collision galaxy until one is released
    assert pool.add(g3.particles, g3.stellar, params_dict(g3, p3), _tracking(g3)) is None
    pool.run(k1, True)
    pool.remove(s1)
    s3 = pool.add(g3.particles, g3.stellar, params_dict(g3, p3), _tracking(g3))
    assert s3 is not None
    pool.run(k2, True)
    _check_same(pool, s0, _solo(g0, p0, k1 + k2, True))
    _check_same(pool, s2, _solo(g2, p2, k1 + k2, True))
    _check_same(pool, s3, _solo(g3, p3, k2, True))
    pool.close()


def test_star_formation_switch_per_galaxy(gpu_lib):
    """A galaxy admitted with star formation off stays exactly its run without
    star formation while a neighbour forms stars in the same steps."""
    (g0, p0), _, _, (g3, p3), _ = _cases()
    pool = GalaxyPool(g0.N + g3.N + 512, 2)
    a = pool.add(g0.particles, g0.stellar, params_dict(g0, p0))
    b = pool.add(g3.particles, g3.stellar, params_dict(g3, p3), _tracking(g3), star_formation=False)
    pool.run(3, True)
    _check_same(pool, a, _solo(g0, p0, 3, True))
    _check_same(pool, b, _solo(g3, p3, 3, False))
    pool.close()


def test_pool_accounting(gpu_lib):
    assert pool_bytes(1 << 20, 16) > pool_bytes(1 << 19, 16) > 0
    pool = GalaxyPool(10000, 2)
    r, s = pool.free()
    assert r == 10000 and s == 2
    g = ic.galaxy_disk(3000, 1)
    a = pool.add(g.particles, g.stellar, params_dict(g, Physics(0.05, 0.5, 0.005)))
    r, s = pool.free()
    assert s == 1 and r == 10000 - 3072
    b = pool.add(g.particles, g.stellar, params_dict(g, Physics(0.05, 0.5, 0.005)))
    assert pool.add(g.particles, g.stellar) is None  # no slot left
    pool.remove(a)
    pool.remove(b)
    assert pool.free() == (10000, 2)
    pool.close()


@pytest.mark.parametrize("comp,com64", [(True, False), (False, True), (True, True)],
                         ids=["compensated", "com64", "both"])
def test_batch_equals_solo_in_precision_modes(gpu_lib, comp, com64):
    """The precision variants (Kahan-compensated far-field sums in the walk, FP64
    internal-node COM) keep the batch guarantee: each galaxy equals its solo run
    in the same mode, bit for bit."""
    from galaxy_sim_b200 import _lib

    cases = _cases()[:4]
    steps = 2
    solos = []
    for g, ph in cases:
        sim = NBodyGPU(0, g.particles, g.stellar, walkGroup=32, walkSplit=1)   # the pool's walk group
        sim.updateParams(**params_dict(g, ph))
        t = _tracking(g)
        if t is not None:
            sim.setTracking(*t)
        sim.setWalkMode(comp)
        sim.setComMode(2 if com64 else 0)
        sim.run(steps, True)
        P, S = sim.readState()
        solos.append((P, S, sim.energy(), sim.getTracking()))
        sim.destroy()
    pool = GalaxyPool(sum(g.N + 256 for g, _ in cases) + 4096, 8)
    _lib.check(_lib.lib().gs_set_walk_mode(pool._ctx, int(comp)), pool._ctx)
    _lib.check(_lib.lib().gs_set_com_mode(pool._ctx, 2 if com64 else 0), pool._ctx)
    slots = [pool.add(g.particles, g.stellar, params_dict(g, ph), _tracking(g)) for g, ph in cases]
    pool.run(steps, True)
    for s, solo in zip(slots, solos):
        _check_same(pool, s, solo)
    pool.close()
