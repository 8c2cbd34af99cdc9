"""Pools beyond gs_run: galaxy sizes at every tile edge, and the NBodyGPU surface
(applyPermutation, uploadBHTree + encodeRefresh + step, getTree) on a slot that
does not sit at the start of the pool. Each must equal the same call sequence on
a single-galaxy context."""
import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200 import morton_tree as mt
from galaxy_sim_b200.autotune import set_
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.pool import GalaxyPool
from galaxy_sim_b200.simulation import Physics, params_dict

pytestmark = pytest.mark.gpu

# walk groups are 32 particles, build tiles 1024, sort tiles 2048 or 4096 keys
EDGE_SIZES = (1, 16, 17, 31, 32, 33, 1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096, 4097, 8193)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def _solo_run(g, kw, steps):
    sim = NBodyGPU(0, g.particles, g.stellar, walkGroup=32, walkSplit=1)
    sim.updateParams(**kw)
    sim.run(steps, True)
    P, S = sim.readState()
    e = sim.energy()
    sim.destroy()
    return P, S, e


@pytest.mark.parametrize("sort_items", [16, 8, 4])
def test_tile_edge_sizes_equal_solo(gpu_lib, sort_items):
    gals = [ic.galaxy_disk(n, 100 + k, gas_frac=0.3 if k % 2 else 0.0) for k, n in enumerate(EDGE_SIZES)]
    kws = [params_dict(g, Physics((0.02, 0.05)[k % 2], (0.5, 0.7)[k % 3 == 0], 0.005, gas_drag=0.25,
                                  sf_eff=0.02)) for k, g in enumerate(gals)]
    pool = GalaxyPool(sum(g.N + 256 for g in gals), len(gals))
    set_(pool._ctx, _lib.TUNE_SORT_ITEMS, sort_items)
    slots = [pool.add(g.particles, g.stellar, kw) for g, kw in zip(gals, kws)]
    pool.run(2, True)
    for g, kw, s in zip(gals, kws, slots):
        P, S, e = _solo_run(g, kw, 2)
        RP, RS = pool.read_state(s)
        assert _same(RP, P) and _same(RS, S), g.N
        assert pool.energy(s) == e, g.N
        assert pool.device_errors(s) == 0, g.N
    pool.close()


def test_apply_permutation_on_a_pool_slot(gpu_lib):
    a, b = ic.galaxy_disk(3000, 1), ic.galaxy_disk(5000, 2, gas_frac=0.3)
    pool = GalaxyPool(a.N + b.N + 512, 2)
    sa = pool.add(a.particles, a.stellar)
    sb = pool.add(b.particles, b.stellar)
    perm = np.random.default_rng(0).permutation(b.N).astype(np.uint32)
    pool.apply_permutation(sb, perm)   # the other galaxy shares the buffers: copy-back path
    P, S = pool.read_state(sb)
    assert _same(P, b.particles[perm]) and _same(S, b.stellar[perm])
    P, S = pool.read_state(sa)
    assert _same(P, a.particles) and _same(S, a.stellar)
    pool.close()


def test_reference_flow_on_a_pool_slot(gpu_lib):
    """main.js's flow (sortAndBuild -> uploadBHTree -> updateParams -> encodeRefresh
    -> step) on the second galaxy of a pool equals it on its own context."""
    other, g = ic.galaxy_disk(2500, 3), ic.disk_16k()
    boot = mt.sortAndBuild(g.particles.ravel(), g.stellar.ravel(), g.N)
    tree = boot["tree"]
    kw = dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5, haloMass=g.halo_mass, haloA=g.halo_a,
              haloCenters=[[0, 0, 0, 0]])
    sim = NBodyGPU(0, boot["sorted"], boot["sortedStellar"], walkGroup=32, walkSplit=1)
    sim.uploadBHTree(tree.nodes, tree.numNodes, tree.levelRanges)
    sim.updateParams(**kw)
    sim.encodeRefresh()
    sim.step()
    want, _ = sim.readState()
    sim.destroy()
    pool = GalaxyPool(other.N + g.N + 512, 2)
    so = pool.add(other.particles, other.stellar, kw)
    sg = pool.add(boot["sorted"], boot["sortedStellar"], kw)
    pool.upload_tree(sg, tree.nodes, tree.numNodes, tree.levelRanges)
    pool.refresh()
    pool.step()
    got, _ = pool.read_state(sg)
    assert _same(got, want)
    assert pool.device_errors(sg) == 0 and pool.device_errors(so) == 0
    # the uploaded tree reads back with the refreshed COM and galaxy-local indices
    nodes, lr, _ = pool.get_tree(sg, want_perm=False)
    assert np.array_equal(nodes["children"], tree.nodes["children"])
    assert np.array_equal(nodes["first"], tree.nodes["first"])
    pool.close()


def test_get_tree_on_a_pool_slot(gpu_lib):
    a, b = ic.galaxy_disk(3000, 4), ic.galaxy_disk(20000, 5)
    sim = NBodyGPU(0, b.particles, b.stellar, walkGroup=32, walkSplit=1)
    sim.sortBuild()
    want_nodes, want_lr, want_perm = sim.getTree()
    sim.destroy()
    pool = GalaxyPool(a.N + b.N + 512, 2)
    pool.add(a.particles, a.stellar)
    sb = pool.add(b.particles, b.stellar)
    pool.sort_build()
    nodes, lr, perm = pool.get_tree(sb)
    assert np.array_equal(perm, want_perm)
    assert np.array_equal(lr, want_lr)
    assert np.array_equal(nodes.view(np.uint8), want_nodes.view(np.uint8))
    pool.close()


def test_readmitted_pool_equals_a_fresh_pool(gpu_lib):
    """bench.py times its pool from the seeded initial conditions after tuning it:
    every galaxy removed, then admitted again in the same order. That must give
    the same slots and the same results as a fresh pool."""
    gals = []
    for k, (n, gas) in enumerate(((3000, 0.3), (7000, 0.0), (1500, 0.3))):
        g = ic.galaxy_disk(n, 50 + k, gas_frac=gas)
        ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25 if gas else 0.0, sf_eff=0.05 if gas else 0.0)
        gals.append((g, ph))
    cap = sum((g.N + 255) // 256 * 256 for g, _ in gals)

    def admit(pool):
        return [pool.add(g.particles, g.stellar, params_dict(g, ph), star_formation=ph.sf_eff > 0)
                for g, ph in gals]

    fresh = GalaxyPool(cap, len(gals))
    want_slots = admit(fresh)
    fresh.run(3, True)
    want = [fresh.read_state(s) for s in want_slots]
    want_e = fresh.energies()
    fresh.close()

    pool = GalaxyPool(cap, len(gals))
    admit(pool)
    pool.run(6, True)
    for s in list(pool.n):
        pool.remove(s)
    slots = admit(pool)
    assert slots == want_slots
    pool.run(3, True)
    for s, (wp, ws) in zip(slots, want):
        gp, gs = pool.read_state(s)
        assert _same(gp, wp) and _same(gs, ws), s
    assert np.array_equal(pool.energies(), want_e)
    pool.close()
