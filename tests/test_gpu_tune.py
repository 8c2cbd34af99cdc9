"""Launch tuning. The walk grid and the sort tile give bit-identical results at
every value. The walk group size (4, 8, 16 or 32 particles per warp) and the
walk split (1, 2, 4 or 8 parts per work item) make each particle take exactly
the same acceptance decisions (identical interaction counts, identical own
leaves) and change only the order of its force sums: forces stay within the
tolerance of the FP64 walk at every setting. The autotuner leaves a valid,
timed choice set on the context."""
import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.autotune import autotune, get, launch_setting, set_
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.pool import GalaxyPool
from galaxy_sim_b200.simulation import Physics, params_dict

pytestmark = pytest.mark.gpu


def _run(g, ph, bps, items, steps=3):
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(**params_dict(g, ph))
    if bps is not None:
        set_(sim._ctx, _lib.TUNE_WALK_BLOCKS_PER_SM, bps)
        set_(sim._ctx, _lib.TUNE_SORT_ITEMS, items)
    sim.run(steps, True)
    P, S = sim.readState()
    e = sim.energy()
    sim.destroy()
    return P, S, e


def test_knobs_do_not_change_results(gpu_lib):
    g = ic.galaxy_disk(20000, 5, Q=1.2, arms=4, gas_frac=0.3)
    ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.02)
    P0, S0, e0 = _run(g, ph, None, None)
    for bps, items in ((1, 8), (4, 16), (8, 8), (7, 4)):
        P, S, e = _run(g, ph, bps, items)
        assert np.array_equal(P.view(np.uint32), P0.view(np.uint32)), (bps, items)
        assert np.array_equal(S.view(np.uint32), S0.view(np.uint32)), (bps, items)
        assert e == e0, (bps, items)


def test_bad_knobs_rejected(gpu_lib):
    g = ic.galaxy_disk(1000, 6)
    sim = NBodyGPU(0, g.particles, g.stellar)
    with pytest.raises(_lib.GalaxyError):
        set_(sim._ctx, _lib.TUNE_SORT_ITEMS, 12)
    with pytest.raises(_lib.GalaxyError):
        set_(sim._ctx, _lib.TUNE_WALK_BLOCKS_PER_SM, 0)
    with pytest.raises(_lib.GalaxyError):
        set_(sim._ctx, _lib.TUNE_WALK_GROUP, 12)
    with pytest.raises(_lib.GalaxyError):
        set_(sim._ctx, _lib.TUNE_WALK_SPLIT, 3)
    with pytest.raises(_lib.GalaxyError):
        set_(sim._ctx, 99, 1)
    sim.destroy()


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)


# (group, split); groups of 32 walk unsplit whatever the split knob says
SETTINGS = [(32, 1), (16, 1), (8, 1), (4, 1), (0, 0), (32, 4), (16, 2), (8, 4), (4, 8), (8, 8), (16, 8), (4, 2)]


@pytest.mark.parametrize("n,eps", [(20000, 0.02), (3000, 0.05), (70001, 0.02), (300, 0.05)])
def test_walk_group_sizes_and_splits_agree(gpu_lib, oracle, n, eps):
    g = ic.galaxy_disk(n, 9, Q=1.2, arms=4, gas_frac=0.3)
    out = {}
    for wg, split in SETTINGS:
        sim = NBodyGPU(0, g.particles, g.stellar)
        sim.updateParams(dt=0.005, G=1.0, epsilon=eps, theta=0.5)
        set_(sim._ctx, _lib.TUNE_WALK_GROUP, wg)
        set_(sim._ctx, _lib.TUNE_WALK_SPLIT, split)
        assert get(sim._ctx, _lib.TUNE_WALK_GROUP) == wg and get(sim._ctx, _lib.TUNE_WALK_SPLIT) == split
        sim.setDebug(True)
        sim.sortBuild()
        nodes, lr, _ = sim.getTree()
        P, _ = sim.readState()
        sim.counters(reset=True)
        sim.step()
        acc, dens = sim.readForces()
        out[wg, split] = (acc, dens, sim.counters(), P, nodes, lr)
        assert sim.deviceErrors() == 0
        sim.destroy()
    ref = out[32, 1]
    P, nodes, lr = ref[3], ref[4], ref[5]
    com64 = oracle.refresh_f64(P, nodes, lr)
    p = oracle.make_params(n, epsilon=eps, theta=0.5, dt=0.005)
    acc64, pot64, dens64, cnt = oracle.walk_f64(p, P, nodes, com64)
    for key, (acc, dens, cnt_dev, _, _, _) in out.items():
        rel = _rel(acc[:, :3].astype(np.float64), acc64)
        assert np.median(rel) <= 2e-5 and np.percentile(rel, 99) <= 1e-3, (key, np.median(rel))
        assert np.median(np.abs(acc[:, 3] - pot64) / np.abs(pot64)) <= 2e-5, key
        assert cnt_dev == ref[2], (key, cnt_dev, ref[2])      # the same decisions
        assert np.array_equal(dens, ref[1]), key              # the same own leaves
        # the sums differ only by rounding
        d = _rel(acc[:, :3].astype(np.float64), ref[0][:, :3].astype(np.float64))
        assert np.median(d) < 1e-6 and np.percentile(d, 99) < 1e-4, (key, np.median(d), np.percentile(d, 99))


def test_split_walk_results_repeat(gpu_lib):
    """A split walk's last part adds the parts' sums in part order, whichever
    part finishes last: the same run twice gives the same bits."""
    g = ic.galaxy_disk(16384, 4, Q=1.5, arms=2)
    runs = []
    for _ in range(2):
        sim = NBodyGPU(0, g.particles, g.stellar, walkGroup=8, walkSplit=8)
        sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
        sim.run(20, False)
        runs.append((sim.readState()[0], sim.energy()))
        assert sim.deviceErrors() == 0
        sim.destroy()
    assert np.array_equal(runs[0][0].view(np.uint32), runs[1][0].view(np.uint32))
    assert runs[0][1] == runs[1][1]


@pytest.mark.parametrize("wg,split", [(32, 1), (8, 4)])
def test_zero_softening_forces_are_finite_and_match_fp64(gpu_lib, oracle, wg, split):
    """epsilon = 0: a particle alone in its leaf sits at the leaf's centre of
    mass (r = 0); the walk opens that leaf and skips the self pair, as the
    reference does, instead of weighing an infinite monopole by zero."""
    g = ic.galaxy_disk(3000, 11)
    sim = NBodyGPU(0, g.particles, g.stellar, walkGroup=wg, walkSplit=split)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.0, theta=0.5)
    sim.setDebug(True)
    sim.sortBuild()
    nodes, lr, _ = sim.getTree()
    P, _ = sim.readState()
    sim.step()
    acc, dens = sim.readForces()
    sim.destroy()
    single = nodes["isLeaf"].astype(bool) & (nodes["count"] == 1)
    assert single.any()                                   # the case arises in this galaxy
    assert np.isfinite(acc).all()
    com64 = oracle.refresh_f64(P, nodes, lr)
    p = oracle.make_params(g.N, epsilon=0.0, theta=0.5, dt=0.005)
    acc64, pot64, dens64, _ = oracle.walk_f64(p, P, nodes, com64)
    rel = _rel(acc[:, :3].astype(np.float64), acc64)
    assert np.median(rel) <= 2e-5 and np.percentile(rel, 99) <= 1e-3, (np.median(rel), np.percentile(rel, 99))
    assert np.median(np.abs(acc[:, 3] - pot64) / np.abs(pot64)) <= 2e-5


def test_autotune_pool(gpu_lib):
    pool = GalaxyPool(40000, 4)
    for k, n in enumerate((3000, 9000, 20000)):
        g = ic.galaxy_disk(n, 20 + k)
        pool.add(g.particles, g.stellar, params_dict(g, Physics(0.05, 0.5, 0.005)))
    res = autotune(pool, steps=2, warmup=1, walk_blocks=(4, 8), sort_items=(8, 16))
    ch = res["choice"]
    assert len(res["ms"]) == 9 and all(t > 0 for t in res["ms"].values())
    assert get(pool._ctx, _lib.TUNE_WALK_GROUP) == (0 if ch["walk_group"] == "by galaxy size" else ch["walk_group"])
    assert get(pool._ctx, _lib.TUNE_WALK_BLOCKS_PER_SM) == ch["walk_blocks_per_sm"]
    assert get(pool._ctx, _lib.TUNE_SORT_ITEMS) == ch["sort_keys_per_thread"]
    assert ch["walk_split"] == "unsplit (several galaxies)"
    pool.run(2, True)
    assert all(pool.device_errors(s) == 0 for s in pool.n)
    pool.close()


def test_autotune_single_galaxy_tunes_the_split(gpu_lib):
    g = ic.galaxy_disk(16384, 21)
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    res = autotune(sim, steps=2, warmup=1, walk_groups=(0, 8), walk_blocks=(7,), sort_items=(16,))
    ch = res["choice"]
    assert len(res["ms"]) == 8 and all(t > 0 for t in res["ms"].values())
    assert get(sim._ctx, _lib.TUNE_WALK_SPLIT) == (0 if ch["walk_split"] == "by galaxy size" else ch["walk_split"])
    eff = launch_setting(sim._ctx)
    assert eff["walk_group"] == 8 and eff["sort_keys_per_thread"] == 16
    assert eff["walk_split"] == (2 if ch["walk_split"] == "by galaxy size" else ch["walk_split"])
    sim.run(2, False)
    assert sim.deviceErrors() == 0
    sim.destroy()


def test_launch_setting_follows_the_size_rules(gpu_lib):
    """The by-size rules of a single-galaxy context, as the library applies them."""
    for n, want in ((4096, (8, 4, 4)), (16384, (8, 2, 4)), (60000, (16, 1, 4)), (200000, (32, 1, 8)),
                    (600000, (32, 1, 16))):
        g = ic.galaxy_disk(n, 30)
        sim = NBodyGPU(0, g.particles, g.stellar)
        eff = launch_setting(sim._ctx)
        assert (eff["walk_group"], eff["walk_split"], eff["sort_keys_per_thread"]) == want, (n, eff)
        set_(sim._ctx, _lib.TUNE_WALK_GROUP, 32)
        set_(sim._ctx, _lib.TUNE_WALK_SPLIT, 4)      # groups of 32 walk unsplit
        assert launch_setting(sim._ctx)["walk_split"] == 1
        sim.destroy()
    pool = GalaxyPool(20000, 2)
    pool._sel(pool.add(ic.galaxy_disk(3000, 31).particles))
    eff = launch_setting(pool._ctx)
    assert eff == {"walk_group": 32, "walk_split": 1, "sort_keys_per_thread": 16}, eff
    pool.close()
