"""Launch tuning. The walk grid and the sort tile give bit-identical results at
every value. The walk group size (8, 16 or 32 particles per warp) makes each
particle take exactly the same acceptance decisions (identical interaction
counts) and changes only the order of its force sums: forces stay within the
tolerance of the FP64 walk at every size. The autotuner leaves a valid, timed
choice set on the context."""
import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.autotune import autotune, get, set_
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
    for bps, items in ((1, 8), (4, 16), (8, 8)):
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
    sim.destroy()


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)


@pytest.mark.parametrize("n,eps", [(20000, 0.02), (3000, 0.05), (70001, 0.02)])
def test_walk_group_sizes_agree(gpu_lib, oracle, n, eps):
    g = ic.galaxy_disk(n, 9, Q=1.2, arms=4, gas_frac=0.3)
    out = {}
    for wg in (32, 16, 8, 4, 0):
        sim = NBodyGPU(0, g.particles, g.stellar)
        sim.updateParams(dt=0.005, G=1.0, epsilon=eps, theta=0.5)
        set_(sim._ctx, _lib.TUNE_WALK_GROUP, wg)
        assert get(sim._ctx, _lib.TUNE_WALK_GROUP) == wg
        sim.setDebug(True)
        sim.sortBuild()
        nodes, lr, _ = sim.getTree()
        P, _ = sim.readState()
        sim.counters(reset=True)
        sim.step()
        acc, dens = sim.readForces()
        out[wg] = (acc, dens, sim.counters(), P, nodes, lr)
        assert sim.deviceErrors() == 0
        sim.destroy()
    P, nodes, lr = out[32][3], out[32][4], out[32][5]
    com64 = oracle.refresh_f64(P, nodes, lr)
    p = oracle.make_params(n, epsilon=eps, theta=0.5, dt=0.005)
    acc64, pot64, dens64, cnt = oracle.walk_f64(p, P, nodes, com64)
    for wg, (acc, dens, cnt_dev, _, _, _) in out.items():
        rel = _rel(acc[:, :3].astype(np.float64), acc64)
        assert np.median(rel) <= 2e-5 and np.percentile(rel, 99) <= 1e-3, (wg, np.median(rel))
        assert np.median(np.abs(acc[:, 3] - pot64) / np.abs(pot64)) <= 2e-5, wg
        assert cnt_dev == out[32][2], (wg, cnt_dev, out[32][2])      # the same decisions
        assert np.array_equal(dens, out[32][1]), wg                  # the same own leaves
        # the sums differ only by rounding
        d = _rel(acc[:, :3].astype(np.float64), out[32][0][:, :3].astype(np.float64))
        assert np.median(d) < 1e-6 and np.percentile(d, 99) < 1e-4, (wg, np.median(d), np.percentile(d, 99))


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
    pool.run(2, True)
    assert all(pool.device_errors(s) == 0 for s in pool.n)
    pool.close()
