"""Launch tuning: every knob value gives bit-identical results, and the
autotuner leaves a valid, timed choice set on the context."""
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
    sim.destroy()


def test_autotune_pool(gpu_lib):
    pool = GalaxyPool(40000, 4)
    for k, n in enumerate((3000, 9000, 20000)):
        g = ic.galaxy_disk(n, 20 + k)
        pool.add(g.particles, g.stellar, params_dict(g, Physics(0.05, 0.5, 0.005)))
    res = autotune(pool, steps=2, warmup=1, walk_blocks=(4, 8), sort_items=(8, 16))
    ch = res["choice"]
    assert len(res["ms"]) == 4 and all(t > 0 for t in res["ms"].values())
    assert get(pool._ctx, _lib.TUNE_WALK_BLOCKS_PER_SM) == ch["walk_blocks_per_sm"]
    assert get(pool._ctx, _lib.TUNE_SORT_ITEMS) == ch["sort_keys_per_thread"]
    pool.run(2, True)
    assert all(pool.device_errors(s) == 0 for s in pool.n)
    pool.close()
