"""Degenerate inputs through the full device path.

* A far outlier stretches the Morton cube so that most particles share their
  codes down to depth 10: leaves there hold many more than 16 particles (the
  reference's MAX_LEVEL leaf rule, mortonTree.js:126), which sends the walk down
  its chunked large-leaf path.
* A cluster of coincident particles gives equal codes, zero-distance pairs and
  depth-10 chains.
Each must build the reference's tree, walk with forces inside the FP64-walk
tolerance, raise no device error, and step identically alone and in a pool.
"""
import numpy as np
import pytest

from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.pool import GalaxyPool

pytestmark = pytest.mark.gpu

KW = dict(dt=0.005, G=1.0, epsilon=0.02, theta=0.5)


def _outlier():
    g = ic.galaxy_disk(6000, 31)
    P = g.particles.copy()
    P[-1, :3] = (3.0e4, -2.0e4, 1.0e4)
    return P, g.stellar


def _cluster():
    g = ic.galaxy_disk(5000, 32)
    P = g.particles.copy()
    P[1000:2200, :3] = P[1000, :3]
    return P, g.stellar


@pytest.mark.parametrize("make", [_outlier, _cluster], ids=["outlier", "cluster"])
def test_degenerate_inputs(gpu_lib, oracle, make):
    P0, S0 = make()
    N = P0.shape[0]
    sim = NBodyGPU(0, P0, S0)
    sim.updateParams(**KW)
    sim.setDebug(True)
    sim.sortBuild()
    nodes, lr, perm = sim.getTree()
    P, _ = sim.readState()
    want = oracle.sort_and_build(P0, S0)
    assert np.array_equal(perm, want["perm"])
    for f in ("isLeaf", "first", "count", "children", "size"):
        assert np.array_equal(nodes[f], want["nodes"][f]), f
    big = int(np.max(want["nodes"]["count"][want["nodes"]["isLeaf"] == 1]))
    sim.step()
    acc, _ = sim.readForces()
    assert sim.deviceErrors() == 0
    com64 = oracle.refresh_f64(P, want["nodes"], want["levelRanges"])
    p = oracle.make_params(N, epsilon=KW["epsilon"], theta=KW["theta"], dt=KW["dt"])
    acc64, _, _, _ = oracle.walk_f64(p, P, want["nodes"], com64)
    rel = np.linalg.norm(acc[:, :3] - acc64, axis=1) / np.maximum(np.linalg.norm(acc64, axis=1), 1e-30)
    assert np.median(rel) < 2e-5 and np.percentile(rel, 99) < 1e-3, (np.median(rel), big)
    sim.destroy()
    if make is _outlier:
        assert big > 16  # the large-leaf path ran
    # full steps alone vs in a pool next to another galaxy
    solo = NBodyGPU(0, P0, S0)
    solo.updateParams(**KW)
    solo.run(3, True)
    want_P, _ = solo.readState()
    solo.destroy()
    other = ic.galaxy_disk(3000, 33)
    pool = GalaxyPool(N + other.N + 512, 2)
    pool.add(other.particles, other.stellar, KW)
    s = pool.add(P0, S0, KW)
    pool.run(3, True)
    got_P, _ = pool.read_state(s)
    assert np.array_equal(got_P.view(np.uint32), want_P.view(np.uint32))
    assert np.all(np.isfinite(got_P))
    assert pool.device_errors(s) == 0
    pool.close()
