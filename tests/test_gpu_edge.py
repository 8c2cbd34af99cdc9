"""Degenerate inputs through the full device path.

* A far outlier stretches the Morton cube so that most particles share their
  codes down to depth 10: leaves there hold many more than 16 particles (the
  reference's MAX_LEVEL leaf rule, mortonTree.js:126), which sends the walk down
  its chunked large-leaf path.
* A cluster of coincident particles gives equal codes, zero-distance pairs and
  depth-10 chains.
Each must build the reference's tree, walk with forces inside the FP64-walk
tolerance, raise no device error, and step identically alone and in a pool.
* Uploaded trees that break the layout rules are flagged, never followed out of
  bounds, and leave the context usable.
"""
import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200 import morton_tree as mt
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
    solo = NBodyGPU(0, P0, S0, walkGroup=32, walkSplit=1)   # a pool's default walk group
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


def _corrupt(nodes, N, how):
    """A copy of a valid BHNode array broken one way (the NBodyGPU upload rules:
    children are a contiguous increasing run after their parent, leaves stay
    inside the particle array)."""
    bad = nodes.copy()
    internal = [k for k in np.where(bad["isLeaf"] == 0)[0] if np.count_nonzero(bad["children"][k] >= 0) >= 2]
    k = internal[len(internal) // 2]
    ch = bad["children"][k]
    first = int(ch[ch >= 0][0])
    slots = np.where(ch >= 0)[0]
    if how == "gap":          # second child skips a node
        bad["children"][k, slots[1]] = first + 2
    elif how == "range":      # a child past the node array
        bad["children"][k, slots[0]] = len(nodes) + 5
    elif how == "backward":   # a child that points back at its parent
        bad["children"][k, slots[0]] = k
    elif how == "leaf":       # a leaf running past the particle array
        leaf = int(np.where(bad["isLeaf"] == 1)[0][-1])
        bad["first"][leaf] = N - 1
        bad["count"][leaf] = 16
    return bad


@pytest.mark.parametrize("how", ["gap", "range", "backward", "leaf"])
def test_malformed_uploaded_tree_is_flagged(gpu_lib, how):
    """uploadBHTree of a tree that breaks the layout rules raises GS_EDEVICE with
    GS_DERR_TREE; the broken nodes become empty leaves, so a step over that tree
    still ends, in bounds, with finite results; and the context stays usable: the
    valid tree uploaded afterwards gives exactly what a fresh context gives."""
    g = ic.disk_16k()
    boot = mt.sortAndBuild(g.particles.ravel(), g.stellar.ravel(), g.N)
    tree = boot["tree"]
    nodes = tree.nodes[: tree.numNodes]
    kw = dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5, haloMass=g.halo_mass, haloA=g.halo_a,
              haloCenters=[[0, 0, 0, 0]])
    fresh = NBodyGPU(0, boot["sorted"], boot["sortedStellar"])
    fresh.uploadBHTree(nodes, tree.numNodes, tree.levelRanges)
    fresh.updateParams(**kw)
    fresh.encodeRefresh()
    fresh.step()
    want, _ = fresh.readState()
    fresh.destroy()

    sim = NBodyGPU(0, boot["sorted"], boot["sortedStellar"])
    sim.updateParams(**kw)
    with pytest.raises(_lib.GalaxyError) as e:
        sim.uploadBHTree(_corrupt(nodes, g.N, how), tree.numNodes, tree.levelRanges)
    assert e.value.code == _lib.GS_EDEVICE
    assert sim.deviceErrors(clear=True) == _lib.DERR_TREE
    sim.encodeRefresh()
    sim.step()
    P, _ = sim.readState()  # raises if the walk over the flagged tree set any error bit
    assert np.all(np.isfinite(P))
    assert sim.deviceErrors() == 0
    # the same context, back on the valid tree from the same start
    sim.writeState(boot["sorted"], boot["sortedStellar"])
    sim.uploadBHTree(nodes, tree.numNodes, tree.levelRanges)
    sim.encodeRefresh()
    sim.step()
    got, _ = sim.readState()
    assert sim.deviceErrors() == 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sim.destroy()


def test_uploaded_dag_walk_is_bounded(gpu_lib):
    """A tree that obeys the upload rules but shares children between parents
    (node k's children are [k+1, k+2] down a chain of 40) has Fibonacci-many
    root-to-leaf paths. The walk's round budget and stack bound end every group
    with GS_DERR_STACK instead of running on; the context stays usable."""
    g = ic.galaxy_disk(64, 41)
    chain = 40
    nodes = np.zeros(chain + 2, _lib.NODE_DTYPE)
    nodes["mass"] = 1.0
    nodes["size"] = 1.0e6          # opened by every particle
    nodes["children"] = -1
    for k in range(chain):
        nodes["children"][k, 0], nodes["children"][k, 1] = k + 1, k + 2
    for j, leaf in enumerate((chain, chain + 1)):
        nodes["isLeaf"][leaf] = 1
        nodes["first"][leaf], nodes["count"][leaf] = 32 * j, 32
    kw = dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(**kw)
    sim.uploadBHTree(nodes, len(nodes))      # passes the layout rules
    assert sim.deviceErrors() == 0
    sim.step()
    with pytest.raises(_lib.GalaxyError) as e:
        sim.readState()
    assert e.value.code == _lib.GS_EDEVICE
    assert sim.deviceErrors(clear=True) & _lib.DERR_STACK
    # the same context walks a proper tree afterwards, exactly like a fresh one
    boot = mt.sortAndBuild(g.particles.ravel(), g.stellar.ravel(), g.N)
    tree = boot["tree"]
    outs = []
    for ctx in (sim, NBodyGPU(0, boot["sorted"], boot["sortedStellar"])):
        ctx.writeState(boot["sorted"], boot["sortedStellar"])
        ctx.updateParams(**kw)
        ctx.uploadBHTree(tree.nodes, tree.numNodes, tree.levelRanges)
        ctx.encodeRefresh()
        ctx.step()
        outs.append(ctx.readState()[0])
        assert ctx.deviceErrors() == 0
        ctx.destroy()
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_sort_lookback_wait_runs_out_and_reports(gpu_lib, oracle):
    """The sort's look-back is the one device-side wait. With a short test limit
    and one tile that never publishes its digit counts (a flag that nothing
    sets), the waits of the tiles after it run out: the kernel returns, the call
    reports GS_EDEVICE with the look-back bit, and the next sort is correct."""
    L = gpu_lib
    codes = np.random.default_rng(17).integers(0, 1 << 30, 12 * 4096 + 5, dtype=np.uint32)
    perm = np.zeros(codes.size, np.uint32)
    want = oracle.radix_sort_indices(codes)
    assert L.gs_test_sort_lookback(0, -1) == _lib.GS_EINVAL
    assert L.gs_test_sort_lookback(4096, 2) == 0
    try:
        rc = L.gs_radix_sort_indices(codes.ctypes.data, codes.size, perm.ctypes.data)
    finally:
        assert L.gs_test_sort_lookback(1 << 20, -1) == 0
    assert rc == _lib.GS_EDEVICE, L.gs_last_error(None)
    assert b"0x1" in L.gs_last_error(None)
    assert L.gs_radix_sort_indices(codes.ctypes.data, codes.size, perm.ctypes.data) == 0
    assert np.array_equal(perm, want)


def test_subnormal_softening_walks_as_none(gpu_lib):
    """epsilon2 below the smallest normal float is walked as no softening (every
    reciprocal square root the walk takes stays a normal number): the steps equal
    those at epsilon = 0 bit for bit and stay finite."""
    g = ic.disk_16k()
    assert 0.0 < np.float32(1e-20 * 1e-20) < np.finfo(np.float32).tiny
    out = []
    for eps in (0.0, 1e-20):
        sim = NBodyGPU(0, g.particles, g.stellar)
        sim.updateParams(dt=0.005, G=1.0, epsilon=eps, theta=0.5)
        sim.run(2, False)
        P, _ = sim.readState()
        assert sim.deviceErrors() == 0
        sim.destroy()
        out.append(P)
    assert np.all(np.isfinite(out[0]))
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))
