"""Generate golden fixtures by running the REFERENCE's own tree-build code.

Run from the repository root (needs the reference checkout, by default at
/root/reference, or at $GS_REFERENCE_ROOT):

    python tests/golden/make_reference_golden.py

src/physics/mortonTree.js and src/physics/bhWorker.js are executed as written,
by the small JavaScript interpreter in oracle/jsmini.py, on seeded inputs:
the crafted cases of make_golden.py plus edge cases (no particles, one
particle, all coincident, two far clusters, codes with bits above 30),
stride-4 positions as the worker reads them, two consecutive worker rebuilds,
and a tree whose node pool runs out (the reference overflows it). Their outputs are stored as they come out
of the reference: reference_mortontree.npz holds the small cases in full,
reference_digests.json larger seeded disks as SHA-256 digests. Tests compare the
C++ oracle and the CUDA path with these files on machines where the reference
itself is absent.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import crafted_cases  # noqa: E402

from galaxy_sim_b200 import initial_conditions as ic  # noqa: E402
from oracle import jsmini as J  # noqa: E402

REFERENCE = os.environ.get("GS_REFERENCE_ROOT", "/root/reference")
MORTON_JS = os.path.join(REFERENCE, "src", "physics", "mortonTree.js")
WORKER_JS = os.path.join(REFERENCE, "src", "physics", "bhWorker.js")


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def extra_cases():
    rng = np.random.default_rng(99)
    cases = {"empty": np.zeros((0, 8), np.float32)}
    P = np.zeros((1, 8), np.float32)
    P[0, :4] = (0.5, -2.0, 3.0, 1.0)
    cases["single"] = P
    P = np.zeros((40, 8), np.float32)
    P[:, :3] = (1.5, -0.25, 7.0)
    P[:, 3] = rng.uniform(0.5, 1.5, 40).astype(np.float32)
    cases["coincident40"] = P
    P = np.zeros((600, 8), np.float32)
    P[:300, :3] = rng.normal(-50.0, 0.3, (300, 3))
    P[300:, :3] = rng.normal(50.0, 0.3, (300, 3))
    P[:, 3] = rng.uniform(0.1, 1.0, 600).astype(np.float32)
    cases["farclusters600"] = P
    return cases


def tree_out(t):
    """(nodes as uint32 words [numNodes, 16], levelRanges [L, 2]) of a MortonTree."""
    nn = int(J.get_prop(t, "numNodes"))
    buf = J.get_prop(t, "_buf")
    nodes = np.frombuffer(bytes(buf.data[: nn * 64]), np.uint32).reshape(-1, 16).copy()
    lr = J.to_numpy(J.get_prop(t, "levelRanges")).astype(np.uint32).reshape(-1, 2)
    return nodes, lr


class Reference:
    """The reference's mortonTree.js exports and one bhWorker.js instance."""

    def __init__(self):
        self.m = J.load_module(MORTON_JS)
        self.sent = []
        self.self_obj = J.JSObject()
        self.self_obj.props["postMessage"] = J.JSFunction(lambda this, msg=None, *rest: self.sent.append(msg))
        J.load_module(WORKER_JS, self_object=self.self_obj)

    def codes(self, P, stride):
        N = P.shape[0]
        codes = J.construct("Uint32Array", [N])
        root = J.call_value(self.m["computeMortonCodes"], None,
                            [J.from_numpy(np.ascontiguousarray(P).reshape(-1)), N, stride, codes])
        return J.to_numpy(codes).astype(np.uint32), float(root)

    def sort(self, codes):
        N = codes.size
        args = [J.from_numpy(codes.astype(np.uint32)), J.construct("Uint32Array", [N]),
                J.construct("Uint32Array", [N]), J.construct("Uint32Array", [1024]), N]
        return J.to_numpy(J.call_value(self.m["radixSortIndices"], None, args)).astype(np.uint32)

    def build(self, sorted_codes, pos3, masses, root, max_particles=None):
        N = sorted_codes.size
        t = J.construct(self.m["MortonTree"], [N if max_particles is None else max_particles])
        J.call_method(t, "build", [J.from_numpy(sorted_codes.astype(np.uint32)),
                                   J.from_numpy(np.ascontiguousarray(pos3, np.float32).reshape(-1)),
                                   J.from_numpy(np.ascontiguousarray(masses, np.float32)), N, root])
        return tree_out(t)

    def sort_and_build(self, P, S, track2):
        N = P.shape[0]
        r = J.call_value(self.m["sortAndBuild"], None,
                         [J.from_numpy(P.reshape(-1)), J.from_numpy(S.reshape(-1)), N, track2])
        nodes, lr = tree_out(J.get_prop(r, "tree"))
        return {"sorted": J.to_numpy(J.get_prop(r, "sorted")).reshape(-1, 8),
                "sortedStellar": J.to_numpy(J.get_prop(r, "sortedStellar")).reshape(-1, 4),
                "perm": J.to_numpy(J.get_prop(r, "perm")).astype(np.uint32),
                "centralIdx": int(J.get_prop(r, "centralIdx")),
                "centralIdx2": int(J.get_prop(r, "centralIdx2")),
                "masses": J.to_numpy(J.get_prop(r, "masses")), "nodes": nodes, "levelRanges": lr}

    def worker(self, msg):
        J.call_value(self.self_obj.props["onmessage"], None, [J.JSObject({"data": J.JSObject(msg)})])
        return self.sent[-1] if self.sent else None


def worker_case(ref, rng, name, P, out):
    """Config, then two rebuilds through the worker protocol (bhWorker.js:13-18)."""
    N = P.shape[0]
    masses = P[:, 3].copy()
    c1, c2 = 0, N // 3
    ref.sent.clear()
    ref.worker({"type": "config", "N": N, "masses": J.from_numpy(masses), "centralIdx": c1, "centralIdx2": c2})
    pos4 = np.concatenate([P[:, :3], rng.normal(0, 1, (N, 1))], 1).astype(np.float32)
    out[f"worker_{name}/masses"] = masses
    out[f"worker_{name}/central_in"] = np.array([c1, c2], np.int64)
    for k in range(2):
        out[f"worker_{name}/pos4_{k}"] = pos4
        msg = ref.worker({"type": "build", "positions": J.from_numpy(pos4.reshape(-1))})
        tree = J.get_prop(msg, "tree")
        nodes = np.frombuffer(bytes(tree.data), np.uint32).reshape(-1, 16).copy()
        assert nodes.shape[0] == int(J.get_prop(msg, "numNodes"))
        perm = J.to_numpy(J.get_prop(msg, "perm")).astype(np.uint32)
        out[f"worker_{name}/nodes_{k}"] = nodes
        out[f"worker_{name}/perm_{k}"] = perm
        out[f"worker_{name}/level_ranges_{k}"] = J.to_numpy(J.get_prop(msg, "levelRanges")).astype(np.uint32)
        out[f"worker_{name}/central_{k}"] = np.array([J.get_prop(msg, "centralIdx"),
                                                      J.get_prop(msg, "centralIdx2")], np.int64)
        out[f"worker_{name}/energy_{k}"] = np.array([J.get_prop(msg, "energy")], np.float64)
        out[f"worker_{name}/bh_{k}"] = np.stack([J.to_numpy(J.get_prop(msg, "bh1")),
                                                 J.to_numpy(J.get_prop(msg, "bh2"))]).astype(np.float32)
        # the next frame: the GPU applied the permutation and the particles moved
        pos4 = pos4[perm].copy()
        pos4[:, :3] += rng.normal(0, 0.01, (N, 3)).astype(np.float32)
        pos4[:, 3] = rng.normal(0, 1, N).astype(np.float32)


def main():
    ref = Reference()
    rng = np.random.default_rng(2026)
    out = {}
    cases = dict(crafted_cases())
    cases.update(extra_cases())
    for name, P in cases.items():
        N = P.shape[0]
        S = np.zeros((N, 4), np.float32)
        S[:, 0] = np.arange(N)
        S[:, 2] = rng.uniform(0, 1, N)
        codes8, root8 = ref.codes(P, 8)
        codes4, root4 = ref.codes(np.ascontiguousarray(P[:, :4]), 4)
        perm = ref.sort(codes8)
        nodes, lr = ref.build(codes8[perm], P[perm, :3], P[perm, 3], root8)
        b = ref.sort_and_build(P, S, N // 2)
        assert np.array_equal(b["perm"], perm)
        out[f"{name}/particles"] = P
        out[f"{name}/stellar"] = S
        out[f"{name}/codes"] = codes8
        out[f"{name}/root_size"] = np.array([root8])
        out[f"{name}/codes_stride4"] = codes4
        out[f"{name}/root_size_stride4"] = np.array([root4])
        out[f"{name}/perm"] = perm
        out[f"{name}/nodes"] = nodes
        out[f"{name}/level_ranges"] = lr
        out[f"{name}/sab_nodes"] = b["nodes"]
        out[f"{name}/sab_sorted"] = b["sorted"]
        out[f"{name}/sab_sorted_stellar"] = b["sortedStellar"]
        out[f"{name}/sab_central"] = np.array([b["centralIdx"], b["centralIdx2"]], np.int64)
        out[f"{name}/sab_masses"] = b["masses"]
    # radixSortIndices on keys with bits above 30 (it orders by the low 30 only) and many ties
    keys = (rng.integers(0, 64, 5000, dtype=np.uint32) << 24) | (rng.integers(0, 4, 5000, dtype=np.uint32) << 30)
    out["sort_highbits/codes"] = keys
    out["sort_highbits/perm"] = ref.sort(keys)
    worker_case(ref, rng, "farclusters600", cases["farclusters600"], out)
    worker_case(ref, rng, "ties300", cases["ties300"], out)
    np.savez_compressed(os.path.join(HERE, "reference_mortontree.npz"), **out)

    digests = {"source": "src/physics/mortonTree.js run by oracle/jsmini.py"}
    g = ic.disk_16k()
    N = g.N
    codes8, root8 = ref.codes(g.particles, 8)
    b = ref.sort_and_build(g.particles, g.stellar, N // 2)
    digests["disk16k"] = {
        "workload": "initial_conditions.disk_16k(): N=16384; sortAndBuild(P, S, N, N/2)",
        "particles_sha256": digest(g.particles), "stellar_sha256": digest(g.stellar),
        "root_size": root8, "codes_sha256": digest(codes8), "perm_sha256": digest(b["perm"]),
        "num_nodes": int(b["nodes"].shape[0]), "level_ranges": b["levelRanges"].tolist(),
        "nodes_sha256": digest(b["nodes"]), "sorted_sha256": digest(b["sorted"]),
        "sorted_stellar_sha256": digest(b["sortedStellar"]),
        "central": [b["centralIdx"], b["centralIdx2"]],
    }
    # a node pool smaller than the tree needs: new MortonTree(0) holds 4096 nodes.
    # The third leaf clause (numNodes + 8 > maxNodes, mortonTree.js:127) turns the
    # node being built into a leaf, but children queued earlier on the same level
    # still get numbers: numNodes ends above maxNodes, the typed-array writes past
    # the pool are dropped and parents keep child indices past it. The fixture
    # records that outcome; the oracle and the CUDA build refuse such a pool.
    g = ic.galaxy_disk(32768, 77)
    P = g.particles
    codes8, root8 = ref.codes(P, 8)
    perm = ref.sort(codes8)
    t = J.construct(ref.m["MortonTree"], [0])
    J.call_method(t, "build", [J.from_numpy(codes8[perm]), J.from_numpy(np.ascontiguousarray(P[perm, :3]).reshape(-1)),
                               J.from_numpy(np.ascontiguousarray(P[perm, 3])), P.shape[0], root8])
    js_nodes = int(J.get_prop(t, "numNodes"))
    kept, lr = tree_out(t)
    full, _ = ref.build(codes8[perm], P[perm, :3], P[perm, 3], root8)
    assert full.shape[0] > 4096 and js_nodes > 4096
    digests["disk32k_pool4096"] = {
        "workload": "initial_conditions.galaxy_disk(32768, 77); new MortonTree(0).build(...) (4096 nodes)",
        "particles_sha256": digest(P), "root_size": root8, "max_nodes": 4096,
        "perm_sha256": digest(perm), "js_num_nodes": js_nodes, "nodes_in_pool": int(kept.shape[0]),
        "full_num_nodes": int(full.shape[0]), "overflow": js_nodes > 4096,
        "level_ranges": lr.tolist(), "nodes_in_pool_sha256": digest(kept),
    }
    with open(os.path.join(HERE, "reference_digests.json"), "w") as f:
        json.dump(digests, f, indent=1)
    print("wrote reference_mortontree.npz, reference_digests.json")


if __name__ == "__main__":
    main()
