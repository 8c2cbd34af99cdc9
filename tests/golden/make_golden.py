"""Generate the committed golden fixtures of the gravity path.

Run from the repository root:  python tests/golden/make_golden.py

The fixtures come from the oracle (oracle/, the CPU restatement of
src/physics/mortonTree.js and src/physics/shaders/nbody_bh.wgsl) on seeded
inputs. They pin the oracle across machines and compilers; the oracle itself
is pinned to the reference by the hand-derived known answers in
tests/test_oracle.py (no JS engine exists to run mortonTree.js here).

Small crafted cases are stored in full (golden_small.npz); the 16384-particle
disk is stored as SHA-256 digests plus a few slices (golden_disk16k.json).
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

import oracle as O  # noqa: E402
from galaxy_sim_b200 import initial_conditions as ic  # noqa: E402


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def topology(nodes):
    """Integer/size fields of BHNodes (COM fields excluded)."""
    return np.stack([nodes["size"].view(np.uint32), nodes["isLeaf"], nodes["first"],
                     nodes["count"]], axis=1).astype(np.uint32), nodes["children"].copy()


def crafted_cases():
    rng = np.random.default_rng(1234)
    cases = {}
    # 1. two particles at opposite cube corners
    P = np.zeros((2, 8), np.float32)
    P[1, :3] = 1.0
    P[:, 3] = 1.0
    cases["corners"] = P
    # 2. 16 clustered + 1 far: root with two leaf children (octants 0 and 7)
    P = np.zeros((17, 8), np.float32)
    P[:16, :3] = rng.uniform(0, 0.1, (16, 3))
    P[16, :3] = 1.0
    P[:, 3] = rng.uniform(0.5, 1.5, 17)
    cases["split17"] = P
    # 3. 20 identical particles: a chain of single-child nodes down to a depth-10 leaf
    P = np.zeros((20, 8), np.float32)
    P[:, :3] = 0.25
    P[:, 3] = 1.0
    cases["identical20"] = P
    # 4. non-finite positions are left out of the bbox and quantised through ToInt32
    P = rng.uniform(-1, 1, (40, 8)).astype(np.float32)
    P[:, 3] = 1.0
    P[3, 0] = np.nan
    P[7, 1] = np.inf
    P[11, 2] = -np.inf
    P[13, 0] = 3e38
    P[13, 1] = np.nan
    cases["nonfinite40"] = P
    # 5. duplicates + ties across a 300-particle clump (stable-sort ties)
    P = np.zeros((300, 8), np.float32)
    P[:, :3] = np.round(rng.uniform(-1, 1, (300, 3)) * 4) / 4
    P[:, 3] = rng.uniform(0.1, 2, 300)
    cases["ties300"] = P
    # 6. uniform cube, 5000 particles
    P = np.zeros((5000, 8), np.float32)
    P[:, :3] = rng.uniform(-3, 3, (5000, 3))
    P[:, 3] = rng.uniform(0.1, 2, 5000)
    cases["cube5000"] = P
    return cases


def main():
    O.build()
    out = {}
    for name, P in crafted_cases().items():
        N = P.shape[0]
        S = np.zeros((N, 4), np.float32)
        S[:, 0] = np.arange(N)
        codes, root = O.compute_morton_codes(P, N, 8)
        perm = O.radix_sort_indices(codes)
        b = O.sort_and_build(P, S)
        assert np.array_equal(b["perm"], perm)
        out[f"{name}/particles"] = P
        out[f"{name}/codes"] = codes
        out[f"{name}/root_size"] = np.array([root])
        out[f"{name}/perm"] = perm
        out[f"{name}/nodes"] = b["nodes"].view(np.uint32).reshape(-1, 16)
        out[f"{name}/level_ranges"] = b["levelRanges"]
    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **out)

    g = ic.disk_16k()
    N = g.N
    b = O.sort_and_build(g.particles, g.stellar)
    codes, root = O.compute_morton_codes(g.particles, N, 8)
    topo, children = topology(b["nodes"])
    refreshed = O.refresh_f32(b["sorted"], b["nodes"], b["levelRanges"])
    p = O.make_params(N, epsilon=0.05, theta=0.5, dt=0.005, haloMass=g.halo_mass, haloA=g.halo_a,
                      haloCenters=g.halo_centers)
    out_p, energy, acc4, dens, cnt = O.step_f32(p, b["sorted"], refreshed, want_forces=True)
    meta = {
        "workload": "disk16k (seed 0): N=16384, Q=1.5, 2 arms, no gas; eps 0.05, theta 0.5, dt 0.005",
        "particles_sha256": digest(g.particles),
        "stellar_sha256": digest(g.stellar),
        "root_size": root,
        "codes_sha256": digest(codes),
        "perm_sha256": digest(b["perm"]),
        "perm_head": b["perm"][:16].tolist(),
        "num_nodes": int(len(b["nodes"])),
        "level_ranges": b["levelRanges"].tolist(),
        "topology_sha256": digest(topo),
        "children_sha256": digest(children),
        "build_com_sha256": digest(b["nodes"]["com"]),
        "build_mass_sha256": digest(b["nodes"]["mass"]),
        "refresh_f32_sha256": digest(np.stack([refreshed["com"][:, 0], refreshed["com"][:, 1],
                                               refreshed["com"][:, 2], refreshed["mass"]], 1)),
        "step_f32_sha256": digest(out_p),
        "energy_f32_sha256": digest(energy),
        "interactions": [int(x) for x in cnt],
        "acc0": acc4[0].tolist(),
    }
    with open(os.path.join(HERE, "golden_disk16k.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
