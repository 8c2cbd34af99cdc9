"""GPU-backed mirror of the exports of galaxy-sim's ``src/physics/mortonTree.js``.

Same names, argument meaning and return values as the JavaScript module, so a
caller of ``computeMortonCodes``, ``radixSortIndices``, ``MortonTree`` and
``sortAndBuild`` can switch to these; every result is computed by the CUDA
library (include/galaxy_b200.h) and matches the JavaScript bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import NODE_DTYPE, check, f32, lib, ptr, u32

WORDS = 16   # mortonTree.js:23
BYTES = 64   # mortonTree.js:24
BUCKET = 16  # mortonTree.js:25
MAX_LEVEL = 10  # mortonTree.js:26


def computeMortonCodes(pos, N: int, stride: int, codes) -> float:
    """mortonTree.js:43-62 — fills ``codes`` (uint32[N]) and returns the root cube size."""
    pos = f32(pos).ravel()
    if N and pos.size < (N - 1) * stride + 3:
        raise ValueError("pos holds fewer than N records")
    out = np.zeros(N, np.uint32)
    root = C.c_double(0.0)
    check(lib().gs_morton_codes(ptr(pos), N, stride, ptr(out), C.byref(root)))
    codes[:N] = out
    return root.value


def radixSortIndices(codes, indices, scratch, counts, N: int):
    """mortonTree.js:68-84 — stable sort by code; returns the gather permutation.

    As in the JavaScript the result lands in one of the two index arrays (here
    always ``scratch``, the array the three-pass JavaScript returns); ``counts``
    is accepted for signature compatibility.
    """
    del counts
    c = u32(np.asarray(codes)[:N])
    out = np.zeros(N, np.uint32)
    check(lib().gs_radix_sort_indices(ptr(c), N, ptr(out)))
    indices[:N] = np.arange(N, dtype=np.uint32)
    scratch[:N] = out
    return scratch


class MortonTree:
    """mortonTree.js:86-185 — a node pool of 2 * maxParticles + 4096 64-byte nodes."""

    def __init__(self, maxParticles: int):
        self.maxNodes = maxParticles * 2 + 4096
        self._nodes = np.zeros(self.maxNodes, NODE_DTYPE)
        self._buf = self._nodes.view(np.uint8)
        self.f32 = self._nodes.view(np.float32)
        self.i32 = self._nodes.view(np.int32)
        self.numNodes = 0
        self.levelRanges = []

    def build(self, codes, pos, masses, N: int, rootSize: float) -> None:
        """BFS bucketed build from Morton-sorted codes, stride-3 positions, masses."""
        nn = C.c_uint32(0)
        nl = C.c_uint32(0)
        lr = np.zeros(64, np.uint32)
        check(lib().gs_tree_build(ptr(u32(np.asarray(codes)[:N])), ptr(f32(np.asarray(pos)[:3 * N])),
                                  ptr(f32(np.asarray(masses)[:N])), N, rootSize, self.maxNodes,
                                  ptr(self._nodes), C.byref(nn), ptr(lr), 32, C.byref(nl)))
        self.numNodes = nn.value
        self.levelRanges = [[int(lr[2 * k]), int(lr[2 * k + 1])] for k in range(nl.value)]

    @property
    def nodes(self):
        return self._nodes[: self.numNodes]

    @property
    def byteLength(self) -> int:
        return self.numNodes * BYTES


def sortAndBuild(particleData, stellarData, N: int, trackIdx2: int = -1) -> dict:
    """mortonTree.js:192-224 — bootstrap sort of 8-float records + stellar records + tree."""
    P = f32(particleData).ravel()[: 8 * N]
    S = f32(stellarData).ravel()[: 4 * N]
    tree = MortonTree(N)
    sorted8 = np.zeros(8 * N, np.float32)
    sorted4 = np.zeros(4 * N, np.float32)
    perm = np.zeros(N, np.uint32)
    masses = np.zeros(N, np.float32)
    nn, nl = C.c_uint32(0), C.c_uint32(0)
    lr = np.zeros(64, np.uint32)
    c1, c2 = C.c_int64(0), C.c_int64(-1)
    check(lib().gs_sort_and_build(ptr(P), ptr(S), N, trackIdx2, ptr(sorted8), ptr(sorted4), ptr(perm),
                                  ptr(tree._nodes), tree.maxNodes, C.byref(nn), ptr(lr), 32,
                                  C.byref(nl), C.byref(c1), C.byref(c2), ptr(masses)))
    tree.numNodes = nn.value
    tree.levelRanges = [[int(lr[2 * k]), int(lr[2 * k + 1])] for k in range(nl.value)]
    return {"sorted": sorted8, "sortedStellar": sorted4, "tree": tree, "perm": perm,
            "centralIdx": c1.value, "centralIdx2": c2.value, "masses": masses}
