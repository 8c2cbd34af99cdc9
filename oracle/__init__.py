"""TEST INFRASTRUCTURE ONLY — ctypes bindings of the CPU oracle (liboracle.so).

The oracle restates galaxy-sim's gravity path on the CPU:

* ``src/physics/mortonTree.js`` — Morton codes (:43-62), the stable LSD radix
  sort (:68-84), the BFS bucketed octree (:107-182), ``sortAndBuild`` (:192-224);
* ``src/physics/bhWorker.js:55-94`` — the asynchronous rebuild;
* ``src/physics/shaders/nbody_bh.wgsl`` — refresh (:289-313), walk + halo +
  kick-drift (:64-181), star formation (:197-268), gather (:319-340),
  compaction (:183-195);
* FP64 references: COM refresh, BH walk with the same acceptance rule on the
  same tree, direct O(N^2) sum, analytic halo.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package, as the test reference or the timed CPU baseline; the product
package ``galaxy_sim_b200`` never does.

Parity pinning: the reference's tests pin only the gather convention
``out[i] = in[perm[i]]`` (test/StarSelection.test.js:51-57); there is no JS
engine or WebGPU stack to run the reference, so the rest is *parity unpinned*
against the reference itself and pinned instead by hand-derived known answers
and committed golden vectors (tests/golden/).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

NODE_DTYPE = np.dtype(
    [
        ("com", "<f4", (3,)),
        ("mass", "<f4"),
        ("size", "<f4"),
        ("isLeaf", "<u4"),
        ("first", "<u4"),
        ("count", "<u4"),
        ("children", "<i4", (8,)),
    ]
)
assert NODE_DTYPE.itemsize == 64


class Params(C.Structure):
    """96-byte Params uniform, nbody_bh.wgsl:19-42 / NBodyGPU.js:253-275."""

    _fields_ = [
        ("dt", C.c_float),
        ("G", C.c_float),
        ("epsilon2", C.c_float),
        ("N", C.c_uint32),
        ("theta", C.c_float),
        ("haloMass", C.c_float),
        ("haloA", C.c_float),
        ("gasDrag", C.c_float),
        ("time", C.c_float),
        ("agingRate", C.c_float),
        ("sfDensity", C.c_float),
        ("sfEff", C.c_float),
        ("sfDt", C.c_float),
        ("haloCount", C.c_uint32),
        ("pad0", C.c_float),
        ("pad1", C.c_float),
        ("haloC1", C.c_float * 4),
        ("haloC2", C.c_float * 4),
    ]


assert C.sizeof(Params) == 96


class PipelineState(C.Structure):
    _fields_ = [
        ("haloC", (C.c_double * 3) * 2),
        ("central", C.c_int64 * 2),
        ("time", C.c_double),
    ]


def make_params(N, dt=0.005, G=1.0, epsilon=0.05, theta=0.5, haloMass=0.0, haloA=1.0,
                gasDrag=0.0, time=0.0, agingRate=25.0, sfDensity=1e9, sfEff=0.0, sfDt=0.0,
                haloCenters=()):
    """Fill Params the way NBodyGPU.updateParams does (NBodyGPU.js:253-275)."""
    p = Params()
    p.dt, p.G = dt, G
    p.epsilon2 = np.float32(float(epsilon) * float(epsilon))   # JS: double product, f32 store
    p.N = N
    p.theta, p.haloMass, p.haloA, p.gasDrag = theta, haloMass, haloA, gasDrag
    p.time, p.agingRate, p.sfDensity, p.sfEff, p.sfDt = time, agingRate, sfDensity, sfEff, sfDt
    p.haloCount = min(len(haloCenters), 2)
    for h, c in enumerate(list(haloCenters)[:2]):
        arr = p.haloC1 if h == 0 else p.haloC2
        for k in range(3):
            arr[k] = c[k]
    return p


_lib = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (system g++ + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, u32, i64, f64 = C.c_void_p, C.c_uint32, C.c_int64, C.c_double
        L.or_part1by2.argtypes, L.or_part1by2.restype = [u32], u32
        L.or_js_toint32.argtypes, L.or_js_toint32.restype = [f64], C.c_int32
        L.or_compute_morton_codes.argtypes = [vp, u32, u32, vp]
        L.or_compute_morton_codes.restype = f64
        L.or_radix_sort_indices.argtypes = [vp, u32, vp]
        L.or_tree_build.argtypes = [vp, vp, vp, u32, f64, u32, vp, vp, u32, vp]
        L.or_tree_build.restype = i64
        L.or_sort_and_build.argtypes = [vp, vp, u32, i64, vp, vp, vp, vp, u32, vp, u32, vp, vp,
                                        vp, vp, vp]
        L.or_sort_and_build.restype = i64
        L.or_worker_build.argtypes = [vp, u32, vp, vp, vp, vp, u32, vp, u32, vp, vp, vp, vp, vp]
        L.or_worker_build.restype = i64
        L.or_apply_permutation.argtypes = [vp, vp, vp, u32, u32]
        L.or_refresh_f32.argtypes = [vp, vp, vp, u32]
        L.or_refresh_f64.argtypes = [vp, vp, u32, vp, u32, vp]
        L.or_step_f32.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]
        L.or_walk_f64.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]
        L.or_direct_f64.argtypes = [vp, vp, vp, u32, vp, vp, C.c_int]
        L.or_halo_f64.argtypes = [vp, vp, vp, u32, vp, vp]
        L.or_star_formation.argtypes = [vp, vp, vp]
        L.or_compact_positions.argtypes = [vp, vp, u32, vp]
        L.or_pcg.argtypes, L.or_pcg.restype = [u32], u32
        L.or_rand01.argtypes, L.or_rand01.restype = [u32, u32], C.c_float
        L.or_imf_sample.argtypes, L.or_imf_sample.restype = [C.c_float, C.c_float], C.c_float
        L.or_full_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, u32, vp, vp]
        L.or_step_f32_sample.argtypes = [vp, vp, vp, vp, vp, u32, C.c_int]
        L.or_full_step.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def part1by2(v: int) -> int:
    return int(lib().or_part1by2(v))


def js_toint32(d: float) -> int:
    return int(lib().or_js_toint32(d))


def compute_morton_codes(pos, N: int, stride: int):
    """mortonTree.js:43-62 -> (codes uint32[N], rootSize float)."""
    pos = _f32(pos).ravel()
    codes = np.zeros(N, np.uint32)
    size = lib().or_compute_morton_codes(_p(pos), N, stride, _p(codes))
    return codes, size


def radix_sort_indices(codes):
    """mortonTree.js:68-84 -> perm uint32[N] (gather order)."""
    codes = np.ascontiguousarray(codes, np.uint32)
    perm = np.zeros(len(codes), np.uint32)
    lib().or_radix_sort_indices(_p(codes), len(codes), _p(perm))
    return perm


def tree_build(sorted_codes, pos3, masses, root_size, max_nodes=None):
    """mortonTree.js:107-182 -> (nodes structured array, level_ranges [L,2])."""
    N = len(sorted_codes)
    if max_nodes is None:
        max_nodes = 2 * N + 4096
    nodes = np.zeros(max_nodes, NODE_DTYPE)
    lr = np.zeros(64, np.uint32)
    nl = np.zeros(1, np.uint32)
    nn = lib().or_tree_build(_p(np.ascontiguousarray(sorted_codes, np.uint32)),
                             _p(_f32(pos3).ravel()), _p(_f32(masses)), N, root_size, max_nodes,
                             _p(nodes), _p(lr), 32, _p(nl))
    if nn < 0:
        raise RuntimeError("oracle tree build overflowed its node pool or level table")
    return nodes[:nn].copy(), lr[: 2 * nl[0]].reshape(-1, 2).copy()


def sort_and_build(particles8, stellar4, track_idx2=-1):
    """mortonTree.js:192-224 (bootstrap)."""
    P = _f32(particles8).reshape(-1, 8)
    S = _f32(stellar4).reshape(-1, 4)
    N = P.shape[0]
    sorted8 = np.zeros_like(P)
    sorted4 = np.zeros_like(S)
    perm = np.zeros(N, np.uint32)
    max_nodes = 2 * N + 4096
    nodes = np.zeros(max_nodes, NODE_DTYPE)
    lr = np.zeros(64, np.uint32)
    nl = np.zeros(1, np.uint32)
    c1 = np.zeros(1, np.int64)
    c2 = np.zeros(1, np.int64)
    masses = np.zeros(N, np.float32)
    root = np.zeros(1, np.float64)
    nn = lib().or_sort_and_build(_p(P), _p(S), N, track_idx2, _p(sorted8), _p(sorted4), _p(perm),
                                 _p(nodes), max_nodes, _p(lr), 32, _p(nl), _p(c1), _p(c2),
                                 _p(masses), _p(root))
    if nn < 0:
        raise RuntimeError("oracle sortAndBuild overflowed")
    return dict(sorted=sorted8, sortedStellar=sorted4, nodes=nodes[:nn].copy(),
                levelRanges=lr[: 2 * nl[0]].reshape(-1, 2).copy(), perm=perm,
                centralIdx=int(c1[0]), centralIdx2=int(c2[0]), masses=masses,
                rootSize=float(root[0]))


def worker_build(pos4, masses, central_idx=0, central_idx2=-1):
    """bhWorker.js:55-94 -> dict like the worker's 'tree' message."""
    pos4 = _f32(pos4).reshape(-1, 4)
    N = pos4.shape[0]
    masses = _f32(masses).copy()
    c1 = np.array([central_idx], np.int64)
    c2 = np.array([central_idx2], np.int64)
    max_nodes = 2 * N + 4096
    nodes = np.zeros(max_nodes, NODE_DTYPE)
    lr = np.zeros(64, np.uint32)
    nl = np.zeros(1, np.uint32)
    perm = np.zeros(N, np.uint32)
    energy = np.zeros(1, np.float64)
    bh1 = np.zeros(3, np.float32)
    bh2 = np.zeros(3, np.float32)
    nn = lib().or_worker_build(_p(pos4), N, _p(masses), _p(c1), _p(c2), _p(nodes), max_nodes,
                               _p(lr), 32, _p(nl), _p(perm), _p(energy), _p(bh1), _p(bh2))
    if nn < 0:
        raise RuntimeError("oracle worker build overflowed")
    return dict(nodes=nodes[:nn].copy(), levelRanges=lr[: 2 * nl[0]].reshape(-1, 2).copy(),
                perm=perm, centralIdx=int(c1[0]), centralIdx2=int(c2[0]), energy=float(energy[0]),
                bh1=bh1, bh2=bh2 if central_idx2 >= 0 else None, masses=masses)


def apply_permutation(src, perm, width):
    src = _f32(src).reshape(-1, width)
    out = np.zeros_like(src)
    lib().or_apply_permutation(_p(src), _p(out), _p(np.ascontiguousarray(perm, np.uint32)),
                               len(perm), width)
    return out


def refresh_f32(particles8, nodes, level_ranges):
    nodes = nodes.copy()
    lr = np.ascontiguousarray(level_ranges, np.uint32)
    lib().or_refresh_f32(_p(_f32(particles8).ravel()), _p(nodes), _p(lr), lr.shape[0])
    return nodes


def refresh_f64(particles8, nodes, level_ranges):
    lr = np.ascontiguousarray(level_ranges, np.uint32)
    com4 = np.zeros((len(nodes), 4), np.float64)
    lib().or_refresh_f64(_p(_f32(particles8).ravel()), _p(np.ascontiguousarray(nodes)),
                         len(nodes), _p(lr), lr.shape[0], _p(com4))
    return com4


def step_f32(params, particles8, nodes, nthreads=0, want_forces=False):
    """nbody_bh.wgsl:64-181 -> (particles_out, energy, acc4|None, density|None, counters)."""
    P = _f32(particles8).reshape(-1, 8)
    N = P.shape[0]
    out = np.zeros_like(P)
    energy = np.zeros(N, np.float32)
    acc4 = np.zeros((N, 4), np.float32) if want_forces else None
    dens = np.zeros(N, np.float32) if want_forces else None
    cnt = np.zeros(3, np.uint64)
    lib().or_step_f32(C.byref(params), _p(P), _p(out), _p(np.ascontiguousarray(nodes)),
                      _p(energy), _p(acc4), _p(dens), _p(cnt), nthreads)
    return out, energy, acc4, dens, cnt


def walk_f64(params, particles8, nodes, com4, nthreads=0):
    """FP64 walk, same acceptance rule, same tree -> (acc3, pot, density, counters)."""
    P = _f32(particles8).reshape(-1, 8)
    N = P.shape[0]
    acc = np.zeros((N, 3), np.float64)
    pot = np.zeros(N, np.float64)
    dens = np.zeros(N, np.float32)
    cnt = np.zeros(3, np.uint64)
    lib().or_walk_f64(C.byref(params), _p(P), _p(np.ascontiguousarray(nodes)),
                      _p(np.ascontiguousarray(com4, np.float64)), _p(acc), _p(pot), _p(dens),
                      _p(cnt), nthreads)
    return acc, pot, dens, cnt


def direct_f64(params, particles8, targets, nthreads=0):
    P = _f32(particles8).reshape(-1, 8)
    t = np.ascontiguousarray(targets, np.uint32)
    acc = np.zeros((len(t), 3), np.float64)
    pot = np.zeros(len(t), np.float64)
    lib().or_direct_f64(C.byref(params), _p(P), _p(t), len(t), _p(acc), _p(pot), nthreads)
    return acc, pot


def halo_f64(params, particles8, targets):
    P = _f32(particles8).reshape(-1, 8)
    t = np.ascontiguousarray(targets, np.uint32)
    acc = np.zeros((len(t), 3), np.float64)
    pot = np.zeros(len(t), np.float64)
    lib().or_halo_f64(C.byref(params), _p(P), _p(t), len(t), _p(acc), _p(pot))
    return acc, pot


def star_formation(params, particles8, stellar4):
    P = _f32(particles8).reshape(-1, 8).copy()
    S = _f32(stellar4).reshape(-1, 4).copy()
    lib().or_star_formation(C.byref(params), _p(P), _p(S))
    return P, S


def compact_positions(particles8, energy):
    P = _f32(particles8).reshape(-1, 8)
    out = np.zeros((P.shape[0], 4), np.float32)
    lib().or_compact_positions(_p(P), _p(_f32(energy)), P.shape[0], _p(out))
    return out


def pcg(v):
    return int(lib().or_pcg(v & 0xFFFFFFFF))


def rand01(i, salt):
    return float(lib().or_rand01(i & 0xFFFFFFFF, salt & 0xFFFFFFFF))


def imf_sample(u1, u2):
    return float(lib().or_imf_sample(u1, u2))


class Pipeline:
    """Oracle of the full per-step sequence the CUDA path runs (oracle/pipeline.cpp)."""

    def __init__(self, particles8, stellar4, params, central=(-1, -1), halo_centers=None,
                 time=0.0, nthreads=0):
        self.P = _f32(particles8).reshape(-1, 8).copy()
        self.S = _f32(stellar4).reshape(-1, 4).copy()
        self.P2 = np.zeros_like(self.P)
        self.S2 = np.zeros_like(self.S)
        self.energy = np.zeros(self.P.shape[0], np.float32)
        self.params = params
        self.state = PipelineState()
        self.state.central[0], self.state.central[1] = central
        self.state.time = time
        if halo_centers is not None:
            for h, c in enumerate(halo_centers[:2]):
                for k in range(3):
                    self.state.haloC[h][k] = float(np.float32(c[k]))
        self.nthreads = nthreads
        self.t_build = 0.0
        self.t_walk = 0.0

    def step(self, do_sf=False, walk_stride=1):
        """One full step; walk_stride > 1 walks every walk_stride-th particle only."""
        tb = np.zeros(1)
        tw = np.zeros(1)
        rc = lib().or_full_step(C.byref(self.params), C.byref(self.state), _p(self.P), _p(self.S),
                                _p(self.P2), _p(self.S2), _p(self.energy), int(do_sf),
                                self.nthreads, int(walk_stride), _p(tb), _p(tw))
        if rc != 0:
            raise RuntimeError("oracle full step failed")
        self.t_build += tb[0]
        self.t_walk += tw[0]
