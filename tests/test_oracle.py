"""The oracle against hand-derived known answers, an independent pure-Python
transcription of src/physics/mortonTree.js (small cases), the one convention
the reference's own tests pin (test/StarSelection.test.js:51-57), and the
committed golden fixtures (tests/golden/)."""
import hashlib
import json
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ---- independent pure-Python transcription (JS number semantics) ----------------------

def js_toint32(d):
    if not math.isfinite(d):
        return 0
    t = math.trunc(d) % 2 ** 32
    return t - 2 ** 32 if t >= 2 ** 31 else t


def js_part1by2(v):
    v &= 0x3FF
    v = (v | (v << 16)) & 0x30000FF
    v = (v | (v << 8)) & 0x300F00F
    v = (v | (v << 4)) & 0x30C30C3
    v = (v | (v << 2)) & 0x9249249
    return v


def js_compute_morton_codes(pos, N, stride):  # mortonTree.js:43-62
    mn = [math.inf] * 3
    mx = [-math.inf] * 3
    for i in range(N):
        x, y, z = (float(pos[i * stride + k]) for k in range(3))
        if not math.isfinite(x + y + z):
            continue
        for k, v in enumerate((x, y, z)):
            if v < mn[k]:
                mn[k] = v
            if v > mx[k]:
                mx[k] = v
    ext = [mx[k] - mn[k] for k in range(3)]
    m = math.nan if any(math.isnan(e) for e in ext) else max(ext)
    size = m * 1.0001 + 1e-9
    s = 1024 / size if size != 0 else math.copysign(math.inf, size)
    codes = []
    for i in range(N):
        q = []
        for k in range(3):
            with np.errstate(all="ignore"):
                v = (float(pos[i * stride + k]) - mn[k]) * s
            q.append(min(js_toint32(v), 1023))
        codes.append(js_part1by2(q[0]) | (js_part1by2(q[1]) << 1) | (js_part1by2(q[2]) << 2))
    return np.array(codes, np.uint32), size


def js_radix_sort(codes):  # mortonTree.js:68-84
    N = len(codes)
    src = list(range(N))
    for p in range(3):
        sh = 10 * p
        counts = [0] * 1024
        for v in src:
            counts[(int(codes[v]) >> sh) & 1023] += 1
        s = 0
        for b in range(1024):
            c = counts[b]
            counts[b] = s
            s += c
        dst = [0] * N
        for v in src:
            d = (int(codes[v]) >> sh) & 1023
            dst[counts[d]] = v
            counts[d] += 1
        src = dst
    return np.array(src, np.uint32)


def js_tree_topology(codes, N):  # mortonTree.js:107-162 (topology only)
    nodes = []
    lr = []
    queue = [(0, N, -1, 0)]
    depth = 0
    max_nodes = 2 * N + 4096
    while queue:
        nxt = []
        start = len(nodes)
        for lo, hi, parent, slot in queue:
            idx = len(nodes)
            node = {"children": [-1] * 8, "isLeaf": 0, "first": 0, "count": 0, "depth": depth}
            nodes.append(node)
            if parent >= 0:
                nodes[parent]["children"][slot] = idx
            count = hi - lo
            if count <= 16 or depth >= 10 or len(nodes) + 8 > max_nodes:
                node.update(isLeaf=1, first=lo, count=count)
            else:
                shift = 27 - 3 * depth
                st = lo
                for k in range(8):
                    end = st
                    while end < hi and ((int(codes[end]) >> shift) & 7) == k:
                        end += 1
                    if end > st:
                        nxt.append((st, end, idx, k))
                    st = end
        lr.append([start, len(nodes) - start])
        queue = nxt
        depth += 1
    return nodes, lr


# ---- known answers ------------------------------------------------------------------------

def test_part1by2_known(oracle):
    for v, want in [(0, 0), (1, 1), (2, 8), (3, 9), (0x3FF, 0x9249249), (0x400, 0), (0x401, 1)]:
        assert oracle.part1by2(v) == want == js_part1by2(v)


def test_toint32_known(oracle):
    for d, want in [(5.9, 5), (-5.9, -5), (2.0 ** 32 + 7, 7), (2.0 ** 31, -2 ** 31),
                    (-(2.0 ** 31) - 1, 2 ** 31 - 1), (float("nan"), 0), (float("inf"), 0),
                    (-float("inf"), 0), (1e300, js_toint32(1e300))]:
        assert oracle.js_toint32(d) == want == js_toint32(d)


def test_codes_corners_known(oracle):
    P = np.zeros((2, 8), np.float32)
    P[1, :3] = 1.0
    codes, root = oracle.compute_morton_codes(P, 2, 8)
    assert root == 1.0 * 1.0001 + 1e-9
    assert codes.tolist() == [0, 0x3FFFFFFF]


def test_sort_stable_known(oracle):
    assert oracle.radix_sort_indices(np.array([5, 3, 5, 3, 0], np.uint32)).tolist() == [4, 1, 3, 0, 2]
    # digits in every 10-bit field, equal keys keep index order
    codes = np.array([1 << 20, 1 << 10, 1, 1 << 10, 0, 1 << 20], np.uint32)
    assert oracle.radix_sort_indices(codes).tolist() == [4, 2, 1, 3, 0, 5]


def test_gather_convention_matches_reference_test(oracle):
    # test/StarSelection.test.js:51-57: out[0]=in[2], out[1]=in[0], out[2]=in[1]
    src = np.arange(3 * 8, dtype=np.float32).reshape(3, 8)
    out = oracle.apply_permutation(src, np.array([2, 0, 1], np.uint32), 8)
    assert np.array_equal(out[0], src[2]) and np.array_equal(out[1], src[0])
    assert np.array_equal(out[2], src[1])


def test_tree_split17_known(oracle):
    d = np.load(os.path.join(GOLDEN, "golden_small.npz"))
    P = d["split17/particles"]
    b = oracle.sort_and_build(P, np.zeros((17, 4), np.float32))
    n = b["nodes"]
    assert b["levelRanges"].tolist() == [[0, 1], [1, 2]]
    assert n["isLeaf"].tolist() == [0, 1, 1]
    assert n["children"][0].tolist() == [1, -1, -1, -1, -1, -1, -1, 2]
    assert (n["first"][1], n["count"][1], n["first"][2], n["count"][2]) == (0, 16, 16, 1)
    assert n["size"][0] == np.float32(b["rootSize"]) and n["size"][1] == np.float32(b["rootSize"] / 2)
    # COM in double, stored f32 (mortonTree.js:130-137)
    m = P[b["perm"], 3].astype(np.float64)
    x = P[b["perm"], 0].astype(np.float64)
    cx = 0.0
    mm = 0.0
    for k in range(16):
        mm += m[k]
        cx += x[k] * m[k]
    assert n["mass"][1] == np.float32(mm) and n["com"][1][0] == np.float32(cx * (1 / mm))


def test_tree_identical20_known(oracle):
    P = np.zeros((20, 8), np.float32)
    P[:, :3] = 0.25
    P[:, 3] = 1.0
    b = oracle.sort_and_build(P, np.zeros((20, 4), np.float32))
    n = b["nodes"]
    assert b["rootSize"] == 1e-9
    assert b["levelRanges"].tolist() == [[d, 1] for d in range(11)]
    for d in range(10):
        assert n["isLeaf"][d] == 0 and n["children"][d].tolist() == [d + 1] + [-1] * 7
    assert (n["isLeaf"][10], n["first"][10], n["count"][10]) == (1, 0, 20)
    assert b["perm"].tolist() == list(range(20))


def test_empty_and_single(oracle):
    codes, root = oracle.compute_morton_codes(np.zeros(0, np.float32), 0, 8)
    assert root == -math.inf and codes.size == 0
    nodes, lr = oracle.tree_build(np.zeros(0, np.uint32), np.zeros(0), np.zeros(0), -math.inf)
    assert lr.tolist() == [[0, 1]] and nodes["isLeaf"].tolist() == [1] and nodes["count"][0] == 0
    P = np.zeros((1, 8), np.float32)
    P[0, 3] = 2.0
    b = oracle.sort_and_build(P, np.zeros((1, 4), np.float32))
    assert b["levelRanges"].tolist() == [[0, 1]] and b["nodes"]["mass"][0] == 2.0


@pytest.mark.parametrize("name", ["corners", "split17", "identical20", "nonfinite40", "ties300"])
def test_oracle_matches_python_transcription(oracle, name):
    d = np.load(os.path.join(GOLDEN, "golden_small.npz"))
    P = d[f"{name}/particles"]
    N = P.shape[0]
    codes, root = oracle.compute_morton_codes(P, N, 8)
    pc, proot = js_compute_morton_codes(P.ravel(), N, 8)
    assert np.array_equal(codes, pc) and (root == proot)
    perm = oracle.radix_sort_indices(codes)
    assert np.array_equal(perm, js_radix_sort(pc))
    nodes, lr = js_tree_topology(pc[perm], N)
    b = oracle.sort_and_build(P, np.zeros((N, 4), np.float32))
    assert b["levelRanges"].tolist() == lr
    got = b["nodes"]
    assert len(got) == len(nodes)
    for k, nd in enumerate(nodes):
        assert got["children"][k].tolist() == nd["children"]
        assert (got["isLeaf"][k], got["first"][k], got["count"][k]) == (nd["isLeaf"], nd["first"], nd["count"])
        assert got["size"][k] == np.float32(root * 0.5 ** nd["depth"])


def test_nonfinite_codes(oracle):
    d = np.load(os.path.join(GOLDEN, "golden_small.npz"))
    P = d["nonfinite40/particles"]
    codes, _ = oracle.compute_morton_codes(P, 40, 8)
    xbits = lambda c: c & 0x9249249  # noqa: E731
    assert xbits(int(codes[3])) == 0          # NaN x -> ToInt32(NaN) = 0
    assert (int(codes[7]) >> 1) & 0x9249249 == 0   # +inf y: (inf - min)*s = inf -> 0


def test_golden_small_fixtures(oracle):
    d = np.load(os.path.join(GOLDEN, "golden_small.npz"))
    names = sorted({k.split("/")[0] for k in d.files})
    for name in names:
        P = d[f"{name}/particles"]
        N = P.shape[0]
        codes, root = oracle.compute_morton_codes(P, N, 8)
        assert np.array_equal(codes, d[f"{name}/codes"]) and root == d[f"{name}/root_size"][0]
        b = oracle.sort_and_build(P, np.zeros((N, 4), np.float32))
        assert np.array_equal(b["perm"], d[f"{name}/perm"])
        assert np.array_equal(b["nodes"].view(np.uint32).reshape(-1, 16), d[f"{name}/nodes"])
        assert np.array_equal(b["levelRanges"], d[f"{name}/level_ranges"])


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_golden_disk16k(oracle):
    from galaxy_sim_b200 import initial_conditions as ic

    meta = json.load(open(os.path.join(GOLDEN, "golden_disk16k.json")))
    g = ic.disk_16k()
    assert _digest(g.particles) == meta["particles_sha256"]
    b = oracle.sort_and_build(g.particles, g.stellar)
    codes, root = oracle.compute_morton_codes(g.particles, g.N, 8)
    assert root == meta["root_size"]
    assert _digest(codes) == meta["codes_sha256"]
    assert _digest(b["perm"]) == meta["perm_sha256"]
    assert b["levelRanges"].tolist() == meta["level_ranges"]
    topo = np.stack([b["nodes"]["size"].view(np.uint32), b["nodes"]["isLeaf"], b["nodes"]["first"],
                     b["nodes"]["count"]], axis=1).astype(np.uint32)
    assert _digest(topo) == meta["topology_sha256"]
    assert _digest(b["nodes"]["children"]) == meta["children_sha256"]
    assert _digest(b["nodes"]["com"]) == meta["build_com_sha256"]
    refreshed = oracle.refresh_f32(b["sorted"], b["nodes"], b["levelRanges"])
    p = oracle.make_params(g.N, epsilon=0.05, theta=0.5, dt=0.005, haloMass=g.halo_mass,
                           haloA=g.halo_a, haloCenters=g.halo_centers)
    out, energy, acc4, dens, cnt = oracle.step_f32(p, b["sorted"], refreshed, want_forces=True)
    assert _digest(out) == meta["step_f32_sha256"]
    assert [int(x) for x in cnt] == meta["interactions"]


def test_worker_build_matches_bootstrap(oracle):
    """bhWorker.js:55-94 on a vec4 readback == sortAndBuild's topology on the same positions."""
    from galaxy_sim_b200 import initial_conditions as ic

    g = ic.disk_16k()
    pos4 = np.concatenate([g.particles[:, :3], np.ones((g.N, 1), np.float32)], 1)
    w = oracle.worker_build(pos4, g.particles[:, 3], 0, -1)
    b = oracle.sort_and_build(g.particles, g.stellar)
    assert np.array_equal(w["perm"], b["perm"])
    assert np.array_equal(w["nodes"], b["nodes"])
    assert w["energy"] == float(g.N)
    assert w["centralIdx"] == b["centralIdx"]


def test_pcg_and_rand01(oracle):
    def pcg(v0):
        v = (v0 * 747796405 + 2891336453) & 0xFFFFFFFF
        v = (((v >> ((v >> 28) + 4)) ^ v) * 277803737) & 0xFFFFFFFF
        return ((v >> 22) ^ v) & 0xFFFFFFFF
    for v in [0, 1, 12345, 0xFFFFFFFF, 0x9E3779B9]:
        assert oracle.pcg(v) == pcg(v)
    for i, salt in [(0, 1), (17, 978), (123456, 4889)]:
        want = np.float32(np.float32(pcg(i ^ ((salt * 0x9E3779B9) & 0xFFFFFFFF))) / np.float32(2 ** 32))
        assert oracle.rand01(i, salt) == want


def test_fp32_walk_close_to_fp64(oracle):
    """The FP32 restatement and the FP64 walk agree to FP32 rounding (same rule, same tree)."""
    from galaxy_sim_b200 import initial_conditions as ic

    g = ic.disk_16k()
    b = oracle.sort_and_build(g.particles, g.stellar)
    nodes = oracle.refresh_f32(b["sorted"], b["nodes"], b["levelRanges"])
    com = oracle.refresh_f64(b["sorted"], b["nodes"], b["levelRanges"])
    p = oracle.make_params(g.N, epsilon=0.05, theta=0.5, dt=0.005)
    _, _, acc4, _, _ = oracle.step_f32(p, b["sorted"], nodes, want_forces=True)
    acc64, pot64, _, _ = oracle.walk_f64(p, b["sorted"], nodes, com)
    rel = np.linalg.norm(acc4[:, :3] - acc64, axis=1) / np.linalg.norm(acc64, axis=1)
    assert np.median(rel) < 1e-5 and np.percentile(rel, 99) < 1e-3
    # against the direct sum: the truncation error of the reference's rule (softened
    # opening distance, theta = 0.5) is about 0.75% median on this disk
    t = np.arange(0, g.N, 64, dtype=np.uint32)
    accd, _ = oracle.direct_f64(p, b["sorted"], t)
    reld = np.linalg.norm(acc64[t] - accd, axis=1) / np.linalg.norm(accd, axis=1)
    assert np.median(reld) < 2e-2
