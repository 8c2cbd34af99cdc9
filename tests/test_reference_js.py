"""The oracle pinned to the reference's own code.

src/physics/mortonTree.js and src/physics/bhWorker.js are plain JavaScript; the
interpreter in oracle/jsmini.py runs their source text. Three layers:

* the interpreter's JavaScript semantics on small snippets (ToInt32, >>>,
  Float32Array rounding, NaN in Math.max, typed-array wrap-around, loops with
  continue, closures, classes and getters);
* where the reference checkout is present, the reference modules read at test
  time, on the crafted golden cases and the seeded 16384-particle disk, against
  the C++ oracle: Morton codes (strides 8 and 4), the sort permutation, the tree
  (every word of every 64-byte node), level ranges, sortAndBuild's outputs and
  two consecutive worker rebuilds, all bit for bit;
* everywhere, the C++ oracle against the fixtures the reference produced
  (tests/golden/reference_mortontree.npz and reference_digests.json, written
  by tests/golden/make_reference_golden.py), so the pin also holds on machines
  without the reference.
"""
import hashlib
import json
import math
import os

import numpy as np
import pytest

from galaxy_sim_b200 import initial_conditions as ic
from oracle import jsmini as J

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
REFERENCE = os.environ.get("GS_REFERENCE_ROOT", "/root/reference")
MORTON_JS = os.path.join(REFERENCE, "src", "physics", "mortonTree.js")
WORKER_JS = os.path.join(REFERENCE, "src", "physics", "bhWorker.js")
have_reference = pytest.mark.skipif(not os.path.exists(MORTON_JS), reason="reference checkout not present")


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _words(nodes):
    return np.ascontiguousarray(nodes).view(np.uint32).reshape(-1, 16)


# ---- the interpreter's semantics --------------------------------------------------------

SNIPPET = r"""
export function int32(x) { return x | 0; }
export function uint(x) { return x >>> 0; }
export function shl(x, s) { return x << s; }
export function f32(x) { const a = new Float32Array(1); a[0] = x; return a[0]; }
export function u32wrap(x) { const a = new Uint32Array(2); a[0] = x; a[1] = -1; return a[0] + a[1]; }
export function maxnan() { return Math.max(1, NaN, 3); }
export function finite(x) { return Number.isFinite(x); }
export function loop() {
  let s = 0;
  for (let i = 0; i < 10; i++) { if (i % 3 === 0) continue; s += i; }
  let k = 0;
  for (let j = 10; j > 0; j -= 2) { if (j === 6) continue; k += j; }
  return [s, k];
}
let counter = 0;
export function bump() { counter++; return counter; }
export class Box {
  constructor(n) { this.n = n; this.items = []; }
  add(v) { this.items.push(v); return this.items.length; }
  get twice() { return this.n * 2; }
}
export function arrow(a) { const f = (x) => x * a; return f(3) + (a ?? 100); }
export function div(a, b) { return a / b; }
export function neg0() { return -0; }
"""


def test_interpreter_semantics():
    m = J.run_source(SNIPPET)
    call = lambda name, *a: J.call_value(m[name], None, list(a))  # noqa: E731
    assert call("int32", 2 ** 31 + 5.7) == -(2 ** 31) + 5
    assert call("int32", -7.9) == -7 and call("int32", math.nan) == 0 and call("int32", math.inf) == 0
    assert call("uint", -1) == 0xFFFFFFFF
    assert call("shl", 1, 31) == -(2 ** 31) and call("shl", 1, 33) == 2
    assert call("f32", 0.1) == float(np.float32(0.1)) and call("f32", 1e39) == math.inf
    assert call("u32wrap", 2 ** 32 + 3) == 3 + 0xFFFFFFFF
    assert math.isnan(call("maxnan"))
    assert call("finite", 1.5) and not call("finite", math.inf) and not call("finite", math.nan)
    assert list(call("loop")) == [1 + 2 + 4 + 5 + 7 + 8, 10 + 8 + 4 + 2]
    assert call("bump") == 1 and call("bump") == 2
    box = J.construct(m["Box"], [21])
    assert J.call_method(box, "add", [5]) == 1 and J.call_method(box, "add", [6]) == 2
    assert J.get_prop(box, "twice") == 42
    assert call("arrow", 2) == 8 and call("arrow", None) != call("arrow", None)   # NaN + 100 -> NaN
    assert call("div", 1, 0) == math.inf and call("div", -1, 0) == -math.inf and math.isnan(call("div", 0, 0))
    assert math.copysign(1.0, call("neg0")) < 0
    with pytest.raises(J.JsSyntaxError):
        J.run_source("export function f() { try { return 1; } catch (e) { return 2; } }")


# ---- the reference's own modules, read at test time, against the C++ oracle -------------

def _ref_sort_and_build(m, P, S, track2):
    N = P.shape[0]
    r = J.call_value(m["sortAndBuild"], None, [J.from_numpy(P.reshape(-1)), J.from_numpy(S.reshape(-1)), N,
                                                track2])
    t = J.get_prop(r, "tree")
    nn = int(J.get_prop(t, "numNodes"))
    return {"perm": J.to_numpy(J.get_prop(r, "perm")).astype(np.uint32),
            "nodes": np.frombuffer(bytes(J.get_prop(t, "_buf").data[: nn * 64]), np.uint32).reshape(-1, 16),
            "levelRanges": J.to_numpy(J.get_prop(t, "levelRanges")).astype(np.uint32).reshape(-1, 2),
            "sorted": J.to_numpy(J.get_prop(r, "sorted")).reshape(-1, 8),
            "sortedStellar": J.to_numpy(J.get_prop(r, "sortedStellar")).reshape(-1, 4),
            "central": (J.get_prop(r, "centralIdx"), J.get_prop(r, "centralIdx2")),
            "masses": J.to_numpy(J.get_prop(r, "masses"))}


def _ref_codes(m, P, stride):
    N = P.shape[0]
    codes = J.construct("Uint32Array", [N])
    root = J.call_value(m["computeMortonCodes"], None, [J.from_numpy(np.ascontiguousarray(P).reshape(-1)), N,
                                                        stride, codes])
    return J.to_numpy(codes).astype(np.uint32), root


@have_reference
def test_reference_mortontree_js_equals_the_oracle(oracle):
    import sys

    sys.path.insert(0, GOLDEN)
    from make_golden import crafted_cases

    m = J.load_module(MORTON_JS)
    cases = dict(crafted_cases())
    cases["disk16k"] = ic.disk_16k().particles
    for name, P in cases.items():
        N = P.shape[0]
        S = np.random.default_rng(N).uniform(0, 1, (N, 4)).astype(np.float32)
        for stride, arr in ((8, P), (4, np.ascontiguousarray(P[:, :4]))):
            got, root = _ref_codes(m, arr, stride)
            want, wroot = oracle.compute_morton_codes(arr, N, stride)
            assert np.array_equal(got, want) and root == wroot, (name, stride)
        r = _ref_sort_and_build(m, P, S, N // 2)
        w = oracle.sort_and_build(P, S, track_idx2=N // 2)
        assert np.array_equal(r["perm"], w["perm"]), name
        assert np.array_equal(r["nodes"], _words(w["nodes"])), name
        assert np.array_equal(r["levelRanges"], w["levelRanges"]), name
        assert np.array_equal(r["sorted"].view(np.uint32), w["sorted"].view(np.uint32)), name
        assert np.array_equal(r["sortedStellar"].view(np.uint32), w["sortedStellar"].view(np.uint32)), name
        assert r["central"] == (w["centralIdx"], w["centralIdx2"]), name
        assert np.array_equal(r["masses"].view(np.uint32), w["masses"].view(np.uint32)), name


@have_reference
def test_reference_worker_js_equals_the_oracle(oracle):
    sent = []
    me = J.JSObject()
    me.props["postMessage"] = J.JSFunction(lambda this, msg=None, *rest: sent.append(msg))
    J.load_module(WORKER_JS, self_object=me)

    def post(msg):
        J.call_value(me.props["onmessage"], None, [J.JSObject({"data": J.JSObject(msg)})])
        return sent[-1] if sent else None

    g = ic.two_galaxy_collision(6000, 3)
    N = g.N
    rng = np.random.default_rng(4)
    masses = g.particles[:, 3].copy()
    c1, c2 = 0, N // 2
    post({"type": "config", "N": N, "masses": J.from_numpy(masses), "centralIdx": c1, "centralIdx2": c2})
    post({"type": "centralMass", "value": 0.5})            # updateCentralMass (NBodyGPU.js / main.js)
    masses[c1] = 0.5
    pos4 = np.concatenate([g.particles[:, :3], rng.normal(0, 1, (N, 1))], 1).astype(np.float32)
    for _ in range(2):
        msg = post({"type": "build", "positions": J.from_numpy(pos4.reshape(-1))})
        w = oracle.worker_build(pos4, masses, c1, c2)
        assert bytes(J.get_prop(msg, "tree").data) == w["nodes"].tobytes()
        assert np.array_equal(J.to_numpy(J.get_prop(msg, "perm")), w["perm"])
        assert np.array_equal(J.to_numpy(J.get_prop(msg, "levelRanges")), w["levelRanges"])
        assert (J.get_prop(msg, "centralIdx"), J.get_prop(msg, "centralIdx2")) == (w["centralIdx"],
                                                                                   w["centralIdx2"])
        assert J.get_prop(msg, "energy") == w["energy"]
        assert np.array_equal(J.to_numpy(J.get_prop(msg, "bh1")), w["bh1"])
        assert np.array_equal(J.to_numpy(J.get_prop(msg, "bh2")), w["bh2"])
        masses, c1, c2 = w["masses"], w["centralIdx"], w["centralIdx2"]
        pos4 = pos4[w["perm"]].copy()
        pos4[:, :3] += rng.normal(0, 0.01, (N, 3)).astype(np.float32)


# ---- the C++ oracle against what the reference produced ---------------------------------

def _fixture():
    return np.load(os.path.join(GOLDEN, "reference_mortontree.npz"))


def _case_names(f):
    return sorted({k.split("/")[0] for k in f.files if not k.startswith(("worker_", "sort_"))})


def test_oracle_equals_reference_fixtures(oracle):
    f = _fixture()
    names = _case_names(f)
    assert {"empty", "single", "coincident40", "farclusters600", "split17", "nonfinite40"} <= set(names)
    for name in names:
        P, S = f[f"{name}/particles"], f[f"{name}/stellar"]
        N = P.shape[0]
        codes, root = oracle.compute_morton_codes(P, N, 8)
        assert np.array_equal(codes, f[f"{name}/codes"]), name
        assert root == f[f"{name}/root_size"][0] or (math.isinf(root) and math.isinf(f[f"{name}/root_size"][0]))
        codes4, root4 = oracle.compute_morton_codes(np.ascontiguousarray(P[:, :4]), N, 4)
        assert np.array_equal(codes4, f[f"{name}/codes_stride4"]), name
        perm = oracle.radix_sort_indices(codes)
        assert np.array_equal(perm, f[f"{name}/perm"]), name
        if N:
            nodes, lr = oracle.tree_build(codes[perm], np.ascontiguousarray(P[perm, :3]), P[perm, 3].copy(), root)
            assert np.array_equal(_words(nodes), f[f"{name}/nodes"]), name
            assert np.array_equal(lr, f[f"{name}/level_ranges"]), name
        w = oracle.sort_and_build(P, S, track_idx2=N // 2)
        assert np.array_equal(_words(w["nodes"]), f[f"{name}/sab_nodes"]), name
        assert np.array_equal(w["levelRanges"], f[f"{name}/level_ranges"]), name
        assert np.array_equal(w["sorted"].view(np.uint32), f[f"{name}/sab_sorted"].view(np.uint32)), name
        assert np.array_equal(w["sortedStellar"].view(np.uint32),
                              f[f"{name}/sab_sorted_stellar"].view(np.uint32)), name
        assert [w["centralIdx"], w["centralIdx2"]] == f[f"{name}/sab_central"].tolist(), name
        assert np.array_equal(w["masses"].view(np.uint32), f[f"{name}/sab_masses"].view(np.uint32)), name
    assert np.array_equal(oracle.radix_sort_indices(f["sort_highbits/codes"]), f["sort_highbits/perm"])


def test_oracle_worker_equals_reference_fixtures(oracle):
    f = _fixture()
    for name in sorted({k.split("/")[0] for k in f.files if k.startswith("worker_")}):
        masses = f[f"{name}/masses"]
        c1, c2 = f[f"{name}/central_in"].tolist()
        for k in range(2):
            w = oracle.worker_build(f[f"{name}/pos4_{k}"], masses, c1, c2)
            assert np.array_equal(_words(w["nodes"]), f[f"{name}/nodes_{k}"]), (name, k)
            assert np.array_equal(w["perm"], f[f"{name}/perm_{k}"]), (name, k)
            assert np.array_equal(w["levelRanges"].reshape(-1), f[f"{name}/level_ranges_{k}"].reshape(-1))
            assert [w["centralIdx"], w["centralIdx2"]] == f[f"{name}/central_{k}"].tolist(), (name, k)
            assert w["energy"] == f[f"{name}/energy_{k}"][0], (name, k)
            assert np.array_equal(np.stack([w["bh1"], w["bh2"]]), f[f"{name}/bh_{k}"]), (name, k)
            masses, c1, c2 = w["masses"], w["centralIdx"], w["centralIdx2"]


def test_oracle_equals_reference_digests(oracle):
    d = json.load(open(os.path.join(GOLDEN, "reference_digests.json")))
    g = ic.disk_16k()
    N = g.N
    e = d["disk16k"]
    assert _digest(g.particles) == e["particles_sha256"], "the seeded disk changed"
    codes, root = oracle.compute_morton_codes(g.particles, N, 8)
    assert _digest(codes) == e["codes_sha256"] and root == e["root_size"]
    w = oracle.sort_and_build(g.particles, g.stellar, track_idx2=N // 2)
    assert _digest(w["perm"]) == e["perm_sha256"]
    assert _digest(_words(w["nodes"])) == e["nodes_sha256"]
    assert w["levelRanges"].tolist() == e["level_ranges"]
    assert _digest(w["sorted"]) == e["sorted_sha256"]
    assert _digest(w["sortedStellar"]) == e["sorted_stellar_sha256"]
    assert [w["centralIdx"], w["centralIdx2"]] == e["central"]
    # MortonTree's third leaf clause with a 4096-node pool: in the reference the
    # children already queued still get numbers past the pool (numNodes ends above
    # maxNodes, the writes past it are dropped); the oracle refuses such a build
    e = d["disk32k_pool4096"]
    assert e["overflow"] and e["js_num_nodes"] > e["max_nodes"]
    g = ic.galaxy_disk(32768, 77)
    P = g.particles
    assert _digest(P) == e["particles_sha256"]
    codes, root = oracle.compute_morton_codes(P, P.shape[0], 8)
    perm = oracle.radix_sort_indices(codes)
    assert _digest(perm) == e["perm_sha256"]
    with pytest.raises(RuntimeError):
        oracle.tree_build(codes[perm], np.ascontiguousarray(P[perm, :3]), P[perm, 3].copy(), root,
                          max_nodes=e["max_nodes"])
    nodes, _ = oracle.tree_build(codes[perm], np.ascontiguousarray(P[perm, :3]), P[perm, 3].copy(), root)
    assert len(nodes) == e["full_num_nodes"]
