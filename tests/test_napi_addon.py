"""The Node-API addon (addon/galaxy_napi.c) through a mock Node-API runtime.

No JavaScript engine exists here, so the addon is compiled against
tests/napi/node_api.h (documented Node-API prototypes) and linked with
tests/napi/mock_node_api.c, a small in-process implementation of those
functions; the tests below play the part of main.js. They check the
marshalling the addon does: typed-array extraction and length checks, the
updateParams object with the reference's defaults, levelRanges as an array of
[start, count] pairs, the tree ArrayBuffer, BigInt device pointers, the
readPositions promise, thrown TypeError / RangeError / library errors, and the
silent no-ops after destroy(). On a GPU the NBodyCUDA call sequence of main.js
must give bit-identical results to the same calls made directly through the C
ABI, and the mortonTree.js exports must equal the oracle bit for bit.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F32, U32, I32 = 7, 6, 5                  # napi_typedarray_type values
K_UNDEF, K_NUM, K_OBJ, K_ARR, K_FUNC, K_TA, K_AB, K_BIGINT, K_PROMISE = 0, 3, 5, 6, 7, 8, 9, 10, 11


class JSError(Exception):
    def __init__(self, name, code, message):
        super().__init__(f"{name} [{code}] {message}")
        self.name, self.code, self.message = name, code, message


class H:
    """A handle to a value of the mock runtime (as opposed to a Python number)."""

    __slots__ = ("p",)

    def __init__(self, p):
        self.p = p


class JS:
    """The addon's exports, called the way JavaScript would call them."""

    def __init__(self, so):
        L = C.CDLL(so)
        vp = C.c_void_p
        for name, res, args in [
            ("mock_env", vp, []), ("mock_load", vp, [vp]), ("mock_number", vp, [C.c_double]),
            ("mock_bool", vp, [C.c_int]), ("mock_undefined", vp, []), ("mock_null", vp, []),
            ("mock_string", vp, [C.c_char_p]), ("mock_object", vp, []), ("mock_array", vp, []),
            ("mock_array_push", None, [vp, vp]), ("mock_set", None, [vp, C.c_char_p, vp]),
            ("mock_arraybuffer", vp, [vp, C.c_size_t]), ("mock_typedarray", vp, [C.c_int, vp, C.c_size_t]),
            ("mock_get", vp, [vp, vp, C.c_char_p]), ("mock_new", vp, [vp, vp, C.c_size_t, vp]),
            ("mock_call_method", vp, [vp, vp, C.c_char_p, C.c_size_t, vp]),
            ("mock_take_exception", C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]),
            ("mock_kind", C.c_int, [vp]), ("mock_num", C.c_double, [vp]), ("mock_bool_of", C.c_int, [vp]),
            ("mock_str", C.c_char_p, [vp]), ("mock_bigint", C.c_uint64, [vp]),
            ("mock_array_len", C.c_uint32, [vp]), ("mock_array_get", vp, [vp, C.c_uint32]),
            ("mock_ta_type", C.c_int, [vp]), ("mock_ta_len", C.c_size_t, [vp]), ("mock_ta_data", vp, [vp]),
            ("mock_ta_buffer", vp, [vp]), ("mock_ab_data", vp, [vp]), ("mock_ab_len", C.c_size_t, [vp]),
            ("mock_promise_state", C.c_int, [vp]), ("mock_promise_result", vp, [vp]),
            ("mock_has_own", C.c_int, [vp, C.c_char_p]), ("mock_prototype", vp, [vp]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.L = L
        self.env = L.mock_env()
        self.exports = H(L.mock_load(self.env))
        self._keep = []

    # values
    def val(self, x):
        L = self.L
        if isinstance(x, H):
            return x.p
        if x is None:
            return L.mock_undefined()
        if isinstance(x, bool):
            return L.mock_bool(int(x))
        if isinstance(x, (int, float, np.floating, np.integer)):
            return L.mock_number(float(x))
        if isinstance(x, str):
            return L.mock_string(x.encode())
        if isinstance(x, np.ndarray):
            kind = {np.dtype(np.float32): F32, np.dtype(np.uint32): U32, np.dtype(np.int32): I32}[x.dtype]
            assert x.flags.c_contiguous
            self._keep.append(x)
            return L.mock_typedarray(kind, x.ctypes.data, x.size)
        if isinstance(x, (list, tuple)):
            a = L.mock_array()
            for e in x:
                L.mock_array_push(a, self.val(e))
            return a
        if isinstance(x, dict):
            o = L.mock_object()
            for k, v in x.items():
                L.mock_set(o, k.encode(), self.val(v))
            return o
        raise TypeError(type(x))

    def _check(self):
        name, code, msg = (C.create_string_buffer(512) for _ in range(3))
        if self.L.mock_take_exception(self.env, name, code, msg, 512):
            raise JSError(name.value.decode(), code.value.decode(), msg.value.decode())

    def _argv(self, args):
        hs = [self.val(a) for a in args]
        arr = (C.c_void_p * max(1, len(hs)))(*hs)
        self._keep.append(arr)
        return arr, len(hs)

    def new(self, cls, *args):
        argv, n = self._argv(args)
        h = self.L.mock_new(self.env, cls.p, n, argv)
        self._check()
        return H(h)

    def call(self, obj, name, *args):
        argv, n = self._argv(args)
        h = self.L.mock_call_method(self.env, obj.p, name.encode(), n, argv)
        self._check()
        return H(h)

    def get(self, obj, key):
        h = self.L.mock_get(self.env, obj.p, key.encode())
        self._check()
        return H(h)

    def kind(self, h):
        return self.L.mock_kind(h.p)

    def promise_state(self, h):
        return self.L.mock_promise_state(h.p)

    def has_own(self, h, key):
        return bool(self.L.mock_has_own(h.p, key.encode()))

    def prototype(self, cls):
        return H(self.L.mock_prototype(cls.p))

    def py(self, h):
        """A Python copy of a returned value (numbers, booleans, strings, BigInts,
        arrays, typed arrays, ArrayBuffers); other values stay handles."""
        L, p = self.L, h.p
        k = L.mock_kind(p)
        if k == K_UNDEF:
            return None
        if k == K_NUM:
            return L.mock_num(p)
        if k == 2:
            return bool(L.mock_bool_of(p))
        if k == 4:
            return L.mock_str(p).decode()
        if k == K_BIGINT:
            return int(L.mock_bigint(p))
        if k == K_ARR:
            return [self.py(H(L.mock_array_get(p, i))) for i in range(L.mock_array_len(p))]
        if k == K_TA:
            dt = {F32: np.float32, U32: np.uint32, I32: np.int32}[L.mock_ta_type(p)]
            n = L.mock_ta_len(p)
            return np.frombuffer((C.c_char * (n * 4)).from_address(L.mock_ta_data(p)), dt).copy()
        if k == K_AB:
            n = L.mock_ab_len(p)
            return bytes((C.c_char * n).from_address(L.mock_ab_data(p)))
        return h


@pytest.fixture(scope="module")
def js(tmp_path_factory):
    from galaxy_sim_b200 import build

    build.build()
    so = str(tmp_path_factory.mktemp("napi") / "galaxy_napi_mock.so")
    cmd = ["gcc", "-O1", "-Wall", "-Wextra", "-Werror", "-shared", "-fPIC",
           "-I", os.path.join(ROOT, "tests", "napi"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "addon", "galaxy_napi.c"), os.path.join(ROOT, "tests", "napi", "mock_node_api.c"),
           "-L", os.path.join(ROOT, "galaxy_sim_b200"), "-lgalaxy_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "galaxy_sim_b200"), "-lm", "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return JS(so)


METHODS = ["applyPermutation", "updateCentralMass", "updateParams", "encodeStarFormation", "uploadBHTree",
           "encodeRefresh", "step", "encodePositionReadback", "readPositions", "destroy", "sortBuild", "run",
           "sync", "energy", "setTracking", "getTracking", "deviceErrors"]


def test_addon_exports_the_nbodygpu_and_mortontree_surface(js):
    cls = js.get(js.exports, "NBodyCUDA")
    assert js.kind(cls) == K_FUNC
    for f in ("computeMortonCodes", "radixSortIndices", "buildTree", "sortAndBuild"):
        assert js.kind(js.get(js.exports, f)) == K_FUNC, f
    assert js.has_own(js.exports, "NBodyCUDA")
    proto = js.prototype(cls)
    for m in METHODS:
        assert js.kind(js.get(proto, m)) == K_FUNC, m
    assert js.has_own(proto, "positionBuffer") and js.has_own(proto, "stellarBuffer")


def test_addon_rejects_bad_arguments_before_any_cuda_call(js):
    cls = js.get(js.exports, "NBodyCUDA")
    with pytest.raises(JSError) as e:
        js.new(cls, 0, "not a typed array")
    assert e.value.name == "TypeError"
    with pytest.raises(JSError) as e:
        js.new(cls, 0, np.zeros(7, np.float32))
    assert e.value.name == "RangeError" and "8 floats" in e.value.message
    with pytest.raises(JSError) as e:
        js.new(cls, 0, np.zeros(16, np.float32), np.zeros(5, np.float32))
    assert e.value.name == "RangeError" and "4 floats" in e.value.message
    with pytest.raises(JSError) as e:
        js.new(cls, -1, np.zeros(16, np.float32))
    assert e.value.name == "RangeError"
    f = js.get(js.exports, "computeMortonCodes")
    with pytest.raises(JSError) as e:
        js.call(js.exports, "computeMortonCodes")
    assert e.value.name == "TypeError"
    with pytest.raises(JSError) as e:
        js.call(js.exports, "computeMortonCodes", np.zeros(30, np.float32), 10, 3, np.zeros(4, np.uint32))
    assert e.value.name == "RangeError"
    assert f


def test_addon_reports_library_errors_as_gs_codes(js):
    """A failing gs_* call becomes an Error whose code names the status and whose
    message is gs_last_error(); without a GPU every CUDA call fails that way."""
    from galaxy_sim_b200 import _lib

    codes = np.arange(4, dtype=np.uint32)[::-1].copy()
    idx = np.zeros(4, np.uint32)
    args = (codes, idx, np.zeros(4, np.uint32), np.zeros(1024, np.uint32), 4)
    cls = js.get(js.exports, "NBodyCUDA")
    if _lib.device_count() == 0:
        with pytest.raises(JSError) as e:
            js.call(js.exports, "radixSortIndices", *args)
        assert e.value.name == "Error" and e.value.code.startswith("GS_E") and e.value.message
        with pytest.raises(JSError) as e:
            js.new(cls, 0, np.zeros(16, np.float32))
        assert e.value.code.startswith("GS_E")
    else:
        h = js.call(js.exports, "radixSortIndices", *args)
        assert list(js.py(h)) == [3, 2, 1, 0]
    # an empty sort is a no-op that returns the indices array
    h = js.call(js.exports, "radixSortIndices", codes, idx, np.zeros(4, np.uint32), np.zeros(1024, np.uint32), 0)
    assert js.kind(h) == K_TA


# ---- on the GPU --------------------------------------------------------------------------

def _params(g):
    return dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5, haloMass=g.halo_mass, haloA=g.halo_a,
                gasDrag=0.25, time=0.0, agingRate=25.0, sfDensity=g.sf_density * 0.2, sfEff=0.5, sfDt=0.005,
                haloCenters=[[0.0, 0.0, 0.0, 0.0]])


@pytest.mark.gpu
def test_addon_nbodycuda_equals_the_c_abi(js, gpu_lib):
    from galaxy_sim_b200 import initial_conditions as ic
    from galaxy_sim_b200 import morton_tree as mt
    from galaxy_sim_b200.nbody_gpu import NBodyGPU

    g = ic.galaxy_disk(6000, 21, gas_frac=0.3)
    N = g.N
    P = np.ascontiguousarray(g.particles.reshape(-1))
    S = np.ascontiguousarray(g.stellar.reshape(-1))
    prm = _params(g)
    # main.js bootstrap (:272-288): sortAndBuild on the host, applyPermutation,
    # uploadBHTree, then frames of updateParams + encodeRefresh + step + encodeStarFormation
    cls = js.get(js.exports, "NBodyCUDA")
    sim = js.new(cls, 0, P, S)
    assert js.py(js.get(sim, "N")) == N and js.py(js.get(sim, "ready")) is True
    boot = js.call(js.exports, "sortAndBuild", P, S, N, -1)
    perm = js.py(js.get(boot, "perm"))
    tree = js.get(boot, "tree")
    buf, num = js.get(tree, "_buf"), int(js.py(js.get(tree, "numNodes")))
    levels = js.py(js.get(tree, "levelRanges"))
    js.call(sim, "updateParams", prm)
    js.call(sim, "applyPermutation", None, perm)
    js.call(sim, "uploadBHTree", buf, num, levels)
    for _ in range(2):
        js.call(sim, "encodeRefresh", None)
        js.call(sim, "step", None)
    js.call(sim, "encodeStarFormation", None)
    js.call(sim, "encodePositionReadback", None)
    out = np.zeros(4 * N, np.float32)
    pr = js.call(sim, "readPositions", out)
    assert js.kind(pr) == K_PROMISE and js.promise_state(pr) == 1
    assert js.py(js.get(sim, "positionBuffer")) != 0 and js.py(js.get(sim, "stellarBuffer")) != 0
    e = js.call(sim, "energy")
    got_e = [js.py(js.get(e, k)) for k in ("eDiag", "eTrue", "mass")] + js.py(js.get(e, "momentum"))

    # the same calls through the C ABI (the Python mirror of NBodyGPU)
    ref = NBodyGPU(0, g.particles, g.stellar)
    ref.updateParams(**prm)
    b = mt.sortAndBuild(g.particles.ravel(), g.stellar.ravel(), N)
    assert np.array_equal(perm, b["perm"])
    assert num == b["tree"].numNodes and levels == [list(map(int, r)) for r in b["tree"].levelRanges]
    ref.applyPermutation(None, b["perm"])
    ref.uploadBHTree(b["tree"].nodes, b["tree"].numNodes, b["tree"].levelRanges)
    for _ in range(2):
        ref.encodeRefresh()
        ref.step()
    ref.encodeStarFormation()
    want = ref.readPositions()
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
    we = ref.energy()
    assert got_e == [we["e_diag"], we["e_true"], we["mass"]] + list(we["momentum"])

    # on-device rebuild and graph-replayed steps, with halo tracking
    js.call(sim, "setTracking", 0, -1, [0.0, 0.0, 0.0])
    ref.setTracking(0, -1, [0.0, 0.0, 0.0], None)
    js.call(sim, "sortBuild")
    js.call(sim, "run", 3, True)
    js.call(sim, "sync", 10000)
    ref.sortBuild()
    ref.run(3, True)
    js.call(sim, "readPositions", out)
    assert np.array_equal(out.view(np.uint32), ref.readPositions().view(np.uint32))
    tr = js.call(sim, "getTracking")
    assert js.py(js.get(tr, "centralIdx")) == ref.getTracking()[0]
    assert js.py(js.call(sim, "deviceErrors")) == 0
    ref.destroy()

    # argument errors on a live simulation, then destroy: later calls are silent no-ops
    with pytest.raises(JSError) as err:
        js.call(sim, "applyPermutation", None, np.zeros(N - 1, np.uint32))
    assert err.value.name == "RangeError"
    with pytest.raises(JSError) as err:
        js.call(sim, "readPositions", np.zeros(4 * N - 1, np.float32))
    assert err.value.name == "RangeError"
    with pytest.raises(JSError) as err:
        js.call(sim, "updateParams", 3)
    assert err.value.name == "TypeError"
    js.call(sim, "destroy")
    assert js.py(js.get(sim, "ready")) is False
    assert js.kind(js.call(sim, "step", None)) == K_UNDEF
    assert js.kind(js.call(sim, "run", 2, True)) == K_UNDEF
    pr = js.call(sim, "readPositions", out)
    assert js.promise_state(pr) == 1


@pytest.mark.gpu
def test_addon_mortontree_exports_equal_the_oracle(js, gpu_lib, oracle):
    from galaxy_sim_b200 import initial_conditions as ic

    g = ic.two_galaxy_collision(5000, 8)
    N = g.N
    P = np.ascontiguousarray(g.particles.reshape(-1))
    S = np.ascontiguousarray(g.stellar.reshape(-1))
    for stride, arr in ((8, P), (4, np.ascontiguousarray(g.particles[:, :4]).reshape(-1))):
        codes = np.zeros(N, np.uint32)
        root = js.py(js.call(js.exports, "computeMortonCodes", arr, N, stride, codes))
        want, wroot = oracle.compute_morton_codes(arr, N, stride)
        assert np.array_equal(codes, want) and root == wroot
    codes, root = oracle.compute_morton_codes(P, N, 8)
    idx = np.zeros(N, np.uint32)
    h = js.call(js.exports, "radixSortIndices", codes, idx, np.zeros(N, np.uint32), np.zeros(1024, np.uint32), N)
    perm = oracle.radix_sort_indices(codes)
    assert np.array_equal(js.py(h), perm) and np.array_equal(idx, perm)
    pos = np.ascontiguousarray(g.particles[perm, :3]).reshape(-1)
    m = np.ascontiguousarray(g.particles[perm, 3])
    t = js.call(js.exports, "buildTree", codes[perm].copy(), pos, m, N, root)
    nodes, lr = oracle.tree_build(codes[perm], pos, m, root)
    num = int(js.py(js.get(t, "numNodes")))
    assert num == len(nodes) and js.py(js.get(t, "maxNodes")) == 2 * N + 4096
    assert js.py(js.get(t, "_buf"))[: 64 * num] == nodes.tobytes()
    assert js.py(js.get(t, "levelRanges")) == lr.tolist()
    b = js.call(js.exports, "sortAndBuild", P, S, N, N // 2)
    w = oracle.sort_and_build(g.particles, g.stellar, track_idx2=N // 2)
    assert np.array_equal(js.py(js.get(b, "perm")), w["perm"])
    assert np.array_equal(js.py(js.get(b, "sorted")).view(np.uint32), w["sorted"].reshape(-1).view(np.uint32))
    assert np.array_equal(js.py(js.get(b, "sortedStellar")).view(np.uint32),
                          w["sortedStellar"].reshape(-1).view(np.uint32))
    assert np.array_equal(js.py(js.get(b, "masses")).view(np.uint32), w["masses"].view(np.uint32))
    assert (js.py(js.get(b, "centralIdx")), js.py(js.get(b, "centralIdx2"))) == (w["centralIdx"], w["centralIdx2"])
    bt = js.get(b, "tree")
    assert js.py(js.get(bt, "_buf"))[: 64 * len(w["nodes"])] == w["nodes"].tobytes()
    # the f32 / i32 views share the tree's buffer, as MortonTree's do
    f32 = js.py(js.get(bt, "f32"))
    assert f32[4] == w["nodes"]["size"][0]
