"""Mirror of galaxy-sim's ``NBodyGPU`` class (src/physics/NBodyGPU.js:14-369).

One instance owns one ``gs_ctx`` of the CUDA library: the same ping-pong
particle and stellar buffers, the same 96-byte Params, the same method names
and argument meaning. ``commandEncoder`` arguments are accepted and ignored:
every call is ordered on the context's CUDA stream, which plays the encoder's
role. Where the JavaScript silently returns while not ``ready`` (after
``destroy``), so do these methods; CUDA failures raise ``GalaxyError``.

Beyond the reference's surface, ``sortBuild`` replaces the Web-Worker rebuild
round trip (bhWorker.js) with an on-device one, and ``run`` replays full steps
(rebuild + walk [+ star formation]) from a CUDA graph.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import NODE_DTYPE, GsDiag, GsParams, check, f32, lib, ptr, u32


def build_params(N, *, dt, G, epsilon, theta=0.5, haloMass=0, haloA=1, gasDrag=0, time=0,
                 agingRate=25, sfDensity=1e9, sfEff=0, sfDt=0, haloCenters=()) -> GsParams:
    """The Params uniform NBodyGPU.updateParams writes (NBodyGPU.js:253-275):
    epsilon * epsilon in double rounded to f32 (the Float32Array store), N
    forced, at most two halo centres."""
    p = GsParams()
    p.dt, p.G = dt, G
    p.epsilon2 = float(np.float32(float(epsilon) * float(epsilon)))  # double product, f32 store
    p.N = int(N)
    p.theta, p.haloMass, p.haloA, p.gasDrag = theta, haloMass, haloA, gasDrag
    p.time, p.agingRate, p.sfDensity, p.sfEff, p.sfDt = time, agingRate, sfDensity, sfEff, sfDt
    hc = list(haloCenters or [])
    p.haloCount = min(len(hc), 2)
    for h, c in enumerate(hc[:2]):
        arr = p.haloC1 if h == 0 else p.haloC2
        for k in range(min(len(c), 4)):
            arr[k] = c[k]
    return p


class NBodyGPU:
    def __init__(self, device, particleData, stellarData=None, walkGroup=None, walkSplit=None):
        """walkGroup: particles a warp walks together (4, 8, 16, 32, or 0 = by
        size, the default of a single-galaxy context; a pool uses 32).
        walkSplit: parts each work item's walk is split into (1, 2, 4, 8, or 0 =
        by size, the default; a pool of several galaxies walks unsplit, 1).
        ``walkGroup=32, walkSplit=1`` gives a galaxy a pool's arithmetic."""
        P = f32(particleData).ravel()
        if P.size % 8:
            raise ValueError("particleData must hold 8 floats per particle")
        self.N = P.size // 8
        self.device = int(device or 0)
        S = None if stellarData is None else f32(stellarData).ravel()
        if S is not None and S.size != 4 * self.N:
            raise ValueError("stellarData must hold 4 floats per particle")
        h = C.c_void_p()
        check(lib().gs_create_on(self.device, self.N, ptr(P), ptr(S), C.byref(h)))
        self._ctx = h
        self.ready = True
        self.levelRanges = None
        self._params = GsParams()
        from ._lib import TUNE_WALK_GROUP, TUNE_WALK_SPLIT

        if walkGroup is not None:
            self._ok(lib().gs_set_tuning(self._ctx, TUNE_WALK_GROUP, int(walkGroup)))
        if walkSplit is not None:
            self._ok(lib().gs_set_tuning(self._ctx, TUNE_WALK_SPLIT, int(walkSplit)))

    # -- reference surface --------------------------------------------------------------
    def _ok(self, rc):
        check(rc, self._ctx)

    def applyPermutation(self, commandEncoder, perm):
        """NBodyGPU.js:225-238: gather out[i] = in[perm[i]], flip both ping-pongs."""
        if not self.ready:
            return
        p = u32(perm)
        if p.size != self.N:
            raise ValueError("perm must hold N indices")
        self._ok(lib().gs_apply_permutation(self._ctx, ptr(p)))

    @property
    def stellarBuffer(self) -> int:
        d = C.c_void_p()
        self._ok(lib().gs_stellar_buffer(self._ctx, C.byref(d)))
        return d.value

    def updateCentralMass(self, mass, idx=0):
        self._ok(lib().gs_update_central_mass(self._ctx, float(mass), int(idx)))

    def updateParams(self, **kw):
        """NBodyGPU.js:253-275 (keyword arguments of ``build_params``)."""
        p = build_params(self.N, **kw)
        self._params = p
        self._ok(lib().gs_update_params(self._ctx, C.byref(p)))

    def encodeStarFormation(self, commandEncoder=None):
        if not self.ready:
            return
        self._ok(lib().gs_star_formation(self._ctx))

    def uploadBHTree(self, treeBuffer, numNodes, levelRanges=None):
        """NBodyGPU.js:288-301: a flat 64-byte-node buffer (bytes, uint8/float32/struct array)."""
        if not self.ready:
            return
        raw = np.frombuffer(memoryview(treeBuffer).cast("B"), np.uint8) if not isinstance(
            treeBuffer, np.ndarray) else treeBuffer.view(np.uint8).ravel()
        nodes = np.ascontiguousarray(raw[: int(numNodes) * 64]).view(NODE_DTYPE)
        lr = None
        nl = 0
        if levelRanges is not None:
            lr = u32(np.asarray(levelRanges, dtype=np.uint32).reshape(-1, 2)[:16])
            nl = lr.shape[0]
            self.levelRanges = [list(map(int, r)) for r in lr]
        self._ok(lib().gs_upload_tree(self._ctx, ptr(nodes), int(numNodes), ptr(lr), nl))

    def encodeRefresh(self, commandEncoder=None):
        """NBodyGPU.js:308-319: COM re-sum from the current positions, deepest level first."""
        if not self.ready:
            return
        self._ok(lib().gs_refresh(self._ctx))

    def step(self, commandEncoder=None):
        """NBodyGPU.js:321-329: walk + halo + kick-drift into the partner buffer, flip."""
        if not self.ready:
            return
        self._ok(lib().gs_step(self._ctx))

    def encodePositionReadback(self, commandEncoder=None, staging=None):
        """NBodyGPU.js:334-341: queue the compaction of vec4(pos, e_i) and its copy to
        host memory behind the work already queued, without waiting (a readback
        already in flight raises GalaxyError GS_ENOTREADY, like the reference's
        one-map rule); readPositions collects it. ``staging`` (N*4 contiguous
        float32, pinned for the copy to overlap later steps) is where it lands; by
        default a buffer of this object. The galaxy's energy diagnostics of the same
        point arrive with it (``readbackEnergy`` after readPositions)."""
        if not self.ready:
            return None
        if staging is None:
            if getattr(self, "_staging", None) is None:
                self._staging = np.zeros(4 * self.N, np.float32)
            staging = self._staging
        buf = np.asarray(staging).reshape(-1)
        if buf.dtype != np.float32 or buf.size < 4 * self.N or not buf.flags.c_contiguous:
            raise ValueError("staging must be contiguous float32 with N*4 elements")
        diag = GsDiag()
        self._ok(lib().gs_encode_position_readback(self._ctx, ptr(buf), C.byref(diag)))
        self._rb = (buf, diag)  # both must outlive the copy
        return None

    def readPositions(self, out=None, timeout_ns=0):
        """NBodyGPU.js:344-348: vec4(pos, e_i) per particle. Awaits the readback
        encodePositionReadback queued (at most timeout_ns, 0 = no limit; a timeout
        raises and leaves it in flight), or reads the current state when none is."""
        rb = getattr(self, "_rb", None)
        if rb is not None:
            self._ok(lib().gs_await_position_readback(self._ctx, int(timeout_ns)))
            self._rb = None
            buf, d = rb
            self.readbackEnergy = {"e_diag": d.e_diag, "e_true": d.e_true,
                                   "momentum": list(d.momentum), "mass": d.mass}
            buf = buf[: 4 * self.N]
        else:
            buf = np.zeros(4 * self.N, np.float32)
            self._ok(lib().gs_read_positions(self._ctx, ptr(buf), int(timeout_ns)))
        if out is not None:
            np.asarray(out).reshape(-1)[: buf.size] = buf
            return out
        return buf.copy() if rb is not None else buf

    @property
    def positionBuffer(self) -> int:
        d = C.c_void_p()
        self._ok(lib().gs_position_buffer(self._ctx, C.byref(d)))
        return d.value

    def destroy(self):
        if getattr(self, "_ctx", None):
            lib().gs_destroy(self._ctx)
            self._ctx = None
        self.ready = False

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- on-device rebuild and full steps --------------------------------------------------
    def setTracking(self, c1=-1, c2=-1, halo1=None, halo2=None):
        h1 = None if halo1 is None else np.asarray(halo1, np.float64)
        h2 = None if halo2 is None else np.asarray(halo2, np.float64)
        self._ok(lib().gs_set_tracking(self._ctx, int(c1), int(c2), ptr(h1), ptr(h2)))

    def getTracking(self):
        c1, c2 = C.c_int64(), C.c_int64()
        h1 = np.zeros(3)
        h2 = np.zeros(3)
        self._ok(lib().gs_get_tracking(self._ctx, C.byref(c1), C.byref(c2), ptr(h1), ptr(h2)))
        return c1.value, c2.value, h1, h2

    def setTime(self, t: float):
        self._ok(lib().gs_set_time(self._ctx, float(t)))

    def setWalkMode(self, compensated: bool):
        """Compensated far-field sums in the walk, one Kahan step per walk round (precision study)."""
        self._ok(lib().gs_set_walk_mode(self._ctx, int(bool(compensated))))

    def setComMode(self, mode: int):
        self._ok(lib().gs_set_com_mode(self._ctx, int(mode)))

    def sortBuild(self):
        self._ok(lib().gs_sort_build(self._ctx))

    def run(self, nsteps: int, starFormation: bool = False):
        self._ok(lib().gs_run(self._ctx, int(nsteps), int(bool(starFormation))))

    def stepKernels(self) -> int:
        """Kernel launches per full step (nodes of the captured step graph)."""
        n = C.c_uint32(0)
        self._ok(lib().gs_step_kernels(self._ctx, C.byref(n)))
        return n.value

    @property
    def stream(self) -> int:
        d = C.c_void_p()
        self._ok(lib().gs_stream(self._ctx, C.byref(d)))
        return d.value or 0

    def sync(self, timeout_ns=0):
        self._ok(lib().gs_sync(self._ctx, int(timeout_ns)))

    def getTree(self, want_perm=True):
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        self._ok(lib().gs_get_tree(self._ctx, None, 0, C.byref(nn), None, 0, C.byref(nl), None))
        nodes = np.zeros(max(nn.value, 1), NODE_DTYPE)
        lr = np.zeros(2 * max(nl.value, 1), np.uint32)
        perm = np.zeros(self.N, np.uint32) if want_perm else None
        self._ok(lib().gs_get_tree(self._ctx, ptr(nodes), nn.value, C.byref(nn), ptr(lr), nl.value,
                                   C.byref(nl), ptr(perm)))
        return nodes[: nn.value], lr[: 2 * nl.value].reshape(-1, 2), perm

    def readState(self):
        P = np.zeros((self.N, 8), np.float32)
        S = np.zeros((self.N, 4), np.float32)
        self._ok(lib().gs_read_state(self._ctx, ptr(P), ptr(S)))
        return P, S

    def writeState(self, particles8=None, stellar4=None):
        P = None if particles8 is None else f32(particles8)
        S = None if stellar4 is None else f32(stellar4)
        self._ok(lib().gs_write_state(self._ctx, ptr(P), ptr(S)))

    def setDebug(self, on=True):
        self._ok(lib().gs_set_debug(self._ctx, int(bool(on))))

    def readForces(self):
        acc = np.zeros((self.N, 4), np.float32)
        dens = np.zeros(self.N, np.float32)
        self._ok(lib().gs_read_forces(self._ctx, ptr(acc), ptr(dens)))
        return acc, dens

    def energy(self) -> dict:
        d = GsDiag()
        self._ok(lib().gs_energy(self._ctx, C.byref(d)))
        return {"e_diag": d.e_diag, "e_true": d.e_true, "momentum": list(d.momentum),
                "mass": d.mass}

    def deviceErrors(self, clear=False) -> int:
        b = C.c_uint32(0)
        self._ok(lib().gs_device_errors(self._ctx, C.byref(b), int(bool(clear))))
        return b.value

    def counters(self, reset=False):
        out = (C.c_uint64 * 3)()
        self._ok(lib().gs_counters(self._ctx, out, int(bool(reset))))
        return list(out)
