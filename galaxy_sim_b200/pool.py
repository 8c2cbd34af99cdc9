"""Many independent galaxies in one context: batches and the serving pool.

The reference runs one simulation per page (one NBodyGPU, one worker). Here a
``GalaxyPool`` owns one ``gs_ctx`` pool: every resident galaxy is stepped by the
same launches (segmented Morton sort, tree build, work-stealing walk) replayed
from one CUDA graph per step, and each galaxy's result equals its solo run.
Galaxies are admitted into free slots and free particle ranges and released
when done, which is what continuous batching needs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import GS_ENOMEM, GalaxyError, GsDiag, check, f32, lib, ptr
from .nbody_gpu import build_params


def device_memory(device: int = 0):
    """(free, total) bytes of a CUDA device."""
    f, t = C.c_uint64(0), C.c_uint64(0)
    check(lib().gs_device_memory(int(device), C.byref(f), C.byref(t)))
    return f.value, t.value


def pool_bytes(capacity: int, max_galaxies: int) -> int:
    """Device bytes of a pool for ``capacity`` particles and ``max_galaxies`` slots."""
    return int(lib().gs_pool_bytes(int(capacity), int(max_galaxies)))


def capacity_for_bytes(budget: int, max_galaxies: int) -> int:
    """Largest particle capacity whose pool fits in ``budget`` bytes."""
    lo, hi = 0, 1 << 27
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if pool_bytes(mid, max_galaxies) <= budget:
            lo = mid
        else:
            hi = mid - 1
    return lo


class GalaxyPool:
    def __init__(self, capacity: int, max_galaxies: int, device: int = 0):
        h = C.c_void_p()
        check(lib().gs_pool_create(int(device), int(capacity), int(max_galaxies), C.byref(h)))
        self._ctx = h
        self.capacity = int(capacity)
        self.max_galaxies = int(max_galaxies)
        self.device = int(device)
        self.n = {}  # slot -> N

    def _ok(self, rc):
        check(rc, self._ctx)

    def _sel(self, slot: int):
        self._ok(lib().gs_select(self._ctx, int(slot)))

    # -- admission -------------------------------------------------------------------------
    def add(self, particles, stellar=None, params: dict | None = None, tracking=None,
            star_formation: bool = True):
        """Admit a galaxy; returns its slot, or None when no slot / particle range is free.

        ``params`` holds NBodyGPU.updateParams keywords; ``tracking`` is
        (c1, c2, halo1, halo2) as in NBodyGPU.setTracking; ``star_formation``
        False keeps run(..., star_formation=True) from acting on this galaxy."""
        P = f32(particles).reshape(-1, 8)
        S = None if stellar is None else f32(stellar).reshape(-1, 4)
        N = P.shape[0]
        prm = build_params(N, **params) if params else None
        slot = C.c_uint32(0)
        rc = lib().gs_pool_add(self._ctx, N, ptr(P), ptr(S), None if prm is None else C.byref(prm),
                               C.byref(slot))
        if rc == GS_ENOMEM:
            return None
        self._ok(rc)
        s = slot.value
        self.n[s] = N
        if tracking is not None:
            self.set_tracking(s, *tracking)
        if not star_formation:
            self._sel(s)
            self._ok(lib().gs_set_star_formation(self._ctx, 0))
        return s

    def remove(self, slot: int):
        self._ok(lib().gs_pool_remove(self._ctx, int(slot)))
        self.n.pop(int(slot), None)

    def free(self):
        """(largest free contiguous particle range, free slots)."""
        r, s = C.c_uint64(0), C.c_uint32(0)
        self._ok(lib().gs_pool_free(self._ctx, C.byref(r), C.byref(s)))
        return r.value, s.value

    def fits(self, N: int) -> bool:
        r, s = self.free()
        return s > 0 and r >= ((N + 255) // 256) * 256

    # -- per-galaxy state ------------------------------------------------------------------
    def set_params(self, slot: int, **kw):
        self._sel(slot)
        p = build_params(self.n[slot], **kw)
        self._ok(lib().gs_update_params(self._ctx, C.byref(p)))

    def set_tracking(self, slot: int, c1=-1, c2=-1, halo1=None, halo2=None):
        self._sel(slot)
        h1 = None if halo1 is None else np.asarray(halo1, np.float64)
        h2 = None if halo2 is None else np.asarray(halo2, np.float64)
        self._ok(lib().gs_set_tracking(self._ctx, int(c1), int(c2), ptr(h1), ptr(h2)))

    def get_tracking(self, slot: int):
        self._sel(slot)
        c1, c2 = C.c_int64(), C.c_int64()
        h1, h2 = np.zeros(3), np.zeros(3)
        self._ok(lib().gs_get_tracking(self._ctx, C.byref(c1), C.byref(c2), ptr(h1), ptr(h2)))
        return c1.value, c2.value, h1, h2

    def read_state(self, slot: int):
        self._sel(slot)
        N = self.n[slot]
        P = np.zeros((N, 8), np.float32)
        S = np.zeros((N, 4), np.float32)
        self._ok(lib().gs_read_state(self._ctx, ptr(P), ptr(S)))
        return P, S

    def write_state(self, slot: int, particles8=None, stellar4=None):
        self._sel(slot)
        P = None if particles8 is None else f32(particles8)
        S = None if stellar4 is None else f32(stellar4)
        self._ok(lib().gs_write_state(self._ctx, ptr(P), ptr(S)))

    def energy(self, slot: int) -> dict:
        self._sel(slot)
        d = GsDiag()
        self._ok(lib().gs_energy(self._ctx, C.byref(d)))
        return {"e_diag": d.e_diag, "e_true": d.e_true, "momentum": list(d.momentum), "mass": d.mass}

    def energies(self) -> np.ndarray:
        """(max_galaxies, 6) array: e_diag, e_true, px, py, pz, mass of every slot."""
        out = (GsDiag * self.max_galaxies)()
        self._ok(lib().gs_pool_energies(self._ctx, out, self.max_galaxies))
        return np.array([[d.e_diag, d.e_true, *d.momentum, d.mass] for d in out])

    def device_errors(self, slot: int, clear=False) -> int:
        self._sel(slot)
        b = C.c_uint32(0)
        self._ok(lib().gs_device_errors(self._ctx, C.byref(b), int(bool(clear))))
        return b.value

    def set_debug(self, enable: bool = True):
        """Keep each walk's pair forces and leaf densities (read_forces), for every galaxy."""
        self._ok(lib().gs_set_debug(self._ctx, int(bool(enable))))

    def read_forces(self, slot: int):
        """{ax, ay, az, phi} per particle (G applied, halo excluded) and own-leaf
        densities of the last walk of one galaxy; needs set_debug(True) first."""
        self._sel(slot)
        N = self.n[slot]
        acc = np.zeros((N, 4), np.float32)
        dens = np.zeros(N, np.float32)
        self._ok(lib().gs_read_forces(self._ctx, ptr(acc), ptr(dens)))
        return acc, dens

    # -- the NBodyGPU surface on one slot ------------------------------------------------------
    def apply_permutation(self, slot: int, perm):
        """NBodyGPU.applyPermutation on one galaxy (out[i] = in[perm[i]], galaxy-local)."""
        self._sel(slot)
        p = np.ascontiguousarray(perm, np.uint32)
        if p.size != self.n[slot]:
            raise ValueError("perm must hold N indices")
        self._ok(lib().gs_apply_permutation(self._ctx, ptr(p)))

    def upload_tree(self, slot: int, nodes, num_nodes: int, level_ranges=None):
        """NBodyGPU.uploadBHTree on one galaxy (BHNode array with galaxy-local indices)."""
        self._sel(slot)
        nd = np.ascontiguousarray(nodes).view(np.uint8)
        lr, nl = None, 0
        if level_ranges is not None:
            lr = np.ascontiguousarray(np.asarray(level_ranges, np.uint32).reshape(-1, 2)[:16])
            nl = lr.shape[0]
        self._ok(lib().gs_upload_tree(self._ctx, ptr(nd), int(num_nodes), ptr(lr), nl))

    def num_nodes(self, slot: int) -> int:
        """Node count of one galaxy's current tree."""
        self._sel(slot)
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        self._ok(lib().gs_get_tree(self._ctx, None, 0, C.byref(nn), None, 0, C.byref(nl), None))
        return nn.value

    def get_tree(self, slot: int, want_perm: bool = True):
        """(nodes, level ranges, permutation of the last rebuild) of one galaxy."""
        from ._lib import NODE_DTYPE

        self._sel(slot)
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        self._ok(lib().gs_get_tree(self._ctx, None, 0, C.byref(nn), None, 0, C.byref(nl), None))
        nodes = np.zeros(max(nn.value, 1), NODE_DTYPE)
        lr = np.zeros(2 * max(nl.value, 1), np.uint32)
        perm = np.zeros(self.n[slot], np.uint32) if want_perm else None
        self._ok(lib().gs_get_tree(self._ctx, ptr(nodes), nn.value, C.byref(nn), ptr(lr), nl.value,
                                   C.byref(nl), ptr(perm)))
        return nodes[: nn.value], lr[: 2 * nl.value].reshape(-1, 2), perm

    def refresh(self):
        """NBodyGPU.encodeRefresh for every resident galaxy."""
        self._ok(lib().gs_refresh(self._ctx))

    def step(self):
        """NBodyGPU.step (walk + halo + kick-drift) for every resident galaxy."""
        self._ok(lib().gs_step(self._ctx))

    def sort_build(self):
        """The on-device rebuild for every resident galaxy."""
        self._ok(lib().gs_sort_build(self._ctx))

    # -- stepping --------------------------------------------------------------------------
    def run(self, nsteps: int, star_formation: bool = False):
        self._ok(lib().gs_run(self._ctx, int(nsteps), int(bool(star_formation))))

    def sync(self, timeout_ns=0):
        self._ok(lib().gs_sync(self._ctx, int(timeout_ns)))

    @property
    def stream(self) -> int:
        d = C.c_void_p()
        self._ok(lib().gs_stream(self._ctx, C.byref(d)))
        return d.value or 0

    @property
    def particles(self) -> int:
        return sum(self.n.values())

    def close(self):
        if getattr(self, "_ctx", None):
            lib().gs_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["GalaxyPool", "GalaxyError", "device_memory", "pool_bytes", "capacity_for_bytes"]
