"""ctypes binding of ``libgalaxy_b200.so`` (declarations in include/galaxy_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgalaxy_b200.so")

GS_OK, GS_EINVAL, GS_ENOMEM, GS_ECUDA, GS_ETIMEDOUT, GS_EDEVICE, GS_ENOTREADY = 0, -1, -2, -3, -4, -5, -6
DERR_LOOKBACK, DERR_STACK, DERR_NODES, DERR_TREE = 0x1, 0x2, 0x4, 0x8
TUNE_WALK_BLOCKS_PER_SM, TUNE_SORT_ITEMS, TUNE_WALK_GROUP, TUNE_WALK_SPLIT = 1, 2, 3, 4

NODE_DTYPE = np.dtype([
    ("com", "<f4", (3,)), ("mass", "<f4"), ("size", "<f4"), ("isLeaf", "<u4"),
    ("first", "<u4"), ("count", "<u4"), ("children", "<i4", (8,)),
])
assert NODE_DTYPE.itemsize == 64


class GsParams(C.Structure):
    """96-byte Params uniform (nbody_bh.wgsl:19-42)."""

    _fields_ = [("dt", C.c_float), ("G", C.c_float), ("epsilon2", C.c_float), ("N", C.c_uint32),
                ("theta", C.c_float), ("haloMass", C.c_float), ("haloA", C.c_float),
                ("gasDrag", C.c_float), ("time", C.c_float), ("agingRate", C.c_float),
                ("sfDensity", C.c_float), ("sfEff", C.c_float), ("sfDt", C.c_float),
                ("haloCount", C.c_uint32), ("pad0", C.c_float), ("pad1", C.c_float),
                ("haloC1", C.c_float * 4), ("haloC2", C.c_float * 4)]


assert C.sizeof(GsParams) == 96


class GsDiag(C.Structure):
    _fields_ = [("e_diag", C.c_double), ("e_true", C.c_double), ("momentum", C.c_double * 3),
                ("mass", C.c_double)]


class GalaxyError(RuntimeError):
    """A non-zero status from the C ABI, with gs_last_error's text."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


# (name, restype, argtypes) for every symbol include/galaxy_b200.h declares
_vp, _u32, _i64, _f32, _f64, _int = C.c_void_p, C.c_uint32, C.c_int64, C.c_float, C.c_double, C.c_int
SIGNATURES = [
    ("gs_last_error", C.c_char_p, [_vp]),
    ("gs_version", C.c_char_p, []),
    ("gs_device_count", _int, [_vp]),
    ("gs_create", _int, [_u32, _vp, _vp, _vp]),
    ("gs_create_on", _int, [_int, _u32, _vp, _vp, _vp]),
    ("gs_destroy", _int, [_vp]),
    ("gs_update_params", _int, [_vp, _vp]),
    ("gs_set_time", _int, [_vp, _f64]),
    ("gs_set_com_mode", _int, [_vp, _int]),
    ("gs_set_star_formation", _int, [_vp, _int]),
    ("gs_set_walk_mode", _int, [_vp, _int]),
    ("gs_set_tuning", _int, [_vp, _int, _int]),
    ("gs_get_tuning", _int, [_vp, _int, _vp]),
    ("gs_get_launch_setting", _int, [_vp, _vp, _vp, _vp]),
    ("gs_update_central_mass", _int, [_vp, _f32, _u32]),
    ("gs_apply_permutation", _int, [_vp, _vp]),
    ("gs_upload_tree", _int, [_vp, _vp, _u32, _vp, _u32]),
    ("gs_refresh", _int, [_vp]),
    ("gs_step", _int, [_vp]),
    ("gs_star_formation", _int, [_vp]),
    ("gs_read_positions", _int, [_vp, _vp, C.c_uint64]),
    ("gs_encode_position_readback", _int, [_vp, _vp, _vp]),
    ("gs_await_position_readback", _int, [_vp, C.c_uint64]),
    ("gs_position_buffer", _int, [_vp, _vp]),
    ("gs_stellar_buffer", _int, [_vp, _vp]),
    ("gs_set_tracking", _int, [_vp, _i64, _i64, _vp, _vp]),
    ("gs_get_tracking", _int, [_vp, _vp, _vp, _vp, _vp]),
    ("gs_sort_build", _int, [_vp]),
    ("gs_run", _int, [_vp, _u32, _int]),
    ("gs_step_kernels", _int, [_vp, _vp]),
    ("gs_stream", _int, [_vp, _vp]),
    ("gs_sync", _int, [_vp, C.c_uint64]),
    ("gs_get_tree", _int, [_vp, _vp, _u32, _vp, _vp, _u32, _vp, _vp]),
    ("gs_read_state", _int, [_vp, _vp, _vp]),
    ("gs_write_state", _int, [_vp, _vp, _vp]),
    ("gs_set_debug", _int, [_vp, _int]),
    ("gs_read_forces", _int, [_vp, _vp, _vp]),
    ("gs_energy", _int, [_vp, _vp]),
    ("gs_device_errors", _int, [_vp, _vp, _int]),
    ("gs_counters", _int, [_vp, _vp, _int]),
    ("gs_morton_codes", _int, [_vp, _u32, _u32, _vp, _vp]),
    ("gs_radix_sort_indices", _int, [_vp, _u32, _vp]),
    ("gs_test_sort_lookback", _int, [_u32, _i64]),
    ("gs_test_fail_alloc", _int, [_i64]),
    ("gs_tree_build", _int, [_vp, _vp, _vp, _u32, _f64, _u32, _vp, _vp, _vp, _u32, _vp]),
    ("gs_sort_and_build", _int, [_vp, _vp, _u32, _i64, _vp, _vp, _vp, _vp, _u32, _vp, _vp, _u32,
                                 _vp, _vp, _vp, _vp]),
    ("gs_device_memory", _int, [_int, _vp, _vp]),
    ("gs_pool_bytes", C.c_uint64, [C.c_uint64, _u32]),
    ("gs_pool_create", _int, [_int, C.c_uint64, _u32, _vp]),
    ("gs_pool_add", _int, [_vp, _u32, _vp, _vp, _vp, _vp]),
    ("gs_pool_remove", _int, [_vp, _u32]),
    ("gs_pool_free", _int, [_vp, _vp, _vp]),
    ("gs_select", _int, [_vp, _u32]),
    ("gs_pool_energies", _int, [_vp, _vp, _u32]),
    ("gs_radix_sort_indices_noalloc", _int, [_vp, _u32, _vp, _vp]),
]

_lib = None


def lib():
    """Load the CUDA library (raises if it is not built: no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m galaxy_sim_b200.build` "
                "(nvcc, sm_100a); the gravity path has no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, ctx=None) -> None:
    if rc != GS_OK:
        msg = lib().gs_last_error(ctx)
        raise GalaxyError(rc, msg.decode() if msg else "")


def ptr(a):
    return None if a is None else a.ctypes.data


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().gs_device_count(C.byref(n))
    return n.value if rc == GS_OK else 0
