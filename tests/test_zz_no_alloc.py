"""The allocation-free sort entry point against the allocating one.

gs_radix_sort_indices_noalloc exists for callers that may not allocate device
memory while they run (a host's per-frame callback, an engine with a device
memory budget fixed at start-up): it takes caller-owned device buffers and
keeps its scratch in a static device array. This test drives it through the C
ABI with device buffers the test owns, twice in a row with different sizes and
key mixes (the second call must not see the first call's leftovers), and
requires exactly the permutation gs_radix_sort_indices returns: integer
results, so the tolerance is zero.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 20


def _reference_perm(L, codes):
    perm = np.zeros(codes.size, np.uint32)
    assert L.gs_radix_sort_indices(codes.ctypes.data, codes.size, perm.ctypes.data) == 0
    return perm


def test_noalloc_sort_matches_allocating_sort_on_two_calls(gpu_lib):
    import torch

    L = gpu_lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(20261203)
    inputs = [
        rng.integers(0, 1 << 30, MAX_N, dtype=np.uint32),              # the maximum size
        (rng.integers(0, 97, 300001, dtype=np.uint32) << 21)           # many ties, and high bits
        | rng.integers(0, 4, 300001, dtype=np.uint32).astype(np.uint32) << 30,
    ]
    for call, codes in enumerate(inputs):
        want = _reference_perm(L, codes)
        d_codes = torch.from_numpy(codes.view(np.int32)).to(dev)
        d_perm = torch.full((codes.size,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize(dev)
        rc = L.gs_radix_sort_indices_noalloc(ctypes.c_void_p(d_codes.data_ptr()), codes.size,
                                             ctypes.c_void_p(d_perm.data_ptr()),
                                             ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, (call, L.gs_last_error(None))
        got = d_perm.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), f"call {call}: permutation differs"


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(gpu_lib):
    import torch

    L = gpu_lib
    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = L.gs_radix_sort_indices_noalloc(ctypes.c_void_p(d.data_ptr()), MAX_N + 1,
                                         ctypes.c_void_p(d.data_ptr()), None)
    assert rc == -1
    assert b"exceeds" in L.gs_last_error(None)
