"""The allocation-free sort entry point, checked against the oracle and the
allocating entry point.

gs_radix_sort_indices_noalloc exists for callers that may not allocate device
memory while they run: a host's per-frame callback, where cudaMalloc/cudaFree
can synchronize the whole device and stall the frame, or an engine whose device
memory budget is fixed at start-up. It takes caller-owned device buffers and
keeps its scratch in a static device array. These tests drive it through the C
ABI with device buffers the test owns:

* after the documented set-up call (N == 0), two calls in a row with different
  sizes and key mixes (the second must not see the first call's leftovers) give
  exactly the permutation of the oracle's radixSortIndices and of
  gs_radix_sort_indices: integer results, so the tolerance is zero;
* after set-up, calls at the maximum size leave the device's free memory
  unchanged;
* a dedicated stream that waits on an event for codes produced on another
  stream, and sizes below, at and just over one sort tile;
* a stream under capture is refused without breaking the capture, and sizes
  beyond the static scratch are refused;
* a look-back wait that runs out comes back as GS_EDEVICE, and the next call
  sorts correctly.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 20


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _noalloc(L, d_codes, n, d_perm, stream):
    return L.gs_radix_sort_indices_noalloc(_vp(d_codes) if d_codes is not None else None, n,
                                           _vp(d_perm) if d_perm is not None else None,
                                           ctypes.c_void_p(stream.cuda_stream) if stream is not None else None)


def _allocating_perm(L, codes):
    perm = np.zeros(codes.size, np.uint32)
    assert L.gs_radix_sort_indices(codes.ctypes.data, codes.size, perm.ctypes.data) == 0
    return perm


def _device(torch, codes):
    dev = torch.device("cuda", 0)
    d_codes = torch.from_numpy(codes.view(np.int32)).to(dev)
    d_perm = torch.full((max(codes.size, 1),), -1, dtype=torch.int32, device=dev)
    return d_codes, d_perm


def test_noalloc_sort_matches_oracle_and_allocating_sort_on_two_calls(gpu_lib, oracle):
    import torch

    L = gpu_lib
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    assert _noalloc(L, None, 0, None, stream) == 0, L.gs_last_error(None)   # set-up
    rng = np.random.default_rng(20261203)
    inputs = [
        rng.integers(0, 1 << 30, MAX_N, dtype=np.uint32),              # the maximum size
        (rng.integers(0, 97, 300001, dtype=np.uint32) << 21)           # many ties, and high bits
        | rng.integers(0, 4, 300001, dtype=np.uint32).astype(np.uint32) << 30,
    ]
    for call, codes in enumerate(inputs):
        want = oracle.radix_sort_indices(codes)
        assert np.array_equal(_allocating_perm(L, codes), want)
        d_codes, d_perm = _device(torch, codes)
        torch.cuda.synchronize()
        rc = _noalloc(L, d_codes, codes.size, d_perm, stream)
        assert rc == 0, (call, L.gs_last_error(None))
        got = d_perm.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), f"call {call}: permutation differs from the oracle"


def test_noalloc_sort_allocates_nothing_after_setup(gpu_lib, oracle):
    import torch

    L = gpu_lib
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    codes = np.random.default_rng(7).integers(0, 1 << 30, MAX_N, dtype=np.uint32)
    d_codes, d_perm = _device(torch, codes)
    assert _noalloc(L, None, 0, None, stream) == 0, L.gs_last_error(None)   # set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        assert _noalloc(L, d_codes, MAX_N, d_perm, stream) == 0, L.gs_last_error(None)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert np.array_equal(d_perm.cpu().numpy().view(np.uint32), oracle.radix_sort_indices(codes))


def test_noalloc_sort_on_a_dedicated_stream_and_small_sizes(gpu_lib, oracle):
    import torch

    L = gpu_lib
    torch.cuda.set_device(0)
    producer, sorter = torch.cuda.Stream(0), torch.cuda.Stream(0)
    rng = np.random.default_rng(99)
    for n in (1, 2, 4095, 4096, 4097, 70000):
        codes = rng.integers(0, 1 << 30, n, dtype=np.uint32)
        codes[: n // 3] = codes[0]                                  # ties
        host = torch.from_numpy(codes.view(np.int32)).pin_memory()
        d_perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()                                    # d_perm is filled before the sort
        with torch.cuda.stream(producer):
            d_codes = torch.empty(n, dtype=torch.int32, device="cuda")
            d_codes.copy_(host, non_blocking=True)                  # produced on another stream
            ready = torch.cuda.Event()
            ready.record(producer)
        sorter.wait_event(ready)
        rc = _noalloc(L, d_codes, n, d_perm, sorter)
        assert rc == 0, (n, L.gs_last_error(None))
        got = d_perm.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, oracle.radix_sort_indices(codes)), n


def test_noalloc_sort_refuses_a_capturing_stream(gpu_lib):
    import torch

    L = gpu_lib
    torch.cuda.set_device(0)
    s = torch.cuda.Stream(0)
    d_codes = torch.arange(64, dtype=torch.int32, device="cuda")
    d_perm = torch.zeros(64, dtype=torch.int32, device="cuda")
    x = torch.zeros(16, device="cuda")
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        rc = _noalloc(L, d_codes, 64, d_perm, s)
    assert rc == -1 and b"capturing" in L.gs_last_error(None)
    g.replay()                                                      # the capture survived
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(gpu_lib):
    import torch

    L = gpu_lib
    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = L.gs_radix_sort_indices_noalloc(_vp(d), MAX_N + 1, _vp(d), None)
    assert rc == -1
    assert b"exceeds" in L.gs_last_error(None)


def test_noalloc_sort_reports_a_lookback_wait_that_runs_out(gpu_lib, oracle):
    import torch

    L = gpu_lib
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    codes = np.random.default_rng(5).integers(0, 1 << 30, 10 * 4096 + 77, dtype=np.uint32)
    d_codes, d_perm = _device(torch, codes)
    torch.cuda.synchronize()
    assert L.gs_test_sort_lookback(4096, 3) == 0   # tile 3 never publishes; waits give up
    try:
        rc = _noalloc(L, d_codes, codes.size, d_perm, stream)
    finally:
        assert L.gs_test_sort_lookback(1 << 20, -1) == 0
    assert rc == -5, L.gs_last_error(None)          # GS_EDEVICE, the call returned
    assert b"look-back" in L.gs_last_error(None)
    assert _noalloc(L, d_codes, codes.size, d_perm, stream) == 0, L.gs_last_error(None)
    assert np.array_equal(d_perm.cpu().numpy().view(np.uint32), oracle.radix_sort_indices(codes))
