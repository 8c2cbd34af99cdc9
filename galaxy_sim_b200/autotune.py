"""Launch autotuner for a context (a single galaxy or a pool).

The knobs never change results (`gs_set_tuning`): the persistent walk grid
(blocks per SM; groups are independent, so fewer resident warps only change the
schedule; below 8 the walk compiled for 72 registers per thread runs) and the sort tile (8 or 16 keys per thread; a stable sort has one
answer). The bucket size (16) and the walk group (one warp of 32 particles)
are not knobs: the first is the reference's tree, the second the warp.

``autotune(ctx_owner)`` times a few full steps of the owner's actual workload
for every candidate (CUDA events on the context's stream, after warm-up steps),
keeps the fastest and leaves it set. It advances the simulation by
(warmup + steps) x candidates steps, so call it on a copy or accept the steps.
"""
from __future__ import annotations

import ctypes as C
import itertools

from ._lib import TUNE_SORT_ITEMS, TUNE_WALK_BLOCKS_PER_SM, GalaxyError, check, lib

WALK_BLOCKS = (6, 7, 8)
SORT_ITEMS = (8, 16)


def get(ctx, knob: int) -> int:
    v = C.c_int(0)
    check(lib().gs_get_tuning(ctx, knob, C.byref(v)), ctx)
    return v.value


def set_(ctx, knob: int, value: int) -> None:
    check(lib().gs_set_tuning(ctx, knob, int(value)), ctx)


def autotune(owner, steps: int = 5, warmup: int = 2, star_formation: bool = False,
             walk_blocks=WALK_BLOCKS, sort_items=SORT_ITEMS, device: int = 0) -> dict:
    """owner: an NBodyGPU or GalaxyPool (anything with ``_ctx``, ``stream`` and
    ``run(n, star_formation)``). Returns {"choice": {...}, "ms": {(bps, items): ms}}."""
    import torch

    ctx = owner._ctx
    ext = torch.cuda.ExternalStream(owner.stream, device=torch.device("cuda", device))
    timing = {}
    for bps, items in itertools.product(walk_blocks, sort_items):
        try:
            set_(ctx, TUNE_WALK_BLOCKS_PER_SM, bps)
            set_(ctx, TUNE_SORT_ITEMS, items)
        except GalaxyError:
            continue  # beyond what this build's kernels were compiled for
        owner.run(warmup, star_formation)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record(ext)
        owner.run(steps, star_formation)
        with torch.cuda.stream(ext):
            e1.record(ext)
        e1.synchronize()
        timing[(bps, items)] = e0.elapsed_time(e1) / steps
    best = min(timing, key=timing.get)
    set_(ctx, TUNE_WALK_BLOCKS_PER_SM, best[0])
    set_(ctx, TUNE_SORT_ITEMS, best[1])
    return {"choice": {"walk_blocks_per_sm": best[0], "sort_keys_per_thread": best[1]},
            "ms": {f"{b}x{i}": round(t, 4) for (b, i), t in timing.items()}}


__all__ = ["autotune", "get", "set_", "WALK_BLOCKS", "SORT_ITEMS"]
