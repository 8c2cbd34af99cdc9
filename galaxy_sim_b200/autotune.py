"""Launch autotuner for a context (a single galaxy or a pool).

Knobs (`gs_set_tuning`):

* walk group size: how many particles a warp walks together, 32 (one lane per
  particle), 16, 8 or 4 (two, four or eight lanes per particle splitting its
  node tests and leaf sources), or 0 = by each galaxy's size. Small galaxies need the
  smaller groups to fill the GPU; large ones walk fastest in groups of 32. The
  group size changes the order of the force sums, so results change at the
  rounding level (inside the force tolerance) with it;
* walk split: how many parts each work item's walk is split into (1, 2, 4 or
  8, or 0 = by size) when the context walks one galaxy. A small galaxy's walk is
  as long as its densest work item; parts walk disjoint subtrees in parallel.
  Like the group size it changes only the order of the force sums. A pool of
  several galaxies walks unsplit, so the tuner skips this knob there;
* the persistent walk grid (blocks per SM; groups are independent, so fewer
  resident warps only change the schedule; below 8 the walk compiled for 72
  registers per thread runs) - never changes results;
* the sort tile depth (4, 8 or 16 keys per thread: tiles of 1024, 2048 or 4096
  keys; a small galaxy sorts in more tiles with the smaller depths; a stable
  sort has one answer) - never changes results.

The bucket size (16) is not a knob: it is the reference's tree
(mortonTree.js:25), and changing it would change every result.

``autotune(owner)`` times a few full steps of the owner's actual workload for
each candidate (CUDA events on the context's stream, after warm-up steps):
first the walk group size, then the walk split, then the walk grid x sort
tile, keeps the fastest
and leaves it set. It advances the simulation by (warmup + steps) x candidates
steps, so call it on a copy or accept the steps.
"""
from __future__ import annotations

import ctypes as C
import itertools

from ._lib import (TUNE_SORT_ITEMS, TUNE_WALK_BLOCKS_PER_SM, TUNE_WALK_GROUP, TUNE_WALK_SPLIT, GalaxyError,
                   check, lib)

WALK_BLOCKS = (6, 7, 8)
SORT_ITEMS = (4, 8, 16)
WALK_GROUPS = (0, 4, 8, 16, 32)
WALK_SPLITS = (0, 1, 2, 4, 8)


def get(ctx, knob: int) -> int:
    v = C.c_int(0)
    check(lib().gs_get_tuning(ctx, knob, C.byref(v)), ctx)
    return v.value


def set_(ctx, knob: int, value: int) -> None:
    check(lib().gs_set_tuning(ctx, knob, int(value)), ctx)


def launch_setting(ctx) -> dict:
    """The setting in effect for the context's selected galaxy after the "by
    size" rules: particles per walk group, walk parts per item, sort keys per thread."""
    g, s, i = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
    check(lib().gs_get_launch_setting(ctx, C.byref(g), C.byref(s), C.byref(i)), ctx)
    return {"walk_group": g.value, "walk_split": s.value, "sort_keys_per_thread": i.value}


def _time(owner, ext, steps, warmup, star_formation):
    import torch

    owner.run(warmup, star_formation)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(ext):
        e0.record(ext)
    owner.run(steps, star_formation)
    with torch.cuda.stream(ext):
        e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def autotune(owner, steps: int = 5, warmup: int = 2, star_formation: bool = False,
             walk_blocks=WALK_BLOCKS, sort_items=SORT_ITEMS, walk_groups=WALK_GROUPS,
             walk_splits=WALK_SPLITS, device: int = 0) -> dict:
    """owner: an NBodyGPU or GalaxyPool (anything with ``_ctx``, ``stream`` and
    ``run(n, star_formation)``). Returns {"choice": {...}, "ms": {...}}."""
    import torch

    ctx = owner._ctx
    ext = torch.cuda.ExternalStream(owner.stream, device=torch.device("cuda", device))
    group_ms = {}
    for wg in walk_groups:
        set_(ctx, TUNE_WALK_GROUP, wg)
        group_ms[wg] = _time(owner, ext, steps, warmup, star_formation)
    best_group = min(group_ms, key=group_ms.get)
    set_(ctx, TUNE_WALK_GROUP, best_group)
    split_ms = {}
    lone = len(getattr(owner, "n", {0: 0})) == 1
    if lone and launch_setting(ctx)["walk_group"] < 32:   # the split applies
        for sp in walk_splits:
            set_(ctx, TUNE_WALK_SPLIT, sp)
            split_ms[sp] = _time(owner, ext, steps, warmup, star_formation)
        best_split = min(split_ms, key=split_ms.get)
        set_(ctx, TUNE_WALK_SPLIT, best_split)
    else:
        best_split = get(ctx, TUNE_WALK_SPLIT)
    timing = {}
    for bps, items in itertools.product(walk_blocks, sort_items):
        try:
            set_(ctx, TUNE_WALK_BLOCKS_PER_SM, bps)
            set_(ctx, TUNE_SORT_ITEMS, items)
        except GalaxyError:
            continue  # beyond what this build's kernels were compiled for
        timing[(bps, items)] = _time(owner, ext, steps, warmup, star_formation)
    best = min(timing, key=timing.get)
    set_(ctx, TUNE_WALK_BLOCKS_PER_SM, best[0])
    set_(ctx, TUNE_SORT_ITEMS, best[1])
    return {"choice": {"walk_group": best_group if best_group else "by galaxy size",
                       "walk_split": (best_split if best_split else "by galaxy size") if split_ms
                       else "unsplit (groups of 32)" if lone else "unsplit (several galaxies)",
                       "walk_blocks_per_sm": best[0], "sort_keys_per_thread": best[1]},
            "ms": {**{f"group{g or 'auto'}": round(t, 4) for g, t in group_ms.items()},
                   **{f"split{p or 'auto'}": round(t, 4) for p, t in split_ms.items()},
                   **{f"{b}x{i}": round(t, 4) for (b, i), t in timing.items()}}}


__all__ = ["autotune", "get", "set_", "launch_setting", "WALK_BLOCKS", "SORT_ITEMS", "WALK_GROUPS", "WALK_SPLITS"]
