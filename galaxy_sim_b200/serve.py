"""Serving independent galaxy simulations on one GPU, with continuous batching.

The reference runs one simulation per browser page. Here a request is a whole
simulation (initial galaxy, Params, number of steps); the ``BatchServer`` keeps
every admitted simulation resident in one ``GalaxyPool`` and advances all of
them with each batched step (one CUDA graph: segmented sort, build and walk
over every resident galaxy). Requests that arrive while others run are
admitted as soon as a slot and a contiguous particle range are free — the pool
is sized from free HBM — and finished ones are read back and released between
steps. Each result is bit-identical to the same simulation run alone.

``PlainServer`` is the one-at-a-time baseline: a fresh single-galaxy context
per request, run to completion in arrival order.

Latencies reported: per batched step (device time, CUDA events on the pool's
stream), per request (arrival to result on the host) and admission queue wait.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import initial_conditions as ic
from .nbody_gpu import NBodyGPU
from .pool import GalaxyPool, capacity_for_bytes, device_memory
from .simulation import Physics, params_dict

PRESETS = ("disk", "sphere", "collision")


@dataclass
class Request:
    rid: int
    arrival: float                    # seconds after the stream starts
    particles: np.ndarray             # (N, 8) float32
    stellar: np.ndarray               # (N, 4) float32
    params: dict                      # NBodyGPU.updateParams keywords
    steps: int
    tracking: tuple | None = None     # NBodyGPU.setTracking arguments
    star_formation: bool = False
    preset: str = ""
    admitted: float | None = None
    finished: float | None = None
    result: tuple | None = None       # (particles, stellar, energy dict)

    @property
    def N(self) -> int:
        return self.particles.shape[0]


def make_request(rid, arrival, preset, N, seed, physics: Physics, steps) -> Request:
    """A request of one of the served presets: a disk, a cold Hernquist sphere
    (a = 1) or two disks on a collision orbit (scaled to N)."""
    if preset == "disk":
        g = ic.galaxy_disk(N, seed, Q=1.5, arms=2)
    elif preset == "sphere":
        g = ic.hernquist_sphere(N, seed, a=1.0)
    elif preset == "collision":
        g = ic.two_galaxy_collision(N, seed, Q=1.5, arms=2)
    else:
        raise ValueError(preset)
    c1, c2 = g.central
    tracking = None
    if c1 >= 0 or c2 >= 0:
        hc = g.halo_centers
        tracking = (c1, c2, hc[0] if len(hc) > 0 else None, hc[1] if len(hc) > 1 else None)
    return Request(rid, arrival, g.particles, g.stellar, params_dict(g, physics), steps, tracking,
                   physics.sf_eff > 0, preset)


def make_stream(n_requests: int, rate: float, seed: int = 0, n_range=(8192, 1 << 20),
                step_range=(100, 2000), presets=PRESETS) -> list:
    """Poisson arrivals at ``rate`` per second; N log-uniform in n_range; preset,
    step count (uniform in step_range) and eps x theta x dt drawn per request."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n_requests):
        t += rng.exponential(1.0 / rate)
        N = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        preset = presets[int(rng.integers(len(presets)))]
        ph = Physics(float(rng.choice([0.02, 0.05])), float(rng.choice([0.5, 0.7])),
                     float(rng.choice([0.0025, 0.005])))
        steps = int(rng.integers(step_range[0], step_range[1] + 1))
        out.append(make_request(rid, t, preset, N, seed * 100003 + rid, ph, steps))
    return out


def _pct(xs, q):
    if not xs:
        return None
    s = sorted(xs)
    return s[min(len(s) - 1, int(q * len(s)))]


def summarize(requests, step_ms, wall_s) -> dict:
    ps = sum(r.N * r.steps for r in requests)
    lat = [r.finished - r.arrival for r in requests]
    wait = [r.admitted - r.arrival for r in requests]
    return {"particle_steps": int(ps), "wall_s": round(wall_s, 3),
            "gpu_busy_s": round(sum(step_ms) / 1e3, 3),
            "value": round(ps / wall_s, 1) if wall_s > 0 else None,
            "step_ms": {"p50": _pct(step_ms, 0.5), "p99": _pct(step_ms, 0.99), "n": len(step_ms)},
            "request_s": {"p50": _pct(lat, 0.5), "p99": _pct(lat, 0.99)},
            "queue_wait_s": {"p50": _pct(wait, 0.5), "p99": _pct(wait, 0.99)}}


class _Timer:
    """Device time of work enqueued on an external CUDA stream (CUDA events)."""

    def __init__(self, stream_ptr: int, device: int):
        import torch

        self.torch = torch
        self.stream = torch.cuda.ExternalStream(stream_ptr, device=torch.device("cuda", device))
        self.pending = []

    def start(self):
        e = self.torch.cuda.Event(enable_timing=True)
        with self.torch.cuda.stream(self.stream):
            e.record(self.stream)
        return e

    def stop(self, e0):
        e1 = self.torch.cuda.Event(enable_timing=True)
        with self.torch.cuda.stream(self.stream):
            e1.record(self.stream)
        self.pending.append((e0, e1))

    def collect(self):
        for _, e1 in self.pending:
            e1.synchronize()
        out = [a.elapsed_time(b) for a, b in self.pending]
        self.pending = []
        return out


class BatchServer:
    """Continuous batching over one GalaxyPool sized from free HBM."""

    def __init__(self, capacity: int | None = None, max_galaxies: int = 64, device: int = 0,
                 hbm_fraction: float = 0.8):
        if capacity is None:
            free, _ = device_memory(device)
            capacity = capacity_for_bytes(int(free * hbm_fraction), max_galaxies)
        self.pool = GalaxyPool(capacity, max_galaxies, device)
        self.device = device

    def close(self):
        self.pool.close()

    def serve(self, requests, clock=time.perf_counter) -> dict:
        pool = self.pool
        todo = deque(sorted(requests, key=lambda r: r.arrival))
        queue = deque()
        active = {}  # slot -> [request, steps left]
        timer = _Timer(pool.stream, self.device)
        step_ms = []
        t0 = clock()
        while todo or queue or active:
            now = clock() - t0
            while todo and todo[0].arrival <= now:
                queue.append(todo.popleft())
            # admission: FIFO while the head fits (a slot and a free particle range)
            while queue and pool.fits(queue[0].N):
                r = queue.popleft()
                slot = pool.add(r.particles, r.stellar, r.params, r.tracking, r.star_formation)
                if slot is None:
                    queue.appendleft(r)
                    break
                r.admitted = clock() - t0
                active[slot] = [r, r.steps]
            if not active:
                if queue:
                    raise RuntimeError(f"request {queue[0].rid} (N={queue[0].N}) can never fit the pool")
                if todo:
                    time.sleep(max(0.0, todo[0].arrival - (clock() - t0)))
                continue
            # one batched step of every resident simulation
            e0 = timer.start()
            pool.run(1, star_formation=True)
            timer.stop(e0)
            done = []
            for slot, a in active.items():
                a[1] -= 1
                if a[1] == 0:
                    done.append(slot)
            for slot in done:  # read back and release (synchronises the stream)
                r = active.pop(slot)[0]
                P, S = pool.read_state(slot)
                r.result = (P, S, pool.energy(slot))
                r.finished = clock() - t0
                pool.remove(slot)
            if len(timer.pending) >= 256:
                step_ms += timer.collect()
        step_ms += timer.collect()
        return summarize(requests, step_ms, clock() - t0)


class PlainServer:
    """One simulation at a time, in arrival order, each in its own context."""

    def __init__(self, device: int = 0):
        self.device = device

    def serve(self, requests, clock=time.perf_counter) -> dict:
        import torch

        step_ms = []
        t0 = clock()
        for r in sorted(requests, key=lambda r: r.arrival):
            now = clock() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            r.admitted = clock() - t0
            sim = NBodyGPU(self.device, r.particles, r.stellar)
            sim.updateParams(**r.params)
            if r.tracking is not None:
                sim.setTracking(*r.tracking)
            ext = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", self.device))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(ext):
                e0.record(ext)
            sim.run(r.steps, r.star_formation)
            with torch.cuda.stream(ext):
                e1.record(ext)
            P, S = sim.readState()
            r.result = (P, S, sim.energy())
            r.finished = clock() - t0
            step_ms += [e0.elapsed_time(e1) / r.steps] * r.steps
            sim.destroy()
        return summarize(requests, step_ms, clock() - t0)


__all__ = ["Request", "make_request", "make_stream", "BatchServer", "PlainServer", "summarize"]
