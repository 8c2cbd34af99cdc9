#!/usr/bin/env python
"""Benchmark of the B200 gravity path: particle-steps/s of the full step.

A step is one pass of the hot path over the whole galaxy: Morton codes, sort,
gather, BFS octree build, COM refresh, Barnes-Hut walk + halo + kick-drift
(+ star formation), replayed from a CUDA graph. Default workload: the single
disk of N = 524288 (30% gas, star formation, eps 0.02, theta 0.5, dt 0.005).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs an independent replica
(the path does not shard; there is no collective): weak scaling, value = all
ranks' particle-steps / the slowest rank's device time.

Timing: after the launch knobs are tuned, the galaxy goes back to its seeded
initial conditions, so every timed leg covers the same early steps of the
workload (the disk contracts, and later steps cost more interactions). Then W
untimed warm-up steps, then K steps, each bracketed by CUDA events on
the context's stream, with a 256 MiB L2 flush (2x the 126 MB L2) between steps;
barrier + synchronize on both sides; max over ranks. ``e2e`` is the same
metric through the C ABI with pinned host buffers, frame by frame as main.js
drives NBodyGPU at one step per frame: upload of the initial state, per step a
Params upload, the step and the position readback (16 B per particle, with the
energy diagnostics of the same point) collected in the next frame as main.js
collects its readback promise, and a final state readback, all inside the
event-timed region. ``precision_modes`` gives the step time of the compensated
walk and of the FP64 internal-node COM refresh on the same workload, each mode
from the initial conditions.

The same line carries the metric's batched and served halves (one GPU):
``batched`` = 96 disks (N log-uniform in [4096, 262144]) stepped as one pool,
one CUDA graph per step, against the same galaxies run back to back in plain
single-galaxy contexts; ``served`` = a seeded Poisson stream of simulation
requests (disk / sphere / collision presets, N log-uniform in [8192, 2^20])
through the continuous-batching server and through a one-at-a-time server,
with per-step and per-request p50/p99 latency and admission queue wait, the
ratio's upper bound for that mix, and a sweep over arrival rates 1/10/50 per s.
``--workload batch96`` and ``--workload serve`` print those alone.

``--impl reference`` times the reference algorithm on the host cores: the CPU
restatement in oracle/ (sort + build single-threaded like the reference's Web
Worker, refresh + walk + kick-drift on all cores), each step a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at N=500k \u03b8=0.5; batched/served vs plain, p50/p99, same GPU"
UNIT = "particle-steps/s"
FLOPS_PER_INTERACTION = 23
L2_FLUSH_BYTES = 256 << 20
GATE_CYCLES = 4_000_000  # ~2 ms device-side delay so the host queues a timed region ahead


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="disk512k")
    ap.add_argument("--theta", type=float, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched/served comparison")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch knobs")
    ap.add_argument("--no-modes", action="store_true", help="skip the precision modes' step times")
    ap.add_argument("--no-sweep", action="store_true", help="serve: skip the arrival-rate sweep")
    ap.add_argument("--no-small", action="store_true", help="skip the config-0 (16384-particle) line")
    ap.add_argument("--no-plain", action="store_true", help="batch96: skip the back-to-back plain runs")
    ap.add_argument("--requests", type=int, default=16, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--min-steps", type=int, default=100, help="serve: fewest steps of a request")
    ap.add_argument("--max-steps", type=int, default=2000, help="serve: most steps of a request")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def rank_max(dist, ms: float, device: str) -> float:
    """The slowest rank's device time: every rank contributes its own ms, all get
    the maximum (one all-reduce, the same call on every rank)."""
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(units_per_rank: float, ws: int, max_ms: float) -> float:
    """Whole-job throughput of ws replicas: all ranks' units over the slowest rank's time."""
    return units_per_rank * ws / (max_ms / 1e3)


def workload(args):
    from galaxy_sim_b200 import simulation as S

    w = S.WORKLOADS[args.workload]
    if args.theta is not None:
        w = S.with_theta(w, args.theta)
    return w


def config_of(w, g, args):
    ph = w.physics
    return {"workload": w.name, "N": int(g.N), "theta": ph.theta, "epsilon": ph.epsilon,
            "dt": ph.dt, "gas_drag": ph.gas_drag, "sf_eff": ph.sf_eff, "bucket": 16,
            "morton_bits": 30, "precision": "fp32 walk, fp32 COM refresh",
            "parallelism": f"replicas x{args.gpus} (no collective)"}


class Clocks:
    """nvidia-smi sampler during the timed region (median SM MHz under load, reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[4]), parts[6:10]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        load = [r for r in rows if r[2] > 10] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4) if r[3][k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(load)}


# Algorithmic bytes of a rebuild: bbox 16, codes 16 + 4, four sort passes of
# 8 B read + 8 B written, gather 4 + 48 read + 48 written, tree flags / scan /
# emit 5, leaf COM 16 per particle; per node 13 (emit) + 8 (leaf lists, an upper
# bound) + 41 (COM cascade).
REBUILD_BYTES_PER_PARTICLE = 16 + 20 + 64 + 100 + 5 + 16
REBUILD_BYTES_PER_NODE = 13 + 8 + 41


def hbm_peak():
    """(GB/s, where it comes from): the measured copy bandwidth of this pool's B200s,
    or the earlier measurement when the peaks file is absent."""
    p = measured_peaks().get("hbm_gbs")
    return (float(p), "measured (MEASURED_PEAKS.json)") if p else (6650.0, "fallback 6.65 TB/s")


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def restart(sim, g, w):
    """Put a Simulation back at its galaxy's seeded initial conditions: particle
    and stellar records, clock, Params and tracked centres, as Simulation sets
    them up (the launch knobs stay)."""
    from galaxy_sim_b200.simulation import params_dict

    gpu = sim.gpu
    gpu.writeState(g.particles, g.stellar)
    gpu.setTime(0.0)
    gpu.updateParams(**params_dict(g, w.physics))
    c1, c2 = g.central
    if c1 >= 0 or c2 >= 0:
        hc = g.halo_centers
        gpu.setTracking(c1, c2, hc[0] if len(hc) > 0 else None, hc[1] if len(hc) > 1 else None)
    sim.sync()


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    from galaxy_sim_b200 import _lib
    from galaxy_sim_b200.simulation import Simulation, params_dict

    torch.cuda.set_device(local)
    dist = init_dist(ws, "nccl")
    w = workload(args)
    g = w.make()
    N = g.N
    sim = Simulation(g, w.physics, device=local)
    ext = torch.cuda.ExternalStream(sim.gpu.stream, device=torch.device("cuda", local))
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    # launch knobs (walk grid, sort tile) timed on this workload; results do not depend on them
    from galaxy_sim_b200.autotune import autotune

    tuned = None
    if not args.no_tune:
        tuned = autotune(sim.gpu, steps=5, warmup=2, star_formation=sim.star_formation, device=local)
        # the tuning steps advanced the galaxy (the disk contracts, so later steps
        # cost more interactions): back to the seeded initial conditions, so the
        # timed steps are steps W .. W + K of the workload, as in the e2e leg and
        # the reference arm
        restart(sim, g, w)
    sim.run(args.warmup)
    sim.sync()
    # kernels per step, counted from the captured step graph: bbox, codes, 4 sort
    # passes, gather, 4 build kernels, walk (+SF fused), diagnostics
    n_launch_step = sim.gpu.stepKernels()
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        with torch.cuda.stream(ext):
            torch.cuda._sleep(GATE_CYCLES)  # the host queues ahead before the first timed step
        for k in range(K):
            with torch.cuda.stream(ext):
                flush.fill_(float(k))          # evict the previous step from L2 (untimed)
                starts[k].record(ext)
            sim.run(1)
            with torch.cuda.stream(ext):
                ends[k].record(ext)
        sim.sync()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    errs = sim.gpu.deviceErrors()
    if errs:
        raise RuntimeError(f"device error word 0x{errs:x} during the timed steps")
    max_ms = rank_max(dist, total_ms, f"cuda:{local}")
    value = job_value(N * K, ws, max_ms)
    clocks = clk.summary()

    # ---- walk kernel, timed alone on the same stream (roofline of the dominant kernel) ----
    sim.gpu.setDebug(True)
    sim.gpu.counters(reset=True)
    sim.gpu.sortBuild()
    sim.gpu.step()
    cnt = sim.gpu.counters(reset=True)
    sim.gpu.setDebug(False)
    interactions = cnt[0] + cnt[1]
    R = 20
    walk_ms, build_ms = [], []
    for _ in range(R):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        with torch.cuda.stream(ext):
            torch.cuda._sleep(2 * GATE_CYCLES)  # no host gap inside the timed pair
            flush.fill_(1.0)
            a.record(ext)
        sim.gpu.sortBuild()
        with torch.cuda.stream(ext):
            b.record(ext)
        sim.gpu.step()
        with torch.cuda.stream(ext):
            c.record(ext)
        sim.sync()
        build_ms.append(a.elapsed_time(b))
        walk_ms.append(b.elapsed_time(c))
    # median: a host stall longer than the gate leaves the device idle inside a pair
    walk_avg = statistics.median(walk_ms)
    import ctypes as _C

    nn, nl = _C.c_uint32(0), _C.c_uint32(0)
    _lib.check(_lib.lib().gs_get_tree(sim.gpu._ctx, None, 0, _C.byref(nn), None, 0, _C.byref(nl), None), sim.gpu._ctx)
    rb_ms = statistics.median(build_ms)
    rbytes = N * REBUILD_BYTES_PER_PARTICLE + nn.value * REBUILD_BYTES_PER_NODE
    hbm, hbm_src = hbm_peak()
    rebuild = {"ms": round(rb_ms, 4), "algorithmic_bytes": int(rbytes), "nodes": int(nn.value),
               "GBps": round(rbytes / (rb_ms / 1e3) / 1e9, 1), "peak_GBps": hbm, "peak_source": hbm_src,
               "frac": round(rbytes / (rb_ms / 1e3) / 1e9 / hbm, 4),
               "bytes_model": f"{REBUILD_BYTES_PER_PARTICLE} B/particle + {REBUILD_BYTES_PER_NODE} B/node"}
    fp32_peak = 148 * 128 * 2 * float(measured_peaks().get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    achieved = interactions * FLOPS_PER_INTERACTION / (walk_avg / 1e3) / 1e12
    roofline = {"kernel": "walk_kernel (BH walk + halo + kick-drift)", "bound": "fp32",
                "achieved": round(achieved, 3), "peak": round(fp32_peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / fp32_peak, 4),
                "peak_source": "nominal FP32 pipe: 148 SM x 128 lanes x 2 x sm_max_mhz "
                               "(MEASURED_PEAKS.json holds no FP32 figure)",
                "algorithmic": f"{interactions / N:.1f} interactions/particle x {N} particles x "
                               f"{FLOPS_PER_INTERACTION} flops per launch",
                "walk_ms": round(walk_avg, 4), "walk_ms_mean": round(sum(walk_ms) / R, 4),
                "walk_samples": R, "sort_build_refresh_ms": round(statistics.median(build_ms), 4),
                "traffic": None,
                "traffic_note": "DRAM bytes per launch come from an ncu capture of the same kernel, "
                                "not from this run (no DRAM counter is read at bench time)"}

    # ---- the precision modes' step time (same workload, same timing) ----
    precision = None
    if not args.no_modes:
        precision = {}
        for name, comp, com in (("fp32", 0, 0), ("compensated", 1, 0), ("com64", 0, 2), ("both", 1, 2)):
            restart(sim, g, w)  # every mode times the same steps of the workload
            sim.gpu.setWalkMode(bool(comp))
            sim.gpu.setComMode(com)
            sim.run(3)
            t = _timed_steps(sim.gpu.stream, local, 20, lambda: sim.run(1), flush)
            precision[name] = round(statistics.median(t), 4)
        sim.gpu.setWalkMode(False)
        sim.gpu.setComMode(0)
        precision["unit"] = "ms per full step, median of 20 (L2 flushed between steps)"
        precision["modes"] = {"fp32": "FP32 walk, FP32 COM", "compensated": "Kahan far-field sums per walk round",
                              "com64": "FP64 internal-node COM", "both": "per-round Kahan sums + FP64 COM"}

    # ---- e2e through the C ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        import ctypes as C

        L = _lib.lib()
        hp = torch.from_numpy(g.particles.reshape(-1)).pin_memory()
        hs = torch.from_numpy(g.stellar.reshape(-1)).pin_memory()
        outp = torch.empty(N * 8, dtype=torch.float32).pin_memory()
        outs = torch.empty(N * 4, dtype=torch.float32).pin_memory()
        # two frame buffers: a frame's positions stay readable while the next lands
        outpos = [torch.empty(N * 4, dtype=torch.float32).pin_memory() for _ in range(2)]
        pd = params_dict(g, w.physics)
        sim.gpu.updateParams(**pd)
        prm = sim.gpu._params
        diags = [_lib.GsDiag(), _lib.GsDiag()]
        ctx = sim.gpu._ctx
        Ke = K
        # untimed warm-up of the same calls: the readback's one-time set-up (its
        # copy stream and pinned block) and the first touch of the host buffers
        _lib.check(L.gs_write_state(ctx, hp.data_ptr(), hs.data_ptr()), ctx)
        for k in range(2):
            _lib.check(L.gs_run(ctx, 1, int(sim.star_formation)), ctx)
            _lib.check(L.gs_encode_position_readback(ctx, outpos[k].data_ptr(), C.byref(diags[k])), ctx)
            _lib.check(L.gs_await_position_readback(ctx, 0), ctx)
        _lib.check(L.gs_read_state(ctx, outp.data_ptr(), outs.data_ptr()), ctx)
        sim.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(ext):
            e0.record(ext)
        _lib.check(L.gs_write_state(ctx, hp.data_ptr(), hs.data_ptr()), ctx)
        for k in range(Ke):
            # one frame of main.js:400-507 at one step per frame: Params with the
            # clock, the step (rebuild on the device), then the frame's position
            # readback (vec4 pos + e_i per particle) with the energy diagnostics of
            # the same point. As in main.js:485-501 the readback resolves while the
            # next frame's step runs, and one is in flight at a time: a frame
            # collects the previous frame's before encoding its own.
            prm.time = k * w.physics.dt
            _lib.check(L.gs_update_params(ctx, C.byref(prm)), ctx)
            _lib.check(L.gs_run(ctx, 1, int(sim.star_formation)), ctx)
            if k:
                _lib.check(L.gs_await_position_readback(ctx, 0), ctx)
            _lib.check(L.gs_encode_position_readback(ctx, outpos[k % 2].data_ptr(),
                                                     C.byref(diags[k % 2])), ctx)
        _lib.check(L.gs_await_position_readback(ctx, 0), ctx)
        diag = diags[(Ke - 1) % 2]
        _lib.check(L.gs_read_state(ctx, outp.data_ptr(), outs.data_ptr()), ctx)
        with torch.cuda.stream(ext):
            e1.record(ext)
        torch.cuda.synchronize()
        te_ms = rank_max(dist, e0.elapsed_time(e1), f"cuda:{local}")
        if not np.isfinite(diag.e_diag) or not all(bool(torch.isfinite(b).all()) for b in outpos):
            raise RuntimeError("non-finite energy or positions in the e2e run")
        e2e = {"value": round(job_value(N * Ke, ws, te_ms), 1), "unit": UNIT,
               "h2d_bytes_per_step": int(round((N * 48 + Ke * 96) / Ke)),
               "d2h_bytes_per_step": int(round((Ke * (48 + 16 * N) + N * 48) / Ke)),
               "path": "gs_write_state (pinned) + K frames of [gs_update_params, gs_run(1), "
                       "gs_encode_position_readback (pinned, 16 B/particle + the energy diagnostics; "
                       "awaited in the next frame, as main.js keeps one readback in flight)] + "
                       "gs_read_state (pinned)",
               "steps": Ke, "ms": round(te_ms, 3)}

    # ---- config 0 (the 16384-particle disk): step and walk time per walk group size ----
    small = None
    if ws == 1 and not args.no_small:
        small = small_disk(local, flush)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, g, steps=5, warmup=1, budget_s=15.0)
    sim.close()
    batched = served = None
    if ws == 1 and not args.no_batch:
        # the metric's batched/served halves: 96 galaxies in one pool vs back-to-back
        # plain runs, and a Poisson request stream through both servers
        batched = batch_compare(local, min(K, 100), max(3, min(args.warmup, 5)))
        served = serve_compare(local, args.requests, args.rate, args.min_steps, args.max_steps,
                               rate_ceiling=(value, batched["value"]),
                               sweep=() if args.no_sweep else (1.0, 10.0, 50.0))
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    step_sorted = sorted(step_ms)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(max_ms / K, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ICs)",
        "config": config_of(w, g, args), "l2": "flush 256 MiB between timed steps",
        "latency_ms": {"p50": round(step_sorted[len(step_sorted) // 2], 5),
                       "p99": round(step_sorted[min(len(step_sorted) - 1, int(0.99 * len(step_sorted)))], 5),
                       "max": round(step_sorted[-1], 5)},
        "interactions_per_particle": round(interactions / N, 2),
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "precision_modes": precision, "config0": small, "rebuild": rebuild,
        "gpu_launches": K * n_launch_step,
        "batched": batched, "served": served, "autotune": tuned,
    }
    print(json.dumps(line), flush=True)


def small_disk(local, flush, steps=50, warmup=5):
    """Config 0 (one disk of N = 16384, eps 0.05, theta 0.5, no gas): full-step and
    walk time at several walk group sizes and splits, the default (both by galaxy
    size) first."""
    import torch

    from galaxy_sim_b200 import _lib
    from galaxy_sim_b200.autotune import launch_setting, set_
    from galaxy_sim_b200.simulation import WORKLOADS, Simulation

    w = WORKLOADS["disk16k"]
    g = w.make()
    out = {"workload": w.name, "N": int(g.N), "theta": w.physics.theta, "epsilon": w.physics.epsilon,
           "unit": "ms", "by_setting": {}}
    for wg, split in ((0, 0), (8, 1), (8, 4), (16, 2), (32, 1)):
        sim = Simulation(g, w.physics, device=local)
        set_(sim.gpu._ctx, _lib.TUNE_WALK_GROUP, wg)
        set_(sim.gpu._ctx, _lib.TUNE_WALK_SPLIT, split)
        if wg == 0:
            out["setting_in_effect"] = launch_setting(sim.gpu._ctx)
        sim.run(warmup)
        t = _timed_steps(sim.gpu.stream, local, steps, lambda: sim.run(1), flush)
        ext = torch.cuda.ExternalStream(sim.gpu.stream, device=torch.device("cuda", local))
        walk = []
        for _ in range(10):
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            with torch.cuda.stream(ext):
                torch.cuda._sleep(GATE_CYCLES // 4)
                flush.fill_(2.0)
                a.record(ext)
            sim.gpu.sortBuild()
            with torch.cuda.stream(ext):
                b.record(ext)
            sim.gpu.step()
            with torch.cuda.stream(ext):
                c.record(ext)
            sim.sync()
            walk.append(b.elapsed_time(c))
        sim.close()
        key = "by_size" if wg == 0 else f"group{wg}_split{split}"
        out["by_setting"][key] = {"ms_per_step": round(statistics.median(t), 4),
                                  "walk_ms": round(statistics.median(walk), 4)}
    d = out["by_setting"]["by_size"]
    out["ms_per_step"], out["walk_ms"] = d["ms_per_step"], d["walk_ms"]
    out["value"] = round(g.N / (d["ms_per_step"] / 1e3), 1)
    eff = out["setting_in_effect"]
    out["walk_group"] = (f"by galaxy size ({eff['walk_group']} particles per warp, walk items in "
                         f"{eff['walk_split']} parts, {eff['sort_keys_per_thread']} sort keys per thread)")
    out["walk_ms_includes"] = "walk kernel + FP64 diagnostics reduction (one gs_step)"
    return out


def cpu_baseline(w, g, steps, warmup, budget_s, nthreads=0):
    """The oracle's full step on the host cores (a bounded sample of the workload).

    Every step runs the complete codes + sort + build (one thread, like the
    reference's Web Worker) and refresh; the walk + kick-drift runs on all
    threads for every stride-th particle, stride chosen so that warmup + steps
    fit the time budget, and its time is scaled by the stride.
    """
    import numpy as np

    import oracle as O
    from galaxy_sim_b200.simulation import params_dict

    O.build()
    pd = params_dict(g, w.physics)
    hc = pd.pop("haloCenters")
    p = O.make_params(g.N, haloCenters=[c[:3] for c in hc], **pd)
    pl = O.Pipeline(g.particles, g.stellar, p, central=g.central, halo_centers=[c[:3] for c in hc],
                    nthreads=nthreads)
    sf = w.physics.sf_eff > 0
    pl.step(sf, 64)                              # probe: build time + 1/64 of the walk
    t_build, walk_full = pl.t_build, pl.t_walk * 64
    per_step = budget_s / max(1, steps + warmup)
    stride = max(1, int(np.ceil(walk_full / max(per_step - t_build, 0.02))))
    for _ in range(warmup):
        pl.step(sf, stride)
    pl.t_build = pl.t_walk = 0.0
    for _ in range(steps):
        pl.step(sf, stride)
    est_step = (pl.t_build + pl.t_walk * stride) / steps
    cores = nthreads or os.cpu_count()
    return {"value": round(g.N / est_step, 1), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} timed steps (+{warmup} warm-up) of {w.name} (N={g.N}): codes+sort+"
                      f"build+refresh on 1 thread (like the reference's Web Worker), walk+integrate "
                      f"of every {stride}-th particle on {cores} threads, walk time scaled x{stride}",
            "build_s_per_step": round(pl.t_build / steps, 4),
            "walk_s_per_step_est": round(pl.t_walk * stride / steps, 4)}


def run_reference(args, ws, rank, local):
    if rank != 0:
        return
    w = workload(args)
    g = w.make()
    cpu = cpu_baseline(w, g, steps=args.steps, warmup=args.warmup, budget_s=150.0)
    line = {
        "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * g.N / cpu["value"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ICs)", "impl": "reference",
        "config": config_of(w, g, args), "l2": "host run (no device caches involved)",
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch96(seed=7):
    from galaxy_sim_b200.simulation import batch96 as make

    return make(seed)


def _timed_steps(stream_ptr, local, K, step, flush):
    """Device time (ms) of K calls of step(), each bracketed by CUDA events on
    the given stream after an L2 flush, with a device-side gate in front."""
    import torch

    ext = torch.cuda.ExternalStream(stream_ptr, device=torch.device("cuda", local))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with torch.cuda.stream(ext):
        torch.cuda._sleep(GATE_CYCLES)
    for k in range(K):
        with torch.cuda.stream(ext):
            flush.fill_(float(k))
            ev[k][0].record(ext)
        step()
        with torch.cuda.stream(ext):
            ev[k][1].record(ext)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def batch_compare(local, K, W, tune=True, plain=True):
    """Batched ensemble (one pool, one graph per step) vs the same galaxies as
    back-to-back plain runs, same GPU, same steps."""
    import torch

    from galaxy_sim_b200.autotune import autotune
    from galaxy_sim_b200.nbody_gpu import NBodyGPU
    from galaxy_sim_b200.pool import GalaxyPool
    from galaxy_sim_b200.simulation import params_dict

    torch.cuda.set_device(local)
    gals = batch96()
    Ntot = sum(g.N for g, _ in gals)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    pool = GalaxyPool(sum((g.N + 255) // 256 * 256 for g, _ in gals), len(gals), local)

    def admit():
        for g, ph in gals:
            pool.add(g.particles, g.stellar, params_dict(g, ph), star_formation=ph.sf_eff > 0)

    admit()
    # launch knobs (walk grid, sort tile) picked by timing this batch; results do not depend on them
    tuned = None
    if tune:
        tuned = autotune(pool, steps=5, warmup=2, star_formation=True, device=local)
        # the trial steps advanced every galaxy: admit them again at their seeded
        # initial conditions (an empty pool gives the same slots and ranges; the
        # knobs stay), so the pool times the same steps as the plain runs below
        for s in list(pool.n):
            pool.remove(s)
        admit()
    pool.run(W, True)
    pool.sync()
    with Clocks(local) as clk:
        bms = _timed_steps(pool.stream, local, K, lambda: pool.run(1, True), flush)
    clocks = clk.summary()
    # the pool's rebuild alone (codes, sort, gather, build, COM), outside the step
    # graph, L2 flushed before each: achieved bandwidth over its algorithmic bytes
    rb = statistics.median(_timed_steps(pool.stream, local, 10, pool.sort_build, flush))
    nodes = sum(pool.num_nodes(sl) for sl in list(pool.n))
    rbytes = Ntot * REBUILD_BYTES_PER_PARTICLE + nodes * REBUILD_BYTES_PER_NODE
    peak, src = hbm_peak()
    rebuild = {"ms": round(rb, 4), "algorithmic_bytes": int(rbytes), "nodes": int(nodes),
               "GBps": round(rbytes / (rb / 1e3) / 1e9, 1), "peak_GBps": peak, "peak_source": src,
               "frac": round(rbytes / (rb / 1e3) / 1e9 / peak, 4),
               "bytes_model": f"{REBUILD_BYTES_PER_PARTICLE} B/particle + {REBUILD_BYTES_PER_NODE} B/node"}
    E = pool.energies()
    pool.close()
    # the same galaxies, one after another, each in its own single-galaxy context
    pms = 0.0
    plain_steps = []
    for g, ph in (gals if plain else []):
        sim = NBodyGPU(local, g.particles, g.stellar)
        sim.updateParams(**params_dict(g, ph))
        sf = ph.sf_eff > 0
        sim.run(W, sf)
        sim.sync()
        t = _timed_steps(sim.stream, local, K, lambda: sim.run(1, sf), flush)
        pms += sum(t)
        plain_steps.append(sum(t) / K)
        sim.destroy()
    b_total = sum(bms)
    srt = sorted(bms)
    value = Ntot * K / (b_total / 1e3)
    plain = Ntot * K / (pms / 1e3) if pms else None
    return {
        "value": round(value, 1), "unit": UNIT, "steps": K, "warmup": W,
        "ms_per_step": round(b_total / K, 4),
        "config": {"workload": "batch96", "galaxies": len(gals), "N_total": Ntot,
                   "N_range": [min(g.N for g, _ in gals), max(g.N for g, _ in gals)],
                   "theta": 0.5, "epsilon": 0.02, "dt": 0.005, "bucket": 16,
                   "l2": "flush 256 MiB between timed steps"},
        "latency_ms": {"p50": round(srt[len(srt) // 2], 4),
                       "p99": round(srt[min(len(srt) - 1, int(0.99 * len(srt)))], 4)},
        "plain_back_to_back": {"value": round(plain, 1), "ms_per_step_all_galaxies": round(pms / K, 4),
                               "ms_per_step_p50_galaxy": round(sorted(plain_steps)[len(plain_steps) // 2], 4)}
        if plain else None,
        "batched_over_plain": round(value / plain, 3) if plain else None,
        "autotune": tuned, "rebuild": rebuild,
        "finite_diagnostics": bool(torch.isfinite(torch.tensor(E)).all()),
        "clocks": clocks,
    }


def serve_compare(local, n_req, rate, min_steps, max_steps, rate_ceiling=(), sweep=()):
    """Served stream (Poisson arrivals) through the continuous-batching server
    and through the one-at-a-time server on the same GPU.

    ``ratio_bound`` is the largest served/plain ratio this mix allows: no server
    can finish the mix's particle-steps faster than the GPU's best measured
    per-particle rate (``rate_ceiling``: the batched server's own device rate, or
    a faster rate measured in the same run), so batched wall time >= particle-steps
    / ceiling and the ratio <= plain wall time x ceiling / particle-steps.
    ``sweep`` repeats the comparison at other arrival rates (half the requests)."""
    import torch

    from galaxy_sim_b200.serve import BatchServer, PlainServer, make_stream

    torch.cuda.set_device(local)

    def both(n, r):
        reqs = make_stream(n, r, seed=11, step_range=(min_steps, max_steps))
        srv = BatchServer(max_galaxies=64, device=local)
        with Clocks(local) as clk:
            b = srv.serve(reqs)
        srv.close()
        reqs2 = make_stream(n, r, seed=11, step_range=(min_steps, max_steps))
        p = PlainServer(local).serve(reqs2)
        return b, p, clk.summary()

    b, p, clocks = both(n_req, rate)
    ps = b["particle_steps"]
    ceiling = max([ps / b["gpu_busy_s"]] + [x for x in rate_ceiling if x])
    bound = {"value": round(p["wall_s"] * ceiling / ps, 3), "rate_ceiling": round(ceiling, 1),
             "plain_wall_s": p["wall_s"], "plain_device_s": p["gpu_busy_s"],
             "batched_wall_s": b["wall_s"], "batched_device_s": b["gpu_busy_s"],
             "particle_steps": ps}
    rows = []
    for r in sweep:
        n = max(4, n_req // 2)
        sb, sp, _ = both(n, r)
        rows.append({"rate_per_s": r, "requests": n, "batched": sb["value"], "plain": sp["value"],
                     "batched_over_plain": round(sb["value"] / sp["value"], 3),
                     "batched_step_ms_p50": sb["step_ms"]["p50"], "batched_step_ms_p99": sb["step_ms"]["p99"]})
    return {"value": b["value"], "unit": UNIT,
            "config": {"workload": "serve", "requests": n_req, "rate_per_s": rate,
                       "N_range": [8192, 1 << 20], "steps_range": [min_steps, max_steps],
                       "presets": ["disk", "sphere", "collision"], "eps": [0.02, 0.05],
                       "theta": [0.5, 0.7], "dt": [0.0025, 0.005]},
            "batched": b, "plain": p, "batched_over_plain": round(b["value"] / p["value"], 3),
            "ratio_bound": bound, "rate_sweep": rows, "clocks": clocks}


def _mode_line(d):
    line = {"metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ICs)"}
    line.update({k: v for k, v in d.items() if k not in ("value", "unit")})
    return line


def run_batch(args, ws, rank, local):
    if rank != 0:
        return
    print(json.dumps(_mode_line(batch_compare(local, args.steps, args.warmup, tune=not args.no_tune,
                                              plain=not args.no_plain))), flush=True)


def run_serve(args, ws, rank, local):
    if rank != 0:
        return
    d = serve_compare(local, args.requests, args.rate, args.min_steps, args.max_steps,
                      sweep=() if args.no_sweep else (1.0, 10.0, 50.0))
    print(json.dumps(_mode_line(d)), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank, local)
    elif args.workload == "batch96":
        run_batch(args, ws, rank, local)
    elif args.workload == "serve":
        run_serve(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
