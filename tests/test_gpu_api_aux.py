"""Calls beyond the NBodyGPU surface.

* Checkpoint and restore: the particle and stellar records (gs_read_state /
  gs_write_state), the simulation clock (gs_set_time) and the tracked centres
  (gs_get_tracking / gs_set_tracking) are the whole state of a galaxy between
  full steps, so a run stopped after 2 steps and resumed in a fresh context for 3
  more equals an uninterrupted 5-step run bit for bit (star formation on, which
  reads the clock; tracked halos on, which read the centres).
* The walk's interaction counters (gs_counters) agree with the FP64 walk of the
  same acceptance rule on the same tree, up to the few borderline acceptances
  that FP32 and FP64 decide differently; reset returns and clears them.
* gs_sync waits for queued work, bounded by a timeout; a wait that times out
  leaves the queued work and the context intact.
* gs_update_params queues its copy without draining the stream; queued updates
  and steps give what the same calls give one at a time.
* The asynchronous position readback (gs_encode_position_readback /
  gs_await_position_readback) delivers the state of the step it followed while
  later steps run, one readback in flight at a time, with a bounded await.
"""
import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.simulation import Physics, Simulation, params_dict

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_checkpoint_restore_continues_bit_identical(gpu_lib):
    g = ic.two_galaxy_collision(20000, 7, gas_frac=0.3)
    ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.05)
    whole = Simulation(g, ph)
    whole.run(5)
    want_P, want_S = whole.gpu.readState()
    want_tr = whole.gpu.getTracking()
    want_e = whole.gpu.energy()
    whole.close()

    first = Simulation(g, ph)
    first.run(2)
    P2, S2 = first.gpu.readState()
    c1, c2, h1, h2 = first.gpu.getTracking()
    first.close()
    t = 0.0  # the clock: a double advanced by the f32 dt once per full step
    for _ in range(2):
        t += float(np.float32(ph.dt))

    resumed = NBodyGPU(0, P2, S2)
    resumed.updateParams(**params_dict(g, ph))
    resumed.setTime(t)
    resumed.setTracking(c1, c2, h1, h2)
    resumed.run(3, True)
    got_P, got_S = resumed.readState()
    got_tr = resumed.getTracking()
    got_e = resumed.energy()
    assert resumed.deviceErrors() == 0
    resumed.destroy()
    assert _same(got_P, want_P) and _same(got_S, want_S)
    assert got_tr[:2] == want_tr[:2]
    assert np.array_equal(got_tr[2], want_tr[2]) and np.array_equal(got_tr[3], want_tr[3])
    assert got_e == want_e


def test_bench_restart_equals_a_fresh_start(gpu_lib):
    """bench.py times its steps from the seeded initial conditions after tuning
    the same context: its restart must leave nothing of the steps before."""
    import os
    import sys
    from types import SimpleNamespace

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    g = ic.two_galaxy_collision(20000, 7, gas_frac=0.3)
    ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.05)
    fresh = Simulation(g, ph)
    fresh.run(3)
    want_P, want_S = fresh.gpu.readState()
    want_tr, want_e = fresh.gpu.getTracking(), fresh.gpu.energy()
    fresh.close()

    sim = Simulation(g, ph)
    sim.run(6)
    bench.restart(sim, g, SimpleNamespace(physics=ph))
    sim.run(3)
    got_P, got_S = sim.gpu.readState()
    got_tr, got_e = sim.gpu.getTracking(), sim.gpu.energy()
    assert sim.gpu.deviceErrors() == 0
    sim.close()
    assert _same(got_P, want_P) and _same(got_S, want_S)
    assert got_tr[:2] == want_tr[:2]
    assert np.array_equal(got_tr[2], want_tr[2]) and np.array_equal(got_tr[3], want_tr[3])
    assert got_e == want_e


def test_walk_counters_match_the_fp64_walk(gpu_lib, oracle):
    g = ic.disk_16k()
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    sim.setDebug(True)
    sim.sortBuild()
    P, _ = sim.readState()
    want = oracle.sort_and_build(g.particles, g.stellar)
    com64 = oracle.refresh_f64(P, want["nodes"], want["levelRanges"])
    sim.counters(reset=True)
    sim.step()
    mono, pairs, visits = sim.counters()
    p = oracle.make_params(g.N, epsilon=0.05, theta=0.5, dt=0.005)
    _, _, _, cnt = oracle.walk_f64(p, P, want["nodes"], com64)
    assert mono > 0 and pairs > 0 and visits >= mono
    assert abs(int(mono) - int(cnt[0])) <= 1e-3 * int(cnt[0]), (mono, cnt[0])
    assert abs(int(pairs) - int(cnt[1])) <= 1e-3 * int(cnt[1]), (pairs, cnt[1])
    assert sim.counters(reset=True) == [mono, pairs, visits]
    assert sim.counters() == [0, 0, 0]
    sim.destroy()


def test_sync_waits_for_queued_steps(gpu_lib):
    g = ic.disk_16k()
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    assert sim.stream != 0
    sim.run(20, False)
    sim.sync(timeout_ns=10_000_000_000)  # returns once the 20 steps are done
    P, _ = sim.readState()
    assert np.all(np.isfinite(P)) and sim.deviceErrors() == 0
    sim.destroy()


def test_sync_timeout_leaves_the_context_usable(gpu_lib):
    """A bounded host wait that expires returns GS_ETIMEDOUT without touching the
    queued work; a later wait sees it finish with no device error."""
    g = ic.disk_16k()
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    sim.run(2000, False)                       # about half a second of queued steps
    with pytest.raises(_lib.GalaxyError) as e:
        sim.sync(timeout_ns=1)
    assert e.value.code == _lib.GS_ETIMEDOUT
    sim.sync(timeout_ns=60_000_000_000)
    P, _ = sim.readState()
    assert np.all(np.isfinite(P)) and sim.deviceErrors() == 0
    sim.destroy()


def test_async_position_readback_follows_its_step(gpu_lib):
    """gs_encode_position_readback / gs_await_position_readback, driven as
    main.js:485-501 drives encodePositionReadback and the readPositions promise
    (NBodyGPU.js:334-348): each frame queues its step, collects the previous
    frame's readback and encodes its own, so a readback is collected after the
    next step was queued. Every readback holds vec4(pos, e_i) and the energy
    diagnostics of the step it followed: the synchronous readback and gs_energy
    of a second context stepped in lock step, bit for bit. One readback is in
    flight at a time (a second encode returns GS_ENOTREADY, leaving the first
    intact); an await with nothing in flight is GS_EINVAL."""
    import ctypes as C

    import torch

    g = ic.disk_16k()
    kw = dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    a, b = NBodyGPU(0, g.particles, g.stellar), NBodyGPU(0, g.particles, g.stellar)
    a.updateParams(**kw)
    b.updateParams(**kw)
    L = _lib.lib()
    bufs = [torch.empty(4 * g.N, dtype=torch.float32).pin_memory() for _ in range(2)]
    diags = [_lib.GsDiag(), _lib.GsDiag()]
    assert L.gs_await_position_readback(a._ctx, 0) == _lib.GS_EINVAL
    got, want = [], []

    def collect(k):
        _lib.check(L.gs_await_position_readback(a._ctx, 0), a._ctx)
        d = diags[k % 2]
        got.append((bufs[k % 2].numpy().copy(), (d.e_diag, d.e_true, *d.momentum, d.mass)))

    for k in range(4):
        a.run(1, False)
        if k:
            collect(k - 1)
        _lib.check(L.gs_encode_position_readback(a._ctx, bufs[k % 2].data_ptr(), C.byref(diags[k % 2])),
                   a._ctx)
        assert L.gs_encode_position_readback(a._ctx, bufs[(k + 1) % 2].data_ptr(), None) == _lib.GS_ENOTREADY
        b.run(1, False)
        e = b.energy()
        want.append((b.readPositions(), (e["e_diag"], e["e_true"], *e["momentum"], e["mass"])))
    collect(3)
    for (gp, gd), (wp, wd) in zip(got, want):
        assert _same(gp, wp)
        assert gd == wd
    assert a.deviceErrors() == 0
    a.destroy()
    b.destroy()


def test_async_position_readback_timeout_and_python_mirror(gpu_lib):
    """A bounded await that expires returns GS_ETIMEDOUT and leaves the readback in
    flight; a later await collects it. The Python mirror's encodePositionReadback
    + readPositions return the positions of the point the readback was encoded at,
    even with more steps queued after it."""
    import torch

    g = ic.disk_16k()
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)
    # pinned: a copy into pageable memory returns only once it is done
    staging = torch.empty(4 * g.N, dtype=torch.float32).pin_memory().numpy()
    sim.run(1000, False)                       # a few hundred ms of queued steps
    sim.encodePositionReadback(staging=staging)
    with pytest.raises(_lib.GalaxyError) as e:
        sim.readPositions(timeout_ns=1)
    assert e.value.code == _lib.GS_ETIMEDOUT
    late = sim.readPositions(timeout_ns=60_000_000_000)
    assert _same(late, sim.readPositions())    # nothing queued since: the same state
    sim.encodePositionReadback()
    sim.run(3, False)
    before = sim.readPositions()
    after = sim.readPositions()
    assert not _same(before, after) and np.all(np.isfinite(before))
    assert sim.readbackEnergy["mass"] > 0 and sim.deviceErrors() == 0
    sim.destroy()


def test_params_updates_queue_without_waiting(gpu_lib):
    """gs_update_params queues its copy behind the work already queued and does
    not drain the stream (a ring of pinned staging entries, each reused only after
    its copy has run). Twenty frames of [update with a new clock and theta, one full
    step] queued without any wait, more frames than the ring has entries, end
    bit-identical to the same frames run with a wait after each."""
    g = ic.disk_16k()
    runs = []
    for wait in (False, True):
        sim = NBodyGPU(0, g.particles, g.stellar)
        for k in range(20):
            sim.updateParams(dt=0.005, G=1.0, epsilon=0.05, theta=0.5 if k % 2 else 0.7, time=0.005 * k)
            sim.run(1, False)
            if wait:
                sim.sync()
        sim.sync()
        runs.append(sim.readState())
        assert sim.deviceErrors() == 0
        sim.destroy()
    assert _same(runs[0][0], runs[1][0]) and _same(runs[0][1], runs[1][1])
