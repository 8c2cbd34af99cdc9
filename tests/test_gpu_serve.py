"""Serving with continuous batching: every request's result is the same alone
and in the mix.

A small stream of mixed presets (disk, sphere, collision with halo tracking),
sizes, step counts and eps/theta/dt goes through a BatchServer whose pool is
too small to hold all of it at once, so requests wait for admission, share
batched steps with whatever else is resident and are released when done. Each
result (particles, stellar records, FP64 diagnostics) must be bit-identical to
the same simulation run alone in its own context.
"""
import numpy as np
import pytest

from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.serve import BatchServer, PlainServer, make_stream

pytestmark = pytest.mark.gpu


def _alone(r, walk_group=None, walk_split=None):
    sim = NBodyGPU(0, r.particles, r.stellar, walkGroup=walk_group, walkSplit=walk_split)
    sim.updateParams(**r.params)
    if r.tracking is not None:
        sim.setTracking(*r.tracking)
    sim.run(r.steps, r.star_formation)
    P, S = sim.readState()
    e = sim.energy()
    sim.destroy()
    return P, S, e


def test_served_results_equal_alone(gpu_lib):
    reqs = make_stream(7, rate=400.0, seed=3, n_range=(1000, 20000), step_range=(2, 9))
    srv = BatchServer(capacity=32768, max_galaxies=3)
    stats = srv.serve(reqs)
    srv.close()
    assert all(r.result is not None for r in reqs)
    assert stats["particle_steps"] == sum(r.N * r.steps for r in reqs)
    assert stats["step_ms"]["n"] >= max(r.steps for r in reqs)
    # the pool held at most three galaxies: some requests had to wait
    assert max(r.admitted - r.arrival for r in reqs) > 0
    for r in reqs:
        P, S, e = _alone(r, walk_group=32, walk_split=1)   # the pool's walk group, unsplit
        RP, RS, re_ = r.result
        assert np.array_equal(RP.view(np.uint32), P.view(np.uint32)), r.rid
        assert np.array_equal(RS.view(np.uint32), S.view(np.uint32)), r.rid
        assert re_ == e, r.rid


def test_plain_server_matches(gpu_lib):
    reqs = make_stream(3, rate=1000.0, seed=4, n_range=(2000, 8000), step_range=(2, 4))
    stats = PlainServer().serve(reqs)
    assert stats["value"] > 0
    for r in reqs:
        P, S, e = _alone(r)
        assert np.array_equal(r.result[0].view(np.uint32), P.view(np.uint32))
