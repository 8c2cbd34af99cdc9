"""Host-side fault injection (nothing faults, traps or hangs on the GPU).

* A device allocation that fails (gs_test_fail_alloc makes the n-th one report
  out-of-memory) at any point while a context is being set up: gs_create returns
  GS_ENOMEM with a message, leaves no context behind and gives back what it had
  allocated; the next context works.
* Admission over budget: a pool with no free contiguous particle range or no
  free slot refuses a galaxy (GS_ENOMEM, None from GalaxyPool.add) without
  touching the galaxies it holds, and admits it once room is made.
"""
import ctypes as C

import numpy as np
import pytest

from galaxy_sim_b200 import _lib
from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.nbody_gpu import NBodyGPU
from galaxy_sim_b200.pool import GalaxyPool, device_memory

pytestmark = pytest.mark.gpu

KW = dict(dt=0.005, G=1.0, epsilon=0.05, theta=0.5)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_device_allocation_failure_unwinds(gpu_lib):
    L = _lib.lib()
    g = ic.disk_16k()
    P = np.ascontiguousarray(g.particles, np.float32)
    S = np.ascontiguousarray(g.stellar, np.float32)
    probe = NBodyGPU(0, g.particles, g.stellar)  # loads the module, so the baseline holds it
    probe.destroy()
    free0, _ = device_memory(0)
    try:
        for nth in (0, 1, 10, 30):  # a context makes about 40 device allocations
            _lib.check(L.gs_test_fail_alloc(nth))
            h = C.c_void_p()
            rc = L.gs_create(g.N, P.ctypes.data, S.ctypes.data, C.byref(h))
            assert rc == _lib.GS_ENOMEM, (nth, rc)
            assert not h.value
            assert "out of memory" in L.gs_last_error(None).decode()
    finally:
        L.gs_test_fail_alloc(-1)
    free1, _ = device_memory(0)
    assert abs(free1 - free0) <= 16 << 20, (free0, free1)
    sim = NBodyGPU(0, g.particles, g.stellar)
    sim.updateParams(**KW)
    sim.run(2, False)
    P2, _ = sim.readState()
    assert np.all(np.isfinite(P2)) and sim.deviceErrors() == 0
    sim.destroy()


def test_pool_refuses_what_does_not_fit(gpu_lib):
    a = ic.galaxy_disk(3000, 1, gas_frac=0.0)
    b = ic.galaxy_disk(2000, 2, gas_frac=0.0)
    c = ic.galaxy_disk(500, 3, gas_frac=0.0)
    # room for a (3072 after alignment) but not also for b (2048 more)
    pool = GalaxyPool(4352, 2)
    sa = pool.add(a.particles, a.stellar, KW)
    assert sa is not None
    assert pool.free() == (4352 - 3072, 1) and not pool.fits(b.N)
    assert pool.add(b.particles, b.stellar, KW) is None
    assert pool.free() == (4352 - 3072, 1)  # the refusal took nothing
    pool.run(2, False)
    solo = NBodyGPU(0, a.particles, a.stellar, walkGroup=32, walkSplit=1)  # the pool's walk group
    solo.updateParams(**KW)
    solo.run(2, False)
    assert _same(pool.read_state(sa)[0], solo.readState()[0])
    solo.destroy()
    pool.remove(sa)
    sb = pool.add(b.particles, b.stellar, KW)
    assert sb is not None
    pool.close()
    # no free slot
    one = GalaxyPool(8192, 1)
    assert one.add(c.particles, c.stellar, KW) is not None
    assert one.add(c.particles, c.stellar, KW) is None
    assert one.free() == (8192 - 512, 0)
    one.close()
