"""Full on-device steps against the oracle's pipeline (oracle/pipeline.cpp).

* One step: the same initial state through gs_run (codes, sort, gather, build,
  refresh, walk + halo + kick-drift + gas drag, star formation) and through
  the oracle. The rebuild is bit-exact, so both end in the same particle order;
  positions and velocities agree to FP32 walk tolerance, and the star-formation
  decisions agree.
* Energy drift over 1000 steps (the third correctness tier): the device run and
  the FP32 oracle run drift by the same small amount.
"""
import numpy as np
import pytest

from galaxy_sim_b200 import initial_conditions as ic
from galaxy_sim_b200.simulation import Physics, Simulation, params_dict

pytestmark = pytest.mark.gpu


def _oracle_pipeline(oracle, g, ph):
    pd = params_dict(g, ph)
    hc = pd.pop("haloCenters")
    p = oracle.make_params(g.N, haloCenters=[c[:3] for c in hc], **pd)
    return oracle.Pipeline(g.particles, g.stellar, p, central=g.central,
                           halo_centers=[c[:3] for c in hc])


def _energy(P, e):
    m = P[:, 3].astype(np.float64)
    return float(np.sum(e.astype(np.float64))), float(np.sum(m * e))


@pytest.mark.parametrize("which", ["disk_gas_sf", "collision"])
def test_one_full_step_matches_oracle(gpu_lib, oracle, which):
    if which == "disk_gas_sf":
        g = ic.disk_512k(N=65536)
        ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.5)
        g.sf_density = g.sf_density * 0.2   # make star formation fire in one step
    else:
        g = ic.two_galaxy_collision(65536, 9, Q=1.5, arms=2, gas_frac=0.0)
        ph = Physics(0.02, 0.5, 0.005)
    sim = Simulation(g, ph)
    sim.run(1)
    P, S = sim.gpu.readState()
    c1, c2, h1, h2 = sim.gpu.getTracking()
    pl = _oracle_pipeline(oracle, g, ph)
    pl.step(do_sf=ph.sf_eff > 0)
    WP, WS = pl.P, pl.S
    scale = np.abs(WP[:, :3]).max()
    vscale = np.abs(WP[:, 4:7]).max()
    assert np.abs(P[:, 3] - WP[:, 3]).max() == 0.0          # same order, same masses
    assert np.abs(P[:, :3] - WP[:, :3]).max() < 1e-5 * scale
    assert np.abs(P[:, 4:7] - WP[:, 4:7]).max() < 1e-4 * vscale
    gas = WP[:, 7] < -0.5
    if which == "disk_gas_sf":
        # densities of own leaves agree wherever both walks visited the same leaf
        assert np.mean(P[gas, 7] == WP[gas, 7]) > 0.999
        formed_w = (pl.S[:, 0] > 0) & (g.stellar[:, 0].min() < 0)
        assert np.mean((S[:, 0] == -1) == (WS[:, 0] == -1)) > 0.999
    else:
        assert (c1, c2) == (int(pl.state.central[0]), int(pl.state.central[1]))
        for h, hc in ((0, h1), (1, h2)):
            want = np.array([pl.state.haloC[h][k] for k in range(3)])
            assert np.abs(hc - want).max() < 1e-9 * max(1.0, np.abs(want).max())
    sim.close()


def test_energy_drift_1000_steps_matches_oracle(gpu_lib, oracle):
    g = ic.disk_16k()
    ph = Physics(0.05, 0.5, 0.005)
    steps = 1000
    sim = Simulation(g, ph)
    sim.run(1)
    e0 = sim.gpu.energy()
    sim.run(steps - 1)
    e1 = sim.gpu.energy()
    gpu_true = (e1["e_true"] - e0["e_true"]) / abs(e0["e_true"])
    gpu_diag = (e1["e_diag"] - e0["e_diag"]) / abs(e0["e_diag"])
    p_mom = np.linalg.norm(np.array(e1["momentum"]) - np.array(e0["momentum"]))
    sim.close()

    pl = _oracle_pipeline(oracle, g, ph)
    pl.step()
    d0 = _energy(pl.P, pl.energy)
    for _ in range(steps - 1):
        pl.step()
    d1 = _energy(pl.P, pl.energy)
    cpu_diag = (d1[0] - d0[0]) / abs(d0[0])
    cpu_true = (d1[1] - d0[1]) / abs(d0[1])
    print(f"\nenergy drift over {steps} steps: device true {gpu_true:+.3e} diag {gpu_diag:+.3e}; "
          f"oracle true {cpu_true:+.3e} diag {cpu_diag:+.3e}; |dp| {p_mom:.2e}")
    assert abs(gpu_true) < 5e-3 and abs(cpu_true) < 5e-3
    assert abs(gpu_true - cpu_true) < 2e-3
    assert abs(gpu_diag - cpu_diag) < 2e-3 + 0.5 * abs(cpu_diag)
