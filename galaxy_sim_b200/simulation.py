"""Headless driver of the gravity path: the physics half of the reference's
frame loop (src/main.js:337-507) with the tree rebuilt on the device every step.

``Simulation`` wires a generated galaxy (initial_conditions.Galaxy) and its
physics parameters into an ``NBodyGPU`` context, the way ``init`` and ``loop``
in main.js do: Params per NBodyGPU.updateParams, halos centred on the tracked
central particles (main.js:276-283, :449-457), star formation once per step
with sfDt = dt (one step per frame).
"""
from __future__ import annotations

from dataclasses import dataclass, replace

from . import initial_conditions as ic
from .nbody_gpu import NBodyGPU


@dataclass(frozen=True)
class Physics:
    epsilon: float
    theta: float
    dt: float
    G: float = 1.0
    gas_drag: float = 0.0
    sf_eff: float = 0.0
    aging_rate: float = 25.0


@dataclass(frozen=True)
class Workload:
    name: str
    make: object          # () -> Galaxy
    physics: Physics
    steps: int


WORKLOADS = {
    # single disk N=16384, eps 0.05, theta 0.5, dt 0.005, no gas, 100 steps
    "disk16k": Workload("disk16k", ic.disk_16k, Physics(0.05, 0.5, 0.005), 100),
    # single disk N=524288, 30% gas + drag + star formation, eps 0.02, theta 0.5
    "disk512k": Workload("disk512k", ic.disk_512k,
                         Physics(0.02, 0.5, 0.005, gas_drag=0.25, sf_eff=0.02), 1000),
    "disk512k_t07": Workload("disk512k_t07", ic.disk_512k,
                             Physics(0.02, 0.7, 0.005, gas_drag=0.25, sf_eff=0.02), 1000),
    # two disks of 262144 with black holes on a parabolic orbit, eps 0.02, theta 0.5
    "collision512k": Workload("collision512k", ic.collision_2x256k, Physics(0.02, 0.5, 0.005), 2000),
}


def batch96(seed: int = 7) -> list:
    """The batched-ensemble workload: 96 disks with N log-uniform in [4096, 262144],
    Q uniform in [1, 2], 2-4 arms, gas fraction 0 or 0.3 (gas: drag + star
    formation), eps 0.02, theta 0.5, dt 0.005. Returns (Galaxy, Physics) pairs."""
    import math

    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for k in range(96):
        N = int(round(math.exp(rng.uniform(math.log(4096), math.log(262144)))))
        Q = float(rng.uniform(1.0, 2.0))
        arms = int(rng.integers(2, 5))
        gas = float(rng.choice([0.0, 0.3]))
        g = ic.galaxy_disk(N, 1000 + k, Q=Q, arms=arms, gas_frac=gas)
        ph = Physics(0.02, 0.5, 0.005, gas_drag=0.25 if gas else 0.0, sf_eff=0.02 if gas else 0.0)
        out.append((g, ph))
    return out


def params_dict(galaxy: "ic.Galaxy", ph: Physics, time: float = 0.0) -> dict:
    """NBodyGPU.updateParams arguments for a galaxy (main.js:414-427)."""
    return dict(dt=ph.dt, G=ph.G, epsilon=ph.epsilon, theta=ph.theta,
                haloMass=galaxy.halo_mass if galaxy.halo_centers else 0.0, haloA=galaxy.halo_a,
                gasDrag=ph.gas_drag, time=time, agingRate=ph.aging_rate,
                sfDensity=galaxy.sf_density, sfEff=ph.sf_eff, sfDt=ph.dt,
                haloCenters=[list(c) + [0.0] for c in galaxy.halo_centers[:2]])


class Simulation:
    def __init__(self, galaxy: "ic.Galaxy", physics: Physics, device: int = 0, com_mode: int = 0):
        self.galaxy = galaxy
        self.physics = physics
        self.gpu = NBodyGPU(device, galaxy.particles, galaxy.stellar)
        self.gpu.updateParams(**params_dict(galaxy, physics))
        c1, c2 = galaxy.central
        if c1 >= 0 or c2 >= 0:
            hc = galaxy.halo_centers
            self.gpu.setTracking(c1, c2, hc[0] if len(hc) > 0 else None,
                                 hc[1] if len(hc) > 1 else None)
        if com_mode:
            self.gpu.setComMode(com_mode)
        self.star_formation = physics.sf_eff > 0.0

    @property
    def N(self) -> int:
        return self.gpu.N

    def run(self, nsteps: int) -> None:
        self.gpu.run(nsteps, self.star_formation)

    def sync(self) -> None:
        self.gpu.sync()

    def close(self) -> None:
        self.gpu.destroy()


def with_theta(w: Workload, theta: float) -> Workload:
    return replace(w, physics=replace(w.physics, theta=theta))
