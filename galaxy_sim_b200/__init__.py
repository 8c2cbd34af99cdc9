"""galaxy_sim_b200 — B200 (sm_100a) gravity path of galaxy-sim.

* ``morton_tree``: the exports of src/physics/mortonTree.js (GPU-backed).
* ``nbody_gpu``: the NBodyGPU class of src/physics/NBodyGPU.js (GPU-backed).
* ``simulation``: headless frame loop (src/main.js physics half) and workloads.
* ``initial_conditions``: seeded galaxy generators (src/physics/InitialConditions.js).

All compute runs in ``libgalaxy_b200.so`` (C ABI: include/galaxy_b200.h).
"""
from . import initial_conditions  # noqa: F401

__all__ = ["initial_conditions", "morton_tree", "nbody_gpu", "simulation"]
