"""Generate the energy-drift fixture of the disk512k workload from the oracle.

Run from the repository root:  python tests/golden/make_drift_golden.py [--steps 1000]

The oracle's pipeline (oracle/pipeline.cpp: the reference's scheme restated in
FP32, with the tree rebuilt from the current positions every step, gas drag and
star formation as in src/physics/shaders/nbody_bh.wgsl) runs the seeded
N = 524288 disk (30% gas, drag 0.25, star formation efficiency 0.02, eps 0.02,
theta 0.5, dt 0.005) for 1000 steps. At step 1 and every 10 steps it records
both energy diagnostics of the state the step wrote: the HUD's unweighted sum
of the specific energies e_i (bhWorker.js:74) and the true energy sum m_i e_i,
each summed in FP64. The run takes about 15 minutes on 8 cores, which is why the
GPU test compares against this committed trajectory instead of rerunning it.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from galaxy_sim_b200.simulation import WORKLOADS, params_dict  # noqa: E402


def energies(P, e):
    m = P[:, 3].astype(np.float64)
    return float(np.sum(e.astype(np.float64))), float(np.sum(m * e.astype(np.float64)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--workload", default="disk512k")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    O.build()
    w = WORKLOADS[a.workload]
    g = w.make()
    pd = params_dict(g, w.physics)
    hc = pd.pop("haloCenters")
    p = O.make_params(g.N, haloCenters=[c[:3] for c in hc], **pd)
    pl = O.Pipeline(g.particles, g.stellar, p, central=g.central, halo_centers=[c[:3] for c in hc])
    sf = w.physics.sf_eff > 0
    rec = []
    t0 = time.time()
    for k in range(1, a.steps + 1):
        pl.step(sf)
        if k == 1 or k % a.every == 0:
            ed, et = energies(pl.P, pl.energy)
            rec.append([k, ed, et])
            print(f"step {k}: e_diag {ed:.9e} e_true {et:.9e} ({time.time() - t0:.0f} s)", flush=True)
    out = {"workload": w.name, "N": int(g.N), "physics": w.physics.__dict__, "steps": a.steps,
           "columns": ["step", "e_diag", "e_true"], "records": rec,
           "generator": "tests/golden/make_drift_golden.py (oracle.Pipeline, FP32 reference scheme)"}
    path = a.out or os.path.join(HERE, f"drift_{w.name}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path)


if __name__ == "__main__":
    main()
