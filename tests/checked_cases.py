"""Small runs through every kernel the checked build guards, shared by
tests/test_checked_build.py (ordinary library, in process) and by a child
process that loads the checked library (LBM2D_LIBRARY):

    python tests/checked_cases.py OUT.npz

- multi-particle sedimentation, 256 x 512, 100 disks, 300 steps, FP64 and
  FP32 (step kernel with listed tiles, particle kernel with pair lists, tile
  lists and history records);
- the C6 Bingham case with stress records, FP32 (omega staged with the
  tile);
- a batch of three runs (two C6, one C1) on the TMA tiles, 40 steps;
- the adjoint of the C3 pair case, FP64 (the forward recompute).
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))


def _sim(pkg, p, pin, steps):
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    sim.step(steps)
    out = {"particles": sim.particles(), "ux": sim.field("ux"), "series": sim.series(),
           "status": np.array(sim.status())}
    sim.close()
    return out


def run_cases(pkg) -> dict:
    cases = pkg.cases
    res = {}
    for prec in (0, 1):
        p, pin = cases.workload_cfg2(prec, 256, 512, 100)
        for k, v in _sim(pkg, p, pin, 300).items():
            res[f"sed{prec}_{k}"] = v
    p, disk = cases.shipped_c6(80, 240)
    p.precision = 1
    p.record_stress = 1
    p.series_every = 5
    p.series_particles = 1
    for k, v in _sim(pkg, p, disk, 300).items():
        res[f"c6_{k}"] = v
    runs = []
    for w in (80, 96):
        q, d = cases.shipped_c6(w, 240)
        q.precision = 1
        runs.append((q, d))
    q = cases.shipped_c1(72, 200, 12.0)
    q.precision = 1
    runs.append((q, cases.pin_array([[36.0, 150.0]], 12.0, 1.25)))
    b = pkg.Batch([q for q, _ in runs])
    b.set_tuning(64, 8, 2)
    for s, (_, d) in zip(b.sims, runs):
        s.set_particles(d)
    b.step(40)
    for i, s in enumerate(b.sims):
        res[f"batch{i}_particles"] = s.particles()
        res[f"batch{i}_status"] = np.array(s.status())
    b.close()
    import adjoint_cases as ac

    p, pin, n0, n1 = ac.build(cases, "c3_pair")
    sim = pkg.Simulation(p.copy(precision=0))
    sim.set_particles(pin)
    j, g = sim.adjoint(n0, n1)
    res["adj_j"] = np.array(j)
    res["adj_grad"] = np.concatenate([np.atleast_1d(np.asarray(g[k], dtype=np.float64))
                                      for k in ("tau_y", "nu", "rho_p", "x0", "y0")])
    res["adj_status"] = np.array(sim.status())
    sim.close()
    res["checked_build"] = np.array(int(pkg.load_library().lbm_checked_build()))
    return res


if __name__ == "__main__":
    pkg = importlib.import_module("2d_nnf_lbm_b200")
    np.savez(sys.argv[1], **run_cases(pkg))
