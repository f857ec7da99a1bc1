"""Run one of the benchmark workloads for a few steps and print a summary.

    python -m 2d_nnf_lbm_b200.run_workload --precision fp32 --steps 30
    python -m 2d_nnf_lbm_b200.run_workload --adjoint --steps 200
    python -m 2d_nnf_lbm_b200.run_workload --batch 32 --steps 7

A short, self-contained run of the library, used for profiling single
kernel launches without the timing harness around them:
  default    the multi-particle sedimentation workload (1024 x 2048 cells,
             512 disks of diameter 16), lbm_step
  --adjoint  the adjoint workload (400 x 1200, one Bingham disk), lbm_adjoint
             with the objective window over the last 100 steps
  --batch N  the first N runs of the batched workload (Bingham single-disk
             runs of widths 128..512), lbm_batch_step with 32 x 8 tiles and
             6 blocks per SM
Prints the step count, the first disk's centre (or J and its gradient) and
the device status.
"""

from __future__ import annotations

import argparse
import importlib
import os
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--particles", type=int, default=512)
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--batch", type=int, default=0)
    a = ap.parse_args(argv)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    pkg = importlib.import_module("2d_nnf_lbm_b200")
    prec = 1 if a.precision == "fp32" else 0
    if a.adjoint:
        p, pin, _ = pkg.cases.workload_cfg5(prec)
        with pkg.Simulation(p) as sim:
            sim.set_particles(pin)
            j, g = sim.adjoint(max(1, a.steps - 100), a.steps)
            print(f"steps {sim.kk}  J {j:.9e}  dJ/dtau_y {g['tau_y']:.9e}  status {sim.status()}")
        return 0
    if a.batch > 0:
        cs = pkg.cases.workload_cfg4(prec)[: a.batch]
        b = pkg.Batch([q for q, _ in cs])
        b.set_tuning(32, 8, 6)
        for s, (_, disks) in zip(b.sims, cs):
            s.set_particles(disks)
        b.step(a.steps)
        parts = b.sims[0].particles()
        print(f"steps {b.sims[0].kk}  run 0 disk at ({parts[0, 0]:.6f}, {parts[0, 1]:.6f})  "
              f"status {max(s.status() for s in b.sims)}")
        b.close()
        return 0
    p, pin = pkg.cases.workload_cfg2(prec, a.nx, a.ny, a.particles)
    with pkg.Simulation(p) as sim:
        sim.set_particles(pin)
        sim.step(a.steps)
        parts = sim.particles()
        print(f"steps {sim.kk}  disk 0 at ({parts[0, 0]:.6f}, {parts[0, 1]:.6f})  "
              f"status {sim.status()}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
