"""Run one of the benchmark workloads for a few steps and print a summary.

    python -m 2d_nnf_lbm_b200.run_workload --precision fp32 --steps 30

A short, self-contained run of the library on the multi-particle
sedimentation workload (1024 x 2048 cells, 512 disks of diameter 16 by
default), used for profiling single kernel launches without the timing
harness around them.  Prints the step count, the first disk's centre and the
device status.
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
    a = ap.parse_args(argv)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    pkg = importlib.import_module("2d_nnf_lbm_b200")
    prec = 1 if a.precision == "fp32" else 0
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
