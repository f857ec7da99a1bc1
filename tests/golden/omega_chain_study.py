"""How far the GPU's per-node omega departs from the reference's omega chain.

In the Bingham collision of 6_FreeFall_YieldStress (C6:867-962) every node
is relaxed with OMEGA_MRT, a single variable that the previous node of the
j-outer / i-inner sweep has just overwritten with its own viscosity
(C6:890 reads it, C6:958 writes it): a serial chain along the sweep.  The
GPU relaxes each node with its own omega of the previous step instead, so
nodes can be updated in any order.  The oracle has both (omega_chain=1 is
the reference's chain, 0 the GPU's rule); this script runs both on the C6
program at reduced size for several yield numbers and reports the
difference in the disk's settling and in the yielded/unyielded field
(C6:947-954):

    python tests/golden/omega_chain_study.py [--nx 80 --ny 300 --steps 12000]

Printed per yield number Y = TAU_Y / ((RHO_S - RHO_F) |A_G| L_C) (C6:30):
the terminal v_y (mean over the last tenth of the run) of both rules, their
relative difference, the largest difference of the disk's y over the run
relative to its total fall, and the fraction of fluid nodes whose
yield flag differs at the end.
"""

from __future__ import annotations

import argparse
import importlib
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def case(nx, ny, y):
    pkg = importlib.import_module("2d_nnf_lbm_b200")
    p, disk = pkg.cases.shipped_c6(nx, ny)
    l_c = float(nx // 4)
    p.tau_y = y * (2.0 - 1.0) * (-p.gravity) * l_c
    p.series_every = 10
    p.series_particles = 1
    p.series_capacity = 1 << 16
    p.record_stress = 1
    return p, disk


def run(args):
    nx, ny, y, steps, chain = args
    from oracle.oracle import Oracle

    p, disk = case(nx, ny, y)
    o = Oracle(p, omega_chain=chain)
    o.set_particles(disk)
    o.step(steps)
    s = o.series()
    img = o.image()
    o.close()
    return s[:, 2 + 1], s[:, 2 + 4], img


def compare(y_hist, v_hist, img, y0):
    """Metrics of rule 0 (GPU) against rule 1 (reference chain)."""
    n = len(v_hist[1])
    tail = slice(n - max(1, n // 10), n)
    v1, v0 = float(np.mean(v_hist[1][tail])), float(np.mean(v_hist[0][tail]))
    fall = float(np.max(np.abs(y_hist[1] - y0)))
    fluid = (img[0] != 10) & (img[1] != 10)
    return {
        "vy_chain": v1, "vy_own": v0,
        "vy_rel_diff": abs(v0 - v1) / max(abs(v1), 1e-300),
        "y_diff_over_fall": float(np.max(np.abs(y_hist[0] - y_hist[1]))) / max(fall, 1e-300),
        "fall": fall,
        "flag_diff_frac": float(np.mean((img[0] == 5)[fluid] != (img[1] == 5)[fluid])),
        "unyielded_frac": float(np.mean((img[1] == 5)[fluid])),
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=80)
    ap.add_argument("--ny", type=int, default=300)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--yields", default="0.033,0.066,0.2,0.5")
    a = ap.parse_args(argv)
    ys = [float(v) for v in a.yields.split(",")]
    jobs = [(a.nx, a.ny, y, a.steps, chain) for y in ys for chain in (1, 0)]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(run, jobs)
    for k, y in enumerate(ys):
        r1, r0 = res[2 * k], res[2 * k + 1]
        _, disk = case(a.nx, a.ny, y)
        m = compare({1: r1[0], 0: r0[0]}, {1: r1[1], 0: r0[1]}, {1: r1[2], 0: r0[2]}, disk[0, 1])
        print(f"Y={y:g} nx={a.nx} ny={a.ny} steps={a.steps}: " +
              ", ".join(f"{key} {val:.4g}" for key, val in m.items()), flush=True)


if __name__ == "__main__":
    main()
