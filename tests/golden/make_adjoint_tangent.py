"""Forward-mode derivatives of the adjoint tests' objective, from the oracle.

For every case of adjoint_cases.py and every gradient entry (tau_y, nu and
per disk rho_p, x0, y0), the tangent build of the oracle
(oracle/liblbm_oracle_tangent.so: the oracle's own source with every real a
value and its derivative) runs the case with that input seeded and returns
J = mean v_y of disk 0 over steps n0..n1 together with dJ/d(input).  These
are the exact derivatives of the oracle's discrete time step, which follows
the reference's Fortran operation by operation: an FP64 reference for the
adjoint that shares no code with the CUDA adjoint kernels and has no
finite-difference truncation error.  The omega rule is the GPU's
(omega_chain=0), as for the finite differences.

    python tests/golden/make_adjoint_tangent.py         # writes adjoint_tangent_<case>.npz
    python tests/golden/make_adjoint_tangent.py --full  # adjoint_tangent_full.npz

--full: the adjoint workload itself (400 x 1200, one Bingham disk D=24,
Bn=5, 4000 steps, J = mean v_y over steps 3000..4000), one process per
gradient entry (about 14 minutes on 8 cores).
"""

from __future__ import annotations

import argparse
import importlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import adjoint_cases as ac  # noqa: E402


def tangent_j(p, pin, n0: int, n1: int, which: str, disk: int) -> tuple[float, float]:
    """J and dJ/d(which of disk) from one tangent run."""
    from oracle.oracle import TangentOracle

    t = TangentOracle(p, which, disk)
    t.set_particles(pin)
    t.step(n0 - 1)
    v, dv = [], []
    for _ in range(n0, n1 + 1):
        t.step(1)
        v.append(t.particles()[0, 4])
        dv.append(t.particles_tangent()[0, 4])
    t.close()
    return ac.objective(np.array(v)), ac.objective(np.array(dv))


def gradient(p, pin, n0: int, n1: int) -> tuple[float, np.ndarray]:
    ents = ac.parameters(pin.shape[0])
    out = [tangent_j(p, pin, n0, n1, e, q) for e, q in ents]
    return out[0][0], np.array([g for _, g in out])


def _full_entry(args):
    which, disk = args
    cases = importlib.import_module("2d_nnf_lbm_b200").cases
    p, pin, info = cases.workload_cfg5(0)
    return tangent_j(p, pin, info["n0"], info["n1"], which, disk)


def full() -> None:
    ents = ac.parameters(1)
    t0 = time.time()
    with mp.get_context("spawn").Pool(len(ents)) as pool:
        out = pool.map(_full_entry, ents)
    j, g = out[0][0], np.array([v for _, v in out])
    np.savez(os.path.join(HERE, "adjoint_tangent_full.npz"), j=j, grad=g,
             names=np.array([f"{e}{'' if q < 0 else q}" for e, q in ents]))
    print(f"full: J={j:.10e} {time.time() - t0:.0f}s")
    for (e, q), v in zip(ents, g):
        print(f"   {e}{'' if q < 0 else q:<3} {v: .12e}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true")
    if ap.parse_args().full:
        full()
        return
    cases = importlib.import_module("2d_nnf_lbm_b200").cases
    for name in ac.CASES:
        t0 = time.time()
        p, pin, n0, n1 = ac.build(cases, name)
        j, g = gradient(p, pin, n0, n1)
        ents = ac.parameters(pin.shape[0])
        np.savez(os.path.join(HERE, f"adjoint_tangent_{name}.npz"), j=j, grad=g,
                 names=np.array([f"{e}{'' if q < 0 else q}" for e, q in ents]), n0=n0, n1=n1)
        print(f"{name}: J={j:.10e} {time.time() - t0:.1f}s")
        for (e, q), v in zip(ents, g):
            print(f"   {e}{'' if q < 0 else q:<3} {v: .12e}")


if __name__ == "__main__":
    main()
