"""Central finite differences of the adjoint test cases on the CPU oracle.

    python tests/golden/make_adjoint_fd.py

For every case of adjoint_cases.py and every gradient entry (tau_y, nu, and
per disk rho_p, x0, y0) the oracle (FP64, the reference's time step) runs the
case with the entry moved by +-delta, delta = 1e-4 * |value| (the relative
step of the adjoint check), and again with delta/2; J is the mean v_y of
disk 0 over the case's window.  The .npz beside this script holds J, both
difference quotients and the entry names; the tests compare lbm_adjoint
against them and check that the two steps agree (the quotients are in
their asymptotic range).
"""

from __future__ import annotations

import importlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import adjoint_cases as ac  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

REL = 1.0e-4


def run_j(p, pin, n0: int, n1: int) -> float:
    o = Oracle(p)
    o.set_particles(pin)
    o.step(n0 - 1)
    v = []
    for _ in range(n0, n1 + 1):
        o.step(1)
        v.append(o.particles()[0, 4])
    o.close()
    return ac.objective(np.array(v))


def fd(p, pin, n0, n1, name, disk, rel):
    delta = rel * abs(ac.base_value(p, pin, name, disk))
    jp = run_j(*ac.perturbed(p, pin, name, disk, +delta), n0, n1)
    jm = run_j(*ac.perturbed(p, pin, name, disk, -delta), n0, n1)
    return (jp - jm) / (2.0 * delta)


def main() -> None:
    cases = importlib.import_module("2d_nnf_lbm_b200").cases
    for name in ac.CASES:
        t0 = time.time()
        p, pin, n0, n1 = ac.build(cases, name)
        j = run_j(p, pin, n0, n1)
        ents = ac.parameters(pin.shape[0])
        g = np.array([fd(p, pin, n0, n1, e, q, REL) for e, q in ents])
        g2 = np.array([fd(p, pin, n0, n1, e, q, 0.5 * REL) for e, q in ents])
        np.savez(os.path.join(HERE, f"adjoint_{name}.npz"), j=j, fd=g, fd_half=g2,
                 names=np.array([f"{e}{'' if q < 0 else q}" for e, q in ents]),
                 n0=n0, n1=n1, rel=REL)
        print(f"{name}: J={j:.6e} {time.time() - t0:.1f}s")
        for (e, q), a, b in zip(ents, g, g2):
            print(f"   {e}{'' if q < 0 else q:<3} {a: .8e} {b: .8e} {abs(a - b) / max(abs(a), 1e-300):.1e}")


if __name__ == "__main__":
    main()
