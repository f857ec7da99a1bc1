"""Small cases of the adjoint tests, shared by make_adjoint_fd.py (which
stores the oracle's central finite differences for them) and the tests.

Each case is (params, disks, n0, n1): J = mean v_y of disk 0 over steps
n0..n1.  The parameters of a gradient are the yield stress tau_y, the
plastic viscosity nu, and per disk rho_p, x0, y0.

  c6_bingham  the C6 program (half-way bounce-back, Papanastasiou, rates
              1.1/1.25/q(omega), offset-wall repulsion) at NX=40 NY=120,
              D=10 rho_p=1.5 at (20, 80), nu=0.05, gravity -1e-5, m=1e5,
              tau_y of yield number 0.05, 400 steps, window 300..400
  c6_wall     as c6_bingham with the disk at (5.8, 80), inside the range of
              the left wall's repulsion
  c1_newton   the C1 program (Zou-He walls, rates 1.1/1.0/1.2/omega, mirror
              walls), NX=40 NY=120, D=10 rho_p=1.5 at (20, 80), gravity
              -1e-5, 400 steps, window 300..400
  c3_pair     the C3 constants (half-way bounce-back, offset walls) with the
              pair-distance contact test, NX=40 NY=120, two disks D=8 at
              (15, 80) rho_p=1.5 and (24.2, 82) rho_p=1.3, within each
              other's repulsion range, 300 steps, window 200..300
"""

from __future__ import annotations

import numpy as np

CASES = ("c6_bingham", "c6_wall", "c1_newton", "c3_pair")


def build(cases, name: str):
    if name in ("c6_bingham", "c6_wall"):
        p, _ = cases.shipped_c6(40, 120)
        p.nu = 0.05
        p.gravity = -1.0e-5
        p.m_pap = 1.0e5
        d, rho_p = 10.0, 1.5
        p.tau_y = 0.05 * (rho_p - 1.0) * 1.0e-5 * d
        p.c_ij = cases.glowinski_cij(rho_p, 1.0, p.gravity, p.pi, d)
        x = 20.0 if name == "c6_bingham" else 5.8
        pin = cases.pin_array([[x, 80.0]], d, rho_p)
        return p, pin, 300, 400
    if name == "c1_newton":
        p = cases.shipped_c1(40, 120, 10.0)
        p.gravity = -1.0e-5
        pin = cases.pin_array([[20.0, 80.0]], 10.0, 1.5)
        return p, pin, 300, 400
    if name == "c3_pair":
        p = cases.shipped_c3(40, 120)
        p.gravity = -1.0e-5
        p.contact_test = 0
        p.series_every = 0
        p.c_ij = cases.glowinski_cij(1.5, 1.0, p.gravity, p.pi, 8.0)
        pin = cases.pin_array([[15.0, 80.0], [24.2, 82.0]], 8.0, np.array([1.5, 1.3]))
        return p, pin, 200, 300
    raise KeyError(name)


def parameters(np_disks: int) -> list[tuple[str, int]]:
    """(name, disk) of every gradient entry, in lbm_adjoint's order."""
    out = [("tau_y", -1), ("nu", -1)]
    for q in range(np_disks):
        out += [("rho_p", q), ("x0", q), ("y0", q)]
    return out


def perturbed(p, pin, name: str, disk: int, delta: float):
    """Copies of (params, disks) with one parameter moved by delta."""
    p2 = p.copy()
    pin2 = np.array(pin, dtype=np.float64, copy=True)
    if name == "tau_y":
        p2.tau_y = p.tau_y + delta
    elif name == "nu":
        p2.nu = p.nu + delta
    elif name == "rho_p":
        pin2[disk, 7] += delta
    elif name == "x0":
        pin2[disk, 0] += delta
    elif name == "y0":
        pin2[disk, 1] += delta
    else:
        raise KeyError(name)
    return p2, pin2


def base_value(p, pin, name: str, disk: int) -> float:
    return {"tau_y": p.tau_y, "nu": p.nu}.get(name) if disk < 0 else \
        float(pin[disk, {"rho_p": 7, "x0": 0, "y0": 1}[name]])


def objective(particles_per_step: np.ndarray) -> float:
    return float(np.mean(particles_per_step))
