"""The CPU oracle against golden vectors from the reference itself.

tests/golden/*.npz hold the state the reference's own Fortran programs reach
on small lattices (generated by tests/golden/make_golden.py, which executes
the shipped C1, C6 and C3 sources with tests/golden/f90run.py).  The oracle,
a C restatement compiled without floating-point contraction, must reproduce
every stored number exactly: populations, velocity, density, body force,
Bingham omega, particle state, and the per-step mean density the reference
writes to its history file.
"""

import os

import numpy as np
import pytest

from oracle.oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def _setup(cases, name):
    if name == "c1_center":
        return cases.shipped_c1(24, 40, 8.0), cases.pin_array([[12.0, 28.0]], 8.0, 1.25), {}
    if name == "c1_walls":
        return cases.shipped_c1(24, 40, 8.0), cases.pin_array([[19.02, 4.98]], 8.0, 1.25), {}
    if name == "c6_bingham":
        p, pin = cases.shipped_c6(24, 60)
        return p, pin, {"omega_chain": 1}  # C6:958 node-to-node omega chain
    if name == "c3_multi":
        p = cases.shipped_c3(48, 72)
        pin = cases.pin_array([[14.0, 50.0], [30.6, 50.0], [24.0, 22.0]], 16.0,
                              float(np.float32(1.01)))
        # the reference's D_PW local starts at zero in the translated run
        return p, pin, {"stale_dpw_init": 0.0}
    if name == "c1_nonnewt":
        p = cases.shipped_c1(24, 40, 8.0)
        p.rheology = 1        # LBM_BINGHAM (Papanastasiou, C1:950-954)
        p.strain_model = 1    # LBM_STRAIN_FEQ (C1:896-948)
        return p, cases.pin_array([[12.0, 28.0]], 8.0, 1.25), {"omega_chain": 1}
    if name in ("c1_bgk", "c1_bgk_biviscous"):
        # C1's main program calling COLLISION (C1:774-841) in place of
        # Collision_MRT; the bi-viscous run at TAU_Y = 1.0D-5
        p = cases.shipped_c1(24, 40, 8.0)
        p.collision = 1  # LBM_COLLISION_BGK
        if name == "c1_bgk_biviscous":
            p.rheology = 1  # LBM_BINGHAM: COLLISION's bi-viscosity branch
            p.tau_y = 1.0e-5
        return p, cases.pin_array([[12.0, 28.0]], 8.0, 1.25), {}
    if name == "c3_casson":
        p = cases.shipped_c3(48, 72)
        p.rheology = 2  # LBM_CASSON
        p.tau_y = 0.5 * (float(np.float32(1.01)) - 1.0) * (-p.gravity) * 16.0  # C3:48
        p.m_pap = float(np.float32(1.0e6))
        pin = cases.pin_array([[14.0, 50.0], [30.6, 50.0], [24.0, 22.0]], 16.0,
                              float(np.float32(1.01)))
        return p, pin, {"stale_dpw_init": 0.0, "omega_chain": 1}
    if name == "c2_dkt":
        p, disks = cases.shipped_c2(30, 112, 3.0, float(np.float32(-5.0e-4)))
        return p, disks, {"stale_dpw_init": 0.0}
    if name == "c4_oscillate":
        p, disk = cases.shipped_c4(40, 30, 10.0, 10.0, 40.0)
        return p, disk, {}
    raise KeyError(name)


CASES = ["c1_center", "c1_walls", "c1_nonnewt", "c1_bgk", "c1_bgk_biviscous", "c6_bingham",
         "c3_multi", "c3_casson", "c2_dkt", "c4_oscillate"]


def _exact(a, b, what):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    if not np.array_equal(a, b):
        d = np.max(np.abs(a - b))
        raise AssertionError(f"{what}: max |diff| {d:.3e} (scale {np.max(np.abs(b)):.3e})")


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_bit_for_bit(cases, name):
    g = _load(name)
    p, pin, kw = _setup(cases, name)
    p.series_every, p.series_particles, p.series_capacity = 1, len(pin), 64
    o = Oracle(p, **kw)
    try:
        o.set_particles(pin)
        o.step(int(g["steps"]))
        assert o.kk == int(g["kk"])
        n1x, n1y = p.nx + 1, p.ny + 1
        _exact(o.f().reshape(n1y, n1x, 9).transpose(2, 1, 0), g["F"], "F after BC")
        _exact(o.field("ux").T, g["UX"], "UX")
        _exact(o.field("uy").T, g["UY"], "UY")
        _exact(o.field("rho").T, g["RHO"], "RHO")
        _exact(o.field("gx").T, g["G"][0], "G(1)")
        _exact(o.field("gy").T, g["G"][1], "G(2)")
        if "OMEGA_BN" in g and p.rheology in (1, 2):  # Bingham, Casson
            _exact(o.field("omega").T, g["OMEGA_BN"], "OMEGA_BN")
        op = o.particles()
        _exact(op[:, 0:2], g["DISK_CENTER"], "CENTER")
        _exact(op[:, 3:6], g["DISK_VELOCITY"], "VELOCITY")
        _exact(op[:, 6:9], g["DISK_FORCE"], "FORCE")
        if name != "c4_oscillate":  # C4's Wan-Turek F_COL never reaches its outputs
            _exact(op[:, 9:11], g["DISK_F_COL"], "F_COL")
        _exact(op[:, 14], g["DISK_M_P"], "M_P")
        _exact(op[:, 15], g["DISK_I_P"], "I_P")
        if "DISK_ANGLE" in g:
            _exact(op[:, 2], g["DISK_ANGLE"], "ANGLE")
        _exact(op[:, 11:14], g["F_H_IN"].T, "F_H_IN")
        s = o.series()
        _exact(s[:, 0], g["UNIT8"][:, 0], "history step numbers")
        _exact(s[:, 1], g["UNIT8"][:, 1], "mean density per step (unit 8)")
        if name == "c4_oscillate":
            # unit 11 (C4:279): KK/T_C, (FORCE(1)+F_H_IN(1))/F_C, FORCE(1)/F_C
            # after this step's lattice pass: FORCE of step k is the force
            # the record of step k+1 starts with (the last one, the final state)
            fx = np.append(s[1:, 2 + 6], op[0, 6])
            u_c, t_c, l_c = p.osc_u, p.osc_period, 10.0
            f_c = 0.5 * u_c * u_c * l_c
            hist = np.stack([s[:, 0] / t_c, (fx + s[:, 2 + 9]) / f_c, fx / f_c], axis=1)
            _exact(hist, g["UNIT11"], "force history (unit 11)")
    finally:
        o.close()


def test_goldens_cover_the_branches_they_claim():
    """The fixtures exercise what their docstrings say (non-trivial values)."""
    w = _load("c1_walls")
    assert np.all(np.abs(w["DISK_F_COL"][0]) > 0)            # wall repulsion active
    c3 = _load("c3_multi")
    assert np.abs(c3["DISK_F_COL"][0, 0]) > 0                 # pair force on disk 1
    c6 = _load("c6_bingham")
    om = c6["OMEGA_BN"]
    assert om.min() < om.max()                                # Bingham omega varies
    assert np.any(c6["DISK_ANGLE"] != 0) or np.any(c6["DISK_VELOCITY"][:, 2] != 0)
    # the BGK runs took COLLISION, not Collision_MRT, and the bi-viscous one
    # has yielded and unyielded nodes (omega = 1/(3 MU_R + 1/2) when unyielded)
    assert not np.array_equal(_load("c1_bgk")["F"], _load("c1_center")["F"])
    bv = _load("c1_bgk_biviscous")["OMEGA_BN"]
    assert 0 < np.count_nonzero(bv < 0.01) < bv.size


def test_oracle_compute_error_matches_reference(cases):
    """COMPUTEERROR (C1:1592-1612) as the reference evaluates it every 1000
    steps (unit 7 of its run): ER at steps 1000 and 2000, and the state."""
    g = _load("c1_error")
    p = cases.shipped_c1(16, 24, 6.0)
    o = Oracle(p)
    try:
        o.set_particles(cases.pin_array([[8.0, 14.0]], 6.0, 1.25))
        ers = []
        for _ in range(2):
            o.step(1000)
            ers.append([float(o.kk), o.compute_error()])
        _exact(np.array(ers), g["UNIT7"], "ER history")
        _exact(o.field("ux").T, g["UX"], "UX")
        _exact(o.particles()[:, 0:2], g["DISK_CENTER"], "CENTER")
    finally:
        o.close()
