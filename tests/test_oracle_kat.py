"""Known-answer tests of the CPU oracle, derived from the mathematics of the
reference routines (no GPU)."""

import numpy as np
import pytest

from oracle.oracle import Oracle


def test_rest_state_halfway_bb_conserves_mass_exactly(cases):
    # closed box, fluid at rest, no particles: streaming and half-way
    # bounce-back conserve mass; each collision multiplies a node's mass by
    # 36*d_mrt (C1:913-921 with d_mrt = 1./36. in REAL(4))
    p = cases.shipped_c3(20, 30)
    o = Oracle(p)
    o.set_particles(np.zeros((0, 8)))
    # INITIALIZE holds RHO = rho0, but its populations sum to
    # rho0*(2*W0 + 8*W1 + 4*W2) with the REAL(4) weights (C1:1162-1164)
    w = p.w_init
    m0 = p.rho0 * (2.0 * w[0] + 8.0 * w[1] + 4.0 * w[2])
    assert o.mean_density() == p.rho0
    o.step(25)
    assert np.all(o.field("ux") == 0.0) and np.all(o.field("uy") == 0.0)
    expect = m0 * (36.0 * p.d_mrt) ** 25
    assert o.mean_density() == pytest.approx(expect, rel=1e-14)
    rho = o.field("rho")
    assert np.ptp(rho) < 1e-14


def test_rest_state_zouhe_stays_at_rest(cases):
    p = cases.shipped_c1(20, 30, 10.0)
    o = Oracle(p)
    o.set_particles(np.zeros((0, 8)))
    o.step(10)
    assert np.max(np.abs(o.field("ux"))) == 0.0
    assert np.max(np.abs(o.field("uy"))) == 0.0


def test_phi_profile_knowns(cases):
    # PHI = 1/2 at distance R, 0 at R + zeta/2 (inclusive), 1 at R - zeta/2 (C1:467-475)
    p = cases.shipped_c1(40, 60, 10.0)
    p.zeta = 2.0
    o = Oracle(p)
    o.set_particles(cases.pin_array([[20.0, 30.0]], 10.0, 1.25))
    phi = o.field("phi")
    assert phi[30, 25] == 0.5 and phi[30, 15] == 0.5
    assert phi[30, 26] == 0.0 and phi[30, 24] == 1.0
    assert phi[30, 20] == 1.0 and phi[30, 30] == 0.0
    # smooth and monotone through the interface along a ray
    r = np.array([phi[30, 20 + k] for k in range(0, 8)])
    assert np.all(np.diff(r) <= 0)
    img = o.image()
    assert img[30, 25] == 10 and img[30, 26] == 0


def test_first_step_particle_update_exact(cases):
    # step 1: FORCE = 0, VP_OLD = 0, V = 0 -> V = (1 - rho0/rho_p) A_G,
    # y += V/2 (C1:250-258), exactly
    p = cases.shipped_c1(40, 60, 10.0)
    o = Oracle(p)
    o.set_particles(cases.pin_array([[20.0, 40.0]], 10.0, 1.25))
    o.step(1)
    s = o.particles()[0]
    v = (1.0 - 1.0 / 1.25) * p.gravity
    assert s[4] == v
    assert s[1] == 40.0 + 0.5 * (v + 0.0)
    assert s[11] == 0.0 and s[12] == 0.0


def _pair(cases, dist, contact, stale=float("inf")):
    p = cases.shipped_c3(80, 80)
    p.gravity = 0.0
    p.rep_zeta = 2.0
    p.contact_test = contact
    p.wall_model = 2
    o = Oracle(p, stale_dpw_init=stale)
    o.set_particles(cases.pin_array([[30.0, 40.0], [30.0 + dist, 40.0]], 16.0, 1.2))
    o.step(1)
    return o.particles()[:, 9:11]


def test_glowinski_pair_force_continuity_and_symmetry(cases):
    # zero at and beyond the cut-off D + zeta, quadratic inside (C3:758-766)
    f_out = _pair(cases, 18.0, 0)
    assert np.all(f_out == 0.0)
    f1 = _pair(cases, 17.9, 0)
    f2 = _pair(cases, 17.8, 0)
    assert f1[0, 0] < 0 < f1[1, 0]  # pushes apart (c_ij > 0 for g < 0 ... sign check below)
    assert np.allclose(f1[0], -f1[1])
    ratio = f2[0, 0] / f1[0, 0]
    assert ratio == pytest.approx(4.0, rel=1e-6)


def test_contact_branch_stale_vs_dpp(cases):
    # overlapping pair: the D_PP test adds the E-term, the stale D_PW = inf
    # of a first call does not (C3:760-763)
    fd = _pair(cases, 15.0, 0)
    fs = _pair(cases, 15.0, 1, stale=float("inf"))
    assert abs(fd[0, 0]) > abs(fs[0, 0]) > 0


def test_bingham_sequential_chain_differs_from_per_node(cases):
    p, disk = cases.shipped_c6(40, 120)
    a = Oracle(p, omega_chain=0)
    b = Oracle(p, omega_chain=1)
    for o in (a, b):
        o.set_particles(disk)
        o.step(30)
    wa, wb = a.field("omega"), b.field("omega")
    assert not np.array_equal(wa, wb)
    assert np.max(np.abs(wa - wb)) < 0.5
    va, vb = a.particles()[0, 4], b.particles()[0, 4]
    assert va == pytest.approx(vb, rel=0.2)


def test_papanastasiou_limits(cases):
    # unyielded (tiny shear) nodes carry omega ~ 1/(3(nu + m tau_y)/rho + 0.5),
    # strongly sheared nodes approach the plastic omega (C6:939-957)
    p, disk = cases.shipped_c6(40, 120)
    o = Oracle(p)
    o.set_particles(disk)
    o.step(50)
    w = o.field("omega")
    w_plastic = 1.0 / (3.0 * p.nu + 0.5)
    w_floor = 1.0 / (3.0 * (p.nu + p.m_pap * p.tau_y) / 1.0 + 0.5)
    assert np.min(w) >= 0.5 * w_floor
    assert np.max(w) <= w_plastic * (1 + 1e-6)
    img = o.image()
    assert set(np.unique(img)) <= {0, 5, 10}
    assert np.any(img == 5) and np.any(img == 10)


def test_next_post_collision_matches_next_step(cases):
    # the state the CUDA path stores (post-collision of the next step) is what
    # the next step streams from
    p = cases.shipped_c1(30, 40, 8.0)
    o = Oracle(p)
    o.set_particles(cases.pin_array([[15.0, 25.0]], 8.0, 1.5))
    o.step(5)
    fnext, _ = o.next_post_collision()
    f_now = o.f()
    assert not np.array_equal(fnext, f_now)
    # mass of the post-collision state = 36*d_mrt * mass of F (C1:911-921)
    assert fnext.sum() == pytest.approx(f_now.sum() * 36.0 * p.d_mrt, rel=1e-14)


def test_bgk_biviscosity_first_step(cases):
    """COLLISION's bi-viscosity model (C1:789-809) on INITIALIZE's state: f
    equals FEQ everywhere, so the shear rate is zero, every node is
    unyielded, and OMEGA_BN = 1/(3 MU_R + 0.5) with MU_R = 1000 NU."""
    from oracle.oracle import Oracle

    p = cases.shipped_c1(12, 16, 4.0)
    p.collision, p.rheology, p.tau_y = 1, 1, 1e-6
    o = Oracle(p)
    o.set_particles(cases.pin_array([[6.0, 9.0]], 4.0, 1.5))
    o.step(1)
    om = o.field("omega")
    assert np.all(om == 1.0 / (3.0 * (1000.0 * p.nu) + 0.5))
    o.close()
