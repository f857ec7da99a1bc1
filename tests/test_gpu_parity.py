"""GPU parity: the CUDA library (through the C ABI) against the CPU oracle.

FP64 plain path: the lattice and particle kernels are built without FMA
contraction and follow the reference's operation order, so the remaining
differences come from sin() (CUDA vs glibc, ~1 ulp) and from the order of the
force reductions (tree vs sequential).  Tolerance: relative 1e-10 on particle
state and fields after up to a few hundred steps, each quantity measured
against the magnitude of its physical group (a torque against force x D).
"""

import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

RTOL64 = 1e-10


def close64(a, b, rtol=RTOL64, what="", scale=None):
    """max|a-b| <= rtol*scale; scale defaults to max|b| (the field's magnitude)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if scale is None:
        scale = np.max(np.abs(b)) if b.size else 0.0
    scale = max(scale, 1e-300)
    err = np.max(np.abs(a - b)) if a.size else 0.0
    assert err <= rtol * scale, f"{what}: max abs err {err:.3e} vs scale {scale:.3e}"


def pair(pkg, p, pin, steps, chain=0):
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    ref = Oracle(p, omega_chain=chain)
    ref.set_particles(pin)
    if steps:
        sim.step(steps)
        ref.step(steps)
    return sim, ref


def compare_all(sim, ref, fields=("ux", "uy", "rho", "phi", "gx", "gy"), rtol=RTOL64):
    assert sim.kk == ref.kk
    gp, rp = sim.particles(), ref.particles()
    # compare each group against the magnitude of its own physical scale, so
    # quantities that vanish by symmetry are measured against their siblings
    d = np.asarray([np.max(ref.state_particles()[:, 17])])
    groups = {
        "position": ([0, 1], None),
        "angle": ([2], max(np.max(np.abs(rp[:, 2])),
                          np.max(np.abs(rp[:, 3:5])) * max(ref.kk, 1) / float(d.max()))),
        "velocity": ([3, 4], None),
        "spin": ([5], np.max(np.abs(rp[:, 3:5])) / float(d.max())),
        "force": ([6, 7], None),
        "torque": ([8], np.max(np.abs(rp[:, 6:8])) * float(d.max())),
        "collision": ([9, 10], np.max(np.abs(rp[:, 9:11])) + np.max(np.abs(rp[:, 6:8]))),
        # F_H_IN = (rho0/rho_p) M (v - v_old): velocity noise times the mass
        "internal": ([11, 12], np.max(np.abs(rp[:, 14])) * np.max(np.abs(rp[:, 3:5]))),
        "internal_t": ([13], np.max(np.abs(rp[:, 15])) * np.max(np.abs(rp[:, 3:5])) / float(d.max())),
        "mass": ([14, 15], None),
    }
    for name, (cols, sc) in groups.items():
        if sc is None:
            sc = np.max(np.abs(rp[:, cols])) if rp.size else 0.0
        close64(gp[:, cols], rp[:, cols], rtol, f"particle {name}", scale=max(sc, 1e-300))
    for f in fields:
        close64(sim.field(f), ref.field(f), rtol, f"field {f}")


@pytest.mark.parametrize("steps", [0, 1, 10, 200])
def test_c1_zouhe_fp64(pkg, cases, steps):
    p = cases.shipped_c1(40, 60, 10.0)
    pin = cases.pin_array([[20.0, 40.0]], 10.0, 1.25)
    sim, ref = pair(pkg, p, pin, steps)
    compare_all(sim, ref)
    assert np.array_equal(sim.image(), ref.image())


def test_c1_offcentre_rotation_fp64(pkg, cases):
    # off-centre disk with initial spin: exercises torque, rotation terms and
    # the wall repulsion of the mirror model near the right wall
    p = cases.shipped_c1(50, 70, 10.0)
    p.gravity = -2e-4
    pin = cases.pin_array([[44.5, 50.25]], 10.0, 1.5, uvw=[[0.0, 0.0, 1e-3]])
    sim, ref = pair(pkg, p, pin, 150)
    compare_all(sim, ref)


def test_series_and_mean_density_fp64(pkg, cases):
    p = cases.shipped_c1(40, 60, 10.0)
    p.series_every = 7
    pin = cases.pin_array([[20.0, 40.0]], 10.0, 1.25)
    sim, ref = pair(pkg, p, pin, 70)
    s, r = sim.series(), ref.series()
    assert s.shape == r.shape == (10, 2 + 12)
    assert np.array_equal(s[:, 0], r[:, 0])
    close64(s[:, 1], r[:, 1], 1e-13, "AvgDen")
    close64(s[:, 2:], r[:, 2:], RTOL64, "history")
    assert abs(sim.mean_density() - ref.mean_density()) < 1e-13


@pytest.mark.parametrize("bc", [0, 1])
def test_c6_bingham_fp64(pkg, cases, bc):
    p, disk = cases.shipped_c6(40, 120)
    p.bc = bc
    p.record_stress = 1
    sim, ref = pair(pkg, p, disk, 120)
    # Papanastasiou with m = 5.5e6 amplifies ulp-level differences of sin()
    compare_all(sim, ref, rtol=1e-8)
    close64(sim.field("omega"), ref.field("omega"), 1e-8, "omega")
    for f in ("tau11", "tau22", "tau12"):
        close64(sim.field(f), ref.field(f), 1e-8, f)
    gi, ri = sim.image(), ref.image()
    # yield flags may differ only where |tau| sits on tau_y within rounding
    assert np.mean(gi != ri) < 1e-3


def test_c1_nonnewtonian_strain_feq_fp64(pkg, cases):
    """C1's non-Newtonian branch: Papanastasiou viscosity with the strain
    rate from m - m_eq(COMPUTEFEQNEW) (C1:896-948), per-node omega."""
    p = cases.shipped_c1(40, 60, 10.0)
    p.rheology = 1
    p.strain_model = 1
    p.record_stress = 1
    sim, ref = pair(pkg, p, cases.pin_array([[20.0, 40.0]], 10.0, 1.25), 80)
    compare_all(sim, ref, rtol=1e-8)
    close64(sim.field("omega"), ref.field("omega"), 1e-8, "omega")
    # C1's m = 1e8 (18x C6's) amplifies the ulp-level sin() differences
    # further in the stresses, which scale with the apparent viscosity
    for f in ("tau11", "tau22", "tau12"):
        close64(sim.field(f), ref.field(f), 1e-7, f)


def test_c3_casson_fp64(pkg, cases):
    """The Casson viscosity of C3's non-Newtonian branch (C3:978-996),
    three disks, per-node omega of the previous step."""
    p = cases.shipped_c3(48, 72)
    p.rheology = 2  # LBM_CASSON
    p.tau_y = 0.5 * (float(np.float32(1.01)) - 1.0) * (-p.gravity) * 16.0
    p.m_pap = float(np.float32(1.0e6))
    p.record_stress = 1
    pin = cases.pin_array([[14.0, 50.0], [30.6, 50.0], [24.0, 22.0]], 16.0,
                          float(np.float32(1.01)))
    sim, ref = pair(pkg, p, pin, 60)
    compare_all(sim, ref, rtol=1e-8)
    close64(sim.field("omega"), ref.field("omega"), 1e-8, "omega")
    for f in ("tau11", "tau22", "tau12"):
        close64(sim.field(f), ref.field(f), 1e-8, f)


def bgk_case(cases, bingham):
    """C1 with the BGK COLLISION (C1:774-841) in place of Collision_MRT; with
    bingham its bi-viscosity model at a yield stress whose threshold
    GAMMA_C = tau_y/(999 nu) = 4e-8 lies inside the range of shear rates
    around the disk, so yielded and unyielded nodes both occur (a larger
    yield stress leaves the whole fluid unyielded at 1000 nu)."""
    p = cases.shipped_c1(40, 60, 8.0)
    p.collision = 1  # LBM_COLLISION_BGK
    p.gravity = -2e-5
    if bingham:
        p.rheology = 1  # LBM_BINGHAM: bi-viscosity under BGK
        p.tau_y = 2e-6
    pin = cases.pin_array([[20.0, 38.0]], 8.0, 1.5)
    return p, pin


@pytest.mark.parametrize("bingham", [0, 1])
def test_bgk_collision_fp64(pkg, cases, bingham):
    """BGK 1e-10; the bi-viscosity switch 1e-8 (as the Papanastasiou path:
    ulp-level differences of sin and of the force order grow where the
    viscosity jumps by a factor of 1000), its omega 1e-7 (near GAMMA_C the
    shear rate comes from f - FEQ differences of ~1e-9 between values of
    ~0.1, eight digits below the populations)."""
    p, pin = bgk_case(cases, bingham)
    sim, ref = pair(pkg, p, pin, 150)
    om = ref.field("omega")
    if bingham:
        assert 0 < np.count_nonzero(om < 0.01) < om.size  # both branches occur
    tol = 1e-8 if bingham else RTOL64
    compare_all(sim, ref, rtol=tol)
    if bingham:
        close64(sim.field("omega"), om, 1e-7, "omega")


@pytest.mark.parametrize("bingham", [0, 1])
def test_bgk_collision_fp32(pkg, cases, bingham):
    p, pin = bgk_case(cases, bingham)
    sim = pkg.Simulation(p.copy(precision=1))
    sim.set_particles(pin)
    ref = Oracle(p)
    ref.set_particles(pin)
    sim.step(150)
    ref.step(150)
    g, r = sim.particles(), ref.particles()
    close64(g[:, 0:2], r[:, 0:2], 1e-4, "position")
    close64(g[:, 3:5], r[:, 3:5], 1e-4, "velocity")
    for f in ("ux", "uy"):
        close64(sim.field(f), ref.field(f), 1e-4, f)
    if bingham:
        # a node at the threshold may take the other branch in FP32: at least
        # 99 % of the nodes agree, each within 1e-3 of the largest omega
        a, b = sim.field("omega"), ref.field("omega")
        agree = np.abs(a - b) <= 1e-3 * np.max(np.abs(b))
        assert np.mean(agree) >= 0.99, np.mean(agree)


@pytest.mark.parametrize("contact", [0, 1])
def test_multiparticle_fp64(pkg, cases, contact):
    rng = np.random.default_rng(3)
    p = cases.shipped_c3(96, 128)
    p.contact_test = contact
    p.gravity = -2e-4
    p.series_particles = 12
    xs = []
    while len(xs) < 12:
        c = np.array([8 + rng.random() * 80, 40 + rng.random() * 80])
        if all(np.hypot(*(c - q)) > 12.5 for q in xs):
            xs.append(c)
    pin = cases.pin_array(np.array(xs), 10.0, 1.0 + rng.random(12) * 0.5)
    sim, ref = pair(pkg, p, pin, 300)
    compare_all(sim, ref, rtol=1e-9)


def test_fp32_shifted_vs_fp64_oracle(pkg, cases):
    p = cases.shipped_c1(60, 120, 12.0)
    p.gravity = -3e-4
    pin = cases.pin_array([[30.0, 80.0]], 12.0, 1.5)
    p32 = p.copy(precision=1)
    sim = pkg.Simulation(p32)
    sim.set_particles(pin)
    ref = Oracle(p)
    ref.set_particles(pin)
    sim.step(500)
    ref.step(500)
    g, r = sim.particles(), ref.particles()
    # trajectory: displacement from the start, relative
    dy_g, dy_r = g[0, 1] - 80.0, r[0, 1] - 80.0
    assert abs(dy_g - dy_r) <= 1e-4 * abs(dy_r), (dy_g, dy_r)
    assert abs(g[0, 4] - r[0, 4]) <= 1e-4 * abs(r[0, 4])
    ux, uxr = sim.field("uy"), ref.field("uy")
    assert np.max(np.abs(ux - uxr)) <= 1e-4 * np.max(np.abs(uxr))


def test_checkpoint_roundtrip_fp64(pkg, cases):
    p, disk = cases.shipped_c6(40, 120)
    a = pkg.Simulation(p)
    a.set_particles(disk)
    a.step(60)
    f, om, parts = a.get_state()
    a.step(40)
    b = pkg.Simulation(p)
    b.set_state(60, f, om, parts)
    b.step(40)
    assert np.array_equal(a.particles(), b.particles())
    assert np.array_equal(a.field("ux"), b.field("ux"))
    # the checkpointed F is the reference's post-BC F of step 60
    ref = Oracle(p)
    ref.set_particles(disk)
    ref.step(60)
    close64(f, ref.f(), RTOL64, "F after BC")


def test_tau_check_rejects(pkg):
    p = pkg.LbmParams(nu=-0.1)
    with pytest.raises(pkg.LbmError) as e:
        pkg.Simulation(p)
    assert e.value.code == -2


# ---- the CUDA path against the reference's own outputs ----------------------
# tests/golden holds states the reference Fortran reaches (see
# tests/golden/make_golden.py).  The single-disk C1 fixtures are compared
# directly; C6 (node-to-node omega chain) and C3 (first-step stale wall
# distance) reach the GPU through the oracle, which matches them exactly.

def _golden(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.npz")
    return dict(np.load(path))


@pytest.mark.parametrize("name,centre", [("c1_center", (12.0, 28.0)), ("c1_walls", (19.02, 4.98))])
@pytest.mark.parametrize("precision,rtol", [(0, RTOL64), (1, 1e-4)])
def test_c1_matches_reference_golden(pkg, cases, name, centre, precision, rtol):
    g = _golden(name)
    p = cases.shipped_c1(24, 40, 8.0)
    p.precision = precision
    sim = pkg.Simulation(p)
    try:
        sim.set_particles(cases.pin_array([list(centre)], 8.0, 1.25))
        sim.step(int(g["steps"]))
        assert sim.kk == int(g["kk"])
        for f, ref in (("ux", g["UX"]), ("uy", g["UY"]), ("rho", g["RHO"]),
                       ("gx", g["G"][0]), ("gy", g["G"][1])):
            close64(sim.field(f).T, ref, rtol, f"field {f}")
        f, _, parts = sim.get_state()
        n1x, n1y = p.nx + 1, p.ny + 1
        close64(f.reshape(n1y, n1x, 9).transpose(2, 1, 0), g["F"], rtol, "F after BC")
        gp = sim.particles()
        close64(gp[:, 0:2], g["DISK_CENTER"], rtol, "centre")
        close64(gp[:, 3:5], g["DISK_VELOCITY"][:, 0:2], rtol, "velocity")
        close64(gp[:, 6:8], g["DISK_FORCE"][:, 0:2], rtol, "force")
        fc = g["DISK_F_COL"]
        close64(gp[:, 9:11], fc, rtol, "wall repulsion", scale=max(np.max(np.abs(fc)), 1e-300))
    finally:
        sim.close()


@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 2e-4)])
def test_compute_error_matches_oracle(pkg, cases, precision, rtol):
    """lbm_compute_error against the oracle's COMPUTEERROR, two calls in a
    row (the second measures the change since the first)."""
    p = cases.shipped_c1(48, 72, 12.0)
    p.precision = precision
    pin = cases.pin_array([[24.0, 50.0]], 12.0, 1.25)
    sim, ref = pair(pkg, p, pin, 30)
    try:
        assert sim.compute_error() == pytest.approx(ref.compute_error(), rel=rtol)
        sim.step(25)
        ref.step(25)
        assert sim.compute_error() == pytest.approx(ref.compute_error(), rel=rtol)
    finally:
        sim.close()
        ref.close()


@pytest.mark.parametrize("nx,precision", [(64, 0), (128, 0), (128, 1)])
def test_wall_column_pass(pkg, cases, nx, precision):
    """NX a multiple of the tile width: the wall column NX is taken by the last
    warp of each tile row; a disk whose PHI ring reaches that column."""
    p = cases.shipped_c1(nx, 48, 10.0)
    p.gravity = -2e-4
    p.wall_model = 2  # no wall repulsion: the disk stays on the wall column
    pin = cases.pin_array([[nx - 5.2, 30.0]], 10.0, 1.5)
    ref = Oracle(p)
    ref.set_particles(pin)
    sim = pkg.Simulation(p.copy(precision=precision))
    sim.set_particles(pin)
    sim.step(80)
    ref.step(80)
    assert ref.field("phi")[20:40, nx].max() > 0.0
    if precision == 0:
        compare_all(sim, ref)
        return
    g, r = sim.particles(), ref.particles()
    for col in (0, 1, 3, 4):  # position (lu), velocity (against |u|)
        scale = np.max(np.abs(r[:, [3, 4]])) if col in (3, 4) else 1.0
        assert abs(g[0, col] - r[0, col]) <= 1e-4 * scale, (col, g[0, col], r[0, col])
    for f in ("ux", "uy", "rho"):
        a, b = sim.field(f), ref.field(f)
        sc = np.max(np.abs(b - (1.0 if f == "rho" else 0.0)))
        assert np.max(np.abs(a - b)) <= 1e-4 * max(sc, 1e-12), f


# ---- case 4: prescribed oscillation, equilibrium boundary, 1.6/1.8 rates ---
def _c4(cases):
    return cases.shipped_c4(40, 30, 10.0, 10.0, 40.0)


@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 2e-4)])
def test_c4_oscillating_cylinder_matches_reference_golden(pkg, cases, precision, rtol):
    """The C4 fixture (the reference's own run, 240 steps): fields, the
    populations after the equilibrium boundary, the disk, and the force
    history the program writes to unit 11."""
    g = _golden("c4_oscillate")
    p, disk = _c4(cases)
    p.precision = precision
    p.series_every, p.series_particles, p.series_capacity = 1, 1, 512
    sim = pkg.Simulation(p)
    try:
        sim.set_particles(disk)
        sim.step(int(g["steps"]))
        for f, ref in (("ux", g["UX"]), ("uy", g["UY"]), ("gx", g["G"][0]), ("gy", g["G"][1])):
            close64(sim.field(f).T, ref, rtol, f"field {f}")
        close64(sim.field("rho").T - 1.0, g["RHO"] - 1.0, rtol, "density deviation")
        f, _, _ = sim.get_state()
        n1x, n1y = p.nx + 1, p.ny + 1
        close64(f.reshape(n1y, n1x, 9).transpose(2, 1, 0), g["F"], rtol, "F after BC")
        gp = sim.particles()
        close64(gp[:, 0:2], g["DISK_CENTER"], 1e-12, "centre")
        close64(gp[:, 3:6], g["DISK_VELOCITY"], 1e-12, "prescribed velocity")
        close64(gp[:, 6:8], g["DISK_FORCE"][:, 0:2], rtol, "force")
        s = sim.series()
        fx = np.append(s[1:, 2 + 6], gp[0, 6])
        f_c = 0.5 * p.osc_u * p.osc_u * 10.0
        hist = np.stack([s[:, 0] / p.osc_period, (fx + s[:, 2 + 9]) / f_c, fx / f_c], axis=1)
        close64(hist, g["UNIT11"], rtol, "force history (unit 11)")
    finally:
        sim.close()


def test_c4_checkpoint_roundtrip(pkg, cases):
    """Restart under the equilibrium boundary: the neighbour values that the
    boundary of the next step needs are rebuilt from the checkpoint."""
    p, disk = _c4(cases)
    a = pkg.Simulation(p)
    a.set_particles(disk)
    a.step(70)
    f, om, parts = a.get_state()
    a.step(30)
    b = pkg.Simulation(p)
    b.set_state(70, f, om, parts)
    b.step(30)
    assert np.array_equal(a.particles(), b.particles())
    assert np.array_equal(a.field("ux"), b.field("ux"))
    assert np.array_equal(a.field("rho"), b.field("rho"))


@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 2e-4)])
def test_c2_two_disks_match_reference_golden(pkg, cases, precision, rtol):
    """Case 2 (DKT, two disks) on the existing kernels against the
    reference's own run: fields, populations, both disks."""
    g = _golden("c2_dkt")
    p, disks = cases.shipped_c2(30, 112, 3.0, float(np.float32(-5.0e-4)))
    p.precision = precision
    sim = pkg.Simulation(p)
    try:
        sim.set_particles(disks)
        sim.step(int(g["steps"]))
        for f, ref in (("ux", g["UX"]), ("uy", g["UY"]), ("gx", g["G"][0]), ("gy", g["G"][1])):
            close64(sim.field(f).T, ref, rtol, f"field {f}")
        f, _, _ = sim.get_state()
        n1x, n1y = p.nx + 1, p.ny + 1
        close64(f.reshape(n1y, n1x, 9).transpose(2, 1, 0), g["F"], rtol, "F after BC")
        gp = sim.particles()
        close64(gp[:, 0:2], g["DISK_CENTER"], rtol, "centre (lu)", scale=1.0)
        close64(gp[:, 3:6], g["DISK_VELOCITY"], rtol, "velocity")
        close64(gp[:, 6:9], g["DISK_FORCE"], rtol, "force")
        close64(gp[:, 2], g["DISK_ANGLE"], rtol, "angle")
    finally:
        sim.close()


def test_full_size_fp32_trajectory_within_1e4(pkg, cases):
    """The throughput workload at its full size (1024 x 2048 cells, 512 disks,
    tau 0.7): FP32-shifted against FP64 plain after 2000 steps, every disk's
    displacement and velocity within 1e-4 of the largest FP64 value.  The
    oracle cannot run this size in seconds; FP64 is pinned to it above."""
    res, pin = {}, None
    for prec in (1, 0):
        p, pin = cases.workload_cfg2(prec, 1024, 2048, 512)
        sim = pkg.Simulation(p)
        sim.set_particles(pin)
        sim.step(2000)
        res[prec] = sim.particles()
        sim.close()
    d32, d64 = res[1][:, 0:2] - pin[:, 0:2], res[0][:, 0:2] - pin[:, 0:2]
    assert np.max(np.linalg.norm(d64, axis=1)) > 1.0  # the disks have moved
    err = np.max(np.linalg.norm(d32 - d64, axis=1))
    assert err <= 1e-4 * np.max(np.linalg.norm(d64, axis=1)), err
    v32, v64 = res[1][:, 3:5], res[0][:, 3:5]
    verr = np.max(np.linalg.norm(v32 - v64, axis=1))
    assert verr <= 1e-4 * np.max(np.linalg.norm(v64, axis=1)), verr


@pytest.mark.parametrize("precision", [1, 0])
def test_full_size_checkpoint_roundtrip(pkg, cases, precision):
    """Restart at the full workload size: a run resumed from a state dump
    matches the uninterrupted run, bit for bit in FP64.  The FP32 dump holds
    f = h + w_k rho0 in double, so an h below 2^-54 in magnitude can lose
    bits on the way back; there the check is 1e-6 of each quantity's scale."""
    p, pin = cases.workload_cfg2(precision, 1024, 2048, 512)
    a = pkg.Simulation(p)
    a.set_particles(pin)
    a.step(200)
    f, om, parts = a.get_state()
    a.step(100)
    b = pkg.Simulation(p)
    b.set_state(200, f, om, parts)
    b.step(100)
    if precision == 0:
        assert np.array_equal(a.particles(), b.particles())
        for name in ("ux", "uy", "rho"):
            assert np.array_equal(a.field(name), b.field(name)), name
    else:
        pa, pb = a.particles(), b.particles()
        close64(pb[:, 0:2], pa[:, 0:2], 1e-6, "position")
        close64(pb[:, 3:5], pa[:, 3:5], 1e-6, "velocity")
        for name in ("ux", "uy", "rho"):
            close64(b.field(name), a.field(name), 1e-6, name)
    a.close()
    b.close()
