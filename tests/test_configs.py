"""The benchmark configurations at their full sizes and run lengths.

Plain method (one disk, 200 x 600, 20,000 steps, history every 10 steps):
the GPU against the oracle's own run of the same inputs
(tests/golden/cfg1_plain.npz, made by tests/golden/make_cfg1.py): the
disk's history (y and v_y, the columns C1:264 writes, and x, u, omega)
every 10 steps, and the corrected velocity and solid fraction at step
20,000.  FP64 within 1e-10 of each quantity's scale over the whole run.
FP32 shifted: the trajectory within 1e-4 over the whole run and the
velocity within 1e-4 during the fall; once the disk rests on the bottom
wall (from about step 8840) the stiff contact model (eps_p = 1e5, C1:702)
turns FP32 differences of the forces into velocity differences of up to
about 1.1e-3 of the peak speed, bounded here at 2e-3.  The frozen gravity
gives a peak particle Reynolds number RHO_P*DIAM*|V|/NU (C1:261) of 20.

Viscoplastic settling (800 x 2400, one Bingham disk D=40): FP32 shifted
against FP64 at full size, the disk history and the yielded/unyielded flag
of every fluid node (C6:947-954).

Multi-particle sedimentation (1024 x 2048, 512 disks): FP32 against FP64
over the configuration's 50,000 steps.  The suspension is chaotic: the
FP32 rounding grows by about e per 12,000 steps, and the worst disk's
displacement error reaches 1.0e-4 of the largest displacement at step
50,000 (RMS over the disks 1.3e-5).
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cfg1_run(pkg, cases, precision, fx):
    p, pin = cases.workload_cfg1(precision)
    assert p.gravity == float(fx["gravity"])
    p.series_capacity = int(fx["steps"]) // 10 + 8
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    sim.step(int(fx["steps"]))
    s = sim.series()
    out = {
        "history": s[:, [0, 2 + 0, 2 + 1, 2 + 3, 2 + 4, 2 + 5]],
        "ux": sim.field("ux"), "uy": sim.field("uy"), "phi": sim.field("phi"),
        "status": sim.status(), "pin": pin, "p": p,
    }
    sim.close()
    return out


def _cfg1_compare(got, fx, rtol, rtol_contact):
    """History and final fields against the fixture.  Velocities are held to
    rtol while the disk falls (its centre more than a diameter above the
    bottom node row) and to rtol_contact once it rests on the wall."""
    h, w = got["history"], fx["history"]
    assert h.shape == w.shape
    assert np.array_equal(h[:, 0], w[:, 0])
    y0, d = got["pin"][0, 1], got["pin"][0, 6]
    vmax = float(np.max(np.abs(w[:, 3:5])))
    fall = float(np.max(np.abs(w[:, 2] - y0)))
    falling = w[:, 2] > 0.5 * d + d
    assert falling[: len(falling) // 3].all()
    for name, col, scale in (("x", 1, fall), ("y", 2, fall)):  # x: lateral drift
        e = np.max(np.abs(h[:, col] - w[:, col]))
        assert e <= rtol * scale, f"history {name}: {e:.3e} vs scale {scale:.3e}"
    for name, col, scale in (("u", 3, vmax), ("v", 4, vmax), ("omega", 5, vmax / d)):
        e = np.abs(h[:, col] - w[:, col])
        assert e[falling].max() <= rtol * scale, f"falling {name}: {e[falling].max():.3e}"
        assert e.max() <= rtol_contact * scale, f"resting {name}: {e.max():.3e}"
    i0, j0 = (int(v) for v in fx["window_origin"])
    n = fx["ux_win"].shape[0]
    win = (slice(j0, j0 + n), slice(i0, i0 + n))
    st = int(fx["stride"])
    for name in ("ux", "uy", "phi"):
        scale = vmax if name != "phi" else 1.0
        e1 = np.max(np.abs(got[name][win] - fx[name + "_win"]))
        e2 = np.max(np.abs(got[name][::st, ::st] - fx[name + "_coarse"]))
        assert max(e1, e2) <= rtol * scale, f"{name}: {max(e1, e2):.3e} vs {scale:.3e}"


@pytest.fixture(scope="module")
def cfg1_fixture():
    path = os.path.join(GOLDEN, "cfg1_plain.npz")
    if not os.path.exists(path):
        pytest.fail("missing tests/golden/cfg1_plain.npz (tests/golden/make_cfg1.py makes it)")
    return np.load(path)


@pytest.mark.parametrize("precision,rtol,rtol_contact", [(0, 1e-10, 1e-10), (1, 1e-4, 2e-3)])
def test_cfg1_plain_matches_oracle_over_20000_steps(pkg, cases, cfg1_fixture, precision, rtol,
                                                    rtol_contact):
    got = _cfg1_run(pkg, cases, precision, cfg1_fixture)
    assert got["status"] == 0
    _cfg1_compare(got, cfg1_fixture, rtol, rtol_contact)
    # peak particle Reynolds number of the fall (C1:261) about 20
    p, pin = got["p"], got["pin"]
    re = pin[0, 7] * pin[0, 6] * np.hypot(got["history"][:, 3], got["history"][:, 4]) / p.nu
    assert 19.0 <= re.max() <= 21.0, re.max()


def _visco(pkg, cases, precision, bn, steps):
    p, pin, info = cases.workload_cfg3(precision, bn)
    p.record_stress = 1
    p.series_every = 10
    p.series_particles = 1
    p.series_capacity = steps // 10 + 8
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    sim.step(steps)
    s = sim.series()
    img = sim.image()
    st = sim.status()
    sim.close()
    return s, img, st, pin


@pytest.mark.parametrize("bn,vtol", [(0.5, 1e-4), (50.0, 3e-4)])
def test_cfg3_viscoplastic_fp32_matches_fp64_full_size(pkg, cases, bn, vtol):
    """800 x 2400 Bingham settling, 20,000 steps: FP32 shifted populations
    against FP64, the disk's position within 1e-4 of its total displacement,
    its velocity within vtol of the largest FP64 speed, and the yield flag
    the same on at least 99.9 % of the fluid nodes.  At Bn = 50 the disk is
    held by the yield stress and creeps at about 5e-4 of U_ref (1.2e-6
    lattice units per step); its FP32 velocity error, about 2.7e-10 there,
    is 1.0e-4 to 1.1e-4 of that creep speed, so the bound is 3e-4."""
    steps = 20000
    s64, img64, st64, pin = _visco(pkg, cases, 0, bn, steps)
    s32, img32, st32, _ = _visco(pkg, cases, 1, bn, steps)
    assert st64 == 0 and st32 == 0
    dy = float(np.max(np.abs(s64[:, 3] - pin[0, 1])))
    vmax = float(np.max(np.abs(s64[:, 6])))
    assert np.max(np.abs(s32[:, 3] - s64[:, 3])) <= 1e-4 * dy
    assert np.max(np.abs(s32[:, 6] - s64[:, 6])) <= vtol * vmax
    fluid = (img64 != 10) & (img32 != 10)
    agree = np.mean((img64 == 5)[fluid] == (img32 == 5)[fluid])
    assert agree >= 0.999, agree


def test_cfg2_fp32_trajectory_over_50000_steps(pkg, cases):
    """512 disks, 1024 x 2048, the configuration's 50,000 steps, FP32 against
    FP64, errors relative to the largest FP64 displacement (speed):
    through 40,000 steps every disk's displacement within 1e-4; at 50,000
    the RMS over the disks within 1e-4 and the worst disk within 2e-4 (the
    chaotic growth of the rounding differences puts it at 1.0e-4 there)."""
    sims = {}
    pin = None
    for prec in (1, 0):
        p, pin = cases.workload_cfg2(prec)
        p.series_every = 0
        sims[prec] = pkg.Simulation(p)
        sims[prec].set_particles(pin)
    done = 0
    for mark in (40000, 50000):
        for s in sims.values():
            s.step(mark - done)
        done = mark
        r32, r64 = sims[1].particles(), sims[0].particles()
        d32, d64 = r32[:, 0:2] - pin[:, 0:2], r64[:, 0:2] - pin[:, 0:2]
        dmax = float(np.max(np.linalg.norm(d64, axis=1)))
        e = np.linalg.norm(d32 - d64, axis=1) / dmax
        vmax = float(np.max(np.linalg.norm(r64[:, 3:5], axis=1)))
        ev = np.linalg.norm(r32[:, 3:5] - r64[:, 3:5], axis=1) / vmax
        if mark == 40000:
            assert e.max() <= 1e-4, e.max()
        else:
            assert np.sqrt(np.mean(e ** 2)) <= 1e-4 and e.max() <= 2e-4, e.max()
            assert np.sqrt(np.mean(ev ** 2)) <= 1e-4 and ev.max() <= 1e-3, ev.max()
    for s in sims.values():
        assert s.status() == 0
        s.close()
