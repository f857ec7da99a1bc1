"""The benchmark configurations at their full sizes and run lengths.

Plain method (one disk, 200 x 600, 20,000 steps, history every 10 steps):
the GPU against the oracle's own run of the same inputs
(tests/golden/cfg1_plain.npz, made by tests/golden/make_cfg1.py): the
disk's history (y and v_y, the columns C1:264 writes, and x, u, omega)
every 10 steps, and the corrected velocity and solid fraction at step
20,000.  FP64 within 1e-10 of each quantity's scale, FP32 shifted within
1e-4.  The frozen gravity gives a peak particle Reynolds number
RHO_P*DIAM*|V|/NU (C1:261) of about 20.

Viscoplastic settling (800 x 2400, one Bingham disk D=40): FP32 shifted
against FP64 at full size, the disk history and the yielded/unyielded flag
of every fluid node (C6:947-954).

Multi-particle sedimentation (1024 x 2048, 512 disks): FP32 against FP64
over the configuration's 50,000 steps.
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


def _cfg1_compare(got, fx, rtol):
    h, w = got["history"], fx["history"]
    assert h.shape == w.shape
    assert np.array_equal(h[:, 0], w[:, 0])
    y0 = got["pin"][0, 1]
    vmax = float(np.max(np.abs(w[:, 3:5])))
    scales = {
        "x": float(np.max(np.abs(w[:, 2] - y0))),  # lateral drift against the fall
        "y": float(np.max(np.abs(w[:, 2] - y0))),
        "u": vmax, "v": vmax,
        "omega": vmax / got["pin"][0, 6],
    }
    x0 = got["pin"][0, 0]
    errs = {
        "x": np.max(np.abs((h[:, 1] - x0) - (w[:, 1] - x0))),
        "y": np.max(np.abs(h[:, 2] - w[:, 2])),
        "u": np.max(np.abs(h[:, 3] - w[:, 3])),
        "v": np.max(np.abs(h[:, 4] - w[:, 4])),
        "omega": np.max(np.abs(h[:, 5] - w[:, 5])),
    }
    for k, e in errs.items():
        assert e <= rtol * scales[k], f"history {k}: {e:.3e} vs scale {scales[k]:.3e}"
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


@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 1e-4)])
def test_cfg1_plain_matches_oracle_over_20000_steps(pkg, cases, cfg1_fixture, precision, rtol):
    got = _cfg1_run(pkg, cases, precision, cfg1_fixture)
    assert got["status"] == 0
    _cfg1_compare(got, cfg1_fixture, rtol)
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


@pytest.mark.parametrize("bn", [0.5, 50.0])
def test_cfg3_viscoplastic_fp32_matches_fp64_full_size(pkg, cases, bn):
    """800 x 2400 Bingham settling, 20,000 steps: FP32 shifted populations
    against FP64, disk position and velocity within 1e-4 of the FP64 scale
    (the total displacement and the largest speed) and the yield flag the
    same on at least 99.9 % of the fluid nodes."""
    steps = 20000
    s64, img64, st64, pin = _visco(pkg, cases, 0, bn, steps)
    s32, img32, st32, _ = _visco(pkg, cases, 1, bn, steps)
    assert st64 == 0 and st32 == 0
    dy = float(np.max(np.abs(s64[:, 3] - pin[0, 1])))
    vmax = float(np.max(np.abs(s64[:, 6])))
    assert np.max(np.abs(s32[:, 3] - s64[:, 3])) <= 1e-4 * dy
    assert np.max(np.abs(s32[:, 6] - s64[:, 6])) <= 1e-4 * vmax
    fluid = (img64 != 10) & (img32 != 10)
    agree = np.mean((img64 == 5)[fluid] == (img32 == 5)[fluid])
    assert agree >= 0.999, agree


def test_cfg2_fp32_trajectory_over_50000_steps(pkg, cases):
    """512 disks, 1024 x 2048, the configuration's 50,000 steps: every disk's
    displacement and velocity in FP32 within 1e-4 of the largest FP64 value."""
    sims = {}
    pin = None
    for prec in (1, 0):
        p, pin = cases.workload_cfg2(prec)
        p.series_every = 0
        sims[prec] = pkg.Simulation(p)
        sims[prec].set_particles(pin)
    for s in sims.values():
        s.step(50000)
    r32, r64 = sims[1].particles(), sims[0].particles()
    for s in sims.values():
        assert s.status() == 0
        s.close()
    d32, d64 = r32[:, 0:2] - pin[:, 0:2], r64[:, 0:2] - pin[:, 0:2]
    dmax = float(np.max(np.linalg.norm(d64, axis=1)))
    vmax = float(np.max(np.linalg.norm(r64[:, 3:5], axis=1)))
    assert np.max(np.linalg.norm(d32 - d64, axis=1)) <= 1e-4 * dmax
    assert np.max(np.linalg.norm(r32[:, 3:5] - r64[:, 3:5], axis=1)) <= 1e-4 * vmax
