"""lbm_batch_*: simulations advanced together in one launch per kernel per
step must reach, each of them, the state the same simulation reaches alone
through lbm_step -- bit for bit in FP64 (same node arithmetic, exact force and
mass sums); within 1e-6 of each quantity's scale in FP32, whose FP32
translation unit lets the compiler contract products into FMAs differently
in the batch kernel and the single-simulation kernel -- across graph
replays, fresh starts and history draining; and bit for bit the same for
every tile shape and grid in both precisions."""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import adjoint_cases as ac  # noqa: E402

pytestmark = pytest.mark.gpu


def mixed_cases(cases, precision):
    out = []
    for name in ("c6_bingham", "c1_newton", "c3_pair"):
        p, pin, _, _ = ac.build(cases, name)
        out.append((p.copy(precision=precision), pin))
    p, pin = cases.shipped_c6(33, 97)  # odd sizes, the disk at its coded start
    p.gravity = -1e-5
    out.append((p.copy(precision=precision), pin))
    p, pin = cases.shipped_c4(40, 30, 10.0, 10.0, 40.0)  # equilibrium boundary, prescribed motion
    out.append((p.copy(precision=precision), pin))
    p = cases.shipped_c1(48, 40, 8.0)  # no particles
    out.append((p.copy(precision=precision), None))
    p = cases.shipped_c1(40, 60, 8.0)  # the BGK collision with the bi-viscosity model
    p.collision, p.rheology, p.tau_y, p.gravity = 1, 1, 2e-6, -2e-5
    out.append((p.copy(precision=precision), cases.pin_array([[20.0, 38.0]], 8.0, 1.5)))
    for p, _ in out:
        p.series_every = 5
        p.series_capacity = 4  # the ring fills: the batch drains between chunks
        p.series_particles = 2
    return out


def run_alone(pkg, p, pin, steps):
    sim = pkg.Simulation(p)
    if pin is not None:
        sim.set_particles(pin)
    sim.step(steps)
    res = state(sim)
    sim.close()
    return res


def state(sim):
    return {
        "parts": sim.particles() if sim.np else np.zeros(0),
        "ux": sim.field("ux"),
        "rho": sim.field("rho"),
        "series": sim.series(),
    }


def assert_same(a, b, what):
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), (what, k)


def assert_close(a, b, what, rtol=1e-6):
    for k in a:
        x, y = np.nan_to_num(np.asarray(a[k])), np.nan_to_num(np.asarray(b[k]))
        if k == "parts" and y.size:
            # position, velocity; the hydrodynamic force, a sum over the disk
            # with cancellation, gets ten times the tolerance
            cols = ((slice(0, 2), rtol), (slice(3, 6), rtol), (slice(6, 9), 10 * rtol))
            for c, tol in cols:
                sc = max(float(np.max(np.abs(y[:, c]))), 1e-300)
                assert np.max(np.abs(x[:, c] - y[:, c])) <= tol * sc, (what, k, c)
            continue
        sc = max(float(np.max(np.abs(y))) if y.size else 0.0, 1e-300)
        assert (np.max(np.abs(x - y)) if y.size else 0.0) <= rtol * sc, (what, k)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_each_simulation_alone(pkg, cases, precision):
    cs = mixed_cases(cases, precision)
    steps = 53  # tuning steps, graph replays and a remainder
    ref = [run_alone(pkg, p, pin, steps) for p, pin in cs]
    b = pkg.Batch([p for p, _ in cs])
    for s, (_, pin) in zip(b.sims, cs):
        if pin is not None:
            s.set_particles(pin)
    b.step(20)
    b.step(steps - 20)
    tx, ty, bpsm = b.tuning()
    assert tx * ty == 256 and bpsm > 0
    for q, s in enumerate(b.sims):
        if precision == 0:
            assert_same(state(s), ref[q], (precision, q))
        else:
            assert_close(state(s), ref[q], (precision, q))
    b.close()


def batch_run(pkg, cs, shape, steps):
    b = pkg.Batch([p for p, _ in cs])
    b.set_tuning(*shape)
    for s, (_, pin) in zip(b.sims, cs):
        s.set_particles(pin)
    b.step(steps)
    assert b.tuning() == shape
    out = [state(s) for s in b.sims]
    b.close()
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_tile_shapes_agree(pkg, cases, precision):
    cs = mixed_cases(cases, precision)[:4]
    ref = batch_run(pkg, cs, (32, 8, 2), 24)
    for shape in ((64, 4, 4), (128, 2, 8), (32, 8, 1)):
        got = batch_run(pkg, cs, shape, 24)
        for q in range(len(cs)):
            assert_same(got[q], ref[q], (shape, q))


def test_batch_rejects_mixed_precision(pkg, cases):
    p = cases.shipped_c1(40, 40, 8.0)
    with pytest.raises(pkg.LbmError):
        pkg.Batch([p.copy(precision=0), p.copy(precision=1)])
    with pytest.raises(pkg.LbmError):
        b = pkg.Batch([p])
        b.set_tuning(48, 4, 2)


@pytest.mark.parametrize("tma", [False, True])
@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 1e-4)])
def test_batch_mrt_runs_match_the_oracle(pkg, cases, precision, rtol, tma):
    """Each MRT run of a batch (the one-node-per-thread kernel at 32 x 8
    tiles, or the TMA-staged kernel) against the oracle's run of the same
    inputs, not against another GPU path: the C6 Bingham case (the GPU's
    per-node omega, oracle rule omega_chain=0, 1e-8 in FP64 as in the
    single-run parity tests), C1 Zou-He and a C3 pair in contact range."""
    from oracle.oracle import Oracle

    cs = []
    for name in ("c6_bingham", "c1_newton", "c3_pair"):
        p, pin, _, _ = ac.build(cases, name)
        p = p.copy(precision=precision)
        p.series_every = 0
        cs.append((name, p, pin))
    steps = 41
    b = pkg.Batch([p for _, p, _ in cs])
    b.set_tuning(*(_tma_shape(precision) if tma else (32, 8, 4)))
    for s, (_, _, pin) in zip(b.sims, cs):
        s.set_particles(pin)
    b.step(steps)
    for s, (name, p, pin) in zip(b.sims, cs):
        tol = 1e-8 if (precision == 0 and name == "c6_bingham") else rtol
        ref = Oracle(p, omega_chain=0)
        ref.set_particles(pin)
        ref.step(steps)
        gp, rp = s.particles(), ref.particles()
        d = float(np.max(pin[:, 6]))
        vmax = max(float(np.max(np.abs(rp[:, 3:5]))), 1e-300)
        disp = max(float(np.max(np.abs(rp[:, 0:2] - pin[:, 0:2]))), 1e-300)
        assert np.max(np.abs(gp[:, 0:2] - rp[:, 0:2])) <= tol * disp, (name, "position")
        assert np.max(np.abs(gp[:, 3:5] - rp[:, 3:5])) <= tol * vmax, (name, "velocity")
        assert np.max(np.abs(gp[:, 5] - rp[:, 5])) <= tol * vmax / d, (name, "spin")
        for fld in ("ux", "uy", "rho"):  # each against its field's magnitude
            g, r = s.field(fld), ref.field(fld)
            sc = float(np.max(np.abs(r)))
            assert np.max(np.abs(g - r)) <= tol * max(sc, 1e-300), (name, fld)
        ref.close()
    b.close()


def _tma_shape(precision):
    return (64, 8, 2)  # the TMA-staged batched tiles, both precisions


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_tma_tiles_match_each_simulation_alone(pkg, cases, precision):
    """The TMA-staged batched kernel (k_step_batch: the single-run step
    kernel's tiles and node arithmetic over every simulation of the batch)
    against each run alone through lbm_step: bit for bit in FP64, within
    1e-6 in FP32; MRT runs only (Bingham, Zou-He, a pair, odd sizes, the
    equilibrium boundary with prescribed motion, no disks)."""
    cs = mixed_cases(cases, precision)[:6]
    steps = 29
    ref = [run_alone(pkg, p, pin, steps) for p, pin in cs]
    b = pkg.Batch([p for p, _ in cs])
    shape = _tma_shape(precision)
    b.set_tuning(*shape)
    for s, (_, pin) in zip(b.sims, cs):
        if pin is not None:
            s.set_particles(pin)
    b.step(11)
    b.step(steps - 11)
    assert b.tuning()[:2] == shape[:2]
    for q, s in enumerate(b.sims):
        if precision == 0:
            assert_same(state(s), ref[q], ("tma", q))
        else:
            assert_close(state(s), ref[q], ("tma", q))
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_tma_tiles_agree_with_scalar_tiles(pkg, cases, precision):
    cs = mixed_cases(cases, precision)[:4]
    ref = batch_run(pkg, cs, (32, 8, 2), 24)
    b = pkg.Batch([p for p, _ in cs])
    shape = _tma_shape(precision)
    b.set_tuning(*shape)
    for s, (_, pin) in zip(b.sims, cs):
        s.set_particles(pin)
    b.step(24)
    got = [state(s) for s in b.sims]
    b.close()
    for q in range(len(cs)):
        if precision == 0:
            assert_same(got[q], ref[q], ("tma-vs-scalar", q))
        else:
            assert_close(got[q], ref[q], ("tma-vs-scalar", q))
