"""lbm_adjoint: gradients of a particle observable against the forward-mode
derivatives of the FP64 oracle (its tangent build, tests/golden/
adjoint_tangent_*.npz, made by tests/golden/make_adjoint_tangent.py: the
FP64 reference adjoint, exact to rounding), against central finite
differences of the FP64 oracle (tests/golden/adjoint_*.npz, made by
tests/golden/make_adjoint_fd.py) and of the GPU's FP64 forward, FP32 against
FP64.

Tolerances: an adjoint entry g matches a difference quotient d(delta) when
|g - d(delta/2)| <= rtol |d(delta/2)| + |d(delta) - d(delta/2)| + floor.
The second term is the quotient's own error: for a central difference the
error of d(delta/2) is about a third of |d(delta) - d(delta/2)|, and it
matters for the initial position, where the solid-fraction profile has a
kink in its second derivative (the measured adjoint errors there are 0.3
to 0.7 of that term).  floor is zero except for the initial position,
whose entries can vanish by symmetry: there it is rtol times the largest
position gradient of the case.  rtol = 1e-6 for the FP64 adjoint, 1e-3 for
the FP32 one.  The objective itself: FP64 within
1e-9 of the oracle's, FP32 within 1e-3.

The torch.autograd.Function below exists only as a test harness: it lets
torch.autograd.grad drive lbm_adjoint for the parameters (tau_y, nu, rho_p,
x0, y0) of one disk.
"""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import adjoint_cases as ac  # noqa: E402

GOLD = os.path.join(HERE, "golden")


def fixture(name):
    return np.load(os.path.join(GOLD, f"adjoint_{name}.npz"))


def grad_vector(g, npd):
    out = [g["tau_y"], g["nu"]]
    for q in range(npd):
        out += [g["rho_p"][q], g["x0"][q], g["y0"][q]]
    return np.array(out)


def check_against_fd(grad, fd, fd_half, rtol, names):
    pos = [k for k, nm in enumerate(names) if nm.startswith(("x0", "y0"))]
    scale = max((abs(fd_half[k]) for k in pos), default=0.0)
    for k, nm in enumerate(names):
        floor = rtol * scale if k in pos else 0.0
        allow = rtol * abs(fd_half[k]) + abs(fd[k] - fd_half[k]) + floor
        assert abs(grad[k] - fd_half[k]) <= allow, (nm, grad[k], fd_half[k], allow)


# ---- CPU: the fixtures ------------------------------------------------------

@pytest.mark.parametrize("name", ac.CASES)
def test_fixture_quotients_converged(name):
    """Both step sizes agree on the parameters that enter smoothly."""
    z = fixture(name)
    for k, nm in enumerate(z["names"]):
        nm = str(nm)
        if nm.startswith(("tau_y", "nu", "rho_p")):
            assert abs(z["fd"][k] - z["fd_half"][k]) <= 1e-6 * abs(z["fd"][k]) + 1e-20, nm


def test_fixture_reproduces_on_the_oracle(cases):
    """One entry recomputed from the oracle matches the stored quotient."""
    sys.path.insert(0, GOLD)
    import make_adjoint_fd as mk

    p, pin, n0, n1 = ac.build(cases, "c6_bingham")
    z = fixture("c6_bingham")
    k = list(map(str, z["names"])).index("rho_p0")
    d = mk.fd(p, pin, n0, n1, "rho_p", 0, mk.REL)
    assert abs(d - z["fd"][k]) <= 1e-12 * abs(z["fd"][k])
    assert abs(mk.run_j(p, pin, n0, n1) - float(z["j"])) <= 1e-15


# ---- CPU: the forward-mode reference -----------------------------------------
# The tangent build of the oracle (oracle/liblbm_oracle_tangent.so) runs the
# oracle's own source with every real a value and its derivative; its
# gradients (tests/golden/adjoint_tangent_*.npz, made by
# tests/golden/make_adjoint_tangent.py) are the exact derivatives of the
# oracle's discrete step: the FP64 reference adjoint, sharing no code with
# the CUDA adjoint kernels.

def tangent_fixture(name):
    return np.load(os.path.join(GOLD, f"adjoint_tangent_{name}.npz"))


def position_scale(names, grad):
    """The largest initial-position gradient of a case: the scale of the
    position entries that vanish by symmetry."""
    return max((abs(grad[k]) for k, nm in enumerate(names) if nm.startswith(("x0", "y0"))),
               default=0.0)


def test_tangent_oracle_values_are_the_ordinary_oracles(cases):
    """Carrying derivatives does not change a value: the tangent run's
    particle state equals the ordinary oracle's bit for bit."""
    from oracle.oracle import Oracle, TangentOracle

    p, pin, _, _ = ac.build(cases, "c3_pair")
    a = Oracle(p)
    a.set_particles(pin)
    a.step(60)
    want = a.particles()
    a.close()
    for which, disk in (("tau_y", -1), ("nu", -1), ("rho_p", 1), ("x0", 0), ("y0", 1)):
        t = TangentOracle(p, which, disk)
        t.set_particles(pin)
        t.step(60)
        assert np.array_equal(t.particles(), want), which
        if which != "tau_y":  # the C3 case is Newtonian: nothing depends on tau_y
            assert np.any(t.particles_tangent() != 0.0), which
        t.close()


def test_tangent_fixture_reproduces(cases):
    sys.path.insert(0, GOLD)
    import make_adjoint_tangent as mt

    p, pin, n0, n1 = ac.build(cases, "c6_bingham")
    z = tangent_fixture("c6_bingham")
    j, g = mt.gradient(p, pin, n0, n1)
    assert j == float(z["j"])
    assert np.array_equal(g, z["grad"])


@pytest.mark.parametrize("name", ac.CASES)
def test_tangent_against_finite_differences(name):
    """The two references agree within the quotient's own error: |t -
    d(delta/2)| <= 2 |d(delta) - d(delta/2)| + 1e-7 |d(delta/2)|, plus 1e-7
    of the case's position scale on the position entries (there the
    quotient of an entry that vanishes by symmetry is rounding noise)."""
    z, t = fixture(name), tangent_fixture(name)
    names = list(map(str, t["names"]))
    assert names == list(map(str, z["names"]))
    assert abs(float(t["j"]) - float(z["j"])) <= 1e-15 * abs(float(z["j"]))
    ps = position_scale(names, t["grad"])
    for k, nm in enumerate(names):
        fd, fh, g = z["fd"][k], z["fd_half"][k], t["grad"][k]
        allow = 2.0 * abs(fd - fh) + 1e-7 * abs(fh) + (1e-7 * ps if nm.startswith(("x0", "y0")) else 0.0)
        assert abs(g - fh) <= allow, (nm, g, fh, allow)


# ---- GPU --------------------------------------------------------------------

def adjoint_run(pkg, p, pin, n0, n1, precision, every=0):
    q = p.copy(precision=precision)
    sim = pkg.Simulation(q)
    sim.set_particles(pin)
    j, g = sim.adjoint(n0, n1, checkpoint_every=every)
    parts = sim.particles()
    sim.close()
    return j, grad_vector(g, pin.shape[0]), parts


@pytest.mark.gpu
@pytest.mark.parametrize("name", ac.CASES)
@pytest.mark.parametrize("precision,rtol,jtol", [(0, 1e-6, 1e-9), (1, 1e-3, 1e-3)])
def test_adjoint_matches_oracle_differences(pkg, cases, name, precision, rtol, jtol):
    p, pin, n0, n1 = ac.build(cases, name)
    z = fixture(name)
    j, g, _ = adjoint_run(pkg, p, pin, n0, n1, precision)
    assert abs(j - float(z["j"])) <= jtol * abs(float(z["j"]))
    check_against_fd(g, z["fd"], z["fd_half"], rtol, list(map(str, z["names"])))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ac.CASES)
@pytest.mark.parametrize("precision,rtol", [(0, 1e-9), (1, 1e-4)])
def test_adjoint_matches_tangent_oracle(pkg, cases, name, precision, rtol):
    """The adjoint against the forward-mode derivatives of the oracle:
    |g - t| <= rtol |t|, plus rtol times the case's position scale on the
    position entries (entries that vanish by symmetry).  Measured: FP64
    within 1.2e-13 of t on tau_y, nu, rho_p and 9e-11 on the positions;
    FP32 within 4.8e-6."""
    p, pin, n0, n1 = ac.build(cases, name)
    t = tangent_fixture(name)
    names = list(map(str, t["names"]))
    j, g, _ = adjoint_run(pkg, p, pin, n0, n1, precision)
    assert abs(j - float(t["j"])) <= (1e-12 if precision == 0 else 1e-5) * abs(float(t["j"]))
    ps = position_scale(names, t["grad"])
    for k, nm in enumerate(names):
        allow = rtol * abs(t["grad"][k]) + (rtol * ps if nm.startswith(("x0", "y0")) else 0.0)
        assert abs(g[k] - t["grad"][k]) <= allow, (nm, g[k], t["grad"][k], allow)


@pytest.mark.gpu
def test_checkpoint_spacing_and_final_state(pkg, cases):
    """Gradients do not depend on the checkpoint spacing; the handle ends at
    step n1 exactly as lbm_step leaves it."""
    p, pin, n0, n1 = ac.build(cases, "c6_bingham")
    ref = None
    for every in (0, 1, 7, 400):
        j, g, parts = adjoint_run(pkg, p, pin, n0, n1, 0, every)
        if ref is None:
            ref = (j, g, parts)
            continue
        assert j == ref[0]
        # entries that vanish by symmetry (x0 here, ~1e-18) carry the
        # summation-order noise of the per-disk FP64 atomics
        assert np.allclose(g, ref[1], rtol=1e-11, atol=1e-15), (every, g, ref[1])
        assert np.array_equal(parts, ref[2])
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    sim.step(n1)
    assert np.array_equal(sim.particles(), ref[2])
    sim.close()


@pytest.mark.gpu
def test_adjoint_rejects_unsupported(pkg, cases):
    p, pin, n0, n1 = ac.build(cases, "c6_bingham")
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    sim.step(1)
    with pytest.raises(pkg.LbmError):  # not at step 0
        sim.adjoint(1, 10)
    sim.close()
    q = p.copy(rheology=2)  # Casson
    sim = pkg.Simulation(q)
    sim.set_particles(pin)
    with pytest.raises(pkg.LbmError):
        sim.adjoint(1, 10)
    with pytest.raises(pkg.LbmError):  # window
        sim.adjoint(10, 5)
    sim.close()


def _autograd_harness(pkg, p, pin, n0, n1, precision):
    import torch

    class Objective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            q = p.copy(precision=precision, tau_y=float(theta[0]), nu=float(theta[1]))
            disks = np.array(pin, copy=True)
            disks[0, 7], disks[0, 0], disks[0, 1] = float(theta[2]), float(theta[3]), float(theta[4])
            sim = pkg.Simulation(q)
            sim.set_particles(disks)
            j, g = sim.adjoint(n0, n1)
            sim.close()
            ctx.save_for_backward(torch.tensor(
                [g["tau_y"], g["nu"], g["rho_p"][0], g["x0"][0], g["y0"][0]], dtype=torch.float64))
            return torch.tensor(j, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout * g

    theta = torch.tensor([p.tau_y, p.nu, pin[0, 7], pin[0, 0], pin[0, 1]], dtype=torch.float64,
                         requires_grad=True)
    j = Objective.apply(theta)
    (g,) = torch.autograd.grad(j, theta)
    return float(j), g.numpy()


@pytest.mark.gpu
def test_autograd_harness_fp32_against_fp64_adjoint_and_differences(pkg, cases):
    p, pin, n0, n1 = ac.build(cases, "c6_bingham")
    z = fixture("c6_bingham")
    j64, g64 = _autograd_harness(pkg, p, pin, n0, n1, 0)
    j32, g32 = _autograd_harness(pkg, p, pin, n0, n1, 1)
    names = list(map(str, z["names"]))
    check_against_fd(g64, z["fd"], z["fd_half"], 1e-6, names)
    check_against_fd(g32, z["fd"], z["fd_half"], 1e-3, names)
    big = [0, 1, 2]  # tau_y, nu, rho_p: FP32 against the FP64 adjoint
    assert np.all(np.abs(g32[big] - g64[big]) <= 1e-3 * np.abs(g64[big]))
    assert abs(j32 - j64) <= 1e-3 * abs(j64)


@pytest.mark.gpu
def test_full_size_adjoint_against_gpu_fp64_differences(pkg, cases):
    """The adjoint workload at its full size (400 x 1200, D=24, Bn=5, 4000
    steps, window 3000..4000, sqrt(N) checkpoints): the FP64 and FP32 adjoints
    against central differences (relative step 1e-4) of the GPU's FP64
    forward, which is pinned to the oracle."""
    p64, pin, info = cases.workload_cfg5(0)
    n0, n1 = info["n0"], info["n1"]

    def run_j(p, disks):
        sim = pkg.Simulation(p)
        sim.set_particles(disks)
        sim.step(n0 - 1)
        v = []
        for _ in range(n0, n1 + 1):
            sim.step(1)
            v.append(sim.particles()[0, 4])
        sim.close()
        return float(np.mean(v))

    j64, g64, _ = adjoint_run(pkg, p64, pin, n0, n1, 0)
    j32, g32, _ = adjoint_run(pkg, p64, pin, n0, n1, 1)
    assert abs(j64 - run_j(p64, pin)) <= 1e-12 * abs(j64)
    ents = ac.parameters(1)
    for k, (name, disk) in enumerate(ents):
        if name == "x0":
            continue  # zero by symmetry
        fds = []
        for rel in (1e-4, 0.5e-4):
            d = rel * abs(ac.base_value(p64, pin, name, disk))
            jp = run_j(*ac.perturbed(p64, pin, name, disk, d))
            jm = run_j(*ac.perturbed(p64, pin, name, disk, -d))
            fds.append((jp - jm) / (2 * d))
        fd, fdh = fds
        for g, rtol in ((g64[k], 1e-6), (g32[k], 1e-3)):
            allow = rtol * abs(fdh) + abs(fd - fdh)
            assert abs(g - fdh) <= allow, (name, g, fdh, allow)
    assert abs(j32 - j64) <= 1e-3 * abs(j64)


@pytest.mark.gpu
def test_full_size_adjoint_against_tangent_oracle(pkg, cases):
    """The adjoint workload at its full size (400 x 1200, 4000 steps,
    sqrt(N) checkpoints) against the forward-mode derivatives of the oracle
    on the same inputs (tests/golden/adjoint_tangent_full.npz, made by
    make_adjoint_tangent.py --full): FP64 within 1e-9, FP32 within 1e-4, of
    each entry (plus that fraction of the position scale on the position
    entries, x0 vanishing by symmetry)."""
    t = np.load(os.path.join(GOLD, "adjoint_tangent_full.npz"))
    names = list(map(str, t["names"]))
    p64, pin, info = cases.workload_cfg5(0)
    ps = position_scale(names, t["grad"])
    for precision, rtol, jtol in ((0, 1e-9, 1e-10), (1, 1e-4, 1e-5)):
        j, g, _ = adjoint_run(pkg, p64, pin, info["n0"], info["n1"], precision)
        assert abs(j - float(t["j"])) <= jtol * abs(float(t["j"])), (precision, j)
        for k, nm in enumerate(names):
            allow = rtol * abs(t["grad"][k]) + (rtol * ps if nm.startswith(("x0", "y0")) else 0.0)
            assert abs(g[k] - t["grad"][k]) <= allow, (precision, nm, g[k], t["grad"][k], allow)
