"""lbm_adjoint: gradients of a particle observable against central finite
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
