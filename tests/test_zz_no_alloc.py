"""lbm_fields_noalloc (static device scratch, no allocation) against the
handle-based output path (lbm_get_field / lbm_get_image) on the same state.

The state and the particle records go to the device in buffers the test
owns; the entry point itself allocates nothing.  Two calls in a row, on
different states, must each match the existing path: the second call shows
the scratch left by the first does not leak into it.  FP64 runs take the
same operations as the output kernel, so the tolerance there is 1e-12 of
each field's magnitude; FP32 runs compare FP64 arithmetic on the widened
state against the FP32 output kernel, 1e-4.
"""

import ctypes

import numpy as np
import pytest

FIELDS = ("ux", "uy", "rho", "phi", "gx", "gy")


def _pin_from_state(ps):
    # LBM_PIN record: x, y, angle, u, v, omega, diam, rho_p
    return np.ascontiguousarray(ps[:, [0, 1, 2, 3, 4, 5, 17, 18]], dtype=np.float64)


def _noalloc_fields(pkg, torch, sim, params):
    f, _, ps = sim.get_state()
    pin = _pin_from_state(ps)
    n1x, n1y = params.nx + 1, params.ny + 1
    dev = torch.device("cuda", 0)
    f_d = torch.from_numpy(f).to(dev)
    pin_d = torch.from_numpy(pin.reshape(-1)).to(dev)
    out_d = torch.full((7 * n1x * n1y,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = pkg.load_library()
    rc = lib.lbm_fields_noalloc(
        ctypes.byref(params), ctypes.c_void_p(f_d.data_ptr()), pin.shape[0],
        ctypes.c_void_p(pin_d.data_ptr()), ctypes.c_void_p(out_d.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.lbm_strerror(rc)
    return out_d.cpu().numpy().reshape(7, n1y, n1x)


def _check(sim, out, rtol):
    for k, name in enumerate(FIELDS):
        ref = sim.field(name)
        scale = max(float(np.max(np.abs(ref))), 1e-300)
        err = float(np.max(np.abs(out[k] - ref)))
        assert err <= rtol * scale, f"{name}: {err:.3e} vs scale {scale:.3e}"
    img = sim.image()
    assert np.array_equal(out[6] == 10.0, img == 10)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,rtol", [(0, 1e-12), (1, 1e-4)])
def test_noalloc_matches_get_field_two_calls(pkg, cases, precision, rtol):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    p = cases.shipped_c1(120, 200, 16.0)
    p.precision = precision
    pin = cases.pin_array([[40.0, 120.0], [62.0, 128.0], [80.0, 90.0]], 16.0, 1.25)
    pin[1, 5] = 2e-3  # one spinning disk, so the rigid-body velocity matters
    sim = pkg.Simulation(p)
    try:
        sim.set_particles(pin)
        sim.step(25)
        first = _noalloc_fields(pkg, torch, sim, p)
        _check(sim, first, rtol)
        sim.step(40)  # a different state for the second call
        second = _noalloc_fields(pkg, torch, sim, p)
        _check(sim, second, rtol)
        assert not np.array_equal(first[0], second[0])
    finally:
        sim.close()


def test_noalloc_rejects_oversize_before_any_work(pkg):
    lib = pkg.load_library()
    p = pkg.LbmParams(nx=2048, ny=8191)  # 17 x 1024 list tiles > 16384
    dummy = ctypes.c_void_p(16)  # never dereferenced: rejected on the host
    rc = lib.lbm_fields_noalloc(ctypes.byref(p), dummy, 0, None, dummy, None)
    assert rc == -11
    assert b"scratch" in lib.lbm_strerror(rc)
    p = pkg.LbmParams(nx=100, ny=100)
    rc = lib.lbm_fields_noalloc(ctypes.byref(p), dummy, 4097, dummy, dummy, None)
    assert rc == -11
    assert lib.lbm_fields_noalloc(ctypes.byref(p), None, 0, None, dummy, None) == -1


def _raw_call(pkg, torch, params, f, pin):
    n1x, n1y = params.nx + 1, params.ny + 1
    dev = torch.device("cuda", 0)
    f_d = torch.from_numpy(np.ascontiguousarray(f)).to(dev)
    pin_d = torch.from_numpy(np.ascontiguousarray(pin).reshape(-1)).to(dev)
    out_d = torch.zeros((7 * n1x * n1y,), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = pkg.load_library()
    rc = lib.lbm_fields_noalloc(
        ctypes.byref(params), ctypes.c_void_p(f_d.data_ptr()), pin.shape[0],
        ctypes.c_void_p(pin_d.data_ptr()), ctypes.c_void_p(out_d.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))
    return rc, out_d.cpu().numpy().reshape(7, n1y, n1x)


@pytest.mark.gpu
def test_noalloc_reports_overflow_and_nonfinite_records(pkg, cases):
    """33 small disks in one 128 x 8 tile: LBM_E_OVERFLOW (the output is
    then incomplete).  A record with a non-finite position: LBM_E_NAN, the
    other disks still evaluated.  A clean call afterwards returns 0: the
    flags of the scratch start at zero on every call."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    p = cases.shipped_c1(200, 40, 2.0)
    n = (p.nx + 1) * (p.ny + 1)
    f = np.tile(np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4), n)  # rest state
    many = cases.pin_array([[3.0 + 3.0 * k, 4.0] for k in range(33)], 2.0, 1.25)
    rc, _ = _raw_call(pkg, torch, p, f, many)
    assert rc == -7
    bad = cases.pin_array([[30.0, 20.0], [60.0, 20.0]], 8.0, 1.25)
    bad[1, 0] = np.nan
    rc, out = _raw_call(pkg, torch, p, f, bad)
    assert rc == -5
    assert out[3, 20, 30] == 1.0  # the finite disk's centre is solid
    rc, out = _raw_call(pkg, torch, p, f, bad[:1])
    assert rc == 0
    assert out[3, 20, 30] == 1.0 and out[3, 20, 60] == 0.0
