"""The failure path of the kernels' bounded waits, exercised without a GPU
fault: a device wait that cannot complete (an mbarrier nothing arrives at)
gives up after its poll limit, the handle reports LBM_E_TIMEOUT and refuses
further steps, and the device stays usable for other handles."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LBM_E_TIMEOUT = -6


def test_expired_wait_sets_timeout_and_device_stays_usable(pkg, cases):
    p = cases.shipped_c1(40, 40, 8.0)
    ref = pkg.Simulation(p)
    ref.step(6)
    want = ref.field("ux")
    ref.close()

    sim = pkg.Simulation(p)
    sim.step(3)
    assert sim.status() == 0
    sim.selftest_wait(256)
    assert sim.status() == LBM_E_TIMEOUT
    with pytest.raises(pkg.LbmError) as err:
        sim.step(1)
    assert err.value.code == LBM_E_TIMEOUT
    sim.close()

    # a new handle on the same device steps as before
    other = pkg.Simulation(p)
    other.step(6)
    assert other.status() == 0
    assert np.array_equal(other.field("ux"), want)
    other.close()


def test_selftest_limit_is_validated(pkg, cases):
    sim = pkg.Simulation(cases.shipped_c1(20, 20, 8.0))
    for bad in (0, -1, (1 << 20) + 1):
        with pytest.raises(pkg.LbmError):
            sim.selftest_wait(bad)
    assert sim.status() == 0
    sim.close()


# ---- failures made on the host: bad states and bad inputs --------------------
# None of these faults the GPU: each is an input that the library's own checks
# turn into a status code: NaN detection, capacity overflows, particles
# leaving the lattice, overlapping input disks.

LBM_E_NAN, LBM_E_OVERFLOW, LBM_E_PARTICLE = -5, -7, -9


def _state_with(sim, node, k, value):
    """The handle's state with population k of node (i, j) replaced."""
    f, om, ps = sim.get_state()
    i, j = node
    n1x = sim.n1x
    f = f.copy()
    f[(j * n1x + i) * 9 + k] = value
    return f, om, ps


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_in_fluid_without_disks_is_reported(pkg, cases, precision):
    """A non-finite population far from any disk (here: no disks at all)
    makes the next step report LBM_E_NAN; the sticky status then refuses
    further steps."""
    p = cases.shipped_c1(64, 40, 8.0)
    p.precision = precision
    sim = pkg.Simulation(p)
    sim.step(5)
    assert sim.status() == 0
    f, om, ps = _state_with(sim, (30, 20), 5, np.nan)
    sim.set_state(sim.kk, f, om, ps)
    sim.step(2)
    assert sim.status() == LBM_E_NAN
    with pytest.raises(pkg.LbmError) as err:
        sim.step(1)
    assert err.value.code == LBM_E_NAN
    sim.close()


def test_fp32_density_beyond_mass_sum_range_is_reported(pkg, cases):
    """FP32: a finite density deviation |rho - rho0| >= 2 is past the range of
    the fixed-point mean-density sum; the step reports LBM_E_OVERFLOW instead
    of writing a saturated history value.  The same state in FP64 steps on.
    The excess put into one node's rest population (about 9.6) is collided
    and streamed before the step sees it: the node keeps about 4/9 of it."""
    for precision, want in ((1, LBM_E_OVERFLOW), (0, 0)):
        p = cases.shipped_c1(64, 40, 8.0)
        p.precision = precision
        p.series_every = 1
        sim = pkg.Simulation(p)
        sim.step(2)
        f, om, ps = _state_with(sim, (30, 20), 0, 10.0)
        sim.set_state(sim.kk, f, om, ps)
        sim.step(1)
        assert sim.status() == want, precision
        sim.close()


def test_more_than_32_disks_on_one_tile_is_reported(pkg, cases):
    """33 small disks in one 128 x 8 list tile exceed its candidate list."""
    p = cases.shipped_c1(200, 40, 2.0)
    xy = [[3.0 + 3.0 * k, 4.0] for k in range(33)]
    sim = pkg.Simulation(p)
    with pytest.raises(pkg.LbmError) as err:
        sim.set_particles(cases.pin_array(xy, 2.0, 1.25))
    assert err.value.code == LBM_E_OVERFLOW
    sim.close()
    # 32 fit
    sim = pkg.Simulation(p)
    sim.set_particles(cases.pin_array(xy[:32], 2.0, 1.25))
    assert sim.status() == 0
    sim.close()


def test_more_than_32_pair_neighbours_is_reported(pkg, cases):
    """A ring of 40 small disks around a large one: the large disk has 40
    pair-list neighbours (more than 32) while no list tile holds more than
    32 disks; the first step's pair-list build reports LBM_E_OVERFLOW."""
    p = cases.shipped_c1(100, 100, 20.0)
    th = 2.0 * np.pi * np.arange(40) / 40.0
    xy = [[50.0, 50.0]] + [[50.0 + 11.0 * np.cos(t), 50.0 + 11.0 * np.sin(t)] for t in th]
    d = np.array([20.0] + [1.0] * 40)
    sim = pkg.Simulation(p)
    sim.set_particles(cases.pin_array(xy, d, 1.25))
    assert sim.status() == 0
    sim.step(1)
    assert sim.status() == LBM_E_OVERFLOW
    sim.close()


def test_disk_driven_out_of_the_lattice_is_reported(pkg, cases):
    """A disk next to the right edge with a large outward velocity (no wall
    repulsion) leaves the lattice in its first step: LBM_E_PARTICLE."""
    p = cases.shipped_c1(40, 40, 4.0)
    p.wall_model = 2  # LBM_WALL_NONE
    disk = cases.pin_array([[37.0, 20.0]], 4.0, 1.25, uvw=[[10.0, 0.0, 0.0]])
    sim = pkg.Simulation(p)
    sim.set_particles(disk)
    sim.step(1)
    assert sim.status() == LBM_E_PARTICLE
    sim.close()


def test_overlapping_input_disks_are_rejected(pkg, cases):
    """lbm_set_particles rejects input disks whose centres are closer than
    the sum of their radii; touching disks are accepted."""
    p = cases.shipped_c1(60, 60, 8.0)
    sim = pkg.Simulation(p)
    with pytest.raises(pkg.LbmError) as err:
        sim.set_particles(cases.pin_array([[20.0, 20.0], [25.0, 20.0]], 8.0, 1.25))
    assert err.value.code == LBM_E_PARTICLE
    with pytest.raises(pkg.LbmError):
        sim.set_particles(cases.pin_array([[20.0, 20.0], [30.0, 30.0], [26.0, 26.0]],
                                          np.array([8.0, 8.0, 4.0]), 1.25))
    sim.set_particles(cases.pin_array([[20.0, 20.0], [28.0, 20.0]], 8.0, 1.25))
    assert sim.status() == 0
    sim.close()


def _overlaps(xy, d):
    """All pairs: some two disks closer than the sum of their radii."""
    e = xy[:, None, :] - xy[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", e, e)
    rs = 0.5 * (d[:, None] + d[None, :])
    np.fill_diagonal(r2, np.inf)
    return bool(np.any(r2 < rs * rs))


@pytest.mark.parametrize("seed", range(8))
def test_overlap_check_matches_all_pairs(pkg, cases, seed):
    """The library's overlap check (a cell grid) against all pairs, on random
    disk sets of mixed diameters: sets built without overlap are accepted,
    the same sets with one disk moved onto another (anywhere, so across cell
    edges too) are rejected."""
    rng = np.random.default_rng(seed)
    nx, ny = 300, 500
    xy, d = [], []
    while len(xy) < 150:
        c = rng.uniform([0.0, 0.0], [nx, ny])
        dd = rng.uniform(2.0, 14.0)
        if all(np.hypot(*(c - q)) >= 0.5 * (dd + e) for q, e in zip(xy, d)):
            xy.append(c)
            d.append(dd)
    xy, d = np.array(xy), np.array(d)
    assert not _overlaps(xy, d)
    p = cases.shipped_c1(nx, ny, 8.0)
    sim = pkg.Simulation(p)
    sim.set_particles(cases.pin_array(xy, d, 1.25))
    a, b = rng.choice(len(xy), 2, replace=False)
    xy2 = xy.copy()
    ang = rng.uniform(0.0, 2 * np.pi)
    xy2[a] = np.clip(xy[b] + 0.45 * (d[a] + d[b]) * np.array([np.cos(ang), np.sin(ang)]),
                     [0.0, 0.0], [nx, ny])
    assert _overlaps(xy2, d)
    with pytest.raises(pkg.LbmError) as err:
        sim.set_particles(cases.pin_array(xy2, d, 1.25))
    assert err.value.code == LBM_E_PARTICLE
    sim.close()
