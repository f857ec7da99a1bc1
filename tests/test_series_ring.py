"""History records through a device ring much smaller than the run.

With series_capacity = 4 and a record every step, the ring wraps every four
steps: before a step writes a slot again, the handle's stream waits for the
copy of the slot's previous record, and the copied mean-density sums are
cleared on the copy stream.  Fifty steps in one lbm_step call and again in
uneven chunks (the series read between calls) must give the same records,
bit for bit, as a run whose ring holds all fifty, in both precisions."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(pkg, cases, precision, capacity, chunks):
    p = cases.shipped_c1(64, 96, 12.0)
    p.precision = precision
    p.series_every = 1
    p.series_particles = 2
    p.series_capacity = capacity
    disks = cases.pin_array([[20.0, 60.0], [44.0, 64.0]], 12.0, np.array([1.25, 1.4]))
    sim = pkg.Simulation(p)
    sim.set_particles(disks)
    got = []
    for c in chunks:
        sim.step(c)
        got.append(sim.series())
    sim.close()
    return np.concatenate(got)


@pytest.mark.parametrize("precision", [0, 1])
def test_small_ring_matches_large_ring_bit_for_bit(pkg, cases, precision):
    want = _run(pkg, cases, precision, 4096, [50])
    assert want.shape[0] == 50
    assert np.array_equal(want[:, 0], np.arange(1, 51))
    one_call = _run(pkg, cases, precision, 4, [50])
    uneven = _run(pkg, cases, precision, 4, [3, 1, 7, 4, 13, 2, 9, 11])
    # every column, including the mean density (column 1)
    assert np.array_equal(one_call, want)
    assert np.array_equal(uneven, want)
    assert np.all(np.isfinite(want))


def test_records_of_many_disks_match_the_particle_state(pkg, cases):
    """700 disks, each recorded every step: the particle kernel stages the
    records of the first disks in shared memory and writes the rest
    directly; every disk's record of the last step (centre, angle,
    velocities, F_H_IN) equals the particle state read back after it, bit
    for bit (both are the same values of the same kernel)."""
    n = 700
    xy = np.array([[12.0 + 13.0 * (k % 28), 12.0 + 14.0 * (k // 28)] for k in range(n)])
    p = cases.shipped_c1(400, 400, 4.0)
    p.precision = 1
    p.series_every = 1
    p.series_particles = n
    p.series_capacity = 8
    sim = pkg.Simulation(p)
    sim.set_particles(cases.pin_array(xy, 4.0, 1.25))
    sim.step(3)
    s = sim.series()
    parts = sim.particles()
    st = sim.status()
    sim.close()
    assert st == 0
    assert s.shape == (3, 2 + 12 * n)
    assert np.array_equal(s[:, 0], [1.0, 2.0, 3.0])
    rec = s[-1, 2:].reshape(n, 12)
    assert np.array_equal(rec[:, 0:6], parts[:, 0:6])
    assert np.array_equal(rec[:, 9:12], parts[:, 11:14])
    assert np.any(rec[:, 4] != 0.0)  # the disks have started to move
