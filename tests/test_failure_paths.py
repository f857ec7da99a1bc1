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
