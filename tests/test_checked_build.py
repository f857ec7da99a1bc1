"""The checked build (liblbm2d_checked.so, compiled with LBM_CHECKED): every
computed index of the step, particle and batch kernels is checked against
its buffer, and a failed check skips the access and reports LBM_E_BOUNDS,
in place of the memory checker, which this GPU pool does not offer.  The
cases of tests/checked_cases.py run once on the ordinary library (in this
process) and once on the checked one (a child process that loads it through
LBM2D_LIBRARY): no check may fire, and the results must be the same -- bit
for bit in FP64, within 1e-6 of each quantity's scale in FP32 (the two
builds may contract FP32 multiply-adds differently), and the adjoint's
gradient within 1e-12 of each entry (its per-disk sums are FP64 atomics,
whose order, and so whose last bits, differ from run to run of any build)."""

import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import checked_cases  # noqa: E402


def test_checked_build_query_without_device(pkg):
    """The ordinary library says it is not the checked build; the checked
    one is built beside it."""
    assert int(pkg.load_library().lbm_checked_build()) == 0
    checked = os.path.join(os.path.dirname(pkg.library_path()), "liblbm2d_checked.so")
    assert os.path.exists(checked)


@pytest.mark.gpu
def test_checked_build_fires_no_check_and_matches(pkg, tmp_path):
    want = checked_cases.run_cases(pkg)
    assert int(want["checked_build"]) == 0
    out = str(tmp_path / "checked.npz")
    env = dict(os.environ)
    env["LBM2D_LIBRARY"] = os.path.join(os.path.dirname(pkg.library_path()), "liblbm2d_checked.so")
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_cases.py"), out], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    got = dict(np.load(out))
    assert int(got["checked_build"]) == 1
    assert set(got) == set(want)
    for k, v in got.items():
        if k == "checked_build":
            continue
        if k.endswith("status"):
            assert int(v) == 0, (k, int(v))  # 0: no LBM_E_BOUNDS, no other error
            continue
        w = want[k]
        assert v.shape == w.shape, k
        if k.startswith(("sed1", "c6", "batch")):  # FP32 runs
            scale = max(float(np.max(np.abs(w))), 1e-300)
            assert np.max(np.abs(v - w)) <= 1e-6 * scale, k
        elif k == "adj_grad":
            assert np.all(np.abs(v - w) <= 1e-12 * np.abs(w)), (v, w)
        else:
            assert np.array_equal(v, w), k
