"""lbm_main, the C++ driver that mirrors the reference's MAIN on the C ABI:
its history, field and restart files against the library's own getters."""

import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "2d_nnf_lbm_b200", "lbm_main")


def test_driver_builds_and_prints_usage():
    assert os.path.exists(DRIVER), "build with __graft_entry__.build()"
    r = subprocess.run([DRIVER, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--case" in r.stdout
    r = subprocess.run([DRIVER, "--case", "c9"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown case" in r.stderr


def _table(path, skip=1):
    with open(path) as fh:
        rows = [l.split() for l in fh.readlines()[skip:] if l.strip()]
    return np.array([[float(v) for v in r] for r in rows])


def _run(args, cwd):
    r = subprocess.run([DRIVER, *args], capture_output=True, text=True, cwd=cwd)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_driver_c1_history_fields_and_restart(pkg, cases, tmp_path):
    nx, ny, steps = 48, 72, 40
    (tmp_path / "p.txt").write_text("24\t50\t12\t1.25")
    out, dump, dump2, dump3 = (tmp_path / d for d in ("out", "dump", "dump2", "dump3"))
    for d in (out, dump, dump2, dump3):
        d.mkdir()
    _run(["--case", "c1", "--nx", str(nx), "--ny", str(ny), "--steps", str(steps),
          "--input", "p.txt", "--out", "out", "--dump", "dump", "--chunk", "16"], tmp_path)

    # the same case through the Python binding
    p = cases.shipped_c1(nx, ny, 12.0)
    p.series_every, p.series_particles, p.series_capacity = 1, 1, 64
    sim = pkg.Simulation(p)
    try:
        sim.set_particles(cases.pin_array([[24.0, 50.0]], 12.0, 1.25))
        sim.step(steps)
        ser = sim.series()
        c_l = float(np.float32(0.25)) / 30.0
        c_t = (c_l * c_l) * p.nu / float(np.float32(0.1))
        c_u = c_l / c_t
        hist = _table(out / "01_ParticleTimehistory.plt")
        assert hist.shape == (steps, 5)
        np.testing.assert_allclose(hist[:, 0], ser[:, 0] * c_t, rtol=1e-15)
        np.testing.assert_allclose(hist[:, 1], ser[:, 2 + 1] * c_l, rtol=1e-15)
        np.testing.assert_allclose(hist[:, 2], ser[:, 2 + 4] * c_u, rtol=1e-15)
        dens = _table(out / "01_AveragedDensity.PLT")
        np.testing.assert_allclose(dens[:, 1], ser[:, 1], rtol=1e-15)
        # Tecplot BLOCK file: 9 variables x (NY+1) rows of NX+1 values
        with open(out / f"02_VelocityField_{steps}.plt") as fh:
            lines = fh.readlines()
        assert lines[0].strip().startswith("VARIABLES") and "F=BLOCK" in lines[1]
        blk = np.array([[float(v) for v in l.split()] for l in lines[2:]])
        assert blk.shape == (9 * (ny + 1), nx + 1)
        np.testing.assert_array_equal(blk[2 * (ny + 1):3 * (ny + 1)], sim.field("ux"))
        np.testing.assert_array_equal(blk[4 * (ny + 1):5 * (ny + 1)], sim.field("rho"))

        # legacy dump -> restart -> dump reproduces the files
        _run(["--case", "c1", "--nx", str(nx), "--ny", str(ny), "--steps", "0", "--input", "p.txt",
              "--out", "out", "--restart", "dump", "--dump", "dump2"], tmp_path)
        for name in ("0_F_output.txt", "0_Particle_output.txt", "0_OmegaBN_output.txt"):
            a, b = _table(dump / name, 0), _table(dump2 / name, 0)
            np.testing.assert_array_equal(a, b)

        # a restarted run continues as lbm_set_state with the dump's content
        # (VP_OLD, F_COL, F_H_IN zero, step counter 0), bit for bit
        _run(["--case", "c1", "--nx", str(nx), "--ny", str(ny), "--steps", "10", "--input", "p.txt",
              "--out", "out", "--restart", "dump", "--dump", "dump3"], tmp_path)
        f_rows = _table(dump / "0_F_output.txt", 0)           # I outer, J inner
        f = f_rows.reshape(nx + 1, ny + 1, 9).transpose(1, 0, 2).reshape(-1)
        om = _table(dump / "0_OmegaBN_output.txt", 0).reshape(nx + 1, ny + 1).T.reshape(-1)
        pr = _table(dump / "0_Particle_output.txt", 0)
        st = np.zeros((1, 20))
        st[0, [0, 1, 3, 4, 5, 9, 10, 11]] = pr[0]
        st[0, 17], st[0, 18], st[0, 19] = 12.0, 1.25, np.inf
        sim.set_state(0, f, om, st)
        sim.step(10)
        got = _table(dump3 / "0_Particle_output.txt", 0)
        q = sim.particles()[0]
        np.testing.assert_array_equal(got[0], q[[0, 1, 3, 4, 5, 6, 7, 8]])
    finally:
        sim.close()


@pytest.mark.gpu
def test_driver_c4_history_matches_reference(tmp_path):
    """lbm_main --case c4 on the C4 fixture's parameters: its
    01_ParticleTimehistory.plt against the reference's unit 11."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "c4_oscillate.npz"))
    _run(["--case", "c4", "--nx", "40", "--ny", "30", "--lc", "10", "--ret", "10", "--tc", "40",
          "--chunk", "64"], tmp_path)
    hist = _table(tmp_path / "01_ParticleTimehistory.plt")
    ref = g["UNIT11"]
    assert hist.shape == ref.shape
    np.testing.assert_allclose(hist[:, 0], ref[:, 0], rtol=1e-15)
    scale = np.max(np.abs(ref[:, 1:]))
    assert np.max(np.abs(hist[:, 1:] - ref[:, 1:])) <= 1e-9 * scale
    dens = _table(tmp_path / "01_AveragedDensity.PLT")
    np.testing.assert_allclose(dens, g["UNIT8"], rtol=1e-12)
