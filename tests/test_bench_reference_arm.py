"""bench.py --impl reference: the reference's algorithm (the oracle, one host
thread) on the bench's workload, printed as one JSON line with the same
metric, unit and direction as the GPU arm; under torchrun only rank 0 runs
it and the other ranks exit 0 without work.  Small lattice, so it runs on
the CPU in a second."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--nx", "64", "--ny", "128", "--particles", "4", "--cpu-seconds", "0.5",
         "--steps", "3", "--warmup", "3"]


def _run(extra_env):
    env = dict(os.environ)
    env.update(extra_env)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", *SMALL], cwd=ROOT,
                          env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "MLUPS (FP32-shifted, multi-particle 64x128, 4 disks)"
    assert d["unit"] == "MLUPS" and d["higher_is_better"] is True
    assert d["value"] > 0.0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 3, 3)
    assert d["config"]["nodes"] == 65 * 129 and d["config"]["particles"] == 4
    assert "smaller than L2" in d["config"]["l2"]
    base = d["cpu_baseline"]
    assert base["kind"] == "port" and base["cores"] == 1
    assert base["value"] == d["value"] and base["unit"] == "MLUPS"
    assert base["host_nproc"] >= 1 and base["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_output():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_l2_note_of_the_bench_workload():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.l2_note(1025 * 2049) == (
        "working set per step 151 MB (fp32) / 302 MB (fp64) > 126 MB L2; no flush")
