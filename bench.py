#!/usr/bin/env python
"""Throughput of the hot path in MLUPS on one B200 (or N independent replicas).

Workload (default): multi-particle sedimentation, 1024x2048 cells
(1025x2049 = 2,100,225 nodes), 512 disks of diameter 16 at seeded
non-overlapping positions in the upper half, density ratios U[1.01, 1.5],
repulsion range 2, tau = 0.7, FP32 shifted populations; the plain FP64 path
is timed on the same workload beside it.  One bench step = one time step of
the whole lattice and all particles.  The per-step working set (two 76 MB
population sweeps in FP32, 151 MB in FP64) exceeds the 126 MB L2, so no
extra flush is needed between steps.

Arms:
  (default)          the CUDA library through its C ABI
  --impl reference   the reference's algorithm on the host cores: the CPU
                     oracle, a C restatement of the Fortran time step with
                     its loop structure (the Fortran itself cannot be built
                     in this image), single-threaded as the reference is

Objects of the JSON line beside the headline (N=1; --parts selects them):
  trajectory_err  FP32 against FP64 on the bench workload over the
                  multi-particle configuration's 50,000 steps
  viscoplastic    the viscoplastic-settling workload (800x2400, one Bingham
                  disk D=40, Bn in {0.5, 2, 10, 50}, 100,000 steps): terminal
                  v_y and yielded/unyielded field of FP32 against FP64, and
                  the Bingham step's MLUPS
  adjoint         lbm_adjoint on the adjoint workload (400x1200, one Bingham
                  disk, 4000 steps, sqrt(N) checkpoints) against the forward
                  time loop; gradients against FP64 central differences
  batch           lbm_batch_step on 256 independent Bingham single-disk runs
                  of uneven sizes against the same runs one after another

--profile-run CASE runs one workload for a few steps with no timing around
it, for ncu captures of single launches: step-fp32 / step-fp64 (the bench
workload), visco (the viscoplastic workload at Bn = 2, FP32), adjoint (the
adjoint workload, objective over the last 100 steps),
batch (the first --batch-sims runs of the batched workload on the
TMA-staged batched kernel).

Multi-GPU: the hot path does not shard (one simulation, one GPU); --gpus N
runs N independent replicas (weak scaling), timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_NODE = {0: 144.0, 1: 72.0}  # FP64 plain / FP32 shifted, Newtonian
BINGHAM_BYTES_PER_NODE = {0: 160.0, 1: 80.0}  # + per-node omega read and written
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) of one k_step<float> launch of the bench workload,
# from ncu (dram__bytes_read.sum + dram__bytes_write.sum, one launch, cold);
# captured with `ncu --set full -k regex:k_step -s 5 -c 1` on
# `python bench.py --profile-run step-fp32 --steps 30` (summary under profiles/)
K_STEP_FP32_TRAFFIC = {"bytes": 112485888.0, "captured_at": "0e24264"}
PARTS = ("fp32", "fp64", "e2e", "trajectory", "viscoplastic", "adjoint", "batch", "cpu")


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--parts", default="all",
                    help="comma list of " + ",".join(PARTS) + " (default all; fp32 always runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint/forward time measurement")
    ap.add_argument("--batch-steps", type=int, default=20000,
                    help="steps of the 256-simulation batch measurement (0: skip)")
    ap.add_argument("--batch-seq-steps", type=int, default=1000,
                    help="steps of each run alone (the sequential comparison)")
    ap.add_argument("--batch-sims", type=int, default=256)
    ap.add_argument("--accuracy-steps", type=int, default=50000,
                    help="steps of the FP32-vs-FP64 trajectory comparison (0: skip)")
    ap.add_argument("--visco-steps", type=int, default=100000,
                    help="steps of each viscoplastic-settling run (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="target CPU time of the bounded oracle sample")
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--particles", type=int, default=512)
    ap.add_argument("--profile-run", default="",
                    choices=["", "step-fp32", "step-fp64", "visco", "adjoint", "batch"])
    a = ap.parse_args(argv)
    parts = set(PARTS) if a.parts == "all" else {s.strip() for s in a.parts.split(",") if s.strip()}
    unknown = parts - set(PARTS)
    if unknown:
        ap.error(f"unknown parts: {sorted(unknown)}")
    if a.no_cpu_baseline:
        parts.discard("cpu")
    if a.no_adjoint:
        parts.discard("adjoint")
    if a.batch_steps <= 0:
        parts.discard("batch")
    if a.accuracy_steps <= 0:
        parts.discard("trajectory")
    if a.visco_steps <= 0:
        parts.discard("viscoplastic")
    parts.add("fp32")
    a.part_set = parts
    return a


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # the GPU work starts once nvidia-smi is sampling (two lines written):
        # its start-up (driver and NVML initialisation, slower on a host
        # with many GPUs) then lies before the warm-up, not inside a short
        # timed region
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            with open(self.path) as fh:
                if sum(1 for _ in fh) >= 2:
                    break
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in rows if num(r[3]) is not None]
        thr = 0.5 * max(pw) if pw else 0.0
        load = [num(r[1]) for r in rows if num(r[3]) is not None and num(r[3]) >= thr]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {
            "sm_mhz": statistics.median(load or sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons,
            "samples": len(rows),
            "power_w_max": max(pw) if pw else None,
        }


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload(pkg, precision, args):
    p, pin = pkg.cases.workload_cfg2(precision, args.nx, args.ny, args.particles)
    p.series_capacity = 1024
    return p, pin


def time_steps(pkg, torch, sim, k):
    ext = torch.cuda.ExternalStream(sim.stream())
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(ext)
    sim.step(k)
    t1.record(ext)
    t1.synchronize()
    return t0.elapsed_time(t1)


def reduce_max(dist, torch, value, device):
    """Max of a per-rank number over all ranks (a replica job takes as long
    as its slowest rank); ``device`` is where the backend reduces: cuda:N for
    NCCL, cpu for gloo."""
    if dist is None:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world, nodes, steps, ms_max):
    """Whole-job MLUPS of `world` replicas that each update `nodes` nodes
    `steps` times, the slowest in `ms_max` milliseconds (weak scaling)."""
    return world * nodes * steps / (ms_max * 1e-3) / 1e6


def run_gpu_path(pkg, torch, args, precision, device, world, dist, clocks=False):
    """Time args.steps steps of the bench workload with CUDA events on the
    library's stream (state resident in HBM).  The step kernel and the
    particle kernel of each step overlap (programmatic dependent launch), so
    the step kernel's launches run back to back and their average duration
    in the timed region is the timed region over the steps.  A second,
    identical pass with events between the launches (which serialises them)
    gives each kernel's own duration."""
    p, pin = workload(pkg, precision, args)
    p.device = device
    sim = pkg.Simulation(p)
    sim.set_particles(pin)
    # the clock sampler starts first (it takes ~0.3 s): the warm-up steps run
    # after that idle gap, and the timed steps right after them
    sampler = ClockSampler(device) if clocks else None
    if sampler:
        sampler.start()
    sim.step(args.warmup)
    sim.series()
    if dist is not None:
        dist.barrier()
    ms = time_steps(pkg, torch, sim, args.steps)
    clk = sampler.stop() if sampler else None
    ms = reduce_max(dist, torch, ms, f"cuda:{device}")
    status = sim.status()
    sim.profile(True)
    sim.step(args.steps)
    (pms, lms), (pn, ln) = sim.profile_read()
    sim.profile(False)
    sim.series()
    parts = sim.particles()
    sim.close()
    nodes = (p.nx + 1) * (p.ny + 1)
    return {
        "ms": ms, "nodes": nodes, "lattice_ms_serialised": lms / max(ln, 1),
        "particle_ms_serialised": pms / max(pn, 1),
        "launches": 2 * args.steps, "clocks": clk, "status": status,
        "finite": bool(np.all(np.isfinite(parts[:, :6]))),
    }


E2E_CHUNK = 256  # steps between drains of the device history ring


def run_e2e(pkg, torch, args, device):
    """Same metric through the public API with host buffers: the disks set
    from pinned host memory, then the time loop with every step's history
    record -- per disk x, y, angle, u, v, omega, FORCE, F_H_IN, and the mean
    density, what the reference writes every step (C1:264, C1:318) -- copied
    to host memory: the library keeps the records in a device ring and
    lbm_get_series drains them every E2E_CHUNK steps, each chunk's records
    read while the next chunk runs.  The device ring holds two chunks, so the
    chunk that runs writes other slots than the one whose records are
    crossing to the host (a one-chunk ring makes every chunk's first step
    wait for the previous chunk's copy)."""
    p, pin = workload(pkg, 1, args)
    p.device = device
    p.series_every = 1
    p.series_particles = pin.shape[0]
    p.series_capacity = 2 * E2E_CHUNK
    sim = pkg.Simulation(p)
    pin_h = torch.from_numpy(pin).pin_memory().numpy()
    sim.set_particles(pin_h)
    sim.step(args.warmup)
    sim.series()
    ext = torch.cuda.ExternalStream(sim.stream())
    # the host buffer the records land in is the caller's, allocated once
    # before the time loop (pinned, so the drains copy straight into it)
    rec_len = sim.series_record_len()
    out = torch.empty((E2E_CHUNK, rec_len), dtype=torch.float64).pin_memory().numpy()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    k = args.steps
    chunks = [min(E2E_CHUNK, k - s0) for s0 in range(0, k, E2E_CHUNK)]
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    t0.record(ext)
    sim.set_particles(pin_h)
    sim.step(chunks[0])
    for i, c in enumerate(chunks):
        if i + 1 < len(chunks):
            sim.step(chunks[i + 1])  # queued before this chunk's records are read
        got = 0
        while got < c:
            got += sim.series_into(out[got:c])
    t1.record(ext)
    t1.synchronize()
    wall = time.perf_counter() - w0
    ms = t0.elapsed_time(t1)
    sim.close()
    nodes = (p.nx + 1) * (p.ny + 1)
    return {
        "value": nodes * k / (ms * 1e-3) / 1e6,
        "unit": "MLUPS",
        "h2d_bytes_per_step": pin.nbytes / k,
        # the record and its fixed-point mean-density sum
        "d2h_bytes_per_step": int(rec_len * 8 + 8),
        "wall_s": wall,
        "output": f"every step's history record ({rec_len} doubles), drained every "
                  f"{E2E_CHUNK} steps",
    }


def trajectory_error(pkg, args, device, steps):
    """FP32-shifted against FP64 plain on the bench workload, outside the
    timed region, at milestones up to `steps` steps (the multi-particle
    configuration runs 50,000): the largest disk displacement error
    relative to the largest FP64 displacement, and the same for the velocity
    (the FP64 path matches the oracle within 1e-10 on the parity cases).
    Control: a second FP64 run whose only change is the disks' initial
    centres rounded to FP32 (what a single-precision input file would hold);
    its departure from the first FP64 run is the suspension's own
    sensitivity to a perturbation of that size."""
    sims = {}
    pin = None
    for prec in (1, 0, "ctl"):
        p, pin = workload(pkg, 0 if prec == "ctl" else prec, args)
        p.device = device
        p.series_every = 0
        sims[prec] = pkg.Simulation(p)
        if prec == "ctl":
            q = pin.copy()
            q[:, 0:2] = q[:, 0:2].astype(np.float32).astype(np.float64)
            sims[prec].set_particles(q)
        else:
            sims[prec].set_particles(pin)
    marks = sorted({m for m in (2000, 10000, 20000, 30000, 40000, steps) if m <= steps})
    tiny = 1e-300
    at = []
    done = 0
    for m in marks:
        for s in sims.values():
            s.step(m - done)
        done = m
        r32, r64 = sims[1].particles(), sims[0].particles()
        d32, d64 = r32[:, 0:2] - pin[:, 0:2], r64[:, 0:2] - pin[:, 0:2]
        v32, v64 = r32[:, 3:5], r64[:, 3:5]
        dmax = max(float(np.max(np.linalg.norm(d64, axis=1))), tiny)
        vmax = max(float(np.max(np.linalg.norm(v64, axis=1))), tiny)
        ed = np.linalg.norm(d32 - d64, axis=1) / dmax
        ev = np.linalg.norm(v32 - v64, axis=1) / vmax
        rc = sims["ctl"].particles()
        ec = np.linalg.norm(rc[:, 0:2] - r64[:, 0:2], axis=1) / dmax
        at.append({
            "steps": m,
            "max_rel_displacement_err": float(ed.max()),
            "rms_rel_displacement_err": float(np.sqrt(np.mean(ed ** 2))),
            "max_rel_velocity_err": float(ev.max()),
            "rms_rel_velocity_err": float(np.sqrt(np.mean(ev ** 2))),
            "max_fp64_displacement": float(np.max(np.linalg.norm(d64, axis=1))),
            "control_max_rel_displacement_err": float(ec.max()),
            "control_rms_rel_displacement_err": float(np.sqrt(np.mean(ec ** 2))),
            "status": [sims[1].status(), sims[0].status(), sims["ctl"].status()],
        })
    for s in sims.values():
        s.close()
    last = at[-1]
    return {
        "steps": steps,
        "max_rel_displacement_err": last["max_rel_displacement_err"],
        "rms_rel_displacement_err": last["rms_rel_displacement_err"],
        "max_rel_velocity_err": last["max_rel_velocity_err"],
        "errors_relative_to": "the largest FP64 displacement (speed) over all disks",
        "tolerance": 1e-4,
        "within_tolerance": bool(last["max_rel_displacement_err"] <= 1e-4 and
                                 last["max_rel_velocity_err"] <= 1e-4),
        "rms_within_tolerance": bool(last["rms_rel_displacement_err"] <= 1e-4),
        "control": "FP64 with the initial centres rounded to FP32, against FP64",
        "control_max_rel_displacement_err": last["control_max_rel_displacement_err"],
        "control_rms_rel_displacement_err": last["control_rms_rel_displacement_err"],
        "milestones": at,
    }


VISCO_BN = (0.5, 2.0, 10.0, 50.0)


def visco_measure(pkg, torch, device, steps, mlups_steps=4000):
    """The viscoplastic-settling workload for each Bingham number: one FP32
    and one FP64 run of `steps` steps (history every 10 steps, stress and
    yield flags kept), compared by the disk's terminal v_y (mean over the
    last tenth of the run) and by the yielded/unyielded flag of every fluid
    node at the end (C6:947-954); then the Bingham step's MLUPS (80 B/node
    FP32, 160 B/node FP64; no stress planes) over `mlups_steps` steps."""
    cases = []
    chunk = 10000
    for bn in VISCO_BN:
        res = {}
        for prec in (1, 0):
            p, pin, info = pkg.cases.workload_cfg3(prec, bn)
            p.device = device
            p.record_stress = 1
            p.series_every = 10
            p.series_particles = 1
            p.series_capacity = chunk // 10 + 8
            sim = pkg.Simulation(p)
            sim.set_particles(pin)
            hist = []
            done = 0
            while done < steps:
                c = min(chunk, steps - done)
                sim.step(c)
                done += c
                hist.append(sim.series())
            h = np.concatenate(hist)
            img = sim.image()
            parts = sim.particles()
            res[prec] = {"vy": h[:, 2 + 4], "y": h[:, 2 + 1], "img": img, "p": parts,
                         "status": sim.status(), "u_ref": info["u_ref"], "tau_y": p.tau_y}
            sim.close()
        n = len(res[0]["vy"])
        tail = slice(n - max(1, n // 10), n)
        v32, v64 = float(np.mean(res[1]["vy"][tail])), float(np.mean(res[0]["vy"][tail]))
        fluid = (res[0]["img"] != 10) & (res[1]["img"] != 10)
        y32, y64 = res[1]["img"] == 5, res[0]["img"] == 5
        agree = float(np.mean((y32 == y64)[fluid]))
        traj = float(np.max(np.abs(res[1]["y"] - res[0]["y"])))
        cases.append({
            "bn": bn, "tau_y": res[0]["tau_y"], "u_ref": res[0]["u_ref"],
            "terminal_vy_fp64": v64, "terminal_vy_fp32": v32,
            "terminal_vy_over_u_ref_fp64": v64 / res[0]["u_ref"],
            "terminal_vy_rel_err": abs(v32 - v64) / max(abs(v64), 1e-300),
            "max_abs_y_err": traj,
            "final_y_fp64": float(res[0]["p"][0, 1]), "final_y_fp32": float(res[1]["p"][0, 1]),
            "unyielded_frac_fp64": float(np.mean(y64[fluid])),
            "unyielded_frac_fp32": float(np.mean(y32[fluid])),
            "yield_flag_agreement": agree,
            "status": [res[1]["status"], res[0]["status"]],
        })
    # Bingham step throughput (no stress planes: the 80 / 160 B/node kernel)
    rate = {}
    for prec in (1, 0):
        p, pin, _ = pkg.cases.workload_cfg3(prec, 2.0)
        p.device = device
        p.series_every = 10
        p.series_capacity = 1024
        sim = pkg.Simulation(p)
        sim.set_particles(pin)
        sim.step(20)
        sim.series()
        ms = time_steps(pkg, torch, sim, mlups_steps)
        sim.series()
        sim.close()
        nodes = (p.nx + 1) * (p.ny + 1)
        rate["fp32" if prec else "fp64"] = {
            "mlups": nodes * mlups_steps / (ms * 1e-3) / 1e6,
            "ms_per_step": ms / mlups_steps,
            "bytes_per_node": BINGHAM_BYTES_PER_NODE[prec],
            "achieved_gbs": BINGHAM_BYTES_PER_NODE[prec] * nodes / (ms / mlups_steps * 1e-3) / 1e9,
        }
    return {
        "workload": "viscoplastic settling 800x2400 (1,923,201 nodes), one Bingham disk D=40 "
                    "rho_p=2, tau_p=0.9, m=1e5, Bn = tau_y D/(nu U_ref), "
                    "U_ref = D^2 (rho_p-1)|g|/nu, |g| from RE_S=0.78 as C6:27-29",
        "steps": steps, "cases": cases, "step_rate": rate,
        "terminal_window": "mean v_y over the last tenth of the run",
        "tolerance": 1e-4,
    }


def adjoint_measure(pkg, torch, device):
    """The adjoint workload (400x1200 lattice, one disk D=24, Bn=5, 4000
    steps, J = mean v_y over steps 3000..4000, sqrt(N) = 63 checkpoints):
    wall time of lbm_adjoint against the forward time loop, both timed with
    CUDA events on the handle's stream (the adjoint call synchronises
    internally, so its interval is its wall time), FP32 and FP64; the FP32
    gradient against the FP64 adjoint and against FP64 central differences
    (relative step 1e-4) of the GPU forward."""
    out = {}
    res = {}
    for prec in (1, 0):
        p, pin, info = pkg.cases.workload_cfg5(prec)
        p.device = device
        n0, n1 = info["n0"], info["n1"]

        def timed(fn):
            sim = pkg.Simulation(p)
            sim.set_particles(pin)
            ext = torch.cuda.ExternalStream(sim.stream())
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(ext)
            r = fn(sim)
            e1.record(ext)
            e1.synchronize()
            sim.close()
            return e0.elapsed_time(e1), r

        timed(lambda s: s.adjoint(n0, n1))  # buffers allocated, code paged in
        fwd = min(timed(lambda s: s.step(n1))[0] for _ in range(2))
        adj, (j, g) = min((timed(lambda s: s.adjoint(n0, n1)) for _ in range(2)),
                          key=lambda t: t[0])
        res[prec] = (j, g)
        out["fp32" if prec else "fp64"] = {"fwd_ms": fwd, "adjoint_ms": adj,
                                           "adjoint_over_fwd": adj / fwd}
    p64, pin, info = pkg.cases.workload_cfg5(0)
    p64.device = device
    n0, n1 = info["n0"], info["n1"]

    def run_j(q, disks):
        sim = pkg.Simulation(q)
        sim.set_particles(disks)
        sim.step(n0 - 1)
        v = []
        for _ in range(n0, n1 + 1):
            sim.step(1)
            v.append(sim.particles()[0, 4])
        sim.close()
        return float(np.mean(v))

    # central differences: parameters at a relative step of 1e-4; the
    # release point at 1e-4 of the disk diameter (a step relative to the
    # coordinate itself, 0.1 lu at y0 = 1032, would measure how the disk
    # sits on the lattice, not the derivative), and again at half that step
    fd, fd_half = {}, {}
    names = ("tau_y", "nu", "rho_p", "x0", "y0")
    col = {"rho_p": 7, "x0": 0, "y0": 1}

    def central(name, d):
        base = {"tau_y": p64.tau_y, "nu": p64.nu}.get(name, None)
        if base is None:
            base = float(pin[0, col[name]])
        jj = []
        for sgn in (1.0, -1.0):
            q = p64.copy()
            disks = np.array(pin, copy=True)
            if name == "tau_y":
                q.tau_y = base + sgn * d
            elif name == "nu":
                q.nu = base + sgn * d
            else:
                disks[0, col[name]] = base + sgn * d
            jj.append(run_j(q, disks))
        return (jj[0] - jj[1]) / (2 * d)

    for name in names:
        if name in ("x0", "y0"):
            d = 1e-4 * float(pin[0, 6])
            fd[name] = central(name, d)
            fd_half[name] = central(name, 0.5 * d)
        else:
            base = {"tau_y": p64.tau_y, "nu": p64.nu, "rho_p": float(pin[0, 7])}[name]
            fd[name] = central(name, 1e-4 * abs(base))
    j32, g32 = res[1]
    j64, g64 = res[0]
    pick = lambda g, k: float(g[k] if k in ("tau_y", "nu") else g[k][0])  # noqa: E731
    # dJ/dx0 vanishes by symmetry (the disk starts on the vertical centre
    # line): it is judged against the scale of dJ/dy0, the others relatively
    rel = [k for k in fd if k != "x0"]
    scale_x = abs(fd["y0"])
    out.update({
        "workload": "Bingham settling 400x1200 (481,601 nodes), disk D=24 rho_p=1.5, Bn=5, "
                    "tau_p=0.9, m=1e5, 4000 steps, J = mean v_y over steps 3000..4000",
        "checkpoint_every": int(round(n1 ** 0.5)),
        "J": j32,
        "grad_fp32": {k: pick(g32, k) for k in fd},
        "grad_fp64": {k: pick(g64, k) for k in fd},
        "fd_fp64": fd,
        "fd_fp64_half_step": fd_half,
        "fd_step": "1e-4 relative (tau_y, nu, rho_p); 1e-4 * D for x0, y0",
        "max_rel_err_fp32_vs_fd": max(abs(pick(g32, k) - fd[k]) / abs(fd[k]) for k in rel),
        "max_rel_err_fp64_vs_fd": max(abs(pick(g64, k) - fd[k]) / abs(fd[k]) for k in rel),
        "max_rel_err_fp32_vs_fp64_adjoint": max(abs(pick(g32, k) - pick(g64, k)) /
                                                abs(pick(g64, k)) for k in rel),
        "x0_abs_err_over_dJdy0": {
            "fp32_vs_fd": abs(pick(g32, "x0") - fd["x0"]) / scale_x,
            "fp64_vs_fd": abs(pick(g64, "x0") - fd["x0"]) / scale_x,
        },
        "tolerance": 1e-3,
    })
    return out


def batch_measure(pkg, torch, device, steps, seq_steps, nsim=256):
    """The batched workload (256 seeded Bingham single-disk runs, widths
    128..512, heights 3x, FP32): one lbm_batch_step of `steps` steps (after
    the tuning steps) against each run alone through lbm_step for
    `seq_steps` steps (the per-step rate of a run alone is steady after its
    warm-up, so its time for `steps` steps is scaled from those); CUDA events
    on the batch's / each handle's stream."""
    cs = pkg.cases.workload_cfg4(1)[:nsim]
    for p, _ in cs:
        p.device = device
    nodes = [(p.nx + 1) * (p.ny + 1) for p, _ in cs]
    b = pkg.Batch([p for p, _ in cs])
    for s, (_, pin) in zip(b.sims, cs):
        s.set_particles(pin)
    b.step(12)  # tuning (9 timed steps) and the first graph capture
    ext = torch.cuda.ExternalStream(b.batch_stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ext)
    b.step(steps)
    e1.record(ext)
    e1.synchronize()
    batch_ms = e0.elapsed_time(e1)
    tuning = b.tuning()
    finite = all(np.all(np.isfinite(s.particles())) for s in b.sims)
    status = max(abs(s.status()) for s in b.sims)
    b.close()
    alone = []
    for p, pin in cs:
        sim = pkg.Simulation(p)
        sim.set_particles(pin)
        sim.step(12)
        ext = torch.cuda.ExternalStream(sim.stream())
        torch.cuda.synchronize()
        e0.record(ext)
        sim.step(seq_steps)
        e1.record(ext)
        e1.synchronize()
        alone.append(e0.elapsed_time(e1) * steps / seq_steps)
        sim.close()
    alone = np.array(alone)
    total = float(np.sum(nodes)) * steps
    return {
        "workload": f"{len(cs)} Bingham single-disk runs (C6), W ~ U[128,512], H = 3W, D = W/10, "
                    "Bn log-uniform [0.1,100], rho_p ~ U[1.2,3], tau_p 0.9, m 1e5, seed 0, FP32",
        "simulations": len(cs), "nodes": int(np.sum(nodes)), "steps": steps,
        "tile": list(tuning[:2]), "blocks_per_sm": tuning[2],
        "batch_ms": batch_ms, "batch_mlups": total / (batch_ms * 1e-3) / 1e6,
        "roofline_frac_80B": total / (batch_ms * 1e-3) * 80.0 / 1e9 / hbm_peak()[0],
        "per_sim_wall_ms_batched": batch_ms,
        "sequential_ms": float(np.sum(alone)),
        "sequential_mlups": total / (float(np.sum(alone)) * 1e-3) / 1e6,
        "sequential_measured_steps": seq_steps,
        "alone_ms_p50": float(np.percentile(alone, 50)), "alone_ms_p99": float(np.percentile(alone, 99)),
        "speedup_vs_sequential": float(np.sum(alone)) / batch_ms,
        "finite": bool(finite), "status": -status,
    }


def host_cpu():
    model = platform.processor() or "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return model, os.cpu_count() or 0


def cpu_baseline(pkg, args, seconds):
    """The oracle (reference loop structure, one thread) on the same workload,
    timed over a bounded number of whole time steps."""
    from oracle.oracle import Oracle

    p, pin = workload(pkg, 0, args)
    nodes = (p.nx + 1) * (p.ny + 1)
    need = 8 * nodes * (len(pin) + 40)
    avail = 0
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    on_the_fly = 1 if avail and avail < 1.5 * need else 0
    o = Oracle(p, phi_on_the_fly=on_the_fly)
    o.set_particles(pin)
    t = time.perf_counter()
    o.step(1)
    first = time.perf_counter() - t
    n = max(1, min(50, int(seconds / max(first, 1e-3))))
    t = time.perf_counter()
    o.step(n)
    dt = time.perf_counter() - t
    o.close()
    model, ncpu = host_cpu()
    return {
        "value": nodes * n / dt / 1e6,
        "unit": "MLUPS",
        "cores": 1,
        "host_cpu": model,
        "host_nproc": ncpu,
        "kind": "port",
        "sample": (f"{n} full time steps of the {args.nx}x{args.ny}, {len(pin)}-disk workload "
                   f"after 1 untimed step ({dt:.1f} s); PHI "
                   + ("recomputed per loop (host memory)" if on_the_fly else
                      "stored per particle over the lattice as in the reference")),
    }


L2_BYTES = 126e6


def l2_note(nodes):
    """How a step's working set compares with the 126 MB L2 (no flush
    between steps, so a bench line needs the larger)."""
    w32, w64 = BYTES_PER_NODE[1] * nodes, BYTES_PER_NODE[0] * nodes
    rel = ">" if w32 > L2_BYTES else "<"
    tail = "; no flush" if w32 > L2_BYTES else "; no flush (smaller than L2: a small case)"
    return (f"working set per step {w32 / 1e6:.0f} MB (fp32) / {w64 / 1e6:.0f} MB (fp64) "
            f"{rel} 126 MB L2{tail}")


def main():
    args = parse_args()
    world, rank, local = dist_env()
    pkg = importlib.import_module("2d_nnf_lbm_b200")
    nodes = (args.nx + 1) * (args.ny + 1)
    cfg = {
        "workload": (f"multi-particle sedimentation {args.nx}x{args.ny} lattice "
                     f"({nodes} nodes), {args.particles} disks D=16, tau=0.7, repulsion 2 lu"),
        "nodes": nodes, "particles": args.particles, "precision": "fp32-shifted (fp64 beside)",
        "l2": l2_note(nodes),
        "parallelism": f"replicas x{world}",
    }
    metric = f"MLUPS (FP32-shifted, multi-particle {args.nx}x{args.ny}, {args.particles} disks)"

    if args.impl == "reference":
        if rank != 0:
            return
        base = cpu_baseline(pkg, args, args.cpu_seconds)
        line = {
            "impl": "reference", "metric": metric, "value": base["value"], "unit": "MLUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    import torch

    if args.profile_run:
        return profile_run(pkg, args)

    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = tdist
    device = local if world > 1 else 0
    parts = args.part_set

    r32 = run_gpu_path(pkg, torch, args, 1, device, world, dist, clocks=True)
    r64 = run_gpu_path(pkg, torch, args, 0, device, world, dist) if "fp64" in parts else None
    e2e = run_e2e(pkg, torch, args, device) if "e2e" in parts else None
    if dist is not None and e2e is not None:
        e2e["value"] = world / reduce_max(dist, torch, 1.0 / e2e["value"], f"cuda:{device}")

    peak, peak_src = hbm_peak()
    # the step kernel's average launch duration in the timed region: its
    # launches run back to back (the particle kernel overlaps them), so it is
    # the timed region over the steps
    kms32 = r32["ms"] / args.steps
    ach32 = BYTES_PER_NODE[1] * r32["nodes"] / (kms32 * 1e-3) / 1e9
    value = job_mlups(world, r32["nodes"], args.steps, r32["ms"])
    line = {
        "metric": metric,
        "value": value,
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": kms32,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic",
        "config": cfg,
        "roofline": {
            "bound": "hbm",
            "achieved": ach32,
            "peak": peak,
            "unit": "GB/s",
            "frac": ach32 / peak,
            "traffic": K_STEP_FP32_TRAFFIC["bytes"],
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                               "k_step<float> launch of this workload, captured at commit "
                               + K_STEP_FP32_TRAFFIC["captured_at"]),
            "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
            else "fallback 6.65 TB/s",
            "bytes_per_node": BYTES_PER_NODE[1],
            "kernel": "k_step<float>",
            "kernel_ms": kms32,
            "kernel_ms_source": "timed region / steps (launches back to back, CUDA events "
                                "on the library stream)",
            "kernel_ms_serialised": r32["lattice_ms_serialised"],
            "particle_kernel_ms_serialised": r32["particle_ms_serialised"],
            "serialised_source": "an identical pass with CUDA events between the launches, "
                                 "which serialises the step and particle kernels",
        },
        "gpu_launches": r32["launches"],
        "clocks": r32["clocks"],
        "status": {"fp32": r32["status"], "finite": r32["finite"]},
    }
    if r64 is not None:
        kms64 = r64["ms"] / args.steps
        ach64 = BYTES_PER_NODE[0] * r64["nodes"] / (kms64 * 1e-3) / 1e9
        value64 = job_mlups(world, r64["nodes"], args.steps, r64["ms"])
        line["fp64"] = {
            "value": value64, "unit": "MLUPS", "ms_per_step": kms64,
            "roofline_frac": ach64 / peak, "achieved_gbs": ach64,
            "kernel_ms_serialised": r64["lattice_ms_serialised"],
            "bytes_per_node": BYTES_PER_NODE[0],
        }
        line["fp32_over_fp64"] = value / value64
        line["status"]["fp64"] = r64["status"]
        line["status"]["finite"] = r32["finite"] and r64["finite"]
    if e2e is not None:
        line["e2e"] = {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step",
                                           "d2h_bytes_per_step")}
        line["e2e"]["output"] = e2e["output"]
    if world == 1 and "trajectory" in parts:
        line["trajectory_err"] = trajectory_error(pkg, args, device, args.accuracy_steps)
    if world == 1 and "viscoplastic" in parts:
        line["viscoplastic"] = visco_measure(pkg, torch, device, args.visco_steps)
    if world == 1 and "adjoint" in parts:
        line["adjoint"] = adjoint_measure(pkg, torch, device)
    if world == 1 and "batch" in parts:
        line["batch"] = batch_measure(pkg, torch, device, args.batch_steps, args.batch_seq_steps,
                                      args.batch_sims)
    if rank == 0 and world == 1 and "cpu" in parts:
        line["cpu_baseline"] = cpu_baseline(pkg, args, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def profile_run(pkg, args):
    """A short run of one workload with no timing around it (ncu captures)."""
    if args.profile_run == "adjoint":
        p, pin, _ = pkg.cases.workload_cfg5(1)
        with pkg.Simulation(p) as sim:
            sim.set_particles(pin)
            j, g = sim.adjoint(max(1, args.steps - 100), args.steps)
            print(f"steps {sim.kk}  J {j:.9e}  dJ/dtau_y {g['tau_y']:.9e}  status {sim.status()}")
        return 0
    if args.profile_run == "batch":
        cs = pkg.cases.workload_cfg4(1)[: args.batch_sims]
        b = pkg.Batch([q for q, _ in cs])
        b.set_tuning(64, 8, 2)  # the TMA-staged batched tiles
        for s, (_, disks) in zip(b.sims, cs):
            s.set_particles(disks)
        b.step(args.steps)
        parts = b.sims[0].particles()
        print(f"steps {b.sims[0].kk}  run 0 disk at ({parts[0, 0]:.6f}, {parts[0, 1]:.6f})  "
              f"status {max(abs(s.status()) for s in b.sims)}")
        b.close()
        return 0
    if args.profile_run == "visco":
        p, pin, _ = pkg.cases.workload_cfg3(1, 2.0)
        with pkg.Simulation(p) as sim:
            sim.set_particles(pin)
            sim.step(args.steps)
            parts = sim.particles()
            print(f"steps {sim.kk}  disk at ({parts[0, 0]:.6f}, {parts[0, 1]:.6f})  "
                  f"status {sim.status()}")
        return 0
    prec = 1 if args.profile_run == "step-fp32" else 0
    p, pin = workload(pkg, prec, args)
    with pkg.Simulation(p) as sim:
        sim.set_particles(pin)
        sim.step(args.steps)
        parts = sim.particles()
        print(f"steps {sim.kk}  disk 0 at ({parts[0, 0]:.6f}, {parts[0, 1]:.6f})  "
              f"status {sim.status()}")
    return 0


if __name__ == "__main__":
    main()
