"""Build liblbm2d.so (the CUDA library behind include/lbm2d.h) in-tree.

Every translation unit is compiled for sm_100a only.  The FP64 lattice
kernel and the particle kernel are built with --fmad=false so that their
arithmetic follows the reference operation by operation; the FP32 kernel
keeps fused multiply-adds.

    python -m 2d_nnf_lbm_b200.build        (or build() from Python)
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblbm2d.so")
BUILD_DIR = os.path.join(HERE, "_build")
# the checked build: every computed index of the step, particle and batch
# kernels checked against its buffer (LBM_CHECKED, lbm_checked_build() == 1)
CHECKED_OUT = os.path.join(HERE, "liblbm2d_checked.so")
CHECKED_BUILD_DIR = os.path.join(HERE, "_build_checked")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
          "--expt-relaxed-constexpr"]

SOURCES = {
    "lbm_fp64.cu": ["--fmad=false"],
    "lbm_fp32.cu": ["--fmad=true"],
    "lbm_particles.cu": ["--fmad=false"],
    "lbm_api.cu": [],
    "lbm_adjoint.cu": ["--fmad=true"],
    "lbm_noalloc.cu": ["--fmad=false"],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, out: str = OUT,
          build_dir: str = BUILD_DIR, defines: tuple = (), driver: bool = True) -> str:
    """Compile and link; ``defines`` (e.g. ("LBM_MINB_F32=6",)) tune launch
    bounds, ``out``/``build_dir`` place a variant elsewhere."""
    os.makedirs(build_dir, exist_ok=True)
    dflags = [f"-D{d}" for d in defines]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "lbm2d.h"))
    objs = []
    logs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s, *headers, __file__]):
            cmd = [nvcc(), *ARCH, *COMMON, *dflags, *extra, "-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            logs.append(r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(out, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", out, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    # the C++ driver that mirrors the reference's MAIN on the C ABI
    drv_src = os.path.join(HERE, "driver", "lbm_main.cpp")
    drv = os.path.join(os.path.dirname(out), "lbm_main")
    if driver and os.path.exists(drv_src) and (force or _stale(drv, [drv_src, out, *headers])):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(HERE, "..", "include"),
               drv_src, "-L", os.path.dirname(out), "-l:" + os.path.basename(out),
               "-Wl,-rpath,$ORIGIN", "-o", drv]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("driver build failed")
    with open(os.path.join(build_dir, "ptxas.log"), "a") as fh:
        fh.write("".join(logs))
    if verbose:
        print("".join(logs))
    return out


def build_checked(verbose: bool = False, force: bool = False) -> str:
    """liblbm2d_checked.so beside liblbm2d.so (no driver of its own)."""
    return build(verbose, force, CHECKED_OUT, CHECKED_BUILD_DIR, ("LBM_CHECKED",), driver=False)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
