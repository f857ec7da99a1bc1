"""C ABI checks that need no GPU: symbols, struct layout, parameter defaults,
argument validation that happens before any CUDA call."""

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbm2d.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load_library()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_struct_matches_header_and_defaults(pkg):
    lib = pkg.load_library()
    p = pkg.LbmParams()
    q = pkg.LbmParams()
    ctypes.memset(ctypes.byref(q), 0, ctypes.sizeof(q))
    assert lib.lbm_params_init(ctypes.byref(q)) == 0
    assert q.struct_size == ctypes.sizeof(pkg.LbmParams)
    # the C defaults and the Python mirror hold the same Fortran-evaluated constants
    for name, _ in pkg.LbmParams._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if name == "w_init":
            assert list(a) == list(b)
        else:
            assert a == b, (name, a, b)


def test_fortran_real4_literals(pkg):
    p = pkg.LbmParams()
    assert p.pi == 3.1415927410125732          # PI=3.14159265359 (C1:3)
    assert p.nu == 0.05000000074505806         # NU=0.05 (C1:23)
    assert p.d_mrt == 0.027777777984738350     # d_mrt=1./36. (C1:881)
    assert p.inv_six == 0.16666667163372040    # Inv_Six=1.0/6.0 (C1:1229)
    assert p.s_e == 1.100000023841858          # omega_e=1.1 (C1:1040)
    assert p.gamma_min == 1.0000000036274937e-15  # 1.0E-15 (C6:939)
    # per-collision mass factor 36*d_mrt of the reference
    assert 36.0 * p.d_mrt - 1.0 == pytest.approx(7.450580596923828e-09, rel=1e-12)


def _create(pkg, p):
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    return lib.lbm_create(ctypes.byref(p), ctypes.byref(h))


def test_create_validation_without_device(pkg):
    p = pkg.LbmParams()
    p.struct_size = 8
    assert _create(pkg, p) == -10  # LBM_E_ABI
    assert _create(pkg, pkg.LbmParams(nu=-0.1)) == -2  # LBM_E_TAU, C1:127-130
    assert _create(pkg, pkg.LbmParams(nx=1)) == -1
    assert _create(pkg, pkg.LbmParams(precision=7)) == -1
    assert _create(pkg, pkg.LbmParams(bc=5)) == -1
    assert _create(pkg, pkg.LbmParams(nu=float("nan"))) == -1


def test_null_arguments(pkg):
    lib = pkg.load_library()
    assert lib.lbm_create(None, None) == -1
    assert lib.lbm_destroy(None) == -1
    assert lib.lbm_step(None, 1) == -1
    assert lib.lbm_params_init(None) == -1
    assert lib.lbm_strerror(-2) == b"relaxation time exceeded 0.5 -> stability problem"


def test_simulation_requires_library(pkg, monkeypatch):
    # no silent fallback: a missing library raises instead of computing on the CPU
    monkeypatch.setattr(pkg.lbm2d, "_LIB", None)
    monkeypatch.setattr(pkg.lbm2d, "library_path", lambda: "/nonexistent/liblbm2d.so")
    with pytest.raises(OSError):
        pkg.lbm2d.load_library()


def test_record_layout_constants(pkg):
    src = open(HEADER).read()
    for name, val in [("LBM_PIN", 8), ("LBM_POUT", 16), ("LBM_STATE_PER", 20),
                      ("LBM_SERIES_HEAD", 2), ("LBM_SERIES_PER", 12)]:
        assert re.search(rf"#define {name} {val}\b", src), name
        assert getattr(pkg.lbm2d, name) == val
    assert np.dtype(np.float64).itemsize == 8


def test_fortran_module_mirrors_header(pkg):
    """include/lbm2d_mod.f90 binds every entry point and lays out LBM_PARAMS
    field by field as lbm_params (no Fortran compiler here, so by text)."""
    mod = open(os.path.join(ROOT, "include", "lbm2d_mod.f90")).read().upper()
    bound = set(n.lower() for n in re.findall(r"NAME='(LBM_[A-Z_0-9]+)'", mod))
    assert set(declared_functions()) == bound
    body = re.search(r"TYPE, BIND\(C\) :: LBM_PARAMS(.*?)END TYPE", mod, re.S).group(1)
    names = []
    for line in body.replace("&\n", " ").split("\n"):
        if "::" in line:
            for n in line.split("::", 1)[1].split(","):
                n = n.strip()
                m = re.match(r"([A-Z_0-9]+)(\((\d+)\))?", n)
                if m:
                    names += [m.group(1).lower()] * (1 if not m.group(3) else 1)
    fields = [f for f, _ in pkg.LbmParams._fields_]
    assert names == fields
