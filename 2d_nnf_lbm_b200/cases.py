"""Parameter sets and particle inputs of the reference cases and workloads.

``shipped_*`` reproduce the PARAMETER arithmetic of the reference programs
exactly as the compiled Fortran evaluates it (REAL(4) literals, left-to-right
evaluation), so a run with them is the reference case.  ``workload_*`` are the
benchmark workloads (the same programs with their PARAMETERs edited to the
workload sizes); their particle inputs are seeded and synthetic.
"""

from __future__ import annotations

import numpy as np

from .lbm2d import (
    LBM_BC_EQUILIBRIUM,
    LBM_BC_HALFWAY_BB,
    LBM_BINGHAM,
    LBM_CONTACT_DPP,
    LBM_CONTACT_STALE_DPW,
    LBM_FP64,
    LBM_MOTION_OSCILLATE,
    LBM_NEWTONIAN,
    LBM_PIN,
    LBM_RATES_FIXED_Q,
    LBM_RATES_Q_OF_OMEGA,
    LBM_WALL_MIRROR,
    LBM_WALL_NONE,
    LBM_WALL_OFFSET,
    LbmParams,
    glowinski_cij,
    mirror_edges,
    r4,
    r4div,
)


# ---- particle input file (0_Particle_Initial_Position.txt) -----------------
def read_particle_file(path: str, n: int, ncols: int) -> np.ndarray:
    """List-directed READ(200,*) of ``n`` records with ``ncols`` values each.

    Mirrors C1:170-175 (x y D rho_p) and C3:145-150 (x y): values are
    separated by blanks, tabs or commas; blank records (the leading tab line
    of the multi-particle file) and CR characters are skipped; a record may
    carry more values than read, which are ignored.
    """
    with open(path, "rb") as fh:
        text = fh.read().decode("ascii", errors="strict")
    rows = []
    for line in text.replace("\r", "").split("\n"):
        toks = line.replace(",", " ").split()
        if not toks:
            continue
        vals = [float(t.replace("d", "e").replace("D", "E")) for t in toks]
        # list-directed input continues onto the next record when short
        if rows and len(rows[-1]) < ncols:
            rows[-1].extend(vals)
            rows[-1] = rows[-1][:ncols]
        else:
            rows.append(vals[:ncols])
        if len(rows) == n and len(rows[-1]) == ncols:
            break
    if len(rows) < n or len(rows[-1]) < ncols:
        raise ValueError(f"{path}: expected {n} records of {ncols} values, got {len(rows)}")
    return np.asarray(rows[:n], dtype=np.float64)


def pin_array(xy, diam, rho_p, uvw=None, angle=None) -> np.ndarray:
    xy = np.asarray(xy, dtype=np.float64).reshape(-1, 2)
    n = xy.shape[0]
    pin = np.zeros((n, LBM_PIN))
    pin[:, 0:2] = xy
    if angle is not None:
        pin[:, 2] = angle
    if uvw is not None:
        pin[:, 3:6] = np.asarray(uvw, dtype=np.float64).reshape(n, 3)
    pin[:, 6] = diam
    pin[:, 7] = rho_p
    return pin


# ---- shipped reference cases -----------------------------------------------
def shipped_c1(nx: int = 240, ny: int = 720, diam: float = 30.0) -> LbmParams:
    """1_Disk_Newtonian (C1:2-93); CIJ uses DISK(1)%DIAM from the input file."""
    p = LbmParams(nx=nx, ny=ny)
    mirror_edges(p)
    p.c_ij = glowinski_cij(r4(1.25), 1.0, p.gravity, p.pi, diam)
    return p


def c1_time_max() -> int:
    """TIME_MAX = INT(1.0/C_T) of C1:35."""
    c_l = r4(0.25) / 30.0
    c_t = (c_l * c_l) * r4(0.05) / r4(0.1)
    return int(1.0 / c_t)


def shipped_c6(nx: int = 80, ny: int = 300) -> tuple[LbmParams, np.ndarray]:
    """6_FreeFall_YieldStress (C6:2-83, C6:161-169); returns params and the disk."""
    p = LbmParams(nx=nx, ny=ny)
    nu = r4(0.025)
    rho_s, rho_f = 2.0, 1.0
    re_s, bn_s = r4(0.78), r4(0.033)
    l_c = float(nx // 4)
    a_g = -(re_s * nu * nu / ((l_c * l_c * l_c) * (rho_s - rho_f) * rho_f))
    tau_y = bn_s * (rho_s - rho_f) * (-a_g) * l_c
    p.nu = nu
    p.bc = LBM_BC_HALFWAY_BB
    p.rheology = LBM_BINGHAM
    p.rate_set = LBM_RATES_Q_OF_OMEGA
    p.s_e, p.s_eps = r4(1.1), 1.25
    p.wall_model = LBM_WALL_OFFSET
    p.contact_test = LBM_CONTACT_STALE_DPW
    p.integrate_angle = 1
    p.gravity = a_g
    p.tau_y = tau_y
    p.m_pap = r4(5.5e6)
    p.zeta = 1.0
    p.rep_zeta = 1.0
    p.eps_p = 0.5
    p.eps_w = p.eps_p
    p.e_p = 10.0
    p.e_w = p.e_p
    p.c_ij = glowinski_cij(rho_s, rho_f, a_g, p.pi, l_c)
    disk = pin_array([[0.5 * float(nx), float(ny) - 7.0 * l_c]], l_c, rho_s)
    return p, disk


def shipped_c2(nx: int = 200, ny: int = 800, l_c: float = 20.0,
               a_g: float | None = None) -> tuple[LbmParams, np.ndarray]:
    """2_DKT_Newtonian (C2:2-88, C2:128-144): two disks D = L_C, rho_p =
    RHO_S = 1.01, at the coded (1/C_L, 7.2/C_L) and (0.97/C_L, 6.8/C_L) with
    C_L = DIAM_PHYSICAL/L_C; half-way bounce-back with the oscillating-wall
    amplitude at its shipped zero (C2:1224-1230), Glowinski repulsion with
    offset walls and the stale D_PW test (C2:735-780), rates 1.1 / 1.25 /
    q(omega) (C2:1029), angle integration (C2:321).  A_G = -9.81/C_G
    (C2:33) unless given; returns params and the two disks."""
    p = LbmParams(nx=nx, ny=ny)
    nu = r4(0.05)
    rho_s = r4(1.01)
    c_l = r4(0.2) / l_c
    if a_g is None:
        c_t = (c_l * c_l) * nu / r4(0.01)
        c_g = c_l * r4(0.01) / (c_t * c_t)
        a_g = -r4(9.81) / c_g
    p.nu = nu
    p.bc = LBM_BC_HALFWAY_BB
    p.rheology = LBM_NEWTONIAN
    p.rate_set = LBM_RATES_Q_OF_OMEGA
    p.s_e, p.s_eps = r4(1.1), 1.25
    p.wall_model = LBM_WALL_OFFSET
    p.contact_test = LBM_CONTACT_STALE_DPW
    p.integrate_angle = 1
    p.gravity = a_g
    p.zeta = 1.0
    p.rep_zeta = 1.0
    p.eps_p = p.eps_w = 1.0
    p.e_p = p.e_w = 20.0
    p.c_ij = glowinski_cij(rho_s, 1.0, a_g, p.pi, l_c)
    xy = [[r4(1.0) / c_l, r4(7.2) / c_l], [r4(0.97) / c_l, r4(6.8) / c_l]]
    return p, pin_array(xy, l_c, rho_s)


def shipped_c4(nx: int = 1500, ny: int = 1000, l_c: float = 50.0, re_t: float = 100.0,
               t_c: float | None = None) -> tuple[LbmParams, np.ndarray]:
    """4_Oscillating_Particle (C4:2-93, C4:197-214): a cylinder D = L_C,
    rho_p = RHO_S = 1, at the centre, driven at u = -U_C cos(2 PI KK/T_C)
    (C4:226), equilibrium boundary on every edge (C4:1219-1275), rates
    1.6 / 1.8 / q(omega) (C4:1018), no gravity.  U_C = RE_T*NU/L_C (C4:30),
    T_C = 5*L_C/U_C (C4:32) unless given; returns params and the disk."""
    p = LbmParams(nx=nx, ny=ny)
    nu = r4(0.025)
    u_c = re_t * nu / l_c
    if t_c is None:
        t_c = 5.0 * l_c / u_c
    p.nu = nu
    p.bc = LBM_BC_EQUILIBRIUM
    p.rate_set = LBM_RATES_Q_OF_OMEGA
    p.s_e, p.s_eps = r4(1.6), r4(1.8)
    p.gravity = 0.0
    p.wall_model = LBM_WALL_NONE
    p.motion = LBM_MOTION_OSCILLATE
    p.osc_u, p.osc_period = u_c, t_c
    p.zeta = 1.0
    disk = pin_array([[0.5 * float(nx), 0.5 * float(ny)]], l_c, 1.0, uvw=[[-u_c, 0.0, 0.0]])
    return p, disk


def shipped_c3(nx: int = 512, ny: int = 512) -> LbmParams:
    """3_MultiParticle_Sedimentation (C3:2-83): D = L_C = 16, RHO_P = RHO_S."""
    p = LbmParams(nx=nx, ny=ny)
    nu = r4div(0.4915, 3.0)
    rho_s = r4(1.01)
    c_l = r4(0.0625) / 16.0
    c_t = (c_l * c_l) * nu / r4(0.01)
    c_g = c_l * r4(0.01) / (c_t * c_t)
    a_g = -r4(9.81) / c_g
    p.nu = nu
    p.bc = LBM_BC_HALFWAY_BB
    p.rheology = LBM_NEWTONIAN
    p.rate_set = LBM_RATES_Q_OF_OMEGA
    p.s_e, p.s_eps = r4(1.1), 1.25
    p.wall_model = LBM_WALL_OFFSET
    p.contact_test = LBM_CONTACT_STALE_DPW
    p.integrate_angle = 0
    p.gravity = a_g
    p.zeta = 1.0
    p.rep_zeta = 1.0
    p.eps_p = 2.0
    p.eps_w = 0.5 * p.eps_p
    p.e_p = 20.0
    p.e_w = 0.5 * p.e_p
    p.c_ij = glowinski_cij(rho_s, 1.0, a_g, p.pi, 16.0)
    return p


# ---- benchmark workloads ------------------------------------------------------
# cfg1: gravity tuned once on the FP64 oracle (tests/golden/make_cfg1.py --tune)
# so that the particle Reynolds number Re_p = rho_p*D*|v|/NU of C1:261
# peaks at about 20 during the fall (19.96, at step ~7170, just before the
# bottom wall slows the disk); frozen here as a constant.
CFG1_GRAVITY = -5.125e-4


def workload_cfg1(precision: int = LBM_FP64) -> tuple[LbmParams, np.ndarray]:
    """Plain method, small: the C1 program at 200x600, D=24 at (100,480),
    rho_p/rho_f=1.5, tau=0.8, SPM thickness 2, history every 10 steps."""
    p = shipped_c1(200, 600, 24.0)
    p.precision = precision
    p.nu = r4((0.8 - 0.5) / 3.0)
    p.zeta = 2.0
    p.gravity = CFG1_GRAVITY
    p.c_ij = glowinski_cij(1.5, 1.0, p.gravity, p.pi, 24.0)
    p.series_every = 10
    p.series_particles = 1
    disk = pin_array([[100.0, 480.0]], 24.0, 1.5)
    return p, disk


CFG2_GRAVITY = -5.0e-5


def workload_cfg2_particles(nx=1024, ny=2048, n=512, diam=16.0, gap=2.0, seed=0):
    """Seeded non-overlapping uniform positions in the upper half.

    x in [R+zeta, NX-R-zeta], y in [NY/2+R+zeta, NY-R-zeta], pairwise
    distance >= D+zeta, rho_p ~ U[1.01, 1.5] from the same generator.  The
    shape follows the 504-disk input of the multi-particle case (C3:145-156).
    """
    rng = np.random.default_rng(seed)
    r = 0.5 * diam
    lo = np.array([r + gap, 0.5 * ny + r + gap])
    hi = np.array([nx - r - gap, ny - r - gap])
    pts = []
    cell = diam + gap
    grid = {}
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > 200000 * n:
            raise RuntimeError("could not place particles")
        c = lo + rng.random(2) * (hi - lo)
        gx, gy = int(c[0] // cell), int(c[1] // cell)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for q in grid.get((gx + dx, gy + dy), ()):
                    if (pts[q][0] - c[0]) ** 2 + (pts[q][1] - c[1]) ** 2 < cell * cell:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            grid.setdefault((gx, gy), []).append(len(pts))
            pts.append(c)
    rho = 1.01 + rng.random(n) * (1.5 - 1.01)
    return pin_array(np.asarray(pts), diam, rho)


def workload_cfg2(precision: int, nx=1024, ny=2048, n=512, seed=0) -> tuple[LbmParams, np.ndarray]:
    """Multi-particle sedimentation: the C3 program at 1024x2048 with 512 disks
    of D=16, repulsion range 2, tau=0.7."""
    p = shipped_c3(nx, ny)
    p.precision = precision
    p.nu = r4((0.7 - 0.5) / 3.0)
    p.gravity = CFG2_GRAVITY
    p.rep_zeta = 2.0
    p.contact_test = LBM_CONTACT_DPP
    p.c_ij = glowinski_cij(1.25, 1.0, p.gravity, p.pi, 16.0)
    p.series_every = 10
    p.series_particles = n
    pin = workload_cfg2_particles(nx, ny, n, 16.0, 2.0, seed)
    return p, pin


def workload_cfg3(precision: int, bn: float, nx=800, ny=2400, diam=40.0) -> tuple[LbmParams, np.ndarray, dict]:
    """Viscoplastic settling: the C6 program at 800x2400, D=40, rho_p=2,
    tau_p=0.9, m=1e5, Bingham number Bn.

    Gravity and the velocity scale follow C6:27-29 with L_C = D:
    A_G = -RE_S*NU^2/(L_C^3 (rho_s-rho_f) rho_f), U_REF = L_C^2 (rho_s-rho_f)(-A_G)/NU,
    and Bn = TAU_Y*L_C/(NU*U_REF) (the BnT column of C6:317), so
    TAU_Y = Bn*NU*U_REF/L_C.
    """
    p, _ = shipped_c6(nx, ny)
    p.precision = precision
    nu = r4((0.9 - 0.5) / 3.0)
    rho_s = 2.0
    re_s = r4(0.78)
    a_g = -(re_s * nu * nu / ((diam ** 3) * (rho_s - 1.0) * 1.0))
    u_ref = diam * diam * (rho_s - 1.0) * (-a_g) / nu
    p.nu = nu
    p.gravity = a_g
    p.tau_y = bn * nu * u_ref / diam
    p.m_pap = 1.0e5
    p.c_ij = glowinski_cij(rho_s, 1.0, a_g, p.pi, diam)
    p.series_every = 10
    disk = pin_array([[0.5 * nx, float(ny) - 7.0 * diam]], diam, rho_s)
    return p, disk, {"u_ref": u_ref, "bn": bn}


def workload_cfg5(precision: int, bn: float = 5.0, nx=400, ny=1200, diam=24.0,
                  rho_s=1.5) -> tuple[LbmParams, np.ndarray, dict]:
    """Adjoint workload: the C6 program at 400x1200, one disk D=24 rho_p=1.5,
    tau_p=0.9, m=1e5, Bingham number Bn; the objective is the disk's mean v_y
    over steps 3000..4000.  Gravity, velocity scale and Bn follow the
    viscoplastic-settling workload: A_G = -RE_S*NU^2/(D^3 (rho_s-1)),
    U_REF = D^2 (rho_s-1)(-A_G)/NU, TAU_Y = Bn*NU*U_REF/D."""
    p, _ = shipped_c6(nx, ny)
    p.precision = precision
    nu = r4((0.9 - 0.5) / 3.0)
    re_s = r4(0.78)
    a_g = -(re_s * nu * nu / ((diam ** 3) * (rho_s - 1.0) * 1.0))
    u_ref = diam * diam * (rho_s - 1.0) * (-a_g) / nu
    p.nu = nu
    p.gravity = a_g
    p.tau_y = bn * nu * u_ref / diam
    p.m_pap = 1.0e5
    p.c_ij = glowinski_cij(rho_s, 1.0, a_g, p.pi, diam)
    disk = pin_array([[0.5 * nx, float(ny) - 7.0 * diam]], diam, rho_s)
    return p, disk, {"u_ref": u_ref, "bn": bn, "n0": 3000, "n1": 4000}


def workload_cfg4(precision: int, n: int = 256, seed: int = 0, tau_p: float = 0.9):
    """Batched persistent solves: n independent Bingham single-disk settling
    runs (the C6 program), seeded: width W ~ U[128, 512] lu (integer), height
    3W, disk D = W/10 at (W/2, 3W - 7D), Bn log-uniform in [0.1, 100],
    rho_p ~ U[1.2, 3.0], tau_p = 0.9, m = 1e5; gravity, U_REF and TAU_Y per
    run as in the viscoplastic-settling workload (L_C = D).  Returns a list
    of (params, disks)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w = int(rng.integers(128, 513))
        bn = float(10.0 ** rng.uniform(-1.0, 2.0))
        rho_s = float(rng.uniform(1.2, 3.0))
        diam = w / 10.0
        p, _ = shipped_c6(w, 3 * w)
        p.precision = precision
        nu = r4((tau_p - 0.5) / 3.0)
        re_s = r4(0.78)
        a_g = -(re_s * nu * nu / ((diam ** 3) * (rho_s - 1.0) * 1.0))
        u_ref = diam * diam * (rho_s - 1.0) * (-a_g) / nu
        p.nu = nu
        p.gravity = a_g
        p.tau_y = bn * nu * u_ref / diam
        p.m_pap = 1.0e5
        p.c_ij = glowinski_cij(rho_s, 1.0, a_g, p.pi, diam)
        disk = pin_array([[0.5 * w, 3.0 * w - 7.0 * diam]], diam, rho_s)
        out.append((p, disk))
    return out


def mlups(nodes: int, steps: int, seconds: float) -> float:
    return nodes * steps / seconds / 1e6


def nodes_of(p: LbmParams) -> int:
    return (p.nx + 1) * (p.ny + 1)


__all__ = [
    "read_particle_file",
    "pin_array",
    "shipped_c1",
    "shipped_c3",
    "shipped_c6",
    "c1_time_max",
    "workload_cfg1",
    "workload_cfg2",
    "workload_cfg2_particles",
    "workload_cfg3",
    "workload_cfg4",
    "workload_cfg5",
    "mlups",
    "nodes_of",
]
