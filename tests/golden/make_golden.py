"""Generate the golden fixtures that pin the CPU oracle to the reference.

Runs the reference's own Fortran programs (read from the reference tree,
parameters shrunk in memory) through tests/golden/f90run.py and stores the
state they reach as .npz files beside this script:

    python tests/golden/make_golden.py [--reference PATH]

Cases (every run is the unmodified main program and subroutines of the file
named; only PARAMETERs and the particle input file are replaced, and in the
c1_bgk cases the collision call of the main program, as described there):

  c1_center  1_Disk_Newtonian (C1), NX=24 NY=40, one disk D=8 rho_p=1.25 at
             (12, 28), 40 steps: Zou-He walls, MRT, SPM coupling, Newton-Euler
  c1_walls   C1 as above with the disk at (19.02, 4.98), 20 steps: the
             mirror-image repulsion of the bottom and right walls (range
             branch; C1's contact stiffness throws a penetrating disk out of
             a lattice this small)
  c6_bingham 6_FreeFall_YieldStress (C6), NX=24 NY=60 (L_C = NX/4 = 6, the
             disk at its coded start (12, 18)), 30 steps: half-way
             bounce-back, Papanastasiou viscosity with the node-to-node omega
             chain, rate set q(omega), angle integration
  c1_nonnewt C1 as c1_center with its non-Newtonian branch switched on
             (NON_NEWTONIAN=.TRUE.): Papanastasiou viscosity with the strain
             rate of C1:896-948 (m_neq against COMPUTEFEQNEW's moments) and
             the node-to-node omega chain
  c1_bgk     C1 as c1_center with its main program calling COLLISION
             (C1:774-841, the single-relaxation BGK routine) in place of
             Collision_MRT: the call the program carries commented out at
             C1:295 is switched in and the Collision_MRT call of C1:296 is
             skipped; nothing else changes
  c1_bgk_biviscous  c1_bgk with NON_NEWTONIAN=.TRUE. and TAU_Y=1.0D-5:
             COLLISION's bi-viscosity branch (GAMMA_C = TAU_Y/(MU_R - MU_0),
             MU_R = 1000 MU_0), about a third of the nodes unyielded at the
             last step
  c1_error   C1 at NX=16 NY=24 with the disk at (8, 14), D=6, 2000 steps:
             the reference's COMPUTEERROR values at steps 1000 and 2000 (unit 7)
  c3_casson  C3 as c3_multi with its non-Newtonian branch switched on
             (NON_NEWTONIAN=.TRUE., Y_g=0.5): the regularised Casson
             viscosity of C3:978-996 with the node-to-node omega chain
  c2_dkt     2_DKT_Newtonian (C2), NX=30 NY=112, L_C=3 (the two disks D=3 at
             the coded (1/C_L, 7.2/C_L) and (0.97/C_L, 6.8/C_L)), A_G=-5E-4,
             40 steps: half-way bounce-back, offset-wall repulsion with the
             stale D_PW test, rates 1.1/1.25/q(omega), angle integration
  c4_oscillate  4_Oscillating_Particle (C4), NX=40 NY=30, L_C=10 (the disk
             D=10 at the centre), RE_T=10 (U_C=0.025), T_C=40 (the loop runs
             INT(6*T_C)=240 steps): prescribed u=-U_C*cos(2*PI*KK/T_C),
             equilibrium boundary on every edge, rate set 1.6/1.8/q(omega)
  c3_multi   3_MultiParticle_Sedimentation (C3), NX=48 NY=72, N_PARTICLE=3
             (D = L_C = 16), 20 steps: pair repulsion including the stale
             D_PW contact test.  The STOP at C3:202, which ends the shipped
             program before its time loop, is skipped.

Each file holds the final populations F (after the boundary conditions of
the last step), UX/UY (corrected), RHO, G, OMEGA_BN (C6), the particle
records and every record the program wrote to its history units.
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import f90run  # noqa: E402

STUBS = ["WRITERESULTS", "WRITE_DOMAINIMAGE", "WRITEIMAGE", "RESULTSPROFILE",
         "WRITE_RESULTSPROFILE"]

CASES = {
    "c1_center": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                      overrides={"NX": "24", "NY": "40", "TIME_MAX": "40"},
                      particles="12\t28\t8\t1.25", steps=40),
    "c1_walls": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                     overrides={"NX": "24", "NY": "40", "TIME_MAX": "20"},
                     particles="19.02\t4.98\t8\t1.25", steps=20),
    "c1_nonnewt": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                       overrides={"NX": "24", "NY": "40", "TIME_MAX": "40", "NON_NEWTONIAN": ".TRUE."},
                       particles="12\t28\t8\t1.25", steps=40),
    "c1_bgk": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                   overrides={"NX": "24", "NY": "40", "TIME_MAX": "40"},
                   particles="12\t28\t8\t1.25", steps=40,
                   edits={295: ("!CALL COLLISION(", "CALL COLLISION(")}, skip_lines=[296]),
    "c1_bgk_biviscous": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                             overrides={"NX": "24", "NY": "40", "TIME_MAX": "40",
                                        "NON_NEWTONIAN": ".TRUE.", "TAU_Y": "1.0D-5"},
                             particles="12\t28\t8\t1.25", steps=40,
                             edits={295: ("!CALL COLLISION(", "CALL COLLISION(")},
                             skip_lines=[296]),
    "c1_error": dict(file="1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90",
                     overrides={"NX": "16", "NY": "24", "TIME_MAX": "2000"},
                     particles="8\t14\t6\t1.25", steps=2000),
    "c6_bingham": dict(file="6_FreeFall_YieldStress/D2Q9_BinghamSediment_Validated_20191127.f90",
                       overrides={"NX": "24", "NY": "60", "TIME_MAX": "30"},
                       particles=None, steps=30),
    "c3_casson": dict(file="3_MultiParticle_Sedimentation/D2Q9_RTParticle_20191003.f90",
                      overrides={"NX": "48", "NY": "72", "TIME_MAX": "20", "N_PARTICLE": "3",
                                 "NON_NEWTONIAN": ".TRUE.", "Y_g": "0.5"},
                      particles="\t\n14\t50\n30.6\t50\n24\t22\n", steps=20, skip_lines=[202]),
    "c2_dkt": dict(file="2_DKT_Newtonian/D2Q9_DKT_Validated_20190926.f90",
                   overrides={"NX": "30", "NY": "112", "L_C": "3.0", "TIME_MAX": "40",
                              "A_G": "-5.0E-4"},
                   particles=None, steps=40),
    "c4_oscillate": dict(file="4_Oscillating_Particle/D2Q9_V7_OscillatingCylinder_Validated.f90",
                         overrides={"NX": "40", "NY": "30", "L_C": "10.0", "RE_T": "10.0",
                                    "T_C": "40.0"},
                         particles=None, steps=240),
    "c3_multi": dict(file="3_MultiParticle_Sedimentation/D2Q9_RTParticle_20191003.f90",
                     overrides={"NX": "48", "NY": "72", "TIME_MAX": "20", "N_PARTICLE": "3"},
                     particles="\t\n14\t50\n30.6\t50\n24\t22\n", steps=20, skip_lines=[202]),
}

PARTICLE_FIELDS = ["CENTER", "VELOCITY", "FORCE", "F_COL", "DIAM", "RHO_P", "M_P", "I_P", "ANGLE"]


def run_case(ref_root, name, spec):
    src = open(os.path.join(ref_root, spec["file"]), encoding="latin-1").read()
    lines = src.split("\n")
    for ln, (old, new) in spec.get("edits", {}).items():  # 1-based line numbers
        if old not in lines[ln - 1]:
            raise SystemExit(f"{name}: line {ln} does not hold {old!r}")
        lines[ln - 1] = lines[ln - 1].replace(old, new, 1)
    src = "\n".join(lines)
    files = {"0_Particle_Initial_Position.txt": spec["particles"]} if spec["particles"] else {}
    t0 = time.time()
    frame, io, prog = f90run.run_program(src, overrides=spec["overrides"], files=files, stubs=STUBS,
                                         skip_lines=spec.get("skip_lines", ()))
    n_used = int(getattr(prog.M, "N_PARTICLE"))
    out = {"steps": np.int64(spec["steps"]), "kk": np.int64(frame["KK"])}
    for k in ("F", "UX", "UY", "RHO", "G", "OMEGA_BN", "DOMAIN_IMAGE"):
        if k in frame:
            out[k] = np.asarray(frame[k])
    for k in ("VP_OLD", "F_H_IN"):  # (1:3, 1:N) per-particle work arrays; (1:3) in C4
        if k in frame:
            v = np.asarray(frame[k])
            out[k] = (v[:, None] if v.ndim == 1 else v)[:, :n_used]
    disks = frame["DISK"][:n_used]  # the main program may declare more than it uses
    for fld in PARTICLE_FIELDS:
        if hasattr(disks[0], fld):
            out["DISK_" + fld] = np.array([np.asarray(getattr(d, fld), dtype=np.float64) for d in disks])
    for unit, recs in io.items():
        recs = [r for r in recs if r]
        if recs and len({len(r) for r in recs}) == 1:
            out[f"UNIT{unit}"] = np.array(recs, dtype=np.float64)
    for k, v in spec["overrides"].items():
        out["PARAM_" + k] = np.array(v)
    print(f"{name}: {time.time() - t0:.1f} s, KK={frame['KK']}, units {sorted(io)}")
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LBM_REFERENCE_DIR"),
                    help="root of the reference project (or LBM_REFERENCE_DIR)")
    ap.add_argument("--case", action="append")
    a = ap.parse_args(argv)
    if not a.reference:
        ap.error("give --reference or set LBM_REFERENCE_DIR")
    for name, spec in CASES.items():
        if a.case and name not in a.case:
            continue
        out = run_case(a.reference, name, spec)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    main()
