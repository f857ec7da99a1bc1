/*
 * lbm_oracle.h -- CPU oracle for the 2D_NNF_LBM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a single-threaded FP64 restatement of
 * the reference Fortran time step, routine by routine, in the reference's
 * own loop structure (per-particle full-lattice PHI arrays, O(Np*N) SPM and
 * force loops, the F_POST copy).  It is the checker for the CUDA library
 * and the timed CPU baseline; nothing in the product links or calls it.
 *
 * Parity pin: the reference Fortran cannot be compiled in this image (no
 * gfortran/flang).  The restatement is pinned against golden vectors that
 * tests/golden/make_golden.py produces by executing the reference's own
 * C1, C6 and C3 sources (PARAMETERs shrunk in memory; the STOP at C3:202
 * skipped) with the Fortran-subset translator tests/golden/f90run.py.  The
 * oracle reproduces all four fixtures bit for bit
 * (tests/test_oracle_golden.py).  Shared by translator and oracle, and so
 * not independently checked: the reading of gfortran's arithmetic (REAL(4)
 * literals, promotion, no contraction) and the zero start of the stale
 * D_PW local.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>
#include "../include/lbm2d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_opts {
    /* 0: each node relaxes with its own omega from the previous step
     *    (the parallel semantics of the CUDA path);
     * 1: the reference's sequential chain -- Collision_MRT calls
     *    ComputeRelaxation_MRT(OMEGA_BN(I,J)) which rewrites the global
     *    OMEGA_MRT that the NEXT node in sweep order uses (C6:958, C6:890). */
    int32_t omega_chain;
    /* 0: PHI stored per particle over the full lattice (C1:76, C3:79);
     * 1: PHI recomputed on the fly in each loop (same arithmetic, O(N) memory). */
    int32_t phi_on_the_fly;
    /* value of the uninitialised D_PW on the first call in STALE mode */
    double stale_dpw_init;
} oracle_opts;

typedef struct oracle oracle;

int  oracle_create(const lbm_params* p, const oracle_opts* o, oracle** out);
void oracle_destroy(oracle* o);
int  oracle_set_particles(oracle* o, int32_t np, const double* pin);
int  oracle_step(oracle* o, int32_t nsteps);
int64_t oracle_kk(const oracle* o);
int  oracle_get_particles(oracle* o, double* out);           /* np*LBM_POUT */
int  oracle_get_field(oracle* o, int32_t which, double* out); /* LBM_FIELD_* */
int  oracle_get_image(oracle* o, int32_t* out);
/* F(0:8,0:NX,0:NY) after boundary conditions of the last step */
int  oracle_get_f(oracle* o, double* out);
/* post-collision populations of the next step (what the CUDA state holds) */
int  oracle_get_next_post_collision(oracle* o, double* out, double* omega_out);
int  oracle_get_series(oracle* o, double* out, int32_t max_records, int32_t* nrec);
int  oracle_series_record_len(const oracle* o);
double oracle_mean_density(oracle* o);
/* COMPUTEERROR: ||u - u_prev|| / ||u||, then u_prev = u (C1:1592-1612) */
int  oracle_compute_error(oracle* o, double* er);
/* the reference's full particle state incl. VP_OLD (np*LBM_STATE_PER) */
int  oracle_get_state_particles(oracle* o, double* out);

/* Tangent build only (liblbm_oracle_tangent.so: the same source compiled as
 * C++ with -DORACLE_TANGENT, every real a value and its derivative): a run
 * that carries the derivative with respect to one input, which = one of
 * ORACLE_SEED_* (disk: the disk of rho_p, x0, y0).  Every other entry point
 * behaves as in the ordinary build and returns the same values;
 * oracle_get_particles_tangent returns the derivatives of what
 * oracle_get_particles returns. */
enum { ORACLE_SEED_TAU_Y = 0, ORACLE_SEED_NU = 1, ORACLE_SEED_RHO_P = 2, ORACLE_SEED_X0 = 3,
       ORACLE_SEED_Y0 = 4 };
int  oracle_create_tangent(const lbm_params* p, const oracle_opts* o, int32_t which,
                           int32_t disk, oracle** out);
int  oracle_get_particles_tangent(oracle* o, double* out); /* np*LBM_POUT */

#ifdef __cplusplus
}
#endif
#endif
