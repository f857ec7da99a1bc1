/*
 * lbm2d.h -- C ABI of the B200 (sm_100a) hot path of 2D_NNF_LBM.
 *
 * One handle = one simulation: a D2Q9 MRT lattice of (NX+1) x (NY+1) nodes
 * (nodes 0..NX, 0..NY, i fastest), rigid disks coupled by the smoothed
 * profile method (SPM), Glowinski soft-sphere repulsion and an explicit
 * Newton-Euler particle update.  The library owns all device memory; the
 * caller owns every host buffer it passes.  Every entry point returns
 * LBM_OK (0) or a negative LBM_E* code.  A handle is used by one host
 * thread at a time.  lbm_step() is asynchronous on the handle's own CUDA
 * stream; every lbm_get_* call synchronises that stream first.
 *
 * Reference interface replaced (the reference is a set of Fortran 90
 * programs; there is no FFI, the "interface" is the in-process subroutine
 * sequence of the time loop, cited per entry point below):
 *   1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90            (C1)
 *   6_FreeFall_YieldStress/D2Q9_BinghamSediment_Validated_20191127.f90 (C6)
 *   3_MultiParticle_Sedimentation/D2Q9_RTParticle_20191003.f90 (C3)
 * A Fortran driver binds these functions through ISO_C_BINDING; a ctypes
 * binding is used by the Python host layer and the tests.
 */
#ifndef LBM2D_H
#define LBM2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM2D_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
    LBM_OK = 0,
    LBM_E_INVALID = -1,   /* bad argument or parameter value                  */
    LBM_E_TAU = -2,       /* relaxation time 1/omega < 0.5 (C1:127-130)        */
    LBM_E_NOMEM = -3,     /* device or host allocation failed                 */
    LBM_E_CUDA = -4,      /* CUDA runtime error (no device, launch failure)   */
    LBM_E_NAN = -5,       /* non-finite density or particle state detected    */
    LBM_E_TIMEOUT = -6,   /* a bounded device-side wait gave up               */
    LBM_E_OVERFLOW = -7,  /* a fixed capacity exceeded: too many particles on
                             one lattice tile or near one particle, or (FP32)
                             a node's |rho - rho0| >= 2, beyond the range of
                             the mean-density sum                             */
    LBM_E_STATE = -8,     /* call out of order (e.g. step before particles)   */
    LBM_E_PARTICLE = -9,  /* particle outside the lattice, or input disks that
                             overlap (lbm_set_particles)                      */
    LBM_E_ABI = -10,      /* struct_size does not match this library          */
    LBM_E_SCRATCH = -11,  /* input larger than lbm_fields_noalloc's scratch   */
    LBM_E_BOUNDS = -12    /* checked build only: a kernel's index check failed
                             and the access was skipped                       */
};

/* ---- variant switches (compile-time PARAMETERs / IF(0|1) blocks upstream) */
enum { LBM_FP64 = 0,            /* plain populations in FP64 (drop-in)        */
       LBM_FP32_SHIFTED = 1 };  /* FP32 storage of f - w_i*rho0, FP32 math    */

enum { LBM_BC_ZOUHE = 0,        /* C1:1250-1258, C1:1341-1363 + corners        */
       LBM_BC_HALFWAY_BB = 1,   /* C6:1206-1219, C6:1285-1294 + corners        */
       LBM_BC_EQUILIBRIUM = 2   /* C4:1219-1275: every edge node takes the
                                   equilibrium of its inward neighbour's density
                                   and velocity of the previous step           */ };

enum { LBM_MOTION_FREE = 0,      /* Newton-Euler (C1:247-259)                   */
       LBM_MOTION_OSCILLATE = 1  /* prescribed u = -osc_u*cos(2*PI*kk/osc_period),
                                    v = w = 0 (C4:222-228); FORCE is still
                                    computed, F_H_IN from this step's change
                                    (C4:270-272)                               */ };

enum { LBM_NEWTONIAN = 0,
       LBM_BINGHAM = 1,         /* Papanastasiou-regularised, C6:913-958       */
       LBM_CASSON = 2 };        /* regularised Casson of the non-Newtonian
                                   branch of C2/C3 (C3:978-996): the strain
                                   rate and omega of LBM_BINGHAM, viscosity
                                   (sqrt(nu) + sqrt(tau_y/g)(1-exp(-sqrt(m g))))^2,
                                   sqrt(nu) + sqrt(m tau_y) at zero shear    */

enum { LBM_RATES_FIXED_Q = 0,   /* C1:1040-1042: s_q given                     */
       LBM_RATES_Q_OF_OMEGA = 1 /* C6:1009-1011: s_q = 8(2-w)/(8-w)            */ };

enum { LBM_STRAIN_MEQ = 0,       /* C6:903-922: m_neq against the moment-space
                                    equilibrium, forcing correction, then 1/rho */
       LBM_STRAIN_FEQ = 1 };     /* C1:896-948: m_neq against the moments of
                                    COMPUTEFEQNEW, 1/rho folded into both terms */

enum { LBM_COLLISION_MRT = 0,    /* Collision_MRT, C1:875-1048 / C6:867-1021     */
       LBM_COLLISION_BGK = 1 };  /* COLLISION, C1:774-841: single-relaxation BGK
                                    with ComputeSourceEquilib_Hydro's forcing
                                    (C1:843-870); with LBM_BINGHAM its
                                    bi-viscosity model (C1:789-809): shear rate
                                    sqrt(4|D12^2 - D11 D22|) from f - FEQ of
                                    the previous collision, nu = MU_R =
                                    1000 nu below GAMMA_C = tau_y/(MU_R - nu),
                                    else nu + tau_y/gamma (C1:51-53)        */

enum { LBM_WALL_MIRROR = 0,     /* C1:737-745: mirror-image wall particles     */
       LBM_WALL_OFFSET = 1,     /* C3:775-783, C6:717-725: wall disk at R out  */
       LBM_WALL_NONE = 2 };

enum { LBM_CONTACT_DPP = 0,       /* pair contact branch tests D_PP (intent)   */
       LBM_CONTACT_STALE_DPW = 1  /* tests the stale wall distance D_PW as the
                                     reference does (C1:721/724, C3:760/763)   */ };

/* ---- parameters -------------------------------------------------------- */
/* Every constant of MODULE PARAM that the hot path reads is a runtime field
 * here.  Values that Fortran evaluates as default-kind REAL(4) literals
 * (PI, 1./36., 1.0/6.0, 1.1, 1.2, 2./9., ...) are passed as the double the
 * Fortran program actually holds; lbm_params_init() fills them that way. */
typedef struct lbm_params {
    int32_t struct_size;      /* must equal sizeof(lbm_params)                 */
    int32_t nx;               /* NX, C1:8                                      */
    int32_t ny;               /* NY, C1:9                                      */
    int32_t precision;        /* LBM_FP64 | LBM_FP32_SHIFTED                   */
    int32_t bc;               /* LBM_BC_*                                      */
    int32_t rheology;         /* LBM_NEWTONIAN | LBM_BINGHAM                   */
    int32_t rate_set;         /* LBM_RATES_*                                   */
    int32_t wall_model;       /* LBM_WALL_*                                    */
    int32_t contact_test;     /* LBM_CONTACT_*                                 */
    int32_t integrate_angle;  /* 1: ANGLE += 0.5(w+w_old) (C6:312)             */
    int32_t series_every;     /* particle history cadence in steps (>= 1)      */
    int32_t series_particles; /* particles per history record (<= np)          */
    int32_t series_capacity;  /* records buffered on the device                */
    int32_t record_stress;    /* 1: keep stress / yield flag / omega fields    */
    int32_t device;           /* CUDA device ordinal                           */
    int32_t motion;           /* LBM_MOTION_*                                  */

    double nu;                /* NU (plastic viscosity Mu_0 for Bingham)       */
    double rho0;              /* RHO0, C1:57                                   */
    double s_e, s_eps, s_q;   /* MRT rates omega_e, omega_eps, omega_q         */
    double d_mrt;             /* d_mrt = 1./36. (C1:881)                       */
    double inv_six;           /* Inv_Six = 1.0/6.0 (C1:1229)                   */
    double w_init[3];         /* COMPUTEFEQNEW W0, W1, W2 (C1:1162-1164)       */
    double pi;                /* PI (C1:3)                                     */
    double zeta;              /* SPM interface thickness DISK%ZITA (C1:177)    */
    double gravity;           /* A_G (C1:45): v += (1-rho0/rho_p)*A_G          */
    double tau_y;             /* TAU_Y                                         */
    double m_pap;             /* M_PAP, Papanastasiou exponent                 */
    double gamma_min;         /* zero-shear guard 1.0E-15 (C6:939)             */
    double rep_zeta;          /* repulsion range ZITA (C1:701)                 */
    double eps_p, eps_w;      /* EPS_P, EPS_W                                  */
    double e_p, e_w;          /* E_P, E_W                                      */
    double c_ij;              /* CIJ = -(RHO_S-RHO_F)*A_G*PI*R^2 (C1:701)      */
    double wall_mirror_top;   /* 2*WALL%EDGE(3) (C1:741)                       */
    double wall_mirror_left;  /* 2*WALL%EDGE(4) (C1:743)                       */
    double osc_u;             /* U_C of LBM_MOTION_OSCILLATE (C4:30)           */
    double osc_period;        /* T_C of LBM_MOTION_OSCILLATE (C4:32)           */
    int32_t strain_model;     /* LBM_STRAIN_* (non-Newtonian strain rate)      */
    int32_t collision;        /* LBM_COLLISION_*                               */
} lbm_params;

/* Particle input record (lbm_set_particles): LBM_PIN doubles per disk. */
#define LBM_PIN 8   /* x, y, angle, u, v, omega, diam, rho_p */

/* Particle output record (lbm_get_particles): LBM_POUT doubles per disk. */
#define LBM_POUT 16
/*  0 x      1 y      2 angle  3 u      4 v      5 omega
 *  6 Fx     7 Fy     8 Tz        hydrodynamic FORCE(1:3)  (C1:546-570)
 *  9 Fcol_x 10 Fcol_y            F_COL (C1:596-769)
 * 11 Fin_x  12 Fin_y  13 Fin_t   F_H_IN (C1:250-252)
 * 14 mass M_P  15 inertia I_P    (C1:178-179)                              */

/* Field selectors for lbm_get_field. */
enum {
    LBM_FIELD_UX = 0,      /* corrected velocity UX (C1:1138-1152)             */
    LBM_FIELD_UY = 1,
    LBM_FIELD_RHO = 2,     /* RHO (C1:1421-1439)                               */
    LBM_FIELD_PHI = 3,     /* total solid fraction sum_p PHI_p (C1:407-484)    */
    LBM_FIELD_GX = 4,      /* SPM body force G (C1:488-542)                    */
    LBM_FIELD_GY = 5,
    LBM_FIELD_TAU11 = 6,   /* STRESS(1:3) of the last collision (C6:947-948)   */
    LBM_FIELD_TAU22 = 7,
    LBM_FIELD_TAU12 = 8,
    LBM_FIELD_OMEGA = 9    /* OMEGA_BN of the last collision (C6:957)          */
};

/* History record: LBM_SERIES_HEAD + series_particles * LBM_SERIES_PER doubles.
 * head: step kk, mean density AvgDen (C1:318; NaN when not evaluated)
 * per particle: x y angle u v omega Fx Fy Tz Fin_x Fin_y Fin_t           */
#define LBM_SERIES_HEAD 2
#define LBM_SERIES_PER 12

typedef struct lbm_sim lbm_sim;

/* Fill *p with the constants of C1 as the Fortran program holds them
 * (REAL(4) literals widened to double), NX/NY = 240/720, FP64, Zou-He. */
int lbm_params_init(lbm_params* p);

/* Allocate the lattice and initialise it to f = f_eq(rho0, 0) as INITIALIZE
 * + COMPUTEFEQNEW do (C1:575-592, C1:1157-1175).  Rejects 1/omega < 0.5
 * with LBM_E_TAU (C1:127-130).  Replaces MAIN's set-up, C1:110-215. */
int lbm_create(const lbm_params* p, lbm_sim** out);
int lbm_destroy(lbm_sim* h);

/* Set np disks from np*LBM_PIN doubles; M_P and I_P follow C1:178-179,
 * VP_OLD and FORCE start at zero as in the reference's static storage.
 * Replaces the particle read C1:170-179 / C3:145-156 / C6:161-169. */
int lbm_set_particles(lbm_sim* h, int32_t np, const double* pin);

/* Advance nsteps time steps.  Each step is one pass of the time loop body
 * C1:241-319 / C6:293-351 / C3:306-399: repulsion, Newton-Euler update,
 * solid fraction, MRT collision, streaming, boundary conditions,
 * macroscopic variables, SPM force field, hydrodynamic force, velocity
 * correction, mean-density check (at history steps). */
int lbm_step(lbm_sim* h, int32_t nsteps);

/* Completed time steps (KK). */
int lbm_get_step(lbm_sim* h, int64_t* kk);

/* Copy the particle state (np*LBM_POUT doubles) to host memory. */
int lbm_get_particles(lbm_sim* h, double* out);

/* Copy one field of (NX+1)*(NY+1) doubles, i fastest (Fortran order of the
 * reference's (0:NX,0:NY) arrays). */
int lbm_get_field(lbm_sim* h, int32_t which, double* out);

/* Copy the DOMAIN_IMAGE codes: 10 particle node (some PHI_p >= 0.5,
 * C1:477-480); for Bingham 5 unyielded / 0 yielded (C6:950-954); else 0. */
int lbm_get_image(lbm_sim* h, int32_t* out);

/* Drain up to max_records history records into out, oldest first; *nrec =
 * number copied.  Record length is lbm_series_record_len(h) doubles.  Each
 * lbm_step call queues the copies of its records after its kernels, on a
 * second stream of the handle, so the steps queued next run while they
 * cross to the host; this call waits only for the copies of the records it
 * returns.  The status returned is that of the last completed lbm_step. */
int lbm_get_series(lbm_sim* h, double* out, int32_t max_records, int32_t* nrec);
int lbm_series_record_len(lbm_sim* h, int32_t* len);

/* Mean density SUM(RHO)/((NX+1)(NY+1)) of the current state (C1:318). */
int lbm_get_mean_density(lbm_sim* h, double* avg);

/* Convergence measure of COMPUTEERROR (C1:1592-1612), which the reference
 * calls every 1000 steps (C1:321-325): ER = sqrt(sum |u - u0|^2 / sum |u|^2)
 * over all nodes, u the corrected velocity of the current step and u0 the
 * velocity of the previous call (zero before the first call, as U0 = UX
 * after INITIALIZE, C1:154-155); the call then keeps u as the new u0. */
int lbm_compute_error(lbm_sim* h, double* er);

/* Checkpoint: the complete dynamic state of step KK, as the reference's
 * restart dump holds it (C1:351-379): f is 9*(NX+1)*(NY+1) doubles in the
 * F(0:8,0:NX,0:NY) order holding F after the boundary conditions of step KK;
 * omega is OMEGA_BN, (NX+1)*(NY+1) doubles (Bingham; may be NULL otherwise);
 * particles is np*LBM_STATE_PER doubles:
 *   0 x 1 y 2 angle 3 u 4 v 5 omega 6-8 VP_OLD 9-11 FORCE 12-13 F_COL
 *   14-16 F_H_IN 17 diam 18 rho_p 19 stale wall distance D_PW
 * Unlike the reference dump, VP_OLD is kept, so a restart continues the
 * internal-mass term exactly. */
#define LBM_STATE_PER 20
int lbm_get_state(lbm_sim* h, double* f, double* omega, double* particles);
int lbm_set_state(lbm_sim* h, int64_t kk, const double* f, const double* omega,
                  int32_t np, const double* particles);

/* Sticky device status (NaN, overflow, timeout); 0 when healthy. */
int lbm_get_status(lbm_sim* h);

/* Check of the failure path of the kernels' bounded waits (no counterpart in
 * the reference): on the handle's stream, one thread waits on a fresh
 * mbarrier that nothing arrives at, with the same bounded wait the step
 * kernel uses, and gives up after `limit` polls (1..1048576), setting the
 * handle's timeout status as a step kernel whose wait expired does.  The
 * handle then reports LBM_E_TIMEOUT from lbm_get_status and refuses further
 * steps (sticky); the device and other handles are unaffected. */
int lbm_selftest_wait(lbm_sim* h, int32_t limit);

/* The handle's CUDA stream (a cudaStream_t), so a caller can order its own
 * work or record events against the library's kernels.  The copies of the
 * history records run on a second, internal stream; lbm_get_series is the
 * way to wait for them.  The reference has no counterpart (it is
 * single-threaded host code). */
int lbm_get_stream(lbm_sim* h, void** stream);

/* Per-kernel device timing, for profiling the time loop (the reference only
 * times the whole run, C1:148, C1:395-397).  While enabled, lbm_step records
 * CUDA events around every launch; lbm_profile_read returns the summed
 * device milliseconds and launch counts of the particle kernel [0] and the
 * lattice kernel [1] since the last enable, and resets them. */
int lbm_profile(lbm_sim* h, int32_t enable);
int lbm_profile_read(lbm_sim* h, double* ms, int64_t* launches);

const char* lbm_strerror(int code);

/* 1 in the checked build of this library (liblbm2d_checked.so: every
 * computed index of the step, particle and batch kernels is checked against
 * its buffer; a failed check skips the access and reports LBM_E_BOUNDS), 0
 * in the ordinary build.  The reference has no counterpart: its Fortran is
 * built without array bounds checks. */
int32_t lbm_checked_build(void);

/* Adjoint gradients of a particle observable (no counterpart in the
 * reference, which has no derivatives).  The objective is the mean of one
 * field of disk `particle` over steps n0..n1 (the record after each step's
 * Newton-Euler update, C1:247-259):
 *   J = sum_{n=n0..n1} state_n[component] / (n1 - n0 + 1).
 * lbm_adjoint runs the forward time loop from step 0 to n1 -- the handle
 * must be at step 0 with its disks set, and is left at step n1 as lbm_step
 * would leave it, history records included -- then the reverse sweep:
 * checkpoints every `checkpoint_every` steps (0: round(sqrt(n1))), each
 * segment recomputed forward and its states reversed through the transposed
 * collision / streaming / boundary / SPM / force / Newton-Euler steps.
 * Device memory kept by the handle: ceil((n1 - 1) / L) checkpoints, two sets
 * of L slots (one set when there is a single segment), each 10 lattice
 * planes, L = checkpoint_every; a segment's recompute runs on a second
 * stream of the handle beside the reverse sweep of the segment after it.
 * The call returns when the sweep is done.
 * grads receives 2 + 3*np doubles:
 *   [LBM_GRAD_TAU_Y] dJ/dtau_y   [LBM_GRAD_NU] dJ/dnu (plastic viscosity)
 *   then per disk p: dJ/drho_p, dJ/dx0, dJ/dy0 at LBM_GRAD_HEAD + 3p.
 * Supported: Newtonian or Bingham (Papanastasiou, m_neq strain rate), Zou-He
 * or half-way bounce-back walls, free motion, at most LBM_ADJ_MAX_PARTICLES
 * disks, with the pair-distance contact test when np > 1; anything else
 * returns LBM_E_INVALID before any work.  The repulsion constants (c_ij)
 * are held fixed. */
#define LBM_ADJ_MAX_PARTICLES 64
enum { LBM_OBJ_X = 0, LBM_OBJ_Y = 1, LBM_OBJ_U = 3, LBM_OBJ_V = 4, LBM_OBJ_W = 5 };
enum { LBM_GRAD_TAU_Y = 0, LBM_GRAD_NU = 1, LBM_GRAD_HEAD = 2, LBM_GRAD_PER = 3 };
typedef struct lbm_objective {
    int32_t struct_size;      /* sizeof(lbm_objective) */
    int32_t particle;         /* observed disk, 0..np-1 */
    int32_t component;        /* LBM_OBJ_* */
    int32_t checkpoint_every; /* steps between checkpoints; 0: round(sqrt(n1)) */
    int64_t n0, n1;           /* window, 1 <= n0 <= n1 */
} lbm_objective;
int lbm_adjoint(lbm_sim* h, const lbm_objective* obj, double* value, double* grads);

/* Batched time steps (no counterpart in the reference, which runs one case
 * per process): nsim independent simulations, each with its own lbm_params
 * (lattice size, rheology, boundary, precision equal for all, device equal
 * for all), advance together, one launch of the particle kernel (one block
 * per simulation) and one of a persistent lattice kernel over every
 * simulation's tiles per step, replayed from a captured CUDA graph.
 * lbm_batch_sim returns simulation i's handle for everything else
 * (lbm_set_particles, the getters, lbm_get_state ...); do not call
 * lbm_step on it while it belongs to a batch.  The first lbm_batch_step
 * picks the lattice kernel by timing each candidate on live steps: the
 * single-run step kernel's TMA pipeline on tiles of 64x8 nodes (at its own
 * occupancy; batches without a BGK run) or the
 * one-node-per-thread kernel at a tile shape of 32x8, 64x4 or 128x2 nodes
 * and a persistent grid of 2, 4 or 6 blocks per SM; the results do not
 * depend on the choice.  lbm_batch_set_tuning fixes it instead (tile_x 0:
 * automatic; the TMA tile shape ignores blocks_per_sm).  The handles belong
 * to the batch: lbm_batch_destroy destroys them. */
typedef struct lbm_batch lbm_batch;
int lbm_batch_create(const lbm_params* params, int32_t nsim, lbm_batch** out);
lbm_sim* lbm_batch_sim(lbm_batch* b, int32_t i);
int lbm_batch_step(lbm_batch* b, int32_t nsteps);
int lbm_batch_tuning(lbm_batch* b, int32_t* tile_x, int32_t* tile_y, int32_t* blocks_per_sm);
int lbm_batch_set_tuning(lbm_batch* b, int32_t tile_x, int32_t tile_y, int32_t blocks_per_sm);
/* The batch's CUDA stream (a cudaStream_t), for the caller's own events. */
int lbm_batch_stream(lbm_batch* b, void** stream);
int lbm_batch_destroy(lbm_batch* b);

/* Output fields of a state held in caller-owned device memory, computed
 * without allocating anything (no counterpart in the reference).
 *
 * For drivers that must not allocate device memory while they run: one that
 * has given all device memory to its own pool or to other solvers, or one
 * that post-processes inside its time loop, where cudaMalloc/cudaFree would
 * synchronise the whole device.  No simulation handle is needed.
 *
 *   p          nx, ny, zeta, pi are read (struct_size must match)
 *   f          device, 9*(NX+1)*(NY+1) doubles: F after the boundary
 *              conditions, F(0:8,0:NX,0:NY) order (as lbm_get_state gives it)
 *   particles  device, np*LBM_PIN doubles (x, y, angle, u, v, omega, diam,
 *              rho_p); may be NULL when np == 0
 *   out        device, 7*(NX+1)*(NY+1) doubles: UX, UY, RHO, PHI, GX, GY as
 *              lbm_get_field gives them, then the image code (10 particle
 *              node, else 0), i fastest
 *   stream     cudaStream_t to run on (NULL: the legacy default stream)
 *
 * The candidate lists of the solid-fraction evaluation live in a fixed
 * static device array, so the lattice may hold at most LBM_NOALLOC_MAX_TILES
 * tiles of 128 x 8 nodes (ceil((NX+1)/128) * ceil((NY+1)/8), e.g. 2047 x
 * 8191) and at most LBM_NOALLOC_MAX_PARTICLES disks; larger inputs return
 * LBM_E_SCRATCH before any work is queued.  Each call clears the scratch it
 * uses, so nothing needs to start at zero.  The first call on a device also
 * looks up the scratch address (make it before any stream capture starts on
 * that device); after cudaDeviceReset the next call looks it up again.  The
 * scratch is shared by all calls on a device: calls that overlap in time on
 * one device race and must be serialised by the caller.  The call returns
 * after its work on `stream` has finished.  LBM_E_OVERFLOW: more than 32
 * disks touch one tile; out is then incomplete (the disks past the 32nd of
 * that tile are left out of its PHI, G and image).  LBM_E_NAN: a particle
 * record holds a non-finite position, velocity or diameter; that disk is
 * left out of out. */
#define LBM_NOALLOC_MAX_TILES 16384
#define LBM_NOALLOC_MAX_PARTICLES 4096
int lbm_fields_noalloc(const lbm_params* p, const double* f, int32_t np,
                       const double* particles, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LBM2D_H */
