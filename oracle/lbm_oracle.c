/*
 * lbm_oracle.c -- CPU oracle (test infrastructure, not product code).
 *
 * Single-threaded FP64 restatement of one time step of the reference
 * Fortran programs.  Every routine follows the reference routine cited in
 * its comment, in the same loop order (J outer, I inner) and with the same
 * left-to-right evaluation of each expression, so that a build without
 * floating-point contraction (-ffp-contract=off) reproduces the Fortran
 * arithmetic operation by operation.  Citations:
 *   C1 = 1_Disk_Newtonian/D2Q9_1P_Validated_20190530.f90
 *   C6 = 6_FreeFall_YieldStress/D2Q9_BinghamSediment_Validated_20191127.f90
 *   C3 = 3_MultiParticle_Sedimentation/D2Q9_RTParticle_20191003.f90
 *
 * The only deliberate departures, all selectable:
 *   - omega_chain=0 relaxes each Bingham node with its own omega of the
 *     previous step instead of the previous node's (C6:958 chain);
 *   - walls move with zero velocity only (every shipped case uses zero);
 *   - the C1 "wall particle" PHI (C1:419-458) only feeds DOMAIN_IMAGE and
 *     is not computed.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The arithmetic type: double, or in the tangent build (C++, ORACLE_TANGENT)
 * a value with its derivative (oracle_dual.h).  RVAL gives the value. */
#ifdef ORACLE_TANGENT
#include "oracle_dual.h"
#else
typedef double real;
#define RVAL(x) (x)
#endif

#define Q 9
static const int CX[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};   /* C1:13 */
static const int CY[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};   /* C1:14 */

typedef struct {
    real center[2], angle, vel[3], diam, force[3], fcol[2];
    real rho_p, m_p, i_p;
    real vp_old[3], fh_in[3];
    real* phi; /* (0:NX,0:NY) or NULL in on-the-fly mode */
} disk_t;

struct oracle {
    lbm_params p;
    oracle_opts opt;
    int nx, ny, n1x, n1y;
    size_t nn;
    real *F, *FPOST, *FEQ, *G, *RHO, *UX, *UY, *OMEGA_BN, *STRESS;
    real *U0, *V0;  /* COMPUTEERROR's previous velocity (allocated on first use) */
    int32_t* IMAGE;
    uint8_t* IS_PARTICLE;
    real omega, omega_mrt[Q];
    real tau_y, nu; /* lbm_params' tau_y and nu in the arithmetic type */
    int np;
    disk_t* disk;
    real stale_dpw;
    int64_t kk;
#ifdef ORACLE_TANGENT
    int seed_which, seed_disk; /* the input whose derivative is carried */
#endif
    /* history */
    double* series;
    int32_t series_len, series_n, series_cap;
};

#define IDX(o, i, j) ((size_t)(i) + (size_t)(o)->n1x * (size_t)(j))
#define FK(o, arr, k, i, j) ((arr)[(size_t)(k) + (size_t)Q * IDX(o, i, j)])

/* ---- COMPUTEFEQNEW, C1:1157-1175 ------------------------------------- */
static void compute_feq(const oracle* o, real ux, real uy, real rho, real* feq) {
    const real W0 = o->p.w_init[0], W1 = o->p.w_init[1], W2 = o->p.w_init[2];
    real U2 = ux * ux + uy * uy;
    feq[0] = W0 * rho * (2. - 3. * U2);
    feq[1] = W1 * rho * (2. + 6. * ux + 9. * ux * ux - 3. * U2);
    feq[2] = W1 * rho * (2. + 6. * uy + 9. * uy * uy - 3. * U2);
    feq[3] = W1 * rho * (2. - 6. * ux + 9. * ux * ux - 3. * U2);
    feq[4] = W1 * rho * (2. - 6. * uy + 9. * uy * uy - 3. * U2);
    feq[5] = W2 * rho * (1. + 3. * (ux + uy) + 9. * ux * uy + 3. * U2);
    feq[6] = W2 * rho * (1. - 3. * (ux - uy) - 9. * ux * uy + 3. * U2);
    feq[7] = W2 * rho * (1. - 3. * (ux + uy) + 9. * ux * uy + 3. * U2);
    feq[8] = W2 * rho * (1. + 3. * (ux - uy) - 9. * ux * uy + 3. * U2);
}

/* ---- ComputeRelaxation_MRT, C1:1029-1048 (fixed q) / C6:1002-1021 ---- */
static void compute_relaxation(const oracle* o, real omega, real* s) {
    real oq = o->p.rate_set == LBM_RATES_Q_OF_OMEGA ? 8. * (2. - omega) / (8. - omega)
                                                      : o->p.s_q;
    s[0] = 0.0; s[1] = o->p.s_e; s[2] = o->p.s_eps; s[3] = 0.0;
    s[4] = oq; s[5] = 0.0; s[6] = oq; s[7] = omega; s[8] = omega;
}

/* ---- INITIALIZE, C1:575-592 ------------------------------------------ */
static void initialize(oracle* o) {
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i) {
            size_t n = IDX(o, i, j);
            o->RHO[n] = o->p.rho0;
            o->UX[n] = 0.0;
            o->UY[n] = 0.0;
            compute_feq(o, o->UX[n], o->UY[n], o->RHO[n], &o->FEQ[Q * n]);
            memcpy(&o->F[Q * n], &o->FEQ[Q * n], Q * sizeof(real));
        }
    memset(o->G, 0, 2 * o->nn * sizeof(real));
}

/* ---- SPM solid fraction of one node, C1:464-476 ----------------------- */
static real phi_node(const oracle* o, const disk_t* d, int i, int j) {
    real X_PC = d->center[0], Y_PC = d->center[1];
    real R_P = 0.5 * d->diam;
    real fi = (real)i, fj = (real)j;
    real D_I = R_P - sqrt((fi - X_PC) * (fi - X_PC) + (fj - Y_PC) * (fj - Y_PC));
    real Z = o->p.zeta, phi = 0.0;
    if (D_I <= -0.5 * Z)
        phi = 0.0;
    else if (fabs(D_I) < 0.5 * Z)
        phi = 0.5 * (sin(o->p.pi * D_I / Z) + 1.0);
    else if (D_I >= 0.5 * Z)
        phi = 1.0;
    return phi;
}

static inline real get_phi(const oracle* o, const disk_t* d, int i, int j) {
    return d->phi ? d->phi[IDX(o, i, j)] : phi_node(o, d, i, j);
}

/* ---- ComputeConcenterationFunction, C1:407-484 (particle part) -------- */
static void compute_concentration(oracle* o) {
    memset(o->IS_PARTICLE, 0, o->nn);
    for (int ip = 0; ip < o->np; ++ip) {
        disk_t* d = &o->disk[ip];
        for (int j = 0; j <= o->ny; ++j)
            for (int i = 0; i <= o->nx; ++i) {
                real phi = phi_node(o, d, i, j);
                if (d->phi) d->phi[IDX(o, i, j)] = phi;
                if (phi >= 0.5) o->IS_PARTICLE[IDX(o, i, j)] = 1;
            }
    }
}

/* ---- Collision_MRT + ComputeSourceEquilib_MRT, C1:875-1027, C6:867-1000 */
static void collision_node(oracle* o, size_t n, const real* S, real* Fn, real* stress_out,
                           int32_t* image_out, real* omega_new) {
    const real d_mrt = o->p.d_mrt;
    real f0 = Fn[0], f1 = Fn[1], f2 = Fn[2], f3 = Fn[3], f4 = Fn[4], f5 = Fn[5], f6 = Fn[6],
           f7 = Fn[7], f8 = Fn[8];
    real M[Q], MF[Q], MEQ[Q], MNE[Q], F1[Q];
    /* C6:878-886 */
    M[0] = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
    M[1] = -4.0 * f0 - f1 - f2 - f3 - f4 + 2.0 * (f5 + f6 + f7 + f8);
    M[2] = 4.0 * f0 - 2.0 * (f1 + f2 + f3 + f4) + (f5 + f6 + f7 + f8);
    M[3] = f1 - f3 + f5 - f6 - f7 + f8;
    M[4] = -2.0 * (f1 - f3) + f5 - f6 - f7 + f8;
    M[5] = f2 - f4 + f5 + f6 - f7 - f8;
    M[6] = -2.0 * (f2 - f4) + f5 + f6 - f7 - f8;
    M[7] = f1 - f2 + f3 - f4;
    M[8] = f5 - f6 + f7 - f8;
    /* ComputeSourceEquilib_MRT, C1:991-1027 (G_X = G_Y = 0) */
    real UX = o->UX[n], UY = o->UY[n], RHO = o->RHO[n];
    real GX = o->G[2 * n], GY = o->G[2 * n + 1];
    real F_X = RHO * (GX + 0.0), F_Y = RHO * (GY + 0.0);
    MF[0] = 0.0;
    MF[1] = 6.0 * (F_X * UX + F_Y * UY);
    MF[2] = -6.0 * (F_X * UX + F_Y * UY);
    MF[3] = F_X;
    MF[4] = -F_X;
    MF[5] = F_Y;
    MF[6] = -F_Y;
    MF[7] = 2.0 * (F_X * UX - F_Y * UY);
    MF[8] = F_Y * UX + F_X * UY;
    real U2 = UX * UX + UY * UY;
    MEQ[0] = RHO;
    MEQ[1] = RHO * (-2.0 + 3. * U2);
    MEQ[2] = RHO * (1.0 - 3. * U2);
    MEQ[3] = RHO * (UX);
    MEQ[4] = RHO * (-UX);
    MEQ[5] = RHO * (UY);
    MEQ[6] = RHO * (-UY);
    MEQ[7] = RHO * (UX * UX - UY * UY);
    MEQ[8] = RHO * (UX * UY);
    /* C6:889; LBM_STRAIN_FEQ: against the moments of COMPUTEFEQNEW, C1:896-908 */
    const int feq_neq = o->p.strain_model == LBM_STRAIN_FEQ;
    if (feq_neq) {
        real FE[Q], ME[Q];
        compute_feq(o, UX, UY, RHO, FE);
        ME[0] = FE[0] + FE[1] + FE[2] + FE[3] + FE[4] + FE[5] + FE[6] + FE[7] + FE[8];
        ME[1] = -4.0 * FE[0] - FE[1] - FE[2] - FE[3] - FE[4] + 2.0 * (FE[5] + FE[6] + FE[7] + FE[8]);
        ME[2] = 4.0 * FE[0] - 2.0 * (FE[1] + FE[2] + FE[3] + FE[4]) + (FE[5] + FE[6] + FE[7] + FE[8]);
        ME[3] = FE[1] - FE[3] + FE[5] - FE[6] - FE[7] + FE[8];
        ME[4] = -2.0 * (FE[1] - FE[3]) + FE[5] - FE[6] - FE[7] + FE[8];
        ME[5] = FE[2] - FE[4] + FE[5] + FE[6] - FE[7] - FE[8];
        ME[6] = -2.0 * (FE[2] - FE[4]) + FE[5] + FE[6] - FE[7] - FE[8];
        ME[7] = FE[1] - FE[2] + FE[3] - FE[4];
        ME[8] = FE[5] - FE[6] + FE[7] - FE[8];
        for (int k = 0; k < Q; ++k) MNE[k] = M[k] - ME[k];
    } else {
        for (int k = 0; k < Q; ++k) MNE[k] = M[k] - MEQ[k];
    }
    /* C1:911 */
    real m[Q];
    for (int k = 0; k < Q; ++k)
        m[k] = S[k] * MEQ[k] + (1. - S[k]) * M[k] + (1. - 0.5 * S[k]) * MF[k];
    /* C1:913-921 */
    Fn[0] = d_mrt * (4.0 * (m[0] - m[1] + m[2]));
    Fn[1] = d_mrt * (4. * m[0] - m[1] - 2. * m[2] + 6. * m[3] - 6. * m[4] + 9. * m[7]);
    Fn[2] = d_mrt * (4.0 * m[0] - m[1] - 2.0 * m[2] + 6.0 * m[5] - 6.0 * m[6] - 9.0 * m[7]);
    Fn[3] = d_mrt * (4.0 * m[0] - m[1] - 2.0 * m[2] - 6.0 * m[3] + 6.0 * m[4] + 9.0 * m[7]);
    Fn[4] = d_mrt * (4.0 * m[0] - m[1] - 2.0 * m[2] - 6.0 * m[5] + 6.0 * m[6] - 9.0 * m[7]);
    Fn[5] = d_mrt * (4.0 * m[0] + 2.0 * m[1] + m[2] + 6.0 * m[3] + 3.0 * m[4] + 6.0 * m[5] +
                     3.0 * m[6] + 9.0 * m[8]);
    Fn[6] = d_mrt * (4.0 * m[0] + 2.0 * m[1] + m[2] - 6.0 * m[3] - 3.0 * m[4] + 6.0 * m[5] +
                     3.0 * m[6] - 9.0 * m[8]);
    Fn[7] = d_mrt * (4.0 * m[0] + 2.0 * m[1] + m[2] - 6.0 * m[3] - 3.0 * m[4] - 6.0 * m[5] -
                     3.0 * m[6] + 9.0 * m[8]);
    Fn[8] = d_mrt * (4.0 * m[0] + 2.0 * m[1] + m[2] + 6.0 * m[3] + 3.0 * m[4] - 6.0 * m[5] -
                     3.0 * m[6] - 9.0 * m[8]);

    /* Chai strain rate, C6:903-916 */
    F1[0] = 4.0 * S[0] * MNE[0] - 4.0 * S[1] * MNE[1] + 4.0 * S[2] * MNE[2];
    F1[1] = 4.0 * S[0] * MNE[0] - 1.0 * S[1] * MNE[1] - 2.0 * S[2] * MNE[2] + 6.0 * S[3] * MNE[3] -
            6.0 * S[4] * MNE[4] + 9.0 * S[7] * MNE[7];
    F1[2] = 4.0 * S[0] * MNE[0] - 1.0 * S[1] * MNE[1] - 2.0 * S[2] * MNE[2] + 6.0 * S[5] * MNE[5] -
            6.0 * S[6] * MNE[6] - 9.0 * S[7] * MNE[7];
    F1[3] = 4.0 * S[0] * MNE[0] - 1.0 * S[1] * MNE[1] - 2.0 * S[2] * MNE[2] - 6.0 * S[3] * MNE[3] +
            6.0 * S[4] * MNE[4] + 9.0 * S[7] * MNE[7];
    F1[4] = 4.0 * S[0] * MNE[0] - 1.0 * S[1] * MNE[1] - 2.0 * S[2] * MNE[2] - 6.0 * S[5] * MNE[5] +
            6.0 * S[6] * MNE[6] - 9.0 * S[7] * MNE[7];
    F1[5] = 4.0 * S[0] * MNE[0] + 2.0 * S[1] * MNE[1] + 1.0 * S[2] * MNE[2] + 6.0 * S[3] * MNE[3] +
            3.0 * S[4] * MNE[4] + 6.0 * S[5] * MNE[5] + 3.0 * S[6] * MNE[6] + 9.0 * S[8] * MNE[8];
    F1[6] = 4.0 * S[0] * MNE[0] + 2.0 * S[1] * MNE[1] + 1.0 * S[2] * MNE[2] - 6.0 * S[3] * MNE[3] -
            3.0 * S[4] * MNE[4] + 6.0 * S[5] * MNE[5] + 3.0 * S[6] * MNE[6] - 9.0 * S[8] * MNE[8];
    F1[7] = 4.0 * S[0] * MNE[0] + 2.0 * S[1] * MNE[1] + 1.0 * S[2] * MNE[2] - 6.0 * S[3] * MNE[3] -
            3.0 * S[4] * MNE[4] - 6.0 * S[5] * MNE[5] - 3.0 * S[6] * MNE[6] + 9.0 * S[8] * MNE[8];
    F1[8] = 4.0 * S[0] * MNE[0] + 2.0 * S[1] * MNE[1] + 1.0 * S[2] * MNE[2] + 6.0 * S[3] * MNE[3] +
            3.0 * S[4] * MNE[4] - 6.0 * S[5] * MNE[5] - 3.0 * S[6] * MNE[6] - 9.0 * S[8] * MNE[8];
    real D11, D22, D12;
    if (feq_neq) { /* C1:940-948: 1/RHO folded into both terms */
        real IR = 1.0 / RHO;
        real ZARIB = -1.5 * d_mrt * IR;
        D11 = ZARIB * (F1[1] + F1[5] + F1[6] + F1[3] + F1[7] + F1[8]);
        D22 = ZARIB * (F1[5] + F1[2] + F1[6] + F1[7] + F1[4] + F1[8]);
        D12 = ZARIB * (F1[5] - F1[6] + F1[7] - F1[8]);
        ZARIB = 0.75 * IR;
        D11 = D11 + ZARIB * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GX * UX));
        D22 = D22 + ZARIB * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GY * UY));
        D12 = D12 + ZARIB * (-S[7] * (GX * UY + GY * UX));
    } else { /* C6:903-916 */
        real ZARIB = -1.5 * d_mrt;
        D11 = ZARIB * (F1[1] + F1[5] + F1[6] + F1[3] + F1[7] + F1[8]) +
              0.75 * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GX * UX));
        D22 = ZARIB * (F1[5] + F1[2] + F1[6] + F1[7] + F1[4] + F1[8]) +
              0.75 * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GY * UY));
        D12 = ZARIB * (F1[5] - F1[6] + F1[7] - F1[8]) + 0.75 * (-S[7] * (GX * UY + GY * UX));
    }
    real NU = o->nu;
    real T11 = NU * 2.0 * D11, T22 = NU * 2.0 * D22, T12 = NU * 2.0 * D12; /* C6:918 */
    if (o->p.rheology == LBM_BINGHAM || o->p.rheology == LBM_CASSON) {
        /* C6:921-958; Casson C3:978-996 */
        real INV_RHO = 1.0 / RHO;
        if (!feq_neq) {
            D11 = D11 * INV_RHO;
            D22 = D22 * INV_RHO;
            D12 = D12 * INV_RHO;
        }
        real GAMMA = sqrt(2.0 * fabs(D11 * D11 + D22 * D22 + 2.0 * (D12 * D12)));
        real NU_A;
        if (o->p.rheology == LBM_CASSON) {
            if (GAMMA < o->p.gamma_min)
                NU_A = sqrt(NU) + sqrt(o->p.m_pap * o->tau_y);
            else {
                NU_A = sqrt(NU) + sqrt(o->tau_y / GAMMA) * (1.0 - exp(-sqrt(o->p.m_pap * GAMMA)));
                NU_A = NU_A * NU_A;
            }
        } else if (GAMMA < o->p.gamma_min)
            NU_A = NU + o->p.m_pap * o->tau_y;
        else
            NU_A = NU + (o->tau_y / GAMMA) * (1.0 - exp(-(o->p.m_pap * GAMMA)));
        T11 = NU_A * 2.0 * D11;
        T22 = NU_A * 2.0 * D22;
        T12 = NU_A * 2.0 * D12;
        real TAU_MAG = sqrt(0.5 * fabs(T11 * T11 + T22 * T22 + 2.0 * (T12 * T12)));
        *image_out = (TAU_MAG <= o->tau_y) ? 5 : 0;
        NU_A = NU_A * INV_RHO;
        *omega_new = 1.0 / (3.0 * NU_A + 0.5);
    }
    stress_out[0] = T11;
    stress_out[1] = T22;
    stress_out[2] = T12;
}

static void collision_mrt(oracle* o) {
    real S[Q];
    int bingham = o->p.rheology == LBM_BINGHAM || o->p.rheology == LBM_CASSON;
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i) {
            size_t n = IDX(o, i, j);
            if (bingham && !o->opt.omega_chain)
                compute_relaxation(o, o->OMEGA_BN[n], S);
            else
                memcpy(S, o->omega_mrt, sizeof S);
            real omega_new = o->OMEGA_BN[n];
            int32_t img = 0;
            collision_node(o, n, S, &o->F[Q * n], &o->STRESS[3 * n], &img, &omega_new);
            if (bingham) {
                o->IMAGE[n] = img;
                o->OMEGA_BN[n] = omega_new;
                /* C6:958: the global rates now follow this node */
                if (o->opt.omega_chain) compute_relaxation(o, omega_new, o->omega_mrt);
            }
        }
}

/* ---- ComputeSourceEquilib_Hydro, C1:843-870: forcing FI and FEQ with
 * G_X = G_Y = 0; the forcing weights are the REAL(4) quotients 4.0/9.0,
 * 1./9., 1./36. ------------------------------------------------------------ */
static void source_equilib_hydro(const oracle* o, real UX, real UY, real RHO, real GX,
                                 real GY, real* FI, real* FEQ) {
    const real W0 = (real)(4.0f / 9.0f), W1 = (real)(1.0f / 9.0f),
                 W2 = (real)(1.0f / 36.0f);
    const real gx = GX + 0.0, gy = GY + 0.0;
    FI[0] = W0 * RHO * (-(3. * UX * gx) - 3. * UY * gy);
    FI[1] = W1 * RHO * ((3. + 6. * UX) * gx - 3. * UY * gy);
    FI[2] = W1 * RHO * (-(3. * UX * gx) + (3. + 6. * UY) * gy);
    FI[3] = W1 * RHO * ((-3. + 6. * UX) * gx - 3. * UY * gy);
    FI[4] = W1 * RHO * (-(3. * UX * gx) + (-3. + 6. * UY) * gy);
    FI[5] = W2 * RHO * ((3. + 6. * UX + 9. * UY) * gx + (3. + 9. * UX + 6. * UY) * gy);
    FI[6] = W2 * RHO * ((-3. + 6. * UX - 9. * UY) * gx + (3. - 9. * UX + 6. * UY) * gy);
    FI[7] = W2 * RHO * ((-3. + 6. * UX + 9. * UY) * gx + (-3. + 9. * UX + 6. * UY) * gy);
    FI[8] = W2 * RHO * ((3. + 6. * UX - 9. * UY) * gx + (-3. - 9. * UX + 6. * UY) * gy);
    compute_feq(o, UX, UY, RHO, FEQ); /* the same expressions as COMPUTEFEQNEW */
}

/* ---- COLLISION, C1:774-841: BGK; with a Bingham rheology the bi-viscosity
 * model (C1:789-809) on f - FEQ of the previous call (FEQ holds it until the
 * node recomputes it), MU_R = 1000 MU_0, GAMMA_C = TAU_Y/(MU_R - MU_0)
 * (C1:49-53, MU_0 = NU). ---------------------------------------------------- */
static void collision_bgk(oracle* o) {
    const int bingham = o->p.rheology == LBM_BINGHAM;
    const real MU_0 = o->nu, MU_R = 1000.0 * MU_0, TAU_Y = o->tau_y;
    const real GAMMA_C = TAU_Y / (MU_R - MU_0);
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i) {
            size_t n = IDX(o, i, j);
            real* f = &o->F[Q * n];
            real* FEQ = &o->FEQ[Q * n];
            const real RHO = o->RHO[n], UX = o->UX[n], UY = o->UY[n];
            real om = o->omega;
            if (bingham) {
                real ZARIB = -1.5 * o->OMEGA_BN[n] / RHO;
                real F_1[Q];
                for (int k = 0; k < Q; ++k) F_1[k] = f[k] - FEQ[k];
                real D11 = ZARIB * (F_1[1] + F_1[5] + F_1[6] + F_1[3] + F_1[7] + F_1[8]);
                real D22 = ZARIB * (F_1[5] + F_1[2] + F_1[6] + F_1[7] + F_1[4] + F_1[8]);
                real D12 = ZARIB * (F_1[5] - F_1[6] + F_1[7] - F_1[8]);
                real GAMMA = sqrt(4.0 * fabs(D12 * D12 - D11 * D22));
                real NU_A;
                if (GAMMA < GAMMA_C) {
                    NU_A = MU_R;
                    o->IMAGE[n] = 5;
                } else {
                    NU_A = MU_0 + TAU_Y / GAMMA;
                    o->IMAGE[n] = 0;
                }
                o->OMEGA_BN[n] = 1.0 / (3.0 * NU_A + 0.5);
                om = o->OMEGA_BN[n];
            }
            real FI[Q];
            source_equilib_hydro(o, UX, UY, RHO, o->G[2 * n], o->G[2 * n + 1], FI, FEQ);
            for (int k = 0; k < Q; ++k)
                f[k] = om * FEQ[k] + (1.0 - om) * f[k] + (1. - 0.5 * om) * FI[k];
        }
}

static void collide(oracle* o) {
    if (o->p.collision == LBM_COLLISION_BGK) collision_bgk(o);
    else collision_mrt(o);
}

/* ---- STREAMING, C1:1181-1217 (pull, out-of-domain sources keep F) ----- */
static void streaming(oracle* o) {
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i)
            for (int k = 0; k < Q; ++k) {
                int io = i - CX[k], jo = j - CY[k];
                if (io >= 0 && io <= o->nx && jo >= 0 && jo <= o->ny)
                    FK(o, o->F, k, i, j) = FK(o, o->FPOST, k, io, jo);
            }
}

/* ---- BOUNDARYCONDITION ------------------------------------------------ */
#define F_(k, i, j) FK(o, o->F, k, i, j)
#define FP_(k, i, j) FK(o, o->FPOST, k, i, j)
static void corners_bb(oracle* o) {
    /* C1:1390-1414 == C6:1364-1386, wall velocity zero */
    const real s6 = o->p.inv_six, c2 = 1.0;
    real Ux_w = 0.0, Uy_w = 0.0, Rho_w;
    int I, J, NX = o->nx, NY = o->ny;
    I = 0; J = 0; Rho_w = o->RHO[IDX(o, I, J)];
    F_(1, I, J) = FP_(3, I, J) - 4.0 * s6 * c2 * Rho_w * (-Ux_w);
    F_(5, I, J) = FP_(7, I, J) - s6 * c2 * Rho_w * (-Ux_w - Uy_w);
    F_(2, I, J) = FP_(4, I, J) - 4.0 * s6 * c2 * Rho_w * (-Uy_w);
    I = 0; J = NY; Rho_w = o->RHO[IDX(o, I, J)];
    F_(1, I, J) = FP_(3, I, J) - 4.0 * s6 * c2 * Rho_w * (-Ux_w);
    F_(8, I, J) = FP_(6, I, J) - s6 * c2 * Rho_w * (-Ux_w + Uy_w);
    F_(4, I, J) = FP_(2, I, J) - 4.0 * s6 * c2 * Rho_w * (Uy_w);
    I = NX; J = NY; Rho_w = o->RHO[IDX(o, I, J)];
    F_(3, I, J) = FP_(1, I, J) - 4.0 * s6 * c2 * Rho_w * (Ux_w);
    F_(7, I, J) = FP_(5, I, J) - s6 * c2 * Rho_w * (Ux_w + Uy_w);
    F_(4, I, J) = FP_(2, I, J) - 4.0 * s6 * c2 * Rho_w * (Uy_w);
    I = NX; J = 0; Rho_w = o->RHO[IDX(o, I, J)];
    F_(2, I, J) = FP_(4, I, J) - 4.0 * s6 * c2 * Rho_w * (-Uy_w);
    F_(6, I, J) = FP_(8, I, J) - s6 * c2 * Rho_w * (Ux_w - Uy_w);
    F_(3, I, J) = FP_(1, I, J) - 4.0 * s6 * c2 * Rho_w * (Ux_w);
}

static void bc_zouhe(oracle* o) {
    /* C1:1222-1417 with UXN=UYN=UXS=UYS=UX_L=UY_L=UX_R=UY_R=0 */
    const real s6 = o->p.inv_six;
    const real UXN = 0.0, UYN = 0.0, UXS = 0.0, UYS = 0.0;
    const real UX_L = 0.0, UY_L = 0.0, UX_R = 0.0, UY_R = 0.0;
    int NX = o->nx, NY = o->ny;
    for (int i = 1; i <= NX - 1; ++i) {
        /* top moving wall C1:1250-1253 */
        real RHON = (F_(0, i, NY) + F_(1, i, NY) + F_(3, i, NY) +
                       2. * (F_(2, i, NY) + F_(6, i, NY) + F_(5, i, NY))) /
                      (1.0 + UYN);
        F_(4, i, NY) = F_(2, i, NY) - 4. * s6 * RHON * UYN;
        F_(8, i, NY) = F_(6, i, NY) - 0.5 * (F_(1, i, NY) - F_(3, i, NY)) + 0.5 * RHON * UXN -
                       s6 * RHON * UYN;
        F_(7, i, NY) = F_(5, i, NY) + 0.5 * (F_(1, i, NY) - F_(3, i, NY)) - 0.5 * RHON * UXN -
                       s6 * RHON * UYN;
        /* bottom moving wall C1:1255-1258 */
        real RHOS = (F_(0, i, 0) + F_(1, i, 0) + F_(3, i, 0) +
                       2. * (F_(4, i, 0) + F_(7, i, 0) + F_(8, i, 0))) /
                      (1.0 - UYS);
        F_(2, i, 0) = F_(4, i, 0) + 4.0 * s6 * RHOS * UYS;
        F_(5, i, 0) = F_(7, i, 0) - 0.5 * (F_(1, i, 0) - F_(3, i, 0)) + 0.5 * RHOS * UXS +
                      s6 * RHOS * UYS;
        F_(6, i, 0) = F_(8, i, 0) + 0.5 * (F_(1, i, 0) - F_(3, i, 0)) - 0.5 * RHOS * UXS +
                      s6 * RHOS * UYS;
    }
    for (int j = 1; j <= NY - 1; ++j) {
        /* left, C1:1341-1345 */
        real RHO_L = (F_(0, 0, j) + F_(2, 0, j) + F_(4, 0, j) +
                        2.0 * (F_(3, 0, j) + F_(6, 0, j) + F_(7, 0, j))) /
                       (1.0 - UX_L);
        F_(5, 0, j) = F_(7, 0, j) - 0.5 * (F_(2, 0, j) - F_(4, 0, j)) + s6 * RHO_L * UX_L +
                      0.5 * RHO_L * UY_L;
        F_(8, 0, j) = F_(6, 0, j) + 0.5 * (F_(2, 0, j) - F_(4, 0, j)) + s6 * RHO_L * UX_L -
                      0.5 * RHO_L * UY_L;
        F_(1, 0, j) = F_(3, 0, j) + 4.0 * s6 * RHO_L * UX_L;
        /* right, C1:1359-1363 */
        real RHO_R = (F_(0, NX, j) + F_(2, NX, j) + F_(4, NX, j) +
                        2.0 * (F_(1, NX, j) + F_(5, NX, j) + F_(8, NX, j))) /
                       (1.0 + UX_R);
        F_(6, NX, j) = F_(8, NX, j) - 0.5 * (F_(2, NX, j) - F_(4, NX, j)) - s6 * RHO_R * UX_R +
                       0.5 * RHO_R * UY_R;
        F_(7, NX, j) = F_(5, NX, j) + 0.5 * (F_(2, NX, j) - F_(4, NX, j)) - s6 * RHO_R * UX_R -
                       0.5 * RHO_R * UY_R;
        F_(3, NX, j) = F_(1, NX, j) - 4.0 * s6 * RHO_R * UX_R;
    }
    corners_bb(o);
}

static void bc_halfway(oracle* o) {
    /* C6:1195-1294 with zero wall velocities */
    const real s6 = o->p.inv_six, c2 = 1.0;
    const real UxN = 0.0, UyN = 0.0, UxS = 0.0, UyS = 0.0;
    const real Ux_L = 0.0, Uy_L = 0.0, Ux_R = 0.0, Uy_R = 0.0;
    int NX = o->nx, NY = o->ny;
    for (int i = 1; i <= NX - 1; ++i) {
        real rN = o->RHO[IDX(o, i, NY)], rS = o->RHO[IDX(o, i, 0)];
        F_(8, i, NY) = FP_(6, i, NY) - s6 * c2 * rN * (-UxN + UyN);
        F_(4, i, NY) = FP_(2, i, NY) - 4.0 * s6 * c2 * rN * (UyN);
        F_(7, i, NY) = FP_(5, i, NY) - s6 * c2 * rN * (UxN + UyN);
        F_(5, i, 0) = FP_(7, i, 0) - s6 * c2 * rS * (-UxS - UyS);
        F_(2, i, 0) = FP_(4, i, 0) - 4.0 * s6 * c2 * rS * (-UyS);
        F_(6, i, 0) = FP_(8, i, 0) - s6 * c2 * rS * (UxS - UyS);
    }
    for (int j = 1; j <= NY - 1; ++j) {
        real rR = o->RHO[IDX(o, NX, j)], rL = o->RHO[IDX(o, 0, j)];
        F_(6, NX, j) = FP_(8, NX, j) - s6 * c2 * rR * (Ux_R - Uy_R);
        F_(3, NX, j) = FP_(1, NX, j) - 4.0 * s6 * c2 * rR * (Ux_R);
        F_(7, NX, j) = FP_(5, NX, j) - s6 * c2 * rR * (Ux_R + Uy_R);
        F_(5, 0, j) = FP_(7, 0, j) - s6 * c2 * rL * (-Ux_L - Uy_L);
        F_(1, 0, j) = FP_(3, 0, j) - 4.0 * s6 * c2 * rL * (-Ux_L);
        F_(8, 0, j) = FP_(6, 0, j) - s6 * c2 * rL * (-Ux_L + Uy_L);
    }
    corners_bb(o);
}
#undef F_
#undef FP_

/* ---- BOUNDARYCONDITION of the oscillating-cylinder case, C4:1219-1275:
 * every edge node takes COMPUTEFEQNEW of the density and velocity that its
 * inward neighbour holds at this point of the step (those of the previous
 * step, after VelocityCorrector); corners take the diagonal neighbour. */
static void bc_equilibrium(oracle* o) {
    const int NX = o->nx, NY = o->ny;
    for (int i = 1; i <= NX - 1; ++i) {                          /* C4:1219-1223 */
        size_t a = IDX(o, i, 1), b = IDX(o, i, NY - 1);
        compute_feq(o, o->UX[a], o->UY[a], o->RHO[a], &FK(o, o->F, 0, i, 0));
        compute_feq(o, o->UX[b], o->UY[b], o->RHO[b], &FK(o, o->F, 0, i, NY));
    }
    for (int j = 1; j <= NY - 1; ++j) {                          /* C4:1263-1266 */
        size_t a = IDX(o, 1, j), b = IDX(o, NX - 1, j);
        compute_feq(o, o->UX[a], o->UY[a], o->RHO[a], &FK(o, o->F, 0, 0, j));
        compute_feq(o, o->UX[b], o->UY[b], o->RHO[b], &FK(o, o->F, 0, NX, j));
    }
    const int ci[4][4] = {{0, 0, 1, 1}, {0, NY, 1, NY - 1}, {NX, NY, NX - 1, NY - 1},
                          {NX, 0, NX - 1, 1}};                    /* C4:1268-1273 */
    for (int c = 0; c < 4; ++c) {
        size_t a = IDX(o, ci[c][2], ci[c][3]);
        compute_feq(o, o->UX[a], o->UY[a], o->RHO[a], &FK(o, o->F, 0, ci[c][0], ci[c][1]));
    }
}

/* ---- MACROSCOPICVARIABLES, C1:1421-1439 ------------------------------- */
static void macroscopic(oracle* o) {
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i) {
            size_t n = IDX(o, i, j);
            const real* f = &o->F[Q * n];
            real rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
            real rinv = 1.0 / rho;
            o->RHO[n] = rho;
            o->UX[n] = rinv * (f[1] + f[5] + f[8] - (f[6] + f[3] + f[7]));
            o->UY[n] = rinv * (f[5] + f[2] + f[6] - (f[7] + f[4] + f[8]));
        }
}

/* ---- ComputeForceField_SPM, C1:488-542 (last particle with PHI>0 wins) - */
static void force_field_spm(oracle* o) {
    for (int j = 0; j <= o->ny; ++j)
        for (int i = 0; i <= o->nx; ++i) {
            size_t n = IDX(o, i, j);
            o->G[2 * n] = 0.0;
            o->G[2 * n + 1] = 0.0;
            for (int ip = 0; ip < o->np; ++ip) {
                const disk_t* d = &o->disk[ip];
                real phi = get_phi(o, d, i, j);
                if (phi > 0.0) {
                    real UX_P = d->vel[0] - d->vel[2] * ((real)j - d->center[1]);
                    real UY_P = d->vel[1] + d->vel[2] * ((real)i - d->center[0]);
                    o->G[2 * n] = phi * (UX_P - o->UX[n]);
                    o->G[2 * n + 1] = phi * (UY_P - o->UY[n]);
                }
            }
        }
}

/* ---- ComputeForce_HYDRO, C1:546-570 ----------------------------------- */
static void force_hydro(oracle* o) {
    for (int ip = 0; ip < o->np; ++ip) {
        disk_t* d = &o->disk[ip];
        real F_P[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j <= o->ny; ++j)
            for (int i = 0; i <= o->nx; ++i) {
                real phi = get_phi(o, d, i, j);
                if (phi > 0.0) {
                    size_t n = IDX(o, i, j);
                    real UX_P = d->vel[0] - d->vel[2] * ((real)j - d->center[1]);
                    real UY_P = d->vel[1] + d->vel[2] * ((real)i - d->center[0]);
                    real rp = o->RHO[n] * phi;
                    F_P[0] = F_P[0] + rp * (o->UX[n] - UX_P);
                    F_P[1] = F_P[1] + rp * (o->UY[n] - UY_P);
                    F_P[2] = F_P[2] + rp * (((real)i - d->center[0]) * (o->UY[n] - UY_P) -
                                            ((real)j - d->center[1]) * (o->UX[n] - UX_P));
                }
            }
        d->force[0] = F_P[0];
        d->force[1] = F_P[1];
        d->force[2] = F_P[2];
    }
}

/* ---- VelocityCorrector, C1:1138-1152 ---------------------------------- */
static void velocity_corrector(oracle* o) {
    for (size_t n = 0; n < o->nn; ++n) {
        o->UX[n] = o->UX[n] + 0.5 * 1.0 * (o->G[2 * n] + 0.0);
        o->UY[n] = o->UY[n] + 0.5 * 1.0 * (o->G[2 * n + 1] + 0.0);
    }
}

/* ---- ComputeCollisionForce, Glowinski model: C1:701-768, C3:739-804 --- */
static void collision_force(oracle* o) {
    const lbm_params* p = &o->p;
    const real ZITA = p->rep_zeta, CIJ = p->c_ij;
    const real EPS_P = p->eps_p, EPS_W = p->eps_w, E_P = p->e_p, E_W = p->e_w;
    real D_PW = o->stale_dpw;
    for (int ip = 0; ip < o->np; ++ip) o->disk[ip].fcol[0] = o->disk[ip].fcol[1] = 0.0;
    if (o->np > 1) {
        for (int ip = 0; ip < o->np - 1; ++ip)
            for (int jp = ip + 1; jp < o->np; ++jp) {
                disk_t *a = &o->disk[ip], *b = &o->disk[jp];
                real dx = a->center[0] - b->center[0], dy = a->center[1] - b->center[1];
                real D_PP = sqrt(dx * dx + dy * dy);
                real rsum = 0.5 * a->diam + 0.5 * b->diam;
                real test = p->contact_test == LBM_CONTACT_STALE_DPW ? D_PW : D_PP;
                real F_PP[2] = {0.0, 0.0};
                if (D_PP > rsum + ZITA) {
                    F_PP[0] = 0.0;
                    F_PP[1] = 0.0;
                } else {
                    real q = (D_PP - 0.5 * a->diam - 0.5 * b->diam - ZITA) / ZITA;
                    if (D_PP <= rsum + ZITA && test > rsum) {
                        F_PP[0] = EPS_P * CIJ * (q * q) * dx / D_PP;
                        F_PP[1] = EPS_P * CIJ * (q * q) * dy / D_PP;
                    } else if (test <= rsum) {
                        real e = E_P * CIJ * (rsum - D_PP) / ZITA;
                        F_PP[0] = (EPS_P * CIJ * (q * q) + e) * dx / D_PP;
                        F_PP[1] = (EPS_P * CIJ * (q * q) + e) * dy / D_PP;
                    }
                }
                a->fcol[0] = a->fcol[0] + F_PP[0];
                a->fcol[1] = a->fcol[1] + F_PP[1];
                b->fcol[0] = b->fcol[0] - F_PP[0];
                b->fcol[1] = b->fcol[1] - F_PP[1];
            }
    }
    if (p->wall_model != LBM_WALL_NONE) {
        for (int ip = 0; ip < o->np; ++ip) {
            disk_t* d = &o->disk[ip];
            real x = d->center[0], y = d->center[1], D = d->diam;
            for (int iw = 1; iw <= 4; ++iw) {
                real R_W[2];
                if (p->wall_model == LBM_WALL_MIRROR) { /* C1:737-745 */
                    if (iw == 1) { R_W[0] = x; R_W[1] = -y; }
                    else if (iw == 2) { R_W[0] = 2.0 * (real)o->nx - x; R_W[1] = y; }
                    else if (iw == 3) { R_W[0] = x; R_W[1] = p->wall_mirror_top - y; }
                    else { R_W[0] = p->wall_mirror_left - x; R_W[1] = y; }
                } else { /* C3:775-783 */
                    if (iw == 1) { R_W[0] = x; R_W[1] = -0.5 * D; }
                    else if (iw == 2) { R_W[0] = (real)o->nx + 0.5 * D; R_W[1] = y; }
                    else if (iw == 3) { R_W[0] = x; R_W[1] = (real)o->ny + 0.5 * D; }
                    else { R_W[0] = -0.5 * D; R_W[1] = y; }
                }
                real ex = x - R_W[0], ey = y - R_W[1];
                D_PW = sqrt(ex * ex + ey * ey);
                real F_PW[2] = {0.0, 0.0};
                if (D_PW > D + ZITA) {
                    F_PW[0] = 0.0;
                    F_PW[1] = 0.0;
                } else {
                    real q = (D_PW - D - ZITA) / ZITA;
                    if (D_PW <= D + ZITA && D_PW > D) {
                        F_PW[0] = EPS_W * CIJ * (q * q) * ex / D_PW;
                        F_PW[1] = EPS_W * CIJ * (q * q) * ey / D_PW;
                    } else if (D_PW <= D) {
                        real e = E_W * CIJ * (D - D_PW) / ZITA;
                        F_PW[0] = (EPS_W * CIJ * (q * q) + e) * ex / D_PW;
                        F_PW[1] = (EPS_W * CIJ * (q * q) + e) * ey / D_PW;
                    }
                }
                d->fcol[0] = d->fcol[0] + F_PW[0];
                d->fcol[1] = d->fcol[1] + F_PW[1];
            }
        }
    }
    o->stale_dpw = D_PW;
}

/* ---- Newton-Euler update inline in MAIN, C1:247-259, C6:300-312 ------- */
static void particle_update(oracle* o) {
    const real RHO0 = o->p.rho0, A_G = o->p.gravity;
    for (int ip = 0; ip < o->np; ++ip) {
        disk_t* d = &o->disk[ip];
        real* V = d->vel;
        real* VO = d->vp_old;
        real* FH = d->fh_in;
        if (o->p.motion == LBM_MOTION_OSCILLATE) {
            /* prescribed oscillation, C4:222-228; F_H_IN of this step's
             * change, C4:270-272 */
            VO[0] = V[0]; VO[1] = V[1]; VO[2] = V[2];
            V[0] = -(o->p.osc_u * cos(((2.0 * o->p.pi) * (real)o->kk) / o->p.osc_period));
            V[1] = 0.0;
            V[2] = 0.0;
            d->center[0] = d->center[0] + 0.5 * (V[0] + VO[0]);
            d->center[1] = d->center[1] + 0.5 * (V[1] + VO[1]);
            FH[0] = (RHO0 / d->rho_p) * d->m_p * (V[0] - VO[0]);
            FH[1] = (RHO0 / d->rho_p) * d->m_p * (V[1] - VO[1]);
            FH[2] = (RHO0 / d->rho_p) * d->i_p * (V[2] - VO[2]);
            continue;
        }
        FH[0] = (RHO0 / d->rho_p) * d->m_p * (V[0] - VO[0]);
        FH[1] = (RHO0 / d->rho_p) * d->m_p * (V[1] - VO[1]);
        FH[2] = (RHO0 / d->rho_p) * d->i_p * (V[2] - VO[2]);
        VO[0] = V[0]; VO[1] = V[1]; VO[2] = V[2];
        V[0] = V[0] + d->force[0] / d->m_p + FH[0] / d->m_p + d->fcol[0] / d->m_p;
        V[1] = V[1] + d->force[1] / d->m_p + FH[1] / d->m_p + (1.0 - RHO0 / d->rho_p) * A_G +
               d->fcol[1] / d->m_p;
        V[2] = V[2] + d->force[2] / d->i_p + FH[2] / d->i_p;
        d->center[0] = d->center[0] + 0.5 * (V[0] + VO[0]);
        d->center[1] = d->center[1] + 0.5 * (V[1] + VO[1]);
        if (o->p.integrate_angle) d->angle = d->angle + 0.5 * (V[2] + VO[2]);
    }
}

static real mean_density(const oracle* o) {
    real s = 0.0;
    /* SUM(Rho) in array element order (C1:318) */
    for (size_t n = 0; n < o->nn; ++n) s += o->RHO[n];
    return s / (real)((o->nx + 1) * (o->ny + 1));
}

static double* series_push(oracle* o) {
    if (o->series_n == o->series_cap) {
        int32_t cap = o->series_cap ? 2 * o->series_cap : 64;
        double* s = (double*)realloc(o->series, (size_t)cap * o->series_len * sizeof(double));
        if (!s) return NULL;
        o->series = s;
        o->series_cap = cap;
    }
    return &o->series[(size_t)o->series_n++ * o->series_len];
}

/* ---- one pass of the time loop body, C1:241-319 ----------------------- */
static void one_step(oracle* o) {
    o->kk += 1;
    collision_force(o);
    particle_update(o);
    double* rec = NULL;
    if (o->p.series_every > 0 && o->kk % o->p.series_every == 0 && o->np > 0) {
        rec = series_push(o);
        if (rec) {
            rec[0] = (double)o->kk;
            rec[1] = NAN;
            int nsp = o->p.series_particles < o->np ? o->p.series_particles : o->np;
            for (int ip = 0; ip < nsp; ++ip) {
                const disk_t* d = &o->disk[ip];
                double* r = &rec[LBM_SERIES_HEAD + LBM_SERIES_PER * ip];
                r[0] = RVAL(d->center[0]); r[1] = RVAL(d->center[1]); r[2] = RVAL(d->angle);
                r[3] = RVAL(d->vel[0]); r[4] = RVAL(d->vel[1]); r[5] = RVAL(d->vel[2]);
                r[6] = RVAL(d->force[0]); r[7] = RVAL(d->force[1]); r[8] = RVAL(d->force[2]);
                r[9] = RVAL(d->fh_in[0]); r[10] = RVAL(d->fh_in[1]); r[11] = RVAL(d->fh_in[2]);
            }
        }
    }
    compute_concentration(o);
    collide(o);
    memcpy(o->FPOST, o->F, Q * o->nn * sizeof(real));
    streaming(o);
    if (o->p.bc == LBM_BC_ZOUHE) bc_zouhe(o);
    else if (o->p.bc == LBM_BC_EQUILIBRIUM) bc_equilibrium(o);
    else bc_halfway(o);
    macroscopic(o);
    force_field_spm(o);
    force_hydro(o);
    velocity_corrector(o);
    if (rec) rec[1] = RVAL(mean_density(o));
}

/* ---- public ----------------------------------------------------------- */
/* which: the seeded input of the tangent build (ORACLE_SEED_*, -1 none) */
static int create_impl(const lbm_params* p, const oracle_opts* opt, int which, int disk,
                       oracle** out) {
    if (!p || !out || p->struct_size != (int32_t)sizeof(lbm_params)) return LBM_E_INVALID;
    if (p->nx < 2 || p->ny < 2) return LBM_E_INVALID;
    oracle* o = (oracle*)calloc(1, sizeof(oracle));
    if (!o) return LBM_E_NOMEM;
    o->p = *p;
    if (opt) o->opt = *opt; else o->opt.stale_dpw_init = INFINITY;
    o->nx = p->nx; o->ny = p->ny; o->n1x = p->nx + 1; o->n1y = p->ny + 1;
    o->nn = (size_t)o->n1x * o->n1y;
    o->tau_y = p->tau_y;
    o->nu = p->nu;
#ifdef ORACLE_TANGENT
    o->seed_which = which;
    o->seed_disk = disk;
    if (which == ORACLE_SEED_TAU_Y) o->tau_y.d = 1.0;
    if (which == ORACLE_SEED_NU) o->nu.d = 1.0;
#else
    (void)which;
    (void)disk;
#endif
    o->F = (real*)calloc(Q * o->nn, sizeof(real));
    o->FPOST = (real*)calloc(Q * o->nn, sizeof(real));
    o->FEQ = (real*)calloc(Q * o->nn, sizeof(real));
    o->G = (real*)calloc(2 * o->nn, sizeof(real));
    o->RHO = (real*)calloc(o->nn, sizeof(real));
    o->UX = (real*)calloc(o->nn, sizeof(real));
    o->UY = (real*)calloc(o->nn, sizeof(real));
    o->OMEGA_BN = (real*)calloc(o->nn, sizeof(real));
    o->STRESS = (real*)calloc(3 * o->nn, sizeof(real));
    o->IMAGE = (int32_t*)calloc(o->nn, sizeof(int32_t));
    o->IS_PARTICLE = (uint8_t*)calloc(o->nn, 1);
    if (!o->F || !o->FPOST || !o->FEQ || !o->G || !o->RHO || !o->UX || !o->UY || !o->OMEGA_BN ||
        !o->STRESS || !o->IMAGE || !o->IS_PARTICLE) {
        oracle_destroy(o);
        return LBM_E_NOMEM;
    }
    /* MAIN, C1:112-113, C1:127-130, C1:151, C1:210 */
    o->omega = 1.0 / (3. * o->nu + 0.5);
    if (1.0 / o->omega < 0.5) { oracle_destroy(o); return LBM_E_TAU; }
    for (size_t n = 0; n < o->nn; ++n) o->OMEGA_BN[n] = o->omega;
    initialize(o);
    compute_relaxation(o, o->omega, o->omega_mrt);
    o->stale_dpw = o->opt.stale_dpw_init;
    o->series_len = LBM_SERIES_HEAD + LBM_SERIES_PER * (p->series_particles > 0 ? p->series_particles : 0);
    *out = o;
    return LBM_OK;
}

int oracle_create(const lbm_params* p, const oracle_opts* opt, oracle** out) {
    return create_impl(p, opt, -1, -1, out);
}

#ifdef ORACLE_TANGENT
int oracle_create_tangent(const lbm_params* p, const oracle_opts* opt, int32_t which,
                          int32_t disk, oracle** out) {
    if (which < ORACLE_SEED_TAU_Y || which > ORACLE_SEED_Y0) return LBM_E_INVALID;
    return create_impl(p, opt, which, disk, out);
}
#endif

void oracle_destroy(oracle* o) {
    if (!o) return;
    for (int ip = 0; ip < o->np; ++ip) free(o->disk[ip].phi);
    free(o->disk);
    free(o->F); free(o->FPOST); free(o->FEQ); free(o->G); free(o->RHO); free(o->UX);
    free(o->UY); free(o->OMEGA_BN); free(o->STRESS); free(o->IMAGE); free(o->IS_PARTICLE);
    free(o->U0); free(o->V0);
    free(o->series);
    free(o);
}

int oracle_set_particles(oracle* o, int32_t np, const double* pin) {
    if (!o || np < 0 || (np > 0 && !pin)) return LBM_E_INVALID;
    for (int ip = 0; ip < o->np; ++ip) free(o->disk[ip].phi);
    free(o->disk);
    o->disk = (disk_t*)calloc(np > 0 ? np : 1, sizeof(disk_t));
    if (!o->disk) return LBM_E_NOMEM;
    o->np = np;
    for (int ip = 0; ip < np; ++ip) {
        disk_t* d = &o->disk[ip];
        const double* r = &pin[LBM_PIN * ip];
        d->center[0] = r[0]; d->center[1] = r[1]; d->angle = r[2];
        d->vel[0] = r[3]; d->vel[1] = r[4]; d->vel[2] = r[5];
        d->diam = r[6]; d->rho_p = r[7];
#ifdef ORACLE_TANGENT
        if (ip == o->seed_disk) {
            if (o->seed_which == ORACLE_SEED_RHO_P) d->rho_p.d = 1.0;
            if (o->seed_which == ORACLE_SEED_X0) d->center[0].d = 1.0;
            if (o->seed_which == ORACLE_SEED_Y0) d->center[1].d = 1.0;
        }
#endif
        /* C1:178-179 */
        d->m_p = d->rho_p * o->p.pi * (0.5 * d->diam) * (0.5 * d->diam);
        d->i_p = 0.5 * d->m_p * (0.5 * d->diam) * (0.5 * d->diam);
        if (!o->opt.phi_on_the_fly) {
            d->phi = (real*)calloc(o->nn, sizeof(real));
            if (!d->phi) return LBM_E_NOMEM;
        }
    }
    compute_concentration(o);
    return LBM_OK;
}

int oracle_step(oracle* o, int32_t nsteps) {
    if (!o || nsteps < 0) return LBM_E_INVALID;
    for (int32_t s = 0; s < nsteps; ++s) one_step(o);
    return LBM_OK;
}

int64_t oracle_kk(const oracle* o) { return o ? o->kk : -1; }

/* one disk's output record (LBM_POUT values) through get (value or derivative) */
#define PARTICLE_RECORD(r, d, get)                                                  \
    do {                                                                            \
        r[0] = get(d->center[0]); r[1] = get(d->center[1]); r[2] = get(d->angle);   \
        r[3] = get(d->vel[0]); r[4] = get(d->vel[1]); r[5] = get(d->vel[2]);        \
        r[6] = get(d->force[0]); r[7] = get(d->force[1]); r[8] = get(d->force[2]);  \
        r[9] = get(d->fcol[0]); r[10] = get(d->fcol[1]);                            \
        r[11] = get(d->fh_in[0]); r[12] = get(d->fh_in[1]); r[13] = get(d->fh_in[2]); \
        r[14] = get(d->m_p); r[15] = get(d->i_p);                                   \
    } while (0)

int oracle_get_particles(oracle* o, double* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (int ip = 0; ip < o->np; ++ip) {
        const disk_t* d = &o->disk[ip];
        double* r = &out[LBM_POUT * ip];
        PARTICLE_RECORD(r, d, RVAL);
    }
    return LBM_OK;
}

#ifdef ORACLE_TANGENT
/* the derivative of every value oracle_get_particles returns, with respect
 * to the seeded input */
int oracle_get_particles_tangent(oracle* o, double* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (int ip = 0; ip < o->np; ++ip) {
        const disk_t* d = &o->disk[ip];
        double* r = &out[LBM_POUT * ip];
        PARTICLE_RECORD(r, d, RDER);
    }
    return LBM_OK;
}
#endif

int oracle_get_state_particles(oracle* o, double* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (int ip = 0; ip < o->np; ++ip) {
        const disk_t* d = &o->disk[ip];
        double* r = &out[LBM_STATE_PER * ip];
        memset(r, 0, LBM_STATE_PER * sizeof(double));
        r[0] = RVAL(d->center[0]); r[1] = RVAL(d->center[1]); r[2] = RVAL(d->angle);
        r[3] = RVAL(d->vel[0]); r[4] = RVAL(d->vel[1]); r[5] = RVAL(d->vel[2]);
        r[6] = RVAL(d->vp_old[0]); r[7] = RVAL(d->vp_old[1]); r[8] = RVAL(d->vp_old[2]);
        r[9] = RVAL(d->force[0]); r[10] = RVAL(d->force[1]); r[11] = RVAL(d->force[2]);
        r[12] = RVAL(d->fcol[0]); r[13] = RVAL(d->fcol[1]);
        r[14] = RVAL(d->fh_in[0]); r[15] = RVAL(d->fh_in[1]); r[16] = RVAL(d->fh_in[2]);
        r[17] = RVAL(d->diam); r[18] = RVAL(d->rho_p);
    }
    return LBM_OK;
}

int oracle_get_field(oracle* o, int32_t which, double* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (size_t n = 0; n < o->nn; ++n) {
        real v;
        switch (which) {
        case LBM_FIELD_UX: v = o->UX[n]; break;
        case LBM_FIELD_UY: v = o->UY[n]; break;
        case LBM_FIELD_RHO: v = o->RHO[n]; break;
        case LBM_FIELD_GX: v = o->G[2 * n]; break;
        case LBM_FIELD_GY: v = o->G[2 * n + 1]; break;
        case LBM_FIELD_TAU11: v = o->STRESS[3 * n]; break;
        case LBM_FIELD_TAU22: v = o->STRESS[3 * n + 1]; break;
        case LBM_FIELD_TAU12: v = o->STRESS[3 * n + 2]; break;
        case LBM_FIELD_OMEGA: v = o->OMEGA_BN[n]; break;
        case LBM_FIELD_PHI: {
            int i = (int)(n % o->n1x), j = (int)(n / o->n1x);
            v = 0.0;
            for (int ip = 0; ip < o->np; ++ip) v += get_phi(o, &o->disk[ip], i, j);
            break;
        }
        default: return LBM_E_INVALID;
        }
        out[n] = RVAL(v);
    }
    return LBM_OK;
}

int oracle_get_image(oracle* o, int32_t* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (size_t n = 0; n < o->nn; ++n)
        out[n] = o->IS_PARTICLE[n] ? 10 : (o->p.rheology == LBM_BINGHAM ? o->IMAGE[n] : 0);
    return LBM_OK;
}

int oracle_get_f(oracle* o, double* out) {
    if (!o || !out) return LBM_E_INVALID;
    for (size_t k = 0; k < Q * o->nn; ++k) out[k] = RVAL(o->F[k]);
    return LBM_OK;
}

int oracle_get_next_post_collision(oracle* o, double* out, double* omega_out) {
    if (!o || !out) return LBM_E_INVALID;
    /* run Collision_MRT of the next step on copies (it does not depend on
     * the particle update that precedes it in the loop) */
    real* F = o->F;
    real* OM = o->OMEGA_BN;
    real* ST = o->STRESS;
    int32_t* IM = o->IMAGE;
    real mrt[Q];
    memcpy(mrt, o->omega_mrt, sizeof mrt);
    real* Fc = (real*)malloc(Q * o->nn * sizeof(real));
    real* Oc = (real*)malloc(o->nn * sizeof(real));
    real* Sc = (real*)malloc(3 * o->nn * sizeof(real));
    int32_t* Ic = (int32_t*)malloc(o->nn * sizeof(int32_t));
    if (!Fc || !Oc || !Sc || !Ic) { free(Fc); free(Oc); free(Sc); free(Ic); return LBM_E_NOMEM; }
    real* FE = o->FEQ;
    real* FEc = (real*)malloc(Q * o->nn * sizeof(real));
    if (!FEc) { free(Fc); free(Oc); free(Sc); free(Ic); return LBM_E_NOMEM; }
    memcpy(FEc, FE, Q * o->nn * sizeof(real));
    memcpy(Fc, F, Q * o->nn * sizeof(real));
    memcpy(Oc, OM, o->nn * sizeof(real));
    o->F = Fc; o->OMEGA_BN = Oc; o->STRESS = Sc; o->IMAGE = Ic; o->FEQ = FEc;
    collide(o);
    for (size_t k = 0; k < Q * o->nn; ++k) out[k] = RVAL(Fc[k]);
    if (omega_out)
        for (size_t n = 0; n < o->nn; ++n) omega_out[n] = RVAL(Oc[n]);
    o->F = F; o->OMEGA_BN = OM; o->STRESS = ST; o->IMAGE = IM; o->FEQ = FE;
    memcpy(o->omega_mrt, mrt, sizeof mrt);
    free(Fc); free(Oc); free(Sc); free(Ic); free(FEc);
    return LBM_OK;
}

int oracle_series_record_len(const oracle* o) { return o ? o->series_len : 0; }

int oracle_get_series(oracle* o, double* out, int32_t max_records, int32_t* nrec) {
    if (!o || !nrec) return LBM_E_INVALID;
    int32_t n = o->series_n < max_records ? o->series_n : max_records;
    if (n > 0 && out) memcpy(out, o->series, (size_t)n * o->series_len * sizeof(double));
    memmove(o->series, o->series + (size_t)n * o->series_len,
            (size_t)(o->series_n - n) * o->series_len * sizeof(double));
    o->series_n -= n;
    *nrec = n;
    return LBM_OK;
}

double oracle_mean_density(oracle* o) { return o ? RVAL(mean_density(o)) : NAN; }

/* ---- COMPUTEERROR, C1:1592-1612 (called at MOD(KK,1000)==0, C1:321-325):
 * I outer, J inner; U0/V0 hold the velocity of the previous call and start
 * as the INITIALIZE velocity, zero (C1:154-155). */
int oracle_compute_error(oracle* o, double* er) {
    if (!o || !er) return LBM_E_INVALID;
    if (!o->U0) {
        o->U0 = (real*)calloc(o->nn, sizeof(real));
        o->V0 = (real*)calloc(o->nn, sizeof(real));
        if (!o->U0 || !o->V0) return LBM_E_NOMEM;
    }
    real err1 = 0.0, err2 = 0.0;
    for (int i = 0; i <= o->nx; ++i)
        for (int j = 0; j <= o->ny; ++j) {
            const size_t n = IDX(o, i, j);
            err1 = err1 + ((o->UX[n] - o->U0[n]) * (o->UX[n] - o->U0[n]) +
                           (o->UY[n] - o->V0[n]) * (o->UY[n] - o->V0[n]));
            err2 = err2 + (o->UX[n] * o->UX[n] + o->UY[n] * o->UY[n]);
            o->U0[n] = o->UX[n];
            o->V0[n] = o->UY[n];
        }
    *er = RVAL(sqrt(err1 / err2));
    return LBM_OK;
}
