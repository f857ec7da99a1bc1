// lbm_lattice.cuh -- the fused lattice kernel of one time step (sm_100a).
//
// One launch per time step k does, for every node in one pass over HBM:
//   pull-stream the stored post-collision populations f*(k)     C1:1181-1217
//   boundary conditions (Zou-He edges / half-way bounce-back)    C1:1222-1417,
//                                                                C6:1195-1390
//   macroscopic rho, u                                           C1:1421-1439
//   SPM solid fraction and body force G (last particle wins)     C1:407-542
//   per-tile partial sums of the hydrodynamic force and torque   C1:546-570
//   velocity correction u += G/2                                 C1:1138-1152
//   MRT collision of step k+1 (+ Papanastasiou viscosity)        C1:875-1048,
//                                                                C6:867-1021
// and writes f*(k+1).  The collision of step k+1 only reads quantities of
// step k (rho, corrected u, G, per-node omega), which is why it can run in the
// same pass as the streaming of step k (C1:292-315 data flow).  Each warp
// adds its (force, torque) sums into exact fixed-point accumulators per
// particle, so results do not depend on block scheduling.
//
// Precision policies:
//   double -- plain populations f, operation order of the reference; the TU
//             is compiled with --fmad=false so products are not contracted.
//   float  -- shifted populations h = f - w_k*rho0 in FP32, FP32 arithmetic;
//             force/torque/mass reductions in FP64.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "lbm_internal.h"

namespace lbm {

enum { MODE_STEP = 0, MODE_OUTPUT = 1, MODE_INIT = 2, MODE_RESTART = 3 };

// exact D2Q9 weights for the shift of the FP32 representation
__device__ __forceinline__ double wexact(int k) {
  return k == 0 ? 4.0 / 9.0 : (k < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
}

// ---------------------------------------------------------------------------
// COMPUTEFEQNEW (C1:1157-1175) in double.
__device__ __forceinline__ void feq_double(const Model& m, double ux, double uy, double rho,
                                           double* feq) {
  const double W0 = m.w_init[0], W1 = m.w_init[1], W2 = m.w_init[2];
  const double U2 = ux * ux + uy * uy;
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

// ---------------------------------------------------------------------------
// Equilibrium boundary (C4:1219-1275): each edge node takes COMPUTEFEQNEW of
// the density and corrected velocity its inward neighbour had in the
// previous step (corners: the diagonal neighbour).  Those values of the
// nodes next to the edges are kept in a ring, one per step parity:
// [par][rho | ux | uy][slot], slots: row j = 1 at i, row j = NY-1 at
// NX+1+i, column i = 1 at 2(NX+1)+j, column i = NX-1 at 2(NX+1)+NY+1+j.
__device__ __forceinline__ int ring_edge_slot(const Geometry& g, int i, int j) {
  const int ii = i < 1 ? 1 : (i > g.nx - 1 ? g.nx - 1 : i);
  if (j == 0) return ii;
  if (j == g.ny) return g.nx + 1 + ii;
  if (i == 0) return 2 * (g.nx + 1) + j;
  return 2 * (g.nx + 1) + g.ny + 1 + j;  // i == NX
}

template <class T>
__device__ __forceinline__ void ring_store(const LatticeArgs& a, int i, int j, int par, T r,
                                           T ux, T uy) {
  const Geometry& g = a.g;
  if (i < 1 || i > g.nx - 1 || j < 1 || j > g.ny - 1) return;
  T* q = static_cast<T*>(a.ring) + (long long)par * 3 * a.ring_n;
  const int n = a.ring_n;
  if (j == 1) { q[i] = r; q[n + i] = ux; q[2 * n + i] = uy; }
  if (j == g.ny - 1) { const int s = g.nx + 1 + i; q[s] = r; q[n + s] = ux; q[2 * n + s] = uy; }
  if (i == 1) { const int s = 2 * (g.nx + 1) + j; q[s] = r; q[n + s] = ux; q[2 * n + s] = uy; }
  if (i == g.nx - 1) {
    const int s = 2 * (g.nx + 1) + g.ny + 1 + j;
    q[s] = r; q[n + s] = ux; q[2 * n + s] = uy;
  }
}

// COMPUTEFEQNEW (C1:1157-1175) in the FP32 shifted form, from dr = rho - rho0:
// h_k = W_k (dr B_k + rho0 (B_k - B_k(0))) + rho0 (W_k B_k(0) - w_k), B_k the
// bracket of COMPUTEFEQNEW, so no O(1) terms cancel.
__device__ __forceinline__ void feq_shift32(const Model& m, float dr, float x, float y, float* h) {
  const float r0 = m.rho0_f;
  const float U2 = x * x + y * y;
  float d[9];  // B_k - B_k(0)
  d[0] = -3.f * U2;
  d[1] = 6.f * x + 9.f * x * x - 3.f * U2;
  d[2] = 6.f * y + 9.f * y * y - 3.f * U2;
  d[3] = -6.f * x + 9.f * x * x - 3.f * U2;
  d[4] = -6.f * y + 9.f * y * y - 3.f * U2;
  d[5] = 3.f * (x + y) + 9.f * x * y + 3.f * U2;
  d[6] = -3.f * (x - y) - 9.f * x * y + 3.f * U2;
  d[7] = -3.f * (x + y) + 9.f * x * y + 3.f * U2;
  d[8] = 3.f * (x - y) - 9.f * x * y + 3.f * U2;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const float W = m.w_init_f[k == 0 ? 0 : (k < 5 ? 1 : 2)];
    const float B = (k == 0 || k < 5 ? 2.f : 1.f) + d[k];
    h[k] = W * (dr * B + r0 * d[k]) + m.eq_c_f[k];
  }
}

// ComputeSourceEquilib_Hydro's forcing (C1:843-870, G_X = G_Y = 0).
template <class T>
__device__ __forceinline__ void bgk_source(const T* W, T rho, T ux, T uy, T gx, T gy, T* FI) {
  gx = gx + (T)0.0;
  gy = gy + (T)0.0;
  FI[0] = W[0] * rho * (-((T)3 * ux * gx) - (T)3 * uy * gy);
  FI[1] = W[1] * rho * (((T)3 + (T)6 * ux) * gx - (T)3 * uy * gy);
  FI[2] = W[1] * rho * (-((T)3 * ux * gx) + ((T)3 + (T)6 * uy) * gy);
  FI[3] = W[1] * rho * (((T)-3 + (T)6 * ux) * gx - (T)3 * uy * gy);
  FI[4] = W[1] * rho * (-((T)3 * ux * gx) + ((T)-3 + (T)6 * uy) * gy);
  FI[5] = W[2] * rho * (((T)3 + (T)6 * ux + (T)9 * uy) * gx + ((T)3 + (T)9 * ux + (T)6 * uy) * gy);
  FI[6] = W[2] * rho * (((T)-3 + (T)6 * ux - (T)9 * uy) * gx + ((T)3 - (T)9 * ux + (T)6 * uy) * gy);
  FI[7] = W[2] * rho * (((T)-3 + (T)6 * ux + (T)9 * uy) * gx + ((T)-3 + (T)9 * ux + (T)6 * uy) * gy);
  FI[8] = W[2] * rho * (((T)3 + (T)6 * ux - (T)9 * uy) * gx + ((T)-3 - (T)9 * ux + (T)6 * uy) * gy);
}

// f of edge node (i, j) from the ring of parity par.  FP64: the reference's
// arithmetic.  FP32 (shifted populations, the ring holding rho - rho0):
// h_k = W_k (drho B_k + rho0 (B_k - B_k(0))) + rho0 (W_k B_k(0) - w_k), with
// B_k the bracket of COMPUTEFEQNEW, so no O(1) terms cancel.
template <class T>
__device__ __forceinline__ void edge_equilibrium(const LatticeArgs& a, int i, int j, int par,
                                                 T* f) {
  const int s = ring_edge_slot(a.g, i, j), n = a.ring_n;
  const T* q = static_cast<const T*>(a.ring) + (long long)par * 3 * n;
  const T r = q[s], ux = q[n + s], uy = q[2 * n + s];
  if (sizeof(T) == 8) {
    double fe[9];
    feq_double(a.m, (double)ux, (double)uy, (double)r, fe);
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (T)fe[k];
    return;
  }
  float h[9];
  feq_shift32(a.m, (float)r, (float)ux, (float)uy, h);
#pragma unroll
  for (int k = 0; k < 9; ++k) f[k] = (T)h[k];
}

// ComputeRelaxation_MRT (C1:1029-1048 fixed q; C6:1002-1021 q of omega).
__device__ __forceinline__ void rates_double(const Model& m, double omega, double* S) {
  const double oq = m.q_of_omega ? 8. * (2. - omega) / (8. - omega) : m.s_q;
  S[0] = 0.0; S[1] = m.s_e; S[2] = m.s_eps; S[3] = 0.0;
  S[4] = oq; S[5] = 0.0; S[6] = oq; S[7] = omega; S[8] = omega;
}

// ---------------------------------------------------------------------------
// SPM solid fraction of one node for one disk (C1:464-476).
__device__ __forceinline__ double phi_double(double di, double dj, double R, double zeta,
                                             double pi) {
  const double D = R - sqrt(di * di + dj * dj);
  double phi = 0.0;
  if (D <= -0.5 * zeta)
    phi = 0.0;
  else if (fabs(D) < 0.5 * zeta)
    phi = 0.5 * (sin(pi * D / zeta) + 1.0);
  else if (D >= 0.5 * zeta)
    phi = 1.0;
  return phi;
}

__device__ __forceinline__ float phi_float(float di, float dj, float R, float zeta, float pi) {
  const float D = R - sqrtf(di * di + dj * dj);
  float phi = 0.0f;
  if (D <= -0.5f * zeta)
    phi = 0.0f;
  else if (fabsf(D) < 0.5f * zeta)
    phi = 0.5f * (__sinf(pi * D / zeta) + 1.0f);  // |argument| < pi/2
  else if (D >= 0.5f * zeta)
    phi = 1.0f;
  return phi;
}

// ---------------------------------------------------------------------------
// Collision_MRT for one node in plain FP64 (C1:886-921; Chai strain rate and
// Papanastasiou viscosity C6:903-958).  Same operations, same order as the
// reference.  Returns the new omega and writes stress / yield code.
struct NodeOut {
  double t11, t22, t12, omega;
  int yield;
};

__device__ __forceinline__ void collide_double(const Model& m, double* f, double RHO, double UX,
                                               double UY, double GX, double GY, const double* S,
                                               bool want_stress, NodeOut& no) {
  const double d_mrt = m.d_mrt;
  const double f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3], f4 = f[4], f5 = f[5], f6 = f[6],
               f7 = f[7], f8 = f[8];
  double M[9], MF[9], MEQ[9];
  M[0] = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
  M[1] = -4.0 * f0 - f1 - f2 - f3 - f4 + 2.0 * (f5 + f6 + f7 + f8);
  M[2] = 4.0 * f0 - 2.0 * (f1 + f2 + f3 + f4) + (f5 + f6 + f7 + f8);
  M[3] = f1 - f3 + f5 - f6 - f7 + f8;
  M[4] = -2.0 * (f1 - f3) + f5 - f6 - f7 + f8;
  M[5] = f2 - f4 + f5 + f6 - f7 - f8;
  M[6] = -2.0 * (f2 - f4) + f5 + f6 - f7 - f8;
  M[7] = f1 - f2 + f3 - f4;
  M[8] = f5 - f6 + f7 - f8;
  const double F_X = RHO * (GX + 0.0), F_Y = RHO * (GY + 0.0);
  MF[0] = 0.0;
  MF[1] = 6.0 * (F_X * UX + F_Y * UY);
  MF[2] = -6.0 * (F_X * UX + F_Y * UY);
  MF[3] = F_X;
  MF[4] = -F_X;
  MF[5] = F_Y;
  MF[6] = -F_Y;
  MF[7] = 2.0 * (F_X * UX - F_Y * UY);
  MF[8] = F_Y * UX + F_X * UY;
  const double U2 = UX * UX + UY * UY;
  MEQ[0] = RHO;
  MEQ[1] = RHO * (-2.0 + 3. * U2);
  MEQ[2] = RHO * (1.0 - 3. * U2);
  MEQ[3] = RHO * (UX);
  MEQ[4] = RHO * (-UX);
  MEQ[5] = RHO * (UY);
  MEQ[6] = RHO * (-UY);
  MEQ[7] = RHO * (UX * UX - UY * UY);
  MEQ[8] = RHO * (UX * UY);
  double mm[9];
#pragma unroll
  for (int k = 0; k < 9; ++k)
    mm[k] = S[k] * MEQ[k] + (1. - S[k]) * M[k] + (1. - 0.5 * S[k]) * MF[k];
  f[0] = d_mrt * (4.0 * (mm[0] - mm[1] + mm[2]));
  f[1] = d_mrt * (4. * mm[0] - mm[1] - 2. * mm[2] + 6. * mm[3] - 6. * mm[4] + 9. * mm[7]);
  f[2] = d_mrt * (4.0 * mm[0] - mm[1] - 2.0 * mm[2] + 6.0 * mm[5] - 6.0 * mm[6] - 9.0 * mm[7]);
  f[3] = d_mrt * (4.0 * mm[0] - mm[1] - 2.0 * mm[2] - 6.0 * mm[3] + 6.0 * mm[4] + 9.0 * mm[7]);
  f[4] = d_mrt * (4.0 * mm[0] - mm[1] - 2.0 * mm[2] - 6.0 * mm[5] + 6.0 * mm[6] - 9.0 * mm[7]);
  f[5] = d_mrt * (4.0 * mm[0] + 2.0 * mm[1] + mm[2] + 6.0 * mm[3] + 3.0 * mm[4] + 6.0 * mm[5] +
                  3.0 * mm[6] + 9.0 * mm[8]);
  f[6] = d_mrt * (4.0 * mm[0] + 2.0 * mm[1] + mm[2] - 6.0 * mm[3] - 3.0 * mm[4] + 6.0 * mm[5] +
                  3.0 * mm[6] - 9.0 * mm[8]);
  f[7] = d_mrt * (4.0 * mm[0] + 2.0 * mm[1] + mm[2] - 6.0 * mm[3] - 3.0 * mm[4] - 6.0 * mm[5] -
                  3.0 * mm[6] + 9.0 * mm[8]);
  f[8] = d_mrt * (4.0 * mm[0] + 2.0 * mm[1] + mm[2] + 6.0 * mm[3] + 3.0 * mm[4] - 6.0 * mm[5] -
                  3.0 * mm[6] - 9.0 * mm[8]);
  if (!want_stress) return;
  // Chai strain rate from S*(m - m_eq) + forcing correction, C6:903-916
  double MNE[9], F1[9];
  if (m.strain_feq) {  // C1:896-908: against the moments of COMPUTEFEQNEW
    double FE[9];
    feq_double(m, UX, UY, RHO, FE);
    MNE[0] = M[0] - (FE[0] + FE[1] + FE[2] + FE[3] + FE[4] + FE[5] + FE[6] + FE[7] + FE[8]);
    MNE[1] = M[1] - (-4.0 * FE[0] - FE[1] - FE[2] - FE[3] - FE[4] + 2.0 * (FE[5] + FE[6] + FE[7] + FE[8]));
    MNE[2] = M[2] - (4.0 * FE[0] - 2.0 * (FE[1] + FE[2] + FE[3] + FE[4]) + (FE[5] + FE[6] + FE[7] + FE[8]));
    MNE[3] = M[3] - (FE[1] - FE[3] + FE[5] - FE[6] - FE[7] + FE[8]);
    MNE[4] = M[4] - (-2.0 * (FE[1] - FE[3]) + FE[5] - FE[6] - FE[7] + FE[8]);
    MNE[5] = M[5] - (FE[2] - FE[4] + FE[5] + FE[6] - FE[7] - FE[8]);
    MNE[6] = M[6] - (-2.0 * (FE[2] - FE[4]) + FE[5] + FE[6] - FE[7] - FE[8]);
    MNE[7] = M[7] - (FE[1] - FE[2] + FE[3] - FE[4]);
    MNE[8] = M[8] - (FE[5] - FE[6] + FE[7] - FE[8]);
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) MNE[k] = M[k] - MEQ[k];
  }
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
  double D11, D22, D12;
  if (m.strain_feq) {  // C1:940-948: 1/RHO folded into both terms
    const double IR = 1.0 / RHO;
    double ZARIB = -1.5 * d_mrt * IR;
    D11 = ZARIB * (F1[1] + F1[5] + F1[6] + F1[3] + F1[7] + F1[8]);
    D22 = ZARIB * (F1[5] + F1[2] + F1[6] + F1[7] + F1[4] + F1[8]);
    D12 = ZARIB * (F1[5] - F1[6] + F1[7] - F1[8]);
    ZARIB = 0.75 * IR;
    D11 = D11 + ZARIB * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GX * UX));
    D22 = D22 + ZARIB * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GY * UY));
    D12 = D12 + ZARIB * (-S[7] * (GX * UY + GY * UX));
  } else {  // C6:903-916
    const double ZARIB = -1.5 * d_mrt;
    D11 = ZARIB * (F1[1] + F1[5] + F1[6] + F1[3] + F1[7] + F1[8]) +
          0.75 * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GX * UX));
    D22 = ZARIB * (F1[5] + F1[2] + F1[6] + F1[7] + F1[4] + F1[8]) +
          0.75 * ((S[7] - S[1]) * (GX * UX + GY * UY) - S[7] * (2.0 * GY * UY));
    D12 = ZARIB * (F1[5] - F1[6] + F1[7] - F1[8]) + 0.75 * (-S[7] * (GX * UY + GY * UX));
  }
  const double NU = m.nu;
  no.t11 = NU * 2.0 * D11;
  no.t22 = NU * 2.0 * D22;
  no.t12 = NU * 2.0 * D12;
  no.yield = 0;
  no.omega = S[7];
  if (m.bingham) {
    const double INV_RHO = 1.0 / RHO;
    if (!m.strain_feq) {
      D11 = D11 * INV_RHO;
      D22 = D22 * INV_RHO;
      D12 = D12 * INV_RHO;
    }
    const double GAMMA = sqrt(2.0 * fabs(D11 * D11 + D22 * D22 + 2.0 * (D12 * D12)));
    double NU_A;
    if (m.casson) {  // C3:985-989
      if (GAMMA < m.gamma_min) {
        NU_A = sqrt(NU) + sqrt(m.m_pap * m.tau_y);
      } else {
        NU_A = sqrt(NU) + sqrt(m.tau_y / GAMMA) * (1.0 - exp(-sqrt(m.m_pap * GAMMA)));
        NU_A = NU_A * NU_A;
      }
    } else if (GAMMA < m.gamma_min) {
      NU_A = NU + m.m_pap * m.tau_y;
    } else {
      NU_A = NU + (m.tau_y / GAMMA) * (1.0 - exp(-(m.m_pap * GAMMA)));
    }
    no.t11 = NU_A * 2.0 * D11;
    no.t22 = NU_A * 2.0 * D22;
    no.t12 = NU_A * 2.0 * D12;
    const double TAU_MAG =
        sqrt(0.5 * fabs(no.t11 * no.t11 + no.t22 * no.t22 + 2.0 * (no.t12 * no.t12)));
    no.yield = (TAU_MAG <= m.tau_y) ? 5 : 0;
    NU_A = NU_A * INV_RHO;
    no.omega = 1.0 / (3.0 * NU_A + 0.5);
  }
}

// Relaxation rates of the FP32 update (s_e, s_eps, s_q, s_nu).
struct Rates32 {
  float s1, s2, sq, sw;
};

// ---------------------------------------------------------------------------
// FP32 node update in moment space, on shifted populations h = f - w*rho0.
// Moments of h are m - rho0*(1,-2,1,0,...); the shift cancels in m - m_eq,
// and the inverse transform adds back rho0*w_k*(36*d_mrt - 1) (zero for an
// exact 1/36).  The nine moments are formed once with pair sums/differences
// and serve both the macroscopic variables and the collision, which then
// works on the moments only.
struct Mom32 {
  float drho, jx, jy, m1, m2, m4, m6, m7, m8;
};

__device__ __forceinline__ Mom32 moments32(const float* h) {
  Mom32 q;
  const float a = h[1] + h[3], b = h[2] + h[4], c = h[5] + h[7], d = h[6] + h[8];
  const float e = h[1] - h[3], g = h[2] - h[4], hh = h[5] - h[7], kk = h[6] - h[8];
  const float ab = a + b, cd = c + d;
  const float hmk = hh - kk, hpk = hh + kk;
  q.drho = h[0] + (ab + cd);
  q.jx = e + hmk;
  q.jy = g + hpk;
  q.m1 = fmaf(2.0f, cd, -ab) - 4.0f * h[0];
  q.m2 = fmaf(4.0f, h[0], cd) - 2.0f * ab;
  q.m4 = fmaf(-2.0f, e, hmk);
  q.m6 = fmaf(-2.0f, g, hpk);
  q.m7 = a - b;
  q.m8 = c - d;
  return q;
}

// Relax the moments (rates r, Guo forcing) and transform back to shifted
// populations; optionally the Chai strain rate / Papanastasiou viscosity.
__device__ __forceinline__ void relax32(const Model& m, const Mom32& q, float rho, float ux,
                                        float uy, float gx, float gy, const Rates32& r,
                                        bool want_stress, NodeOut& no, float* h) {
  const float FX = rho * gx, FY = rho * gy;
  const float uxx = ux * ux, uyy = uy * uy;
  const float ru2 = 3.0f * rho * (uxx + uyy);
  const float e1 = fmaf(-2.0f, q.drho, ru2);
  const float e2 = q.drho - ru2;
  const float e4 = -rho * ux;
  const float e6 = -rho * uy;
  const float e7 = rho * (uxx - uyy);
  const float e8 = rho * (ux * uy);
  const float fu = fmaf(FX, ux, FY * uy);
  const float cw = 1.0f - 0.5f * r.sw, cq = 1.0f - 0.5f * r.sq;
  const float p0 = q.drho;
  const float p1 = fmaf(r.s1, e1 - q.m1, q.m1) + (6.0f - 3.0f * r.s1) * fu;
  const float p2 = fmaf(r.s2, e2 - q.m2, q.m2) - (6.0f - 3.0f * r.s2) * fu;
  const float p3 = q.jx + FX;
  const float p5 = q.jy + FY;
  const float p4 = fmaf(r.sq, e4 - q.m4, q.m4) - cq * FX;
  const float p6 = fmaf(r.sq, e6 - q.m6, q.m6) - cq * FY;
  const float p7 = fmaf(r.sw, e7 - q.m7, q.m7) + cw * (2.0f * fmaf(FX, ux, -FY * uy));
  const float p8 = fmaf(r.sw, e8 - q.m8, q.m8) + cw * fmaf(FY, ux, FX * uy);
  const float d = m.d_mrt_f;
  const float A = fmaf(4.0f, p0, -p1) - 2.0f * p2;
  const float B = fmaf(4.0f, p0, 2.0f * p1) + p2;
  const float X = 6.0f * (p3 - p4), Y = 6.0f * (p5 - p6);
  const float X2 = fmaf(6.0f, p3, 3.0f * p4), Y2 = fmaf(6.0f, p5, 3.0f * p6);
  const float P7 = 9.0f * p7, P8 = 9.0f * p8;
  const float AP = A + P7, AM = A - P7, BP = B + P8, BM = B - P8;
  const float XpY = X2 + Y2, XmY = X2 - Y2;
  h[0] = fmaf(d, 4.0f * (p0 - p1 + p2), m.shift_f[0]);
  h[1] = fmaf(d, AP + X, m.shift_f[1]);
  h[3] = fmaf(d, AP - X, m.shift_f[3]);
  h[2] = fmaf(d, AM + Y, m.shift_f[2]);
  h[4] = fmaf(d, AM - Y, m.shift_f[4]);
  h[5] = fmaf(d, BP + XpY, m.shift_f[5]);
  h[7] = fmaf(d, BP - XpY, m.shift_f[7]);
  h[6] = fmaf(d, BM - XmY, m.shift_f[6]);
  h[8] = fmaf(d, BM + XmY, m.shift_f[8]);
  if (!want_stress) return;
  // closed form of the Chai strain rate (C6:903-916) with S0 = S3 = S5 = 0
  const float n1 = q.m1 - e1, n7 = q.m7 - e7, n8 = q.m8 - e8;
  const float t1 = 9.0f * r.s1 * n1, t7 = 27.0f * r.sw * n7;
  const float gu = gx * ux + gy * uy;
  float D11 = -d * (t1 + t7) + 0.75f * ((r.sw - r.s1) * gu - r.sw * (2.0f * gx * ux));
  float D22 = -d * (t1 - t7) + 0.75f * ((r.sw - r.s1) * gu - r.sw * (2.0f * gy * uy));
  float D12 = -54.0f * d * r.sw * n8 + 0.75f * (-r.sw * (gx * uy + gy * ux));
  if (m.strain_feq) {  // C1:940-948 divides both terms by rho (FP32: the
    // moments of COMPUTEFEQNEW equal the moment-space equilibrium here)
    const float ir = 1.0f / rho;
    D11 *= ir;
    D22 *= ir;
    D12 *= ir;
  }
  const float NU = m.nu_f;
  no.t11 = NU * 2.0f * D11;
  no.t22 = NU * 2.0f * D22;
  no.t12 = NU * 2.0f * D12;
  no.yield = 0;
  no.omega = r.sw;
  if (m.bingham) {
    // The divisions and the square root of the strain rate use the hardware
    // approximations (relative errors of a few 2^-23, far below the FP32
    // populations' own rounding after the collision); 1 - e^(-m gamma) keeps
    // expm1f, whose accuracy at small m gamma the plug regions need.
    const float inv_rho = __fdividef(1.0f, rho);
    if (!m.strain_feq) {
      D11 *= inv_rho;
      D22 *= inv_rho;
      D12 *= inv_rho;
    }
    const float g2 = 2.0f * fabsf(D11 * D11 + D22 * D22 + 2.0f * (D12 * D12));
    const float gam = g2 > 0.0f ? g2 * rsqrtf(g2) : 0.0f;
    const float ty = m.tau_y_f;
    float nua;
    if (m.casson) {
      if (gam < m.gamma_min_f) {
        nua = sqrtf(NU) + sqrtf(m.m_pap_f * ty);
      } else {
        nua = sqrtf(NU) + sqrtf(ty / gam) * -expm1f(-sqrtf(m.m_pap_f * gam));
        nua = nua * nua;
      }
    } else if (gam < m.gamma_min_f) {
      nua = NU + m.m_pap_f * ty;
    } else {
      // 1 - e^(-m gamma) by expm1f: no cancellation where m gamma is small;
      // above m gamma = 18 it rounds to exactly 1 in FP32 (e^-18 < 2^-25),
      // so yielded fluid skips the exponential
      const float mg = m.m_pap_f * gam;
      nua = NU + __fdividef(ty, gam) * (mg > 18.0f ? 1.0f : -expm1f(-mg));
    }
    const float t11 = nua * 2.0f * D11, t22 = nua * 2.0f * D22, t12 = nua * 2.0f * D12;
    no.t11 = t11;
    no.t22 = t22;
    no.t12 = t12;
    if (m.record_stress) {  // the yield flag is kept only with the stress record
      const float tm = sqrtf(0.5f * fabsf(t11 * t11 + t22 * t22 + 2.0f * (t12 * t12)));
      no.yield = (tm <= ty) ? 5 : 0;
    }
    no.omega = __fdividef(1.0f, 3.0f * (nua * inv_rho) + 0.5f);
  }
}

// ---------------------------------------------------------------------------
// Pull streaming + boundary conditions for one node.  Sources outside the
// lattice keep the node's own post-collision value (C1:1195-1199); the
// boundary routine then overwrites the unknowns.  Wall velocities are zero
// in every reference case, which reduces the moving-wall terms to +-0.
template <class T>
__device__ __forceinline__ void pull_bc(const T* __restrict__ src, const Geometry& g, int bc,
                                        int i, int j, T* f) {
  const long long P = g.plane;
  const long long n = (long long)j * g.pitch + i;
  const int pt = g.pitch;
  const bool L = (i == 0), R = (i == g.nx), B = (j == 0), U = (j == g.ny);
  const T* s0 = src + n;
  f[0] = s0[0];
  f[1] = !L ? s0[plane_of(1) * P - 1] : s0[plane_of(1) * P];
  f[2] = !B ? s0[plane_of(2) * P - pt] : s0[plane_of(2) * P];
  f[3] = !R ? s0[plane_of(3) * P + 1] : s0[plane_of(3) * P];
  f[4] = !U ? s0[plane_of(4) * P + pt] : s0[plane_of(4) * P];
  f[5] = (!L && !B) ? s0[plane_of(5) * P - pt - 1] : s0[plane_of(5) * P];
  f[6] = (!R && !B) ? s0[plane_of(6) * P - pt + 1] : s0[plane_of(6) * P];
  f[7] = (!R && !U) ? s0[plane_of(7) * P + pt + 1] : s0[plane_of(7) * P];
  f[8] = (!L && !U) ? s0[plane_of(8) * P + pt - 1] : s0[plane_of(8) * P];
  if (!(L || R || B || U)) return;
  // own post-collision populations F_POST(k,i,j)
#define FPOST(k) src[plane_of(k) * P + n]
  if ((L || R) && (B || U)) {
    // corners: half-way bounce-back of 3 of the 5 unknowns (C1:1390-1414)
    if (L && B) { f[1] = FPOST(3); f[5] = FPOST(7); f[2] = FPOST(4); }
    else if (L && U) { f[1] = FPOST(3); f[8] = FPOST(6); f[4] = FPOST(2); }
    else if (R && U) { f[3] = FPOST(1); f[7] = FPOST(5); f[4] = FPOST(2); }
    else { f[2] = FPOST(4); f[6] = FPOST(8); f[3] = FPOST(1); }
    return;
  }
  if (bc == 1 /* LBM_BC_HALFWAY_BB, C6:1206-1219, C6:1285-1294 */) {
    if (U) { f[8] = FPOST(6); f[4] = FPOST(2); f[7] = FPOST(5); }
    else if (B) { f[5] = FPOST(7); f[2] = FPOST(4); f[6] = FPOST(8); }
    else if (R) { f[6] = FPOST(8); f[3] = FPOST(1); f[7] = FPOST(5); }
    else { f[5] = FPOST(7); f[1] = FPOST(3); f[8] = FPOST(6); }
  } else { /* Zou-He, C1:1250-1258 (top/bottom), C1:1341-1363 (left/right) */
    if (U) {
      f[4] = f[2];
      f[8] = f[6] - (T)0.5 * (f[1] - f[3]);
      f[7] = f[5] + (T)0.5 * (f[1] - f[3]);
    } else if (B) {
      f[2] = f[4];
      f[5] = f[7] - (T)0.5 * (f[1] - f[3]);
      f[6] = f[8] + (T)0.5 * (f[1] - f[3]);
    } else if (L) {
      f[5] = f[7] - (T)0.5 * (f[2] - f[4]);
      f[8] = f[6] + (T)0.5 * (f[2] - f[4]);
      f[1] = f[3];
    } else {
      f[6] = f[8] - (T)0.5 * (f[2] - f[4]);
      f[7] = f[5] + (T)0.5 * (f[2] - f[4]);
      f[3] = f[1];
    }
  }
#undef FPOST
}

template <class T>
__device__ __forceinline__ void pull_interior(const T* __restrict__ src, const Geometry& g,
                                              long long n, T* f) {
  const long long P = g.plane;
  const int pt = g.pitch;
  const T* s0 = src + n;
  f[0] = s0[0];
  f[1] = s0[plane_of(1) * P - 1];
  f[2] = s0[plane_of(2) * P - pt];
  f[3] = s0[plane_of(3) * P + 1];
  f[4] = s0[plane_of(4) * P + pt];
  f[5] = s0[plane_of(5) * P - pt - 1];
  f[6] = s0[plane_of(6) * P - pt + 1];
  f[7] = s0[plane_of(7) * P + pt + 1];
  f[8] = s0[plane_of(8) * P + pt - 1];
}

// ---------------------------------------------------------------------------
// Warp sums of three values with 12 shuffles instead of 30: after the
// exchange over lane bit 4 a lane keeps two of four partial sums (the fourth
// is zero), after bit 3 one, then three plain levels.  Returns the total of
// a in lanes 0-7, of b in lanes 8-15, of c in lanes 16-23.
__device__ __forceinline__ double warp_sum3(double a, double b, double c, int lane) {
  const bool hi = (lane & 16) != 0, mid = (lane & 8) != 0;
  double k0 = hi ? c : a, k1 = hi ? 0.0 : b;
  const double s0 = hi ? a : c, s1 = hi ? b : 0.0;
  k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
  k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
  double k = mid ? k1 : k0;
  k += __shfl_xor_sync(0xffffffffu, mid ? k0 : k1, 8);
  k += __shfl_xor_sync(0xffffffffu, k, 4);
  k += __shfl_xor_sync(0xffffffffu, k, 2);
  k += __shfl_xor_sync(0xffffffffu, k, 1);
  return k;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Exact, order-independent accumulation of a double into two int64 words:
// v = hi*2^-20 + lo*2^-62 (|v| < 2^43).  Integer sums commute, so the
// result does not depend on which warp adds first.
__device__ __forceinline__ void facc_add(unsigned long long* hi, unsigned long long* lo, double v) {
  const double t = v * FHI;
  const double h = floor(t);
  const double l = rint((t - h) * FLO);
  atomicAdd(hi, (unsigned long long)(long long)h);
  atomicAdd(lo, (unsigned long long)(long long)l);
}

#ifndef LBM_MINB_F32
#define LBM_MINB_F32 1
#endif
#ifndef LBM_MINB_F64
#define LBM_MINB_F64 1
#endif

// FP32 node share of the mean-density sum in units of 2^-40: drho rounded to
// a multiple of 2^-30 by a 32-bit conversion (|drho| < 2; beyond that it
// saturates), then widened, which is cheaper than a 64-bit conversion.
__device__ __forceinline__ long long mass_share32(float drho) {
  return (long long)__float2int_rn(drho * 0x1p30f) * 1024;
}

// Lattice health, once per warp and tile: a node whose density is not
// finite (a blow-up anywhere in the fluid, with or without disks nearby)
// sets ST_NAN; in FP32 a finite |rho - rho0| >= 2, beyond the range of
// mass_share32, sets ST_OVERFLOW.  Every lane of the warp calls it; nodes
// outside the lattice pass drho = 0.
template <class T>
__device__ __forceinline__ void lattice_health(int* status, T drho, int lane) {
  const bool bad = sizeof(T) == 8 ? !isfinite((double)drho) : !(fabsf((float)drho) < 2.0f);
  if (__any_sync(0xffffffffu, bad)) {
    const bool nf = __any_sync(0xffffffffu, !isfinite((double)drho));
    if (lane == 0) atomicOr(status, nf ? ST_NAN : ST_OVERFLOW);
  }
}

// One tile of BX x BY nodes (block (bxi, byi) of the lattice), one node per
// thread; BX*BY threads.  The tile lies inside one LTX x LTY list tile.
// mass_local (MODE_STEP): when given, lane 0 adds the warp's fixed-point
// mean-density share there instead of to the history slot (the caller adds
// the total once); integer sums, so the result is the same.
// BGK: whether the body carries the BGK collision at all (a kernel that only
// ever sees MRT models leaves it out and keeps its register budget).
template <class T, int MODE, int BX, int BY, bool BGK = true>
__device__ __forceinline__ void lattice_body(const LatticeArgs& a, int bxi, int byi,
                                             long long* mass_local = nullptr) {
  static_assert(LTX % BX == 0 && LTY % BY == 0 && BX % 32 == 0, "tile inside a list tile");
  constexpr bool F64 = sizeof(T) == 8;
  __shared__ int s_idx[MAX_TILE_CAND];
  __shared__ double s_px[MAX_TILE_CAND], s_py[MAX_TILE_CAND], s_pr[MAX_TILE_CAND];
  __shared__ double s_pu[MAX_TILE_CAND], s_pv[MAX_TILE_CAND], s_pw[MAX_TILE_CAND];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int i = bxi * BX + (tid & (BX - 1));
  const int j = byi * BY + tid / BX;
  const int tile = ((byi * BY) / LTY) * a.g.ltx + (bxi * BX) / LTX;
  const Geometry& g = a.g;
  const Model& m = a.m;
  (void)warp;

  // ---- step number and the particles touching this tile -----------------
  // Every warp reads the count itself, so tiles without particles never wait
  // at a barrier; with particles, warp 0 stages them in shared memory sorted
  // by index (the last particle with PHI>0 sets G, C1:500-507).
  int kk = 0;        // parity of the step number
  int rslot = -1;    // history slot of this step
  int ncand = 0;
  if (MODE != MODE_INIT) {
    int c = 0, buf = 0, kl = 0, rs = -1;
    if (lane == 0) {
      if (MODE == MODE_STEP || MODE == MODE_RESTART) kl = (int)(a.step & 1);
      if (MODE == MODE_STEP) rs = a.rec_slot;
      buf = a.tile_cur[a.step & 1];
      c = a.tile_count[(long long)buf * a.ntiles + tile];
    }
    kk = __shfl_sync(0xffffffffu, kl, 0);
    rslot = __shfl_sync(0xffffffffu, rs, 0);
    c = __shfl_sync(0xffffffffu, c, 0);
    buf = __shfl_sync(0xffffffffu, buf, 0);
    if (c > a.tile_cap) {
      if (tid == 0) atomicOr(a.status, ST_OVERFLOW);
      c = a.tile_cap;
    }
    ncand = c;
    if (ncand > 0) {
      if (tid < 32) {
        const long long tbase = (long long)buf * a.ntiles + tile;
        const int pv = lane < ncand ? a.tile_list[tbase * a.tile_cap + lane] : 0x7fffffff;
        int rank = 0;
#pragma unroll 8
        for (int o = 0; o < 32; ++o) rank += (__shfl_sync(0xffffffffu, pv, o) < pv);
        if (lane < ncand) {
          const PRef p{const_cast<double*>(a.ps) + pv, a.npad};
          s_idx[rank] = pv;
          s_px[rank] = p[P_X];
          s_py[rank] = p[P_Y];
          s_pr[rank] = 0.5 * p[P_D];
          s_pu[rank] = p[P_U];
          s_pv[rank] = p[P_V];
          s_pw[rank] = p[P_W];
        }
      }
      __syncthreads();
    }
  }

  const bool act = (i <= g.nx) && (j <= g.ny);
  const long long n = (long long)j * g.pitch + i;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  const bool initial = (MODE == MODE_INIT) || (MODE == MODE_OUTPUT && a.initial);

  // ---- populations after streaming and boundary conditions -------------
  T f[9];
  if (act) {
    if (initial) {
      double feq[9];
      feq_double(m, 0.0, 0.0, m.rho0, feq);
#pragma unroll
      for (int k = 0; k < 9; ++k) f[k] = F64 ? (T)feq[k] : (T)(feq[k] - wexact(k) * m.rho0);
    } else if (MODE == MODE_RESTART || (MODE == MODE_OUTPUT && a.src_post_bc)) {
#pragma unroll
      for (int k = 0; k < 9; ++k) f[k] = src[plane_of(k) * g.plane + n];
    } else {
      const bool interior = bxi > 0 && byi > 0 && (bxi + 1) * BX <= g.nx &&
                            (byi + 1) * BY <= g.ny;
      const bool on_edge = i == 0 || i == g.nx || j == 0 || j == g.ny;
      if (interior)
        pull_interior<T>(src, g, n, f);
      else if (m.bc == BC_EQUILIBRIUM && on_edge)
        edge_equilibrium<T>(a, i, j, (int)((a.step - 1) & 1), f);
      else
        pull_bc<T>(src, g, m.bc, i, j, f);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (T)0;
  }

  // ---- macroscopic variables (C1:1421-1439) ----------------------------
  T rho, drho, ux, uy;
  Mom32 mq;
  if (initial) {
    if (!F64) {
      float hq[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) hq[k] = (float)f[k];
      mq = moments32(hq);
    }
    rho = F64 ? (T)m.rho0 : (T)m.rho0_f;
    drho = (T)0;
    ux = (T)0;
    uy = (T)0;
  } else if (F64) {
    rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    drho = rho - (T)m.rho0;
    const T rinv = (T)1.0 / rho;
    ux = rinv * (f[1] + f[5] + f[8] - (f[6] + f[3] + f[7]));
    uy = rinv * (f[5] + f[2] + f[6] - (f[7] + f[4] + f[8]));
  } else {
    float hq[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) hq[k] = (float)f[k];
    mq = moments32(hq);
    drho = (T)mq.drho;
    rho = (T)(m.rho0_f + mq.drho);
    const float rinv = __fdividef(1.0f, (float)rho);
    ux = (T)(mq.jx * rinv);
    uy = (T)(mq.jy * rinv);
  }
  if (!act) {
    rho = (T)1;
    drho = (T)0;
    ux = uy = (T)0;
  }
  if (MODE == MODE_STEP) lattice_health<T>(a.status, drho, lane);

  // ---- SPM: G (last particle with PHI>0 wins) and the hydrodynamic force -
  T gx = (T)0, gy = (T)0;
  double phisum = 0.0;
  bool pnode = false;
  for (int c = 0; c < ncand; ++c) {
    double fx = 0.0, fy = 0.0, tz = 0.0;
    bool hit = false;
    if (act) {
      const double di = (double)i - s_px[c];
      const double dj = (double)j - s_py[c];
      T phi;
      if (F64)
        phi = (T)phi_double(di, dj, s_pr[c], m.zeta, m.pi);
      else
        phi = (T)phi_float((float)di, (float)dj, (float)s_pr[c], m.zeta_f, m.pi_f);
      if (phi > (T)0) {
        hit = true;
        const T uxp = (T)s_pu[c] - (T)s_pw[c] * (T)dj;
        const T uyp = (T)s_pv[c] + (T)s_pw[c] * (T)di;
        if (!initial) {
          gx = phi * (uxp - ux);
          gy = phi * (uyp - uy);
        }
        if (MODE == MODE_STEP) {
          const T rp = rho * phi;
          fx = (double)(rp * (ux - uxp));
          fy = (double)(rp * (uy - uyp));
          tz = (double)(rp * ((T)di * (uy - uyp) - (T)dj * (ux - uxp)));
        }
        phisum += (double)phi;
        if (phi >= (T)0.5) pnode = true;
      }
    }
    if (MODE == MODE_STEP && __any_sync(0xffffffffu, hit)) {
      fx = warp_sum(fx);
      fy = warp_sum(fy);
      tz = warp_sum(tz);
      if (lane == 0) {
        unsigned long long* acc = a.facc + s_idx[c];
        const long long st = a.npad;
        facc_add(acc, acc + st, fx);
        facc_add(acc + 2 * st, acc + 3 * st, fy);
        facc_add(acc + 4 * st, acc + 5 * st, tz);
      }
    }
  }

  // ---- velocity correction (C1:1138-1152) --------------------------------
  const T uxc = ux + (T)0.5 * (gx + (T)0.0);
  const T uyc = uy + (T)0.5 * (gy + (T)0.0);
  if (MODE != MODE_OUTPUT && m.bc == BC_EQUILIBRIUM && act)
    ring_store<T>(a, i, j, (int)(a.step & 1), F64 ? rho : drho, uxc, uyc);

  if (MODE == MODE_OUTPUT) {
    if (act) {
      const long long nn = (long long)(g.nx + 1) * (g.ny + 1);
      const long long o = (long long)j * (g.nx + 1) + i;
      a.out[o] = (double)uxc;
      a.out[nn + o] = (double)uyc;
      a.out[2 * nn + o] = F64 ? (double)rho : m.rho0 + (double)drho;
      a.out[3 * nn + o] = phisum;
      a.out[4 * nn + o] = (double)gx;
      a.out[5 * nn + o] = (double)gy;
      a.out[6 * nn + o] = pnode ? 10.0 : 0.0;
      if (a.out_f) {
#pragma unroll
        for (int k = 0; k < 9; ++k)
          a.out_f[o * 9 + k] = F64 ? (double)f[k] : (double)f[k] + wexact(k) * m.rho0;
      }
    }
    return;
  }

  // ---- mean density at history steps (C1:318): fixed-point, order-free ---
  // (each node's share rounded to fixed point, as the TMA step kernel does,
  // so both give the same integer total)
  if (MODE == MODE_STEP && rslot >= 0) {
    long long q = !act ? 0
                  : F64 ? __double2ll_rn((double)drho * MASS_FIX)
                        : mass_share32((float)drho);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_down_sync(0xffffffffu, q, o);
    if (lane == 0) {
      if (mass_local) *mass_local += q;
      else atomicAdd(a.mass_acc + rslot, (unsigned long long)q);
    }
  }

  // ---- collision of the next step ---------------------------------------
  if (!act) return;
  NodeOut no;
  no.omega = m.omega;
  no.yield = 0;
  no.t11 = no.t22 = no.t12 = 0.0;
  const bool want_stress = m.bingham || m.record_stress;
  const bool node_omega = m.bingham && MODE != MODE_INIT;
  if (BGK && m.bgk) {
    // COLLISION (C1:774-841).  Bingham: the bi-viscosity model on f - FEQ of
    // the node's previous collision (from its stored density and velocity;
    // INITIALIZE's equilibrium at the first step, the restored state's own
    // after a restart), with the node's previous omega.
    T* pm = static_cast<T*>(a.pm_dst);
    if (F64) {
      double om = m.omega;
      if (m.bingham) {
        double fp[9];
        if (MODE == MODE_STEP) {
          const T* q = static_cast<const T*>(a.pm_src);
          feq_double(m, (double)q[g.plane + n], (double)q[2 * g.plane + n], (double)q[n], fp);
        } else if (MODE == MODE_INIT) {
          feq_double(m, 0.0, 0.0, m.rho0, fp);
        } else {
          feq_double(m, (double)uxc, (double)uyc, (double)rho, fp);
        }
        const double omp = node_omega ? (double)static_cast<const T*>(a.om_src)[n] : m.omega;
        const double ZARIB = -1.5 * omp / (double)rho;
        double F_1[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) F_1[k] = (double)f[k] - fp[k];
        const double D11 = ZARIB * (F_1[1] + F_1[5] + F_1[6] + F_1[3] + F_1[7] + F_1[8]);
        const double D22 = ZARIB * (F_1[5] + F_1[2] + F_1[6] + F_1[7] + F_1[4] + F_1[8]);
        const double D12 = ZARIB * (F_1[5] - F_1[6] + F_1[7] - F_1[8]);
        const double GAMMA = sqrt(4.0 * fabs(D12 * D12 - D11 * D22));
        double NU_A;
        if (GAMMA < m.gamma_c) {
          NU_A = m.mu_r;
          no.yield = 5;
        } else {
          NU_A = m.nu + m.tau_y / GAMMA;
        }
        om = 1.0 / (3.0 * NU_A + 0.5);
        no.omega = om;
      }
      double FE[9], FI[9];
      bgk_source<double>(m.w_src, (double)rho, (double)uxc, (double)uyc, (double)gx, (double)gy, FI);
      feq_double(m, (double)uxc, (double)uyc, (double)rho, FE);
#pragma unroll
      for (int k = 0; k < 9; ++k)
        f[k] = (T)(om * FE[k] + (1.0 - om) * (double)f[k] + (1. - 0.5 * om) * FI[k]);
    } else {
      float om = m.omega_f;
      const float dr = (float)drho, rf = (float)rho, xf = (float)uxc, yf = (float)uyc;
      if (m.bingham) {
        float hp[9];
        if (MODE == MODE_STEP) {
          const T* q = static_cast<const T*>(a.pm_src);
          feq_shift32(m, (float)q[n], (float)q[g.plane + n], (float)q[2 * g.plane + n], hp);
        } else if (MODE == MODE_INIT) {
          feq_shift32(m, 0.0f, 0.0f, 0.0f, hp);
        } else {
          feq_shift32(m, dr, xf, yf, hp);
        }
        const float omp = node_omega ? (float)static_cast<const T*>(a.om_src)[n] : m.omega_f;
        const float ZARIB = -1.5f * omp / rf;
        float F_1[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) F_1[k] = (float)f[k] - hp[k];
        const float D11 = ZARIB * (F_1[1] + F_1[5] + F_1[6] + F_1[3] + F_1[7] + F_1[8]);
        const float D22 = ZARIB * (F_1[5] + F_1[2] + F_1[6] + F_1[7] + F_1[4] + F_1[8]);
        const float D12 = ZARIB * (F_1[5] - F_1[6] + F_1[7] - F_1[8]);
        const float GAMMA = sqrtf(4.0f * fabsf(D12 * D12 - D11 * D22));
        float NU_A;
        if (GAMMA < m.gamma_c_f) {
          NU_A = m.mu_r_f;
          no.yield = 5;
        } else {
          NU_A = m.nu_f + m.tau_y_f / GAMMA;
        }
        om = 1.0f / (3.0f * NU_A + 0.5f);
        no.omega = om;
      }
      float FE[9], FI[9];
      bgk_source<float>(m.w_src_f, rf, xf, yf, (float)gx, (float)gy, FI);
      feq_shift32(m, dr, xf, yf, FE);
#pragma unroll
      for (int k = 0; k < 9; ++k)
        f[k] = (T)(om * FE[k] + (1.0f - om) * (float)f[k] + (1.0f - 0.5f * om) * FI[k]);
    }
    if (m.bingham && pm) {
      pm[n] = F64 ? rho : drho;
      pm[g.plane + n] = uxc;
      pm[2 * g.plane + n] = uyc;
    }
  } else if (F64) {
    double S[9];
    if (node_omega) {
      rates_double(m, (double)static_cast<const T*>(a.om_src)[n], S);
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) S[k] = m.S_uni[k];
    }
    double fd[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) fd[k] = (double)f[k];
    collide_double(m, fd, (double)rho, (double)uxc, (double)uyc, (double)gx, (double)gy, S,
                   want_stress, no);
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (T)fd[k];
  } else {
    Rates32 r;
    r.s1 = m.s_e_f;
    r.s2 = m.s_eps_f;
    if (node_omega) {
      const float w = (float)static_cast<const T*>(a.om_src)[n];
      r.sw = w;
      r.sq = m.q_of_omega ? 8.0f * (2.0f - w) / (8.0f - w) : m.sq_uni_f;
    } else {
      r.sw = m.omega_f;
      r.sq = m.sq_uni_f;
    }
    float hf[9];
    relax32(m, mq, (float)rho, (float)uxc, (float)uyc, (float)gx, (float)gy, r, want_stress, no,
            hf);
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (T)hf[k];
  }
  T* __restrict__ dst = static_cast<T*>(a.dst);
#pragma unroll
  for (int k = 0; k < 9; ++k) dst[plane_of(k) * g.plane + n] = f[k];
  if (m.bingham) static_cast<T*>(a.om_dst)[n] = (T)no.omega;
  if (m.record_stress) {
    const int slot = (int)((kk + 1) & 1);
    T* rec = static_cast<T*>(a.rec) + (long long)slot * 4 * g.plane;
    rec[n] = (T)no.t11;
    rec[g.plane + n] = (T)no.t22;
    rec[2 * g.plane + n] = (T)no.t12;
    rec[3 * g.plane + n] = (T)no.yield;
  }
}

template <class T, int MODE>
__global__ void __launch_bounds__(TPB, sizeof(T) == 8 ? LBM_MINB_F64 : LBM_MINB_F32)
    k_lattice(const LatticeArgs a) {
  lattice_body<T, MODE, TX, TY>(a, blockIdx.x, blockIdx.y);
}


// ---------------------------------------------------------------------------
// Persistent, warp-specialised, TMA-pipelined time step (the launch lbm_step
// uses).
//
// Tile = TR rows x TW nodes, one node per consumer thread.  Each population
// plane of a tile is one TMA box of TR rows x (TW + 2H) elements, taken from
// row j - c_y and starting H elements left of the tile (H = one 16-byte
// vector), so the streamed value of node (i, j) sits at column i - c_x + H
// of the box row.  One producer warp runs up to NSTAGE tiles ahead: it waits
// until the consumers released a stage, stages the particles that touch the
// tile, and issues the nine TMA boxes; the stage's "full" barrier completes
// when both have landed.  The consumer warps wait on "full", compute their
// nodes, release the stage on its "empty" barrier and store.  No block-wide
// barrier is taken inside the loop.  Boxes that reach past the lattice are
// zero-filled by the TMA unit; the nodes on the lattice edge gather their
// populations from global memory with the boundary conditions instead.
constexpr int STEP_CONSUMERS = 512;              // consumer threads (16 warps)
constexpr int STEP_TPB = STEP_CONSUMERS + 32;    // + one producer warp

// TWv: nodes per tile row (the single-run kernel: 128 FP32, 64 FP64; the
// batched kernel: 64, which leaves fewer threads idle on narrow lattices)
template <class T, int TWv = (sizeof(T) == 8 ? 64 : 128)>
struct Stage {
  static constexpr int H = 16 / (int)sizeof(T);               // halo: one 16-byte vector
  static constexpr int TW = TWv;                              // nodes per tile row
  static constexpr int TR = STEP_CONSUMERS / TW;              // tile rows (8 or 4)
  static constexpr int BW = TW + 2 * H;                       // box width (544 bytes)
  static constexpr int PLANE = TR * BW;                       // elements per plane box
  static constexpr int BYTES = 9 * PLANE * (int)sizeof(T);     // the population boxes
  // a Bingham model's node omega of the tile, one box without halo after
  // the populations (a global load per node on the collision's path otherwise)
  static constexpr int OM_BYTES = TR * TW * (int)sizeof(T);
  static constexpr int SLOT = BYTES + OM_BYTES;                // one stage
  // offset of population k of a node from its column in the stage
  __host__ __device__ static constexpr int off(int k) {
    return plane_of(k) * PLANE + ((k == 1 || k == 5 || k == 8) ? -1 : (k == 3 || k == 6 || k == 7) ? 1 : 0);
  }
};

#ifndef LBM_STEP_STAGES
#define LBM_STEP_STAGES 3
#endif
constexpr int NSTAGE = LBM_STEP_STAGES;

// Particles touching one tile, staged by the producer warp (one per stage).
// One lane per candidate: the consumers cull them with a warp ballot.
static_assert(MAX_TILE_CAND <= 32, "one candidate per lane");
struct TileCand {
  double px[MAX_TILE_CAND], py[MAX_TILE_CAND], pd[MAX_TILE_CAND];  // pd: diameter
  double pu[MAX_TILE_CAND], pv[MAX_TILE_CAND], pw[MAX_TILE_CAND];
  int idx[MAX_TILE_CAND];
  int n;
  int bx, by;  // the tile in this stage
  // batched step only: the tile's simulation, its buffers and step, and the
  // slot of the shared ring that holds its LatticeArgs
  int sim, rslot, aslot, pad;
  long long step;
  const void* src;
  void* dst;
  const void* om_src;
  void* om_dst;
};

template <class T, class ST = Stage<T>>
constexpr int step_smem() {
  return NSTAGE * ST::SLOT + 2 * 8 * NSTAGE + 64 + NSTAGE * (int)sizeof(TileCand);
}

// Bounded wait on an mbarrier phase; false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
        "selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

template <class T, class ST = Stage<T>>
__device__ __forceinline__ void tma_tile(const CUtensorMap* tm, uint32_t dst, uint32_t mbar,
                                         int bx, int by) {
  const int x = bx * ST::TW - ST::H;  // a multiple of H: 16-byte aligned
  const int y0 = by * ST::TR;
  // three boxes of three planes: row shifts c_y = 0, +1, -1 (plane_of)
#pragma unroll
  for (int gq = 0; gq < 3; ++gq) {
    const int cy = gq == 0 ? 0 : (gq == 1 ? 1 : -1);
    const uint32_t d = dst + (uint32_t)(3 * gq * ST::PLANE * (int)sizeof(T));
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(d),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y0 - cy), "r"(3 * gq), "r"(mbar)
        : "memory");
  }
}

// The node omega of tile (bx, by) of a Bingham model: one 2-D box of TR
// rows x TW nodes, no halo (x = bx * TW is a multiple of 16 bytes).
template <class T, class ST = Stage<T>>
__device__ __forceinline__ void tma_omega(const CUtensorMap* tm, uint32_t dst, uint32_t mbar,
                                          int bx, int by) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(bx * ST::TW), "r"(by * ST::TR), "r"(mbar)
      : "memory");
}

// Candidate particles of one tile.  No latency sits between a free ring
// slot and its TMA issue: the count and the list row come in one round trip
// before the slot is waited for (the whole row is read before the count is
// known); after the TMA issue each lane copies its disk's state into the
// stage with cp.async, tracked by the stage's "full" barrier, so the
// producer never waits for it.
struct CandList {
  int n, idx;  // lane c: candidate c
};

__device__ __forceinline__ CandList cand_list(const LatticeArgs& a, int lt, int buf, int lane) {
  CandList c{0, 0};
  if (buf < 0) return c;  // a tile that no disk can reach
  if (!LBM_IN(lt, a.ntiles, a.status)) return c;
  const long long tbase = (long long)buf * a.ntiles + lt;
  c.n = a.tile_count[tbase];
  if (lane < a.tile_cap) c.idx = a.tile_list[tbase * a.tile_cap + lane];
  return c;
}

__device__ __forceinline__ void cp_async8(const void* smem, const void* gmem) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
}

// Fill C for tile (bx, by) and make the second arrival on the stage's
// "full" barrier fb once the copies have landed.
__device__ __forceinline__ void cand_copy(const LatticeArgs& a, CandList c, int bx, int by,
                                          TileCand& C, int lane, uint32_t fb) {
  if (c.n > a.tile_cap) {
    if (lane == 0) atomicOr(a.status, ST_OVERFLOW);
    c.n = a.tile_cap;
  }
  if (lane < c.n) {
    C.idx[lane] = c.idx;
    if (LBM_IN(c.idx, a.np, a.status)) {
      const double* p = a.ps + c.idx;
      const long long st = a.npad;
      cp_async8(&C.px[lane], p + P_X * st);
      cp_async8(&C.py[lane], p + P_Y * st);
      cp_async8(&C.pd[lane], p + P_D * st);
      cp_async8(&C.pu[lane], p + P_U * st);
      cp_async8(&C.pv[lane], p + P_V * st);
      cp_async8(&C.pw[lane], p + P_W * st);
    }
  }
  // the barrier's phase waits for this lane's copies (pending count +1 now,
  // -1 when they land); c.n is warp-uniform
  if (c.n > 0) asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(fb) : "memory");
  __syncwarp();
  if (lane == 0) {
    C.bx = bx;
    C.by = by;
    C.n = c.n;
    mbar_arrive(fb);
  }
}

#ifndef LBM_STEP_MINB_F32
#define LBM_STEP_MINB_F32 2
#endif


// Per-launch buffers of one simulation's step: the single-run kernel takes
// them from its arguments, the batched kernel from the stage's simulation.
template <class T>
struct StepIO {
  const T* src;     // f*(k), read by the edge gathers (the boxes come by TMA)
  T* dst;           // f*(k+1)
  const T* om_src;  // per-node omega of the Bingham models
  T* om_dst;
  long long step;   // the launch's step k
};

// One node's values between the stage read and the collision.
template <class T>
struct NodeVals {
  T f[9];
  T rho, drho, ux, uy, gx, gy;
  Mom32 mq;
};

// Node (i, j) of a staged tile: populations after streaming and the
// boundary conditions, macroscopic variables, lattice health, SPM body force
// (the highest-index disk with PHI > 0 sets G) and the warp's force sums.
// Every lane of the warp calls it (act: the node is in the lattice; edge:
// it gathers its populations from global memory); q points at the node's
// stage elements.  PDL: the force accumulators are touched only after
// griddepcontrol.wait (the particle kernel that zeroes them may still run).
template <class T, bool PDL, class ST = Stage<T>>
__device__ __forceinline__ void node_gather(const LatticeArgs& a, const StepIO<T>& io,
                                            const TileCand& C, T* const q, int i, int j,
                                            bool act, bool edge, int lane, bool& waited,
                                            NodeVals<T>& v) {
  constexpr bool F64 = sizeof(T) == 8;
  const Geometry& g = a.g;
  const Model& m = a.m;
  const T* __restrict__ src = io.src;
  // ---- streaming + boundary conditions --------------------------------
  // Nodes inside the lattice take the streamed values from the stage;
  // nodes on its edge gather theirs with the boundary conditions.
  T* const f = v.f;
  if (!edge) {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = q[ST::off(k)];
  } else if (act) {
    if (m.bc == BC_EQUILIBRIUM)
      edge_equilibrium<T>(a, i, j, (int)((io.step - 1) & 1), f);
    else
      pull_bc<T>(src, g, m.bc, i, j, f);
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = (T)0;
  }

  // ---- macroscopic variables (C1:1421-1439) ---------------------------
  T rho, drho, ux, uy;
  Mom32& mq = v.mq;
  if (F64) {
    rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    drho = rho - (T)m.rho0;
    const T rinv = (T)1.0 / rho;
    ux = rinv * (f[1] + f[5] + f[8] - (f[6] + f[3] + f[7]));
    uy = rinv * (f[5] + f[2] + f[6] - (f[7] + f[4] + f[8]));
  } else {
    float hq[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) hq[k] = (float)f[k];
    mq = moments32(hq);
    drho = (T)mq.drho;
    rho = (T)(m.rho0_f + mq.drho);
    const float rinv = __fdividef(1.0f, (float)rho);
    ux = (T)(mq.jx * rinv);
    uy = (T)(mq.jy * rinv);
  }
  if (!act) {
    rho = (T)1;
    drho = (T)0;
    ux = uy = (T)0;
  }
  lattice_health<T>(a.status, drho, lane);
  // FP64 reads f back from the stage after the particle loop instead of
  // holding 18 registers across it; edge nodes park theirs there first
  if (F64 && edge && act) {
#pragma unroll
    for (int k = 0; k < 9; ++k) q[ST::off(k)] = f[k];
  }

  // ---- SPM body force (the highest-index particle with PHI>0 sets G,
  //      C1:500-507) and force sums ---------------------------------------
  T gx = (T)0, gy = (T)0;
  int gbest = -1;
  // Only the candidates whose disk reaches this warp's 32 nodes of row j
  // are visited: for the others every node of the segment is at least
  // R + zeta/2 + 1e-3 from the centre, so PHI is 0 there in either
  // precision (rounding of the node distance is far below 1e-3) and the
  // skipped iterations would add nothing.
  unsigned near = 0;
  {
    bool nr = false;
    if (lane < C.n) {  // the warp's nodes: columns i - lane .. i - lane + 31
      const double dl = (double)(i - lane) - C.px[lane], dr = dl + 31.0;
      const double dx = dl > 0.0 ? dl : (dr < 0.0 ? -dr : 0.0);
      const double dy = (double)j - C.py[lane];
      const double reach = 0.5 * C.pd[lane] + 0.5 * m.zeta + 1e-3;
      nr = dx * dx + dy * dy < reach * reach;
    }
    near = __ballot_sync(0xffffffffu, nr);
  }
  while (near) {
    const int c = __ffs(near) - 1;
    near &= near - 1;
    double fx = 0.0, fy = 0.0, tz = 0.0;
    bool hit = false;
    if (act) {
      const double di = (double)i - C.px[c];
      const double dj = (double)j - C.py[c];
      T phi;
      if (F64)
        phi = (T)phi_double(di, dj, 0.5 * C.pd[c], m.zeta, m.pi);
      else
        phi = (T)phi_float((float)di, (float)dj, (float)(0.5 * C.pd[c]), m.zeta_f, m.pi_f);
      if (phi > (T)0) {
        hit = true;
        const T uxp = (T)C.pu[c] - (T)C.pw[c] * (T)dj;
        const T uyp = (T)C.pv[c] + (T)C.pw[c] * (T)di;
        if (C.idx[c] > gbest) {
          gbest = C.idx[c];
          gx = phi * (uxp - ux);
          gy = phi * (uyp - uy);
        }
        const T rp = rho * phi;
        fx = (double)(rp * (ux - uxp));
        fy = (double)(rp * (uy - uyp));
        tz = (double)(rp * ((T)di * (uy - uyp) - (T)dj * (ux - uxp)));
      }
    }
    if (__any_sync(0xffffffffu, hit)) {
      // warp totals of (Fx, Fy, Tz) in lanes 0, 8, 16
      const double tot = warp_sum3(fx, fy, tz, lane);
      if (PDL && !waited) {  // the particle kernel has zeroed the accumulators
        asm volatile("griddepcontrol.wait;" ::: "memory");
        waited = true;
      }
      const int comp = lane >> 3;
      if ((lane & 7) == 0 && comp < 3 && LBM_IN(C.idx[c], a.np, a.status)) {
        const long long st = a.npad;
        unsigned long long* acc = a.facc + C.idx[c] + 2 * comp * st;
        facc_add(acc, acc + st, tot);
      }
    }
  }
  if (F64 && act) {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = q[ST::off(k)];
  }
  v.rho = rho;
  v.drho = drho;
  v.ux = ux;
  v.uy = uy;
  v.gx = gx;
  v.gy = gy;
}

// Velocity correction and collision of the next step of node (i, j) (row
// offset nd), then its stores.  omn: the node's omega of the previous step
// (Bingham models; read by the caller before it releases the stage).
template <class T, bool STRESS>
__device__ __forceinline__ void node_collide(const LatticeArgs& a, const StepIO<T>& io,
                                             NodeVals<T>& v, int i, int j, long long nd,
                                             T om_node) {
  constexpr bool F64 = sizeof(T) == 8;
  const Model& m = a.m;
  const long long P = a.g.plane;
  if (!LBM_IN(nd, P, a.status)) return;  // every store below is at offset nd of a plane
  T* __restrict__ dst = io.dst;
  // ---- velocity correction (C1:1138-1152) and collision of the next step
  const T uxc = v.ux + (T)0.5 * (v.gx + (T)0.0);
  const T uyc = v.uy + (T)0.5 * (v.gy + (T)0.0);
  if (m.bc == BC_EQUILIBRIUM)
    ring_store<T>(a, i, j, (int)(io.step & 1), F64 ? v.rho : v.drho, uxc, uyc);
  const bool want_stress = STRESS;
  const bool bingham = STRESS && m.bingham;
  NodeOut no;
  no.omega = m.omega;
  no.yield = 0;
  no.t11 = no.t22 = no.t12 = 0.0;
  T omn = (T)m.omega;
  if (bingham) omn = om_node;
  if (F64) {
    double S[9];
    if (bingham) {
      rates_double(m, (double)omn, S);
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) S[k] = m.S_uni[k];
    }
    double fd[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) fd[k] = (double)v.f[k];
    collide_double(m, fd, (double)v.rho, (double)uxc, (double)uyc, (double)v.gx, (double)v.gy, S,
                   want_stress, no);
#pragma unroll
    for (int k = 0; k < 9; ++k) v.f[k] = (T)fd[k];
  } else {
    Rates32 r;
    r.s1 = m.s_e_f;
    r.s2 = m.s_eps_f;
    if (bingham) {
      const float w = (float)omn;
      r.sw = w;
      r.sq = m.q_of_omega ? 8.0f * (2.0f - w) / (8.0f - w) : m.sq_uni_f;
    } else {
      r.sw = m.omega_f;
      r.sq = m.sq_uni_f;
    }
    float hf[9];
    relax32(m, v.mq, (float)v.rho, (float)uxc, (float)uyc, (float)v.gx, (float)v.gy, r,
            want_stress, no, hf);
#pragma unroll
    for (int k = 0; k < 9; ++k) v.f[k] = (T)hf[k];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) dst[plane_of(k) * P + nd] = v.f[k];
  if (bingham) io.om_dst[nd] = (T)no.omega;
  if (STRESS && m.record_stress) {
    const int slot = (int)((io.step + 1) & 1);
    T* rec = static_cast<T*>(a.rec) + (long long)slot * 4 * P;
    rec[nd] = (T)no.t11;
    rec[P + nd] = (T)no.t22;
    rec[2 * P + nd] = (T)no.t12;
    rec[3 * P + nd] = (T)no.yield;
  }
}

// STRESS: the model needs the strain rate (Bingham viscosity or recorded
// stress); the Newtonian instantiation carries none of that code.
template <class T, bool STRESS>
__device__ __forceinline__ void step_body(const LatticeArgs& a, const CUtensorMap& tm,
                                          const CUtensorMap& tmo) {
  constexpr bool F64 = sizeof(T) == 8;
  constexpr uint32_t WAIT = 1u << 20;
  using ST = Stage<T>;
  extern __shared__ __align__(128) unsigned char s_raw[];
  T* const stage_w = reinterpret_cast<T*>(s_raw);
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(s_raw);
  const uint32_t full0 = s_base + NSTAGE * ST::SLOT;  // NSTAGE "full" barriers
  const uint32_t empty0 = full0 + 8 * NSTAGE;          // NSTAGE "empty" barriers
  TileCand* cands = reinterpret_cast<TileCand*>(s_raw + NSTAGE * ST::SLOT + 16 * NSTAGE + 64);

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const Geometry& g = a.g;
  const Model& m = a.m;
  const int ntx = (g.nx + 1 + ST::TW - 1) / ST::TW;
  const int nty = (g.ny + 1 + ST::TR - 1) / ST::TR;

  if (tid == STEP_CONSUMERS) {  // the producer's descriptors, before its first issue
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm)) : "memory");
    if (STRESS) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmo)) : "memory");
  }
  if (tid == 0) {
    for (int st = 0; st < NSTAGE; ++st) {
      // "full": the TMA boxes (expect_tx) and the candidates, two arrivals
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(full0 + 8 * st) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty0 + 8 * st),
                   "r"(STEP_CONSUMERS / 32)
                   : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // every CTA is resident: the next step's particle kernel may be scheduled
  // (it waits for this grid before it touches anything)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (warp == STEP_CONSUMERS / 32) {
    // ================= producer warp =====================================
    // Tiles come from one queue shared by all CTAs (work_ctr[step & 1]): the
    // step tiles of the list tiles in tile_order of the previous step's list
    // buffer, the tiles no disk can reach first (a disk moves less than the
    // Verlet skin between list builds).  Those need nothing from this step's
    // particle kernel, which may still be running; the first tile that lists
    // disks waits for it (griddepcontrol.wait), and by then every
    // particle-free tile has been handed out.  Taking tiles one at a time
    // from the queue keeps the CTAs finishing together.
    int* ctr = a.work_ctr + (a.step & 1);
    constexpr int SX = LTX / ST::TW, SY = LTY / ST::TR, S = SX * SY;  // step tiles per list tile
    const int Q = S * a.ntiles;
    // Queue entries blockIdx.x and gridDim.x + blockIdx.x are this CTA's
    // without an atomic; the shared counter hands out the rest from 2 x grid
    // on.  The list buffer of the previous step, its order and unlisted count
    // are read together with both buffers' candidates for those two entries,
    // so the first TMA issue waits for one round trip.
    const int base = 2 * (int)gridDim.x;
    int t0 = (int)blockIdx.x, t1 = (int)gridDim.x + (int)blockIdx.x, t2 = 0;
    int L0 = 0, L1 = 0, L2 = 0, nu = 0, bo = 0;
    if (lane == 0) {
      // odd steps take each group of the order reversed (tile_order[2 buf + 1])
      const int dir = (int)(a.step & 1);
      const int* o0 = a.tile_order + (long long)dir * a.ntiles;
      const int* o1 = a.tile_order + (long long)(2 + dir) * a.ntiles;
      bo = a.tile_cur[(a.step - 1) & 1];
      const int nu0 = a.n_unlisted[0], nu1 = a.n_unlisted[1];
      const int a0 = t0 < Q ? o0[t0 / S] : 0, a1 = t0 < Q ? o1[t0 / S] : 0;
      const int b0 = t1 < Q ? o0[t1 / S] : 0, b1 = t1 < Q ? o1[t1 / S] : 0;
      t2 = base + atomicAdd(ctr, 1);
      nu = bo ? nu1 : nu0;
      L0 = bo ? a1 : a0;
      L1 = bo ? b1 : b0;
    }
    const int buf_old = __shfl_sync(0xffffffffu, bo, 0);
    const int* order = a.tile_order + (long long)(2 * buf_old + (int)(a.step & 1)) * a.ntiles;
    int buf = -1;
    bool waited = false;
    int sidx = 0;
    uint32_t epar = 0;  // per-stage parity of the next "empty" completion
    uint32_t fpar = 0;  // per-stage parity of the next "full" completion
    int n = 0;          // tiles issued
    bool alive = true;

    // One queue entry: false once the queue is exhausted or the consumers
    // gave up.
    auto issue = [&](int t, int L) -> bool {
      if (t >= Q) return false;
      if ((unsigned)L >= (unsigned)a.ntiles) {  // never for a built order; no stray tile
        if (lane == 0) atomicOr(a.status, ST_OVERFLOW);
        return true;
      }
      const int sub = t % S, ly = L / g.ltx, lx = L - ly * g.ltx;
      const int bx = lx * SX + sub % SX, by = ly * SY + sub / SX;
      if (bx >= ntx || by >= nty) return true;  // past the lattice: no slot
      const bool listed = t / S >= __shfl_sync(0xffffffffu, nu, 0);
      if (listed && !waited) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        int bn = 0;
        if (lane == 0) bn = a.tile_cur[a.step & 1];
        buf = __shfl_sync(0xffffffffu, bn, 0);
        waited = true;
      }
      const CandList cl =
          cand_list(a, ((by * ST::TR) / LTY) * g.ltx + (bx * ST::TW) / LTX, listed ? buf : -1, lane);
      if (n >= NSTAGE) {
        bool ok = true;
        if (lane == 0) {
          ok = mbar_wait(empty0 + 8 * sidx, (epar >> sidx) & 1u, WAIT);
          if (!ok) atomicOr(a.status, ST_TIMEOUT);
        }
        epar ^= 1u << sidx;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          // consumers gave up: let the boxes already in flight land (bounded)
          if (lane == 0) {
            for (int st = 0; st < NSTAGE; ++st)
              mbar_wait(full0 + 8 * st, ((fpar >> st) & 1u) ^ 1u, WAIT);
          }
          alive = false;
          return false;
        }
      }
      const uint32_t fb = full0 + 8 * sidx;
      if (lane == 0) {
        if (bx * ST::TW >= g.nx) {
          // every node of the tile is on the right edge (the last column of
          // an NX that is a multiple of TW) and gathers from global memory:
          // no stage data
          mbar_arrive(fb);
        } else {
          // boxes reaching past the lattice are filled with zeros; they
          // still deliver their full byte count
          const bool om = STRESS && m.bingham;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                       "r"((uint32_t)(ST::BYTES + (om ? ST::OM_BYTES : 0)))
                       : "memory");
          tma_tile<T>(&tm, s_base + sidx * ST::SLOT, fb, bx, by);
          if (om) tma_omega<T>(&tmo, s_base + sidx * ST::SLOT + ST::BYTES, fb, bx, by);
        }
      }
      // the candidates, while the boxes are in flight; second arrival
      cand_copy(a, cl, bx, by, cands[sidx], lane, fb);
      fpar ^= 1u << sidx;
      sidx = sidx + 1 == NSTAGE ? 0 : sidx + 1;
      ++n;
      return true;
    };

    // Lane 0 runs the queue with three (index, list tile) register pairs
    // that rotate through "take" (atomicAdd issued), "look up" (order load
    // issued) and "issue", so neither latency is waited for while the ring
    // has work.
    for (;;) {
      if (lane == 0) L2 = t2 < Q ? order[t2 / S] : 0;
      if (!issue(__shfl_sync(0xffffffffu, t0, 0), __shfl_sync(0xffffffffu, L0, 0))) break;
      if (lane == 0) t0 = base + atomicAdd(ctr, 1);
      if (!issue(__shfl_sync(0xffffffffu, t1, 0), __shfl_sync(0xffffffffu, L1, 0))) break;
      if (lane == 0) {
        L0 = t0 < Q ? order[t0 / S] : 0;
        t1 = base + atomicAdd(ctr, 1);
      }
      if (!issue(__shfl_sync(0xffffffffu, t2, 0), __shfl_sync(0xffffffffu, L2, 0))) break;
      if (lane == 0) {
        L1 = t1 < Q ? order[t1 / S] : 0;
        t2 = base + atomicAdd(ctr, 1);
      }
    }
    if (alive) {
      // end marker: a stage whose tile column is -1
      bool ok = true;
      if (lane == 0) {
        if (n >= NSTAGE) {
          ok = mbar_wait(empty0 + 8 * sidx, (epar >> sidx) & 1u, WAIT);
          if (!ok) atomicOr(a.status, ST_TIMEOUT);
        }
        if (ok) {
          cands[sidx].bx = -1;
          mbar_arrive(full0 + 8 * sidx);  // both arrivals of the stage
          mbar_arrive(full0 + 8 * sidx);
        }
      }
    }
    // this grid completes only after this step's particle kernel, so the
    // next one (waiting on this grid) never overlaps it
    if (!waited) asm volatile("griddepcontrol.wait;" ::: "memory");
    return;
  }

  // ================= consumer warps ========================================
  const int rslot = a.rec_slot;
  bool waited = false;  // griddepcontrol.wait done (before the first force sum)
  const int tr = tid / ST::TW, tc = tid - tr * ST::TW;  // row and column in the tile
  const StepIO<T> io{static_cast<const T*>(a.src), static_cast<T*>(a.dst),
                     static_cast<const T*>(a.om_src), static_cast<T*>(a.om_dst), a.step};
  const int pt = g.pitch;
  int sidx = 0;
  uint32_t fpar = 0;  // per-stage parity of the next "full" completion
  // this thread's fixed-point share of the mean-density sum (rho - rho0 of
  // each of its nodes in units of 2^-40, rounded once per node: FP64 at
  // 2^-40, FP32 at 2^-30 by mass_share32), summed over the
  // warp and added to the history slot once when the warp leaves the loop:
  // integer sums, so the total does not depend on the order
  long long mass_q = 0;

  for (;; sidx = (sidx + 1 == NSTAGE ? 0 : sidx + 1)) {
    if (!mbar_wait(full0 + 8 * sidx, (fpar >> sidx) & 1u, WAIT)) {
      if (lane == 0) atomicOr(a.status, ST_TIMEOUT);
      return;
    }
    fpar ^= 1u << sidx;
    const int bx = cands[sidx].bx, by = cands[sidx].by;  // set by the producer
    if (bx < 0) break;  // the producer's end marker
    const int i = bx * ST::TW + tc;
    const int j = by * ST::TR + tr;
    const long long nd = (long long)j * pt + i;
    // A warp lies in one tile row: warp-uniform "has a lattice node".
    const bool warp_live = (j <= g.ny) && (bx * ST::TW + (tc & ~31) <= g.nx);
    if (!warp_live) {
      __syncwarp();
      if (lane == 0) mbar_arrive(empty0 + 8 * sidx);
      continue;
    }
    const TileCand& C = cands[sidx];
    const bool act = (i <= g.nx) && (j <= g.ny);
    const bool edge = (i == 0) || (i >= g.nx) || (j == 0) || (j >= g.ny);
    // this node's nine stage elements: planes in plane_of order, the row
    // shift is in the box, the column shift -c_x is applied in ST::off.  Pull
    // streaming is a bijection, so no other node reads these elements.
    T* const slot = stage_w + sidx * (ST::SLOT / (int)sizeof(T));
    T* const q = slot + tr * ST::BW + ST::H + tc;
    // the staged omega (none in a tile whose nodes all gather: bx * TW >= NX)
    const T* const omq = (STRESS && m.bingham && bx * ST::TW < g.nx)
                             ? slot + ST::BYTES / (int)sizeof(T) + tid
                             : nullptr;
    NodeVals<T> v;
    node_gather<T, true>(a, io, C, q, i, j, act, edge, lane, waited, v);
    // the node's omega, from the stage while it is still this tile's
    const T omn = (STRESS && m.bingham && act) ? (omq ? *omq : io.om_src[nd]) : (T)0;
    // the stage and its candidates are consumed
    __syncwarp();
    if (lane == 0) mbar_arrive(empty0 + 8 * sidx);

    // ---- mean density at history steps (C1:318): fixed-point, order-free -
    if (rslot >= 0 && act)
      mass_q += F64 ? __double2ll_rn((double)v.drho * MASS_FIX)
                    : mass_share32((float)v.drho);
    if (act) node_collide<T, STRESS>(a, io, v, i, j, nd, omn);
  }
  if (rslot >= 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass_q += __shfl_down_sync(0xffffffffu, mass_q, o);
    if (lane == 0 && mass_q != 0) atomicAdd(a.mass_acc + rslot, (unsigned long long)mass_q);
  }
}

// FP32: two CTAs per SM; FP64: one (with 17 warps, one SM sub-partition
// holds 5 of them, which caps FP64 at 96 registers per thread).
template <class T, bool STRESS>
__global__ void __launch_bounds__(STEP_TPB, sizeof(T) == 8 ? 1 : LBM_STEP_MINB_F32)
    k_step(const LatticeArgs a, const __grid_constant__ CUtensorMap tm,
           const __grid_constant__ CUtensorMap tmo) {
  step_body<T, STRESS>(a, tm, tmo);
}

// tm: the population buffer read; tmo: its omega buffer (Bingham models;
// any map otherwise, not read)
template <class T>
cudaError_t launch_step_tma(const LatticeArgs& a, const CUtensorMap* tm, const CUtensorMap* tmo,
                            cudaStream_t s) {
  using ST = Stage<T>;
  constexpr int SMEM = step_smem<T>();
  const int sx = (a.m.bingham || a.m.record_stress) ? 1 : 0;
  void (*const kern)(const LatticeArgs, const CUtensorMap, const CUtensorMap) =
      sx ? k_step<T, true> : k_step<T, false>;
  static int grid_of[2][64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (grid_of[sx][dev] == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, STEP_TPB, SMEM);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    // one SM stays free for the particle kernel that runs beside the
    // particle-free tiles (it fills an SM's register file on its own)
    grid_of[sx][dev] = (per_sm > 0 ? per_sm : 1) * (sms > 1 ? sms - 1 : 1);
  }
  const int ntiles = ((a.g.nx + 1 + ST::TW - 1) / ST::TW) * ((a.g.ny + 1 + ST::TR - 1) / ST::TR);
  const int grid = ntiles < grid_of[sx][dev] ? ntiles : grid_of[sx][dev];
  // Programmatic dependent launch: the kernel may start as soon as the
  // particle kernel before it on the stream allows (griddepcontrol.
  // launch_dependents); it waits for that kernel (griddepcontrol.wait) before
  // the tiles that need its results.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(STEP_TPB);
  cfg.dynamicSmemBytes = SMEM;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a, *tm, *tmo);
}

// ---------------------------------------------------------------------------
// Batched step on the TMA pipeline: the warp-specialised step of k_step over
// the tiles of every simulation of a batch (MRT models; a batch with a BGK
// run takes the one-node-per-thread kernel below), in tiles of 64 x 8 nodes
// (a batch's lattices are often narrow: 128-wide tiles left about a sixth
// of their threads without a node on 129-513-node rows).  Tiles are numbered
// simulation by simulation (row-major inside one, BatchSim::first), and
// block b takes a contiguous range of them, so it stays in one or two
// simulations.  Entering a simulation, the producer reads its device
// counters (step number, ping-pong buffer, history slot, list buffer: a
// captured graph replays unchanged) and picks the tensor maps of that buffer
// and of its omega (four per simulation, in global memory).  Per tile it issues the boxes,
// stages the candidates and notes the tile's simulation, buffers and step in
// the stage; the simulation's LatticeArgs go into a slot of a small shared
// ring that the consumers read their model from.  A slot is rewritten only
// after every consumer warp has finished the tile that used it (warps are at
// most NSTAGE tiles apart, the ring holds 2 NSTAGE).  The node arithmetic is
// k_step's (node_gather, node_collide).  Launches do not overlap: the
// batched particle kernel runs between two.
constexpr int BATCH_ARGS_SLOTS = 2 * NSTAGE;

template <class T>
using BatchStage = Stage<T, BATCH_TMA_TW>;
static_assert(BatchStage<float>::TR == BATCH_TMA_TR && BatchStage<double>::TR == BATCH_TMA_TR,
              "batched TMA tile");

template <class T>
constexpr int batch_step_smem() {
  return step_smem<T, BatchStage<T>>() + BATCH_ARGS_SLOTS * (int)sizeof(LatticeArgs);
}

template <class T, bool STRESS>
__global__ void __launch_bounds__(STEP_TPB, sizeof(T) == 8 ? 1 : LBM_STEP_MINB_F32)
    k_step_batch(const BatchSim* __restrict__ sims, int nsim,
                 const CUtensorMap* __restrict__ tmaps, long long total) {
  constexpr bool F64 = sizeof(T) == 8;
  constexpr uint32_t WAIT = 1u << 20;
  using ST = BatchStage<T>;
  static_assert(sizeof(LatticeArgs) % 8 == 0 && sizeof(TileCand) % 8 == 0, "8-byte words");
  extern __shared__ __align__(128) unsigned char s_raw[];
  T* const stage_w = reinterpret_cast<T*>(s_raw);
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(s_raw);
  const uint32_t full0 = s_base + NSTAGE * ST::SLOT;
  const uint32_t empty0 = full0 + 8 * NSTAGE;
  unsigned char* const cand_raw = s_raw + NSTAGE * ST::SLOT + 16 * NSTAGE + 64;
  TileCand* cands = reinterpret_cast<TileCand*>(cand_raw);
  LatticeArgs* ring = reinterpret_cast<LatticeArgs*>(cand_raw + NSTAGE * sizeof(TileCand));
  __shared__ int s_ring_sim[BATCH_ARGS_SLOTS];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (tid < BATCH_ARGS_SLOTS) s_ring_sim[tid] = -1;
  if (tid == 0) {
    for (int st = 0; st < NSTAGE; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(full0 + 8 * st) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty0 + 8 * st),
                   "r"(STEP_CONSUMERS / 32)
                   : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const long long per = (total + gridDim.x - 1) / gridDim.x;
  const long long t_lo = (long long)blockIdx.x * per;
  const long long t_hi = t_lo + per < total ? t_lo + per : total;

  if (warp == STEP_CONSUMERS / 32) {
    // ================= producer warp =====================================
    int q = 0;
    if (lane == 0) {  // the last simulation whose first tile is <= t_lo
      int lo = 0, hi = nsim - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sims[mid].first <= t_lo) lo = mid;
        else hi = mid - 1;
      }
      q = lo;
    }
    q = __shfl_sync(0xffffffffu, q, 0);
    // the simulation being staged, from its device counters
    long long first = 0, next = 0, kk = 0;
    int ntx = 1, ltx = 1, nx = 0, buf = 0, lbuf = 0, rslot = -1;
    const CUtensorMap* tm = nullptr;
    bool om = false;
    auto enter = [&](int sq) {
      const BatchSim& B = sims[sq];
      long long k = 0, f0 = 0, f1 = 0;
      int b = 0, lb = 0, rs = -1;
      if (lane == 0) {
        k = *B.kk;
        b = (int)((B.par0 + k - 1) & 1);
        rs = *B.rec_slot;
        lb = B.a.tile_cur[k & 1];
        f0 = B.first;
        f1 = sq + 1 < nsim ? sims[sq + 1].first : total;
      }
      kk = __shfl_sync(0xffffffffu, k, 0);
      buf = __shfl_sync(0xffffffffu, b, 0);
      rslot = __shfl_sync(0xffffffffu, rs, 0);
      lbuf = __shfl_sync(0xffffffffu, lb, 0);
      first = __shfl_sync(0xffffffffu, f0, 0);
      next = __shfl_sync(0xffffffffu, f1, 0);
      ntx = B.nbx;
      ltx = B.a.g.ltx;
      nx = B.a.g.nx;
      tm = tmaps + 4 * sq + buf;
      om = STRESS && B.a.m.bingham;
    };
    if (t_lo < t_hi) enter(q);
    int sidx = 0, n = 0;
    uint32_t epar = 0, fpar = 0;
    bool alive = true;
    for (long long t = t_lo; t < t_hi; ++t) {
      while (t >= next) enter(++q);
      const BatchSim& B = sims[q];
      const int local = (int)(t - first);
      const int by = local / ntx, bx = local - by * ntx;
      const CandList cl =
          cand_list(B.a, ((by * ST::TR) / LTY) * ltx + (bx * ST::TW) / LTX, lbuf, lane);
      if (n >= NSTAGE) {
        bool ok = true;
        if (lane == 0) {
          ok = mbar_wait(empty0 + 8 * sidx, (epar >> sidx) & 1u, WAIT);
          if (!ok) atomicOr(B.a.status, ST_TIMEOUT);
        }
        epar ^= 1u << sidx;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          if (lane == 0) {
            for (int st = 0; st < NSTAGE; ++st)
              mbar_wait(full0 + 8 * st, ((fpar >> st) & 1u) ^ 1u, WAIT);
          }
          alive = false;
          break;
        }
      }
      // the simulation's arguments into the ring slot of this tile
      const int slot = n % BATCH_ARGS_SLOTS;
      if (s_ring_sim[slot] != q) {
        const unsigned long long* from = reinterpret_cast<const unsigned long long*>(&B.a);
        unsigned long long* to = reinterpret_cast<unsigned long long*>(&ring[slot]);
        for (int w = lane; w < (int)(sizeof(LatticeArgs) / 8); w += 32) to[w] = from[w];
        __syncwarp();
        if (lane == 0) s_ring_sim[slot] = q;
      }
      TileCand& C = cands[sidx];
      const uint32_t fb = full0 + 8 * sidx;
      if (lane == 0) {
        C.sim = q;
        C.rslot = rslot;
        C.aslot = slot;
        C.step = kk;
        C.src = B.f[buf];
        C.dst = B.f[buf ^ 1];
        C.om_src = B.om[buf];
        C.om_dst = B.om[buf ^ 1];
        if (bx * ST::TW >= nx) {
          mbar_arrive(fb);  // every node on the right edge gathers from global memory
        } else {
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                       "r"((uint32_t)(ST::BYTES + (om ? ST::OM_BYTES : 0)))
                       : "memory");
          tma_tile<T, ST>(tm, s_base + sidx * ST::SLOT, fb, bx, by);
          if (om) tma_omega<T, ST>(tm + 2, s_base + sidx * ST::SLOT + ST::BYTES, fb, bx, by);
        }
      }
      cand_copy(B.a, cl, bx, by, C, lane, fb);
      fpar ^= 1u << sidx;
      sidx = sidx + 1 == NSTAGE ? 0 : sidx + 1;
      ++n;
    }
    if (alive) {
      bool ok = true;
      if (lane == 0) {
        if (n >= NSTAGE) ok = mbar_wait(empty0 + 8 * sidx, (epar >> sidx) & 1u, WAIT);
        if (ok) {
          cands[sidx].bx = -1;
          mbar_arrive(full0 + 8 * sidx);
          mbar_arrive(full0 + 8 * sidx);
        }
      }
    }
    return;
  }

  // ================= consumer warps ========================================
  bool waited = true;  // no programmatic dependence: the particles are done
  const int tr = tid / ST::TW, tc = tid - tr * ST::TW;
  int sidx = 0;
  uint32_t fpar = 0;
  // the warp's mean-density share of the current simulation's history slot,
  // added when the warp moves to another simulation or leaves
  long long mass_q = 0;
  int cur = -1, cur_rslot = -1;
  unsigned long long* cur_mass = nullptr;
  auto flush_mass = [&]() {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass_q += __shfl_down_sync(0xffffffffu, mass_q, o);
    if (lane == 0 && mass_q != 0 && cur_mass && cur_rslot >= 0)
      atomicAdd(cur_mass + cur_rslot, (unsigned long long)mass_q);
    mass_q = 0;
  };
  for (;; sidx = (sidx + 1 == NSTAGE ? 0 : sidx + 1)) {
    if (!mbar_wait(full0 + 8 * sidx, (fpar >> sidx) & 1u, WAIT)) {
      // the producer wrote no status word for a stage it never filled: the
      // current simulation's (or the first one's) takes the timeout
      if (lane == 0) atomicOr(sims[cur >= 0 ? cur : 0].a.status, ST_TIMEOUT);
      return;
    }
    fpar ^= 1u << sidx;
    const TileCand& C = cands[sidx];
    const int bx = C.bx, by = C.by;
    if (bx < 0) break;
    const LatticeArgs& a = ring[C.aslot];
    if (C.sim != cur) {
      flush_mass();
      cur = C.sim;
      cur_rslot = C.rslot;
      cur_mass = a.mass_acc;
    }
    const Geometry& g = a.g;
    const StepIO<T> io{static_cast<const T*>(C.src), static_cast<T*>(C.dst),
                       static_cast<const T*>(C.om_src), static_cast<T*>(C.om_dst), C.step};
    const int i = bx * ST::TW + tc;
    const int j = by * ST::TR + tr;
    const long long nd = (long long)j * g.pitch + i;
    const bool warp_live = (j <= g.ny) && (bx * ST::TW + (tc & ~31) <= g.nx);
    if (!warp_live) {
      __syncwarp();
      if (lane == 0) mbar_arrive(empty0 + 8 * sidx);
      continue;
    }
    const bool act = (i <= g.nx) && (j <= g.ny);
    const bool edge = (i == 0) || (i >= g.nx) || (j == 0) || (j >= g.ny);
    T* const slot = stage_w + sidx * (ST::SLOT / (int)sizeof(T));
    T* const qp = slot + tr * ST::BW + ST::H + tc;
    const T* const omq = (STRESS && a.m.bingham && bx * ST::TW < g.nx)
                             ? slot + ST::BYTES / (int)sizeof(T) + tid
                             : nullptr;
    NodeVals<T> v;
    node_gather<T, false, ST>(a, io, C, qp, i, j, act, edge, lane, waited, v);
    // the node's omega, from the stage while it is still this tile's
    const T omn = (STRESS && a.m.bingham && act) ? (omq ? *omq : io.om_src[nd]) : (T)0;
    // the stage and its candidates are consumed (the ring slot is not)
    __syncwarp();
    if (lane == 0) mbar_arrive(empty0 + 8 * sidx);
    if (cur_rslot >= 0 && cur_mass != nullptr && act)
      mass_q += F64 ? __double2ll_rn((double)v.drho * MASS_FIX) : mass_share32((float)v.drho);
    if (act) node_collide<T, STRESS>(a, io, v, i, j, nd, omn);
  }
  flush_mass();
}

template <class T>
cudaError_t batch_tma_prepare(int stress, int* blocks_per_sm) {
  constexpr int SMEM = batch_step_smem<T>();
  void (*const kern)(const BatchSim*, int, const CUtensorMap*, long long) =
      stress ? k_step_batch<T, true> : k_step_batch<T, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, STEP_TPB, SMEM);
}

template <class T>
cudaError_t launch_batch_tma(const BatchSim* sims, int nsim, const CUtensorMap* tmaps,
                             long long total, int stress, int grid, cudaStream_t s) {
  constexpr int SMEM = batch_step_smem<T>();
  if (stress)
    k_step_batch<T, true><<<grid, STEP_TPB, SMEM, s>>>(sims, nsim, tmaps, total);
  else
    k_step_batch<T, false><<<grid, STEP_TPB, SMEM, s>>>(sims, nsim, tmaps, total);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched step: a persistent grid over the work items (simulation, tile) of
// every simulation in the batch; block b takes a contiguous range of items,
// so it stays inside one or two simulations.  When it enters a simulation it
// stages that simulation's arguments in shared memory, with the ping-pong
// buffers, the step number and the history slot taken from the simulation's
// device counters (so a captured graph replays unchanged).  The node
// arithmetic is the scalar step's, so results do not depend on the tile
// shape or the grid.  BGK: some simulation of the batch uses the BGK collision.
// FP32 MRT: six blocks per SM (40 registers, a few spilled) hide more of the
// gather latency than four at 64 registers; the BGK variant keeps four
// (its larger body would spill much more at 40); FP64 takes the compiler's
// register count.
#ifndef LBM_BATCH_MINB_F32
#define LBM_BATCH_MINB_F32 6
#endif
template <class T, int BX, int BY, bool BGK>
__global__ void __launch_bounds__(BX * BY, sizeof(T) == 8 ? 0 : (BGK ? 4 : LBM_BATCH_MINB_F32))
    k_lattice_batch(const BatchSim* __restrict__ sims, int nsim, long long total) {
  __shared__ LatticeArgs s_a;
  __shared__ int s_sim;
  const long long per = (total + gridDim.x - 1) / gridDim.x;
  const long long i0 = (long long)blockIdx.x * per;
  const long long i1 = i0 + per < total ? i0 + per : total;
  long long qfirst = 0, qend = -1;  // items of the staged simulation
  int nbx = 1;
  // lane 0: the warp's mean-density share for the staged simulation's
  // history slot, added once when the block leaves the simulation
  long long mass_q = 0;
  unsigned long long* mass_ptr = nullptr;
  for (long long item = i0; item < i1; ++item) {
    __syncthreads();  // the previous tile is done with s_a and the candidates
    if (item >= qend) {
      if ((threadIdx.x & 31) == 0 && mass_ptr && mass_q)
        atomicAdd(mass_ptr, (unsigned long long)mass_q);
      mass_q = 0;
      if (threadIdx.x == 0) {
        int lo = 0, hi = nsim - 1;  // last simulation with first <= item
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sims[mid].first <= item) lo = mid;
          else hi = mid - 1;
        }
        s_sim = lo;
      }
      __syncthreads();
      const int q = s_sim;
      const BatchSim& B = sims[q];
      const int* src = reinterpret_cast<const int*>(&B.a);
      int* dst = reinterpret_cast<int*>(&s_a);
      for (int w = threadIdx.x; w < (int)(sizeof(LatticeArgs) / 4); w += BX * BY) dst[w] = src[w];
      __syncthreads();
      if (threadIdx.x == 0) {
        const long long k = *B.kk;
        const int b = (int)((B.par0 + k - 1) & 1);
        s_a.step = k;
        s_a.rec_slot = *B.rec_slot;
        s_a.src = B.f[b];
        s_a.dst = B.f[b ^ 1];
        s_a.om_src = B.om[b];
        s_a.om_dst = B.om[b ^ 1];
        s_a.pm_src = B.pm[b];
        s_a.pm_dst = B.pm[b ^ 1];
      }
      __syncthreads();
      qfirst = B.first;
      qend = q + 1 < nsim ? sims[q + 1].first : total;
      nbx = B.nbx;
      mass_ptr = (s_a.rec_slot >= 0 && s_a.mass_acc) ? s_a.mass_acc + s_a.rec_slot : nullptr;
    }
    const long long t = item - qfirst;
    lattice_body<T, MODE_STEP, BX, BY, BGK>(s_a, (int)(t % nbx), (int)(t / nbx), &mass_q);
  }
  if ((threadIdx.x & 31) == 0 && mass_ptr && mass_q) atomicAdd(mass_ptr, (unsigned long long)mass_q);
}

template <class T, bool BGK>
void launch_batch_shape(const BatchSim* sims, int nsim, long long total, int shape, int grid,
                        cudaStream_t s) {
  switch (shape) {
    case 0: k_lattice_batch<T, 32, 8, BGK><<<grid, 256, 0, s>>>(sims, nsim, total); break;
    case 1: k_lattice_batch<T, 64, 4, BGK><<<grid, 256, 0, s>>>(sims, nsim, total); break;
    default: k_lattice_batch<T, 128, 2, BGK><<<grid, 256, 0, s>>>(sims, nsim, total); break;
  }
}

template <class T>
cudaError_t launch_batch(const BatchSim* sims, int nsim, long long total, int shape, int bgk,
                         int grid, cudaStream_t s) {
  if (bgk) launch_batch_shape<T, true>(sims, nsim, total, shape, grid, s);
  else launch_batch_shape<T, false>(sims, nsim, total, shape, grid, s);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_mode(const LatticeArgs& a, cudaStream_t s, int mode) {
  dim3 grid(a.g.nbx, a.g.nby);
  switch (mode) {
    case MODE_STEP: k_lattice<T, MODE_STEP><<<grid, TPB, 0, s>>>(a); break;  // BGK steps
    case MODE_OUTPUT: k_lattice<T, MODE_OUTPUT><<<grid, TPB, 0, s>>>(a); break;
    case MODE_INIT: k_lattice<T, MODE_INIT><<<grid, TPB, 0, s>>>(a); break;
    default: k_lattice<T, MODE_RESTART><<<grid, TPB, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

}  // namespace lbm
