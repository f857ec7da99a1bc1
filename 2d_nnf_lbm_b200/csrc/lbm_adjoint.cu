// lbm_adjoint.cu -- reverse-mode (adjoint) kernels of one time step (sm_100a).
//
// The forward level n (the step kernel) maps, node by node,
//   f*(n) --pull + BC--> F(n) --> rho, u_pred, G (SPM, last disk wins),
//   u = u_pred + G/2, FORCE(n) = sum rho*phi*(u_pred - u_p)     C1:546-570
//   f*(n+1) = M^-1 [m - S(m - m_eq) + (1 - S/2) m_F]             C1:875-1048
//   omega(n+1) = 1/(3 nu_A/rho + 1/2), nu_A Papanastasiou        C6:903-958
// and the particle kernel of step n+1 maps (records n, FORCE(n)) to records
// n+1 (C1:247-259, C6:300-312).  The kernels below run the transposed
// Jacobians of those maps, level by level from the last step back to the
// first:
//   k_adj_lattice   one node per thread: gathers dJ/df*(n+1) from
//                   dJ/dF(n+1) by the transposed pull (a gather along +c_k;
//                   bounce-back terms at the wall node itself), re-derives
//                   the forward intermediates from f*(n) and the records of
//                   step n, and writes dJ/dF(n), dJ/domega(n); per-disk
//                   sums of dJ/d(x, y, u, v, w) go to FP64 accumulators,
//                   dJ/dnu and dJ/dtau_y to one FP64 slot per block.
//   k_adj_particles one thread per disk: the transposed Newton-Euler update
//                   and repulsion (walls and pairs), the objective's own
//                   term, dJ/drho_p.
// The collision is differentiated in moment space: with the orthogonal D2Q9
// transform, M^-T = D^-1 M, D = diag(9, 36, 36, 6, 12, 6, 12, 4, 4), and the
// strain rate of C6:903-916 reduces to sums of S*m_neq moments,
//   D11 = kappa(-y1/4 - 3y7/4) + 3/4((s7-s1)G.u - 2 s7 Gx ux), y = S*m_neq,
// kappa = 36*d_mrt the scale of the reference's inverse transform.
// T = float: populations and node arithmetic in FP32 (the forward's shifted
// populations); reductions in FP64.  T = double: FP64 throughout.
#include <cuda_runtime.h>

#include "lbm_lattice.cuh"

namespace lbm {

namespace {

__device__ __forceinline__ int cxk(int k) { return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0); }
__device__ __forceinline__ int cyk(int k) { return k == 2 || k == 5 || k == 6 ? 1 : (k == 4 || k == 7 || k == 8 ? -1 : 0); }
__device__ __forceinline__ int oppk(int k) { return k == 0 ? 0 : (k < 5 ? ((k + 1) & 3) + 1 : ((k - 3) & 3) + 5); }

// Unknown k of node (i, j) that the boundary sets by half-way bounce-back
// from the node's own post-collision population opp(k): the corners (both
// boundary kinds, C1:1390-1414) and, for LBM_BC_HALFWAY_BB, the edges
// (C6:1206-1219, C6:1285-1294).
__device__ __forceinline__ bool bb_set(const Geometry& g, int bc, int k, int i, int j) {
  const bool L = i == 0, R = i == g.nx, B = j == 0, U = j == g.ny;
  if ((L || R) && (B || U)) {
    if (L && B) return k == 1 || k == 5 || k == 2;
    if (L && U) return k == 1 || k == 8 || k == 4;
    if (R && U) return k == 3 || k == 7 || k == 4;
    return k == 2 || k == 6 || k == 3;
  }
  if (bc != 1) return false;
  if (U) return k == 8 || k == 4 || k == 7;
  if (B) return k == 5 || k == 2 || k == 6;
  if (R) return k == 6 || k == 3 || k == 7;
  if (L) return k == 5 || k == 1 || k == 8;
  return false;
}

// dJ/dr(k) of the raw pulled value r(k) of node (i, j) -- the value before
// the boundary routine: F*(k, x - c_k), or the node's own F*(k) when that
// source lies outside -- from dJ/dF of the node after the boundary routine.
template <class T>
__device__ __forceinline__ T adj_raw(const T* __restrict__ A, const Geometry& g, int bc, int k,
                                     int i, int j) {
  const long long P = g.plane;
  const long long n = (long long)j * g.pitch + i;
#define AA(q) A[plane_of(q) * P + n]
  const bool L = i == 0, R = i == g.nx, B = j == 0, U = j == g.ny;
  if (!(L || R || B || U)) return AA(k);
  if (((L || R) && (B || U)) || bc == 1) return bb_set(g, bc, k, i, j) ? (T)0 : AA(k);
  // Zou-He with zero wall velocity (C1:1250-1258, C1:1341-1363)
  const T h = (T)0.5;
  if (U) {
    switch (k) {
      case 1: return AA(1) - h * AA(8) + h * AA(7);
      case 2: return AA(2) + AA(4);
      case 3: return AA(3) + h * AA(8) - h * AA(7);
      case 5: return AA(5) + AA(7);
      case 6: return AA(6) + AA(8);
      case 0: return AA(0);
      default: return (T)0;
    }
  }
  if (B) {
    switch (k) {
      case 1: return AA(1) - h * AA(5) + h * AA(6);
      case 3: return AA(3) + h * AA(5) - h * AA(6);
      case 4: return AA(4) + AA(2);
      case 7: return AA(7) + AA(5);
      case 8: return AA(8) + AA(6);
      case 0: return AA(0);
      default: return (T)0;
    }
  }
  if (L) {
    switch (k) {
      case 2: return AA(2) - h * AA(5) + h * AA(8);
      case 4: return AA(4) + h * AA(5) - h * AA(8);
      case 7: return AA(7) + AA(5);
      case 6: return AA(6) + AA(8);
      case 3: return AA(3) + AA(1);
      case 0: return AA(0);
      default: return (T)0;
    }
  }
  switch (k) {  // R
    case 2: return AA(2) - h * AA(6) + h * AA(7);
    case 4: return AA(4) + h * AA(6) - h * AA(7);
    case 8: return AA(8) + AA(6);
    case 5: return AA(5) + AA(7);
    case 1: return AA(1) + AA(3);
    case 0: return AA(0);
    default: return (T)0;
  }
#undef AA
}

// dJ/df*(k) of node (i, j): the transpose of pull streaming + boundary.
template <class T>
__device__ __forceinline__ void adj_gather(const T* __restrict__ A, const Geometry& g, int bc,
                                           int i, int j, T* a) {
  const long long P = g.plane;
  const int pt = g.pitch;
  const long long n = (long long)j * pt + i;
  if (i >= 2 && i <= g.nx - 2 && j >= 2 && j <= g.ny - 2) {
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = A[plane_of(k) * P + n + cxk(k) + (long long)cyk(k) * pt];
    return;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    T v = (T)0;
    const int xi = i + cxk(k), xj = j + cyk(k);
    if (xi >= 0 && xi <= g.nx && xj >= 0 && xj <= g.ny) v += adj_raw<T>(A, g, bc, k, xi, xj);
    const int si = i - cxk(k), sj = j - cyk(k);
    if (!(si >= 0 && si <= g.nx && sj >= 0 && sj <= g.ny)) v += adj_raw<T>(A, g, bc, k, i, j);
    const int ko = oppk(k);
    if (bb_set(g, bc, ko, i, j)) v += A[plane_of(ko) * P + n];
    a[k] = v;
  }
}

// The D2Q9 moments of C6:878-886.
template <class T>
__device__ __forceinline__ void moments9(const T* f, T* m) {
  const T s14 = f[1] + f[2] + f[3] + f[4], s58 = f[5] + f[6] + f[7] + f[8];
  m[0] = f[0] + s14 + s58;
  m[1] = (T)-4 * f[0] - s14 + (T)2 * s58;
  m[2] = (T)4 * f[0] - (T)2 * s14 + s58;
  m[3] = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  m[4] = (T)-2 * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
  m[5] = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
  m[6] = (T)-2 * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
  m[7] = f[1] - f[2] + f[3] - f[4];
  m[8] = f[5] - f[6] + f[7] - f[8];
}

// M^T a (the adjoint of m = M f).
template <class T>
__device__ __forceinline__ void moments9_t(const T* a, T* f) {
  const T c0 = a[0] - a[1] - (T)2 * a[2];
  const T d0 = a[0] + (T)2 * a[1] + a[2];
  f[0] = a[0] - (T)4 * a[1] + (T)4 * a[2];
  f[1] = c0 + a[3] - (T)2 * a[4] + a[7];
  f[2] = c0 + a[5] - (T)2 * a[6] - a[7];
  f[3] = c0 - a[3] + (T)2 * a[4] + a[7];
  f[4] = c0 - a[5] + (T)2 * a[6] - a[7];
  f[5] = d0 + a[3] + a[4] + a[5] + a[6] + a[8];
  f[6] = d0 - a[3] - a[4] + a[5] + a[6] - a[8];
  f[7] = d0 - a[3] - a[4] - a[5] - a[6] + a[8];
  f[8] = d0 + a[3] + a[4] - a[5] - a[6] - a[8];
}

__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float texp(float x) { return expf(x); }
__device__ __forceinline__ double texp(double x) { return exp(x); }
__device__ __forceinline__ float tcos(float x) { return cosf(x); }
__device__ __forceinline__ double tcos(double x) { return cos(x); }
__device__ __forceinline__ float texpm1(float x) { return expm1f(x); }
__device__ __forceinline__ double texpm1(double x) { return expm1(x); }

// Taylor coefficients: g1 = (1 - e^-x)/x = sum_k (-1)^(k+1) x^(k-1)/k! and
// r = (1 - e^-x - x e^-x)/x^2 = sum_k (-1)^k (k-1) x^(k-2)/k!; 1/k! below.
#define LBM_IF(k) (1.0 / (k))
__device__ __forceinline__ double inv_fact(int k) {
  constexpr double F[15] = {1.0, 1.0, LBM_IF(2.0), LBM_IF(6.0), LBM_IF(24.0), LBM_IF(120.0),
                            LBM_IF(720.0), LBM_IF(5040.0), LBM_IF(40320.0), LBM_IF(362880.0),
                            LBM_IF(3628800.0), LBM_IF(39916800.0), LBM_IF(479001600.0),
                            LBM_IF(6227020800.0), LBM_IF(87178291200.0)};
  return F[k];
}
#undef LBM_IF
__device__ __forceinline__ double g1_coef(int k) { return (k % 2 ? 1.0 : -1.0) * inv_fact(k); }
__device__ __forceinline__ double r_coef(int k) { return (k % 2 ? -1.0 : 1.0) * (k - 1) * inv_fact(k); }

// g1 and r for x >= 0 without cancellation: the series below x = 0.1 (terms
// to x^7 in FP32, x^13 in FP64; the first omitted term is below the type's
// rounding), expm1 above.  The Papanastasiou viscosity is
// nu + tau_y m g1(m gamma) and its derivative in gamma -tau_y m^2 r(m gamma).
template <class T>
__device__ __forceinline__ void papanastasiou_terms(T x, T* g1, T* r) {
  constexpr int K = sizeof(T) == 8 ? 14 : 8;
  if (x < (T)0.1) {
    T sg = (T)g1_coef(K), sr = (T)r_coef(K);
#pragma unroll
    for (int k = K - 1; k >= 1; --k) sg = sg * x + (T)g1_coef(k);
#pragma unroll
    for (int k = K - 1; k >= 2; --k) sr = sr * x + (T)r_coef(k);
    *g1 = sg;
    *r = sr;
    return;
  }
  const T ix = (T)1 / x;
  const T em = -texpm1(-x);
  *g1 = em * ix;
  *r = (em - x * texp(-x)) * ix * ix;
}

template <class T>
__device__ __forceinline__ T phi_of(T di, T dj, T R, const Model& m) {
  if (sizeof(T) == 8) return (T)phi_double((double)di, (double)dj, (double)R, m.zeta, m.pi);
  return (T)phi_float((float)di, (float)dj, (float)R, m.zeta_f, m.pi_f);
}

constexpr int ADJ_TPB = TPB;

}  // namespace

template <class T>
__global__ void __launch_bounds__(ADJ_TPB) k_adj_lattice(const AdjLatticeArgs a) {
  const Geometry& g = a.g;
  const Model& m = a.m;
  __shared__ double s_x[ADJ_MAX_PARTICLES], s_y[ADJ_MAX_PARTICLES], s_r[ADJ_MAX_PARTICLES];
  __shared__ double s_u[ADJ_MAX_PARTICLES], s_v[ADJ_MAX_PARTICLES], s_w[ADJ_MAX_PARTICLES];
  __shared__ double s_ax[ADJ_MAX_PARTICLES], s_ay[ADJ_MAX_PARTICLES], s_at[ADJ_MAX_PARTICLES];
  __shared__ int s_idx[ADJ_MAX_PARTICLES];
  __shared__ int s_nc;
  __shared__ double s_g[ADJ_TPB / 32][2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i = blockIdx.x * TX + (tid % TX), j = blockIdx.y * TY + (tid / TX);
  // the next particle adjoint kernel may launch; it waits for this grid
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  // disks whose support reaches this block, in index order (records of step
  // n, written by the forward pass)
  if (tid == 0) {
    int c = 0;
    if (!a.level0) {
      const double i0 = blockIdx.x * TX, i1 = i0 + TX - 1, j0 = blockIdx.y * TY, j1 = j0 + TY - 1;
      for (int p = 0; p < a.np; ++p) {
        const PRef P{const_cast<double*>(a.ps) + p, a.npad};
        const double x = P[P_X], y = P[P_Y], r = 0.5 * P[P_D];
        const double rs = r + 0.5 * m.zeta + 1.0;
        if (x + rs < i0 || x - rs > i1 || y + rs < j0 || y - rs > j1) continue;
        s_idx[c] = p;
        s_x[c] = x;
        s_y[c] = y;
        s_r[c] = r;
        s_u[c] = P[P_U];
        s_v[c] = P[P_V];
        s_w[c] = P[P_W];
        ++c;
      }
    }
    s_nc = c;
  }
  __syncthreads();
  const int nc = s_nc;
  const bool act = i <= g.nx && j <= g.ny;
  const long long n = (long long)j * g.pitch + i;
  const T rho0 = (T)m.rho0;
  double gnu = 0.0, gty = 0.0;

  // ---- forward intermediates ---------------------------------------------
  T h[9];
  if (a.level0 || !act) {
    double fe[9];
    feq_double(m, 0.0, 0.0, m.rho0, fe);
#pragma unroll
    for (int k = 0; k < 9; ++k) h[k] = (T)(fe[k] - wexact(k) * m.rho0);
  } else {
    pull_bc<T>(static_cast<const T*>(a.fs), g, m.bc, i, j, h);
    if (sizeof(T) == 8) {
#pragma unroll
      for (int k = 0; k < 9; ++k) h[k] = h[k] - (T)(wexact(k) * m.rho0);
    }
  }
  // every global load of the node is issued here, before the arithmetic:
  // omega(n), dJ/dF(n+1) of the transposed pull, dJ/domega(n+1)
  const bool node_omega = m.bingham && !a.level0;
  const T om = node_omega && act ? static_cast<const T*>(a.oms)[n] : (T)m.omega;
  T ahs[9];
  if (a.a_in && act) {
    adj_gather<T>(static_cast<const T*>(a.a_in), g, m.bc, i, j, ahs);
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) ahs[k] = (T)0;
  }
  const T awo = (m.bingham && a.aw_in && act) ? static_cast<const T*>(a.aw_in)[n] : (T)0;
  T mh[9];
  moments9<T>(h, mh);
  T drho, rho, upx, upy;
  if (a.level0 || !act) {
    drho = (T)0;
    rho = rho0;
    upx = upy = (T)0;
  } else {
    drho = mh[0];
    rho = rho0 + drho;
    upx = mh[3] / rho;
    upy = mh[5] / rho;
  }
  int win = -1;
  T phw = (T)0, usxw = (T)0, usyw = (T)0;
  if (act) {
    for (int c = 0; c < nc; ++c) {
      const T di = (T)((double)i - s_x[c]), dj = (T)((double)j - s_y[c]);
      const T phi = phi_of<T>(di, dj, (T)s_r[c], m);
      if (phi > (T)0) {
        win = c;
        phw = phi;
        usxw = (T)s_u[c] - (T)s_w[c] * dj;
        usyw = (T)s_v[c] + (T)s_w[c] * di;
      }
    }
  }
  T Gx = (T)0, Gy = (T)0;
  if (win >= 0) {
    Gx = phw * (usxw - upx);
    Gy = phw * (usyw - upy);
  }
  const T ux = upx + (T)0.5 * Gx, uy = upy + (T)0.5 * Gy;
  const T sw = om;
  const T i8w = (T)1 / ((T)8 - om);
  const T sq = m.q_of_omega ? (T)8 * ((T)2 - om) * i8w : (T)m.s_q;
  const T s1 = (T)m.s_e, s2 = (T)m.s_eps;
  const T kap = (T)a.kappa;
  const T U2 = ux * ux + uy * uy;
  const T mne1 = mh[1] + (T)2 * drho - (T)3 * rho * U2;
  const T mne4 = mh[4] + rho * ux, mne6 = mh[6] + rho * uy;
  const T mne7 = mh[7] - rho * (ux * ux - uy * uy), mne8 = mh[8] - rho * ux * uy;
  const T Fx = rho * Gx, Fy = rho * Gy;
  const T mf4 = -Fx, mf6 = -Fy, mf7 = (T)2 * (Fx * ux - Fy * uy), mf8 = Fy * ux + Fx * uy;

  // f*(n+1) = kappa M^-1 m' + const  ->  dJ/dm' = kappa D^-1 M dJ/df*
  T am[9];
  moments9<T>(ahs, am);
  {
    const T k36 = kap * (T)(1.0 / 36.0);
    am[0] *= (T)4 * k36;
    am[1] *= k36;
    am[2] *= k36;
    am[3] *= (T)6 * k36;
    am[4] *= (T)3 * k36;
    am[5] *= (T)6 * k36;
    am[6] *= (T)3 * k36;
    am[7] *= (T)9 * k36;
    am[8] *= (T)9 * k36;
  }
  // m' = M - S m_neq + (1 - S/2) m_F
  T aM[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) aM[k] = am[k];
  T an1 = -s1 * am[1], an2 = -s2 * am[2], an4 = -sq * am[4], an6 = -sq * am[6];
  T an7 = -sw * am[7], an8 = -sw * am[8];
  T asq = -(mne4 + (T)0.5 * mf4) * am[4] - (mne6 + (T)0.5 * mf6) * am[6];
  T asw = -(mne7 + (T)0.5 * mf7) * am[7] - (mne8 + (T)0.5 * mf8) * am[8];
  T arho = (T)0, aux = (T)0, auy = (T)0, aGx = (T)0, aGy = (T)0;

  // Papanastasiou viscosity and omega(n+1) (C6:903-958)
  if (m.bingham) {
    const T y1 = s1 * mne1, y7 = sw * mne7, y8 = sw * mne8;
    const T Pg = Gx * ux + Gy * uy;
    const T D11 = kap * ((T)-0.25 * y1 - (T)0.75 * y7) +
                  (T)0.75 * ((sw - s1) * Pg - (T)2 * sw * Gx * ux);
    const T D22 = kap * ((T)-0.25 * y1 + (T)0.75 * y7) +
                  (T)0.75 * ((sw - s1) * Pg - (T)2 * sw * Gy * uy);
    const T D12 = kap * ((T)-1.5 * y8) + (T)0.75 * (-sw * (Gx * uy + Gy * ux));
    const T ir = (T)1 / rho;
    const T d11 = D11 * ir, d22 = D22 * ir, d12 = D12 * ir;
    const T gam = tsqrt((T)2 * fabs(d11 * d11 + d22 * d22 + (T)2 * (d12 * d12)));
    const T nu = (T)m.nu, ty = (T)m.tau_y, mp = (T)m.m_pap;
    const bool low = gam < (T)m.gamma_min;
    T g1 = (T)1, rq = (T)0.5;
    if (!low) papanastasiou_terms<T>(mp * gam, &g1, &rq);
    const T nuA = nu + ty * mp * g1;
    const T wout = (T)1 / ((T)3 * nuA * ir + (T)0.5);
    const T az = -wout * wout * awo;
    const T anuA = (T)3 * az * ir;
    arho += (T)-3 * nuA * ir * ir * az;
    gnu += (double)anuA;
    gty += (double)(anuA * mp * g1);
    const T agam = low ? (T)0 : -anuA * ty * mp * mp * rq;
    T ad11 = (T)0, ad22 = (T)0, ad12 = (T)0;
    if (gam > (T)0) {
      const T q = (T)2 * agam / gam;
      ad11 = q * d11;
      ad22 = q * d22;
      ad12 = (T)2 * q * d12;
    }
    arho -= (ad11 * d11 + ad22 * d22 + ad12 * d12) * ir;
    const T aD11 = ad11 * ir, aD22 = ad22 * ir, aD12 = ad12 * ir;
    const T ay1 = (T)-0.25 * kap * (aD11 + aD22);
    const T ay7 = (T)0.75 * kap * (aD22 - aD11);
    const T ay8 = (T)-1.5 * kap * aD12;
    const T aP = (T)0.75 * (sw - s1) * (aD11 + aD22);
    asw += (T)0.75 * Pg * (aD11 + aD22) - (T)1.5 * (Gx * ux * aD11 + Gy * uy * aD22) -
           (T)0.75 * (Gx * uy + Gy * ux) * aD12 + mne7 * ay7 + mne8 * ay8;
    an1 += s1 * ay1;
    an7 += sw * ay7;
    an8 += sw * ay8;
    aGx += aP * ux - (T)1.5 * sw * ux * aD11 - (T)0.75 * sw * uy * aD12;
    aGy += aP * uy - (T)1.5 * sw * uy * aD22 - (T)0.75 * sw * ux * aD12;
    aux += aP * Gx - (T)1.5 * sw * Gx * aD11 - (T)0.75 * sw * Gy * aD12;
    auy += aP * Gy - (T)1.5 * sw * Gy * aD22 - (T)0.75 * sw * Gx * aD12;
  }

  // m_neq = M - m_eq(rho, u)
  aM[1] += an1; aM[2] += an2; aM[4] += an4; aM[6] += an6; aM[7] += an7; aM[8] += an8;
  {
    const T q1 = -an1, q2 = -an2, q4 = -an4, q6 = -an6, q7 = -an7, q8 = -an8;
    arho += q1 * ((T)-2 + (T)3 * U2) + q2 * ((T)1 - (T)3 * U2) - q4 * ux - q6 * uy +
            q7 * (ux * ux - uy * uy) + q8 * ux * uy;
    aux += (T)6 * rho * ux * (q1 - q2) - rho * q4 + (T)2 * rho * ux * q7 + rho * uy * q8;
    auy += (T)6 * rho * uy * (q1 - q2) - rho * q6 - (T)2 * rho * uy * q7 + rho * ux * q8;
  }
  // forcing moments m_F(rho G, u) (C1:995-1016)
  {
    const T b1 = ((T)1 - (T)0.5 * s1) * am[1], b2 = ((T)1 - (T)0.5 * s2) * am[2];
    const T b3 = am[3], b4 = ((T)1 - (T)0.5 * sq) * am[4];
    const T b5 = am[5], b6 = ((T)1 - (T)0.5 * sq) * am[6];
    const T b7 = ((T)1 - (T)0.5 * sw) * am[7], b8 = ((T)1 - (T)0.5 * sw) * am[8];
    const T aFx = (T)6 * ux * (b1 - b2) + b3 - b4 + (T)2 * ux * b7 + uy * b8;
    const T aFy = (T)6 * uy * (b1 - b2) + b5 - b6 - (T)2 * uy * b7 + ux * b8;
    aux += (T)6 * Fx * (b1 - b2) + (T)2 * Fx * b7 + Fy * b8;
    auy += (T)6 * Fy * (b1 - b2) - (T)2 * Fy * b7 + Fx * b8;
    arho += aFx * Gx + aFy * Gy;
    aGx += rho * aFx;
    aGy += rho * aFy;
  }
  // rates of omega (C6:1002-1021)
  {
    T aom = asw;
    if (m.q_of_omega) aom += asq * (T)-48 * i8w * i8w;
    if (node_omega) {
      if (act) static_cast<T*>(a.aw_out)[n] = aom;
    } else if (act) {
      gnu += (double)(aom * (T)(-3.0 * m.omega * m.omega));  // omega = 1/(3 nu + 1/2)
    }
  }
  // u = u_pred + G/2 (C1:1138-1152); G = phi (u_p - u_pred) of the winner
  T aupx = aux, aupy = auy;
  aGx += (T)0.5 * aux;
  aGy += (T)0.5 * auy;
  if (win >= 0) {
    aupx -= phw * aGx;
    aupy -= phw * aGy;
  }

  // ---- disks: G of the winner, FORCE(n), phi and the rigid velocity --------
  // dJ/dFORCE(n) comes from the particle adjoint kernel launched before this
  // one, which also clears a_p after reading it: wait for it here.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (tid < nc) {
    const int p = s_idx[tid];
    s_ax[tid] = a.a_h[p];
    s_ay[tid] = a.a_h[a.npad + p];
    s_at[tid] = a.a_h[2 * a.npad + p];
  }
  __syncthreads();
  for (int c = 0; c < nc; ++c) {
    double cx = 0.0, cy = 0.0, cu = 0.0, cv = 0.0, cw = 0.0;
    if (act) {
      const T di = (T)((double)i - s_x[c]), dj = (T)((double)j - s_y[c]);
      const T phi = phi_of<T>(di, dj, (T)s_r[c], m);
      if (phi > (T)0) {
        const T W = (T)s_w[c];
        const T usx = (T)s_u[c] - W * dj, usy = (T)s_v[c] + W * di;
        T aphi = (T)0, ausx = (T)0, ausy = (T)0, adi = (T)0, adj = (T)0;
        if (c == win) {
          aphi += aGx * (usx - upx) + aGy * (usy - upy);
          ausx += phw * aGx;
          ausy += phw * aGy;
        }
        const T aHx = (T)s_ax[c], aHy = (T)s_ay[c], aT = (T)s_at[c];
        const T ex = upx - usx, ey = upy - usy;
        const T tq = di * ey - dj * ex;
        const T sdot = aHx * ex + aHy * ey + aT * tq;
        arho += phi * sdot;
        aphi += rho * sdot;
        const T rp = rho * phi;
        const T aex = rp * (aHx - aT * dj), aey = rp * (aHy + aT * di);
        aupx += aex;
        aupy += aey;
        ausx -= aex;
        ausy -= aey;
        adi += rp * aT * ey;
        adj -= rp * aT * ex;
        cu = (double)ausx;
        cv = (double)ausy;
        cw = (double)(-dj * ausx + di * ausy);
        adj -= W * ausx;
        adi += W * ausy;
        const T r = tsqrt(di * di + dj * dj);
        const T Dd = (T)s_r[c] - r;
        const T zh = (T)(0.5 * m.zeta);
        if (Dd > -zh && Dd < zh && r > (T)0) {
          const T k = (T)(m.pi / m.zeta);
          const T aD = aphi * (T)0.5 * k * tcos(k * Dd) / r;
          adi -= aD * di;
          adj -= aD * dj;
        }
        cx = -(double)adi;
        cy = -(double)adj;
      }
    }
    const bool any = __any_sync(0xffffffffu, cx != 0.0 || cy != 0.0 || cu != 0.0 || cv != 0.0 ||
                                                 cw != 0.0);
    if (any) {
      cx = warp_sum(cx);
      cy = warp_sum(cy);
      cu = warp_sum(cu);
      cv = warp_sum(cv);
      cw = warp_sum(cw);
      if (lane == 0) {
        const int p = s_idx[c];
        const long long st = a.npad;
        atomicAdd(a.a_p + p, cx);
        atomicAdd(a.a_p + st + p, cy);
        atomicAdd(a.a_p + 2 * st + p, cu);
        atomicAdd(a.a_p + 3 * st + p, cv);
        atomicAdd(a.a_p + 4 * st + p, cw);
      }
    }
  }

  // u_pred = j / rho; rho = rho0 + sum h, j = sum c h
  if (act && !a.level0) {
    const T ir = (T)1 / rho;
    arho -= (aupx * upx + aupy * upy) * ir;
    aM[0] += arho;
    aM[3] += aupx * ir;
    aM[5] += aupy * ir;
    T ah[9];
    moments9_t<T>(aM, ah);
    T* out = static_cast<T*>(a.a_out);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[plane_of(k) * g.plane + n] = ah[k];
  }

  // ---- dJ/dnu, dJ/dtau_y: one slot per block, fixed order ------------------
  gnu = warp_sum(gnu);
  gty = warp_sum(gty);
  if (lane == 0) {
    s_g[warp][0] = gnu;
    s_g[warp][1] = gty;
  }
  __syncthreads();
  if (tid == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < ADJ_TPB / 32; ++w) {
      t0 += s_g[w][0];
      t1 += s_g[w][1];
    }
    double* slot = a.gacc + 2 * ((long long)blockIdx.y * gridDim.x + blockIdx.x);
    slot[0] += t0;
    slot[1] += t1;
  }
}

// ---------------------------------------------------------------------------
// Glowinski repulsion magnitude g(r) along the centre line and g'(r)
// (C1:701-768, C3:739-804): range rc = contact + zeta; g = eps C q^2,
// q = (r - rc)/zeta, plus E C (contact - r)/zeta when overlapping.
__device__ __forceinline__ void glowinski(double r, double contact, double zeta, double eps,
                                          double E, double C, double* gv, double* gd) {
  *gv = 0.0;
  *gd = 0.0;
  if (r > contact + zeta) return;
  const double q = (r - contact - zeta) / zeta;
  *gv = eps * C * q * q;
  *gd = 2.0 * eps * C * q / zeta;
  if (r <= contact) {
    *gv += E * C * (contact - r) / zeta;
    *gd -= E * C / zeta;
  }
}

__global__ void __launch_bounds__(ADJ_MAX_PARTICLES) k_adj_particles(const AdjParticleArgs a) {
  __shared__ double s_fx[ADJ_MAX_PARTICLES], s_fy[ADJ_MAX_PARTICLES];
  const int p = threadIdx.x;
  // launched as a programmatic dependent of the lattice adjoint kernel of
  // the same step: its per-disk sums and dJ/dF must be complete
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const long long st = a.npad;
  double aX = 0, aY = 0, aUp = 0, aVp = 0, aWp = 0, aUO = 0, aVO = 0, aWO = 0;
  double x = 0, y = 0, D = 0, M = 1, I = 1;
  if (p < a.np) {
    const PRef Q{const_cast<double*>(a.prev) + p, a.npad};
    const PRef C{const_cast<double*>(a.cur) + p, a.npad};
    double s[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] = a.a_state[k * st + p];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      s[k] += a.a_p[k * st + p];
      a.a_p[k * st + p] = 0.0;
    }
    if (p == a.obj_p && a.n >= a.n0 && a.n <= a.n1) {
      const int c = a.obj_c == P_X ? 0 : a.obj_c == P_Y ? 1 : a.obj_c == P_U ? 2
                  : a.obj_c == P_V ? 3 : 4;
      s[c] += a.obj_w;
    }
    // X(n) = X(n-1) + (V(n) + V(n-1))/2; V(n) = V + (FORCE + F_H_IN + F_COL)/M
    // (+ buoyancy); F_H_IN/M = (rho0/rho_p)(V - V_OLD) (C1:247-259)
    const double rhop = Q[P_RHO];
    M = Q[P_M];
    I = Q[P_I];
    x = Q[P_X];
    y = Q[P_Y];
    D = Q[P_D];
    const double rr = a.rho0 / rhop;
    const double bx = s[2] + 0.5 * s[0], by = s[3] + 0.5 * s[1], bw = s[4];
    aX = s[0];
    aY = s[1];
    aUp = 0.5 * s[0] + bx + s[5] + rr * bx;
    aVp = 0.5 * s[1] + by + s[6] + rr * by;
    aWp = bw + s[7] + rr * bw;
    aUO = -rr * bx;
    aVO = -rr * by;
    aWO = -rr * bw;
    a.a_h[p] = bx / M;
    a.a_h[st + p] = by / M;
    a.a_h[2 * st + p] = bw / I;
    s_fx[p] = bx / M;
    s_fy[p] = by / M;
    const double hx = C[P_FX], hy = C[P_FY], tz = C[P_TZ], fcx = C[P_FCX], fcy = C[P_FCY];
    const double du = Q[P_U] - Q[P_UO], dv = Q[P_V] - Q[P_VO], dw = Q[P_W] - Q[P_WO];
    a.a_rho[p] += -(bx * (hx + fcx) + by * (hy + fcy)) / (M * rhop) -
                  rr / rhop * (bx * du + by * dv) + by * a.rho0 * a.gravity / (rhop * rhop) -
                  bw * tz / (I * rhop) - rr / rhop * bw * dw;
  }
  __syncthreads();
  if (p < a.np) {
    const double fx = s_fx[p], fy = s_fy[p];
    // walls (C1:737-745 mirror images, C3:775-783 wall disks): the image
    // lies along one axis, e = s*(coordinate) + const with s = 2 or 1
    if (a.wall_model != 2) {
      for (int iw = 1; iw <= 4; ++iw) {
        double e, sc;
        const bool ydir = (iw == 1 || iw == 3);
        if (a.wall_model == 0) {
          sc = 2.0;
          e = iw == 1 ? 2.0 * y : iw == 2 ? 2.0 * x - 2.0 * (double)a.nx
            : iw == 3 ? 2.0 * y - a.mirror_top : 2.0 * x - a.mirror_left;
        } else {
          sc = 1.0;
          e = iw == 1 ? y + 0.5 * D : iw == 2 ? x - (double)a.nx - 0.5 * D
            : iw == 3 ? y - (double)a.ny - 0.5 * D : x + 0.5 * D;
        }
        const double r = fabs(e);
        double gv, gd;
        glowinski(r, D, a.rep_zeta, a.eps_w, a.e_w, a.c_ij, &gv, &gd);
        if (ydir) aY += sc * gd * fy;
        else aX += sc * gd * fx;
      }
    }
    // pairs: F_p = g(r) e/r, e = X_p - X_q; dF/de = g' e e^T/r^2 + g/r (I - e e^T/r^2)
    for (int q = 0; q < a.np; ++q) {
      if (q == p) continue;
      const PRef Qq{const_cast<double*>(a.prev) + q, a.npad};
      const double ex = x - Qq[P_X], ey = y - Qq[P_Y];
      const double r = sqrt(ex * ex + ey * ey);
      if (!(r > 0.0)) continue;
      double gv, gd;
      glowinski(r, 0.5 * D + 0.5 * Qq[P_D], a.rep_zeta, a.eps_p, a.e_p, a.c_ij, &gv, &gd);
      if (gv == 0.0 && gd == 0.0) continue;
      const double nx_ = ex / r, ny_ = ey / r;
      const double dfx = fx - s_fx[q], dfy = fy - s_fy[q];
      const double en = nx_ * dfx + ny_ * dfy;
      const double t = gv / r;
      aX += gd * en * nx_ + t * (dfx - en * nx_);
      aY += gd * en * ny_ + t * (dfy - en * ny_);
    }
    a.a_state[p] = aX;
    a.a_state[st + p] = aY;
    a.a_state[2 * st + p] = aUp;
    a.a_state[3 * st + p] = aVp;
    a.a_state[4 * st + p] = aWp;
    a.a_state[5 * st + p] = aUO;
    a.a_state[6 * st + p] = aVO;
    a.a_state[7 * st + p] = aWO;
  }
}

template <class K, class A>
cudaError_t launch_pdl(K kernel, dim3 grid, int block, const A& a, cudaStream_t s, int pdl) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(block);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

cudaError_t launch_adj_lattice_fp32(const AdjLatticeArgs& a, cudaStream_t s, int pdl) {
  return launch_pdl(k_adj_lattice<float>, dim3(a.g.nbx, a.g.nby), ADJ_TPB, a, s, pdl);
}
cudaError_t launch_adj_lattice_fp64(const AdjLatticeArgs& a, cudaStream_t s, int pdl) {
  return launch_pdl(k_adj_lattice<double>, dim3(a.g.nbx, a.g.nby), ADJ_TPB, a, s, pdl);
}
cudaError_t launch_adj_particles(const AdjParticleArgs& a, cudaStream_t s) {
  return launch_pdl(k_adj_particles, dim3(1), ADJ_MAX_PARTICLES, a, s, 1);
}

__global__ void k_set_ll(long long* p, long long v) { *p = v; }

cudaError_t launch_set_ll(long long* p, long long v, cudaStream_t s) {
  k_set_ll<<<1, 1, 0, s>>>(p, v);
  return cudaGetLastError();
}

}  // namespace lbm
