// lbm_particles.cu -- particle kernel of one time step (sm_100a).
//
// One block of PBLK threads, particles strided over the threads:
//   1. cell list of disk centres (counting sort into cells of edge
//      >= D_max + repulsion range), so each disk only tests the disks of its
//      3x3 neighbour cells;
//   2. Glowinski repulsion, pairs then walls (C1:701-768, C3:739-804); each
//      disk sums its pair forces in ascending partner order, which is the
//      order in which the reference's IP<JP double loop accumulates them;
//   3. Newton-Euler update with the internal-mass term (C1:247-259,
//      C6:300-312) and the history record (C1:264, C6:315-318);
//   4. per-tile candidate lists for the lattice kernel's SPM evaluation.
// Built with --fmad=false: the FP64 arithmetic is operation-for-operation the
// reference's, so the particle update is bit-identical for identical inputs.
#include <cuda_runtime.h>

#include "lbm_internal.h"

namespace lbm {

constexpr int PBLK = 256;
constexpr int MAX_NEIGH = 32;

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ int cell_index(const ParticleArgs& a, double x, double y) {
  const int cx = clampi((int)floor(x / a.cell_size), 0, a.ncx - 1);
  const int cy = clampi((int)floor(y / a.cell_size), 0, a.ncy - 1);
  return cy * a.ncx + cx;
}

// Pair force of (lo, hi), lo < hi, as the reference evaluates F_PP for
// IP = lo, JP = hi (C3:758-766); the contact branch tests D_PP or the stale
// wall distance D_PW.
__device__ __forceinline__ void pair_force(const ParticleArgs& a, const double* A, const double* B,
                                           double test_stale, double* F) {
  const double ZITA = a.rep_zeta, CIJ = a.c_ij, EPS_P = a.eps_p, E_P = a.e_p;
  const double dx = A[P_X] - B[P_X], dy = A[P_Y] - B[P_Y];
  const double D_PP = sqrt(dx * dx + dy * dy);
  const double rsum = 0.5 * A[P_D] + 0.5 * B[P_D];
  const double test = a.contact == 1 ? test_stale : D_PP;
  F[0] = 0.0;
  F[1] = 0.0;
  if (D_PP > rsum + ZITA) return;
  const double q = (D_PP - 0.5 * A[P_D] - 0.5 * B[P_D] - ZITA) / ZITA;
  if (D_PP <= rsum + ZITA && test > rsum) {
    F[0] = EPS_P * CIJ * (q * q) * dx / D_PP;
    F[1] = EPS_P * CIJ * (q * q) * dy / D_PP;
  } else if (test <= rsum) {
    const double e = E_P * CIJ * (rsum - D_PP) / ZITA;
    F[0] = (EPS_P * CIJ * (q * q) + e) * dx / D_PP;
    F[1] = (EPS_P * CIJ * (q * q) + e) * dy / D_PP;
  }
}

__device__ void build_tiles(const ParticleArgs& a, int tid) {
  // clear the tiles of the previous boxes
  for (int p = tid; p < a.np; p += PBLK) {
    const int4 tb = a.tbox[p];
    for (int ty = 0; ty < tb.w; ++ty)
      for (int tx = 0; tx < tb.z; ++tx) {
        const int nbx = (a.nx + 1 + TX - 1) / TX;
        a.tile_count[(tb.y + ty) * nbx + tb.x + tx] = 0;
      }
  }
  __syncthreads();
  const int nbx = (a.nx + 1 + TX - 1) / TX;
  for (int p = tid; p < a.np; p += PBLK) {
    const double* P = a.ps + (long long)p * PS;
    const double r = 0.5 * P[P_D] + 0.5 * a.zeta + 1.0;
    int i0 = (int)ceil(P[P_X] - r), i1 = (int)floor(P[P_X] + r);
    int j0 = (int)ceil(P[P_Y] - r), j1 = (int)floor(P[P_Y] + r);
    i0 = max(i0, 0);
    j0 = max(j0, 0);
    i1 = min(i1, a.nx);
    j1 = min(j1, a.ny);
    int4 tb = make_int4(0, 0, 0, 0);
    if (i0 <= i1 && j0 <= j1 && isfinite(P[P_X]) && isfinite(P[P_Y])) {
      tb.x = i0 / TX;
      tb.y = j0 / TY;
      tb.z = i1 / TX - tb.x + 1;
      tb.w = j1 / TY - tb.y + 1;
      if (tb.z * tb.w > a.max_slots) {
        atomicOr(a.status, ST_OVERFLOW);
        tb = make_int4(0, 0, 0, 0);
      }
    }
    for (int ty = 0; ty < tb.w; ++ty)
      for (int tx = 0; tx < tb.z; ++tx) {
        const int t = (tb.y + ty) * nbx + tb.x + tx;
        const int slot = atomicAdd(&a.tile_count[t], 1);
        if (slot < a.tile_cap)
          a.tile_list[(long long)t * a.tile_cap + slot] = p;
        else
          atomicOr(a.status, ST_OVERFLOW);
      }
    a.tbox[p] = tb;
  }
}

__global__ void __launch_bounds__(PBLK) k_particles(const ParticleArgs a) {
  __shared__ long long s_kk;
  __shared__ int s_sum[PBLK];
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_kk = *a.kk + 1;
    *a.kk = s_kk;
  }
  __syncthreads();
  const long long kk = s_kk;

  // ---- 1. cell list ------------------------------------------------------
  const int ncells = a.ncx * a.ncy;
  if (a.np > 1) {
    for (int c = tid; c < ncells; c += PBLK) a.cell_count[c] = 0;
    __syncthreads();
    for (int p = tid; p < a.np; p += PBLK) {
      const double* P = a.ps + (long long)p * PS;
      const int c = cell_index(a, P[P_X], P[P_Y]);
      a.cell_of[p] = c;
      atomicAdd(&a.cell_count[c], 1);
    }
    __syncthreads();
    const int chunk = (ncells + PBLK - 1) / PBLK;
    const int c0 = tid * chunk, c1 = min(ncells, c0 + chunk);
    int local = 0;
    for (int c = c0; c < c1; ++c) local += a.cell_count[c];
    s_sum[tid] = local;
    __syncthreads();
    if (tid == 0) {
      int run = 0;
      for (int t = 0; t < PBLK; ++t) {
        const int v = s_sum[t];
        s_sum[t] = run;
        run += v;
      }
    }
    __syncthreads();
    int run = s_sum[tid];
    for (int c = c0; c < c1; ++c) {
      const int v = a.cell_count[c];
      a.cell_start[c] = run;
      a.cell_count[c] = run;  // becomes the scatter cursor
      run += v;
    }
    if (tid == 0) a.cell_start[ncells] = a.np;
    __syncthreads();
    for (int p = tid; p < a.np; p += PBLK) {
      const int slot = atomicAdd(&a.cell_count[a.cell_of[p]], 1);
      a.cell_items[slot] = p;
    }
  }
  const double stale = *a.stale_dpw;  // D_PW left over from the previous call
  __syncthreads();

  // ---- 2./3. repulsion, Newton-Euler update, history ----------------------
  const bool rec = a.series != nullptr && a.series_every > 0 && (kk % a.series_every) == 0;
  const long long rslot = rec ? (kk / a.series_every - 1) % a.series_cap : 0;
  if (rec && tid == 0) {
    a.series[rslot * a.series_len + 0] = (double)kk;
    a.series[rslot * a.series_len + 1] = __longlong_as_double(0x7ff8000000000000LL);
  }
  for (int p = tid; p < a.np; p += PBLK) {
    double* P = a.ps + (long long)p * PS;
    double fcx = 0.0, fcy = 0.0;
    if (a.np > 1) {
      int nb[MAX_NEIGH];
      int nn = 0;
      const int c = a.cell_of[p];
      const int cx = c % a.ncx, cy = c / a.ncx;
      for (int yy = max(cy - 1, 0); yy <= min(cy + 1, a.ncy - 1); ++yy)
        for (int xx = max(cx - 1, 0); xx <= min(cx + 1, a.ncx - 1); ++xx) {
          const int cc = yy * a.ncx + xx;
          for (int s = a.cell_start[cc]; s < a.cell_start[cc + 1]; ++s) {
            const int q = a.cell_items[s];
            if (q == p) continue;
            const double* Q = a.ps + (long long)q * PS;
            const double dx = P[P_X] - Q[P_X], dy = P[P_Y] - Q[P_Y];
            const double lim = 0.5 * P[P_D] + 0.5 * Q[P_D] + a.rep_zeta;
            if (dx * dx + dy * dy > 1.0000001 * lim * lim + 1e-12) continue;
            if (nn < MAX_NEIGH) {
              int k = nn++;
              while (k > 0 && nb[k - 1] > q) {
                nb[k] = nb[k - 1];
                --k;
              }
              nb[k] = q;
            } else {
              atomicOr(a.status, ST_OVERFLOW);
            }
          }
        }
      for (int k = 0; k < nn; ++k) {
        const int q = nb[k];
        double F[2];
        if (q < p) {
          pair_force(a, a.ps + (long long)q * PS, P, stale, F);
          fcx = fcx - F[0];
          fcy = fcy - F[1];
        } else {
          pair_force(a, P, a.ps + (long long)q * PS, stale, F);
          fcx = fcx + F[0];
          fcy = fcy + F[1];
        }
      }
    }
    // walls (C1:735-768 mirror images; C3:775-804 wall disks)
    if (a.wall_model != 2) {
      const double ZITA = a.rep_zeta, CIJ = a.c_ij, EPS_W = a.eps_w, E_W = a.e_w;
      const double x = P[P_X], y = P[P_Y], D = P[P_D];
      double D_PW = stale;
      for (int iw = 1; iw <= 4; ++iw) {
        double rw0, rw1;
        if (a.wall_model == 0) {
          if (iw == 1) { rw0 = x; rw1 = -y; }
          else if (iw == 2) { rw0 = 2.0 * (double)a.nx - x; rw1 = y; }
          else if (iw == 3) { rw0 = x; rw1 = a.mirror_top - y; }
          else { rw0 = a.mirror_left - x; rw1 = y; }
        } else {
          if (iw == 1) { rw0 = x; rw1 = -0.5 * D; }
          else if (iw == 2) { rw0 = (double)a.nx + 0.5 * D; rw1 = y; }
          else if (iw == 3) { rw0 = x; rw1 = (double)a.ny + 0.5 * D; }
          else { rw0 = -0.5 * D; rw1 = y; }
        }
        const double ex = x - rw0, ey = y - rw1;
        D_PW = sqrt(ex * ex + ey * ey);
        double F0 = 0.0, F1 = 0.0;
        if (!(D_PW > D + ZITA)) {
          const double q = (D_PW - D - ZITA) / ZITA;
          if (D_PW <= D + ZITA && D_PW > D) {
            F0 = EPS_W * CIJ * (q * q) * ex / D_PW;
            F1 = EPS_W * CIJ * (q * q) * ey / D_PW;
          } else if (D_PW <= D) {
            const double e = E_W * CIJ * (D - D_PW) / ZITA;
            F0 = (EPS_W * CIJ * (q * q) + e) * ex / D_PW;
            F1 = (EPS_W * CIJ * (q * q) + e) * ey / D_PW;
          }
        }
        fcx = fcx + F0;
        fcy = fcy + F1;
      }
      if (p == a.np - 1) *a.stale_dpw = D_PW;
    }
    P[P_FCX] = fcx;
    P[P_FCY] = fcy;

    // Newton-Euler with internal-mass correction (C1:250-258, C6:312)
    const double RHO0 = a.rho0;
    const double rr = RHO0 / P[P_RHO];
    const double M = P[P_M], I = P[P_I];
    const double fh0 = rr * M * (P[P_U] - P[P_UO]);
    const double fh1 = rr * M * (P[P_V] - P[P_VO]);
    const double fh2 = rr * I * (P[P_W] - P[P_WO]);
    const double vo0 = P[P_U], vo1 = P[P_V], vo2 = P[P_W];
    const double v0 = P[P_U] + P[P_FX] / M + fh0 / M + fcx / M;
    const double v1 = P[P_V] + P[P_FY] / M + fh1 / M + (1.0 - RHO0 / P[P_RHO]) * a.gravity + fcy / M;
    const double v2 = P[P_W] + P[P_TZ] / I + fh2 / I;
    P[P_FHX] = fh0;
    P[P_FHY] = fh1;
    P[P_FHT] = fh2;
    P[P_UO] = vo0;
    P[P_VO] = vo1;
    P[P_WO] = vo2;
    P[P_U] = v0;
    P[P_V] = v1;
    P[P_W] = v2;
    P[P_X] = P[P_X] + 0.5 * (v0 + vo0);
    P[P_Y] = P[P_Y] + 0.5 * (v1 + vo1);
    if (a.integrate_angle) P[P_ANG] = P[P_ANG] + 0.5 * (v2 + vo2);
    if (!isfinite(P[P_X]) || !isfinite(P[P_Y]) || !isfinite(v0) || !isfinite(v1))
      atomicOr(a.status, ST_NAN);
    else if (P[P_X] < 0.0 || P[P_X] > (double)a.nx || P[P_Y] < 0.0 || P[P_Y] > (double)a.ny)
      atomicOr(a.status, ST_PARTICLE);
    if (rec && p < a.series_np) {
      double* r = a.series + rslot * a.series_len + 2 + 12LL * p;
      r[0] = P[P_X]; r[1] = P[P_Y]; r[2] = P[P_ANG];
      r[3] = v0; r[4] = v1; r[5] = v2;
      r[6] = P[P_FX]; r[7] = P[P_FY]; r[8] = P[P_TZ];
      r[9] = fh0; r[10] = fh1; r[11] = fh2;
    }
  }
  __syncthreads();

  // ---- 4. tile candidate lists ----------------------------------------------
  build_tiles(a, tid);
}

__global__ void __launch_bounds__(PBLK) k_tiles_only(const ParticleArgs a) {
  build_tiles(a, threadIdx.x);
}

cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s) {
  k_particles<<<1, PBLK, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_tiles_only(const ParticleArgs& a, cudaStream_t s) {
  k_tiles_only<<<1, PBLK, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace lbm
