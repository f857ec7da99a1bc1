// lbm_particles.cu -- particle kernel of one time step (sm_100a).
//
// One block of PBLK threads; the particle centres and diameters are staged in
// shared memory:
//   0. FORCE of the previous lattice step, decoded from the exact fixed-point
//      accumulators the lattice kernel filled (ComputeForce_HYDRO, C1:546-570);
//   1. Verlet pair lists (cut-off + SKIN) rebuilt from a hashed cell grid only
//      when some disk moved more than SKIN/2 since the last build;
//   2. Glowinski repulsion, pairs then walls (C1:701-768, C3:739-804); each
//      disk sums its pair forces in ascending partner order, the order in
//      which the reference's IP<JP double loop accumulates them;
//      Newton-Euler update with the internal-mass term (C1:247-259,
//      C6:300-312) and the history record (C1:264, C6:315-318);
//   3. per-tile candidate lists for the lattice kernel's SPM evaluation,
//      rebuilt (radius R + zeta/2 + 1 + SKIN) into the idle buffer only when
//      some disk moved more than SKIN/2 from where the lists were built.
// Built with --fmad=false: the FP64 arithmetic is operation-for-operation the
// reference's, so the particle update is bit-identical for identical inputs.
#include <cuda_runtime.h>
#include <cstddef>

#include "lbm_internal.h"

namespace lbm {

constexpr int PBLK = 512;
constexpr int HASH = 4096;  // power of two

struct PShared {
  int cnt[HASH + 1];
  int start[HASH + 1];
  int items[MAX_PARTICLES];
  int key[MAX_PARTICLES];
  double x[MAX_PARTICLES], y[MAX_PARTICLES], d[MAX_PARTICLES];
  int scan[PBLK / 32];
};
// History steps: the records of the first REC_STAGE disks (12 doubles each)
// are staged in the pair hash's part of the shared memory (cnt .. key, dead
// after the pair lists are built) and written out coalesced.  Written one
// disk per thread, 12 doubles at a 96-byte stride, every store of a warp
// touches 32 sectors, and all of them go through the one SM this kernel
// runs on.
constexpr int REC_STAGE =
    (int)((2 * (HASH + 1) + 2 * MAX_PARTICLES) * sizeof(int) / (12 * sizeof(double)));
static_assert(offsetof(PShared, x) >= (size_t)REC_STAGE * 12 * sizeof(double),
              "record staging fits in front of the centre arrays");

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Pair force of (lo, hi), lo < hi, as the reference evaluates F_PP for
// IP = lo, JP = hi (C3:758-766); the contact branch tests D_PP or the stale
// wall distance D_PW.
__device__ __forceinline__ void pair_force(const ParticleArgs& a, double ax, double ay, double ad,
                                           double bx, double by, double bd, double test_stale,
                                           double* F) {
  const double ZITA = a.rep_zeta, CIJ = a.c_ij, EPS_P = a.eps_p, E_P = a.e_p;
  const double dx = ax - bx, dy = ay - by;
  const double D_PP = sqrt(dx * dx + dy * dy);
  const double rsum = 0.5 * ad + 0.5 * bd;
  const double test = a.contact == 1 ? test_stale : D_PP;
  F[0] = 0.0;
  F[1] = 0.0;
  if (D_PP > rsum + ZITA) return;
  const double q = (D_PP - 0.5 * ad - 0.5 * bd - ZITA) / ZITA;
  if (D_PP <= rsum + ZITA && test > rsum) {
    F[0] = EPS_P * CIJ * (q * q) * dx / D_PP;
    F[1] = EPS_P * CIJ * (q * q) * dy / D_PP;
  } else if (test <= rsum) {
    const double e = E_P * CIJ * (rsum - D_PP) / ZITA;
    F[0] = (EPS_P * CIJ * (q * q) + e) * dx / D_PP;
    F[1] = (EPS_P * CIJ * (q * q) + e) * dy / D_PP;
  }
}

// Insert disk p into the candidate lists of the tiles within R + zeta/2 + 1
// + SKIN of (x, y); atomics are issued four at a time so latencies overlap.
__device__ __forceinline__ void insert_tiles(const ParticleArgs& a, int p, double x, double y,
                                             double D, int buf) {
  const double r = 0.5 * D + 0.5 * a.zeta + 1.0 + SKIN;
  int i0 = max((int)ceil(x - r), 0), i1 = min((int)floor(x + r), a.nx);
  int j0 = max((int)ceil(y - r), 0), j1 = min((int)floor(y + r), a.ny);
  if (!(i0 <= i1 && j0 <= j1) || !isfinite(x) || !isfinite(y)) return;
  const int tx0 = i0 / LTX, ty0 = j0 / LTY, ntx = i1 / LTX - tx0 + 1, nty = j1 / LTY - ty0 + 1;
  int* cnt = a.tile_count + (long long)buf * a.ntiles;
  int* lst = a.tile_list + (long long)buf * a.ntiles * a.tile_cap;
  const int nt = ntx * nty;
  for (int t0 = 0; t0 < nt; t0 += 4) {
    int tt[4], sl[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u;
      tt[u] = -1;
      if (t < nt) {
        const int ty = t / ntx, tx = t - ty * ntx;
        const int tile = (ty0 + ty) * a.nbx + tx0 + tx;
        if (LBM_IN(tile, a.ntiles, a.status)) {
          tt[u] = tile;
          sl[u] = atomicAdd(&cnt[tile], 1);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (tt[u] < 0) continue;
      if (sl[u] < a.tile_cap)
        lst[(long long)tt[u] * a.tile_cap + sl[u]] = p;
      else
        atomicOr(a.status, ST_OVERFLOW);
    }
  }
}

// Order of the list tiles of buffer buf for the step kernel's tile queue:
// the tiles without disks first, then those with, each group in index order
// (tile_order[2 buf]) and each group reversed (tile_order[2 buf + 1], for odd
// steps: a step then starts on the rows the previous one wrote last, which
// are still in L2); n_unlisted[buf] = size of the first group.  Run by one
// block.
__device__ void build_tile_order(const ParticleArgs& a, int buf) {
  __shared__ int s_w[PBLK / 32];
  __shared__ int s_base[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x / 32;
  const int* cnt = a.tile_count + (long long)buf * a.ntiles;
  int* ord = a.tile_order + (long long)(2 * buf) * a.ntiles;
  int* rev = ord + a.ntiles;
  int nu = 0;
  for (int t = tid; t < a.ntiles; t += blockDim.x) nu += cnt[t] == 0 ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) nu += __shfl_xor_sync(0xffffffffu, nu, o);
  if (lane == 0) s_w[warp] = nu;
  if (tid == 0) s_base[0] = s_base[1] = 0;
  __syncthreads();
  int total_u = 0;
  for (int w = 0; w < nw; ++w) total_u += s_w[w];
  __syncthreads();
  for (int c0 = 0; c0 < a.ntiles; c0 += blockDim.x) {
    const int t = c0 + tid;
    const bool in = t < a.ntiles;
    const bool un = in && cnt[t] == 0;
    // counts packed as unlisted | listed << 16 (at most 1024 per chunk)
    const int v = (un ? 1 : 0) | ((in && !un) ? 1 << 16 : 0);
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    int before = 0, chunk = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) before += s_w[w];
      chunk += s_w[w];
    }
    const int ex = before + inc - v;
    if (un) {
      const int pos = s_base[0] + (ex & 0xffff);
      if (LBM_IN(pos, total_u, a.status)) {
        ord[pos] = t;
        rev[total_u - 1 - pos] = t;
      }
    } else if (in) {
      const int pos = total_u + s_base[1] + (ex >> 16);
      if (LBM_IN(pos, a.ntiles, a.status) && LBM_IN(pos - total_u, a.ntiles - total_u, a.status)) {
        ord[pos] = t;
        rev[a.ntiles - 1 + total_u - pos] = t;
      }
    }
    __syncthreads();
    if (tid == 0) {
      s_base[0] += chunk & 0xffff;
      s_base[1] += chunk >> 16;
    }
    __syncthreads();
  }
  if (tid == 0) a.n_unlisted[buf] = total_u;
}

__device__ __forceinline__ int cell_key(const ParticleArgs& a, double x, double y) {
  const int cx = clampi((int)floor(x / a.cell_size), 0, a.ncx - 1);
  const int cy = clampi((int)floor(y / a.cell_size), 0, a.ncy - 1);
  return cy * a.ncx + cx;
}

// Verlet lists: hash the staged centres into HASH buckets (counting sort),
// then collect, for each disk, the partners within cut-off + SKIN in
// ascending index order.
__device__ void rebuild_pairs(const ParticleArgs& a, PShared& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int b = tid; b <= HASH; b += PBLK) S.cnt[b] = 0;
  __syncthreads();
  for (int p = tid; p < a.np; p += PBLK) {
    const int key = cell_key(a, S.x[p], S.y[p]);
    S.key[p] = key;
    atomicAdd(&S.cnt[key & (HASH - 1)], 1);
  }
  __syncthreads();
  constexpr int PER = HASH / PBLK;
  int loc[PER];
  int sum = 0;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    loc[u] = S.cnt[tid * PER + u];
    sum += loc[u];
  }
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) S.scan[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < PBLK / 32 ? S.scan[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += v;
    }
    if (lane < PBLK / 32) S.scan[lane] = wi - w;
  }
  __syncthreads();
  int run = S.scan[warp] + incl - sum;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    S.start[tid * PER + u] = run;
    S.cnt[tid * PER + u] = run;  // scatter cursor
    run += loc[u];
  }
  if (tid == PBLK - 1) S.start[HASH] = run;
  __syncthreads();
  for (int p = tid; p < a.np; p += PBLK) {
    const int slot = atomicAdd(&S.cnt[S.key[p] & (HASH - 1)], 1);
    if (LBM_IN(slot, a.np, a.status)) S.items[slot] = p;
  }
  __syncthreads();
  for (int p = tid; p < a.np; p += PBLK) {
    const double px = S.x[p], py = S.y[p], pd = S.d[p];
    int nbl[MAX_NEIGH];
    int nn = 0;
    const int key = S.key[p];
    const int cx = key % a.ncx, cy = key / a.ncx;
    for (int yy = max(cy - 1, 0); yy <= min(cy + 1, a.ncy - 1); ++yy)
      for (int xx = max(cx - 1, 0); xx <= min(cx + 1, a.ncx - 1); ++xx) {
        const int ck = yy * a.ncx + xx;
        const int b = ck & (HASH - 1);
        for (int s = S.start[b]; s < S.start[b + 1]; ++s) {
          const int q = S.items[s];
          if (!LBM_IN(q, a.np, a.status) || q == p || S.key[q] != ck) continue;
          const double dx = px - S.x[q], dy = py - S.y[q];
          const double lim = 0.5 * pd + 0.5 * S.d[q] + a.rep_zeta + SKIN;
          if (dx * dx + dy * dy > lim * lim) continue;
          if (nn < MAX_NEIGH) {
            int k = nn++;
            while (k > 0 && nbl[k - 1] > q) {
              nbl[k] = nbl[k - 1];
              --k;
            }
            nbl[k] = q;
          } else {
            atomicOr(a.status, ST_OVERFLOW);
          }
        }
      }
    for (int k = 0; k < nn; ++k) a.nbr[(long long)k * a.npad + p] = nbl[k];
    a.nbr_count[p] = nn;
    a.nbr_xy[p] = px;
    a.nbr_xy[a.npad + p] = py;
  }
}

__device__ __forceinline__ void particles_body(const ParticleArgs& a);

__global__ void __launch_bounds__(PBLK) k_particles(const ParticleArgs a) { particles_body(a); }

// Batched: block b runs the particle step of simulation b.
__global__ void __launch_bounds__(PBLK) k_particles_batch(const ParticleArgs* __restrict__ args) {
  particles_body(args[blockIdx.x]);
}

__device__ __forceinline__ void particles_body(const ParticleArgs& a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PShared& S = *reinterpret_cast<PShared*>(smem_raw);
  __shared__ long long s_kk;
  __shared__ int s_pairs, s_tiles;
  const int tid = threadIdx.x;
  // Launched as a programmatic dependent of the previous step's lattice
  // kernel: resident early, it waits here for that kernel (whose force sums
  // it decodes and whose particle reads must end before the update below).
  // Then the lattice kernel of this step may start its particle-free tiles.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (tid == 0) {
    const long long k1 = *a.kk + 1;
    s_kk = k1;
    *a.kk = k1;
    s_pairs = *a.pair_rebuild;
    s_tiles = 0;
    // the tile queue of the next step (its last user, the step kernel of
    // step k1 - 1, has completed)
    a.work_ctr[(k1 + 1) & 1] = 0;
    const bool r = a.series != nullptr && a.series_every > 0 && (k1 % a.series_every) == 0;
    const long long slot = r ? (k1 / a.series_every - 1) % a.series_cap : -1;
    *a.rec_slot = (int)slot;  // read by the lattice kernel of this step
    if (r) {
      a.series[slot * a.series_len + 0] = (double)k1;
      a.series[slot * a.series_len + 1] = __longlong_as_double(0x7ff8000000000000LL);
    }
  }
  const double stale = *a.stale_dpw;  // D_PW left over from the previous call
  __syncthreads();
  const long long kk = s_kk;
  const bool rec = a.series != nullptr && a.series_every > 0 && (kk % a.series_every) == 0;
  const long long rslot = rec ? (kk / a.series_every - 1) % a.series_cap : 0;

  // ---- 0. FORCE of the last lattice step; stage centres ------------------
  for (int p = tid; p < a.np; p += PBLK) {
    const PRef P{a.ps + p, a.npad};
    if (a.decode_force) {
      unsigned long long* acc = a.facc + p;
      const long long st = a.npad;
      const double fx = decode_force(acc[0], acc[st]);
      const double fy = decode_force(acc[2 * st], acc[3 * st]);
      const double tz = decode_force(acc[4 * st], acc[5 * st]);
#pragma unroll
      for (int k = 0; k < 6; ++k) acc[k * st] = 0ull;
      P[P_FX] = fx;
      P[P_FY] = fy;
      P[P_TZ] = tz;
      if (!isfinite(fx) || !isfinite(fy) || !isfinite(tz)) atomicOr(a.status, ST_NAN);
    }
    const double x = P[P_X], y = P[P_Y];
    S.x[p] = x;
    S.y[p] = y;
    S.d[p] = P[P_D];
    if (a.np > 1) {
      const double ddx = x - a.nbr_xy[p], ddy = y - a.nbr_xy[a.npad + p];
      if (!(ddx * ddx + ddy * ddy <= 0.25 * SKIN * SKIN)) s_pairs = 1;
    }
  }
  __syncthreads();

  // ---- 1. pair lists -------------------------------------------------------
  if (a.np > 1 && s_pairs) {
    rebuild_pairs(a, S);
    if (tid == 0) *a.pair_rebuild = 0;
  }

  // ---- 2. repulsion, Newton-Euler update, history -------------------------
  double* const rstage = reinterpret_cast<double*>(smem_raw);
  if (rec) __syncthreads();  // the pair search has finished with the hash
  for (int p = tid; p < a.np; p += PBLK) {
    const PRef P{a.ps + p, a.npad};
    // issue every global load of this disk before the dependent arithmetic
    const double u0 = P[P_U], u1 = P[P_V], u2 = P[P_W];
    const double uo0 = P[P_UO], uo1 = P[P_VO], uo2 = P[P_WO];
    const double frx = P[P_FX], fry = P[P_FY], frt = P[P_TZ];
    const double rhop = P[P_RHO], M = P[P_M], I = P[P_I], ang = P[P_ANG];
    const double xt = P[P_XT], yt = P[P_YT];
    const double px = S.x[p], py = S.y[p], pd = S.d[p];
    // The neighbour count and the first 8 list entries load together (the
    // list has room for MAX_NEIGH entries of every disk; those past the
    // count are masked below), and the wall forces, which need neither, are
    // formed while they are in flight.  The sums keep the order of the
    // reference: the pairs, then walls 1 to 4.
    int nn = 0, nraw[8];
    if (a.np > 1) {
      nn = a.nbr_count[p];
#pragma unroll
      for (int k = 0; k < 8; ++k) nraw[k] = a.nbr[(long long)k * a.npad + p];
    }
    double wf0[4] = {0.0, 0.0, 0.0, 0.0}, wf1[4] = {0.0, 0.0, 0.0, 0.0};
    // walls (C1:735-768 mirror images; C3:775-804 wall disks)
    if (a.wall_model != 2) {
      const double ZITA = a.rep_zeta, CIJ = a.c_ij, EPS_W = a.eps_w, E_W = a.e_w;
      const double x = px, y = py, D = pd;
      double D_PW = stale;
#pragma unroll
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
        wf0[iw - 1] = F0;
        wf1[iw - 1] = F1;
      }
      if (p == a.np - 1) *a.stale_dpw = D_PW;
    }
    double fcx = 0.0, fcy = 0.0;
    if (a.np > 1) {
      if (!LBM_IN(nn, MAX_NEIGH + 1, a.status)) nn = 0;
      int nbl[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) nbl[k] = k < nn ? nraw[k] : 0;
      for (int k = 0; k < nn; ++k) {
        const int q = k < 8 ? nbl[k] : a.nbr[(long long)k * a.npad + p];
        if (!LBM_IN(q, a.np, a.status)) continue;
        double F[2];
        if (q < p) {
          pair_force(a, S.x[q], S.y[q], S.d[q], px, py, pd, stale, F);
          fcx = fcx - F[0];
          fcy = fcy - F[1];
        } else {
          pair_force(a, px, py, pd, S.x[q], S.y[q], S.d[q], stale, F);
          fcx = fcx + F[0];
          fcy = fcy + F[1];
        }
      }
    }
    if (a.wall_model != 2) {
#pragma unroll
      for (int iw = 0; iw < 4; ++iw) {
        fcx = fcx + wf0[iw];
        fcy = fcy + wf1[iw];
      }
    }
    P[P_FCX] = fcx;
    P[P_FCY] = fcy;

    // Newton-Euler with internal-mass correction (C1:250-258, C6:312), or
    // the prescribed oscillation (C4:222-228) with F_H_IN of this step's
    // velocity change (C4:270-272)
    const double RHO0 = a.rho0;
    const double rr = RHO0 / rhop;
    double fh0, fh1, fh2, v0, v1, v2;
    if (a.motion == MOTION_OSCILLATE) {
      v0 = -(a.osc_u * cos(((2.0 * a.pi) * (double)s_kk) / a.osc_period));
      v1 = 0.0;
      v2 = 0.0;
      fh0 = rr * M * (v0 - u0);
      fh1 = rr * M * (v1 - u1);
      fh2 = rr * I * (v2 - u2);
    } else {
      fh0 = rr * M * (u0 - uo0);
      fh1 = rr * M * (u1 - uo1);
      fh2 = rr * I * (u2 - uo2);
      v0 = u0 + frx / M + fh0 / M + fcx / M;
      v1 = u1 + fry / M + fh1 / M + (1.0 - RHO0 / rhop) * a.gravity + fcy / M;
      v2 = u2 + frt / I + fh2 / I;
    }
    const double nx_ = px + 0.5 * (v0 + u0);
    const double ny_ = py + 0.5 * (v1 + u1);
    P[P_FHX] = fh0;
    P[P_FHY] = fh1;
    P[P_FHT] = fh2;
    P[P_UO] = u0;
    P[P_VO] = u1;
    P[P_WO] = u2;
    P[P_U] = v0;
    P[P_V] = v1;
    P[P_W] = v2;
    P[P_X] = nx_;
    P[P_Y] = ny_;
    const double nang = a.integrate_angle ? ang + 0.5 * (v2 + u2) : ang;
    if (a.integrate_angle) P[P_ANG] = nang;
    if (!isfinite(nx_) || !isfinite(ny_) || !isfinite(v0) || !isfinite(v1))
      atomicOr(a.status, ST_NAN);
    else if (nx_ < 0.0 || nx_ > (double)a.nx || ny_ < 0.0 || ny_ > (double)a.ny)
      atomicOr(a.status, ST_PARTICLE);
    if (rec && p < a.series_np) {
      double* r = p < REC_STAGE ? rstage + 12LL * p : a.series + rslot * a.series_len + 2 + 12LL * p;
      r[0] = nx_; r[1] = ny_; r[2] = nang;
      r[3] = v0; r[4] = v1; r[5] = v2;
      r[6] = frx; r[7] = fry; r[8] = frt;
      r[9] = fh0; r[10] = fh1; r[11] = fh2;
    }
    if (a.hist && kk < a.hist_n) {
      double* hr = a.hist + kk * (long long)PS * a.npad + p;
      for (int f = 0; f < PS; ++f) hr[(long long)f * a.npad] = P[f];
    }
    const double tdx = nx_ - xt, tdy = ny_ - yt;
    if (!(tdx * tdx + tdy * tdy <= 0.25 * SKIN * SKIN)) s_tiles = 1;
  }
  __syncthreads();
  if (rec) {  // the staged records, coalesced
    const int n = 12 * (a.series_np < REC_STAGE ? a.series_np : REC_STAGE);
    double* const dst = a.series + rslot * a.series_len + 2;
    for (int e = tid; e < n; e += PBLK) dst[e] = rstage[e];
  }

  // ---- 3. tile candidate lists ---------------------------------------------
  // The lattice kernel of this step, already running, sorts its tiles by the
  // lists of the previous step (tile_cur[(k-1)&1]); a rebuild goes into the
  // other buffer, published as tile_cur[k&1].
  const int cur = a.tile_cur[(s_kk - 1) & 1];
  if (!s_tiles && tid == 0) a.tile_cur[s_kk & 1] = cur;
  if (s_tiles) {
    const int buf = 1 - cur;
    int* cnt = a.tile_count + (long long)buf * a.ntiles;
    for (int t = tid; t < a.ntiles; t += PBLK) cnt[t] = 0;
    __syncthreads();
    for (int p = tid; p < a.np; p += PBLK) {  // new centres, written above
      const PRef P{a.ps + p, a.npad};
      const double x = P[P_X], y = P[P_Y];
      insert_tiles(a, p, x, y, P[P_D], buf);
      P[P_XT] = x;
      P[P_YT] = y;
    }
    __syncthreads();
    build_tile_order(a, buf);
    __syncthreads();
    if (tid == 0) a.tile_cur[s_kk & 1] = buf;
  }
}

// After set_particles / set_state: tile lists into buffer 0 (cleared by the
// host) and a pair-list rebuild request for the next particle kernel.
__global__ void __launch_bounds__(256) k_tiles_only(const ParticleArgs a) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.np; p += gridDim.x * blockDim.x) {
    const PRef P{a.ps + p, a.npad};
    insert_tiles(a, p, P[P_X], P[P_Y], P[P_D], 0);
    P[P_XT] = P[P_X];
    P[P_YT] = P[P_Y];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.tile_cur[0] = a.tile_cur[1] = 0;
    *a.pair_rebuild = 1;
  }
}

// The batched particle kernel's shared-memory size, set on the current
// device before any launch (and so before any graph capture).
cudaError_t prepare_particles_batch() {
  return cudaFuncSetAttribute(k_particles_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(PShared));
}

cudaError_t launch_particles_batch(const ParticleArgs* args, int nsim, cudaStream_t s) {
  k_particles_batch<<<nsim, PBLK, sizeof(PShared), s>>>(args);
  return cudaGetLastError();
}

cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s) {
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_particles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(PShared));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(PBLK);
  cfg.dynamicSmemBytes = sizeof(PShared);
  cfg.stream = s;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_particles, a);
}

__global__ void __launch_bounds__(PBLK) k_tile_order(const ParticleArgs a, int buf) {
  build_tile_order(a, buf);
}

cudaError_t launch_tile_order(const ParticleArgs& a, int buf, cudaStream_t s) {
  k_tile_order<<<1, PBLK, 0, s>>>(a, buf);
  return cudaGetLastError();
}

cudaError_t launch_tiles_only(const ParticleArgs& a, cudaStream_t s) {
  const int blocks = (a.np + 255) / 256 > 0 ? (a.np + 255) / 256 : 1;
  k_tiles_only<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace lbm
