// lbm_api.cu -- C ABI of include/lbm2d.h: handle life cycle, the per-step
// launch sequence, and the getters/setters.
//
// Per time step the host enqueues two kernels on the handle's stream:
//   k_particles  repulsion, Newton-Euler update, history, tile lists
//   k_step       stream + BC + macro + SPM + force sums + correction +
//                collision of the next step (persistent, TMA-fed)
// The post-collision populations live in a ping-pong pair: after step K,
// f[cur] holds f*(K+1) and f[cur^1] holds f*(K), from which the output
// kernel re-derives the fields of step K (F after BC, rho, u, G, PHI) on
// demand without touching the state.
#include <algorithm>
#include <cmath>
#include <deque>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm2d.h"
#include "lbm_internal.h"

using namespace lbm;

struct lbm_sim {
  CUtensorMap tm[2];   // TMA descriptors of f[0], f[1] for the step kernel
  CUtensorMap tmo[2];  // and of om[0], om[1] (Bingham models; else copies of tm)
  lbm_params p;
  cudaStream_t stream = nullptr;
  Geometry g{};
  Model m{};
  int prec = 0;
  size_t esz = 8;
  void* f[2] = {nullptr, nullptr};
  void* om[2] = {nullptr, nullptr};
  void* pm[2] = {nullptr, nullptr};  // previous-collision macros (BGK bi-viscosity)
  void* rec = nullptr;
  void* ring = nullptr;  // equilibrium boundary: T[2][3][ring_n]
  int ring_n = 0;
  int cur = 0;
  bool prev_post_bc = false;
  int64_t kk = 0;
  // particles
  int np = 0;
  int np_cap = 0;
  double* ps = nullptr;                // [PS][npad]
  int npad = 32;
  unsigned long long* facc = nullptr;  // [6][npad] FORCE accumulators
  int* rec_slot = nullptr;
  int* tile_count = nullptr;
  int* tile_list = nullptr;
  int* tile_cur = nullptr;
  int* tile_order = nullptr;  // [2 buffers][forward, reversed][ntiles]
  int* n_unlisted = nullptr;  // [2]
  int* work_ctr = nullptr;    // [2]
  int tile_cap = MAX_TILE_CAND;
  int* nbr = nullptr;
  int* nbr_count = nullptr;
  double* nbr_xy = nullptr;
  int* pair_rebuild = nullptr;
  double* ps_pin = nullptr;     // pinned staging of the particle upload [PS][npad]
  size_t ps_pin_n = 0;          // its size in doubles
  bool partials_valid = false;  // facc holds FORCE of the last lattice step
  int ncx = 1, ncy = 1;
  double cell_size = 1.0;
  // scalars
  unsigned long long* mass_acc = nullptr;
  long long* d_kk = nullptr;
  double* stale_dpw = nullptr;
  int* h_status = nullptr;  // pinned copy of d_status, refreshed after each call
  int* d_status = nullptr;  // sticky ST_* bits written by the kernels
  // history
  double* series = nullptr;
  int series_len = LBM_SERIES_HEAD;
  int series_cap = 0;
  int series_np = 0;
  int64_t drained_kk = 0;      // records of steps <= drained_kk are in host_series
  int64_t copied_kk = 0;       // records of steps <= copied_kk have their copies queued
  std::vector<double> host_series;
  size_t host_series_read = 0;
  // pinned staging ring of the history records and their mean-density sums,
  // filled by copies on copy_stream queued after the kernels that wrote them
  // (so the next steps' kernels run while they cross to the host)
  double* series_pin = nullptr;              // [series_pcap][series_len]
  unsigned long long* mass_pin = nullptr;    // [series_pcap]
  int series_pcap = 0;
  struct SeriesBatch {
    long long r_end;  // records [drained record, r_end) complete with ev
    cudaEvent_t ev;
  };
  std::deque<SeriesBatch> series_pending;
  std::vector<cudaEvent_t> series_ev_free;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_fork = nullptr;  // the kernels that wrote a batch, on stream
  int64_t ring_free = 0;  // the stream has waited for the copies of records < ring_free
  // COMPUTEERROR: velocity of the previous call, per-block partial sums
  double* u0 = nullptr;       // [2][nodes]
  double* err_part = nullptr;
  // output scratch
  double* out = nullptr;
  double* out_f = nullptr;
  int64_t out_kk = -1;
  // per-kernel profiling (lbm_profile)
  bool prof = false;
  std::vector<cudaEvent_t> ev;  // 3 per profiled step
  size_t ev_used = 0;
  double prof_ms[2] = {0.0, 0.0};
  int64_t prof_n[2] = {0, 0};
  // adjoint sweep (lbm_adjoint), allocated on first use and kept
  unsigned char* adj_slots = nullptr;  // [nslots][10 planes]: f*(n) then omega(n)
  int adj_nslots = 0;
  std::vector<CUtensorMap> adj_tm;     // TMA descriptor of each slot's f*
  std::vector<CUtensorMap> adj_tmo;    // and of its omega plane
  unsigned char* adj_ck = nullptr;     // [nck][10 planes] checkpoints
  int adj_nck = 0;
  double* adj_ckp = nullptr;           // [nck+1][ckp_len]: records, FORCE sums, D_PW
  double* adj_hist = nullptr;          // [nhist][PS][npad] particle records of every step
  long long adj_nhist = 0;
  void* adj_a[2] = {nullptr, nullptr};  // dJ/dF, T[9 planes]
  void* adj_w[2] = {nullptr, nullptr};  // dJ/domega, T[plane]
  double* adj_state = nullptr;         // [8][npad]
  double* adj_p = nullptr;             // [5][npad]
  double* adj_h = nullptr;             // [3][npad]
  double* adj_rho = nullptr;           // [npad]
  double* adj_g = nullptr;             // [blocks][2]
  int adj_npad = 0;
  bool adj_record = false;  // the particle kernel writes adj_hist (forward pass)
  cudaStream_t adj_rs = nullptr;  // recompute stream of the reverse sweep
  // recompute done with slot set 0/1, reverse done with set 0/1, fork/join
  cudaEvent_t adj_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace {

constexpr int NOUT = 7;  // ux uy rho phi gx gy pnode

int cuda_fail(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return LBM_E_NOMEM;
  return LBM_E_CUDA;
}

#define CK(expr)                                 \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return cuda_fail(e_); \
  } while (0)

template <class T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(e);
  }
  return LBM_OK;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// All copies are ordered on the handle's (non-blocking) stream; copies to the
// host wait for completion.
cudaError_t h2d(lbm_sim* h, void* dst, const void* src, size_t bytes) {
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
}
cudaError_t d2h(lbm_sim* h, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(h->stream);
}

long long nodes(const lbm_sim* h) { return (long long)(h->p.nx + 1) * (h->p.ny + 1); }

int sticky_status(const lbm_sim* h) {
  const int s = *(volatile int*)h->h_status;  // as of the last completed copy
  if (s & ST_NAN) return LBM_E_NAN;
  if (s & ST_OVERFLOW) return LBM_E_OVERFLOW;
  if (s & ST_TIMEOUT) return LBM_E_TIMEOUT;
  if (s & ST_BOUNDS) return LBM_E_BOUNDS;
  if (s & ST_PARTICLE) return LBM_E_PARTICLE;
  return LBM_OK;
}

// Synchronising variant for the getters.
int refreshed_status(lbm_sim* h) {
  if (cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return LBM_E_CUDA;
  return sticky_status(h);
}

LatticeArgs lattice_args(lbm_sim* h) {
  LatticeArgs a{};
  a.g = h->g;
  a.m = h->m;
  a.src = h->f[h->cur];
  a.dst = h->f[h->cur ^ 1];
  a.om_src = h->om[h->cur];
  a.om_dst = h->om[h->cur ^ 1];
  a.pm_src = h->pm[h->cur];
  a.pm_dst = h->pm[h->cur ^ 1];
  a.ps = h->ps;
  a.np = h->np;
  a.npad = h->npad;
  a.step = h->kk;
  a.rec_slot = -1;
  if (h->series && h->p.series_every > 0 && h->kk > 0 && h->kk % h->p.series_every == 0)
    a.rec_slot = (int)((h->kk / h->p.series_every - 1) % h->series_cap);
  a.tile_count = h->tile_count;
  a.tile_list = h->tile_list;
  a.tile_cur = h->tile_cur;
  a.tile_order = h->tile_order;
  a.n_unlisted = h->n_unlisted;
  a.work_ctr = h->work_ctr;
  a.tile_cap = h->tile_cap;
  a.ntiles = h->g.ltx * h->g.lty;
  a.facc = h->facc;
  a.mass_acc = h->series ? h->mass_acc : nullptr;
  a.status = h->d_status;
  a.rec = h->rec;
  a.ring = h->ring;
  a.ring_n = h->ring_n;
  return a;
}

ParticleArgs particle_args(lbm_sim* h) {
  ParticleArgs a{};
  a.ps = h->ps;
  a.np = h->np;
  a.npad = h->npad;
  a.rec_slot = h->rec_slot;
  a.facc = h->facc;
  a.decode_force = h->partials_valid ? 1 : 0;
  a.tile_count = h->tile_count;
  a.tile_list = h->tile_list;
  a.tile_cur = h->tile_cur;
  a.tile_order = h->tile_order;
  a.n_unlisted = h->n_unlisted;
  a.work_ctr = h->work_ctr;
  a.tile_cap = h->tile_cap;
  a.ntiles = h->g.ltx * h->g.lty;
  a.nbx = h->g.ltx;
  a.nbr = h->nbr;
  a.nbr_count = h->nbr_count;
  a.nbr_xy = h->nbr_xy;
  a.pair_rebuild = h->pair_rebuild;
  a.wall_model = h->p.wall_model;
  a.contact = h->p.contact_test;
  a.rep_zeta = h->p.rep_zeta;
  a.eps_p = h->p.eps_p;
  a.eps_w = h->p.eps_w;
  a.e_p = h->p.e_p;
  a.e_w = h->p.e_w;
  a.c_ij = h->p.c_ij;
  a.mirror_top = h->p.wall_mirror_top;
  a.mirror_left = h->p.wall_mirror_left;
  a.rho0 = h->p.rho0;
  a.gravity = h->p.gravity;
  a.integrate_angle = h->p.integrate_angle;
  a.ncx = h->ncx;
  a.ncy = h->ncy;
  a.cell_size = h->cell_size;
  a.stale_dpw = h->stale_dpw;
  a.kk = h->d_kk;
  a.series = h->series;
  a.mass_acc = h->series ? h->mass_acc : nullptr;
  a.series_every = h->p.series_every;
  a.series_cap = h->series_cap;
  a.series_len = h->series_len;
  a.series_np = h->series_np;
  a.status = h->d_status;
  a.nx = h->p.nx;
  a.ny = h->p.ny;
  a.zeta = h->p.zeta;
  a.motion = h->p.motion;
  a.osc_u = h->p.osc_u;
  a.osc_period = h->p.osc_period;
  a.pi = h->p.pi;
  a.hist = h->adj_record ? h->adj_hist : nullptr;
  a.hist_n = h->adj_record ? h->adj_nhist : 0;
  return a;
}

cudaError_t launch_lattice(lbm_sim* h, const LatticeArgs& a, int mode) {
  // the BGK collision (C1:774-841) runs in the one-node-per-thread step
  if (mode == 0 && h->m.bgk)
    return h->prec == LBM_FP64 ? launch_bgk_step_fp64(a, h->stream)
                               : launch_bgk_step_fp32(a, h->stream);
  if (h->prec == LBM_FP64) {
    switch (mode) {
      case 0: return launch_step_fp64(a, &h->tm[h->cur], &h->tmo[h->cur], h->stream);
      case 1: return launch_output_fp64(a, h->stream);
      case 2: return launch_init_fp64(a, h->stream);
      default: return launch_restart_fp64(a, h->stream);
    }
  }
  switch (mode) {
    case 0: return launch_step_fp32(a, &h->tm[h->cur], &h->tmo[h->cur], h->stream);
    case 1: return launch_output_fp32(a, h->stream);
    case 2: return launch_init_fp32(a, h->stream);
    default: return launch_restart_fp32(a, h->stream);
  }
}

// History records.  Record r (step (r+1)*every) sits in slot r % series_cap
// of the device ring.  series_enqueue queues, on the copy stream after the
// kernels that wrote them (an event of the handle's stream), the copies of
// the records not yet queued into the pinned staging ring (slot
// r % series_pcap), with their mean-density sums, and clears those sums on
// the device; before a step writes a slot again, ring_wait makes the
// handle's stream wait for the copy of the slot's previous record.
// series_absorb_one waits for the oldest queued batch only and moves it into
// host_series.
int series_absorb_one(lbm_sim* h) {
  const lbm_sim::SeriesBatch b = h->series_pending.front();
  CK(cudaEventSynchronize(b.ev));
  h->series_pending.pop_front();
  h->series_ev_free.push_back(b.ev);
  const int every = h->p.series_every;
  const long long r0 = h->drained_kk / every;
  const size_t len = (size_t)h->series_len;
  const size_t old = h->host_series.size();
  h->host_series.resize(old + (size_t)(b.r_end - r0) * len);
  double* dst = h->host_series.data() + old;
  const double nn = (double)nodes(h);
  for (long long r = r0; r < b.r_end; ++r, dst += len) {
    const long long ps = r % h->series_pcap;
    std::memcpy(dst, h->series_pin + ps * len, len * sizeof(double));
    // AvgDen = rho0 + sum(rho - rho0)/N from the fixed-point accumulator
    dst[1] = h->p.rho0 + (double)(long long)h->mass_pin[ps] / MASS_FIX / nn;
  }
  h->drained_kk = b.r_end * every;
  return LBM_OK;
}

int series_enqueue(lbm_sim* h) {
  const int every = h->p.series_every;
  if (!h->series || every <= 0) {
    h->copied_kk = h->drained_kk = h->kk;
    return LBM_OK;
  }
  const long long r0 = h->copied_kk / every, r1 = h->kk / every;
  if (r1 <= r0) return LBM_OK;
  int rc;
  while (!h->series_pending.empty() && r1 - h->drained_kk / every > h->series_pcap)
    if ((rc = series_absorb_one(h))) return rc;
  const size_t len = (size_t)h->series_len;
  const long long cap = h->series_cap, pcap = h->series_pcap;
  CK(cudaEventRecord(h->copy_fork, h->stream));
  CK(cudaStreamWaitEvent(h->copy_stream, h->copy_fork, 0));
  for (long long r = r0; r < r1;) {
    const long long ds = r % cap, ps = r % pcap;
    const long long cnt = std::min(r1 - r, std::min(cap - ds, pcap - ps));
    CK(cudaMemcpyAsync(h->series_pin + ps * len, h->series + ds * len, cnt * len * sizeof(double),
                       cudaMemcpyDeviceToHost, h->copy_stream));
    CK(cudaMemcpyAsync(h->mass_pin + ps, h->mass_acc + ds, cnt * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, h->copy_stream));
    // the slots start at zero again before the ring comes back to them
    CK(cudaMemsetAsync(h->mass_acc + ds, 0, cnt * sizeof(unsigned long long), h->copy_stream));
    r += cnt;
  }
  cudaEvent_t ev = nullptr;
  if (!h->series_ev_free.empty()) {
    ev = h->series_ev_free.back();
    h->series_ev_free.pop_back();
  } else {
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  CK(cudaEventRecord(ev, h->copy_stream));
  h->series_pending.push_back({r1, ev});
  h->copied_kk = r1 * every;
  return LBM_OK;
}

// Every record of steps up to kk into host_series.
int drain_series(lbm_sim* h) {
  int rc = series_enqueue(h);
  if (rc) return rc;
  while (!h->series_pending.empty())
    if ((rc = series_absorb_one(h))) return rc;
  return LBM_OK;
}

// Drop the queued batches (callers synchronise the handle's stream first;
// the copies are waited for here) and the records not yet drained.
void series_reset(lbm_sim* h, long long kk) {
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for (const auto& b : h->series_pending) h->series_ev_free.push_back(b.ev);
  h->series_pending.clear();
  h->drained_kk = h->copied_kk = kk;
  h->ring_free = h->p.series_every > 0 ? kk / h->p.series_every + h->series_cap : 0;
}

// Before the step that writes record r: the handle's stream waits for the
// copy (and the cleared sum) of the record that held its slot before,
// r - series_cap, unless it has already waited for it or the host has seen
// that copy complete.
int ring_wait(lbm_sim* h, long long r) {
  const long long prev = r - h->series_cap;
  if (prev < 0 || r < h->ring_free) return LBM_OK;
  const long long drained = h->drained_kk / h->p.series_every;
  if (prev < drained) {  // absorbed: its copy has completed
    h->ring_free = drained + h->series_cap;
    return LBM_OK;
  }
  // queued (enqueue_step queues a record's copy before its slot comes back)
  for (const auto& b : h->series_pending) {
    if (b.r_end > prev) {
      CK(cudaStreamWaitEvent(h->stream, b.ev, 0));
      h->ring_free = b.r_end + h->series_cap;
      return LBM_OK;
    }
  }
  return LBM_E_STATE;
}

// Fields of step kk in h->out (and F after BC in h->out_f when want_f).
int compute_output(lbm_sim* h, bool want_f) {
  if (h->out_kk == h->kk && (!want_f || h->out_f)) return LBM_OK;
  LatticeArgs a = lattice_args(h);
  a.src = h->f[h->cur ^ 1];
  a.om_src = h->om[h->cur ^ 1];
  a.out = h->out;
  a.out_f = want_f ? h->out_f : nullptr;
  a.src_post_bc = h->prev_post_bc ? 1 : 0;
  a.initial = (h->kk == 0 && !h->prev_post_bc) ? 1 : 0;
  CK(launch_lattice(h, a, 1));
  CK(cudaStreamSynchronize(h->stream));
  h->out_kk = h->kk;
  return LBM_OK;
}

int setup_particle_buffers(lbm_sim* h, int np, double dmax) {
  // buffers of the same sizes are kept and cleared, so a driver that resets
  // its disks between runs pays no allocation
  const int npad = (std::max(np, 1) + 31) / 32 * 32;
  const int series_np = std::max(0, std::min(h->p.series_particles, np));
  const int series_len = LBM_SERIES_HEAD + LBM_SERIES_PER * series_np;
  const int series_cap = std::max(1, h->p.series_capacity);
  const bool keep_p = h->ps && npad == h->npad;
  const bool keep_s = h->series && h->p.series_every > 0 && series_len == h->series_len &&
                      series_cap == h->series_cap;
  if (!keep_p) {
    dfree(h->ps); dfree(h->facc); dfree(h->nbr); dfree(h->nbr_count); dfree(h->nbr_xy);
    h->ps = nullptr; h->facc = nullptr; h->nbr = nullptr; h->nbr_count = nullptr;
    h->nbr_xy = nullptr;
  }
  // records of the old disk set (its record length) are dropped
  series_reset(h, h->kk);
  h->host_series.clear();
  h->host_series_read = 0;
  if (!keep_s) {
    dfree(h->series); dfree(h->mass_acc);
    h->series = nullptr; h->mass_acc = nullptr;
    if (h->series_pin) cudaFreeHost(h->series_pin);
    if (h->mass_pin) cudaFreeHost(h->mass_pin);
    h->series_pin = nullptr;
    h->mass_pin = nullptr;
  }
  h->np = np;
  h->partials_valid = false;
  // pair search cells cover the Verlet radius D_max + repulsion range + SKIN
  h->cell_size = std::max(1.0, dmax + h->p.rep_zeta + SKIN) * (1.0 + 1e-9);
  h->ncx = std::max(1, (int)std::floor((double)h->p.nx / h->cell_size) + 1);
  h->ncy = std::max(1, (int)std::floor((double)h->p.ny / h->cell_size) + 1);
  int rc;
  h->npad = npad;
  const size_t npa = (size_t)h->npad;
  if (!keep_p) {
    if ((rc = dalloc(&h->ps, npa * PS))) return rc;
    if ((rc = dalloc(&h->facc, npa * 6))) return rc;
    if ((rc = dalloc(&h->nbr, npa * MAX_NEIGH))) return rc;
    if ((rc = dalloc(&h->nbr_count, npa))) return rc;
    if ((rc = dalloc(&h->nbr_xy, npa * 2))) return rc;
  }
  CK(cudaMemsetAsync(h->ps, 0, sizeof(double) * npa * PS, h->stream));
  CK(cudaMemsetAsync(h->facc, 0, sizeof(unsigned long long) * npa * 6, h->stream));
  CK(cudaMemsetAsync(h->nbr_count, 0, sizeof(int) * npa, h->stream));
  CK(cudaMemsetAsync(h->nbr_xy, 0, sizeof(double) * npa * 2, h->stream));
  CK(cudaMemsetAsync(h->tile_count, 0, sizeof(int) * 2 * h->g.ltx * h->g.lty, h->stream));
  h->series_np = series_np;
  h->series_len = series_len;
  h->series_cap = series_cap;
  if (h->p.series_every > 0) {
    if (!keep_s) {
      if ((rc = dalloc(&h->series, (size_t)h->series_cap * h->series_len))) return rc;
      if ((rc = dalloc(&h->mass_acc, (size_t)h->series_cap))) return rc;
      h->series_pcap = 2 * h->series_cap;
      if (cudaHostAlloc(reinterpret_cast<void**>(&h->series_pin),
                        sizeof(double) * h->series_pcap * h->series_len, cudaHostAllocDefault) !=
              cudaSuccess ||
          cudaHostAlloc(reinterpret_cast<void**>(&h->mass_pin),
                        sizeof(unsigned long long) * h->series_pcap, cudaHostAllocDefault) !=
              cudaSuccess)
        return LBM_E_NOMEM;
    }
    CK(cudaMemsetAsync(h->mass_acc, 0, sizeof(unsigned long long) * h->series_cap, h->stream));
  }
  return LBM_OK;
}

void particle_record(const lbm_params& p, double* P, double x, double y, double ang, double u,
                     double v, double w, double diam, double rho_p) {
  std::memset(P, 0, sizeof(double) * PS);
  P[P_X] = x;
  P[P_Y] = y;
  P[P_ANG] = ang;
  P[P_U] = u;
  P[P_V] = v;
  P[P_W] = w;
  P[P_D] = diam;
  P[P_RHO] = rho_p;
  // M_P and I_P as C1:178-179
  P[P_M] = rho_p * p.pi * (0.5 * diam) * (0.5 * diam);
  P[P_I] = 0.5 * P[P_M] * (0.5 * diam) * (0.5 * diam);
}

int launch_tiles(lbm_sim* h) {
  ParticleArgs pa = particle_args(h);
  CK(cudaMemsetAsync(h->tile_count, 0, sizeof(int) * 2 * h->g.ltx * h->g.lty, h->stream));
  CK(cudaMemsetAsync(h->work_ctr, 0, 2 * sizeof(int), h->stream));
  CK(launch_tiles_only(pa, h->stream));
  CK(launch_tile_order(pa, 0, h->stream));
  CK(launch_tile_order(pa, 1, h->stream));
  return LBM_OK;
}

// Particle records with FORCE of the last lattice step: while the
// accumulators hold it (the next particle kernel decodes them on the
// device), decode them here the same way.
int read_particles(lbm_sim* h, std::vector<double>& buf) {
  const size_t npad = (size_t)h->npad;
  std::vector<double> soa(npad * PS);
  CK(d2h(h, soa.data(), h->ps, soa.size() * sizeof(double)));
  buf.assign((size_t)std::max(h->np, 1) * PS, 0.0);
  for (int i = 0; i < h->np; ++i)
    for (int f = 0; f < PS; ++f) buf[(size_t)i * PS + f] = soa[(size_t)f * npad + i];
  if (h->partials_valid && h->np > 0) {
    std::vector<unsigned long long> acc(npad * 6);
    CK(d2h(h, acc.data(), h->facc, acc.size() * sizeof(unsigned long long)));
    for (int i = 0; i < h->np; ++i) {
      double* P = &buf[(size_t)i * PS];
      P[P_FX] = decode_force(acc[i], acc[npad + i]);
      P[P_FY] = decode_force(acc[2 * npad + i], acc[3 * npad + i]);
      P[P_TZ] = decode_force(acc[4 * npad + i], acc[5 * npad + i]);
    }
  }
  return LBM_OK;
}

// Upload np AoS records (PS doubles each) into the SoA device layout,
// through the handle's pinned staging buffer (a direct DMA copy).  Both
// callers (lbm_set_particles, lbm_set_state) synchronise the stream before
// the call and after it, so no copy from the buffer is in flight when it is
// refilled.
int write_particles(lbm_sim* h, const std::vector<double>& buf) {
  const size_t npad = (size_t)h->npad;
  const size_t n = npad * PS;
  if (h->ps_pin_n < n) {
    if (h->ps_pin) cudaFreeHost(h->ps_pin);
    h->ps_pin = nullptr;
    h->ps_pin_n = 0;
    if (cudaHostAlloc(reinterpret_cast<void**>(&h->ps_pin), n * sizeof(double),
                      cudaHostAllocDefault) != cudaSuccess)
      return LBM_E_NOMEM;
    h->ps_pin_n = n;
  }
  double* soa = h->ps_pin;
  std::fill(soa, soa + n, 0.0);
  for (int i = 0; i < h->np; ++i)
    for (int f = 0; f < PS; ++f) soa[(size_t)f * npad + i] = buf[(size_t)i * PS + f];
  CK(h2d(h, h->ps, soa, n * sizeof(double)));
  return LBM_OK;
}

// Whether two input disks overlap (centre distance below the sum of the
// radii), on the host in O(np + cells): a linked-cell grid over the lattice
// whose cells are at least the largest diameter wide (so two overlapping
// disks lie in the same or in adjacent cells) and few enough (about np) that
// clearing it costs no more than the disks.  Centres lie in [0, nx] x [0, ny]
// (checked by the caller).
bool disks_overlap(const double* pin, int np, double dmax, int nx, int ny) {
  if (np < 2 || !(dmax > 0.0)) return false;
  const double cs = std::max(dmax, std::sqrt((nx + 1.0) * (ny + 1.0) / np));
  const int ncx = (int)std::floor(nx / cs) + 1, ncy = (int)std::floor(ny / cs) + 1;
  std::vector<int> head((size_t)ncx * ncy, -1), next((size_t)np), cell((size_t)np);
  for (int i = 0; i < np; ++i) {
    const double* r = pin + (size_t)LBM_PIN * i;
    const int cx = std::min(ncx - 1, (int)(r[0] / cs)), cy = std::min(ncy - 1, (int)(r[1] / cs));
    cell[(size_t)i] = cy * ncx + cx;
    next[(size_t)i] = head[(size_t)cell[(size_t)i]];
    head[(size_t)cell[(size_t)i]] = i;
  }
  for (int i = 0; i < np; ++i) {
    const double* a = pin + (size_t)LBM_PIN * i;
    const int cx = cell[(size_t)i] % ncx, cy = cell[(size_t)i] / ncx;
    for (int y = std::max(0, cy - 1); y <= std::min(ncy - 1, cy + 1); ++y)
      for (int x = std::max(0, cx - 1); x <= std::min(ncx - 1, cx + 1); ++x)
        for (int j = head[(size_t)y * ncx + x]; j >= 0; j = next[(size_t)j]) {
          if (j <= i) continue;
          const double* b = pin + (size_t)LBM_PIN * j;
          const double ex = a[0] - b[0], ey = a[1] - b[1], rs = 0.5 * (a[6] + b[6]);
          if (ex * ex + ey * ey < rs * rs) return true;
        }
  }
  return false;
}

template <class T>
void to_pitched(const double* src_dense, std::vector<unsigned char>& buf, const lbm_sim* h,
                int planes, bool aos9, bool shift) {
  const int n1x = h->p.nx + 1, n1y = h->p.ny + 1;
  buf.assign((size_t)planes * h->g.plane * sizeof(T), 0);
  T* d = reinterpret_cast<T*>(buf.data());
  static const double w[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                              1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
  for (int k = 0; k < planes; ++k)
    for (int j = 0; j < n1y; ++j)
      for (int i = 0; i < n1x; ++i) {
        const size_t o = (size_t)j * n1x + i;
        double v = aos9 ? src_dense[o * 9 + k] : src_dense[(size_t)k * n1x * n1y + o];
        if (shift) v -= w[k] * h->p.rho0;
        const int pl = planes == 9 ? plane_of(k) : k;  // population planes (plane_of)
        d[(size_t)pl * h->g.plane + (size_t)j * h->g.pitch + i] = (T)v;
      }
}

template <class T>
void from_pitched(const std::vector<unsigned char>& buf, double* dst, const lbm_sim* h) {
  const int n1x = h->p.nx + 1, n1y = h->p.ny + 1;
  const T* s = reinterpret_cast<const T*>(buf.data());
  for (int j = 0; j < n1y; ++j)
    for (int i = 0; i < n1x; ++i) dst[(size_t)j * n1x + i] = (double)s[(size_t)j * h->g.pitch + i];
}

int profile_flush(lbm_sim* h) {
  if (h->ev_used == 0) return LBM_OK;
  CK(cudaStreamSynchronize(h->stream));
  for (size_t b = 0; b + 2 < h->ev_used; b += 3) {
    float t0 = 0.f, t1 = 0.f;
    CK(cudaEventElapsedTime(&t0, h->ev[b], h->ev[b + 1]));
    CK(cudaEventElapsedTime(&t1, h->ev[b + 1], h->ev[b + 2]));
    h->prof_ms[0] += t0;
    h->prof_ms[1] += t1;
    h->prof_n[0] += 1;
    h->prof_n[1] += 1;
  }
  h->ev_used = 0;
  return LBM_OK;
}

cudaError_t record_event(lbm_sim* h) {
  if (h->ev_used == h->ev.size()) {
    cudaEvent_t e;
    cudaError_t err = cudaEventCreate(&e);
    if (err != cudaSuccess) return err;
    h->ev.push_back(e);
  }
  return cudaEventRecord(h->ev[h->ev_used++], h->stream);
}

// Tensor maps over the population buffers, 3-D (x = pitch, y = NY+1,
// z = 9 planes), box = one step-kernel tile of the three planes that share a
// row shift (plane_of).  The encoder comes
// from the driver through the runtime, so no link against libcuda is needed.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// TMA descriptor of the step kernel's reads from the population buffer at base;
// tw x rows nodes per tile (default: the single-run step kernel's tile).
int encode_f_map(const lbm_sim* h, void* base, CUtensorMap* out, int tw = 0, int rows = 0) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      fn == nullptr || q != cudaDriverEntryPointSuccess)
    return LBM_E_CUDA;
  EncodeTiledFn enc = reinterpret_cast<EncodeTiledFn>(fn);
  const cuuint64_t dims[3] = {(cuuint64_t)h->g.pitch, (cuuint64_t)(h->p.ny + 1), 9};
  const cuuint64_t strides[2] = {(cuuint64_t)h->g.pitch * h->esz,
                                 (cuuint64_t)h->g.plane * h->esz};
  if (tw <= 0) tw = step_tile_width((int)h->esz);
  if (rows <= 0) rows = step_box_rows((int)h->esz);
  const cuuint32_t box[3] = {(cuuint32_t)(tw + 2 * (16 / (int)h->esz)), (cuuint32_t)rows, 3};
  const cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(out, h->esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                   3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LBM_OK : LBM_E_CUDA;
}

// TMA descriptor of the step kernel's reads of the node omega at base (one
// plane): 2-D, box = one tile (TW nodes x TR rows), no halo.
int encode_om_map(const lbm_sim* h, void* base, CUtensorMap* out, int tw = 0, int rows = 0) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      fn == nullptr || q != cudaDriverEntryPointSuccess)
    return LBM_E_CUDA;
  EncodeTiledFn enc = reinterpret_cast<EncodeTiledFn>(fn);
  const cuuint64_t dims[2] = {(cuuint64_t)h->g.pitch, (cuuint64_t)(h->p.ny + 1)};
  const cuuint64_t strides[1] = {(cuuint64_t)h->g.pitch * h->esz};
  if (tw <= 0) tw = step_tile_width((int)h->esz);
  if (rows <= 0) rows = step_box_rows((int)h->esz);
  const cuuint32_t box[2] = {(cuuint32_t)tw, (cuuint32_t)rows};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = enc(out, h->esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                   2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LBM_OK : LBM_E_CUDA;
}

int make_tensor_maps(lbm_sim* h) {
  for (int b = 0; b < 2; ++b) {
    int rc = encode_f_map(h, h->f[b], &h->tm[b]);
    if (rc) return rc;
    h->tmo[b] = h->tm[b];
    if (h->om[b] && (rc = encode_om_map(h, h->om[b], &h->tmo[b]))) return rc;
  }
  return LBM_OK;
}

void destroy_buffers(lbm_sim* h) {
  // history copies still in flight on the copy stream read the device ring
  // and write the pinned staging ring: let them finish before anything goes
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  if (h->adj_rs) cudaStreamSynchronize(h->adj_rs);
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  h->ev.clear();
  for (int b = 0; b < 2; ++b) {
    dfree(h->f[b]);
    dfree(h->om[b]);
    dfree(h->pm[b]);
  }
  dfree(h->rec);
  dfree(h->ring);
  dfree(h->ps); dfree(h->facc); dfree(h->nbr); dfree(h->nbr_count); dfree(h->nbr_xy);
  dfree(h->tile_count); dfree(h->tile_list); dfree(h->tile_cur); dfree(h->pair_rebuild);
  dfree(h->tile_order); dfree(h->n_unlisted); dfree(h->work_ctr);
  dfree(h->rec_slot);
  dfree(h->mass_acc);
  dfree(h->d_kk); dfree(h->stale_dpw);
  dfree(h->series); dfree(h->out); dfree(h->out_f); dfree(h->d_status);
  dfree(h->u0); dfree(h->err_part);
  if (h->series_pin) cudaFreeHost(h->series_pin);
  if (h->mass_pin) cudaFreeHost(h->mass_pin);
  if (h->ps_pin) cudaFreeHost(h->ps_pin);
  for (const auto& b : h->series_pending) cudaEventDestroy(b.ev);
  for (cudaEvent_t e : h->series_ev_free) cudaEventDestroy(e);
  dfree(h->adj_slots); dfree(h->adj_ck); dfree(h->adj_ckp); dfree(h->adj_hist);
  for (int b = 0; b < 2; ++b) {
    dfree(h->adj_a[b]);
    dfree(h->adj_w[b]);
  }
  dfree(h->adj_state); dfree(h->adj_p); dfree(h->adj_h); dfree(h->adj_rho); dfree(h->adj_g);
  for (cudaEvent_t e : h->adj_ev)
    if (e) cudaEventDestroy(e);
  if (h->adj_rs) cudaStreamDestroy(h->adj_rs);
  if (h->h_status) cudaFreeHost(h->h_status);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->copy_fork) cudaEventDestroy(h->copy_fork);
  if (h->stream) cudaStreamDestroy(h->stream);
}

constexpr int ERR_BLOCKS = 592, ERR_TPB = 256;

// Per block: sum of |u - u0|^2 and |u|^2 over a fixed strided set of nodes
// reduced by a fixed tree (deterministic), and u0 = u.
__global__ void __launch_bounds__(ERR_TPB) k_error(const double* ux, const double* uy,
                                                   double* u0, double* v0, long long nn,
                                                   double* part) {
  __shared__ double s1[ERR_TPB], s2[ERR_TPB];
  double e1 = 0.0, e2 = 0.0;
  for (long long n = blockIdx.x * (long long)ERR_TPB + threadIdx.x; n < nn;
       n += (long long)gridDim.x * ERR_TPB) {
    const double x = ux[n], y = uy[n], dx = x - u0[n], dy = y - v0[n];
    e1 += dx * dx + dy * dy;
    e2 += x * x + y * y;
    u0[n] = x;
    v0[n] = y;
  }
  s1[threadIdx.x] = e1;
  s2[threadIdx.x] = e2;
  __syncthreads();
  for (int w = ERR_TPB / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1[0];
    part[2 * blockIdx.x + 1] = s2[0];
  }
}

// One time step on the handle's stream: particle kernel, then the step
// kernel (the body of lbm_step's loop).
int enqueue_step(lbm_sim* h) {
  const int every = h->p.series_every;
  if (h->series && every > 0 && (h->kk + 1) / every - h->copied_kk / every > h->series_cap) {
    int rc = series_enqueue(h);  // the ring slots are copied before reuse
    if (rc) return rc;
  }
  if (h->series && every > 0 && (h->kk + 1) % every == 0) {
    int rc = ring_wait(h, (h->kk + 1) / every - 1);
    if (rc) return rc;
  }
  if (h->prof) {
    if (h->ev_used + 3 > 3 * 65536) {
      int rc = profile_flush(h);
      if (rc) return rc;
    }
    CK(record_event(h));
  }
  ParticleArgs pa = particle_args(h);
  CK(launch_particles(pa, h->stream));
  if (h->prof) CK(record_event(h));
  h->kk += 1;
  LatticeArgs a = lattice_args(h);
  CK(launch_lattice(h, a, 0));
  if (h->prof) CK(record_event(h));
  h->cur ^= 1;
  h->prev_post_bc = false;
  h->partials_valid = true;
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_compute_error(lbm_sim* h, double* er) {
  if (!h || !er) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const long long nn = nodes(h);
  if (!h->u0) {
    int rc = dalloc(&h->u0, (size_t)2 * nn);
    if (!rc) rc = dalloc(&h->err_part, (size_t)2 * ERR_BLOCKS);
    if (rc) return rc;
    // the previous velocity starts as INITIALIZE's, zero (C1:154-155)
    CK(cudaMemsetAsync(h->u0, 0, sizeof(double) * 2 * nn, h->stream));
  }
  int rc = compute_output(h, false);  // corrected velocity of step kk in out[0], out[1]
  if (rc) return rc;
  k_error<<<ERR_BLOCKS, ERR_TPB, 0, h->stream>>>(h->out, h->out + nn, h->u0, h->u0 + nn, nn,
                                                 h->err_part);
  CK(cudaGetLastError());
  std::vector<double> part((size_t)2 * ERR_BLOCKS);
  CK(d2h(h, part.data(), h->err_part, part.size() * sizeof(double)));
  double e1 = 0.0, e2 = 0.0;
  for (int b = 0; b < ERR_BLOCKS; ++b) {
    e1 += part[2 * (size_t)b];
    e2 += part[2 * (size_t)b + 1];
  }
  *er = std::sqrt(e1 / e2);
  return refreshed_status(h);
}

static_assert(lbm::BC_EQUILIBRIUM == LBM_BC_EQUILIBRIUM, "kernel switch values");
static_assert(lbm::MOTION_OSCILLATE == LBM_MOTION_OSCILLATE, "kernel switch values");

int lbm_params_init(lbm_params* p) {
  if (!p) return LBM_E_INVALID;
  std::memset(p, 0, sizeof(*p));
  p->struct_size = (int32_t)sizeof(lbm_params);
  // C1 PARAMETERs as the Fortran holds them (REAL(4) literals widened)
  const float f1_36 = 1.0f / 36.0f, f1_6 = 1.0f / 6.0f;
  p->nx = 240;
  p->ny = 720;
  p->precision = LBM_FP64;
  p->bc = LBM_BC_ZOUHE;
  p->rheology = LBM_NEWTONIAN;
  p->rate_set = LBM_RATES_FIXED_Q;
  p->wall_model = LBM_WALL_MIRROR;
  p->contact_test = LBM_CONTACT_STALE_DPW;
  p->integrate_angle = 0;
  p->series_every = 1;
  p->series_particles = 1;
  p->series_capacity = 4096;
  p->record_stress = 0;
  p->device = 0;
  p->nu = (double)0.05f;
  p->rho0 = 1.0;
  p->s_e = (double)1.1f;
  p->s_eps = 1.0;
  p->s_q = (double)1.2f;
  p->d_mrt = (double)f1_36;
  p->inv_six = (double)f1_6;
  p->w_init[0] = (double)(2.0f / 9.0f);
  p->w_init[1] = (double)(1.0f / 18.0f);
  p->w_init[2] = (double)(1.0f / 36.0f);
  p->pi = (double)3.14159265359f;
  p->zeta = 1.0;
  const double c_l = (double)0.25f / 30.0;
  const double c_t = (c_l * c_l) * p->nu / (double)0.1f;
  const double c_g = c_l * (double)0.01f / (c_t * c_t);
  p->gravity = -(double)9.81f / c_g;
  p->tau_y = 1.0 * p->nu * 1.0 / 30.0;
  p->m_pap = (double)1.0e8f;
  p->gamma_min = (double)1.0e-15f;
  p->rep_zeta = 2.0;
  p->eps_p = 1.0e5;
  p->eps_w = 0.5 * p->eps_p;
  p->e_p = 2.0e5;
  p->e_w = 0.5 * p->e_p;
  const double D = 30.0;
  p->c_ij = -((((((double)1.25f - 1.0) * p->gravity) * p->pi) * 0.5) * D * 0.5) * D;
  const double edge3 = 0.5 * (double)p->ny + 0.5 * (2.0 * (double)p->ny);
  const double edge4 = 0.5 * (double)p->nx - 0.5 * (2.0 * (double)p->nx);
  p->wall_mirror_top = 2.0 * edge3;
  p->wall_mirror_left = 2.0 * edge4;
  return LBM_OK;
}

int lbm_create(const lbm_params* pin, lbm_sim** out) {
  if (!pin || !out) return LBM_E_INVALID;
  *out = nullptr;
  if (pin->struct_size != (int32_t)sizeof(lbm_params)) return LBM_E_ABI;
  const lbm_params& p = *pin;
  if (p.nx < 2 || p.ny < 2 || (long long)(p.nx + 1) * (p.ny + 1) > (1LL << 31)) return LBM_E_INVALID;
  if (p.precision != LBM_FP64 && p.precision != LBM_FP32_SHIFTED) return LBM_E_INVALID;
  if (p.bc != LBM_BC_ZOUHE && p.bc != LBM_BC_HALFWAY_BB && p.bc != LBM_BC_EQUILIBRIUM)
    return LBM_E_INVALID;
  if (p.motion != LBM_MOTION_FREE && p.motion != LBM_MOTION_OSCILLATE) return LBM_E_INVALID;
  if (p.strain_model != LBM_STRAIN_MEQ && p.strain_model != LBM_STRAIN_FEQ) return LBM_E_INVALID;
  if (p.collision != LBM_COLLISION_MRT && p.collision != LBM_COLLISION_BGK) return LBM_E_INVALID;
  if (p.collision == LBM_COLLISION_BGK && p.rheology == LBM_CASSON) return LBM_E_INVALID;
  if (p.motion == LBM_MOTION_OSCILLATE && (!std::isfinite(p.osc_u) || !(p.osc_period > 0.0)))
    return LBM_E_INVALID;
  if (p.rheology != LBM_NEWTONIAN && p.rheology != LBM_BINGHAM && p.rheology != LBM_CASSON)
    return LBM_E_INVALID;
  if (p.wall_model < 0 || p.wall_model > 2 || p.contact_test < 0 || p.contact_test > 1)
    return LBM_E_INVALID;
  if (!std::isfinite(p.nu) || !(p.rho0 > 0.0) || !(p.zeta > 0.0) || !(p.rep_zeta > 0.0) ||
      !(p.d_mrt > 0.0))
    return LBM_E_INVALID;
  const double omega = 1.0 / (3. * p.nu + 0.5);
  if (!(1.0 / omega >= 0.5)) return LBM_E_TAU;  // C1:127-130: IF(1.0/OMEGA < 0.5) STOP
  if (p.series_every < 0 || p.series_capacity < 0 || p.series_particles < 0) return LBM_E_INVALID;

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LBM_E_CUDA;
  if (p.device < 0 || p.device >= ndev) return LBM_E_INVALID;
  if (cudaSetDevice(p.device) != cudaSuccess) return LBM_E_CUDA;

  lbm_sim* h = new (std::nothrow) lbm_sim();
  if (!h) return LBM_E_NOMEM;
  h->p = p;
  h->prec = p.precision;
  h->esz = h->prec == LBM_FP64 ? 8 : 4;
  h->g.nx = p.nx;
  h->g.ny = p.ny;
  h->g.pitch = ((p.nx + 1) + 31) / 32 * 32;
  h->g.plane = (long long)h->g.pitch * (p.ny + 1);
  h->g.nbx = (p.nx + 1 + TX - 1) / TX;
  h->g.nby = (p.ny + 1 + TY - 1) / TY;
  h->g.ltx = (p.nx + 1 + LTX - 1) / LTX;
  h->g.lty = (p.ny + 1 + LTY - 1) / LTY;
  Model& m = h->m;
  m.bc = p.bc;
  m.bingham = p.rheology == LBM_BINGHAM || p.rheology == LBM_CASSON;
  m.casson = p.rheology == LBM_CASSON;
  m.strain_feq = p.strain_model == LBM_STRAIN_FEQ;
  m.q_of_omega = p.rate_set == LBM_RATES_Q_OF_OMEGA;
  m.record_stress = p.record_stress ? 1 : 0;
  m.rho0 = p.rho0;
  m.nu = p.nu;
  m.omega = omega;
  m.s_e = p.s_e;
  m.s_eps = p.s_eps;
  m.s_q = p.s_q;
  m.d_mrt = p.d_mrt;
  m.pi = p.pi;
  m.zeta = p.zeta;
  m.tau_y = p.tau_y;
  m.m_pap = p.m_pap;
  m.gamma_min = p.gamma_min;
  for (int k = 0; k < 3; ++k) m.w_init[k] = p.w_init[k];
  // rates at the uniform omega, ComputeRelaxation_MRT (C1:1029-1048, C6:1002-1021)
  const double oq = m.q_of_omega ? 8. * (2. - omega) / (8. - omega) : p.s_q;
  const double S_uni[9] = {0.0, p.s_e, p.s_eps, 0.0, oq, 0.0, oq, omega, omega};
  for (int k = 0; k < 9; ++k) m.S_uni[k] = S_uni[k];
  static const double w[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                              1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
  for (int k = 0; k < 9; ++k) m.shift_f[k] = (float)(p.rho0 * w[k] * (36.0 * p.d_mrt - 1.0));
  m.rho0_f = (float)p.rho0;
  m.nu_f = (float)p.nu;
  m.d_mrt_f = (float)p.d_mrt;
  m.pi_f = (float)p.pi;
  m.zeta_f = (float)p.zeta;
  m.tau_y_f = (float)p.tau_y;
  m.m_pap_f = (float)p.m_pap;
  m.gamma_min_f = (float)p.gamma_min;
  m.s_e_f = (float)p.s_e;
  m.s_eps_f = (float)p.s_eps;
  m.sq_uni_f = (float)oq;
  m.omega_f = (float)omega;
  for (int k = 0; k < 3; ++k) m.w_init_f[k] = (float)p.w_init[k];
  for (int k = 0; k < 9; ++k) {  // rho0*(W_k*B_k(u=0) - w_k), B(0) = 2 (k<5) or 1
    const double W = p.w_init[k == 0 ? 0 : (k < 5 ? 1 : 2)];
    m.eq_c_f[k] = (float)(p.rho0 * (W * (k < 5 ? 2.0 : 1.0) - w[k]));
  }
  // COLLISION (C1:774-841): MU_R = 1000.0*MU_0, GAMMA_C = TAU_Y/(MU_R-MU_0)
  // (C1:49-53, MU_0 = NU); the forcing weights of ComputeSourceEquilib_Hydro
  // are REAL(4) quotients (C1:847)
  m.bgk = p.collision == LBM_COLLISION_BGK;
  m.mu_r = 1000.0 * p.nu;
  m.gamma_c = p.tau_y / (m.mu_r - p.nu);
  m.w_src[0] = (double)(4.0f / 9.0f);
  m.w_src[1] = (double)(1.0f / 9.0f);
  m.w_src[2] = (double)(1.0f / 36.0f);
  m.mu_r_f = (float)m.mu_r;
  m.gamma_c_f = (float)m.gamma_c;
  for (int k = 0; k < 3; ++k) m.w_src_f[k] = (float)m.w_src[k];

  int rc = LBM_OK;
  auto fail = [&](int code) {
    destroy_buffers(h);
    delete h;
    return code;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->copy_fork, cudaEventDisableTiming) != cudaSuccess)
    return fail(LBM_E_CUDA);
  if (cudaHostAlloc(reinterpret_cast<void**>(&h->h_status), sizeof(int), cudaHostAllocDefault) !=
      cudaSuccess)
    return fail(LBM_E_NOMEM);
  *h->h_status = 0;
  if ((rc = dalloc(&h->d_status, 1))) return fail(rc);
  cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream);
  const size_t fbytes = (size_t)9 * h->g.plane * h->esz;
  for (int b = 0; b < 2; ++b) {
    if (cudaMalloc(&h->f[b], fbytes) != cudaSuccess) return fail(LBM_E_NOMEM);
    if (m.bingham && cudaMalloc(&h->om[b], (size_t)h->g.plane * h->esz) != cudaSuccess)
      return fail(LBM_E_NOMEM);
    if (m.bgk && m.bingham && cudaMalloc(&h->pm[b], (size_t)3 * h->g.plane * h->esz) != cudaSuccess)
      return fail(LBM_E_NOMEM);
  }
  if (m.record_stress &&
      cudaMalloc(&h->rec, (size_t)2 * 4 * h->g.plane * h->esz) != cudaSuccess)
    return fail(LBM_E_NOMEM);
  if (p.bc == LBM_BC_EQUILIBRIUM) {
    h->ring_n = 2 * (p.nx + 1) + 2 * (p.ny + 1);
    const size_t rb = (size_t)2 * 3 * h->ring_n * h->esz;
    if (cudaMalloc(&h->ring, rb) != cudaSuccess) return fail(LBM_E_NOMEM);
    cudaMemsetAsync(h->ring, 0, rb, h->stream);
  }
  if ((rc = make_tensor_maps(h))) return fail(rc);
  const int ntiles = h->g.ltx * h->g.lty;
  if ((rc = dalloc(&h->tile_count, (size_t)2 * ntiles))) return fail(rc);
  if ((rc = dalloc(&h->tile_list, (size_t)2 * ntiles * h->tile_cap))) return fail(rc);
  if ((rc = dalloc(&h->tile_cur, 2))) return fail(rc);
  if ((rc = dalloc(&h->tile_order, (size_t)4 * ntiles))) return fail(rc);
  if ((rc = dalloc(&h->n_unlisted, 2))) return fail(rc);
  if ((rc = dalloc(&h->work_ctr, 2))) return fail(rc);
  cudaMemsetAsync(h->work_ctr, 0, 2 * sizeof(int), h->stream);
  if ((rc = dalloc(&h->pair_rebuild, 1))) return fail(rc);
  if ((rc = dalloc(&h->rec_slot, 1))) return fail(rc);
  cudaMemsetAsync(h->rec_slot, 0xff, sizeof(int), h->stream);
  cudaMemsetAsync(h->tile_cur, 0, 2 * sizeof(int), h->stream);
  cudaMemsetAsync(h->pair_rebuild, 0, sizeof(int), h->stream);
  if ((rc = dalloc(&h->d_kk, 1))) return fail(rc);
  if ((rc = dalloc(&h->stale_dpw, 1))) return fail(rc);
  if ((rc = dalloc(&h->out, (size_t)NOUT * nodes(h)))) return fail(rc);
  cudaMemsetAsync(h->f[0], 0, fbytes, h->stream);
  cudaMemsetAsync(h->f[1], 0, fbytes, h->stream);
  cudaMemsetAsync(h->tile_count, 0, sizeof(int) * 2 * ntiles, h->stream);
  cudaMemsetAsync(h->d_kk, 0, sizeof(long long), h->stream);
  const double inf = INFINITY;
  cudaMemcpyAsync(h->stale_dpw, &inf, sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if ((rc = setup_particle_buffers(h, 0, 0.0))) return fail(rc);
  {  // empty lists: the tile queue order of both buffers
    ParticleArgs pa = particle_args(h);
    if (launch_tile_order(pa, 0, h->stream) != cudaSuccess ||
        launch_tile_order(pa, 1, h->stream) != cudaSuccess)
      return fail(LBM_E_CUDA);
  }
  // f*(1) = collision of step 1 applied to INITIALIZE's state (C1:151, C1:296)
  h->cur = 0;
  LatticeArgs a = lattice_args(h);
  a.src = nullptr;
  a.dst = h->f[0];
  a.om_dst = h->om[0];
  a.pm_dst = h->pm[0];
  if (launch_lattice(h, a, 2) != cudaSuccess) return fail(LBM_E_CUDA);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(LBM_E_CUDA);
  *out = h;
  return LBM_OK;
}

int lbm_destroy(lbm_sim* h) {
  if (!h) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  destroy_buffers(h);
  delete h;
  return LBM_OK;
}

int lbm_set_particles(lbm_sim* h, int32_t np, const double* pin) {
  if (!h || np < 0 || np > MAX_PARTICLES || (np > 0 && !pin)) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  double dmax = 0.0;
  for (int i = 0; i < np; ++i) {
    const double* r = pin + (size_t)LBM_PIN * i;
    for (int k = 0; k < LBM_PIN; ++k)
      if (!std::isfinite(r[k])) return LBM_E_INVALID;
    if (!(r[6] > 0.0) || !(r[7] > 0.0)) return LBM_E_INVALID;
    if (r[0] < 0.0 || r[0] > h->p.nx || r[1] < 0.0 || r[1] > h->p.ny) return LBM_E_PARTICLE;
    dmax = std::max(dmax, r[6]);
  }
  // overlapping input disks (no reference input holds any; the repulsion
  // model's contact branch is for disks that come into contact while moving)
  if (disks_overlap(pin, np, dmax, h->p.nx, h->p.ny)) return LBM_E_PARTICLE;
  // kernels still in flight may read the particle buffers reused below
  CK(cudaStreamSynchronize(h->stream));
  int rc = setup_particle_buffers(h, np, dmax);
  if (rc) return rc;
  std::vector<double> buf((size_t)std::max(np, 1) * PS, 0.0);
  for (int i = 0; i < np; ++i) {
    const double* r = pin + (size_t)LBM_PIN * i;
    particle_record(h->p, &buf[(size_t)i * PS], r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]);
  }
  if ((rc = write_particles(h, buf))) return rc;
  if ((rc = launch_tiles(h))) return rc;
  h->out_kk = -1;
  series_reset(h, h->kk);
  return refreshed_status(h);
}

int lbm_step(lbm_sim* h, int32_t nsteps) {
  if (!h || nsteps < 0) return LBM_E_INVALID;
  int st = sticky_status(h);
  if (st) return st;
  cudaSetDevice(h->p.device);
  for (int32_t s = 0; s < nsteps; ++s) {
    int rc = enqueue_step(h);
    if (rc) return rc;
  }
  if (h->series) {
    int rc = series_enqueue(h);  // this call's records, copied behind its kernels
    if (rc) return rc;
  }
  h->out_kk = -1;
  CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  return LBM_OK;
}

int lbm_get_step(lbm_sim* h, int64_t* kk) {
  if (!h || !kk) return LBM_E_INVALID;
  *kk = h->kk;
  return LBM_OK;
}

int lbm_get_particles(lbm_sim* h, double* out) {
  if (!h || (!out && h->np > 0)) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  std::vector<double> buf;
  int rc = read_particles(h, buf);
  if (rc) return rc;
  for (int i = 0; i < h->np; ++i) {
    const double* P = &buf[(size_t)i * PS];
    double* r = out + (size_t)LBM_POUT * i;
    r[0] = P[P_X]; r[1] = P[P_Y]; r[2] = P[P_ANG];
    r[3] = P[P_U]; r[4] = P[P_V]; r[5] = P[P_W];
    r[6] = P[P_FX]; r[7] = P[P_FY]; r[8] = P[P_TZ];
    r[9] = P[P_FCX]; r[10] = P[P_FCY];
    r[11] = P[P_FHX]; r[12] = P[P_FHY]; r[13] = P[P_FHT];
    r[14] = P[P_M]; r[15] = P[P_I];
  }
  return refreshed_status(h);
}

int lbm_get_field(lbm_sim* h, int32_t which, double* out) {
  if (!h || !out) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const long long nn = nodes(h);
  const int n1x = h->p.nx + 1, n1y = h->p.ny + 1;
  if (which >= LBM_FIELD_UX && which <= LBM_FIELD_GY) {
    int rc = compute_output(h, false);
    if (rc) return rc;
    const int slot = which == LBM_FIELD_UX ? 0 : which == LBM_FIELD_UY ? 1 :
                     which == LBM_FIELD_RHO ? 2 : which == LBM_FIELD_PHI ? 3 :
                     which == LBM_FIELD_GX ? 4 : 5;
    CK(d2h(h, out, h->out + (size_t)slot * nn, nn * sizeof(double)));
    return refreshed_status(h);
  }
  if (which == LBM_FIELD_OMEGA) {
    if (!h->m.bingham || h->kk == 0) {
      for (long long i = 0; i < nn; ++i) out[i] = h->m.omega;
      return LBM_OK;
    }
    std::vector<unsigned char> buf((size_t)h->g.plane * h->esz);
    CK(d2h(h, buf.data(), h->om[h->cur ^ 1], buf.size()));
    if (h->prec == LBM_FP64) from_pitched<double>(buf, out, h); else from_pitched<float>(buf, out, h);
    return LBM_OK;
  }
  if (which >= LBM_FIELD_TAU11 && which <= LBM_FIELD_TAU12) {
    if (!h->rec) return LBM_E_STATE;
    if (h->kk == 0) {
      for (long long i = 0; i < nn; ++i) out[i] = 0.0;
      return LBM_OK;
    }
    const int slot = (int)(h->kk & 1);
    const int comp = which - LBM_FIELD_TAU11;
    std::vector<unsigned char> buf((size_t)h->g.plane * h->esz);
    const size_t off = ((size_t)slot * 4 + comp) * h->g.plane * h->esz;
    CK(d2h(h, buf.data(), static_cast<unsigned char*>(h->rec) + off, buf.size()));
    if (h->prec == LBM_FP64) from_pitched<double>(buf, out, h); else from_pitched<float>(buf, out, h);
    (void)n1x; (void)n1y;
    return LBM_OK;
  }
  return LBM_E_INVALID;
}

int lbm_get_image(lbm_sim* h, int32_t* out) {
  if (!h || !out) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const long long nn = nodes(h);
  int rc = compute_output(h, false);
  if (rc) return rc;
  std::vector<double> pn(nn), yd;
  CK(d2h(h, pn.data(), h->out + 6 * nn, nn * sizeof(double)));
  if (h->m.bingham && h->rec && h->kk > 0) {
    yd.resize(nn);
    std::vector<unsigned char> buf((size_t)h->g.plane * h->esz);
    const size_t off = ((size_t)(h->kk & 1) * 4 + 3) * h->g.plane * h->esz;
    CK(d2h(h, buf.data(), static_cast<unsigned char*>(h->rec) + off, buf.size()));
    if (h->prec == LBM_FP64) from_pitched<double>(buf, yd.data(), h);
    else from_pitched<float>(buf, yd.data(), h);
  }
  for (long long i = 0; i < nn; ++i)
    out[i] = pn[i] > 5.0 ? 10 : (yd.empty() ? 0 : (int32_t)yd[i]);
  return refreshed_status(h);
}

int lbm_series_record_len(lbm_sim* h, int32_t* len) {
  if (!h || !len) return LBM_E_INVALID;
  *len = h->series_len;
  return LBM_OK;
}

int lbm_get_series(lbm_sim* h, double* out, int32_t max_records, int32_t* nrec) {
  if (!h || !nrec || max_records < 0) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const size_t len = (size_t)h->series_len;
  // wait only for the oldest batches the request needs: steps queued after
  // them keep running while the caller reads these
  int rc = series_enqueue(h);
  if (rc) return rc;
  if (out && h->host_series_read == h->host_series.size() && h->p.series_every > 0) {
    // nothing held on the host: whole batches go straight from the pinned
    // staging ring to the caller
    const int every = h->p.series_every;
    const double nn = (double)nodes(h);
    size_t n = 0;
    while (!h->series_pending.empty()) {
      const lbm_sim::SeriesBatch b = h->series_pending.front();
      const long long r0 = h->drained_kk / every;
      if (n + (size_t)(b.r_end - r0) > (size_t)max_records) break;
      CK(cudaEventSynchronize(b.ev));
      h->series_pending.pop_front();
      h->series_ev_free.push_back(b.ev);
      for (long long r = r0; r < b.r_end; ++r, ++n) {
        const long long ps = r % h->series_pcap;
        double* dst = out + n * len;
        std::memcpy(dst, h->series_pin + ps * len, len * sizeof(double));
        dst[1] = h->p.rho0 + (double)(long long)h->mass_pin[ps] / MASS_FIX / nn;
      }
      h->drained_kk = b.r_end * every;
    }
    if (n > 0) {
      *nrec = (int32_t)n;
      return sticky_status(h);
    }
  }
  while ((h->host_series.size() - h->host_series_read) / len < (size_t)max_records &&
         !h->series_pending.empty())
    if ((rc = series_absorb_one(h))) return rc;
  const size_t avail = (h->host_series.size() - h->host_series_read) / len;
  const size_t n = std::min<size_t>(avail, (size_t)max_records);
  if (n && out)
    std::memcpy(out, h->host_series.data() + h->host_series_read, n * len * sizeof(double));
  h->host_series_read += n * len;
  if (h->host_series_read == h->host_series.size()) {
    h->host_series.clear();
    h->host_series_read = 0;
  }
  *nrec = (int32_t)n;
  return sticky_status(h);  // as of the last lbm_step; no wait for later steps
}

int lbm_get_mean_density(lbm_sim* h, double* avg) {
  if (!h || !avg) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const long long nn = nodes(h);
  int rc = compute_output(h, false);
  if (rc) return rc;
  std::vector<double> r(nn);
  CK(d2h(h, r.data(), h->out + 2 * nn, nn * sizeof(double)));
  double s = 0.0;
  for (long long i = 0; i < nn; ++i) s += r[i];
  *avg = s / (double)nn;
  return std::isfinite(*avg) ? LBM_OK : LBM_E_NAN;
}

int lbm_get_state(lbm_sim* h, double* f, double* omega, double* particles) {
  if (!h) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  const long long nn = nodes(h);
  if (f) {
    if (!h->out_f) {
      int rc = dalloc(&h->out_f, (size_t)9 * nn);
      if (rc) return rc;
    }
    h->out_kk = -1;
    int rc = compute_output(h, true);
    if (rc) return rc;
    CK(d2h(h, f, h->out_f, (size_t)9 * nn * sizeof(double)));
  }
  if (omega) {
    int rc = lbm_get_field(h, LBM_FIELD_OMEGA, omega);
    if (rc) return rc;
  }
  if (particles && h->np > 0) {
    std::vector<double> buf;
    int rc = read_particles(h, buf);
    if (rc) return rc;
    double stale = 0.0;
    CK(d2h(h, &stale, h->stale_dpw, sizeof(double)));
    for (int i = 0; i < h->np; ++i) {
      const double* P = &buf[(size_t)i * PS];
      double* r = particles + (size_t)LBM_STATE_PER * i;
      r[0] = P[P_X]; r[1] = P[P_Y]; r[2] = P[P_ANG];
      r[3] = P[P_U]; r[4] = P[P_V]; r[5] = P[P_W];
      r[6] = P[P_UO]; r[7] = P[P_VO]; r[8] = P[P_WO];
      r[9] = P[P_FX]; r[10] = P[P_FY]; r[11] = P[P_TZ];
      r[12] = P[P_FCX]; r[13] = P[P_FCY];
      r[14] = P[P_FHX]; r[15] = P[P_FHY]; r[16] = P[P_FHT];
      r[17] = P[P_D]; r[18] = P[P_RHO]; r[19] = stale;
    }
  }
  return refreshed_status(h);
}

int lbm_set_state(lbm_sim* h, int64_t kk, const double* f, const double* omega, int32_t np,
                  const double* particles) {
  if (!h || !f || kk < 0 || np < 0 || np > MAX_PARTICLES || (np > 0 && !particles))
    return LBM_E_INVALID;
  if (h->m.bingham && !omega) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  CK(cudaStreamSynchronize(h->stream));
  double dmax = 0.0;
  for (int i = 0; i < np; ++i) {
    const double* r = particles + (size_t)LBM_STATE_PER * i;
    if (!(r[17] > 0.0) || !(r[18] > 0.0)) return LBM_E_INVALID;
    dmax = std::max(dmax, r[17]);
  }
  int rc = setup_particle_buffers(h, np, dmax);
  if (rc) return rc;
  std::vector<double> buf((size_t)std::max(np, 1) * PS, 0.0);
  double stale = INFINITY;
  for (int i = 0; i < np; ++i) {
    const double* r = particles + (size_t)LBM_STATE_PER * i;
    double* P = &buf[(size_t)i * PS];
    particle_record(h->p, P, r[0], r[1], r[2], r[3], r[4], r[5], r[17], r[18]);
    P[P_UO] = r[6]; P[P_VO] = r[7]; P[P_WO] = r[8];
    P[P_FX] = r[9]; P[P_FY] = r[10]; P[P_TZ] = r[11];
    P[P_FCX] = r[12]; P[P_FCY] = r[13];
    P[P_FHX] = r[14]; P[P_FHY] = r[15]; P[P_FHT] = r[16];
    stale = r[19];
  }
  if ((rc = write_particles(h, buf))) return rc;
  CK(h2d(h, h->stale_dpw, &stale, sizeof(double)));
  const long long kkl = kk;
  CK(h2d(h, h->d_kk, &kkl, sizeof(long long)));
  // F after BC of step kk into the "previous" buffer
  std::vector<unsigned char> pb;
  const int prev = h->cur ^ 1;
  if (h->prec == LBM_FP64) to_pitched<double>(f, pb, h, 9, true, false);
  else to_pitched<float>(f, pb, h, 9, true, true);
  CK(h2d(h, h->f[prev], pb.data(), pb.size()));
  CK(cudaStreamSynchronize(h->stream));  // pb is reused below
  if (h->m.bingham) {
    if (h->prec == LBM_FP64) to_pitched<double>(omega, pb, h, 1, false, false);
    else to_pitched<float>(omega, pb, h, 1, false, false);
    CK(h2d(h, h->om[prev], pb.data(), pb.size()));
    CK(cudaStreamSynchronize(h->stream));
  }
  h->kk = kk;
  series_reset(h, kk);
  h->host_series.clear();
  h->host_series_read = 0;
  if ((rc = launch_tiles(h))) return rc;
  // collision of step kk+1 from the restored state
  LatticeArgs a = lattice_args(h);
  a.src = h->f[prev];
  a.om_src = h->om[prev];
  a.dst = h->f[h->cur];
  a.om_dst = h->om[h->cur];
  a.pm_dst = h->pm[h->cur];
  CK(launch_lattice(h, a, 3));
  CK(cudaStreamSynchronize(h->stream));
  h->prev_post_bc = true;
  h->out_kk = -1;
  return refreshed_status(h);
}

int lbm_get_stream(lbm_sim* h, void** stream) {
  if (!h || !stream) return LBM_E_INVALID;
  *stream = (void*)h->stream;
  return LBM_OK;
}

int lbm_profile(lbm_sim* h, int32_t enable) {
  if (!h) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  int rc = profile_flush(h);
  if (rc) return rc;
  h->prof = enable != 0;
  h->prof_ms[0] = h->prof_ms[1] = 0.0;
  h->prof_n[0] = h->prof_n[1] = 0;
  return LBM_OK;
}

int lbm_profile_read(lbm_sim* h, double* ms, int64_t* launches) {
  if (!h || !ms || !launches) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  int rc = profile_flush(h);
  if (rc) return rc;
  ms[0] = h->prof_ms[0];
  ms[1] = h->prof_ms[1];
  launches[0] = h->prof_n[0];
  launches[1] = h->prof_n[1];
  h->prof_ms[0] = h->prof_ms[1] = 0.0;
  h->prof_n[0] = h->prof_n[1] = 0;
  return LBM_OK;
}

int lbm_get_status(lbm_sim* h) {
  if (!h) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  CK(d2h(h, h->h_status, h->d_status, sizeof(int)));
  return sticky_status(h);
}

int lbm_selftest_wait(lbm_sim* h, int32_t limit) {
  if (!h || limit < 1 || limit > (1 << 20)) return LBM_E_INVALID;
  cudaSetDevice(h->p.device);
  CK(launch_wait_selftest(h->d_status, (uint32_t)limit, h->stream));
  CK(d2h(h, h->h_status, h->d_status, sizeof(int)));
  return LBM_OK;
}

int32_t lbm_checked_build(void) {
#ifdef LBM_CHECKED
  return 1;
#else
  return 0;
#endif
}

const char* lbm_strerror(int code) {
  switch (code) {
    case LBM_OK: return "ok";
    case LBM_E_INVALID: return "invalid argument or parameter";
    case LBM_E_TAU: return "relaxation time exceeded 0.5 -> stability problem";
    case LBM_E_NOMEM: return "out of memory";
    case LBM_E_CUDA: return "CUDA error (no device or launch failure)";
    case LBM_E_NAN: return "non-finite density or particle state";
    case LBM_E_TIMEOUT: return "bounded device wait expired";
    case LBM_E_OVERFLOW:
      return "fixed capacity exceeded (particles per lattice tile or neighbours per particle, "
             "or an FP32 density deviation of 2 or more)";
    case LBM_E_STATE: return "call out of order";
    case LBM_E_PARTICLE: return "particle outside the lattice";
    case LBM_E_ABI: return "lbm_params.struct_size mismatch";
    case LBM_E_SCRATCH: return "lattice or particle count exceeds the fixed no-alloc scratch";
    case LBM_E_BOUNDS: return "a kernel index check failed (checked build)";
    default: return "unknown error";
  }
}

}  // extern "C"

// ===========================================================================
// Adjoint sweep.  Forward: the time loop from step 0 to n1, keeping every
// step's particle records and, every L steps, a checkpoint of the state
// after that step (f*, omega, records, FORCE sums, D_PW).  Reverse, segment
// by segment from the last: restore the checkpoint into the first slot of
// the segment's slot set, recompute the segment forward with the step kernel
// writing each f*(n), omega(n) into its own slot, then run the level kernels
// from the segment's last level to its first, each followed by the particle
// kernel of the step before.  Two slot sets: the recompute of a segment runs
// on a second stream while the level kernels of the segment after it run on
// the handle's stream, so the two latency-bound kernel chains share the SMs.
namespace {

size_t adj_slot_bytes(const lbm_sim* h) { return (size_t)10 * h->g.plane * h->esz; }
size_t adj_ckp_len(const lbm_sim* h) { return (size_t)(PS + 6) * h->npad + 1; }

int adj_reserve(lbm_sim* h, int nslots, int nck, long long nhist) {
  int rc;
  const size_t sb = adj_slot_bytes(h);
  if (nslots > h->adj_nslots) {
    dfree(h->adj_slots);
    h->adj_nslots = 0;
    if ((rc = dalloc(&h->adj_slots, sb * nslots))) return rc;
    h->adj_tm.assign(nslots, CUtensorMap{});
    h->adj_tmo.assign(nslots, CUtensorMap{});
    const size_t pb = (size_t)h->g.plane * h->esz;
    for (int s = 0; s < nslots; ++s) {
      if ((rc = encode_f_map(h, h->adj_slots + sb * s, &h->adj_tm[s]))) return rc;
      h->adj_tmo[s] = h->adj_tm[s];
      if (h->m.bingham &&
          (rc = encode_om_map(h, h->adj_slots + sb * s + 9 * pb, &h->adj_tmo[s])))
        return rc;
    }
    h->adj_nslots = nslots;
  }
  if (nck > h->adj_nck || h->adj_npad != h->npad) {
    dfree(h->adj_ck);
    dfree(h->adj_ckp);
    h->adj_nck = 0;
    if (nck > 0 && (rc = dalloc(&h->adj_ck, sb * nck))) return rc;
    if ((rc = dalloc(&h->adj_ckp, adj_ckp_len(h) * (nck + 1)))) return rc;
    h->adj_nck = nck;
  }
  if (nhist > h->adj_nhist || h->adj_npad != h->npad) {
    dfree(h->adj_hist);
    h->adj_nhist = 0;
    if ((rc = dalloc(&h->adj_hist, (size_t)nhist * PS * h->npad))) return rc;
    h->adj_nhist = nhist;
  }
  if (!h->adj_a[0]) {
    for (int b = 0; b < 2; ++b) {
      if ((rc = dalloc(reinterpret_cast<unsigned char**>(&h->adj_a[b]), 9 * h->g.plane * h->esz)))
        return rc;
      if ((rc = dalloc(reinterpret_cast<unsigned char**>(&h->adj_w[b]), h->g.plane * h->esz)))
        return rc;
    }
    if ((rc = dalloc(&h->adj_g, (size_t)2 * h->g.nbx * h->g.nby))) return rc;
  }
  if (!h->adj_rs) {
    CK(cudaStreamCreateWithFlags(&h->adj_rs, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->adj_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (h->adj_npad != h->npad) {
    dfree(h->adj_state); dfree(h->adj_p); dfree(h->adj_h); dfree(h->adj_rho);
    const size_t np = (size_t)h->npad;
    if ((rc = dalloc(&h->adj_state, 8 * np)) || (rc = dalloc(&h->adj_p, 5 * np)) ||
        (rc = dalloc(&h->adj_h, 3 * np)) || (rc = dalloc(&h->adj_rho, np)))
      return rc;
    h->adj_npad = h->npad;
  }
  return LBM_OK;
}

// Small state (records, FORCE sums, D_PW) into / out of checkpoint entry c.
cudaError_t adj_save_small(lbm_sim* h, int c) {
  double* d = h->adj_ckp + adj_ckp_len(h) * c;
  const size_t np = (size_t)h->npad;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(d, h->ps, PS * np * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(d + PS * np, h->facc, 6 * np * sizeof(double),
                           cudaMemcpyDeviceToDevice, h->stream)) != cudaSuccess)
    return e;
  return cudaMemcpyAsync(d + (PS + 6) * np, h->stale_dpw, sizeof(double),
                         cudaMemcpyDeviceToDevice, h->stream);
}

int adj_load_small(lbm_sim* h, int c, long long kk, bool partials) {
  const double* d = h->adj_ckp + adj_ckp_len(h) * c;
  const size_t np = (size_t)h->npad;
  CK(cudaMemcpyAsync(h->ps, d, PS * np * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->facc, d + PS * np, 6 * np * sizeof(double), cudaMemcpyDeviceToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(h->stale_dpw, d + (PS + 6) * np, sizeof(double), cudaMemcpyDeviceToDevice,
                     h->stream));
  h->kk = kk;
  CK(launch_set_ll(h->d_kk, kk, h->stream));
  h->partials_valid = partials;
  return launch_tiles(h);
}

// f* and omega of the current state (f[cur], om[cur]) into a 10-plane block.
cudaError_t adj_save_fields(lbm_sim* h, unsigned char* dst) {
  const size_t pb = (size_t)h->g.plane * h->esz;
  cudaError_t e = cudaMemcpyAsync(dst, h->f[h->cur], 9 * pb, cudaMemcpyDeviceToDevice, h->stream);
  if (e != cudaSuccess || !h->m.bingham) return e;
  return cudaMemcpyAsync(dst + 9 * pb, h->om[h->cur], pb, cudaMemcpyDeviceToDevice, h->stream);
}

// One forward step reading slot s and writing slot s + 1.
int adj_step_slots(lbm_sim* h, int s) {
  const size_t sb = adj_slot_bytes(h), pb = (size_t)h->g.plane * h->esz;
  unsigned char* src = h->adj_slots + sb * s;
  unsigned char* dst = src + sb;
  ParticleArgs pa = particle_args(h);
  CK(launch_particles(pa, h->stream));
  h->kk += 1;
  LatticeArgs a = lattice_args(h);
  a.src = src;
  a.dst = dst;
  a.om_src = src + 9 * pb;
  a.om_dst = dst + 9 * pb;
  if (h->prec == LBM_FP64) CK(launch_step_fp64(a, &h->adj_tm[s], &h->adj_tmo[s], h->stream));
  else CK(launch_step_fp32(a, &h->adj_tm[s], &h->adj_tmo[s], h->stream));
  h->partials_valid = true;
  return LBM_OK;
}

AdjParticleArgs adj_particle_args(lbm_sim* h, const lbm_objective* obj, long long n) {
  AdjParticleArgs q{};
  const size_t rec = (size_t)PS * h->npad;
  q.prev = h->adj_hist + rec * (n - 1);
  q.cur = h->adj_hist + rec * n;
  q.a_state = h->adj_state;
  q.a_p = h->adj_p;
  q.a_h = h->adj_h;
  q.a_rho = h->adj_rho;
  q.np = h->np;
  q.npad = h->npad;
  q.n = n;
  q.n0 = obj->n0;
  q.n1 = obj->n1;
  q.obj_p = obj->particle;
  q.obj_c = obj->component;
  q.obj_w = 1.0 / (double)(obj->n1 - obj->n0 + 1);
  q.wall_model = h->p.wall_model;
  q.rep_zeta = h->p.rep_zeta;
  q.eps_p = h->p.eps_p;
  q.eps_w = h->p.eps_w;
  q.e_p = h->p.e_p;
  q.e_w = h->p.e_w;
  q.c_ij = h->p.c_ij;
  q.mirror_top = h->p.wall_mirror_top;
  q.mirror_left = h->p.wall_mirror_left;
  q.rho0 = h->p.rho0;
  q.gravity = h->p.gravity;
  q.nx = h->p.nx;
  q.ny = h->p.ny;
  return q;
}

cudaError_t adj_level(lbm_sim* h, long long n, const unsigned char* slot, const void* a_in,
                      const void* aw_in, void* a_out, void* aw_out, int pdl) {
  AdjLatticeArgs a{};
  a.g = h->g;
  a.m = h->m;
  const size_t pb = (size_t)h->g.plane * h->esz;
  a.fs = slot;
  a.oms = slot ? slot + 9 * pb : nullptr;
  a.a_in = a_in;
  a.aw_in = aw_in;
  a.a_out = a_out;
  a.aw_out = aw_out;
  a.ps = h->adj_hist + (size_t)PS * h->npad * n;
  a.a_h = h->adj_h;
  a.a_p = h->adj_p;
  a.gacc = h->adj_g;
  a.np = h->np;
  a.npad = h->npad;
  a.level0 = n == 0 ? 1 : 0;
  a.kappa = 36.0 * h->p.d_mrt;
  return h->prec == LBM_FP64 ? launch_adj_lattice_fp64(a, h->stream, pdl)
                             : launch_adj_lattice_fp32(a, h->stream, pdl);
}

}  // namespace

extern "C" int lbm_adjoint(lbm_sim* h, const lbm_objective* obj, double* value, double* grads) {
  if (!h || !obj || !grads || obj->struct_size != (int32_t)sizeof(lbm_objective))
    return LBM_E_INVALID;
  const lbm_params& p = h->p;
  if (h->kk != 0 || h->np < 1 || h->np > ADJ_MAX_PARTICLES) return LBM_E_INVALID;
  if (obj->particle < 0 || obj->particle >= h->np || obj->n0 < 1 || obj->n1 < obj->n0 ||
      obj->checkpoint_every < 0)
    return LBM_E_INVALID;
  const int comp = obj->component;
  if (comp != LBM_OBJ_X && comp != LBM_OBJ_Y && comp != LBM_OBJ_U && comp != LBM_OBJ_V &&
      comp != LBM_OBJ_W)
    return LBM_E_INVALID;
  if ((p.bc != LBM_BC_ZOUHE && p.bc != LBM_BC_HALFWAY_BB) ||
      (p.rheology != LBM_NEWTONIAN && p.rheology != LBM_BINGHAM) ||
      p.strain_model != LBM_STRAIN_MEQ || p.motion != LBM_MOTION_FREE ||
      p.collision != LBM_COLLISION_MRT ||
      (h->np > 1 && p.contact_test != LBM_CONTACT_DPP))
    return LBM_E_INVALID;
  int st = sticky_status(h);
  if (st) return st;
  cudaSetDevice(p.device);
  const long long N = obj->n1;
  const long long nlev = N - 1;  // lattice levels 1..N-1 act on the objective
  long long L = obj->checkpoint_every > 0 ? obj->checkpoint_every
                                          : std::max<long long>(1, std::llround(std::sqrt((double)N)));
  L = std::max<long long>(1, std::min<long long>(L, std::max<long long>(nlev, 1)));
  const int C = nlev > 0 ? (int)((nlev + L - 1) / L) : 0;
  const int nsets = C >= 2 ? 2 : 1;
  int rc = adj_reserve(h, nsets * (int)L, C, N + 1);
  if (rc) return rc;
  const size_t rec = (size_t)PS * h->npad;
  const size_t sb = adj_slot_bytes(h);

  // ---- forward --------------------------------------------------------------
  CK(cudaMemcpyAsync(h->adj_hist, h->ps, rec * sizeof(double), cudaMemcpyDeviceToDevice,
                     h->stream));
  std::vector<char> ck_partials(C + 1, 0);
  h->adj_record = true;  // the particle kernel stores each step's records
  for (long long n = 1; n <= N && rc == LBM_OK; ++n) {
    if ((n - 1) % L == 0 && (n - 1) / L < C) {
      const int c = (int)((n - 1) / L);
      cudaError_t e = adj_save_fields(h, h->adj_ck + sb * c);
      if (e == cudaSuccess) e = adj_save_small(h, c);
      if (e != cudaSuccess) rc = cuda_fail(e);
      ck_partials[c] = h->partials_valid ? 1 : 0;
    }
    if (rc == LBM_OK) rc = enqueue_step(h);
  }
  h->adj_record = false;
  if (rc) return rc;
  h->out_kk = -1;
  CK(adj_save_small(h, C));  // state after step N, put back at the end
  const bool final_partials = h->partials_valid;

  // ---- reverse --------------------------------------------------------------
  const size_t np = (size_t)h->npad;
  CK(cudaMemsetAsync(h->adj_state, 0, 8 * np * sizeof(double), h->stream));
  CK(cudaMemsetAsync(h->adj_p, 0, 5 * np * sizeof(double), h->stream));
  CK(cudaMemsetAsync(h->adj_h, 0, 3 * np * sizeof(double), h->stream));
  CK(cudaMemsetAsync(h->adj_rho, 0, np * sizeof(double), h->stream));
  CK(cudaMemsetAsync(h->adj_g, 0, 2 * (size_t)h->g.nbx * h->g.nby * sizeof(double), h->stream));
  struct Restore {  // recomputed steps record no history and no profile
    lbm_sim* h;
    int every;
    bool prof;
    ~Restore() {
      h->p.series_every = every;
      h->prof = prof;
    }
  } restore{h, h->p.series_every, h->prof};
  h->p.series_every = 0;
  h->prof = false;
  CK(launch_adj_particles(adj_particle_args(h, obj, N), h->stream));
  // The recompute stream starts after everything enqueued so far and the
  // handle's stream ends after everything the recompute stream was given.
  CK(cudaEventRecord(h->adj_ev[4], h->stream));
  CK(cudaStreamWaitEvent(h->adj_rs, h->adj_ev[4], 0));
  int ain = 0;
  bool have = false;
  {
    struct Join {
      lbm_sim* h;
      ~Join() {
        cudaEventRecord(h->adj_ev[4], h->adj_rs);
        cudaStreamWaitEvent(h->stream, h->adj_ev[4], 0);
      }
    } join{h};
    // Segment c into slot set c & 1, on the recompute stream (the step and
    // particle launchers take the handle's stream, switched for the call).
    auto recompute = [&](int c) -> int {
      const int set = c & 1;
      const long long t0 = (long long)c * L;
      const long long hi = std::min<long long>(t0 + L, nlev);
      // the level kernels of segment c + 2 are done reading the set
      CK(cudaStreamWaitEvent(h->adj_rs, h->adj_ev[2 + set], 0));
      struct Switch {
        lbm_sim* h;
        cudaStream_t own;
        ~Switch() { h->stream = own; }
      } sw{h, h->stream};
      h->stream = h->adj_rs;
      const int base = set * (int)L;
      CK(cudaMemcpyAsync(h->adj_slots + sb * base, h->adj_ck + sb * c, sb,
                         cudaMemcpyDeviceToDevice, h->stream));
      int r = adj_load_small(h, c, t0, ck_partials[c] != 0);
      for (int s = 0; r == LBM_OK && t0 + 1 + s < hi; ++s) r = adj_step_slots(h, base + s);
      if (r) return r;
      CK(cudaEventRecord(h->adj_ev[set], h->stream));
      return LBM_OK;
    };
    if (C > 0) rc = recompute(C - 1);
    for (int c = C - 1; c >= 0 && rc == LBM_OK; --c) {
      if (c > 0 && (rc = recompute(c - 1))) break;
      const int set = c & 1;
      const long long t0 = (long long)c * L;
      const long long hi = std::min<long long>(t0 + L, nlev);
      CK(cudaStreamWaitEvent(h->stream, h->adj_ev[set], 0));
      for (long long n = hi; n >= t0 + 1; --n) {
        const unsigned char* slot = h->adj_slots + sb * (size_t)(set * L + n - t0 - 1);
        // the first level of a segment follows a wait on the recompute
        // stream: no early start there
        CK(adj_level(h, n, slot, have ? h->adj_a[ain] : nullptr, have ? h->adj_w[ain] : nullptr,
                     h->adj_a[ain ^ 1], h->adj_w[ain ^ 1], n == hi ? 0 : 1));
        have = true;
        ain ^= 1;
        CK(launch_adj_particles(adj_particle_args(h, obj, n), h->stream));
      }
      CK(cudaEventRecord(h->adj_ev[2 + set], h->stream));
    }
  }  // the recompute stream joins the handle's stream here
  if (rc) return rc;
  // level 0: the collision of step 1 from INITIALIZE's state (nu, tau_y only)
  CK(adj_level(h, 0, nullptr, have ? h->adj_a[ain] : nullptr, have ? h->adj_w[ain] : nullptr,
               nullptr, nullptr, 1));
  // the handle back at step N
  if ((rc = adj_load_small(h, C, N, final_partials))) return rc;

  // ---- results ----------------------------------------------------------------
  std::vector<double> sv(8 * np), rv(np), gv(2 * (size_t)h->g.nbx * h->g.nby);
  CK(d2h(h, sv.data(), h->adj_state, sv.size() * sizeof(double)));
  CK(d2h(h, rv.data(), h->adj_rho, rv.size() * sizeof(double)));
  CK(d2h(h, gv.data(), h->adj_g, gv.size() * sizeof(double)));
  std::vector<double> hist((size_t)(N + 1) * rec);
  CK(d2h(h, hist.data(), h->adj_hist, hist.size() * sizeof(double)));
  CK(cudaStreamSynchronize(h->stream));
  double gnu = 0.0, gty = 0.0;
  for (size_t b = 0; b < gv.size(); b += 2) {
    gnu += gv[b];
    gty += gv[b + 1];
  }
  grads[LBM_GRAD_TAU_Y] = gty;
  grads[LBM_GRAD_NU] = gnu;
  for (int q = 0; q < h->np; ++q) {
    grads[LBM_GRAD_HEAD + LBM_GRAD_PER * q + 0] = rv[q];
    grads[LBM_GRAD_HEAD + LBM_GRAD_PER * q + 1] = sv[q];
    grads[LBM_GRAD_HEAD + LBM_GRAD_PER * q + 2] = sv[np + q];
  }
  if (value) {
    const int field = comp == LBM_OBJ_X ? P_X : comp == LBM_OBJ_Y ? P_Y : comp == LBM_OBJ_U ? P_U
                    : comp == LBM_OBJ_V ? P_V : P_W;
    double s = 0.0;
    for (long long n = obj->n0; n <= obj->n1; ++n)
      s += hist[rec * n + (size_t)field * np + obj->particle];
    *value = s / (double)(obj->n1 - obj->n0 + 1);
  }
  return refreshed_status(h);
}

// ===========================================================================
// Batched time steps.  All simulations of a batch advance in lockstep on the
// batch's stream: per step one launch of k_particles_batch (block b =
// simulation b) and one of the batched lattice kernel: k_step_batch (the
// TMA-staged tiles of the step kernel) or k_lattice_batch (one node per
// thread, any tile shape; the only one for BGK runs), whichever the
// autotuner timed fastest.  Steps run from a captured graph of
// BATCH_GRAPH_STEPS steps once the kernel, tile shape and grid are chosen.
struct lbm_batch {
  std::vector<lbm_sim*> sims;
  int device = 0;
  int prec = 0;
  int bgk = 0;             // some simulation uses the BGK collision
  int stress = 0;          // some simulation needs the strain rate (TMA kernel variant)
  int tma_bpsm = 0;        // resident blocks per SM of the TMA-staged kernel (0: not usable)
  CUtensorMap* d_tmaps = nullptr;  // [4 nsim]: each simulation's f[0], f[1], om[0], om[1]
  int nsm = 148;
  cudaStream_t stream = nullptr;
  BatchSim* d_sims = nullptr;
  ParticleArgs* d_pargs = nullptr;
  std::vector<BatchSim> h_sims;
  std::vector<ParticleArgs> h_pargs;
  long long total = 0;     // work items at the current shape
  int shape = -1;          // tuned (or fixed) tile shape, -1: not yet
  int bpsm = 0;            // persistent blocks per SM
  bool fixed = false;      // set by lbm_batch_set_tuning
  cudaGraphExec_t exec = nullptr;
  int graph_shape = -1, graph_bpsm = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

namespace {

constexpr int BATCH_GRAPH_STEPS = 8;
constexpr int BATCH_BPSM[3] = {2, 4, 6};

int batch_grid(const lbm_batch* b) {
  const long long g = (long long)(b->shape == BATCH_SHAPE_TMA ? b->tma_bpsm : b->bpsm) * b->nsm;
  return (int)std::max<long long>(1, std::min<long long>(g, b->total));
}

// Per-simulation arguments at tile shape `shape`, uploaded to the device.
// Tile width and height of shape (the TMA shape's depend on the precision).
int batch_tile_x(const lbm_batch*, int shape) {
  return shape == BATCH_SHAPE_TMA ? BATCH_TMA_TW : batch_bx(shape);
}
int batch_tile_y(const lbm_batch*, int shape) {
  return shape == BATCH_SHAPE_TMA ? BATCH_TMA_TR : batch_by(shape);
}

int batch_upload(lbm_batch* b, int shape) {
  const int n = (int)b->sims.size();
  const int bx = batch_tile_x(b, shape), by = batch_tile_y(b, shape);
  long long first = 0;
  for (int q = 0; q < n; ++q) {
    lbm_sim* h = b->sims[q];
    BatchSim& B = b->h_sims[q];
    B.a = lattice_args(h);
    for (int k = 0; k < 2; ++k) {
      B.f[k] = h->f[k];
      B.om[k] = h->om[k];
      B.pm[k] = h->pm[k];
    }
    B.kk = h->d_kk;
    B.rec_slot = h->rec_slot;
    B.par0 = (int)(((long long)h->cur - h->kk) & 1);
    B.nbx = (h->p.nx + 1 + bx - 1) / bx;
    B.first = first;
    first += (long long)B.nbx * ((h->p.ny + 1 + by - 1) / by);
    b->h_pargs[q] = particle_args(h);
  }
  b->total = first;
  CK(cudaMemcpyAsync(b->d_sims, b->h_sims.data(), n * sizeof(BatchSim), cudaMemcpyHostToDevice,
                     b->stream));
  CK(cudaMemcpyAsync(b->d_pargs, b->h_pargs.data(), n * sizeof(ParticleArgs),
                     cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));  // the host arrays are pageable and reused
  return LBM_OK;
}

cudaError_t batch_launch_lattice(lbm_batch* b) {
  const int n = (int)b->sims.size();
  if (b->shape == BATCH_SHAPE_TMA)
    return b->prec == LBM_FP64 ? launch_batch_tma_fp64(b->d_sims, n, b->d_tmaps, b->total,
                                                       b->stress, batch_grid(b), b->stream)
                               : launch_batch_tma_fp32(b->d_sims, n, b->d_tmaps, b->total,
                                                       b->stress, batch_grid(b), b->stream);
  return b->prec == LBM_FP64 ? launch_batch_fp64(b->d_sims, n, b->total, b->shape, b->bgk,
                                                 batch_grid(b), b->stream)
                             : launch_batch_fp32(b->d_sims, n, b->total, b->shape, b->bgk,
                                                 batch_grid(b), b->stream);
}

cudaError_t batch_launch_step(lbm_batch* b) {
  cudaError_t e = launch_particles_batch(b->d_pargs, (int)b->sims.size(), b->stream);
  if (e != cudaSuccess) return e;
  return batch_launch_lattice(b);
}

// Host bookkeeping of s completed batch steps.
void batch_advance(lbm_batch* b, int s) {
  for (lbm_sim* h : b->sims) {
    h->kk += s;
    h->cur ^= (s & 1);
    h->prev_post_bc = false;
    h->partials_valid = true;
    h->out_kk = -1;
  }
}

// Steps every simulation can take before its history ring is full.
long long batch_room(const lbm_batch* b) {
  long long room = 1LL << 40;
  for (const lbm_sim* h : b->sims) {
    const int every = h->p.series_every;
    if (!h->series || every <= 0) continue;
    const long long last = (h->series_cap + h->drained_kk / every + 1) * (long long)every - 1;
    room = std::min(room, last - h->kk);
  }
  return room;
}

int batch_tune(lbm_batch* b, int32_t& left) {
  // one timed step per candidate: the TMA-staged kernel (MRT batches), then
  // each (shape, blocks per SM) of the one-node-per-thread kernel; results
  // do not depend on the choice
  float best = 1e30f;
  int bs = 0, bb = BATCH_BPSM[0];
  std::vector<int> shapes;
  if (b->tma_bpsm > 0) shapes.push_back(BATCH_SHAPE_TMA);
  for (int sh = 0; sh < BATCH_SHAPES; ++sh) shapes.push_back(sh);
  for (const int sh : shapes) {
    if (left <= 0) break;
    int rc = batch_upload(b, sh);
    if (rc) return rc;
    b->shape = sh;
    const int ngrid = sh == BATCH_SHAPE_TMA ? 1 : 3;
    for (int k = 0; k < ngrid && left > 0 && batch_room(b) > 0; ++k) {
      b->bpsm = sh == BATCH_SHAPE_TMA ? b->tma_bpsm : BATCH_BPSM[k];
      CK(launch_particles_batch(b->d_pargs, (int)b->sims.size(), b->stream));
      CK(cudaEventRecord(b->ev[0], b->stream));
      CK(batch_launch_lattice(b));
      CK(cudaEventRecord(b->ev[1], b->stream));
      CK(cudaEventSynchronize(b->ev[1]));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
      batch_advance(b, 1);
      --left;
      if (ms < best) {
        best = ms;
        bs = sh;
        bb = b->bpsm;
      }
      // the next launch decodes the force sums this one left
      for (ParticleArgs& pa : b->h_pargs) pa.decode_force = 1;
      CK(cudaMemcpyAsync(b->d_pargs, b->h_pargs.data(), b->h_pargs.size() * sizeof(ParticleArgs),
                         cudaMemcpyHostToDevice, b->stream));
      CK(cudaStreamSynchronize(b->stream));
    }
  }
  b->shape = bs;
  b->bpsm = bb;
  return batch_upload(b, bs);
}

}  // namespace

extern "C" {

int lbm_batch_create(const lbm_params* params, int32_t nsim, lbm_batch** out) {
  if (!params || !out || nsim < 1) return LBM_E_INVALID;
  *out = nullptr;
  for (int q = 1; q < nsim; ++q)
    if (params[q].precision != params[0].precision || params[q].device != params[0].device)
      return LBM_E_INVALID;
  lbm_batch* b = new (std::nothrow) lbm_batch();
  if (!b) return LBM_E_NOMEM;
  auto fail = [&](int rc) {
    lbm_batch_destroy(b);
    return rc;
  };
  b->device = params[0].device;
  b->prec = params[0].precision;
  for (int q = 0; q < nsim; ++q) b->bgk |= params[q].collision == LBM_COLLISION_BGK;
  for (int q = 0; q < nsim; ++q) {
    lbm_sim* h = nullptr;
    int rc = lbm_create(&params[q], &h);
    if (rc) return fail(rc);
    b->sims.push_back(h);
  }
  cudaSetDevice(b->device);
  if (cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
    return fail(LBM_E_CUDA);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess ||
      prepare_particles_batch() != cudaSuccess)
    return fail(LBM_E_CUDA);
  int rc;
  if ((rc = dalloc(&b->d_sims, nsim)) || (rc = dalloc(&b->d_pargs, nsim))) return fail(rc);
  b->h_sims.resize(nsim);
  b->h_pargs.resize(nsim);
  // the TMA-staged kernel: every simulation's tensor maps, and its occupancy
  // (which also sets its shared-memory size, before any graph capture)
  for (lbm_sim* h : b->sims) b->stress |= (h->m.bingham || h->m.record_stress) ? 1 : 0;
  if (!b->bgk) {
    std::vector<CUtensorMap> tm(4 * (size_t)nsim);
    for (int q = 0; q < nsim; ++q) {
      lbm_sim* h = b->sims[q];
      for (int k = 0; k < 2; ++k) {
        CUtensorMap* fm = &tm[4 * (size_t)q + k];
        CUtensorMap* om = &tm[4 * (size_t)q + 2 + k];
        if ((rc = encode_f_map(h, h->f[k], fm, BATCH_TMA_TW, BATCH_TMA_TR))) return fail(rc);
        *om = *fm;
        if (h->om[k] && (rc = encode_om_map(h, h->om[k], om, BATCH_TMA_TW, BATCH_TMA_TR)))
          return fail(rc);
      }
    }
    if ((rc = dalloc(&b->d_tmaps, tm.size()))) return fail(rc);
    if (cudaMemcpy(b->d_tmaps, tm.data(), tm.size() * sizeof(CUtensorMap),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(LBM_E_CUDA);
    const cudaError_t e = b->prec == LBM_FP64 ? batch_tma_prepare_fp64(b->stress, &b->tma_bpsm)
                                              : batch_tma_prepare_fp32(b->stress, &b->tma_bpsm);
    if (e != cudaSuccess) return fail(cuda_fail(e));
  }
  *out = b;
  return LBM_OK;
}

lbm_sim* lbm_batch_sim(lbm_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->sims.size()) return nullptr;
  return b->sims[i];
}

int lbm_batch_tuning(lbm_batch* b, int32_t* tile_x, int32_t* tile_y, int32_t* blocks_per_sm) {
  if (!b || !tile_x || !tile_y || !blocks_per_sm) return LBM_E_INVALID;
  *tile_x = b->shape < 0 ? 0 : batch_tile_x(b, b->shape);
  *tile_y = b->shape < 0 ? 0 : batch_tile_y(b, b->shape);
  *blocks_per_sm = b->shape < 0 ? 0 : b->bpsm;
  return LBM_OK;
}

int lbm_batch_set_tuning(lbm_batch* b, int32_t tile_x, int32_t tile_y, int32_t blocks_per_sm) {
  if (!b) return LBM_E_INVALID;
  if (tile_x == 0) {
    b->fixed = false;
    b->shape = -1;
    return LBM_OK;
  }
  int sh = -1;
  for (int q = 0; q < BATCH_SHAPES; ++q)
    if (batch_bx(q) == tile_x && batch_by(q) == tile_y) sh = q;
  // the TMA-staged tiles run at their own occupancy (blocks_per_sm ignored)
  if (b->tma_bpsm > 0 && tile_x == batch_tile_x(b, BATCH_SHAPE_TMA) &&
      tile_y == batch_tile_y(b, BATCH_SHAPE_TMA)) {
    b->shape = BATCH_SHAPE_TMA;
    b->bpsm = b->tma_bpsm;
    b->fixed = true;
    return LBM_OK;
  }
  if (sh < 0 || blocks_per_sm < 1 || blocks_per_sm > 64) return LBM_E_INVALID;
  b->shape = sh;
  b->bpsm = blocks_per_sm;
  b->fixed = true;
  return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int32_t nsteps) {
  if (!b || nsteps < 0) return LBM_E_INVALID;
  cudaSetDevice(b->device);
  for (lbm_sim* h : b->sims) {
    int st = sticky_status(h);
    if (st) return st;
    CK(cudaStreamSynchronize(h->stream));  // the handles' own work first
  }
  int rc;
  int32_t left = nsteps;
  if (left == 0) return LBM_OK;
  // a simulation whose force sums are not yet valid (fresh, restarted) takes
  // one step with its own decode flag before the rest can be uniform
  if (b->shape < 0) {
    if ((rc = batch_tune(b, left))) return rc;
  } else {
    if ((rc = batch_upload(b, b->shape))) return rc;
  }
  while (left > 0) {
    long long room = batch_room(b);
    if (room <= 0) {
      CK(cudaStreamSynchronize(b->stream));
      for (lbm_sim* h : b->sims)
        if ((rc = drain_series(h))) return rc;
      continue;
    }
    bool uniform = true;
    for (const ParticleArgs& pa : b->h_pargs) uniform = uniform && pa.decode_force == 1;
    const long long chunk = std::min<long long>(left, room);
    if (uniform && chunk >= BATCH_GRAPH_STEPS) {
      if (!b->exec || b->graph_shape != b->shape || b->graph_bpsm != b->bpsm) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int s = 0; s < BATCH_GRAPH_STEPS && e == cudaSuccess; ++s) e = batch_launch_step(b);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          return LBM_E_CUDA;
        }
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e);
        b->graph_shape = b->shape;
        b->graph_bpsm = b->bpsm;
      }
      const long long reps = chunk / BATCH_GRAPH_STEPS;
      for (long long r = 0; r < reps; ++r) CK(cudaGraphLaunch(b->exec, b->stream));
      batch_advance(b, (int)(reps * BATCH_GRAPH_STEPS));
      left -= (int32_t)(reps * BATCH_GRAPH_STEPS);
      continue;
    }
    CK(batch_launch_step(b));
    batch_advance(b, 1);
    --left;
    if (!uniform) {
      for (ParticleArgs& pa : b->h_pargs) pa.decode_force = 1;
      CK(cudaMemcpyAsync(b->d_pargs, b->h_pargs.data(), b->h_pargs.size() * sizeof(ParticleArgs),
                         cudaMemcpyHostToDevice, b->stream));
      CK(cudaStreamSynchronize(b->stream));
    }
  }
  for (lbm_sim* h : b->sims)
    CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  int worst = LBM_OK;
  for (lbm_sim* h : b->sims) {
    int st = sticky_status(h);
    if (st && !worst) worst = st;
  }
  return worst;
}

int lbm_batch_stream(lbm_batch* b, void** stream) {
  if (!b || !stream) return LBM_E_INVALID;
  *stream = b->stream;
  return LBM_OK;
}

int lbm_batch_destroy(lbm_batch* b) {
  if (!b) return LBM_E_INVALID;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (lbm_sim* h : b->sims) lbm_destroy(h);
  dfree(b->d_sims);
  dfree(b->d_pargs);
  dfree(b->d_tmaps);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return LBM_OK;
}

}  // extern "C"
