// lbm_noalloc.cu -- lbm_fields_noalloc: the output fields (corrected
// velocity, density, solid fraction, SPM body force, particle image) of a
// lattice state held in caller-owned device memory, computed without
// allocating anything.
//
// Who needs it: a driver that must not allocate device memory while it runs,
// for instance one that has handed all device memory to its own pool or to
// other solvers, or one that post-processes from inside its time loop, where
// cudaMalloc/cudaFree would synchronise the whole device and stall its other
// streams.  lbm_get_field needs a simulation handle and the buffers lbm_create
// allocated; this entry point needs neither.
//
// Scratch: the per-tile candidate lists of the SPM evaluation live in one
// fixed, file-scope device array (NaScratch below, about 2.1 MB per device),
// so the largest lattice is LBM_NOALLOC_MAX_TILES list tiles of 128 x 8
// nodes and at most LBM_NOALLOC_MAX_PARTICLES disks; larger inputs are
// rejected with LBM_E_SCRATCH before anything is launched.  Every call first
// clears the tile counters and the overflow flag itself, so nothing has to
// start at zero.  All calls on one device share that one array: calls that
// overlap in time on the same device (different streams or host threads)
// race on it and must be serialised by the caller.
//
// The arithmetic is the output kernel's FP64 path (C1:1421-1439 macroscopic
// variables, C1:464-480 solid fraction and image, C1:488-507 body force with
// the last particle winning, C1:1138-1152 velocity correction), compiled with
// --fmad=false like the other FP64 translation units.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/lbm2d.h"
#include "lbm_internal.h"
#include "lbm_lattice.cuh"

namespace lbm {
namespace {

constexpr int NA_MAX_TILES = LBM_NOALLOC_MAX_TILES;
constexpr int NA_MAX_PARTICLES = LBM_NOALLOC_MAX_PARTICLES;
constexpr int NA_CAP = MAX_TILE_CAND;  // candidates per list tile

struct NaScratch {
  int count[NA_MAX_TILES];
  int list[NA_MAX_TILES * NA_CAP];
  int overflow;
  int nonfinite;
};

static __device__ __align__(256) NaScratch na_scratch;

// Device address of na_scratch, looked up once per device and context: the
// cache holds the driver's unique id of the context the address belongs to,
// so after a cudaDeviceReset (a new primary context, the module loaded
// again) the next call looks the address up again instead of using a
// dangling one.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
std::mutex na_mutex;
struct NaCache {
  NaScratch* ptr;
  unsigned long long ctx_id;
};
NaCache na_cache[64] = {};
CtxGetCurrentFn na_ctx_current = nullptr;
CtxGetIdFn na_ctx_id = nullptr;

// The id of the calling thread's current context (0 when none is current
// or the driver lacks cuCtxGetId).
unsigned long long current_ctx_id() {
  if (!na_ctx_current || !na_ctx_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return 0;
    na_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    na_ctx_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (na_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (na_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

__global__ void k_na_clear(NaScratch* s, int ntiles) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x)
    s->count[t] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s->overflow = 0;
    s->nonfinite = 0;
  }
}

// Disk p into the lists of every list tile within R + zeta/2 + 1 of its
// centre (PHI > 0 needs R - dist > -zeta/2).
__global__ void k_na_insert(NaScratch* s, const double* pin, int np, int nx, int ny, int ltx,
                            double zeta) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const double* r = pin + (long long)p * LBM_PIN;
  const double x = r[0], y = r[1], rad = 0.5 * r[6] + 0.5 * zeta + 1.0;
  if (!isfinite(x) || !isfinite(y) || !isfinite(rad) || !isfinite(r[3]) || !isfinite(r[4]) ||
      !isfinite(r[5])) {
    atomicExch(&s->nonfinite, 1);  // reported as LBM_E_NAN; the disk is left out
    return;
  }
  const int i0 = max((int)ceil(x - rad), 0), i1 = min((int)floor(x + rad), nx);
  const int j0 = max((int)ceil(y - rad), 0), j1 = min((int)floor(y + rad), ny);
  if (i0 > i1 || j0 > j1) return;
  for (int ty = j0 / LTY; ty <= j1 / LTY; ++ty)
    for (int tx = i0 / LTX; tx <= i1 / LTX; ++tx) {
      const int t = ty * ltx + tx;
      const int slot = atomicAdd(&s->count[t], 1);
      if (slot < NA_CAP)
        s->list[t * NA_CAP + slot] = p;
      else
        atomicExch(&s->overflow, 1);
    }
}

// One node per thread, blocks of 32 x 8 nodes inside one list tile.  The
// candidates of the tile are staged in shared memory in ascending index
// order, so the last disk with PHI > 0 sets G and PHI sums in index order.
__global__ void __launch_bounds__(256) k_na_fields(const NaScratch* s, const double* f,
                                                   const double* pin, double* out, int nx,
                                                   int ny, int ltx, double zeta, double pi) {
  __shared__ double s_px[NA_CAP], s_py[NA_CAP], s_pr[NA_CAP];
  __shared__ double s_pu[NA_CAP], s_pv[NA_CAP], s_pw[NA_CAP];
  const int tid = threadIdx.x, lane = tid & 31;
  const int i = blockIdx.x * 32 + lane;
  const int j = blockIdx.y * 8 + tid / 32;
  const int tile = blockIdx.y * ltx + (blockIdx.x * 32) / LTX;
  int nc = min(s->count[tile], NA_CAP);
  if (tid < 32) {
    const int pv = lane < nc ? s->list[tile * NA_CAP + lane] : 0x7fffffff;
    int rank = 0;
    for (int o = 0; o < 32; ++o) rank += (__shfl_sync(0xffffffffu, pv, o) < pv);
    if (lane < nc) {
      const double* r = pin + (long long)pv * LBM_PIN;
      s_px[rank] = r[0];
      s_py[rank] = r[1];
      s_pr[rank] = 0.5 * r[6];
      s_pu[rank] = r[3];
      s_pv[rank] = r[4];
      s_pw[rank] = r[5];
    }
  }
  __syncthreads();
  if (i > nx || j > ny) return;
  const long long o = (long long)j * (nx + 1) + i;
  const double* F = f + o * 9;
  const double f0 = F[0], f1 = F[1], f2 = F[2], f3 = F[3], f4 = F[4], f5 = F[5], f6 = F[6],
               f7 = F[7], f8 = F[8];
  const double rho = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
  const double rinv = 1.0 / rho;
  const double ux = rinv * (f1 + f5 + f8 - (f6 + f3 + f7));
  const double uy = rinv * (f5 + f2 + f6 - (f7 + f4 + f8));
  double gx = 0.0, gy = 0.0, phisum = 0.0;
  bool pnode = false;
  for (int c = 0; c < nc; ++c) {
    const double di = (double)i - s_px[c];
    const double dj = (double)j - s_py[c];
    const double phi = phi_double(di, dj, s_pr[c], zeta, pi);
    if (phi > 0.0) {
      const double uxp = s_pu[c] - s_pw[c] * dj;
      const double uyp = s_pv[c] + s_pw[c] * di;
      gx = phi * (uxp - ux);
      gy = phi * (uyp - uy);
      phisum += phi;
      if (phi >= 0.5) pnode = true;
    }
  }
  const long long nn = (long long)(nx + 1) * (ny + 1);
  out[o] = ux + 0.5 * (gx + 0.0);
  out[nn + o] = uy + 0.5 * (gy + 0.0);
  out[2 * nn + o] = rho;
  out[3 * nn + o] = phisum;
  out[4 * nn + o] = gx;
  out[5 * nn + o] = gy;
  out[6 * nn + o] = pnode ? 10.0 : 0.0;
}

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" int lbm_fields_noalloc(const lbm_params* p, const double* f, int32_t np,
                                  const double* particles, double* out, void* stream) {
  if (!p || !f || !out || np < 0 || (np > 0 && !particles)) return LBM_E_INVALID;
  if (p->struct_size != (int32_t)sizeof(lbm_params)) return LBM_E_ABI;
  if (p->nx < 1 || p->ny < 1 || !(p->zeta > 0.0) || !std::isfinite(p->zeta) ||
      !std::isfinite(p->pi))
    return LBM_E_INVALID;
  const int ltx = (p->nx + 1 + LTX - 1) / LTX, lty = (p->ny + 1 + LTY - 1) / LTY;
  if ((long long)ltx * lty > NA_MAX_TILES || np > NA_MAX_PARTICLES) return LBM_E_SCRATCH;
  const int ntiles = ltx * lty;

  // Set-up, once per device (and again after the device's context was
  // replaced): the device address of the static scratch, with that device
  // current.  The first call on a device does this, so it should come
  // before any stream capture.
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LBM_E_CUDA;
  NaScratch* s = nullptr;
  {
    std::lock_guard<std::mutex> lock(na_mutex);
    unsigned long long id = current_ctx_id();
    if (!na_cache[dev].ptr || id == 0 || id != na_cache[dev].ctx_id) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, na_scratch) != cudaSuccess || !ptr) return LBM_E_CUDA;
      na_cache[dev].ptr = static_cast<NaScratch*>(ptr);
      // the runtime has made the device's context current by now
      na_cache[dev].ctx_id = id ? id : current_ctx_id();
    }
    s = na_cache[dev].ptr;
  }

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_na_clear<<<(ntiles + 255) / 256, 256, 0, st>>>(s, ntiles);
  if (np > 0)
    k_na_insert<<<(np + 127) / 128, 128, 0, st>>>(s, particles, np, p->nx, p->ny, ltx, p->zeta);
  const dim3 grid((p->nx + 1 + 31) / 32, (p->ny + 1 + 7) / 8);
  k_na_fields<<<grid, 256, 0, st>>>(s, f, particles, out, p->nx, p->ny, ltx, p->zeta, p->pi);
  if (cudaGetLastError() != cudaSuccess) return LBM_E_CUDA;

  // The flags decide the return code: wait for this call's work.
  int flags[2] = {0, 0};
  if (cudaMemcpyAsync(flags, &s->overflow, sizeof(flags), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return LBM_E_CUDA;
  if (flags[1]) return LBM_E_NAN;
  return flags[0] ? LBM_E_OVERFLOW : LBM_OK;
}
