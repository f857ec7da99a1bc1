// lbm_fp32.cu -- FP32 shifted-population instantiation of the lattice kernel
// (h = f - w_k*rho0 stored and computed in FP32; reductions in FP64).
#include "lbm_lattice.cuh"

namespace lbm {
cudaError_t launch_init_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_INIT);
}
cudaError_t launch_step_fp32(const LatticeArgs& a, const CUtensorMap* tm, const CUtensorMap* tmo,
                             cudaStream_t s) {
  return launch_step_tma<float>(a, tm, tmo, s);
}
cudaError_t launch_output_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_OUTPUT);
}
cudaError_t launch_restart_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_RESTART);
}
cudaError_t launch_batch_fp32(const BatchSim* sims, int nsim, long long total, int shape,
                              int bgk, int grid, cudaStream_t s) {
  return launch_batch<float>(sims, nsim, total, shape, bgk, grid, s);
}
// The failure path of the bounded wait: one thread waits on a fresh
// mbarrier that nothing arrives at (phase 0 never completes), gives up after
// `limit` polls and flags the timeout as the step kernel does.
__global__ void k_wait_selftest(int* status, uint32_t limit) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x != 0) return;
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (!mbar_wait(b, 0, limit)) atomicOr(status, ST_TIMEOUT);
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(b) : "memory");
}

cudaError_t launch_wait_selftest(int* status, uint32_t limit, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(status, limit);
  return cudaGetLastError();
}
cudaError_t launch_batch_tma_fp32(const BatchSim* sims, int nsim, const CUtensorMap* tmaps,
                                  long long total, int stress, int grid, cudaStream_t s) {
  return launch_batch_tma<float>(sims, nsim, tmaps, total, stress, grid, s);
}
cudaError_t batch_tma_prepare_fp32(int stress, int* blocks_per_sm) {
  return batch_tma_prepare<float>(stress, blocks_per_sm);
}
cudaError_t launch_bgk_step_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_STEP);
}
}  // namespace lbm
