// lbm_fp32.cu -- FP32 shifted-population instantiation of the lattice kernel
// (h = f - w_k*rho0 stored and computed in FP32; reductions in FP64).
#include "lbm_lattice.cuh"

namespace lbm {
cudaError_t launch_init_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_INIT);
}
cudaError_t launch_step_fp32(const LatticeArgs& a, const CUtensorMap* tm, cudaStream_t s) {
  return launch_step_tma<float>(a, tm, s);
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
cudaError_t launch_bgk_step_fp32(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<float>(a, s, MODE_STEP);
}
}  // namespace lbm
