// lbm_fp64.cu -- FP64 plain-population instantiation of the lattice kernel.
// Built with --fmad=false: every product and sum rounds on its own, in the
// reference's order, so the only differences from the FP64 oracle come from
// sin() and from the order of the force reductions.
#include "lbm_lattice.cuh"

namespace lbm {
cudaError_t launch_init_fp64(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<double>(a, s, MODE_INIT);
}
cudaError_t launch_step_fp64(const LatticeArgs& a, const CUtensorMap* tm, const CUtensorMap* tmo,
                             cudaStream_t s) {
  return launch_step_tma<double>(a, tm, tmo, s);
}
cudaError_t launch_output_fp64(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<double>(a, s, MODE_OUTPUT);
}
cudaError_t launch_restart_fp64(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<double>(a, s, MODE_RESTART);
}
cudaError_t launch_batch_fp64(const BatchSim* sims, int nsim, long long total, int shape,
                              int bgk, int grid, cudaStream_t s) {
  return launch_batch<double>(sims, nsim, total, shape, bgk, grid, s);
}
cudaError_t launch_batch_tma_fp64(const BatchSim* sims, int nsim, const CUtensorMap* tmaps,
                                  long long total, int stress, int grid, cudaStream_t s) {
  return launch_batch_tma<double>(sims, nsim, tmaps, total, stress, grid, s);
}
cudaError_t batch_tma_prepare_fp64(int stress, int* blocks_per_sm) {
  return batch_tma_prepare<double>(stress, blocks_per_sm);
}
cudaError_t launch_bgk_step_fp64(const LatticeArgs& a, cudaStream_t s) {
  return launch_mode<double>(a, s, MODE_STEP);
}
}  // namespace lbm
