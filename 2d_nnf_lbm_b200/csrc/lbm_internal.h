// lbm_internal.h -- structures shared by the host orchestration (lbm_api.cu)
// and the sm_100a kernels (lbm_lattice.cuh, lbm_particles.cu).
//
// HBM layout of one simulation:
//   populations  f[2][9][NY+1][pitch]   structure of arrays, ping-pong pair;
//                pitch = NX+1 rounded up to 32 elements so every row starts
//                on a 128 B (FP32) / 256 B (FP64) boundary
//   omega        om[2][NY+1][pitch]     per-node Bingham relaxation rate
//   particles    ps[np][PS]             one 192 B FP64 record per disk
//   tile lists   tile_count[ntiles], tile_list[ntiles][tile_cap]
//   partials     part[np][max_slots][3] per-tile hydrodynamic force sums
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lbm {

// Lattice tile = one thread block, one node per thread.
constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TPB = TX * TY;
constexpr int MAX_TILE_CAND = 32;  // particles that may touch one tile

// Particle record (doubles).
enum : int {
  P_X = 0, P_Y, P_ANG, P_U, P_V, P_W,   // CENTER, ANGLE, VELOCITY
  P_UO, P_VO, P_WO,                     // VP_OLD
  P_FX, P_FY, P_TZ,                     // FORCE (hydrodynamic)
  P_FCX, P_FCY,                         // F_COL
  P_FHX, P_FHY, P_FHT,                  // F_H_IN
  P_D, P_RHO, P_M, P_I,                 // DIAM, RHO_P, M_P, I_P
  P_R0, P_R1, P_R2,
  PS
};

// Sticky status bits.
enum : int {
  ST_NAN = 1,
  ST_OVERFLOW = 2,
  ST_TIMEOUT = 4,
  ST_PARTICLE = 8,
};

struct Geometry {
  int nx, ny;        // cells; nodes 0..nx, 0..ny
  int pitch;         // elements per row
  long long plane;   // elements per population plane = pitch*(ny+1)
  int nbx, nby;      // tiles
};

struct Model {
  int bc;            // LBM_BC_*
  int bingham;       // 1: Papanastasiou
  int q_of_omega;    // 1: s_q = 8(2-w)/(8-w)
  int record_stress; // 1: write stress/yield ring
  double rho0, nu, omega, s_e, s_eps, s_q, d_mrt, pi, zeta;
  double tau_y, m_pap, gamma_min;
  double w_init[3];
  double shift_c[9]; // FP32 shifted: rho0*w_k*(36*d_mrt - 1)
};

struct ParticleArgs {
  double* ps;
  int np;
  int4* tbox;            // per particle (tx0, ty0, ntx, nty)
  int* tile_count;
  int* tile_list;
  int tile_cap;
  int max_slots;
  // repulsion
  int wall_model, contact;
  double rep_zeta, eps_p, eps_w, e_p, e_w, c_ij, mirror_top, mirror_left;
  double rho0, gravity;
  int integrate_angle;
  // cell list scratch
  int* cell_count;       // ncells + 1
  int* cell_start;       // ncells + 1
  int* cell_items;       // np
  int* cell_of;          // np
  int ncx, ncy;
  double cell_size;
  double* stale_dpw;
  // bookkeeping
  long long* kk;
  double* series;
  int series_every, series_cap, series_len, series_np;
  int* status;
  int nx, ny;
  double zeta;           // SPM interface thickness (tile box radius)
};

struct LatticeArgs {
  Geometry g;
  Model m;
  const void* src;       // f read (post-collision, or post-BC in restart)
  void* dst;             // f written
  const void* om_src;
  void* om_dst;
  const double* ps;
  double* ps_force;      // same array, written by the last block only
  int np;
  const int* tile_count;
  const int* tile_list;
  int tile_cap;
  const int4* tbox;
  double* partials;
  int max_slots;
  unsigned int* ticket;
  double* mass_partials;
  const long long* kk;
  double* series;
  int series_every, series_cap, series_len;
  int* status;
  // stress ring: 2 slots x (tau11, tau22, tau12, yield) fields
  void* rec;             // T[2][4][NY+1][pitch]
  // output mode
  double* out;           // [7][NY+1][NX+1]: ux uy rho phi gx gy image
  double* out_f;         // [9*(NX+1)*(NY+1)] post-BC F in F(0:8,i,j) order, may be null
  int src_post_bc;       // 1: src already holds post-BC populations
  int initial;           // 1: state is INITIALIZE (rho0, u=0, G=0)
};

// Launchers (defined in lbm_fp64.cu / lbm_fp32.cu).
cudaError_t launch_init_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_step_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_output_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_restart_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_init_fp32(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_step_fp32(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_output_fp32(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_restart_fp32(const LatticeArgs& a, cudaStream_t s);

// Particle kernel (lbm_particles.cu).
cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s);
// Tile lists only (after set_particles / set_state, before the first step).
cudaError_t launch_tiles_only(const ParticleArgs& a, cudaStream_t s);

}  // namespace lbm
