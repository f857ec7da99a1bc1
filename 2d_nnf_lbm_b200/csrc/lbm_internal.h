// lbm_internal.h -- structures shared by the host orchestration (lbm_api.cu)
// and the sm_100a kernels (lbm_lattice.cuh, lbm_particles.cu).
//
// HBM layout of one simulation:
//   populations  f[2][9][NY+1][pitch]   structure of arrays, ping-pong pair;
//                pitch = NX+1 rounded up to 32 elements so every row starts
//                on a 128 B (FP32) / 256 B (FP64) boundary
//   omega        om[2][NY+1][pitch]     per-node Bingham relaxation rate
//   particles    ps[PS][npad]           structure of arrays, npad = np rounded to 32
//   force sums   facc[6][npad]          exact fixed-point FORCE accumulators
//   tile lists   tile_count[2][ntiles], tile_list[2][ntiles][tile_cap]
//   pair lists   nbr_count[npad], nbr[MAX_NEIGH][npad]  (Verlet lists with skin)
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace lbm {

// Switch values of lbm_params the kernels test (equal to the lbm2d.h enums;
// lbm_api.cu asserts it).
constexpr int BC_EQUILIBRIUM = 2;     // LBM_BC_EQUILIBRIUM
constexpr int MOTION_OSCILLATE = 1;   // LBM_MOTION_OSCILLATE

// Scalar lattice kernels: one node per thread, blocks of TX x TY nodes.
constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TPB = TX * TY;
// Particle candidate lists are kept per list tile of LTX x LTY nodes; a step
// kernel tile (128 x 4 FP32 or 64 x 8 FP64 nodes) lies inside one list tile.
constexpr int LTX = 128;
constexpr int LTY = 8;
constexpr int MAX_TILE_CAND = 32;   // particles that may touch one tile
constexpr int MAX_PARTICLES = 4096; // particles per simulation (shared-memory staging)
constexpr int MAX_NEIGH = 32;       // pair-list entries per particle
constexpr double SKIN = 2.0;        // Verlet skin (lattice units) of pair and tile lists
constexpr double MASS_FIX = 1099511627776.0;  // 2^40: fixed-point scale of the mass sum
// FORCE accumulators: v = hi*2^-20 + lo*2^-62 (both exact integer sums)
constexpr double FHI = 1048576.0;                  // 2^20
constexpr double FLO = 4398046511104.0;            // 2^42
constexpr double FDEC_HI = 1.0 / 1048576.0;        // 2^-20
constexpr double FDEC_LO = 1.0 / 4611686018427387904.0;  // 2^-62

// Particle record (doubles).
enum : int {
  P_X = 0, P_Y, P_ANG, P_U, P_V, P_W,   // CENTER, ANGLE, VELOCITY
  P_UO, P_VO, P_WO,                     // VP_OLD
  P_FX, P_FY, P_TZ,                     // FORCE (hydrodynamic)
  P_FCX, P_FCY,                         // F_COL
  P_FHX, P_FHY, P_FHT,                  // F_H_IN
  P_D, P_RHO, P_M, P_I,                 // DIAM, RHO_P, M_P, I_P
  P_XT, P_YT,                           // centre at the last tile-list build
  P_R2,
  PS
};

// Field f of particle p in the structure-of-arrays particle state.
struct PRef {
  double* base;  // &ps[p]
  int stride;    // npad
  __host__ __device__ double& operator[](int f) const { return base[(long long)f * stride]; }
};

// Sticky status bits.
enum : int {
  ST_NAN = 1,
  ST_OVERFLOW = 2,
  ST_TIMEOUT = 4,
  ST_PARTICLE = 8,
  ST_BOUNDS = 16,  // checked build: an index check failed, the access was skipped
};

// Index checks of the checked build (compiled with LBM_CHECKED): an index
// outside [0, n) of its buffer sets ST_BOUNDS in the handle's status word and
// the guarded access is skipped, so a wrong index shows as LBM_E_BOUNDS
// instead of reading or writing memory it should not.  The ordinary build
// compiles every check to true.
#ifdef LBM_CHECKED
__device__ __forceinline__ bool lbm_in_range(long long i, long long n, int* status) {
  if (i >= 0 && i < n) return true;
  atomicOr(status, ST_BOUNDS);
  return false;
}
#define LBM_IN(i, n, st) lbm_in_range((long long)(i), (long long)(n), (st))
#else
#define LBM_IN(i, n, st) true
#endif

struct Geometry {
  int nx, ny;        // cells; nodes 0..nx, 0..ny
  int pitch;         // elements per row
  long long plane;   // elements per population plane = pitch*(ny+1)
  int nbx, nby;      // scalar-kernel blocks
  int ltx, lty;      // list tiles
};

// Population k lives in plane plane_of(k) of a population buffer.  The planes
// are grouped by the row shift c_y of the pull (0: k=0,1,3; +1: k=2,5,6;
// -1: k=4,7,8), so one 3-D TMA box of depth 3 fetches the three planes that
// share a row offset.
__host__ __device__ constexpr int plane_of(int k) {
  return k == 2 ? 3 : k == 3 ? 2 : k == 4 ? 6 : k == 5 ? 4 : k == 6 ? 5 : k;
}

struct Model {
  int bc;            // LBM_BC_*
  int bingham;       // 1: per-node viscosity (Papanastasiou Bingham or Casson)
  int casson;        // 1: the Casson viscosity function
  int strain_feq;    // 1: strain rate of C1 (m_neq against COMPUTEFEQNEW's moments)
  int q_of_omega;    // 1: s_q = 8(2-w)/(8-w)
  int record_stress; // 1: write stress/yield ring
  double rho0, nu, omega, s_e, s_eps, s_q, d_mrt, pi, zeta;
  double tau_y, m_pap, gamma_min;
  double w_init[3];
  double S_uni[9];   // rates at the uniform omega (Newtonian nodes)
  // FP32 copies, so kernels never convert per node
  float rho0_f, nu_f, d_mrt_f, pi_f, zeta_f, tau_y_f, m_pap_f, gamma_min_f;
  float s_e_f, s_eps_f, sq_uni_f, omega_f;
  float shift_f[9];  // rho0*w_k*(36*d_mrt - 1)
  // equilibrium boundary in FP32: COMPUTEFEQNEW weights and, per k,
  // rho0*(W_k*B_k(u=0) - w_k) of the shifted form
  float w_init_f[3], eq_c_f[9];
  // LBM_COLLISION_BGK (COLLISION, C1:774-841): bi-viscosity MU_R = 1000 nu,
  // GAMMA_C = tau_y/(MU_R - nu); ComputeSourceEquilib_Hydro's forcing weights
  // (the REAL(4) quotients 4/9, 1/9, 1/36)
  int bgk;
  double mu_r, gamma_c, w_src[3];
  float mu_r_f, gamma_c_f, w_src_f[3];
};

struct ParticleArgs {
  double* ps;                // [PS][npad]
  int np, npad;
  unsigned long long* facc;  // [6][npad]
  int decode_force;          // 1: FORCE = decoded accumulators (then zeroed)
  int* tile_count;           // [2][ntiles]
  int* tile_list;            // [2][ntiles][tile_cap]
  int* tile_cur;             // [2]: list buffer valid for step k at [k&1]
  int* tile_order;           // [2][2][ntiles]: list tiles, those without disks first;
                             // forward and with each group reversed
  int* n_unlisted;           // [2]: how many list tiles have no disk
  int* work_ctr;             // [2]: step-kernel tile queue of step k at [k&1]
  int tile_cap;
  int ntiles, nbx;
  int motion;                // LBM_MOTION_*
  double osc_u, osc_period, pi;
  int* nbr;                  // [MAX_NEIGH][npad]
  int* nbr_count;            // [npad]
  double* nbr_xy;            // [2][npad] centres at the last pair-list build
  int* pair_rebuild;         // 1: rebuild the pair lists before use
  // repulsion
  int wall_model, contact;
  double rep_zeta, eps_p, eps_w, e_p, e_w, c_ij, mirror_top, mirror_left;
  double rho0, gravity;
  int integrate_angle;
  int ncx, ncy;
  double cell_size;
  double* stale_dpw;
  // bookkeeping
  long long* kk;
  int* rec_slot;             // history slot of this step, -1 if none
  double* series;
  unsigned long long* mass_acc;  // [series_cap] fixed-point sum of rho - rho0
  int series_every, series_cap, series_len, series_np;
  int* status;
  int nx, ny;
  double zeta;               // SPM interface thickness (tile box radius)
  // adjoint forward pass: record of step k into hist[k][PS][npad] (k < hist_n)
  double* hist;
  long long hist_n;
};

struct LatticeArgs {
  Geometry g;
  Model m;
  const void* src;       // f read (post-collision, or post-BC in restart)
  void* dst;             // f written
  const void* om_src;
  void* om_dst;
  // LBM_COLLISION_BGK with a Bingham rheology: the density (FP32: rho - rho0)
  // and corrected velocity of each node's previous collision, T[3][plane]
  const void* pm_src;
  void* pm_dst;
  const double* ps;      // [PS][npad]
  int np, npad;
  const int* tile_count; // [2][ntiles]
  const int* tile_list;
  const int* tile_cur;   // [2]: list buffer valid for step k at [k&1]
  const int* tile_order; // [2][2][ntiles]: list tiles, those without disks first;
                         // forward and with each group reversed (odd steps)
  const int* n_unlisted; // [2]
  int* work_ctr;         // [2]: tile queue of step k at [k&1], zero at the start
  int tile_cap;
  int ntiles;
  // equilibrium boundary: density (FP32: rho - rho0) and corrected velocity
  // of the nodes next to the edges, T[2 parities][3][ring_n]
  void* ring;
  int ring_n;
  unsigned long long* facc;  // [6][npad]
  long long step;        // lattice step of this launch
  int rec_slot;          // history slot of this step (-1: none)
  unsigned long long* mass_acc;
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
cudaError_t launch_step_fp64(const LatticeArgs& a, const CUtensorMap* tm, const CUtensorMap* tmo,
                             cudaStream_t s);
cudaError_t launch_output_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_restart_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_init_fp32(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_step_fp32(const LatticeArgs& a, const CUtensorMap* tm, const CUtensorMap* tmo,
                             cudaStream_t s);
cudaError_t launch_output_fp32(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_restart_fp32(const LatticeArgs& a, cudaStream_t s);
// One time step of the BGK collision (one node per thread).
cudaError_t launch_bgk_step_fp64(const LatticeArgs& a, cudaStream_t s);
cudaError_t launch_bgk_step_fp32(const LatticeArgs& a, cudaStream_t s);

// TMA box of the step kernel: one tile row (128 FP32 / 64 FP64 nodes) plus
// a 16-byte vector of halo on each side; 512 / row-width rows; one plane.
inline int step_tile_width(int esz) { return esz == 8 ? 64 : 128; }
inline int step_box_width(int esz) { return step_tile_width(esz) + 2 * (16 / esz); }
inline int step_box_rows(int esz) { return 512 / (esz == 8 ? 64 : 128); }

// Particle kernel (lbm_particles.cu).
cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s);
// tile_order / n_unlisted of list buffer buf from its counts.
cudaError_t launch_tile_order(const ParticleArgs& a, int buf, cudaStream_t s);
// Tile lists (into buffer 0) and a pair-list rebuild request, after
// set_particles / set_state.
cudaError_t launch_tiles_only(const ParticleArgs& a, cudaStream_t s);

// ---------------------------------------------------------------------------
// Batched time steps (lbm_batch_*): many independent simulations advance in
// one launch of the particle kernel (one block per simulation) and one of
// the lattice kernel (a persistent grid over every simulation's tiles).
struct BatchSim {
  LatticeArgs a;       // the simulation's lattice arguments; src/dst, om_src/
                       // om_dst, step and rec_slot are set on the device
  void* f[2];
  void* om[2];
  void* pm[2];         // previous-collision macros (BGK bi-viscosity), or null
  long long* kk;       // step counter (the particle kernel increments it)
  int* rec_slot;       // history slot of the step (written by the particle kernel)
  int par0;            // f[(par0 + kk - 1) & 1] holds f*(kk) at lattice step kk
  int nbx;             // tiles per row at the batch tile shape
  long long first;     // first work item of this simulation
};

// Batch tile shapes (nodes): 0: 32 x 8, 1: 64 x 4, 2: 128 x 2 (one node per
// thread); BATCH_SHAPE_TMA: the TMA-staged step kernel's pipeline on tiles of
// 64 x 8 nodes, MRT models only.
constexpr int BATCH_SHAPES = 3;
constexpr int BATCH_SHAPE_TMA = 3;
constexpr int BATCH_TMA_TW = 64, BATCH_TMA_TR = 8;  // its tile, both precisions
__host__ __device__ constexpr int batch_bx(int shape) { return shape == 0 ? 32 : (shape == 1 ? 64 : 128); }
__host__ __device__ constexpr int batch_by(int shape) { return 256 / batch_bx(shape); }

cudaError_t launch_batch_fp32(const BatchSim* sims, int nsim, long long total, int shape,
                              int bgk, int grid, cudaStream_t s);
cudaError_t launch_batch_fp64(const BatchSim* sims, int nsim, long long total, int shape,
                              int bgk, int grid, cudaStream_t s);
// The TMA-staged batched step: tensor maps of f[0], f[1] per simulation
// (tmaps[4 q + b]) and of om[0], om[1] (tmaps[4 q + 2 + b]), BatchSim::first /
// nbx counted in step-kernel tiles.
cudaError_t launch_batch_tma_fp32(const BatchSim* sims, int nsim, const CUtensorMap* tmaps,
                                  long long total, int stress, int grid, cudaStream_t s);
cudaError_t launch_batch_tma_fp64(const BatchSim* sims, int nsim, const CUtensorMap* tmaps,
                                  long long total, int stress, int grid, cudaStream_t s);
// Sets the kernel's shared-memory size and returns its resident blocks per SM
// (call before any graph capture).
cudaError_t batch_tma_prepare_fp32(int stress, int* blocks_per_sm);
cudaError_t batch_tma_prepare_fp64(int stress, int* blocks_per_sm);
cudaError_t prepare_particles_batch();
cudaError_t launch_wait_selftest(int* status, uint32_t limit, cudaStream_t s);
cudaError_t launch_particles_batch(const ParticleArgs* args, int nsim, cudaStream_t s);

// ---------------------------------------------------------------------------
// Adjoint (reverse-mode) sweep, lbm_adjoint.cu.  Level n of the forward is
// the step kernel that reads f*(n), omega(n) and the particle records of
// step n and produces FORCE(n), f*(n+1), omega(n+1); the particle kernel of
// step n+1 then maps (records n, FORCE(n)) to records n+1.
constexpr int ADJ_MAX_PARTICLES = 64;

// Adjoint field of the populations: a[k] is dJ/dF(k) of the populations
// after streaming and boundary conditions, stored like f (plane_of(k) planes).
struct AdjLatticeArgs {
  Geometry g;
  Model m;
  const void* fs;       // f*(n) (T planes); unused at level 0
  const void* oms;      // omega(n) (T), Bingham
  const void* a_in;     // dJ/dF(n+1) (T planes), null: zero
  const void* aw_in;    // dJ/domega(n+1) (T), null: zero
  void* a_out;          // dJ/dF(n) (T planes); unused at level 0
  void* aw_out;         // dJ/domega(n) (T), Bingham
  const double* ps;     // particle records of step n, [PS][npad]
  const double* a_h;    // dJ/dFORCE(n), [3][npad] (x, y, torque)
  double* a_p;          // += lattice part of dJ/d(records n): [5][npad] x y u v w
  double* gacc;         // [blocks][2] += (dJ/dnu, dJ/dtau_y), one slot per block
  int np, npad;
  int level0;           // 1: the collision of step 1 from INITIALIZE's state
  double kappa;         // 36*d_mrt: the scale of the collision's inverse transform
};

struct AdjParticleArgs {
  const double* prev;   // records of step n-1
  const double* cur;    // records of step n
  double* a_state;      // [8][npad] dJ/d(state): x y u v w uo vo wo, n -> n-1 in place
  double* a_p;          // [5][npad] lattice part at step n, zeroed here
  double* a_h;          // [3][npad] out: dJ/dFORCE(n-1)
  double* a_rho;        // [npad] += dJ/drho_p
  int np, npad;
  long long n, n0, n1;  // reverse of the particle update of step n; objective window
  int obj_p, obj_c;     // observed disk and record field (P_X, P_Y, P_U, P_V, P_W)
  double obj_w;         // 1 / (n1 - n0 + 1)
  int wall_model;
  double rep_zeta, eps_p, eps_w, e_p, e_w, c_ij, mirror_top, mirror_left;
  double rho0, gravity;
  int nx, ny;
};

// pdl: launch as a programmatic dependent of the previous kernel (which must
// be the particle adjoint kernel: the lattice kernel waits for it only
// before reading dJ/dFORCE and adding to a_p).
cudaError_t launch_adj_lattice_fp32(const AdjLatticeArgs& a, cudaStream_t s, int pdl);
cudaError_t launch_adj_lattice_fp64(const AdjLatticeArgs& a, cudaStream_t s, int pdl);
cudaError_t launch_adj_particles(const AdjParticleArgs& a, cudaStream_t s);
cudaError_t launch_set_ll(long long* p, long long v, cudaStream_t s);

// Host and device decode the force accumulators the same way.
__host__ __device__ inline double decode_force(unsigned long long hi, unsigned long long lo) {
  return (double)(long long)hi * FDEC_HI + (double)(long long)lo * FDEC_LO;
}

}  // namespace lbm
