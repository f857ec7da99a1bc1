// lbm_main -- the reference's PROGRAM MAIN on liblbm2d.so (C ABI only).
//
// Runs one of the shipped cases the way its driver does (C1:97-399,
// C6:87-395, C3:87-440): constants of MODULE PARAM, the particle input file
// 0_Particle_Initial_Position.txt, the time loop, and the output files with
// the reference's names and columns:
//   00_Simulation_Parameters.txt   lattice and conversion constants
//   01_ParticleTimehistory.plt     C1: T,Y,Uy,Re_P,E_t (C1:142, C1:264)
//                                  C6: T,Y,X,ANG,Ux,Uy,OMG,Fx,BnT,Cd,ReT (C6:129, C6:315-318)
//   01_ClusterTimehistory.plt      C3: header only, as shipped (C3:129, C3:362)
//   01_AveragedDensity.PLT         Iteration, Density_Averaged every step (C1:318-319)
//   01_ErrorHistory.PLT            Iteration, Error every 1000 steps (C1:321-325)
//   02_VelocityField_<KK>.plt      Tecplot BLOCK field file (WriteResults, C1:1443-1491)
//   00_Simulation.TXT              LastIteration, RunTime, LastError (C1:398)
// and the restart dump of WRITE_OUTPUT / READ_INPUT (C1:351-379, C1:185-209):
//   0_F_output.txt 0_UX_output.txt 0_UY_output.txt 0_RHO_output.txt
//   0_Gspm_output.txt 0_OmegaBN_output.txt 0_Particle_output.txt
//   0_OmegaMRT_output.txt, one record per node with I outer and J inner.
// Numbers are written with 17 significant digits (the reference's
// list-directed output rounds differently; the columns are the same).  A
// restart keeps what the dump holds: centre, velocity and FORCE of each
// disk; VP_OLD, F_COL and F_H_IN start at zero as in a fresh reference
// process, and the step counter starts at 0 (C1:235).
//
//   C4 (4_Oscillating_Particle, C4:93-381): history Itr,F_D,F_L (C4:279),
//   the disk in code, the particle dump named 0_P1_output.txt (C4:342).
//
//   lbm_main --case c1|c6|c3|c4 [--nx N] [--ny N] [--steps N] [--input FILE]
//            [--precision fp64|fp32] [--out DIR] [--fields-every N]
//            [--dump DIR] [--restart DIR] [--device N] [--chunk N]
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "lbm2d.h"

namespace {

struct Opts {
  std::string cas = "c1", input = "0_Particle_Initial_Position.txt", out = ".", dump, restart;
  int nx = -1, ny = -1, steps = -1, precision = LBM_FP64, device = 0, fields_every = 0;
  int chunk = 1000;
  double lc = -1, ret = -1, tc = -1;  // C4 PARAMETER overrides (L_C, RE_T, T_C)
};

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "lbm_main: %s\n", msg.c_str());
  std::exit(2);
}

void check(int rc, const char* what) {
  if (rc != LBM_OK) die(std::string(what) + ": " + lbm_strerror(rc));
}

double r4(double x) { return (double)(float)x; }  // a default-kind REAL literal

// Case constants as MODULE PARAM evaluates them (REAL(4) literals widened).
struct Case {
  lbm_params p;
  double c_l = 0, c_t = 0, c_u = 0, c_g = 0, u_c = 1, l_c = 30, rho_s = 1.25, diam = 30;
  double t_c = 0, f_c = 0;  // C4: oscillation period and force scale
  int np = 1, time_max = 0, time_sample = 0;
  std::vector<double> pin;  // np * LBM_PIN
};

void mirror_edges(lbm_params& p) {  // 2*WALL%EDGE(3), 2*WALL%EDGE(4), C1:157-164
  const double edge3 = 0.5 * (double)p.ny + 0.5 * (2.0 * (double)p.ny);
  const double edge4 = 0.5 * (double)p.nx - 0.5 * (2.0 * (double)p.nx);
  p.wall_mirror_top = 2.0 * edge3;
  p.wall_mirror_left = 2.0 * edge4;
}

double glowinski_cij(double rho_s, double rho_f, double a_g, double pi, double d) {
  return -((((((rho_s - rho_f) * a_g) * pi) * 0.5) * d) * 0.5) * d;  // C1:701
}

// List-directed READ(200,*) of n records of k values (blank records skipped).
std::vector<double> read_records(const std::string& path, int n, int k) {
  std::ifstream f(path, std::ios::binary);
  if (!f) die("cannot open " + path);
  std::vector<double> v;
  std::string tok;
  std::string all((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  for (char& c : all)
    if (c == ',' || c == '\t' || c == '\r') c = ' ';
  std::istringstream in(all);
  while ((int)v.size() < n * k && in >> tok) {
    for (char& c : tok)
      if (c == 'd' || c == 'D') c = 'e';
    v.push_back(std::strtod(tok.c_str(), nullptr));
  }
  if ((int)v.size() < n * k) die(path + ": too few values");
  return v;
}

Case make_case(const Opts& o) {
  Case c;
  check(lbm_params_init(&c.p), "lbm_params_init");
  lbm_params& p = c.p;
  const double PI = p.pi;
  if (o.cas == "c1") {  // 1_Disk_Newtonian, C1:2-93
    p.nx = o.nx > 0 ? o.nx : 240;
    p.ny = o.ny > 0 ? o.ny : 720;
    mirror_edges(p);
    c.l_c = 30.0;
    c.c_l = r4(0.25) / c.l_c;
    c.c_t = (c.c_l * c.c_l) * p.nu / r4(0.1);
    c.c_u = c.c_l / c.c_t;
    c.c_g = c.c_l * r4(0.01) / (c.c_t * c.c_t);
    c.time_max = (int)(1.0 / c.c_t);
    c.np = 1;
    const std::vector<double> r = read_records(o.input, 1, 4);  // x y D rho_p, C1:170-175
    c.diam = r[2];
    c.rho_s = r4(1.25);
    p.c_ij = glowinski_cij(c.rho_s, 1.0, p.gravity, PI, c.diam);
    c.pin = {r[0], r[1], 0, 0, 0, 0, r[2], r[3]};
  } else if (o.cas == "c6") {  // 6_FreeFall_YieldStress, C6:2-83, C6:161-169
    p.nx = o.nx > 0 ? o.nx : 80;
    p.ny = o.ny > 0 ? o.ny : 300;
    const double nu = r4(0.025), rho_s = 2.0, rho_f = 1.0, re_s = r4(0.78), bn_s = r4(0.033);
    c.l_c = (double)(p.nx / 4);
    const double a_g = -(re_s * nu * nu / ((c.l_c * c.l_c * c.l_c) * (rho_s - rho_f) * rho_f));
    p.nu = nu;
    p.bc = LBM_BC_HALFWAY_BB;
    p.rheology = LBM_BINGHAM;
    p.rate_set = LBM_RATES_Q_OF_OMEGA;
    p.s_e = r4(1.1);
    p.s_eps = 1.25;
    p.wall_model = LBM_WALL_OFFSET;
    p.contact_test = LBM_CONTACT_STALE_DPW;
    p.integrate_angle = 1;
    p.gravity = a_g;
    p.tau_y = bn_s * (rho_s - rho_f) * (-a_g) * c.l_c;
    p.m_pap = r4(5.5e6);
    p.zeta = 1.0;
    p.rep_zeta = 1.0;
    p.eps_p = 0.5;
    p.eps_w = p.eps_p;
    p.e_p = 10.0;
    p.e_w = p.e_p;
    p.c_ij = glowinski_cij(rho_s, rho_f, a_g, PI, c.l_c);
    p.record_stress = 1;
    c.rho_s = rho_s;
    c.diam = c.l_c;
    c.u_c = (c.l_c * c.l_c) * (rho_s - rho_f) * (-a_g) / nu;
    c.time_max = (int)std::lround(r4(1.6) * c.l_c * c.l_c / nu);
    c.np = 1;
    c.pin = {0.5 * (double)p.nx, (double)p.ny - 7.0 * c.l_c, 0, 0, 0, 0, c.l_c, rho_s};
  } else if (o.cas == "c4") {  // 4_Oscillating_Particle, C4:2-93, C4:197-214
    p.nx = o.nx > 0 ? o.nx : 1500;
    p.ny = o.ny > 0 ? o.ny : 1000;
    const double nu = r4(0.025), re_t = o.ret > 0 ? o.ret : 100.0;
    c.l_c = o.lc > 0 ? o.lc : 50.0;
    c.u_c = re_t * nu / c.l_c;                        // C4:30
    c.t_c = o.tc > 0 ? o.tc : 5.0 * c.l_c / c.u_c;    // C4:32
    c.f_c = 0.5 * c.u_c * c.u_c * c.l_c;              // C4:33
    p.nu = nu;
    p.bc = LBM_BC_EQUILIBRIUM;
    p.rate_set = LBM_RATES_Q_OF_OMEGA;
    p.s_e = r4(1.6);
    p.s_eps = r4(1.8);
    p.gravity = 0.0;
    p.wall_model = LBM_WALL_NONE;
    p.motion = LBM_MOTION_OSCILLATE;
    p.osc_u = c.u_c;
    p.osc_period = c.t_c;
    c.time_max = (int)(6.0 * c.t_c);                  // DO WHILE(KK<INT(6.0*T_C))
    c.np = 1;
    c.rho_s = 1.0;
    c.diam = c.l_c;
    c.pin = {0.5 * (double)p.nx, 0.5 * (double)p.ny, 0, -c.u_c, 0, 0, c.l_c, 1.0};
  } else if (o.cas == "c3") {  // 3_MultiParticle_Sedimentation, C3:2-83, C3:145-156
    p.nx = o.nx > 0 ? o.nx : 512;
    p.ny = o.ny > 0 ? o.ny : 512;
    const double nu = (double)(0.4915f / 3.0f);
    c.rho_s = r4(1.01);
    c.l_c = 16.0;
    c.c_l = r4(0.0625) / c.l_c;
    c.c_t = (c.c_l * c.c_l) * nu / r4(0.01);
    c.c_u = c.c_l / c.c_t;
    c.c_g = c.c_l * r4(0.01) / (c.c_t * c.c_t);
    const double a_g = -r4(9.81) / c.c_g;
    p.nu = nu;
    p.bc = LBM_BC_HALFWAY_BB;
    p.rate_set = LBM_RATES_Q_OF_OMEGA;
    p.s_e = r4(1.1);
    p.s_eps = 1.25;
    p.wall_model = LBM_WALL_OFFSET;
    p.contact_test = LBM_CONTACT_STALE_DPW;
    p.gravity = a_g;
    p.zeta = 1.0;
    p.rep_zeta = 1.0;
    p.eps_p = 2.0;
    p.eps_w = 0.5 * p.eps_p;
    p.e_p = 20.0;
    p.e_w = 0.5 * p.e_p;
    p.c_ij = glowinski_cij(c.rho_s, 1.0, a_g, PI, c.l_c);
    c.diam = c.l_c;
    c.time_max = (int)std::lround(r4(24.0) / c.c_t);
    c.time_sample = (int)std::lround(1.0 / c.c_t);
    std::vector<double> r;
    {  // N_PARTICLE = 504 records of x y, or as many as the file holds
      std::ifstream f(o.input);
      if (!f) die("cannot open " + o.input);
      int count = 0;
      std::string line;
      while (std::getline(f, line)) {
        std::istringstream in(line);
        double a, b;
        if (in >> a >> b) ++count;
      }
      c.np = count < 504 ? count : 504;
    }
    r = read_records(o.input, c.np, 2);
    for (int i = 0; i < c.np; ++i) {
      const double rec[LBM_PIN] = {r[2 * i], r[2 * i + 1], 0, 0, 0, 0, c.diam, c.rho_s};
      c.pin.insert(c.pin.end(), rec, rec + LBM_PIN);
    }
  } else {
    die("unknown case " + o.cas);
  }
  p.precision = o.precision;
  p.device = o.device;
  p.series_every = 1;
  p.series_particles = c.np < 4 ? c.np : 4;
  p.series_capacity = 2 * o.chunk + 16;
  return c;
}

std::string fmt(double v) {
  char b[40];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

std::string path_in(const std::string& dir, const std::string& name) {
  return dir.empty() || dir == "." ? name : dir + "/" + name;
}

// Tecplot BLOCK field file of WriteResults (C1:1443-1491).
void write_fields(lbm_sim* h, const lbm_params& p, long long kk, const std::string& dir) {
  const size_t n1x = p.nx + 1, n1y = p.ny + 1, nn = n1x * n1y;
  std::vector<double> ux(nn), uy(nn), rho(nn), t11(nn, 0.0), t22(nn, 0.0), t12(nn, 0.0);
  std::vector<int32_t> img(nn);
  check(lbm_get_field(h, LBM_FIELD_UX, ux.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_UY, uy.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_RHO, rho.data()), "lbm_get_field");
  check(lbm_get_image(h, img.data()), "lbm_get_image");
  if (p.record_stress) {
    check(lbm_get_field(h, LBM_FIELD_TAU11, t11.data()), "lbm_get_field");
    check(lbm_get_field(h, LBM_FIELD_TAU22, t22.data()), "lbm_get_field");
    check(lbm_get_field(h, LBM_FIELD_TAU12, t12.data()), "lbm_get_field");
  }
  std::ofstream f(path_in(dir, "02_VelocityField_" + std::to_string(kk) + ".plt"));
  f << " VARIABLES =X/D, Y/D, UX, UY, RHO,Solid_Nodes,TAU_11,TAU_22,TAU_12\n";
  f << " ZONE I=" << n1x << " J=" << n1y << " , F=BLOCK\n";
  auto block = [&](auto value) {
    for (size_t j = 0; j < n1y; ++j) {
      for (size_t i = 0; i < n1x; ++i) f << ' ' << fmt(value(i, j));
      f << '\n';
    }
  };
  block([](size_t i, size_t) { return (double)i; });
  block([](size_t, size_t j) { return (double)j; });
  block([&](size_t i, size_t j) { return ux[j * n1x + i]; });
  block([&](size_t i, size_t j) { return uy[j * n1x + i]; });
  block([&](size_t i, size_t j) { return rho[j * n1x + i]; });
  block([&](size_t i, size_t j) { return (double)img[j * n1x + i]; });
  block([&](size_t i, size_t j) { return t11[j * n1x + i]; });
  block([&](size_t i, size_t j) { return t22[j * n1x + i]; });
  block([&](size_t i, size_t j) { return t12[j * n1x + i]; });
}

// WRITE_OUTPUT block (C1:351-379): one record per node, I outer, J inner.
void write_dump(lbm_sim* h, const Case& c, const std::string& dir) {
  const lbm_params& p = c.p;
  const size_t n1x = p.nx + 1, n1y = p.ny + 1, nn = n1x * n1y;
  std::vector<double> F(9 * nn), om(nn), ux(nn), uy(nn), rho(nn), gx(nn), gy(nn),
      ps((size_t)c.np * LBM_STATE_PER);
  check(lbm_get_state(h, F.data(), om.data(), ps.data()), "lbm_get_state");
  check(lbm_get_field(h, LBM_FIELD_UX, ux.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_UY, uy.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_RHO, rho.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_GX, gx.data()), "lbm_get_field");
  check(lbm_get_field(h, LBM_FIELD_GY, gy.data()), "lbm_get_field");
  std::ofstream f51(path_in(dir, "0_F_output.txt")), f52(path_in(dir, "0_UX_output.txt")),
      f53(path_in(dir, "0_UY_output.txt")), f54(path_in(dir, "0_RHO_output.txt")),
      f55(path_in(dir, "0_Gspm_output.txt")), f56(path_in(dir, "0_OmegaBN_output.txt")),
      f57(path_in(dir, c.p.motion == LBM_MOTION_OSCILLATE ? "0_P1_output.txt" : "0_Particle_output.txt")), f59(path_in(dir, "0_OmegaMRT_output.txt"));
  if (!f51 || !f57) die("cannot write the dump into " + dir);
  for (size_t i = 0; i < n1x; ++i)
    for (size_t j = 0; j < n1y; ++j) {
      const size_t o = j * n1x + i;
      for (int k = 0; k < 9; ++k) f51 << ' ' << fmt(F[o * 9 + k]);
      f51 << '\n';
      f52 << ' ' << fmt(ux[o]) << '\n';
      f53 << ' ' << fmt(uy[o]) << '\n';
      f54 << ' ' << fmt(rho[o]) << '\n';
      f55 << ' ' << fmt(gx[o]) << ' ' << fmt(gy[o]) << '\n';
      f56 << ' ' << fmt(om[o]) << '\n';
    }
  for (int ip = 0; ip < c.np; ++ip) {  // CENTER, VELOCITY, FORCE
    const double* r = &ps[(size_t)ip * LBM_STATE_PER];
    const int cols[8] = {0, 1, 3, 4, 5, 9, 10, 11};
    for (int k : cols) f57 << ' ' << fmt(r[k]);
    f57 << '\n';
  }
  // OMEGA_MRT of the uniform relaxation rate (C1:1029-1048 / C6:1002-1021)
  const double om0 = 1.0 / (3. * p.nu + 0.5);
  const double oq = p.rate_set == LBM_RATES_Q_OF_OMEGA ? 8. * (2. - om0) / (8. - om0) : p.s_q;
  const double s[9] = {0.0, p.s_e, p.s_eps, 0.0, oq, 0.0, oq, om0, om0};
  for (double v : s) f59 << ' ' << fmt(v);
  f59 << '\n';
}

// READ_INPUT block (C1:185-209): F after the boundary conditions, OMEGA_BN,
// and per disk CENTER, VELOCITY, FORCE.
void read_dump(lbm_sim* h, const Case& c, const std::string& dir) {
  const lbm_params& p = c.p;
  const size_t n1x = p.nx + 1, n1y = p.ny + 1, nn = n1x * n1y;
  const std::vector<double> Fio = read_records(path_in(dir, "0_F_output.txt"), (int)nn, 9);
  const std::vector<double> omio = read_records(path_in(dir, "0_OmegaBN_output.txt"), (int)nn, 1);
  const std::vector<double> pr = read_records(path_in(dir, c.p.motion == LBM_MOTION_OSCILLATE ? "0_P1_output.txt" : "0_Particle_output.txt"), c.np, 8);
  std::vector<double> F(9 * nn), om(nn), ps((size_t)c.np * LBM_STATE_PER, 0.0);
  size_t r = 0;
  for (size_t i = 0; i < n1x; ++i)
    for (size_t j = 0; j < n1y; ++j, ++r) {
      const size_t o = j * n1x + i;
      for (int k = 0; k < 9; ++k) F[o * 9 + k] = Fio[r * 9 + k];
      om[o] = omio[r];
    }
  for (int ip = 0; ip < c.np; ++ip) {
    double* s = &ps[(size_t)ip * LBM_STATE_PER];
    const double* q = &pr[(size_t)ip * 8];
    s[0] = q[0]; s[1] = q[1];
    s[3] = q[2]; s[4] = q[3]; s[5] = q[4];
    s[9] = q[5]; s[10] = q[6]; s[11] = q[7];
    s[17] = c.pin[(size_t)ip * LBM_PIN + 6];
    s[18] = c.pin[(size_t)ip * LBM_PIN + 7];
    s[19] = INFINITY;
  }
  check(lbm_set_state(h, 0, F.data(), om.data(), c.np, ps.data()), "lbm_set_state");
}

Opts parse(int argc, char** argv) {
  Opts o;
  for (int a = 1; a < argc; ++a) {
    const std::string k = argv[a];
    auto val = [&]() -> std::string {
      if (a + 1 >= argc) die("missing value for " + k);
      return argv[++a];
    };
    if (k == "--help" || k == "-h") {
      std::printf(
          "lbm_main --case c1|c6|c3|c4 [--nx N] [--ny N] [--steps N] [--input FILE]\n"
          "         [--precision fp64|fp32] [--out DIR] [--fields-every N]\n"
          "         [--dump DIR] [--restart DIR] [--device N] [--chunk N]\n"
          "         [--lc L_C] [--ret RE_T] [--tc T_C]   (c4 PARAMETERs)\n");
      std::exit(0);
    } else if (k == "--case") o.cas = val();
    else if (k == "--nx") o.nx = std::atoi(val().c_str());
    else if (k == "--ny") o.ny = std::atoi(val().c_str());
    else if (k == "--steps") o.steps = std::atoi(val().c_str());
    else if (k == "--input") o.input = val();
    else if (k == "--out") o.out = val();
    else if (k == "--dump") o.dump = val();
    else if (k == "--restart") o.restart = val();
    else if (k == "--device") o.device = std::atoi(val().c_str());
    else if (k == "--fields-every") o.fields_every = std::atoi(val().c_str());
    else if (k == "--chunk") o.chunk = std::max(1, std::atoi(val().c_str()));
    else if (k == "--lc") o.lc = std::atof(val().c_str());
    else if (k == "--ret") o.ret = std::atof(val().c_str());
    else if (k == "--tc") o.tc = std::atof(val().c_str());
    else if (k == "--precision") {
      const std::string v = val();
      if (v == "fp64") o.precision = LBM_FP64;
      else if (v == "fp32") o.precision = LBM_FP32_SHIFTED;
      else die("precision must be fp64 or fp32");
    } else die("unknown option " + k);
  }
  return o;
}

}  // namespace

int main(int argc, char** argv) {
  const Opts o = parse(argc, argv);
  Case c = make_case(o);
  const lbm_params& p = c.p;
  const int steps = o.steps >= 0 ? o.steps : c.time_max;
  const double omega = 1.0 / (3. * p.nu + 0.5);

  {  // 00_Simulation_Parameters.txt (C1:114-121)
    std::ofstream f(path_in(o.out, "00_Simulation_Parameters.txt"));
    f << " **********************\n Lattice Parameter\n";
    f << " TAU_LB= " << fmt(1.0 / omega) << "\n U_LB_max= " << fmt(c.u_c) << "\n Tau_Y_LB= "
      << fmt(p.tau_y) << "\n A_G= " << fmt(p.gravity) << "\n MAX_ITR = " << c.time_max << "\n";
    f << " **********************\n Transformation Coefficients\n";
    f << " C_L (cm)= " << fmt(c.c_l) << "\n C_T (sec)= " << fmt(c.c_t) << "\n C_U (cm/s)= "
      << fmt(c.c_u) << "\n C_g (m/s^2)= " << fmt(c.c_g) << "\n";
  }
  lbm_sim* h = nullptr;
  check(lbm_create(&p, &h), "lbm_create");  // LBM_E_TAU replaces C1:127-130
  check(lbm_set_particles(h, c.np, c.pin.data()), "lbm_set_particles");
  if (!o.restart.empty()) read_dump(h, c, o.restart);

  std::ofstream f7(path_in(o.out, "01_ErrorHistory.PLT")), f8(path_in(o.out, "01_AveragedDensity.PLT"));
  f7 << " VARIABLES=Iteration,Error\n";
  f8 << " VARIABLES=Iteration,Density_Averaged\n";
  std::ofstream f11;
  if (o.cas == "c3") {
    f11.open(path_in(o.out, "01_ClusterTimehistory.plt"));
    f11 << " VARIABLES=T,UX_AVG,UY_AVG,UX_FLC,UY_FLC,PHI,DX,DY\n";
  } else {
    f11.open(path_in(o.out, "01_ParticleTimehistory.plt"));
    f11 << (o.cas == "c1"   ? " VARIABLES=T,Y,Uy,Re_P,E_t\n"
            : o.cas == "c4" ? " VARIABLES=Itr,F_D,F_L\n"
                            : " VARIABLES=T,Y,X,ANG,Ux,Uy,OMG,Fx,BnT,Cd,ReT\n");
  }

  const auto t0 = std::chrono::steady_clock::now();
  int32_t len = 0;
  check(lbm_series_record_len(h, &len), "lbm_series_record_len");
  std::vector<double> rec((size_t)len * (o.chunk + 8));
  double er = 1.0;
  long long kk = 0;
  // C4 writes after the lattice pass (C4:279): the row of step k carries the
  // force of step k, which the record of step k+1 starts with
  long long c4_k = -1;
  double c4_fhx = 0.0;
  auto c4_row = [&](double fx) {
    f11 << ' ' << fmt((double)c4_k / c.t_c) << ' ' << fmt((fx + c4_fhx) / c.f_c) << ' '
        << fmt(fx / c.f_c) << '\n';
  };
  while (kk < steps) {
    int n = (int)std::min<long long>(o.chunk, steps - kk);
    if (o.fields_every > 0) n = std::min<long long>(n, o.fields_every - kk % o.fields_every);
    if (kk % 1000 != 0) n = std::min<long long>(n, 1000 - kk % 1000);
    check(lbm_step(h, n), "lbm_step");
    kk += n;
    int32_t nrec = 0;
    check(lbm_get_series(h, rec.data(), o.chunk + 8, &nrec), "lbm_get_series");
    for (int r = 0; r < nrec; ++r) {
      const double* R = &rec[(size_t)r * len];
      const double k = R[0], avg = R[1];
      f8 << ' ' << (long long)k << ' ' << fmt(avg) << '\n';
      if (o.cas == "c3" || c.np < 1) continue;
      const double* d = R + LBM_SERIES_HEAD;  // x y angle u v omega Fx Fy Tz Fin_x Fin_y Fin_t
      const double x = d[0], y = d[1], ang = d[2], u = d[3], v = d[4], w = d[5];
      if (o.cas == "c4") {
        if (c4_k >= 0) c4_row(d[6]);
        c4_k = (long long)k;
        c4_fhx = d[9];
      } else if (o.cas == "c1") {  // C1:261-264
        const double re_p = c.pin[7] * c.diam * std::sqrt(u * u + v * v) / p.nu;
        const double dp = 0.5 * r4(0.25);  // 0.5*DIAM_PHYSICAL
        const double e_t = 0.5 * (c.rho_s * p.pi * (dp * dp)) * (u * u + v * v) * (c.c_u * c.c_u);
        f11 << ' ' << fmt(k * c.c_t) << ' ' << fmt(y * c.c_l) << ' ' << fmt(v * c.c_u) << ' '
            << fmt(re_p) << ' ' << fmt(e_t) << '\n';
      } else {  // C6:315-318
        const double L = c.l_c;
        f11 << ' ' << fmt(k * p.nu / (L * L)) << ' ' << fmt(y) << ' ' << fmt(x) << ' ' << fmt(ang)
            << ' ' << fmt(u) << ' ' << fmt(v / c.u_c) << ' ' << fmt(w) << ' ' << fmt(d[6] + d[9])
            << ' ' << fmt(p.tau_y * L / (p.nu * -v)) << ' ' << fmt((d[7] + d[10]) / (p.nu * -v))
            << ' ' << fmt(-v * L / p.nu) << '\n';
      }
    }
    if (kk % 1000 == 0) {  // C1:321-325
      check(lbm_compute_error(h, &er), "lbm_compute_error");
      f7 << ' ' << kk << ' ' << fmt(er) << '\n';
    }
    if (o.fields_every > 0 && kk % o.fields_every == 0) write_fields(h, p, kk, o.out);
  }
  if (o.cas == "c4" && c4_k >= 0) {  // the last row: the final state's force
    std::vector<double> po((size_t)c.np * LBM_POUT);
    check(lbm_get_particles(h, po.data()), "lbm_get_particles");
    c4_row(po[6]);
  }
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (o.fields_every <= 0) write_fields(h, p, kk, o.out);  // C1:392
  if (!o.dump.empty()) write_dump(h, c, o.dump);
  {
    std::ofstream f9(path_in(o.out, "00_Simulation.TXT"));
    f9 << " LastIteration= " << kk << " RunTime= " << fmt(secs) << " LastError= " << fmt(er)
       << '\n';
  }
  std::printf("steps %lld  %.3f s  %.1f MLUPS\n", kk, secs,
              (double)(p.nx + 1) * (p.ny + 1) * (double)kk / secs / 1e6);
  check(lbm_destroy(h), "lbm_destroy");
  return 0;
}
