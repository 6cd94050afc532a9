// Oracle harness: drives the reference solver's OWN classes (compiled from the
// unmodified reference sources by oracle/Makefile) on a case written here, and
// dumps fields for the parity tests.  Test infrastructure only: nothing in the
// product links or runs this.
//
// The harness mirrors the reference's main() (Z4_Mercury/main.cpp:27-99):
// Param -> Grid_Preprocess -> build_topology -> Field -> SingularEdgeRegistry
// -> Halo -> EdgeOwnerSyncPattern -> MercurySolver.  It then overrides the
// initial state (the reference only ships uniform initial conditions,
// Z4_Mercury/include/2_Initial.h:134-215) and calls the reference's own
// StepOnce() (Z4_Mercury/src/MercurySolver_Driver.cpp:21-61).
//
// Usage:  mercury_ref <job-file>
// The job file holds "key value" lines; see oracle/mercury_oracle.py.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "00_Mercury_Const.h"
#include "0_basic/MPI_WRAPPER.h"
#include "1_grid/1_MPCNS_Grid.h"
#include "2_topology/Topology.h"
#include "2_topology/TopologyBuilder.h"
#include "3_field/Field.h"
#include "4_halo/Halo.h"
#include "4_halo/HaloEdgeOwner.h"
#include "7_metric/SingularEdgeRegistry.h"
#include "MercuryGridValidation.h"

// The harness needs the solver's private step and field members; it is the
// test driver, so it opens the class the way a unit-test friend would.
#define private public
#define protected public
#include "MercurySolver.h"
#undef private
#undef protected

namespace fs = std::filesystem;

namespace {

std::map<std::string, std::string> g_job;

std::string job_str(const std::string &k, const std::string &def = "") {
  auto it = g_job.find(k);
  return it == g_job.end() ? def : it->second;
}
double job_dbl(const std::string &k, double def) {
  auto it = g_job.find(k);
  return it == g_job.end() ? def : std::stod(it->second);
}
long job_int(const std::string &k, long def) {
  auto it = g_job.find(k);
  return it == g_job.end() ? def : std::stol(it->second);
}

// ---------------------------------------------------------------- RNG
// Seeded exactly as the workload definition states: std::mt19937_64 with
// seed 20261203 + solve_id, uniforms formed as (x >> 11) * 2^-53.
struct Uniform {
  std::mt19937_64 g;
  explicit Uniform(uint64_t seed) : g(seed) {}
  double next() { return (double)(g() >> 11) * 0x1.0p-53; }
  double sym(double a) { return -a + 2.0 * a * next(); }
};

// ---------------------------------------------------------------- case files
void write_text(const fs::path &p, const std::string &s) {
  std::ofstream f(p);
  f << s;
}

std::string setup_general() {
  std::ostringstream o;
  o << "double  CFL " << job_dbl("cfl", 0.4) << "\n";
  o << "double  yee 0.125\n";
  o << "double  max_Time 1e30\n";
  o << "int     output_step 0\n";
  o << "int     output_residual " << job_int("output_residual", 0) << "\n";
  o << "double  Archive_Output_Time 1e30\n";
  o << "bool    post_static_output 0\n";
  o << "bool    output_dec_jedge 0\n";
  o << "int     dimension 3\n";
  o << "int     ngg " << job_int("ngg", 4) << "\n";
  o << "bool    continue_calc 0\n";
  o << "bool    continue_calc_index 0\n";
  o << "int     Read_Method 2\n";
  o << "int     max_Nstep " << job_int("steps", 1) << "\n";
  o << "int     corner_treat 2\n";
  o << "double  eta_max_mercury " << job_dbl("eta_max", 1.25e7) << "\n";
  o << "int     ns 2\n";
  o << "double  mole_mass1 0.001\n";
  o << "double  mole_mass2 0.023\n";
  o << "LIST==================================================================\n";
  o << "constant        5\n(double)\n";
  o << "gamma           NA              R_uni       mu_mag             q_e\n";
  o << "1.6667          6.02E23         8.314       1.256637061e-6     1.602E-19\n";
  o << "LIST==================================================================\n";
  o << "double  scale 1.0\n";
  o << "END_OF_FILE\n";
  return o.str();
}

std::string setup_initial() {
  // REF is the reference's own production normalisation
  // (Z4_Mercury/9999setup/1_Initial_condition.txt:1-7).
  std::ostringstream o;
  o << "LIST==================================================================\n";
  o << "REF             6\n(double)\n";
  o << "U               T               n           Molecular_mass  B_ref   L_ref\n";
  o << "4.031E5         1.7407E5        4E7         0.001           1E-9    2.44E6\n";
  o << "LIST==================================================================\n";
  o << "LIST==================================================================\n";
  o << "INITIAL         9\n(double)\n";
  o << "U               T               n           Molecular_mass  c_y     c_z     Bx      By      Bz\n";
  o << job_str("initial_line",
               "4.03112887E5 1.7407E5 4E7 0.001 1.240347346E-1 0.0 -1.52E-8 8.4E-9 -8.5E-9")
    << "\n";
  o << "LIST==================================================================\n";
  o << "END_OF_FILE\n";
  return o.str();
}

std::string setup_boundary() {
  std::ostringstream o;
  o << "LIST==================================================================\n";
  o << "Boundary_Priority      5\n(int)\n";
  o << "Pole                   Outflow     Absorbing   Solid_Surface   Farfield\n";
  o << "0                      4           2           3               1\n";
  o << "LIST==================================================================\n";
  o << "LIST==================================================================\n";
  o << "Boundary_Farfield      5\n(double)\n";
  o << "U                      T           n           c_y             c_z\n";
  o << job_str("farfield_line", "4.03112887E5 1.7407E5 4E7 1.240347346E-1 0.0") << "\n";
  o << "LIST==================================================================\n";
  o << "LIST==================================================================\n";
  o << "Boundary_Solid_Surface 1\n(double)\n";
  o << "T\n288\n";
  o << "LIST==================================================================\n";
  o << "END_OF_FILE\n";
  return o.str();
}

std::string setup_mhd() {
  std::ostringstream o;
  o << "int     num_of_dipole " << job_int("num_of_dipole", 0) << "\n";
  o << "LIST==================================================================\n";
  o << "Dipole1         7\n(double)\n";
  o << "x0              y0              z0          mx          my          mz          a\n";
  o << job_str("dipole_line", "0.0 0.0 0.0 0.0 0.0 -2.83E19 0.0") << "\n";
  o << "LIST==================================================================\n";
  o << "bool    is_Mercury_resistance " << job_int("resistive", 0) << "\n";
  o << "double  mercury_eta_r_inner " << job_dbl("eta_r_inner", 0.84) << "\n";
  o << "double  mercury_eta_r_outer " << job_dbl("eta_r_outer", 1.04) << "\n";
  o << "double  mercury_eta_width " << job_dbl("eta_width", 0.02) << "\n";
  o << "double  implicit_resistive_ksp_rtol " << job_dbl("ksp_rtol", 5e-3) << "\n";
  o << "double  implicit_resistive_ksp_atol " << job_dbl("ksp_atol", 1e-8) << "\n";
  o << "int     implicit_resistive_ksp_max_it " << job_int("ksp_max_it", 200) << "\n";
  o << "bool    is_Ambipolar_Efield " << job_int("ambipolar", 1) << "\n";
  o << "double  r_min " << job_dbl("hall_r_min", 0.0) << "\n";
  o << "double  r_max " << job_dbl("hall_r_max", 0.0) << "\n";
  o << "double  arti_eta_max " << job_dbl("arti_eta_max", 0.0) << "\n";
  o << "double  J_range_start " << job_dbl("arti_J_start", 800.0) << "\n";
  o << "double  J_range_on " << job_dbl("arti_J_on", 3000.0) << "\n";
  o << "bool    is_local_artificial_resistivity " << job_int("local_arti", 0) << "\n";
  o << "double  local_arti_eta_max " << job_dbl("local_arti_eta_max", 0.1) << "\n";
  o << "double  local_arti_x0 " << job_dbl("local_arti_x0", 1.53) << "\n";
  o << "double  local_arti_y0 " << job_dbl("local_arti_y0", 0.0) << "\n";
  o << "double  local_arti_z0 " << job_dbl("local_arti_z0", 0.25) << "\n";
  o << "double  local_arti_r_decay " << job_dbl("local_arti_r_decay", 0.05) << "\n";
  o << "double  local_arti_r_cutoff " << job_dbl("local_arti_r_cutoff", 0.05) << "\n";
  o << "END_OF_FILE\n";
  return o.str();
}

const char *kFvbnd =
    "FVBND 1 3\nNo_Boundary_Condition\nSolid_Surface\nSymmetry\nFarfield\nInflow\nOutflow\nPole\n"
    "Generic_#1\nGeneric_#2\nGeneric_#3\nPERIOD-X\nperiod_X\nPERIOD-Y\nperiod_Y\nPERIOD-Z\nperiod_Z\n"
    "BOUNDARIES\n";

void write_grid_binary(const fs::path &p, const std::vector<std::string> &names,
                       const std::vector<std::array<int, 3>> &dims,
                       const std::vector<std::vector<double>> &xyz /* per block: x,y,z k-j-i */) {
  std::ofstream f(p, std::ios::binary);
  int32_t nb = (int32_t)names.size();
  f.write((const char *)&nb, 4);
  for (auto &n : names) {
    int32_t len = (int32_t)n.size() + 1;
    f.write((const char *)&len, 4);
    f.write(n.c_str(), len);
  }
  for (auto &d : dims)
    for (int a = 0; a < 3; ++a) {
      int32_t v = d[a];
      f.write((const char *)&v, 4);
    }
  for (auto &b : xyz) f.write((const char *)b.data(), (std::streamsize)(b.size() * sizeof(double)));
}

// Config "cube": one periodic block of n0 x n1 x n2 cells on the unit box
// ("n" holds one count for a cube or three per-axis counts), periodic in
// every direction, nodes x_a = xi_a + amp*sin(2 pi xi_b)*sin(2 pi xi_c) for
// cyclic (a, b, c), xi_a = index / n_a.  Periodic connectivity uses negative
// block ids (src/1_grid/1_MPCNS_Grid.cpp:455-464).
void cube_counts(int nc[3]) {
  std::istringstream is(job_str("n", "32"));
  is >> nc[0];
  if (!(is >> nc[1] >> nc[2])) nc[1] = nc[2] = nc[0];
}

void write_cube_case(const fs::path &geo) {
  int nc[3];
  cube_counts(nc);
  const double amp = job_dbl("amp", 0.05);
  const int np0 = nc[0] + 1, np1 = nc[1] + 1, np2 = nc[2] + 1;
  const double two_pi = 2.0 * std::acos(-1.0);
  std::vector<double> x((size_t)np0 * np1 * np2), y(x.size()), z(x.size());
  for (int k = 0; k < np2; ++k)
    for (int j = 0; j < np1; ++j)
      for (int i = 0; i < np0; ++i) {
        const double a = (double)i / nc[0], b = (double)j / nc[1], c = (double)k / nc[2];
        const size_t o = ((size_t)k * np1 + j) * np0 + i;
        x[o] = a + amp * std::sin(two_pi * b) * std::sin(two_pi * c);
        y[o] = b + amp * std::sin(two_pi * c) * std::sin(two_pi * a);
        z[o] = c + amp * std::sin(two_pi * a) * std::sin(two_pi * b);
      }
  std::vector<double> blk;
  blk.insert(blk.end(), x.begin(), x.end());
  blk.insert(blk.end(), y.begin(), y.end());
  blk.insert(blk.end(), z.begin(), z.end());
  write_grid_binary(geo / "grid   0.grd", {"Fluid"}, {{np0, np1, np2}}, {blk});

  fs::create_directories(geo / "boundary_condition");
  write_text(geo / "boundary_condition" / "boundary   0.txt", "\t0\n");
  write_text(geo / "boundary_condition" / "boundary_name.fvbnd", kFvbnd);
  write_text(geo / "boundary_condition" / "parallel   0.txt", "\t1\t0\n\t0\nimin\timax\tjmin\tjmax\tkmin\tkmax\ts_r_id\ts_flag\tr_flag\tPhysic_Name\n");
  // Six periodic face pairs, both directions listed as in the reference's own
  // geometry fixtures (Z0_NULL/CASE/geometry.tar.gz).
  std::ostringstream in;
  const std::string N[3] = {std::to_string(np0), std::to_string(np1), std::to_string(np2)};
  auto face = [&](int axis, bool hi) {
    std::string r[3];
    for (int a = 0; a < 3; ++a) {
      if (a == axis)
        r[a] = (hi ? N[a] : "1") + std::string("\t") + (hi ? N[a] : "1");
      else if (a == (axis + 2) % 3)
        r[a] = "-1\t-" + N[a];  // second tangential direction carries the sign mark
      else
        r[a] = "1\t" + N[a];
    }
    return r[0] + "\t" + r[1] + "\t" + r[2];
  };
  in << "\t6\n\t6\nimin\timax\tjmin\tjmax\tkmin\tkmax\tid\tPhysic_Name\n";
  for (int axis = 0; axis < 3; ++axis) {
    in << face(axis, false) << "\t-1\tFluid\n" << face(axis, true) << "\t-1\tFluid\n";
    in << face(axis, true) << "\t-1\tFluid\n" << face(axis, false) << "\t-1\tFluid\n";
  }
  write_text(geo / "boundary_condition" / "inner   0.txt", in.str());
}

// Case "lattice": the periodic curvilinear unit cube of the "cube" case cut
// into bx x by x bz aligned blocks of n^3 cells each (block id
// (p * by + q) * bz + r for lattice position (p, q, r)).  Every block face is
// an inner patch joined to the neighbouring block's opposite face, listed
// from both sides with the "cube" case's orientation marks; a patch that
// wraps around the box carries negative block ids (periodic,
// src/1_grid/1_MPCNS_Grid.cpp:455-464).  No physical or parallel patches.
void write_lattice_case(const fs::path &geo) {
  const int n = (int)job_int("n", 4);
  int nb[3] = {2, 2, 2};
  std::istringstream(job_str("nb", "2 2 2")) >> nb[0] >> nb[1] >> nb[2];
  const double amp = job_dbl("amp", 0.05);
  const int np = n + 1;
  const double two_pi = 2.0 * std::acos(-1.0);
  const int nblock = nb[0] * nb[1] * nb[2];
  auto bid = [&](int p, int q, int r) { return (p * nb[1] + q) * nb[2] + r; };
  std::vector<std::string> names(nblock, "Fluid");
  std::vector<std::array<int, 3>> dims(nblock, {np, np, np});
  std::vector<std::vector<double>> xyz(nblock);
  for (int p = 0; p < nb[0]; ++p)
    for (int q = 0; q < nb[1]; ++q)
      for (int r = 0; r < nb[2]; ++r) {
        const size_t m = (size_t)np * np * np;
        std::vector<double> blk(3 * m);
        for (int k = 0; k < np; ++k)
          for (int j = 0; j < np; ++j)
            for (int i = 0; i < np; ++i) {
              const double a = (double)(p * n + i) / (nb[0] * n), b = (double)(q * n + j) / (nb[1] * n),
                           c = (double)(r * n + k) / (nb[2] * n);
              const size_t o = ((size_t)k * np + j) * np + i;
              blk[o] = a + amp * std::sin(two_pi * b) * std::sin(two_pi * c);
              blk[m + o] = b + amp * std::sin(two_pi * c) * std::sin(two_pi * a);
              blk[2 * m + o] = c + amp * std::sin(two_pi * a) * std::sin(two_pi * b);
            }
        xyz[bid(p, q, r)] = std::move(blk);
      }
  write_grid_binary(geo / "grid   0.grd", names, dims, xyz);

  fs::create_directories(geo / "boundary_condition");
  std::string bnd, par = "\t" + std::to_string(nblock) + "\t0\n";
  for (int b = 0; b < nblock; ++b) {
    bnd += "\t0\n";
    par += "\t0";
  }
  par += "\nimin\timax\tjmin\tjmax\tkmin\tkmax\ts_r_id\ts_flag\tr_flag\tPhysic_Name\n";
  write_text(geo / "boundary_condition" / "boundary   0.txt", bnd);
  write_text(geo / "boundary_condition" / "boundary_name.fvbnd", kFvbnd);
  write_text(geo / "boundary_condition" / "parallel   0.txt", par);
  const std::string N = std::to_string(np);
  auto face = [&](int axis, bool hi) {
    std::string rg[3];
    for (int a = 0; a < 3; ++a) {
      if (a == axis)
        rg[a] = (hi ? N : "1") + std::string("\t") + (hi ? N : "1");
      else if (a == (axis + 2) % 3)
        rg[a] = "-1\t-" + N;
      else
        rg[a] = "1\t" + N;
    }
    return rg[0] + "\t" + rg[1] + "\t" + rg[2];
  };
  std::ostringstream in;
  in << "\t" << 6 * nblock << "\n";
  for (int b = 0; b < nblock; ++b) in << "\t6";
  in << "\nimin\timax\tjmin\tjmax\tkmin\tkmax\tid\tPhysic_Name\n";
  for (int p = 0; p < nb[0]; ++p)
    for (int q = 0; q < nb[1]; ++q)
      for (int r = 0; r < nb[2]; ++r) {
        const int pos[3] = {p, q, r};
        for (int axis = 0; axis < 3; ++axis)
          for (int hi = 0; hi < 2; ++hi) {
            int t[3] = {p, q, r};
            const bool wrap = hi ? pos[axis] == nb[axis] - 1 : pos[axis] == 0;
            t[axis] = (pos[axis] + (hi ? 1 : nb[axis] - 1)) % nb[axis];
            const int sgn = wrap ? -1 : 1;
            in << face(axis, hi) << "\t" << sgn * (bid(p, q, r) + 1) << "\tFluid\n"
               << face(axis, !hi) << "\t" << sgn * (bid(t[0], t[1], t[2]) + 1) << "\tFluid\n";
          }
      }
  write_text(geo / "boundary_condition" / "inner   0.txt", in.str());
}

// Config "shell": 6-panel gnomonic (equiangular) cubed-sphere shell,
// r in [1, r_out] with r_k = r_out^(k/nr); panel p has local axes
// (i: xi angle, j: eta angle, k: radius), right-handed.  Shared panel-edge
// nodes are bitwise identical (tan of the edge angles is set to +-1 exactly
// and the angle grid is symmetric), so the reference's mesh transfer sees
// conformal interfaces.  Inner boundary r = 1: "Coupled-Solid" (the name the
// reference registers its solid-wall handlers under); outer r = r_out: Farfield.
void shell_dir(int p, double ta, double tb, double d[3]) {
  switch (p) {
    case 0: d[0] = 1.0; d[1] = ta; d[2] = tb; break;
    case 1: d[0] = -ta; d[1] = 1.0; d[2] = tb; break;
    case 2: d[0] = -1.0; d[1] = -ta; d[2] = tb; break;
    case 3: d[0] = ta; d[1] = -1.0; d[2] = tb; break;
    case 4: d[0] = -tb; d[1] = ta; d[2] = 1.0; break;
    default: d[0] = tb; d[1] = ta; d[2] = -1.0; break;
  }
}
double shell_tan(int i, int n) {
  const int q = 2 * i - n;
  if (q == n) return 1.0;
  if (q == -n) return -1.0;
  return std::tan(((double)q / (double)n) * (std::acos(-1.0) / 4.0));
}
void shell_node(int p, int i, int j, int k, int na, int nr, double r_out, double out[3]) {
  double d[3];
  shell_dir(p, shell_tan(i, na), shell_tan(j, na), d);
  const double inv = 1.0 / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double r = (k == 0) ? 1.0 : (k == nr ? r_out : std::pow(r_out, (double)k / (double)nr));
  for (int a = 0; a < 3; ++a) out[a] = r * d[a] * inv;
}

void write_shell_case(const fs::path &geo) {
  const int na = (int)job_int("na", 48), nr = (int)job_int("nr", 96);
  const double r_out = job_dbl("r_out", 8.0);
  const int ni = na + 1, nk = nr + 1;
  std::vector<std::string> names(6, "Fluid");
  std::vector<std::array<int, 3>> dims(6, {ni, ni, nk});
  std::vector<std::vector<double>> xyz(6);
  for (int p = 0; p < 6; ++p) {
    auto &b = xyz[p];
    b.resize((size_t)3 * ni * ni * nk);
    const size_t npts = (size_t)ni * ni * nk;
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < ni; ++j)
        for (int i = 0; i < ni; ++i) {
          double x[3];
          shell_node(p, i, j, k, na, nr, r_out, x);
          const size_t o = ((size_t)k * ni + j) * ni + i;
          b[o] = x[0];
          b[npts + o] = x[1];
          b[2 * npts + o] = x[2];
        }
  }
  write_grid_binary(geo / "grid   0.grd", names, dims, xyz);

  // panel edge e: 0 = (i = 0), 1 = (i = na), 2 = (j = 0), 3 = (j = na); nodes along the
  // other angular index t at r = 1
  auto edge_pt = [&](int p, int e, int t, double out[3]) {
    const int i = e == 0 ? 0 : e == 1 ? na : t;
    const int j = e == 2 ? 0 : e == 3 ? na : t;
    shell_node(p, i, j, 0, na, nr, r_out, out);
  };
  struct Conn {
    int q, f;
    bool reversed;
  };
  Conn conn[6][4];
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e) {
      bool found = false;
      for (int q = 0; q < 6 && !found; ++q)
        for (int f = 0; f < 4 && !found; ++f) {
          if (q == p) continue;
          for (int rev = 0; rev < 2 && !found; ++rev) {
            bool ok = true;
            for (int t = 0; t <= na && ok; ++t) {
              double a[3], b[3];
              edge_pt(p, e, t, a);
              edge_pt(q, f, rev ? na - t : t, b);
              ok = a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
            }
            if (ok) {
              conn[p][e] = {q, f, rev != 0};
              found = true;
            }
          }
        }
      if (!found) {
        std::fprintf(stderr, "shell: panel %d edge %d has no partner\n", p, e);
        std::exit(3);
      }
    }
  // inner patches, 1-based node ranges; the normal dimension has sub == sup,
  // the angular tangential is sign-marked (paired with the partner's angular
  // tangential), the radial tangential is unmarked and runs 1..nk on both sides.
  const std::string A = std::to_string(ni), K = std::to_string(nk);
  auto ranges = [&](int e, bool rev) {
    std::string r[3];
    const bool on_i = (e == 0 || e == 1);
    const std::string fixed = (e == 0 || e == 2) ? "1" : A;
    const std::string ang = rev ? ("-" + A + "\t-1") : ("-1\t-" + A);
    r[on_i ? 0 : 1] = fixed + "\t" + fixed;
    r[on_i ? 1 : 0] = ang;
    r[2] = "1\t" + K;
    return r[0] + "\t" + r[1] + "\t" + r[2];
  };
  std::ostringstream in;
  in << "\t24\n\t4\t4\t4\t4\t4\t4\nimin\timax\tjmin\tjmax\tkmin\tkmax\tid\tPhysic_Name\n";
  // Each side of a connection must list, as its partner, exactly the range
  // line the partner lists for itself (src/1_grid/1_MPCNS_Grid.cpp:473-509
  // pairs patches by equal ranges); a reversed connection is therefore
  // written descending on the side with the larger (panel, edge) key.
  auto own_line = [&](int p, int e) {
    const Conn &c = conn[p][e];
    const bool upper = (p * 4 + e) > (c.q * 4 + c.f);
    return ranges(e, upper && c.reversed);
  };
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e) {
      const Conn &c = conn[p][e];
      in << own_line(p, e) << "\t" << (p + 1) << "\tFluid\n";
      in << own_line(c.q, c.f) << "\t" << (c.q + 1) << "\tFluid\n";
    }
  fs::create_directories(geo / "boundary_condition");
  write_text(geo / "boundary_condition" / "inner   0.txt", in.str());
  std::ostringstream bc;
  const std::string M = std::to_string(na), R = std::to_string(nr);
  for (int p = 0; p < 6; ++p) {
    bc << "\t2\n";
    bc << "0\t" << M << "\t0\t" << M << "\t0\t0\t17\n";
    bc << "0\t" << M << "\t0\t" << M << "\t" << R << "\t" << R << "\t4\n";
  }
  write_text(geo / "boundary_condition" / "boundary   0.txt", bc.str());
  std::string fv = kFvbnd;
  fv.replace(fv.find("BOUNDARIES"), 10, "Coupled-Solid\nBOUNDARIES");
  write_text(geo / "boundary_condition" / "boundary_name.fvbnd", fv);
  write_text(geo / "boundary_condition" / "parallel   0.txt",
             "\t6\t0\n\t0\t0\t0\t0\t0\t0\nimin\timax\tjmin\tjmax\tkmin\tkmax\ts_r_id\ts_flag\tr_flag\tPhysic_Name\n");
}

void write_case(const fs::path &work) {
  fs::create_directories(work / "CASE" / "setup");
  fs::create_directories(work / "CASE" / "geometry");
  write_text(work / "CASE/setup/filenames",
             "0_General_Setting.txt\n1_Initial_condition.txt\n2_Boundary_Condition.txt\n3_MHD_Control.txt\n###END###\n");
  write_text(work / "CASE/setup/0_General_Setting.txt", setup_general());
  write_text(work / "CASE/setup/1_Initial_condition.txt", setup_initial());
  write_text(work / "CASE/setup/2_Boundary_Condition.txt", setup_boundary());
  write_text(work / "CASE/setup/3_MHD_Control.txt", setup_mhd());
  const std::string kind = job_str("case", "cube");
  if (kind == "cube")
    write_cube_case(work / "CASE" / "geometry");
  else if (kind == "lattice")
    write_lattice_case(work / "CASE" / "geometry");
  else if (kind == "shell")
    write_shell_case(work / "CASE" / "geometry");
  else {
    std::fprintf(stderr, "unknown case %s\n", kind.c_str());
    std::exit(2);
  }
}

// ---------------------------------------------------------------- dumps
// Dump format (little endian): "MHDDUMP1", int32 nrec; per record:
//   int32 name_len, name bytes, int32 block, int32 lo[3], int32 hi[3], int32 ncomp,
//   then (hi-lo product)*ncomp doubles in the reference's (i,j,k,m) order.
struct Dumper {
  std::ofstream f;
  int32_t nrec = 0;
  std::streampos count_pos;
  explicit Dumper(const fs::path &p) : f(p, std::ios::binary) {
    f.write("MHDDUMP1", 8);
    count_pos = f.tellp();
    f.write((const char *)&nrec, 4);
  }
  void rec(const std::string &name, int block, const int lo[3], const int hi[3], int ncomp,
           const double *data) {
    int32_t len = (int32_t)name.size();
    f.write((const char *)&len, 4);
    f.write(name.data(), len);
    int32_t b = block;
    f.write((const char *)&b, 4);
    for (int a = 0; a < 3; ++a) {
      int32_t v = lo[a];
      f.write((const char *)&v, 4);
    }
    for (int a = 0; a < 3; ++a) {
      int32_t v = hi[a];
      f.write((const char *)&v, 4);
    }
    int32_t nc = ncomp;
    f.write((const char *)&nc, 4);
    size_t n = (size_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * ncomp;
    f.write((const char *)data, (std::streamsize)(n * sizeof(double)));
    ++nrec;
  }
  ~Dumper() {
    f.seekp(count_pos);
    f.write((const char *)&nrec, 4);
  }
};

void dump_field(Dumper &d, Field *fld, const std::string &name, const std::string &tag = "") {
  const int fid = fld->field_id(name);
  for (int ib = 0; ib < fld->num_blocks(); ++ib) {
    FieldBlock &F = fld->field(fid, ib);
    if (!F.is_allocated()) continue;
    const Int3 lo = F.get_lo(), hi = F.get_hi();
    const int l[3] = {lo.i, lo.j, lo.k}, h[3] = {hi.i, hi.j, hi.k};
    d.rec(tag + name, ib, l, h, fld->descriptor(fid).ncomp, F.raw_data().GetV3().data());
  }
}

void dump_grid(Dumper &d, Grid *grd) {
  for (int ib = 0; ib < grd->nblock; ++ib) {
    Block &b = grd->grids(ib);
    double3D *arrs[6] = {&b.x, &b.y, &b.z, &b.dual_x, &b.dual_y, &b.dual_z};
    const char *names[6] = {"node_x", "node_y", "node_z", "dual_x", "dual_y", "dual_z"};
    for (int a = 0; a < 6; ++a) {
      double3D &A = *arrs[a];
      const int g = A.Getghostmesh();
      const int l[3] = {-g, -g, -g};
      const int h[3] = {A.Getsize1() - g, A.Getsize2() - g, A.Getsize3() - g};
      d.rec(names[a], ib, l, h, 1, A.GetA3().data());
    }
  }
}

std::vector<std::string> split_ws(const std::string &s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

// ---------------------------------------------------------------- initial state
// Orszag-Tang vortex on both ion fluids (every block of the periodic box): rho = 1, p = 0.6,
// v = (-sin 2 pi y, sin 2 pi x, 0), B = curl A with
// A_z = (cos 4 pi x / (4 pi) + cos 2 pi y / (2 pi)) / sqrt(4 pi), i.e.
// B = (-sin 2 pi y, sin 4 pi x, 0) / sqrt(4 pi).  Multiplicative noise
// (1 + U[-a, a]) is applied to every conserved component and to every edge
// potential A.dr before the discrete curl, so div B starts at roundoff.
// Edge potentials live on the periodic index set [0, n) and are wrapped, so
// periodic alias faces receive identical fluxes.
void set_orszag_tang(MercurySolver &S) {
  Field *fld = S.fld_;
  Grid *grd = S.grd_;
  const double pi = std::acos(-1.0);
  const double gamma = S.gamma_;
  const double noise = job_dbl("noise", 1e-3);
  Uniform rng(20261203ull + (uint64_t)job_int("solve_id", 0));
  // cells per block and blocks per axis: one periodic block ("cube"), or the
  // "lattice" case's bx x by x bz blocks of equal size tiling the periodic box
  int nc[3], nb[3] = {1, 1, 1};
  cube_counts(nc);
  if (job_str("case", "cube") == "lattice") std::istringstream(job_str("nb", "2 2 2")) >> nb[0] >> nb[1] >> nb[2];
  const int n0 = nc[0], n1 = nc[1], n2 = nc[2];  // cells per direction of a block
  const int N0 = n0 * nb[0], N1 = n1 * nb[1], N2 = n2 * nb[2];
  auto bid = [&](int p, int q, int r) { return (p * nb[1] + q) * nb[2] + r; };
  for (int p = 0; p < nb[0]; ++p)
    for (int q = 0; q < nb[1]; ++q)
      for (int r = 0; r < nb[2]; ++r) {
        const int ib = bid(p, q, r);
        FieldBlock &UH = fld->field(S.fid_.fid_U_H, ib);
        FieldBlock &UN = fld->field(S.fid_.fid_U_Na, ib);
        Block &blk = grd->grids(ib);
        for (int i = 0; i < n0; ++i)
          for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k) {
              const double x = blk.dual_x(i + 1, j + 1, k + 1);
              const double y = blk.dual_y(i + 1, j + 1, k + 1);
              const double rho = 1.0, pr = 0.6;
              const double u = -std::sin(2.0 * pi * y), v = std::sin(2.0 * pi * x), w = 0.0;
              const double qv[5] = {rho, rho * u, rho * v, rho * w,
                                    pr / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)};
              for (FieldBlock *U : {&UH, &UN})
                for (int m = 0; m < 5; ++m) (*U)(i, j, k, m) = qv[m] * (1.0 + rng.sym(noise));
            }
      }
  // Edge potentials A_z * dz on the periodic edge set of the whole box
  // (global indices I = p * n0 + i, ...), each evaluated on the block that
  // holds the edge's lower node.
  auto Az = [&](double x, double y) {
    return (std::cos(4.0 * pi * x) / (4.0 * pi) + std::cos(2.0 * pi * y) / (2.0 * pi)) /
           std::sqrt(4.0 * pi);
  };
  std::vector<double> ax((size_t)N0 * N1 * N2), ay(ax.size()), az(ax.size());
  auto idx = [&](int i, int j, int k) { return ((size_t)i * N1 + j) * N2 + k; };
  auto edge_val = [&](int I, int J, int K, int di, int dj, int dk) {
    Block &blk = grd->grids(bid(I / n0, J / n1, K / n2));
    const int i0 = I % n0, j0 = J % n1, k0 = K % n2, i1 = i0 + di, j1 = j0 + dj, k1 = k0 + dk;
    const double xa = blk.x(i0, j0, k0), ya = blk.y(i0, j0, k0), za = blk.z(i0, j0, k0);
    const double xb = blk.x(i1, j1, k1), yb = blk.y(i1, j1, k1), zb = blk.z(i1, j1, k1);
    return Az(0.5 * (xa + xb), 0.5 * (ya + yb)) * (zb - za);
  };
  for (int i = 0; i < N0; ++i)
    for (int j = 0; j < N1; ++j)
      for (int k = 0; k < N2; ++k) ax[idx(i, j, k)] = edge_val(i, j, k, 1, 0, 0) * (1.0 + rng.sym(noise));
  for (int i = 0; i < N0; ++i)
    for (int j = 0; j < N1; ++j)
      for (int k = 0; k < N2; ++k) ay[idx(i, j, k)] = edge_val(i, j, k, 0, 1, 0) * (1.0 + rng.sym(noise));
  for (int i = 0; i < N0; ++i)
    for (int j = 0; j < N1; ++j)
      for (int k = 0; k < N2; ++k) az[idx(i, j, k)] = edge_val(i, j, k, 0, 0, 1) * (1.0 + rng.sym(noise));
  auto wi = [&](int a) { return ((a % N0) + N0) % N0; };
  auto wj = [&](int a) { return ((a % N1) + N1) % N1; };
  auto wk = [&](int a) { return ((a % N2) + N2) % N2; };
  // Face fluxes = discrete curl of the edge potential, same stencil as the
  // reference's CurlEdgeToFace (Z4_Mercury/src/operators/CTOperators.cpp:6-56)
  // with multiplier +1; block faces on a shared boundary get identical values.
  for (int p = 0; p < nb[0]; ++p)
    for (int q = 0; q < nb[1]; ++q)
      for (int r = 0; r < nb[2]; ++r) {
        const int ib = bid(p, q, r);
        const int I0 = p * n0, J0 = q * n1, K0 = r * n2;
        auto EX = [&](int i, int j, int k) { return ax[idx(wi(I0 + i), wj(J0 + j), wk(K0 + k))]; };
        auto EY = [&](int i, int j, int k) { return ay[idx(wi(I0 + i), wj(J0 + j), wk(K0 + k))]; };
        auto EZ = [&](int i, int j, int k) { return az[idx(wi(I0 + i), wj(J0 + j), wk(K0 + k))]; };
        FieldBlock &Bx = fld->field(S.fid_.fid_B.xi, ib);
        FieldBlock &By = fld->field(S.fid_.fid_B.eta, ib);
        FieldBlock &Bz = fld->field(S.fid_.fid_B.zeta, ib);
        for (int i = 0; i <= n0; ++i)
          for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k)
              Bx(i, j, k, 0) = (EY(i, j, k) - EY(i, j, k + 1)) + (EZ(i, j + 1, k) - EZ(i, j, k));
        for (int i = 0; i < n0; ++i)
          for (int j = 0; j <= n1; ++j)
            for (int k = 0; k < n2; ++k)
              By(i, j, k, 0) = (EX(i, j, k + 1) - EX(i, j, k)) + (EZ(i, j, k) - EZ(i + 1, j, k));
        for (int i = 0; i < n0; ++i)
          for (int j = 0; j < n1; ++j)
            for (int k = 0; k <= n2; ++k)
              Bz(i, j, k, 0) = (EX(i, j, k) - EX(i, j + 1, k)) + (EY(i + 1, j, k) - EY(i, j, k));
      }
}

// Magnetosphere start: the reference's uniform solar wind (Common_Initial,
// Z4_Mercury/include/2_Initial.h:134-215) for H+, and Na+ at a number-density
// fraction f of it with the same velocity and temperature:
// rho_Na = f (M_Na / M_H) rho_H, p_Na = f p_H, on every allocated cell.
void set_na_fraction(MercurySolver &S) {
  Field *fld = S.fld_;
  const double f = job_dbl("na_fraction", 1e-3);
  const double g = S.gamma_;
  for (int ib = 0; ib < fld->num_blocks(); ++ib) {
    FieldBlock &UH = fld->field(S.fid_.fid_U_H, ib);
    FieldBlock &UN = fld->field(S.fid_.fid_U_Na, ib);
    const Int3 lo = UH.get_lo(), hi = UH.get_hi();
    for (int i = lo.i; i < hi.i; ++i)
      for (int j = lo.j; j < hi.j; ++j)
        for (int k = lo.k; k < hi.k; ++k) {
          const double rho = UH(i, j, k, 0);
          const double u = UH(i, j, k, 1) / rho, v = UH(i, j, k, 2) / rho, w = UH(i, j, k, 3) / rho;
          const double p = (g - 1.0) * (UH(i, j, k, 4) - 0.5 * rho * (u * u + v * v + w * w));
          const double rn = f * (S.M_Na / S.M_H) * rho, pn = f * p;
          UN(i, j, k, 0) = rn;
          UN(i, j, k, 1) = rn * u;
          UN(i, j, k, 2) = rn * v;
          UN(i, j, k, 3) = rn * w;
          UN(i, j, k, 4) = pn / (g - 1.0) + 0.5 * rn * (u * u + v * v + w * w);
        }
  }
}

// ---------------------------------------------------------------- sync probe
// Unique-code probe of one sync group, following the reference's own halo
// test method (Z0_NULL/test/halo_comm/Z0_HaloCommTest.cpp:361-398): every
// allocated DOF of every field of the group gets a distinct integer code
// (owned DOFs) or NaN (ghost DOFs), the group is synchronised, and the dump
// shows for every DOF which code (and sign) landed there.
void probe_group(MercurySolver &S, const std::string &group, Dumper &d) {
  Field *fld = S.fld_;
  std::vector<std::string> names = split_ws(job_str("probe_fields"));
  double code = 1.0;
  for (auto &name : names) {
    const int fid = fld->field_id(name);
    for (int ib = 0; ib < fld->num_blocks(); ++ib) {
      FieldBlock &F = fld->field(fid, ib);
      if (!F.is_allocated()) continue;
      const Int3 lo = F.get_lo(), hi = F.get_hi(), ilo = F.inner_lo(), ihi = F.inner_hi();
      const int nc = fld->descriptor(fid).ncomp;
      for (int i = lo.i; i < hi.i; ++i)
        for (int j = lo.j; j < hi.j; ++j)
          for (int k = lo.k; k < hi.k; ++k)
            for (int m = 0; m < nc; ++m) {
              const bool owned = i >= ilo.i && i < ihi.i && j >= ilo.j && j < ihi.j && k >= ilo.k && k < ihi.k;
              F(i, j, k, m) = owned ? code : std::nan("");
              code += 1.0;
            }
    }
  }
  for (auto &name : names) dump_field(d, fld, name, "before:");
  S.mercury_bound_.Sync(group);
  for (auto &name : names) dump_field(d, fld, name, "after:");
}

// Hall radial taper per edge, evaluated by the reference's own
// HallRadialTaperEdge_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:16-25)
// on the owned edges (the range BuildHallFaceEMF_Rusanov_diff_ uses), zero elsewhere.
void dump_taper(MercurySolver &S, Dumper &d) {
  Field *fld = S.fld_;
  const int fids[3] = {S.fid_.fid_Ehall.xi, S.fid_.fid_Ehall.eta, S.fid_.fid_Ehall.zeta};
  const StaggerLocation locs[3] = {StaggerLocation::EdgeXi, StaggerLocation::EdgeEt, StaggerLocation::EdgeZe};
  const char *names[3] = {"taper_xi", "taper_eta", "taper_zeta"};
  for (int a = 0; a < 3; ++a)
    for (int ib = 0; ib < fld->num_blocks(); ++ib) {
      FieldBlock &E = fld->field(fids[a], ib);
      const Int3 lo = E.get_lo(), hi = E.get_hi(), ilo = E.inner_lo(), ihi = E.inner_hi();
      const int ni = hi.i - lo.i, nj = hi.j - lo.j, nk = hi.k - lo.k;
      std::vector<double> t((size_t)ni * nj * nk, 0.0);
      for (int i = ilo.i; i < ihi.i; ++i)
        for (int j = ilo.j; j < ihi.j; ++j)
          for (int k = ilo.k; k < ihi.k; ++k)
            t[((size_t)(i - lo.i) * nj + (j - lo.j)) * nk + (k - lo.k)] = S.HallRadialTaperEdge_(ib, locs[a], i, j, k);
      const int l[3] = {lo.i, lo.j, lo.k}, h[3] = {hi.i, hi.j, hi.k};
      d.rec(std::string("static:") + names[a], ib, l, h, 1, t.data());
    }
  // and at the owned cell centres (HallRadialTaper_ of the singular-edge Hall
  // EMF, Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:51), zero elsewhere
  for (int ib = 0; ib < fld->num_blocks(); ++ib) {
    FieldBlock &U = fld->field(S.fid_.fid_U_H, ib);
    Block &blk = S.grd_->grids(ib);
    const Int3 lo = U.get_lo(), hi = U.get_hi(), ilo = U.inner_lo(), ihi = U.inner_hi();
    const int ni = hi.i - lo.i, nj = hi.j - lo.j, nk = hi.k - lo.k;
    std::vector<double> t((size_t)ni * nj * nk, 0.0);
    for (int i = ilo.i; i < ihi.i; ++i)
      for (int j = ilo.j; j < ihi.j; ++j)
        for (int k = ilo.k; k < ihi.k; ++k)
          t[((size_t)(i - lo.i) * nj + (j - lo.j)) * nk + (k - lo.k)] =
              S.HallRadialTaper_(blk.dual_x(i + 1, j + 1, k + 1), blk.dual_y(i + 1, j + 1, k + 1),
                                 blk.dual_z(i + 1, j + 1, k + 1));
    const int l[3] = {lo.i, lo.j, lo.k}, h[3] = {hi.i, hi.j, hi.k};
    d.rec("static:taper_cell", ib, l, h, 1, t.data());
  }
}

// Local artificial resistivity per edge as the reference fills it on its first
// use (AddLocalArtificialResistivityToEdgeEMF_,
// Z4_Mercury/src/physics/MercurySolver_MagExplicit_Resis.cpp:117-158): the harness triggers that fill
// once before stepping (the E field is zeroed at the start of every step, so
// the extra contribution is discarded) and dumps the arrays over the E box.
void dump_local_eta(MercurySolver &S, Dumper &d) {
  S.AddLocalArtificialResistivityToEdgeEMF_();
  Field *fld = S.fld_;
  const int fids[3] = {S.fid_.fid_E.xi, S.fid_.fid_E.eta, S.fid_.fid_E.zeta};
  const char *names[3] = {"local_arti_eta_xi", "local_arti_eta_eta", "local_arti_eta_zeta"};
  for (int a = 0; a < 3; ++a)
    for (int ib = 0; ib < fld->num_blocks(); ++ib) {
      FieldBlock &E = fld->field(fids[a], ib);
      auto &eta = a == 0 ? S.local_arti_eta_xi_[ib] : a == 1 ? S.local_arti_eta_eta_[ib] : S.local_arti_eta_ze_[ib];
      const Int3 lo = E.get_lo(), hi = E.get_hi();
      const int ni = hi.i - lo.i, nj = hi.j - lo.j, nk = hi.k - lo.k;
      std::vector<double> t((size_t)ni * nj * nk, 0.0);
      for (int i = lo.i; i < hi.i; ++i)
        for (int j = lo.j; j < hi.j; ++j)
          for (int k = lo.k; k < hi.k; ++k) t[((size_t)(i - lo.i) * nj + (j - lo.j)) * nk + (k - lo.k)] = eta(i, j, k);
      const int l[3] = {lo.i, lo.j, lo.k}, h[3] = {hi.i, hi.j, hi.k};
      d.rec(std::string("static:") + names[a], ib, l, h, 1, t.data());
    }
}

// Implicit-resistivity coefficient per edge as the reference evaluates it for
// its unknowns (ImplicitResistiveEtaAtEdge_,
// Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:228-258) on every edge of the owned
// range, zero elsewhere.
void dump_eta_res(MercurySolver &S, Dumper &d) {
  Field *fld = S.fld_;
  const int fids[3] = {S.fid_.fid_Eres.xi, S.fid_.fid_Eres.eta, S.fid_.fid_Eres.zeta};
  const TOPO::EntityAxis axes[3] = {TOPO::EntityAxis::Xi, TOPO::EntityAxis::Eta, TOPO::EntityAxis::Zeta};
  const char *names[3] = {"eta_res_xi", "eta_res_eta", "eta_res_zeta"};
  for (int a = 0; a < 3; ++a)
    for (int ib = 0; ib < fld->num_blocks(); ++ib) {
      FieldBlock &E = fld->field(fids[a], ib);
      const Int3 lo = E.get_lo(), hi = E.get_hi(), ilo = E.inner_lo(), ihi = E.inner_hi();
      const int ni = hi.i - lo.i, nj = hi.j - lo.j, nk = hi.k - lo.k;
      std::vector<double> t((size_t)ni * nj * nk, 0.0);
      for (int i = ilo.i; i < ihi.i; ++i)
        for (int j = ilo.j; j < ihi.j; ++j)
          for (int k = ilo.k; k < ihi.k; ++k)
            t[((size_t)(i - lo.i) * nj + (j - lo.j)) * nk + (k - lo.k)] =
                S.ImplicitResistiveEtaAtEdge_(TOPO::make_edge(0, ib, i, j, k, axes[a]));
      const int l[3] = {lo.i, lo.j, lo.k}, h[3] = {hi.i, hi.j, hi.k};
      d.rec(std::string("static:") + names[a], ib, l, h, 1, t.data());
    }
}

// Edge alias classes exactly as ReduceEdgeAliasCandidatesToOwners_ consumes
// them (Z4_Mercury/src/physics/MercurySolver_Current.cpp:8-35): classes with a
// global id and more than one member, sorted by global id; per class the owner
// and the members in their stored order.  Record layout (int32 each):
//   [global_id, nmem, owner_axis, oi, oj, ok, owner_sign, (axis, i, j, k, sign) * nmem]
void dump_edge_classes(TOPO::Topology &topo, Dumper &d) {
  std::vector<const TOPO::EquivClass *> cls;
  for (const auto &c : topo.edges.classes)
    if (c.global_id >= 0 && c.members.size() > 1) cls.push_back(&c);
  std::sort(cls.begin(), cls.end(), [](const auto *a, const auto *b) { return a->global_id < b->global_id; });
  std::vector<double> buf;
  for (const auto *c : cls) {
    buf.push_back(c->global_id);
    buf.push_back((double)c->members.size());
    const auto &o = c->owner;
    buf.push_back((int)o.entity.axis);
    buf.push_back(o.entity.i);
    buf.push_back(o.entity.j);
    buf.push_back(o.entity.k);
    buf.push_back(o.orient_sign);
    buf.push_back(o.entity.block);
    for (const auto &m : c->members) {
      buf.push_back((int)m.entity.axis);
      buf.push_back(m.entity.i);
      buf.push_back(m.entity.j);
      buf.push_back(m.entity.k);
      buf.push_back(m.orient_sign);
      buf.push_back(m.entity.block);
    }
  }
  const int l[3] = {0, 0, 0}, h[3] = {(int)buf.size(), 1, 1};
  d.rec("edge_alias_classes", -1, l, h, 1, buf.data());
}

// The reference's topology patch lists (TOPO::Topology, built by
// TOPO::build_topology, src/2_topology/TopologyBuilder.cpp:436) as int32
// records, so that a multi-block table builder can be pinned patch for patch:
//   record "topo_faces":    per inner patch  this_block nb_block direction nb_direction
//                           this_box_node lo[3] hi[3]  nb_box_node lo[3] hi[3]  perm[3] sign[3] offset[3]
//   record "topo_edges":    per inner edge patch  this_block nb_block dir1 dir2 this lo/hi nb lo/hi perm sign offset
//   record "topo_vertices": per inner vertex patch  this_block nb_block dir1 dir2 dir3 this lo/hi nb lo/hi perm sign offset
//   record "topo_physical": per physical patch  this_block direction bc_id this lo/hi
//   record "topo_phys_edges" / "topo_phys_vertices": physical edge / vertex patches (block dir1 dir2 [dir3] lo/hi)
void dump_topology(TOPO::Topology &t, Dumper &d) {
  auto box = [](std::vector<double> &b, const Box3 &x) {
    for (int v : {x.lo.i, x.lo.j, x.lo.k, x.hi.i, x.hi.j, x.hi.k}) b.push_back(v);
  };
  auto tr = [](std::vector<double> &b, const TOPO::IndexTransform &x) {
    for (int a = 0; a < 3; ++a) b.push_back(x.perm[a]);
    for (int a = 0; a < 3; ++a) b.push_back(x.sign[a]);
    for (int v : {x.offset.i, x.offset.j, x.offset.k}) b.push_back(v);
  };
  auto emit = [&](const char *name, std::vector<double> &b) {
    if (b.empty()) b.push_back(-1.0);
    const int l[3] = {0, 0, 0}, h[3] = {(int)b.size(), 1, 1};
    d.rec(name, -1, l, h, 1, b.data());
  };
  std::vector<double> f, e, v, p, pe, pv;
  for (const auto &x : t.inner_patches) {
    for (int q : {x.this_block, x.nb_block, x.direction, x.nb_direction, (int)x.is_coupling}) f.push_back(q);
    box(f, x.this_box_node);
    box(f, x.nb_box_node);
    tr(f, x.trans);
  }
  for (const auto &x : t.inner_edge_patches) {
    for (int q : {x.this_block, x.nb_block, x.dir1, x.dir2, (int)x.is_coupling}) e.push_back(q);
    box(e, x.this_box_node);
    box(e, x.nb_box_node);
    tr(e, x.trans);
  }
  for (const auto &x : t.inner_vertex_patches) {
    for (int q : {x.this_block, x.nb_block, x.dir1, x.dir2, x.dir3, (int)x.is_coupling}) v.push_back(q);
    box(v, x.this_box_node);
    box(v, x.nb_box_node);
    tr(v, x.trans);
  }
  for (const auto &x : t.physical_patches) {
    for (int q : {x.this_block, x.direction, x.bc_id}) p.push_back(q);
    box(p, x.this_box_node);
  }
  for (const auto &x : t.physical_edge_patches) {
    for (int q : {x.this_block, x.dir1, x.dir2}) pe.push_back(q);
    box(pe, x.this_box_node);
  }
  for (const auto &x : t.physical_vertex_patches) {
    for (int q : {x.this_block, x.dir1, x.dir2, x.dir3}) pv.push_back(q);
    box(pv, x.this_box_node);
  }
  emit("topo_faces", f);
  emit("topo_edges", e);
  emit("topo_vertices", v);
  emit("topo_physical", p);
  emit("topo_phys_edges", pe);
  emit("topo_phys_vertices", pv);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <job-file>\n", argv[0]);
    return 2;
  }
  {
    std::ifstream jf(argv[1]);
    std::string line;
    while (std::getline(jf, line)) {
      auto sp = line.find(' ');
      if (line.empty() || line[0] == '#' || sp == std::string::npos) continue;
      g_job[line.substr(0, sp)] = line.substr(sp + 1);
    }
  }
  const fs::path out = fs::absolute(job_str("out", "oracle_dump.bin"));
  const fs::path work = fs::absolute(job_str("workdir", "oracle_work"));
  fs::create_directories(work);
  write_case(work);
  fs::current_path(work);

  int myid = 0;
  PARALLEL::mpi_initial(argc, argv);
  PARALLEL::mpi_rank(&myid);
  PetscInitialize(&argc, &argv, NULL, NULL);
  if (job_int("ksp_force", 0)) oracle_ksp_force_tolerances(job_dbl("ksp_rtol", 1e-13), job_dbl("ksp_atol", 0.0), (int)job_int("ksp_max_it", 200));

  Param *par = new Param;
  par->ReadParam(myid);
  Grid *grd = new Grid;
  grd->Grid_Preprocess(par);
  TOPO::Topology topology = TOPO::build_topology(*grd, myid, par->GetInt("dimension"));
  const int ngg = par->GetInt("ngg");
  Field *fld = new Field(grd, par, ngg);
  MercurySolver::RegisterFields(fld, ngg);
  MercurySolver::RegisterCouplingChannels(fld, topology, par->GetInt("dimension"), ngg);
  METRIC::SingularEdgeRegistry singular_edges;
  singular_edges.build(topology, *fld, *grd, myid);
  singular_edges.validate_or_abort();
  Halo *hal = new Halo(fld, &topology);
  hal->set_topology_equiv(&topology);
  MercurySolver::RegisterHaloFields(fld, hal);
  HALO_OWNER::EdgeOwnerSyncPattern edge_owner_pat;
  HALO_OWNER::build_edge_owner_sync_pattern(topology, edge_owner_pat);
  {
    MercurySolver S(grd, &topology, fld, hal, par, &topology, &edge_owner_pat, &singular_edges);
    Dumper d(out);
    const std::string mode = job_str("mode", "run");
    if (mode == "probe") {
      if (job_int("dump_grid", 0)) dump_grid(d, grd);
      probe_group(S, job_str("probe_group"), d);
    } else if (mode == "classes") {
      dump_edge_classes(topology, d);
    } else if (mode == "topology") {
      dump_topology(topology, d);
      dump_edge_classes(topology, d);
    } else {
      const std::string init = job_str("init", "ot");
      if (init == "ot") set_orszag_tang(S);
      if (init == "na_fraction") set_na_fraction(S);
      if (!job_str("read_restart").empty()) {
        // resume the state from a restart file through the reference's own
        // reader (IOModule::ReadRestartBinFile, src/6_io/IOModule_Bin.cpp:234-420)
        S.io_.Change_RestartPath(job_str("read_restart"));
        S.io_.ReadRestartBinFile();
      }
      S.mercury_bound_.Sync("Ucell");
      S.mercury_bound_.Sync("Bface");
      // Advance() begins with UpdateDerivedFields_ and the step-0 control
      // update (Z4_Mercury/src/MercurySolver_Driver.cpp:6-13).
      S.UpdateDerivedFields_();
      S.control_.UpdateSwitches(*S.run_data_);
      const auto static_fields = split_ws(job_str("dump_static"));
      for (auto &name : static_fields) dump_field(d, fld, name, "static:");
      if (job_int("dump_grid", 0)) dump_grid(d, grd);
      if (job_int("dump_taper", 0)) dump_taper(S, d);
      if (job_int("local_arti", 0)) dump_local_eta(S, d);
      if (job_int("resistive", 0)) dump_eta_res(S, d);
      const auto state_fields = split_ws(job_str("dump_fields", "U_H U_Na B_xi B_eta B_zeta"));
      const long steps = job_int("steps", 1);
      std::vector<long> at;
      for (auto &s : split_ws(job_str("dump_at", "0 " + std::to_string(steps)))) at.push_back(std::stol(s));
      auto dump_state = [&](long step) {
        for (long a : at)
          if (a == step) {
            const std::string tag = "step" + std::to_string(step) + ":";
            if (job_int("calc_divb", 0)) S.calc_divB();  // the reference's output-step diagnostic
            for (auto &name : state_fields) dump_field(d, fld, name, tag);
            const double meta[2] = {S.dt, S.run_data_->time};
            const int l[3] = {0, 0, 0}, h[3] = {1, 1, 2};
            d.rec(tag + "dt_time", -1, l, h, 1, meta);
          }
      };
      dump_state(0);
      // wall time of the StepOnce calls after the first time_from (warm-up) steps
      const long time_from = job_int("time_from", 0);
      double stepping = 0.0;
      for (long s = 1; s <= steps; ++s) {
        const auto t0 = std::chrono::steady_clock::now();
        S.StepOnce();
        if (s > time_from) stepping += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        dump_state(s);
      }
      if (!job_str("write_restart").empty()) {
        // the reference's own restart writer (IOModule::WriteRestartBinFile,
        // src/6_io/IOModule_Bin.cpp:168-232), with the step count and time of
        // this run
        S.io_.Change_RestartPath(job_str("write_restart"));
        S.io_.WriteRestartBinFile((int)(job_int("restart_step0", 0) + steps), S.run_data_->time);
      }
      if (!job_str("write_rundata").empty()) {
        // the reference's run-data file (IOModule::WriteRunDataFile), from its
        // default ./DATA/RunData.bin
        fs::create_directories("DATA");
        S.io_.WriteRunDataFile();
        fs::copy_file("DATA/RunData.bin", job_str("write_rundata"), fs::copy_options::overwrite_existing);
      }
      if (!job_str("write_tecplot").empty()) {
        // the reference's own checkpoint plot file (IOModule::WriteTecplotBinFile,
        // src/6_io/IOModule_Tecplot.cpp:749-1017, in the AllNode mode and with
        // the variables MercurySolver's constructor selects), written to its
        // default ./DATA/ path and copied to the requested one
        fs::create_directories("DATA");
        S.io_.WriteTecplotBinFile((int)steps, S.run_data_->time);
        for (const auto &e : fs::directory_iterator("DATA"))
          if (e.path().extension() == ".plt")
            fs::copy_file(e.path(), job_str("write_tecplot"), fs::copy_options::overwrite_existing);
      }
      {
        // wall time of the StepOnce calls alone (setup and dumps excluded)
        long cells = 0;
        for (int ib = 0; ib < fld->num_blocks(); ++ib) {
          FieldBlock &U = fld->field(S.fid_.fid_U_H, ib);
          if (!U.is_allocated()) continue;
          const Int3 h = U.inner_hi();
          cells += (long)h.i * h.j * h.k;
        }
        const double meta[3] = {stepping, (double)(steps - std::min(steps, time_from)), (double)cells};
        const int l[3] = {0, 0, 0}, h[3] = {1, 1, 3};
        d.rec("timing", -1, l, h, 1, meta);
      }
    }
  }
  delete hal;
  delete fld;
  delete par;
  delete grd;
  PetscFinalize();
  PARALLEL::mpi_finalize();
  return 0;
}
