// FP64 kernels of the explicit multi-fluid Hall-MHD step on sm_100a.
//
// Each kernel restates one pass of the reference step in the reference's own
// operation order (the build disables FMA contraction), so that the FP64 path
// reproduces the reference to roundoff.  The stencils are HBM-bound: they read
// a neighbourhood of state, derived and static fields and write one result per
// DOF; threads map (k, j, i) -> (x, y, z) so that warps read contiguous k rows.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "mhd_layout.cuh"
#include "mhd_step.cuh"

namespace mhd {

namespace {

// Component indices (global numbering) used by the kernels.
constexpr int cUH = 0, cUN = 5;
constexpr int cBX = kComp.first[MHD_B_XI], cBY = kComp.first[MHD_B_ETA], cBZ = kComp.first[MHD_B_ZETA];
constexpr int cPVH = kComp.first[MHD_PV_H], cPVN = kComp.first[MHD_PV_NA], cUP = kComp.first[MHD_U_PLUS];
constexpr int cBC = kComp.first[MHD_B_CELL], cBIC = kComp.first[MHD_BIND_CELL], cJC = kComp.first[MHD_J_CELL];
constexpr int cJX = kComp.first[MHD_J_XI], cJY = kComp.first[MHD_J_ETA], cJZ = kComp.first[MHD_J_ZETA];
constexpr int cEX = kComp.first[MHD_E_XI], cEY = kComp.first[MHD_E_ETA], cEZ = kComp.first[MHD_E_ZETA];
constexpr int cHX = kComp.first[MHD_EHALL_XI], cHY = kComp.first[MHD_EHALL_ETA], cHZ = kComp.first[MHD_EHALL_ZETA];
constexpr int cEFX = kComp.first[MHD_EFACE_XI], cEFY = kComp.first[MHD_EFACE_ETA], cEFZ = kComp.first[MHD_EFACE_ZETA];
constexpr int cEHC = kComp.first[MHD_EHC], cHB = kComp.first[MHD_HALL_BETA];
constexpr int cJAC = kComp.first[MHD_JAC], cJDX = kComp.first[MHD_JDXI], cJDY = kComp.first[MHD_JDET],
              cJDZ = kComp.first[MHD_JDZE];
constexpr int cAX = kComp.first[MHD_AREA_XI], cAY = kComp.first[MHD_AREA_ETA], cAZ = kComp.first[MHD_AREA_ZETA];
constexpr int cDLX = kComp.first[MHD_DL_XI], cDLY = kComp.first[MHD_DL_ETA], cDLZ = kComp.first[MHD_DL_ZETA];
constexpr int cDRX = kComp.first[MHD_DR_XI], cDRY = kComp.first[MHD_DR_ETA], cDRZ = kComp.first[MHD_DR_ZETA];
constexpr int cBFX = kComp.first[MHD_HODGE_FACE_XI], cBFY = kComp.first[MHD_HODGE_FACE_ETA],
              cBFZ = kComp.first[MHD_HODGE_FACE_ZETA];
constexpr int cALX = kComp.first[MHD_HODGE_EDGE_XI], cALY = kComp.first[MHD_HODGE_EDGE_ETA],
              cALZ = kComp.first[MHD_HODGE_EDGE_ZETA];
constexpr int cWB = kComp.first[MHD_BCELL_W], cWJ = kComp.first[MHD_JCELL_W];
constexpr int cBAX = kComp.first[MHD_BADD_XI], cBAY = kComp.first[MHD_BADD_ETA], cBAZ = kComp.first[MHD_BADD_ZETA];
constexpr int cPHOTO = kComp.first[MHD_PHOTO], cCX = kComp.first[MHD_CELL_X], cCY = kComp.first[MHD_CELL_Y],
              cCZ = kComp.first[MHD_CELL_Z];
constexpr int cTPX = kComp.first[MHD_TAPER_XI], cTPY = kComp.first[MHD_TAPER_ETA], cTPZ = kComp.first[MHD_TAPER_ZETA];

// std::max / std::min semantics (first argument wins ties, incl. signed zeros).
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

struct Num {
  double nH, nNa, ne_eff, chiH, chiNa, wH, wNa;
};

// Hall_Num_Limiter (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:111-157)
__device__ __forceinline__ Num num_limiter(const Consts &c, double rhoH, double rhoNa) {
  Num d;
  const double rH = dmax(rhoH, 0.0), rN = dmax(rhoNa, 0.0);
  d.nH = rH / c.M_H * c.M_ref;
  d.nNa = rN / c.M_Na * c.M_ref;
  const double ne_true = d.nH + d.nNa;
  d.ne_eff = sqrt(ne_true * ne_true + c.ne_hall_floor * c.ne_hall_floor);
  if (ne_true > 1.0e-300) {
    d.chiH = d.nH / ne_true;
    d.chiNa = d.nNa / ne_true;
  } else {
    d.chiH = 1.0;
    d.chiNa = 0.0;
  }
  d.wH = d.nH / d.ne_eff;
  d.wNa = d.nNa / d.ne_eff;
  return d;
}

struct Idx {
  int i, j, k;
};

// Thread -> logical index over [lo, hi) per axis (x -> k, y -> j, z -> i).
__device__ __forceinline__ bool thread_index(const int lo[3], const int hi[3], Idx &p) {
  p.k = lo[2] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  p.j = lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  p.i = lo[0] + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  return p.i < hi[0] && p.j < hi[1] && p.k < hi[2];
}

#define AT(c, i, j, k) (B.comp(c)[B.off((i), (j), (k))])

// ------------------------------------------------------------------ timestep
// Compute_Timestep (Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:8-141):
// dt = CFL * V / sum_faces (|u_n| + c_f) |A| over both species; the global
// minimum is a warp-shuffle + CTA reduction and one atomicMin per CTA on the
// bit pattern (dt > 0, so the unsigned order is the numeric order).
__device__ __forceinline__ double fast_cf(double cs2, double vA2, double vAn2) {
  const double term = cs2 + vA2;
  double disc = term * term - 4.0 * cs2 * vAn2;
  if (disc < 0.0) disc = 0.0;
  return sqrt(0.5 * (term + sqrt(disc)));
}
__device__ __forceinline__ double face_term(const Consts &c, double ax, double ay, double az, bool outward_plus, double ux,
                                            double uy, double uz, double Bx, double By, double Bz, double B2, double rho,
                                            double cs2) {
  const double An = sqrt(ax * ax + ay * ay + az * az);
  if (An <= 0.0) return 0.0;
  double nx = ax / An, ny = ay / An, nz = az / An;
  if (!outward_plus) {
    nx = -nx;
    ny = -ny;
    nz = -nz;
  }
  const double un = ux * nx + uy * ny + uz * nz;
  const double Bn = Bx * nx + By * ny + Bz * nz;
  const double vA2 = c.inver_MA2 * B2 / rho;
  const double vAn2 = c.inver_MA2 * (Bn * Bn) / rho;
  return (fabs(un) + fast_cf(cs2, vA2, vAn2)) * An;
}

__global__ void k_timestep(BlockView B, Consts c, Scalars *S) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  Idx p;
  double dtl = 1e100;
  if (thread_index(lo, hi, p)) {
    const int i = p.i, j = p.j, k = p.k;
    const double Vol = fabs(AT(cJAC, i, j, k));
    if (Vol > 0.0) {
      const double Bx = AT(cBC, i, j, k), By = AT(cBC + 1, i, j, k), Bz = AT(cBC + 2, i, j, k);
      const double B2 = Bx * Bx + By * By + Bz * Bz;
      const double a0[3] = {AT(cJDX, i, j, k), AT(cJDX + 1, i, j, k), AT(cJDX + 2, i, j, k)};
      const double a1[3] = {AT(cJDX, i + 1, j, k), AT(cJDX + 1, i + 1, j, k), AT(cJDX + 2, i + 1, j, k)};
      const double b0[3] = {AT(cJDY, i, j, k), AT(cJDY + 1, i, j, k), AT(cJDY + 2, i, j, k)};
      const double b1[3] = {AT(cJDY, i, j + 1, k), AT(cJDY + 1, i, j + 1, k), AT(cJDY + 2, i, j + 1, k)};
      const double c0[3] = {AT(cJDZ, i, j, k), AT(cJDZ + 1, i, j, k), AT(cJDZ + 2, i, j, k)};
      const double c1[3] = {AT(cJDZ, i, j, k + 1), AT(cJDZ + 1, i, j, k + 1), AT(cJDZ + 2, i, j, k + 1)};
      for (int s = 0; s < 2; ++s) {
        const int u0 = s ? cUN : cUH;
        const double rho = dmax(AT(u0, i, j, k), 1e-2);
        const double ux = AT(u0 + 1, i, j, k) / rho, uy = AT(u0 + 2, i, j, k) / rho, uz = AT(u0 + 3, i, j, k) / rho;
        const double E = AT(u0 + 4, i, j, k);
        const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
        const double pr = (c.gamma - 1.0) * (E - ke);
        const double cs2 = c.gamma * pr / rho;
        double den = 0.0;
        den += face_term(c, a0[0], a0[1], a0[2], false, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        den += face_term(c, a1[0], a1[1], a1[2], true, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        den += face_term(c, b0[0], b0[1], b0[2], false, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        den += face_term(c, b1[0], b1[1], b1[2], true, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        den += face_term(c, c0[0], c0[1], c0[2], false, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        den += face_term(c, c1[0], c1[1], c1[2], true, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
        if (den > 0.0) dtl = dmin(dtl, c.CFL * Vol / den);
      }
    }
  }
  // warp + CTA min
  for (int o = 16; o > 0; o >>= 1) dtl = dmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
  __shared__ double red[32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  if ((tid & 31) == 0) red[tid >> 5] = dtl;
  __syncthreads();
  if (tid < 32) {
    double v = tid < (nthr + 31) / 32 ? red[tid] : 1e100;
    for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tid == 0) atomicMin(&S->dt_bits, (unsigned long long)__double_as_longlong(v));
  }
}

// ------------------------------------------------------------------ ideal EMF
// AssembleOneDirectionEMF_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ideal.cpp:433-594)
__device__ __forceinline__ void shift1(int axis, int &i, int &j, int &k, int s) {
  if (axis == 0) i += s;
  else if (axis == 1) j += s;
  else k += s;
}
__device__ __forceinline__ double cell_u_contra(const BlockView &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  const int cm = axis == 0 ? cJDX : axis == 1 ? cJDY : cJDZ;
  const double kx = 0.5 * (AT(cm, i, j, k) + AT(cm, ip, jp, kp));
  const double ky = 0.5 * (AT(cm + 1, i, j, k) + AT(cm + 1, ip, jp, kp));
  const double kz = 0.5 * (AT(cm + 2, i, j, k) + AT(cm + 2, ip, jp, kp));
  const double inv_jac = 1.0 / (fabs(AT(cJAC, i, j, k)) + 1.0e-30);
  return (kx * AT(cUP, i, j, k) + ky * AT(cUP + 1, i, j, k) + kz * AT(cUP + 2, i, j, k)) * inv_jac;
}
__device__ __forceinline__ int bcomp(int axis) { return axis == 0 ? cBX : axis == 1 ? cBY : cBZ; }
__device__ __forceinline__ int bacomp(int axis) { return axis == 0 ? cBAX : axis == 1 ? cBAY : cBAZ; }
__device__ __forceinline__ double face_tot(const BlockView &B, int axis, int i, int j, int k) {
  return AT(bcomp(axis), i, j, k) + AT(bacomp(axis), i, j, k);
}
__device__ __forceinline__ double cell_beta_ind(const BlockView &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return 0.5 * (AT(bcomp(axis), i, j, k) + AT(bcomp(axis), ip, jp, kp));
}
__device__ __forceinline__ double cell_beta_tot(const BlockView &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return 0.5 * (face_tot(B, axis, i, j, k) + face_tot(B, axis, ip, jp, kp));
}
__device__ __forceinline__ double emf_flux(const BlockView &B, int ba, int fa, int iL, int jL, int kL, int iR, int jR,
                                           int kR, double bff) {
  const double btL = cell_beta_tot(B, ba, iL, jL, kL), btR = cell_beta_tot(B, ba, iR, jR, kR);
  const double biL = cell_beta_ind(B, ba, iL, jL, kL), biR = cell_beta_ind(B, ba, iR, jR, kR);
  const double ufL = cell_u_contra(B, fa, iL, jL, kL), ufR = cell_u_contra(B, fa, iR, jR, kR);
  const double ubL = cell_u_contra(B, ba, iL, jL, kL), ubR = cell_u_contra(B, ba, iR, jR, kR);
  const double GL = ufL * btL - ubL * bff, GR = ufR * btR - ubR * bff;
  const double r = dmax(fabs(ufL), fabs(ufR));
  return 0.5 * (GL + GR) - 0.5 * r * (biR - biL);
}

// One thread per face over [-1, inner_hi + 1) per axis (the one locally
// evaluated ghost layer of Ideal.cpp:548-555), all three face families.
__global__ void k_face_emf(BlockView B) {
  const int lo[3] = {-1, -1, -1}, hi[3] = {B.n[0] + 2, B.n[1] + 2, B.n[2] + 2};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  for (int fa = 0; fa < 3; ++fa) {
    // face family fa has inner_hi = n + 1 along fa, n elsewhere
    bool in = true;
    const int q[3] = {i, j, k};
    for (int a = 0; a < 3; ++a) in = in && q[a] < B.n[a] + (a == fa ? 1 : 0) + 1;
    if (!in) continue;
    int iL = i, jL = j, kL = k;
    shift1(fa, iL, jL, kL, -1);
    const double bff = face_tot(B, fa, i, j, k);
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    if (fa == 0) {
      const double Ge = emf_flux(B, 1, 0, iL, jL, kL, i, j, k, bff);
      const double Gz = emf_flux(B, 2, 0, iL, jL, kL, i, j, k, bff);
      e1 = Gz;
      e2 = -Ge;
    } else if (fa == 1) {
      const double Gx = emf_flux(B, 0, 1, iL, jL, kL, i, j, k, bff);
      const double Gz = emf_flux(B, 2, 1, iL, jL, kL, i, j, k, bff);
      e0 = -Gz;
      e2 = Gx;
    } else {
      const double Gx = emf_flux(B, 0, 2, iL, jL, kL, i, j, k, bff);
      const double Ge = emf_flux(B, 1, 2, iL, jL, kL, i, j, k, bff);
      e0 = Ge;
      e1 = -Gx;
    }
    const int ce = fa == 0 ? cEFX : fa == 1 ? cEFY : cEFZ;
    AT(ce, i, j, k) = e0;
    AT(ce + 1, i, j, k) = e1;
    AT(ce + 2, i, j, k) = e2;
  }
}

__device__ __forceinline__ double max_abs_u4(const BlockView &B, int axis, int i0, int j0, int k0, int i1, int j1, int k1,
                                             int i2, int j2, int k2, int i3, int j3, int k3) {
  double a = 0.0;
  a = dmax(a, fabs(cell_u_contra(B, axis, i0, j0, k0)));
  a = dmax(a, fabs(cell_u_contra(B, axis, i1, j1, k1)));
  a = dmax(a, fabs(cell_u_contra(B, axis, i2, j2, k2)));
  a = dmax(a, fabs(cell_u_contra(B, axis, i3, j3, k3)));
  return a;
}

__device__ __forceinline__ double pe_node(const BlockView &B, int i, int j, int k) {
  double sum = 0.0;
  for (int di = -1; di <= 0; ++di)
    for (int dj = -1; dj <= 0; ++dj)
      for (int dk = -1; dk <= 0; ++dk)
        sum += AT(cPVH + 3, i + di, j + dj, k + dk) + AT(cPVN + 3, i + di, j + dj, k + dk);
  return 0.125 * sum;
}

// AssembleEdgeEMF_FromFaceE_Ideal_ (Ideal.cpp:138-372) followed by
// AddAmbipolarEdgeEMF_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ambipo.cpp:3-143)
// on the owned edges of all three families.  E ghosts are not written (the
// Eedge sync fills them later; nothing reads them before).
__global__ void k_edge_emf(BlockView B, Consts c) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  const double Cuct = 0.5;
  const double pc = (c.rho_ref * c.U_ref) / (c.q_e * c.L_ref * c.B_ref * c.n_ref);
  if (i < B.n[0]) {  // xi edges: i in [0,n), j,k in [0,n]
    const double Ec = 0.25 * (AT(cEFY, i, j, k) + AT(cEFY, i, j, k - 1) + AT(cEFZ, i, j, k) + AT(cEFZ, i, j - 1, k));
    const double ae = max_abs_u4(B, 1, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
    const double az = max_abs_u4(B, 2, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
    const double d1 = AT(cBZ, i, j, k) - AT(cBZ, i, j - 1, k);
    const double d2 = AT(cBY, i, j, k) - AT(cBY, i, j, k - 1);
    double e = Ec + Cuct * (0.5 * ae * d1 - 0.5 * az * d2);
    if (c.ambipolar) {
      const double p0 = pe_node(B, i, j, k), p1 = pe_node(B, i + 1, j, k);
      double rH = 0.0, rN = 0.0;
      for (int dj = -1; dj <= 0; ++dj)
        for (int dk = -1; dk <= 0; ++dk) {
          rH += AT(cUH, i, j + dj, k + dk);
          rN += AT(cUN, i, j + dj, k + dk);
        }
      const Num d = num_limiter(c, 0.25 * rH, 0.25 * rN);
      e -= pc * (p1 - p0) / d.ne_eff;
    }
    AT(cEX, i, j, k) = e;
  }
  if (j < B.n[1]) {  // eta edges
    const double Ec = 0.25 * (AT(cEFX + 1, i, j, k) + AT(cEFX + 1, i, j, k - 1) + AT(cEFZ + 1, i, j, k) +
                              AT(cEFZ + 1, i - 1, j, k));
    const double az = max_abs_u4(B, 2, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
    const double ax = max_abs_u4(B, 0, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
    const double d1 = AT(cBX, i, j, k) - AT(cBX, i, j, k - 1);
    const double d2 = AT(cBZ, i, j, k) - AT(cBZ, i - 1, j, k);
    double e = Ec + Cuct * (0.5 * az * d1 - 0.5 * ax * d2);
    if (c.ambipolar) {
      const double p0 = pe_node(B, i, j, k), p1 = pe_node(B, i, j + 1, k);
      double rH = 0.0, rN = 0.0;
      for (int di = -1; di <= 0; ++di)
        for (int dk = -1; dk <= 0; ++dk) {
          rH += AT(cUH, i + di, j, k + dk);
          rN += AT(cUN, i + di, j, k + dk);
        }
      const Num d = num_limiter(c, 0.25 * rH, 0.25 * rN);
      e -= pc * (p1 - p0) / d.ne_eff;
    }
    AT(cEY, i, j, k) = e;
  }
  if (k < B.n[2]) {  // zeta edges
    const double Ec = 0.25 * (AT(cEFX + 2, i, j, k) + AT(cEFX + 2, i, j - 1, k) + AT(cEFY + 2, i, j, k) +
                              AT(cEFY + 2, i - 1, j, k));
    const double ax = max_abs_u4(B, 0, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
    const double ae = max_abs_u4(B, 1, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
    const double d1 = AT(cBY, i, j, k) - AT(cBY, i - 1, j, k);
    const double d2 = AT(cBX, i, j, k) - AT(cBX, i, j - 1, k);
    double e = Ec + Cuct * (0.5 * ax * d1 - 0.5 * ae * d2);
    if (c.ambipolar) {
      const double p0 = pe_node(B, i, j, k), p1 = pe_node(B, i, j, k + 1);
      double rH = 0.0, rN = 0.0;
      for (int di = -1; di <= 0; ++di)
        for (int dj = -1; dj <= 0; ++dj) {
          rH += AT(cUH, i + di, j + dj, k);
          rN += AT(cUN, i + di, j + dj, k);
        }
      const Num d = num_limiter(c, 0.25 * rH, 0.25 * rN);
      e -= pc * (p1 - p0) / d.ne_eff;
    }
    AT(cEZ, i, j, k) = e;
  }
}

// ------------------------------------------------------------------ Hall EMF
// BuildHallFaceEMF_Rusanov_diff_ step 1 (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:110-146)
// over the allocated cell range [-g, n + g).
__global__ void k_hall_cell(BlockView B, Consts c, int g) {
  const int lo[3] = {-g, -g, -g}, hi[3] = {B.n[0] + g, B.n[1] + g, B.n[2] + g};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  const Num d = num_limiter(c, AT(cUH, i, j, k), AT(cUN, i, j, k));
  const double alpha = c.hall_coef / d.ne_eff;
  const double Jx = AT(cJC, i, j, k), Jy = AT(cJC + 1, i, j, k), Jz = AT(cJC + 2, i, j, k);
  const double Bx = AT(cBC, i, j, k), By = AT(cBC + 1, i, j, k), Bz = AT(cBC + 2, i, j, k);
  AT(cEHC, i, j, k) = alpha * (Jy * Bz - Jz * By);
  AT(cEHC + 1, i, j, k) = alpha * (Jz * Bx - Jx * Bz);
  AT(cEHC + 2, i, j, k) = alpha * (Jx * By - Jy * Bx);
  AT(cHB, i, j, k) = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
}

// BuildHallFaceEMF_Rusanov_diff_ steps 2-4 (Hall.cpp:148-400): Hall edge EMF
// with whistler-LLF diffusion (C_wh = 0.1) and the per-edge radial taper.
__global__ void k_hall_edge(BlockView B) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  const double eps = 1e-14, Cwh = 0.1;
  if (i < B.n[0]) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (AT(cEHC + q, i, j - 1, k - 1) + AT(cEHC + q, i, j - 1, k) + AT(cEHC + q, i, j, k - 1) +
                      AT(cEHC + q, i, j, k));
    const double Ecen = Ec[0] * AT(cDRX, i, j, k) + Ec[1] * AT(cDRX + 1, i, j, k) + Ec[2] * AT(cDRX + 2, i, j, k);
    const double be = dmax(dmax(AT(cHB, i, j - 1, k - 1), AT(cHB, i, j - 1, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
    const double L = dmax(AT(cDLX, i, j, k), eps);
    const double Abz = 0.5 * (AT(cAZ, i, j, k) + AT(cAZ, i, j - 1, k));
    const double ihe = L / dmax(Abz, eps);
    const double mue = Cwh * be * ihe * ihe;
    const double Abe = 0.5 * (AT(cAY, i, j, k) + AT(cAY, i, j, k - 1));
    const double ihz = L / dmax(Abe, eps);
    const double muz = Cwh * be * ihz * ihz;
    const double d1 = AT(cBZ, i, j, k) - AT(cBZ, i, j - 1, k);
    const double d2 = AT(cBY, i, j, k) - AT(cBY, i, j, k - 1);
    AT(cHX, i, j, k) = AT(cTPX, i, j, k) * (Ecen + 0.5 * mue * d1 - 0.5 * muz * d2);
  }
  if (j < B.n[1]) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (AT(cEHC + q, i - 1, j, k - 1) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j, k - 1) +
                      AT(cEHC + q, i, j, k));
    const double Ecen = Ec[0] * AT(cDRY, i, j, k) + Ec[1] * AT(cDRY + 1, i, j, k) + Ec[2] * AT(cDRY + 2, i, j, k);
    const double be = dmax(dmax(AT(cHB, i - 1, j, k - 1), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
    const double L = dmax(AT(cDLY, i, j, k), eps);
    const double Abx = 0.5 * (AT(cAX, i, j, k) + AT(cAX, i, j, k - 1));
    const double ihz = L / dmax(Abx, eps);
    const double muz = Cwh * be * ihz * ihz;
    const double Abz = 0.5 * (AT(cAZ, i, j, k) + AT(cAZ, i - 1, j, k));
    const double ihx = L / dmax(Abz, eps);
    const double mux = Cwh * be * ihx * ihx;
    const double d1 = AT(cBX, i, j, k) - AT(cBX, i, j, k - 1);
    const double d2 = AT(cBZ, i, j, k) - AT(cBZ, i - 1, j, k);
    AT(cHY, i, j, k) = AT(cTPY, i, j, k) * (Ecen + 0.5 * muz * d1 - 0.5 * mux * d2);
  }
  if (k < B.n[2]) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (AT(cEHC + q, i - 1, j - 1, k) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j - 1, k) +
                      AT(cEHC + q, i, j, k));
    const double Ecen = Ec[0] * AT(cDRZ, i, j, k) + Ec[1] * AT(cDRZ + 1, i, j, k) + Ec[2] * AT(cDRZ + 2, i, j, k);
    const double be = dmax(dmax(AT(cHB, i - 1, j - 1, k), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j - 1, k), AT(cHB, i, j, k)));
    const double L = dmax(AT(cDLZ, i, j, k), eps);
    const double Abe = 0.5 * (AT(cAY, i, j, k) + AT(cAY, i - 1, j, k));
    const double ihx = L / dmax(Abe, eps);
    const double mux = Cwh * be * ihx * ihx;
    const double Abx = 0.5 * (AT(cAX, i, j, k) + AT(cAX, i, j - 1, k));
    const double ihe = L / dmax(Abx, eps);
    const double mue = Cwh * be * ihe * ihe;
    const double d1 = AT(cBY, i, j, k) - AT(cBY, i - 1, j, k);
    const double d2 = AT(cBX, i, j, k) - AT(cBX, i, j - 1, k);
    AT(cHZ, i, j, k) = AT(cTPZ, i, j, k) * (Ecen + 0.5 * mux * d1 - 0.5 * mue * d2);
  }
}

// E += Ehall on owned edges (MagneticRHS.cpp:135-147).
__global__ void k_add_hall(BlockView B) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  if (i < B.n[0]) AT(cEX, i, j, k) += AT(cHX, i, j, k);
  if (j < B.n[1]) AT(cEY, i, j, k) += AT(cHY, i, j, k);
  if (k < B.n[2]) AT(cEZ, i, j, k) += AT(cHZ, i, j, k);
}

// ------------------------------------------------------------------ fluid RHS + update
// Scheme_U_ (Z4_Mercury/src/physics/MercurySolver_FluidRHS.cpp:3-202): Rusanov
// face flux.  The cell kernel evaluates both faces of each direction itself
// (the same deterministic function the reference stores in F_xi/F_eta/F_zeta),
// so the divergence is bitwise the reference's without the flux scratch.
__device__ __forceinline__ void rusanov(const BlockView &B, const Consts &c, int u0, int pv0, double k1, double k2,
                                        double k3, int iL, int jL, int kL, int i, int j, int k, double out[5]) {
  const double g = c.gamma;
  const double rhoL = AT(u0, iL, jL, kL), uL = AT(pv0, iL, jL, kL), vL = AT(pv0 + 1, iL, jL, kL),
               wL = AT(pv0 + 2, iL, jL, kL), pL = AT(pv0 + 3, iL, jL, kL);
  const double rhoR = AT(u0, i, j, k), uR = AT(pv0, i, j, k), vR = AT(pv0 + 1, i, j, k), wR = AT(pv0 + 2, i, j, k),
               pR = AT(pv0 + 3, i, j, k);
  const double reL = pL / (g - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL);
  const double reR = pR / (g - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR);
  const double UL[5] = {rhoL, rhoL * uL, rhoL * vL, rhoL * wL, reL};
  const double UR[5] = {rhoR, rhoR * uR, rhoR * vR, rhoR * wR, reR};
  const double kk = k1 * k1 + k2 * k2 + k3 * k3;
  const double uvwL = k1 * uL + k2 * vL + k3 * wL, uvwR = k1 * uR + k2 * vR + k3 * wR;
  const double cL = sqrt(dmax(0.0, g * pL / dmax(rhoL, 1e-30))), cR = sqrt(dmax(0.0, g * pR / dmax(rhoR, 1e-30)));
  const double rad = dmax(fabs(uvwL) + cL * sqrt(kk), fabs(uvwR) + cR * sqrt(kk));
  const double FL[5] = {rhoL * uvwL, rhoL * uvwL * uL + k1 * pL, rhoL * uvwL * vL + k2 * pL, rhoL * uvwL * wL + k3 * pL,
                        uvwL * (reL + pL)};
  const double FR[5] = {rhoR * uvwR, rhoR * uvwR * uR + k1 * pR, rhoR * uvwR * vR + k2 * pR, rhoR * uvwR * wR + k3 * pR,
                        uvwR * (reR + pR)};
#pragma unroll
  for (int m = 0; m < 5; ++m) out[m] = 0.5 * (FL[m] + FR[m]) - 0.5 * rad * (UR[m] - UL[m]);
}

// ZeroRHS_ + Scheme_U_ + AddSourceToRHS_Fluid (FluidRHS.cpp:206-527) +
// ApplyUpdate_Euler_ (Z4_Mercury/src/physics/MercurySolver_Advance.cpp:73-147)
// for one owned cell (both species), and B_face += dt * (-curl E) for the
// owned faces at the same (i, j, k) (CTOperators.cpp:6-56 with multiplier -1).
__global__ void k_update(BlockView B, Consts c, Scalars *S, int account) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  const double dt = __longlong_as_double((long long)S->dt_bits);
  if (!(dt >= 1e-7) || !isfinite(dt)) {
    if (i == 0 && j == 0 && k == 0) S->status = MHD_ERR_DT;
    return;  // the reference aborts here; the state stays at the last valid step
  }
  if (account && i == 0 && j == 0 && k == 0) {  // run_data_ bookkeeping (Driver.cpp:40-45)
    S->dt = dt;
    S->time += dt;
    S->step += 1;
  }
  // ---- faces: B += dt * RHS_B
  if (j < B.n[1] && k < B.n[2]) {
    const double rb = -1.0 * ((AT(cEY, i, j, k) - AT(cEY, i, j, k + 1)) + (AT(cEZ, i, j + 1, k) - AT(cEZ, i, j, k)));
    AT(cBX, i, j, k) += dt * rb;
  }
  if (i < B.n[0] && k < B.n[2]) {
    const double rb = -1.0 * ((AT(cEX, i, j, k + 1) - AT(cEX, i, j, k)) + (AT(cEZ, i, j, k) - AT(cEZ, i + 1, j, k)));
    AT(cBY, i, j, k) += dt * rb;
  }
  if (i < B.n[0] && j < B.n[1]) {
    const double rb = -1.0 * ((AT(cEX, i, j, k) - AT(cEX, i, j + 1, k)) + (AT(cEY, i + 1, j, k) - AT(cEY, i, j, k)));
    AT(cBZ, i, j, k) += dt * rb;
  }
  if (i >= B.n[0] || j >= B.n[1] || k >= B.n[2]) return;
  // ---- cell: fluid RHS of both species, then U^{n+1}
  double R[2][5];
  const double invJ = 1.0 / AT(cJAC, i, j, k);
  for (int s = 0; s < 2; ++s) {
    const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double Fm[5], Fp[5];
    double dx[5], dy[5], dz[5];
    rusanov(B, c, u0, pv0, AT(cJDX, i, j, k), AT(cJDX + 1, i, j, k), AT(cJDX + 2, i, j, k), i - 1, j, k, i, j, k, Fm);
    rusanov(B, c, u0, pv0, AT(cJDX, i + 1, j, k), AT(cJDX + 1, i + 1, j, k), AT(cJDX + 2, i + 1, j, k), i, j, k, i + 1, j,
            k, Fp);
    for (int m = 0; m < 5; ++m) dx[m] = Fp[m] - Fm[m];
    rusanov(B, c, u0, pv0, AT(cJDY, i, j, k), AT(cJDY + 1, i, j, k), AT(cJDY + 2, i, j, k), i, j - 1, k, i, j, k, Fm);
    rusanov(B, c, u0, pv0, AT(cJDY, i, j + 1, k), AT(cJDY + 1, i, j + 1, k), AT(cJDY + 2, i, j + 1, k), i, j, k, i, j + 1,
            k, Fp);
    for (int m = 0; m < 5; ++m) dy[m] = Fp[m] - Fm[m];
    rusanov(B, c, u0, pv0, AT(cJDZ, i, j, k), AT(cJDZ + 1, i, j, k), AT(cJDZ + 2, i, j, k), i, j, k - 1, i, j, k, Fm);
    rusanov(B, c, u0, pv0, AT(cJDZ, i, j, k + 1), AT(cJDZ + 1, i, j, k + 1), AT(cJDZ + 2, i, j, k + 1), i, j, k, i, j,
            k + 1, Fp);
    for (int m = 0; m < 5; ++m) dz[m] = Fp[m] - Fm[m];
    for (int m = 0; m < 5; ++m) {
      r[m] -= dx[m] * invJ;
      r[m] -= dy[m] * invJ;
      r[m] -= dz[m] * invJ;
    }
    for (int m = 0; m < 5; ++m) R[s][m] = r[m];
  }
  // ---- sources (FluidRHS.cpp:206-527)
  {
    const double Tn0 = 1000.0, sk1 = 5.0e-5, sk2 = 1.0e-5;
    const double a1_Na = (c.L_ref / c.U_ref) * (c.m_Na / c.rho_ref) * 1e6;
    const double a4 = (c.L_ref / c.U_ref);
    const double a5 = (3.0 * c.L_ref * c.k_Boltz * c.n_ref) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref);
    const double a6 = (1.0e6 * c.L_ref * c.k_Boltz) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref * (c.gamma - 1.0));
    const double upx = AT(cUP, i, j, k), upy = AT(cUP + 1, i, j, k), upz = AT(cUP + 2, i, j, k);
    const double Bx = AT(cBC, i, j, k), By = AT(cBC + 1, i, j, k), Bz = AT(cBC + 2, i, j, k);
    const double Jx = AT(cJC, i, j, k), Jy = AT(cJC + 1, i, j, k), Jz = AT(cJC + 2, i, j, k);
    const double sjbx = Jy * Bz - Jz * By, sjby = Jz * Bx - Jx * Bz, sjbz = Jx * By - Jy * Bx;
    const Num num = num_limiter(c, AT(cUH, i, j, k), AT(cUN, i, j, k));
    double dpex = 0.0, dpey = 0.0, dpez = 0.0;
    if (c.ambipolar) {
      const double Vol = fabs(AT(cJAC, i, j, k));
      double ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0, cxm = 0, cym = 0, czm = 0;
      if (Vol > 0.0) {
        ax = 0.5 * (AT(cJDX, i - 1, j, k) + AT(cJDX, i, j, k)) / Vol;
        ay = 0.5 * (AT(cJDX + 1, i - 1, j, k) + AT(cJDX + 1, i, j, k)) / Vol;
        az = 0.5 * (AT(cJDX + 2, i - 1, j, k) + AT(cJDX + 2, i, j, k)) / Vol;
        bx = 0.5 * (AT(cJDY, i, j - 1, k) + AT(cJDY, i, j, k)) / Vol;
        by = 0.5 * (AT(cJDY + 1, i, j - 1, k) + AT(cJDY + 1, i, j, k)) / Vol;
        bz = 0.5 * (AT(cJDY + 2, i, j - 1, k) + AT(cJDY + 2, i, j, k)) / Vol;
        cxm = 0.5 * (AT(cJDZ, i, j, k - 1) + AT(cJDZ, i, j, k)) / Vol;
        cym = 0.5 * (AT(cJDZ + 1, i, j, k - 1) + AT(cJDZ + 1, i, j, k)) / Vol;
        czm = 0.5 * (AT(cJDZ + 2, i, j, k - 1) + AT(cJDZ + 2, i, j, k)) / Vol;
      }
      const double pip = AT(cPVH + 3, i + 1, j, k) + AT(cPVN + 3, i + 1, j, k);
      const double pim = AT(cPVH + 3, i - 1, j, k) + AT(cPVN + 3, i - 1, j, k);
      const double pjp = AT(cPVH + 3, i, j + 1, k) + AT(cPVN + 3, i, j + 1, k);
      const double pjm = AT(cPVH + 3, i, j - 1, k) + AT(cPVN + 3, i, j - 1, k);
      const double pkp = AT(cPVH + 3, i, j, k + 1) + AT(cPVN + 3, i, j, k + 1);
      const double pkm = AT(cPVH + 3, i, j, k - 1) + AT(cPVN + 3, i, j, k - 1);
      dpex = 0.5 * (ax * (pip - pim) + bx * (pjp - pjm) + cxm * (pkp - pkm));
      dpey = 0.5 * (ay * (pip - pim) + by * (pjp - pjm) + cym * (pkp - pkm));
      dpez = 0.5 * (az * (pip - pim) + bz * (pjp - pjm) + czm * (pkp - pkm));
    }
    const double sss = AT(cPHOTO, i, j, k);
    const double x = AT(cCX, i, j, k), y = AT(cCY, i, j, k), z = AT(cCZ, i, j, k);
    const double rho_cyl = sqrt(y * y + z * z);
    const double vst = (x < 0.0 && rho_cyl < 1.0) ? sk2 : sk1;
    for (int s = 0; s < 2; ++s) {
      const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
      double *r = R[s];
      const double nS = s ? num.nNa : num.nH;
      const double chi = s ? num.wNa : num.wH;
      const double rho = dmax(AT(u0, i, j, k), 0.0);
      const double u = AT(pv0, i, j, k), v = AT(pv0 + 1, i, j, k), w = AT(pv0 + 2, i, j, k);
      const double u2 = u * u + v * v + w * w;
      const double subx = (v - upy) * Bz - (w - upz) * By;
      const double suby = (w - upz) * Bx - (u - upx) * Bz;
      const double subz = (u - upx) * By - (v - upy) * Bx;
      const double subu = subx * u + suby * v + subz * w;
      const double sjbu = sjbx * u + sjby * v + sjbz * w;
      const double dpeu = dpex * u + dpey * v + dpez * w;
      const double Ts0 = AT(pv0 + 4, i, j, k) * c.T_ref;
      double b1, b2;
      if (!s) {
        b1 = vst * (Tn0 - Ts0) * (c.M_H / (c.M_H + c.M_Na));
        b2 = (c.M_Na / (c.M_H + c.M_Na)) * vst;
      } else {
        b1 = vst * (Tn0 - Ts0) * (c.M_Na / (c.M_Na + c.M_Na));
        b2 = (c.M_Na / (c.M_Na + c.M_Na)) * vst;
      }
      r[1] += c.momentum_induce_coeff * nS * subx + c.momentum_hall_coeff * chi * sjbx;
      r[2] += c.momentum_induce_coeff * nS * suby + c.momentum_hall_coeff * chi * sjby;
      r[3] += c.momentum_induce_coeff * nS * subz + c.momentum_hall_coeff * chi * sjbz;
      r[4] += c.momentum_induce_coeff * nS * subu + c.momentum_hall_coeff * chi * sjbu;
      if (c.ambipolar) {
        r[1] -= chi * dpex;
        r[2] -= chi * dpey;
        r[3] -= chi * dpez;
        r[4] -= chi * dpeu;
      }
      if (s) {
        r[0] += a1_Na * sss;
        r[4] += a6 * sss * Tn0;
      }
      r[1] -= a4 * rho * u * vst;
      r[2] -= a4 * rho * v * vst;
      r[3] -= a4 * rho * w * vst;
      r[4] -= a4 * rho * u2 * vst;
      r[4] += a5 * nS * b1;
      r[4] += a4 * rho * u2 * b2;
    }
  }
  const int64_t o = B.off(i, j, k);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    B.Unext[(int64_t)(cUH + m) * B.total + o] = B.U[(int64_t)(cUH + m) * B.total + o] + dt * R[0][m];
    B.Unext[(int64_t)(cUN + m) * B.total + o] = B.U[(int64_t)(cUN + m) * B.total + o] + dt * R[1][m];
  }
}

// ------------------------------------------------------------------ derived fields
// calc_Bcell (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:3-90), owned cells.
// Thread (0,0,0) of the launch also re-arms the dt accumulator for the next
// step (every reader of this step's dt has finished by stream order).
__global__ void k_bcell(BlockView B, Scalars *S, int rearm) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  Idx p;
  const bool in = thread_index(lo, hi, p);
  if (rearm && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0 &&
      threadIdx.z == 0)
    S->dt_bits = (unsigned long long)__double_as_longlong(1e100);
  if (!in) return;
  const int i = p.i, j = p.j, k = p.k;
  const double pt[6] = {-AT(cBX, i, j, k) - AT(cBAX, i, j, k), AT(cBX, i + 1, j, k) + AT(cBAX, i + 1, j, k),
                        -AT(cBY, i, j, k) - AT(cBAY, i, j, k), AT(cBY, i, j + 1, k) + AT(cBAY, i, j + 1, k),
                        -AT(cBZ, i, j, k) - AT(cBAZ, i, j, k), AT(cBZ, i, j, k + 1) + AT(cBAZ, i, j, k + 1)};
  const double pi_[6] = {-AT(cBX, i, j, k), AT(cBX, i + 1, j, k), -AT(cBY, i, j, k),
                         AT(cBY, i, j + 1, k), -AT(cBZ, i, j, k), AT(cBZ, i, j, k + 1)};
  double bxt = 0, byt = 0, bzt = 0, bxi = 0, byi = 0, bzi = 0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const double wx = AT(cWB + q, i, j, k), wy = AT(cWB + 6 + q, i, j, k), wz = AT(cWB + 12 + q, i, j, k);
    bxt += wx * pt[q];
    byt += wy * pt[q];
    bzt += wz * pt[q];
    bxi += wx * pi_[q];
    byi += wy * pi_[q];
    bzi += wz * pi_[q];
  }
  AT(cBC, i, j, k) = bxt;
  AT(cBC + 1, i, j, k) = byt;
  AT(cBC + 2, i, j, k) = bzt;
  AT(cBIC, i, j, k) = bxi;
  AT(cBIC + 1, i, j, k) = byi;
  AT(cBIC + 2, i, j, k) = bzi;
}

// CurlAdjFaceToEdge (Z4_Mercury/src/operators/CTOperators.cpp:59-110) then the
// alpha scaling of Calc_J_Edge (Z4_Mercury/src/physics/MercurySolver_Current.cpp:140-190).
__global__ void k_jedge(BlockView B) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  if (i < B.n[0]) {
    const double v = ((AT(cBFY, i, j, k - 1) * AT(cBY, i, j, k - 1) - AT(cBFY, i, j, k) * AT(cBY, i, j, k)) +
                      (AT(cBFZ, i, j, k) * AT(cBZ, i, j, k) - AT(cBFZ, i, j - 1, k) * AT(cBZ, i, j - 1, k))) * 1.0;
    AT(cJX, i, j, k) = v * AT(cALX, i, j, k);
  }
  if (j < B.n[1]) {
    const double v = ((AT(cBFX, i, j, k) * AT(cBX, i, j, k) - AT(cBFX, i, j, k - 1) * AT(cBX, i, j, k - 1)) +
                      (AT(cBFZ, i - 1, j, k) * AT(cBZ, i - 1, j, k) - AT(cBFZ, i, j, k) * AT(cBZ, i, j, k))) * 1.0;
    AT(cJY, i, j, k) = v * AT(cALY, i, j, k);
  }
  if (k < B.n[2]) {
    const double v = ((AT(cBFX, i, j - 1, k) * AT(cBX, i, j - 1, k) - AT(cBFX, i, j, k) * AT(cBX, i, j, k)) +
                      (AT(cBFY, i, j, k) * AT(cBY, i, j, k) - AT(cBFY, i - 1, j, k) * AT(cBY, i - 1, j, k))) * 1.0;
    AT(cJZ, i, j, k) = v * AT(cALZ, i, j, k);
  }
}

// calc_Jcell (Current.cpp:203-243), owned cells.
__global__ void k_jcell(BlockView B) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  const double s[12] = {AT(cJX, i, j, k),         AT(cJX, i, j + 1, k),     AT(cJX, i, j, k + 1),
                        AT(cJX, i, j + 1, k + 1), AT(cJY, i, j, k),         AT(cJY, i + 1, j, k),
                        AT(cJY, i, j, k + 1),     AT(cJY, i + 1, j, k + 1), AT(cJZ, i, j, k),
                        AT(cJZ, i + 1, j, k),     AT(cJZ, i, j + 1, k),     AT(cJZ, i + 1, j + 1, k)};
  double jx = 0, jy = 0, jz = 0;
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    jx += AT(cWJ + q, i, j, k) * s[q];
    jy += AT(cWJ + 12 + q, i, j, k) * s[q];
    jz += AT(cWJ + 24 + q, i, j, k) * s[q];
  }
  AT(cJC, i, j, k) = jx;
  AT(cJC + 1, i, j, k) = jy;
  AT(cJC + 2, i, j, k) = jz;
}

// calc_PV + calc_Uplus (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:159-301)
// over the allocated cell range [-g, n + g), ghosts included.
__global__ void k_pv_uplus(BlockView B, Consts c, int g) {
  const int lo[3] = {-g, -g, -g}, hi[3] = {B.n[0] + g, B.n[1] + g, B.n[2] + g};
  Idx p;
  if (!thread_index(lo, hi, p)) return;
  const int i = p.i, j = p.j, k = p.k;
  double vel[2][3];
  for (int s = 0; s < 2; ++s) {
    const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
    const double coeff = s ? c.state_coeff_Na : c.state_coeff_H;
    const double rho = dmax(AT(u0, i, j, k), 1e-12);
    const double u = AT(u0 + 1, i, j, k) / rho, v = AT(u0 + 2, i, j, k) / rho, w = AT(u0 + 3, i, j, k) / rho;
    const double E = AT(u0 + 4, i, j, k);
    const double ke = 0.5 * rho * (u * u + v * v + w * w);
    double eint = E - ke;
    if (eint < 0.0) eint = 0.0;
    double pr = (c.gamma - 1.0) * eint;
    pr = dmax(pr, 1e-12);
    const double T = pr / (rho * coeff);
    AT(pv0, i, j, k) = u;
    AT(pv0 + 1, i, j, k) = v;
    AT(pv0 + 2, i, j, k) = w;
    AT(pv0 + 3, i, j, k) = pr;
    AT(pv0 + 4, i, j, k) = T;
    vel[s][0] = u;
    vel[s][1] = v;
    vel[s][2] = w;
  }
  const double rH = dmax(AT(cUH, i, j, k), 0.0), rN = dmax(AT(cUN, i, j, k), 0.0);
  const Num d = num_limiter(c, rH, rN);
  for (int q = 0; q < 3; ++q) {
    const double uH = rH > 1e-20 ? vel[0][q] : 0.0;
    const double uN = rN > 1e-20 ? vel[1][q] : 0.0;
    AT(cUP + q, i, j, k) = d.chiH * uH + d.chiNa * uN;
  }
}

#undef AT

// ------------------------------------------------------------------ sync and alias kernels
// One flattened copy table: dst <- sign * src, element offsets into the arena;
// bit 62 of an offset marks a U component (current buffer chosen at launch).
__global__ void k_copy(const int64_t *__restrict__ dst, const int64_t *__restrict__ src, const double *__restrict__ sign,
                       int n, double *arena, int64_t ucur_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  constexpr int64_t kU = int64_t(1) << 62;
  int64_t s = src[t], d = dst[t];
  if (s & kU) s = (s & ~kU) + ucur_off;
  if (d & kU) d = (d & ~kU) + ucur_off;
  arena[d] = sign[t] * arena[s];
}

// ReduceEdgeAliasCandidatesToOwners_ (Current.cpp:3-57): one thread per class,
// members summed in stored order from 0.0.
__global__ void k_alias(const int32_t *__restrict__ offset, const int64_t *__restrict__ member,
                        const double *__restrict__ msign, const int64_t *__restrict__ owner,
                        const double *__restrict__ osign, int n_classes, double *arena) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_classes) return;
  const int a = offset[t], b = offset[t + 1];
  double sum = 0.0;
  for (int q = a; q < b; ++q) sum += msign[q] * arena[member[q]];
  arena[owner[t]] = osign[t] * sum / (double)(b - a);
}

}  // namespace

// ------------------------------------------------------------------ launchers
static dim3 grid_for(const int lo[3], const int hi[3], dim3 blk) {
  return dim3((unsigned)((hi[2] - lo[2] + blk.x - 1) / blk.x), (unsigned)((hi[1] - lo[1] + blk.y - 1) / blk.y),
              (unsigned)((hi[0] - lo[0] + blk.z - 1) / blk.z));
}
static const dim3 kBlk(32, 4, 2);

void launch_timestep(const BlockView &B, const Consts &c, Scalars *S, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  k_timestep<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, c, S);
}
void launch_face_emf(const BlockView &B, cudaStream_t st) {
  const int lo[3] = {-1, -1, -1}, hi[3] = {B.n[0] + 2, B.n[1] + 2, B.n[2] + 2};
  k_face_emf<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B);
}
void launch_edge_emf(const BlockView &B, const Consts &c, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  k_edge_emf<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, c);
}
void launch_hall_cell(const BlockView &B, const Consts &c, int g, cudaStream_t st) {
  const int lo[3] = {-g, -g, -g}, hi[3] = {B.n[0] + g, B.n[1] + g, B.n[2] + g};
  k_hall_cell<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, c, g);
}
void launch_hall_edge(const BlockView &B, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  k_hall_edge<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B);
}
void launch_add_hall(const BlockView &B, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  k_add_hall<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B);
}
void launch_update(const BlockView &B, const Consts &c, Scalars *S, int account, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  k_update<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, c, S, account);
}
void launch_bcell(const BlockView &B, Scalars *S, int rearm, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  k_bcell<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, S, rearm);
}
void launch_jedge(const BlockView &B, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0] + 1, B.n[1] + 1, B.n[2] + 1};
  k_jedge<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B);
}
void launch_jcell(const BlockView &B, cudaStream_t st) {
  const int lo[3] = {0, 0, 0}, hi[3] = {B.n[0], B.n[1], B.n[2]};
  k_jcell<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B);
}
void launch_pv_uplus(const BlockView &B, const Consts &c, int g, cudaStream_t st) {
  const int lo[3] = {-g, -g, -g}, hi[3] = {B.n[0] + g, B.n[1] + g, B.n[2] + g};
  k_pv_uplus<<<grid_for(lo, hi, kBlk), kBlk, 0, st>>>(B, c, g);
}
void launch_copy(const int64_t *dst, const int64_t *src, const double *sign, int n, double *arena, int64_t ucur_off,
                 cudaStream_t st) {
  if (n <= 0) return;
  k_copy<<<(n + 255) / 256, 256, 0, st>>>(dst, src, sign, n, arena, ucur_off);
}
void launch_alias(const int32_t *offset, const int64_t *member, const double *msign, const int64_t *owner,
                  const double *osign, int n_classes, double *arena, cudaStream_t st) {
  if (n_classes <= 0) return;
  k_alias<<<(n_classes + 127) / 128, 128, 0, st>>>(offset, member, msign, owner, osign, n_classes, arena);
}

}  // namespace mhd
