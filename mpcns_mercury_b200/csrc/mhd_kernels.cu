// FP64 kernels of the explicit multi-fluid Hall-MHD step on sm_100a, run by
// the batched engine (mhd_engine.cuh): every kernel is a persistent
// grid-stride loop over the tile work-list of all active solves.
//
// Each kernel restates one pass of the reference step in the reference's own
// operation order (the library is built without FMA contraction), so the
// FP64 path reproduces the reference bitwise.  Restructurings that keep the
// arithmetic identical:
//   * the contravariant velocity u^a = (K^a . U_plus) / (|J| + 1e-30) of every
//     cell (cell_u_contra, Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ideal.cpp:180-199)
//     is computed once per step into UCON instead of up to 16 times per edge;
//   * the fluid update runs one work item per (cell, species);
//   * B_cell/Bind_cell and J_edge share one pass over the face fluxes;
//   * the next step's CFL dt is reduced in the same pass that refreshes the
//     primitive variables (both read U and B_cell after their syncs).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "mhd_engine.cuh"
#include "mhd_kernels.cuh"

namespace mhd {

namespace {

constexpr int cUH = 0, cUN = 5;
constexpr int cBX = kComp.first[MHD_B_XI], cBY = kComp.first[MHD_B_ETA], cBZ = kComp.first[MHD_B_ZETA];
constexpr int cPVH = kComp.first[MHD_PV_H], cPVN = kComp.first[MHD_PV_NA], cUP = kComp.first[MHD_U_PLUS];
constexpr int cBC = kComp.first[MHD_B_CELL], cBIC = kComp.first[MHD_BIND_CELL], cJC = kComp.first[MHD_J_CELL];
constexpr int cJX = kComp.first[MHD_J_XI], cJY = kComp.first[MHD_J_ETA], cJZ = kComp.first[MHD_J_ZETA];
constexpr int cEX = kComp.first[MHD_E_XI], cEY = kComp.first[MHD_E_ETA], cEZ = kComp.first[MHD_E_ZETA];
constexpr int cHX = kComp.first[MHD_EHALL_XI], cHY = kComp.first[MHD_EHALL_ETA], cHZ = kComp.first[MHD_EHALL_ZETA];
constexpr int cEFX = kComp.first[MHD_EFACE_XI], cEFY = kComp.first[MHD_EFACE_ETA], cEFZ = kComp.first[MHD_EFACE_ZETA];
constexpr int cEHC = kComp.first[MHD_EHC], cHB = kComp.first[MHD_HALL_BETA], cUC = kComp.first[MHD_UCON];
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

// One block's fields for the current step: U = current buffer.
struct V {
  double *U, *Un, *M;
  int64_t total, si, sj;
  int G, n0, n1, n2;
  __device__ __forceinline__ double *c(int comp) const {
    return comp < kNumUComps ? U + (int64_t)comp * total : M + (int64_t)(comp - kNumUComps) * total;
  }
  __device__ __forceinline__ int64_t off(int i, int j, int k) const {
    return (int64_t)(i + G) * si + (int64_t)(j + G) * sj + (k + G);
  }
};
#define AT(cc, i, j, k) (B.c(cc)[B.off((i), (j), (k))])

struct Item {
  int s;       // solve
  int species; // kCells2 only
  int i, j, k;
  bool in;     // inside the kernel's range
};

// Work-item loop: for every tile of range `KIND` of every active solve, call
// f(S, B, item).  Tile lookup: two binary searches by thread 0, broadcast
// through shared memory.
template <int KIND, class F>
__device__ __forceinline__ void for_items(const Dir &D, F &&f) {
  __shared__ int sh[3];
  const int total = D.solve_tile_prefix[KIND][D.nsolves];
  const int tid = threadIdx.x;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    if (tid == 0) {
      const int *sp = D.solve_tile_prefix[KIND];
      int lo = 0, hi = D.nsolves;  // largest s with sp[s] <= w
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sp[mid] <= w) lo = mid; else hi = mid;
      }
      const int s = lo;
      const int lw = w - sp[s];
      const int *bp = D.solves[s].tile_prefix[KIND];
      int blo = 0, bhi = D.solves[s].nblocks;
      while (bhi - blo > 1) {
        const int mid = (blo + bhi) >> 1;
        if (bp[mid] <= lw) blo = mid; else bhi = mid;
      }
      sh[0] = s;
      sh[1] = blo;
      sh[2] = lw - bp[blo];
    }
    __syncthreads();
    const int s = sh[0], b = sh[1];
    int t = sh[2];
    __syncthreads();
    if (!solve_active(D, s)) continue;  // inactive solve (the whole CTA agrees)
    const DevSolve &S = D.solves[s];
    const DevBlock &DB = S.blocks[b];
    const RangeBox r = range_of(KIND, DB.n, S.c.nghost);
    Item it;
    it.s = s;
    it.species = 0;
    if (KIND == kCells2) {
      it.species = t & 1;
      t >>= 1;
    }
    const int tk = (r.hi[2] - r.lo[2] + kTileK - 1) / kTileK;
    const int tj = (r.hi[1] - r.lo[1] + kTileJ - 1) / kTileJ;
    const int bk = t % tk, bj = (t / tk) % tj, bi = t / (tk * tj);
    it.k = r.lo[2] + bk * kTileK + (tid % kTileK);
    it.j = r.lo[1] + bj * kTileJ + ((tid / kTileK) % kTileJ);
    it.i = r.lo[0] + bi * kTileI + (tid / (kTileK * kTileJ));
    it.in = it.i < r.hi[0] && it.j < r.hi[1] && it.k < r.hi[2];
    V B;
    const int cur = D.state[s].cur;
    B.U = DB.U[cur];
    B.Un = DB.U[cur ^ 1];
    B.M = DB.M;
    B.total = DB.total;
    B.si = DB.si;
    B.sj = DB.sj;
    B.G = DB.G;
    B.n0 = DB.n[0];
    B.n1 = DB.n[1];
    B.n2 = DB.n[2];
    f(S, B, it);
  }
}

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

__device__ __forceinline__ void shift1(int axis, int &i, int &j, int &k, int s) {
  if (axis == 0) i += s;
  else if (axis == 1) j += s;
  else k += s;
}

// ------------------------------------------------------------------ ideal EMF
__device__ __forceinline__ int bcomp(int axis) { return axis == 0 ? cBX : axis == 1 ? cBY : cBZ; }
__device__ __forceinline__ int bacomp(int axis) { return axis == 0 ? cBAX : axis == 1 ? cBAY : cBAZ; }
__device__ __forceinline__ double face_tot(const V &B, int axis, int i, int j, int k) {
  return AT(bcomp(axis), i, j, k) + AT(bacomp(axis), i, j, k);
}
__device__ __forceinline__ double cell_beta_ind(const V &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return 0.5 * (AT(bcomp(axis), i, j, k) + AT(bcomp(axis), ip, jp, kp));
}
__device__ __forceinline__ double cell_beta_tot(const V &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return 0.5 * (face_tot(B, axis, i, j, k) + face_tot(B, axis, ip, jp, kp));
}
__device__ __forceinline__ double ucon(const V &B, int axis, int i, int j, int k) { return AT(cUC + axis, i, j, k); }

// flux() of AssembleOneDirectionEMF_ (Ideal.cpp:517-536)
__device__ __forceinline__ double emf_flux(const V &B, int ba, int fa, int iL, int jL, int kL, int iR, int jR, int kR,
                                           double bff) {
  const double btL = cell_beta_tot(B, ba, iL, jL, kL), btR = cell_beta_tot(B, ba, iR, jR, kR);
  const double biL = cell_beta_ind(B, ba, iL, jL, kL), biR = cell_beta_ind(B, ba, iR, jR, kR);
  const double ufL = ucon(B, fa, iL, jL, kL), ufR = ucon(B, fa, iR, jR, kR);
  const double ubL = ucon(B, ba, iL, jL, kL), ubR = ucon(B, ba, iR, jR, kR);
  const double GL = ufL * btL - ubL * bff, GR = ufR * btR - ubR * bff;
  const double r = dmax(fabs(ufL), fabs(ufR));
  return 0.5 * (GL + GR) - 0.5 * r * (biR - biL);
}

// AssembleOneDirectionEMF_ (Ideal.cpp:433-594) for all three face families on
// [-1, inner_hi + 1) (the one locally evaluated ghost layer, Ideal.cpp:548-555).
__global__ void __launch_bounds__(kTileThreads) k_face_emf(Dir D) {
  for_items<kExt>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const int q[3] = {i, j, k}, n[3] = {B.n0, B.n1, B.n2};
#pragma unroll 1
    for (int fa = 0; fa < 3; ++fa) {
      bool in = true;
      for (int a = 0; a < 3; ++a) in = in && q[a] < n[a] + (a == fa ? 1 : 0) + 1;
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
      const int64_t o = B.off(i, j, k);
      B.c(ce)[o] = e0;
      B.c(ce + 1)[o] = e1;
      B.c(ce + 2)[o] = e2;
    }
  });
}

__device__ __forceinline__ double max_abs_u4(const V &B, int axis, int i0, int j0, int k0, int i1, int j1, int k1,
                                             int i2, int j2, int k2, int i3, int j3, int k3) {
  double a = 0.0;
  a = dmax(a, fabs(ucon(B, axis, i0, j0, k0)));
  a = dmax(a, fabs(ucon(B, axis, i1, j1, k1)));
  a = dmax(a, fabs(ucon(B, axis, i2, j2, k2)));
  a = dmax(a, fabs(ucon(B, axis, i3, j3, k3)));
  return a;
}
__device__ __forceinline__ double pe_node(const V &B, int i, int j, int k) {
  double sum = 0.0;
  for (int di = -1; di <= 0; ++di)
    for (int dj = -1; dj <= 0; ++dj)
      for (int dk = -1; dk <= 0; ++dk)
        sum += AT(cPVH + 3, i + di, j + dj, k + dk) + AT(cPVN + 3, i + di, j + dj, k + dk);
  return 0.125 * sum;
}

// AssembleEdgeEMF_FromFaceE_Ideal_ (Ideal.cpp:138-372) + AddAmbipolarEdgeEMF_
// (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ambipo.cpp:3-143) on the owned edges.
__global__ void __launch_bounds__(kTileThreads) k_edge_emf(Dir D) {
  for_items<kBox>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const Consts &c = S.c;
    const int i = it.i, j = it.j, k = it.k;
    const double Cuct = 0.5;
    const double pc = (c.rho_ref * c.U_ref) / (c.q_e * c.L_ref * c.B_ref * c.n_ref);
    if (i < B.n0) {
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
        e -= pc * (p1 - p0) / num_limiter(c, 0.25 * rH, 0.25 * rN).ne_eff;
      }
      AT(cEX, i, j, k) = e;
    }
    if (j < B.n1) {
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
        e -= pc * (p1 - p0) / num_limiter(c, 0.25 * rH, 0.25 * rN).ne_eff;
      }
      AT(cEY, i, j, k) = e;
    }
    if (k < B.n2) {
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
        e -= pc * (p1 - p0) / num_limiter(c, 0.25 * rH, 0.25 * rN).ne_eff;
      }
      AT(cEZ, i, j, k) = e;
    }
  });
}

// ------------------------------------------------------------------ Hall EMF
// BuildHallFaceEMF_Rusanov_diff_ step 1 (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:110-146).
__global__ void __launch_bounds__(kTileThreads) k_hall_cell(Dir D) {
  for_items<kAlloc>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const int64_t o = B.off(i, j, k);
    const Num d = num_limiter(S.c, B.c(cUH)[o], B.c(cUN)[o]);
    const double alpha = S.c.hall_coef / d.ne_eff;
    const double Jx = B.c(cJC)[o], Jy = B.c(cJC + 1)[o], Jz = B.c(cJC + 2)[o];
    const double Bx = B.c(cBC)[o], By = B.c(cBC + 1)[o], Bz = B.c(cBC + 2)[o];
    B.c(cEHC)[o] = alpha * (Jy * Bz - Jz * By);
    B.c(cEHC + 1)[o] = alpha * (Jz * Bx - Jx * Bz);
    B.c(cEHC + 2)[o] = alpha * (Jx * By - Jy * Bx);
    B.c(cHB)[o] = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
  });
}

// BuildHallFaceEMF_Rusanov_diff_ steps 2-4 (Hall.cpp:148-400).
__global__ void __launch_bounds__(kTileThreads) k_hall_edge(Dir D) {
  for_items<kBox>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const double eps = 1e-14, Cwh = 0.1;
    if (i < B.n0) {
      double Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = 0.25 * (AT(cEHC + q, i, j - 1, k - 1) + AT(cEHC + q, i, j - 1, k) + AT(cEHC + q, i, j, k - 1) +
                        AT(cEHC + q, i, j, k));
      const double Ecen = Ec[0] * AT(cDRX, i, j, k) + Ec[1] * AT(cDRX + 1, i, j, k) + Ec[2] * AT(cDRX + 2, i, j, k);
      const double be =
          dmax(dmax(AT(cHB, i, j - 1, k - 1), AT(cHB, i, j - 1, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
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
    if (j < B.n1) {
      double Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = 0.25 * (AT(cEHC + q, i - 1, j, k - 1) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j, k - 1) +
                        AT(cEHC + q, i, j, k));
      const double Ecen = Ec[0] * AT(cDRY, i, j, k) + Ec[1] * AT(cDRY + 1, i, j, k) + Ec[2] * AT(cDRY + 2, i, j, k);
      const double be =
          dmax(dmax(AT(cHB, i - 1, j, k - 1), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
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
    if (k < B.n2) {
      double Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = 0.25 * (AT(cEHC + q, i - 1, j - 1, k) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j - 1, k) +
                        AT(cEHC + q, i, j, k));
      const double Ecen = Ec[0] * AT(cDRZ, i, j, k) + Ec[1] * AT(cDRZ + 1, i, j, k) + Ec[2] * AT(cDRZ + 2, i, j, k);
      const double be =
          dmax(dmax(AT(cHB, i - 1, j - 1, k), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j - 1, k), AT(cHB, i, j, k)));
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
  });
}

// E += Ehall on owned edges (Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:135-147).
__global__ void __launch_bounds__(kTileThreads) k_add_hall(Dir D) {
  for_items<kBox>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int64_t o = B.off(it.i, it.j, it.k);
    if (it.i < B.n0) B.c(cEX)[o] += B.c(cHX)[o];
    if (it.j < B.n1) B.c(cEY)[o] += B.c(cHY)[o];
    if (it.k < B.n2) B.c(cEZ)[o] += B.c(cHZ)[o];
  });
}

// ------------------------------------------------------------------ fluid update
// Rusanov face flux of Scheme_U_ (Z4_Mercury/src/physics/MercurySolver_FluidRHS.cpp:36-104).
__device__ __forceinline__ void rusanov(const V &B, double g, int u0, int pv0, double k1, double k2, double k3, int iL,
                                        int jL, int kL, int i, int j, int k, double out[5]) {
  const double rhoL = AT(u0, iL, jL, kL), uL = AT(pv0, iL, jL, kL), vL = AT(pv0 + 1, iL, jL, kL),
               wL = AT(pv0 + 2, iL, jL, kL), pL = AT(pv0 + 3, iL, jL, kL);
  const double rhoR = AT(u0, i, j, k), uR = AT(pv0, i, j, k), vR = AT(pv0 + 1, i, j, k), wR = AT(pv0 + 2, i, j, k),
               pR = AT(pv0 + 3, i, j, k);
  const double reL = pL / (g - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL);
  const double reR = pR / (g - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR);
  const double kk = k1 * k1 + k2 * k2 + k3 * k3;
  const double uvwL = k1 * uL + k2 * vL + k3 * wL, uvwR = k1 * uR + k2 * vR + k3 * wR;
  const double cL = sqrt(dmax(0.0, g * pL / dmax(rhoL, 1e-30))), cR = sqrt(dmax(0.0, g * pR / dmax(rhoR, 1e-30)));
  const double rad = dmax(fabs(uvwL) + cL * sqrt(kk), fabs(uvwR) + cR * sqrt(kk));
  out[0] = 0.5 * (rhoL * uvwL + rhoR * uvwR) - 0.5 * rad * (rhoR - rhoL);
  out[1] = 0.5 * ((rhoL * uvwL * uL + k1 * pL) + (rhoR * uvwR * uR + k1 * pR)) - 0.5 * rad * (rhoR * uR - rhoL * uL);
  out[2] = 0.5 * ((rhoL * uvwL * vL + k2 * pL) + (rhoR * uvwR * vR + k2 * pR)) - 0.5 * rad * (rhoR * vR - rhoL * vL);
  out[3] = 0.5 * ((rhoL * uvwL * wL + k3 * pL) + (rhoR * uvwR * wR + k3 * pR)) - 0.5 * rad * (rhoR * wR - rhoL * wL);
  out[4] = 0.5 * (uvwL * (reL + pL) + uvwR * (reR + pR)) - 0.5 * rad * (reR - reL);
}

// ZeroRHS_ + Scheme_U_ + AddSourceToRHS_Fluid (FluidRHS.cpp:206-527) +
// ApplyUpdate_Euler_ (Z4_Mercury/src/physics/MercurySolver_Advance.cpp:73-147)
// for one owned cell and one ion species; the state goes to the other buffer.
__global__ void __launch_bounds__(kTileThreads, 2) k_fluid(Dir D) {
  for_items<kCells2>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const Consts &c = S.c;
    const double dt = __longlong_as_double((long long)D.state[it.s].dt_bits);
    if (!(dt >= 1e-7) || !isfinite(dt)) return;  // the reference aborts; k_flip records the status
    const int i = it.i, j = it.j, k = it.k, s = it.species;
    const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
    const double g = c.gamma;
    const double invJ = 1.0 / AT(cJAC, i, j, k);
    // r[m] = ((0 - dx[m]/J) - dy[m]/J) - dz[m]/J, accumulated direction by
    // direction (the per-component operation sequence of Scheme_U_'s divergence)
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int dir = 0; dir < 3; ++dir) {
      const int cm = dir == 0 ? cJDX : dir == 1 ? cJDY : cJDZ;
      int ip = i, jp = j, kp = k, im = i, jm = j, km = k;
      shift1(dir, ip, jp, kp, 1);
      shift1(dir, im, jm, km, -1);
      double Fm[5], Fp[5];
      rusanov(B, g, u0, pv0, AT(cm, i, j, k), AT(cm + 1, i, j, k), AT(cm + 2, i, j, k), im, jm, km, i, j, k, Fm);
      rusanov(B, g, u0, pv0, AT(cm, ip, jp, kp), AT(cm + 1, ip, jp, kp), AT(cm + 2, ip, jp, kp), i, j, k, ip, jp, kp,
              Fp);
#pragma unroll
      for (int m = 0; m < 5; ++m) r[m] -= (Fp[m] - Fm[m]) * invJ;
    }
    // sources (FluidRHS.cpp:206-527)
    const double Tn0 = 1000.0, sk1 = 5.0e-5, sk2 = 1.0e-5;
    const double a4 = (c.L_ref / c.U_ref);
    const double a5 = (3.0 * c.L_ref * c.k_Boltz * c.n_ref) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref);
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
    const double x = AT(cCX, i, j, k), y = AT(cCY, i, j, k), z = AT(cCZ, i, j, k);
    const double rho_cyl = sqrt(y * y + z * z);
    const double vst = (x < 0.0 && rho_cyl < 1.0) ? sk2 : sk1;
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
      const double a1_Na = (c.L_ref / c.U_ref) * (c.m_Na / c.rho_ref) * 1e6;
      const double a6 = (1.0e6 * c.L_ref * c.k_Boltz) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref * (c.gamma - 1.0));
      const double sss = AT(cPHOTO, i, j, k);
      r[0] += a1_Na * sss;
      r[4] += a6 * sss * Tn0;
    }
    r[1] -= a4 * rho * u * vst;
    r[2] -= a4 * rho * v * vst;
    r[3] -= a4 * rho * w * vst;
    r[4] -= a4 * rho * u2 * vst;
    r[4] += a5 * nS * b1;
    r[4] += a4 * rho * u2 * b2;
    const int64_t o = B.off(i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m) B.Un[(int64_t)(u0 + m) * B.total + o] = B.U[(int64_t)(u0 + m) * B.total + o] + dt * r[m];
  });
}

// B_face += dt * (-curl E) on the owned faces (CTOperators.cpp:6-56 with multiplier -1).
__global__ void __launch_bounds__(kTileThreads) k_bface(Dir D) {
  for_items<kBox>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const double dt = __longlong_as_double((long long)D.state[it.s].dt_bits);
    if (!(dt >= 1e-7) || !isfinite(dt)) return;
    const int i = it.i, j = it.j, k = it.k;
    if (j < B.n1 && k < B.n2) {
      const double rb = -1.0 * ((AT(cEY, i, j, k) - AT(cEY, i, j, k + 1)) + (AT(cEZ, i, j + 1, k) - AT(cEZ, i, j, k)));
      AT(cBX, i, j, k) += dt * rb;
    }
    if (i < B.n0 && k < B.n2) {
      const double rb = -1.0 * ((AT(cEX, i, j, k + 1) - AT(cEX, i, j, k)) + (AT(cEZ, i, j, k) - AT(cEZ, i + 1, j, k)));
      AT(cBY, i, j, k) += dt * rb;
    }
    if (i < B.n0 && j < B.n1) {
      const double rb = -1.0 * ((AT(cEX, i, j, k) - AT(cEX, i, j + 1, k)) + (AT(cEY, i + 1, j, k) - AT(cEY, i, j, k)));
      AT(cBZ, i, j, k) += dt * rb;
    }
  });
}

// ------------------------------------------------------------------ derived fields
// calc_Bcell (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:3-90) on owned cells and
// CurlAdjFaceToEdge + alpha scaling of Calc_J_Edge (CTOperators.cpp:59-110,
// Z4_Mercury/src/physics/MercurySolver_Current.cpp:140-190) on owned edges.
__global__ void __launch_bounds__(kTileThreads) k_bcell_jedge(Dir D) {
  for_items<kBox>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    if (i < B.n0 && j < B.n1 && k < B.n2) {
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
      const int64_t o = B.off(i, j, k);
      B.c(cBC)[o] = bxt;
      B.c(cBC + 1)[o] = byt;
      B.c(cBC + 2)[o] = bzt;
      B.c(cBIC)[o] = bxi;
      B.c(cBIC + 1)[o] = byi;
      B.c(cBIC + 2)[o] = bzi;
    }
    if (i < B.n0) {
      const double v = ((AT(cBFY, i, j, k - 1) * AT(cBY, i, j, k - 1) - AT(cBFY, i, j, k) * AT(cBY, i, j, k)) +
                        (AT(cBFZ, i, j, k) * AT(cBZ, i, j, k) - AT(cBFZ, i, j - 1, k) * AT(cBZ, i, j - 1, k))) * 1.0;
      AT(cJX, i, j, k) = v * AT(cALX, i, j, k);
    }
    if (j < B.n1) {
      const double v = ((AT(cBFX, i, j, k) * AT(cBX, i, j, k) - AT(cBFX, i, j, k - 1) * AT(cBX, i, j, k - 1)) +
                        (AT(cBFZ, i - 1, j, k) * AT(cBZ, i - 1, j, k) - AT(cBFZ, i, j, k) * AT(cBZ, i, j, k))) * 1.0;
      AT(cJY, i, j, k) = v * AT(cALY, i, j, k);
    }
    if (k < B.n2) {
      const double v = ((AT(cBFX, i, j - 1, k) * AT(cBX, i, j - 1, k) - AT(cBFX, i, j, k) * AT(cBX, i, j, k)) +
                        (AT(cBFY, i, j, k) * AT(cBY, i, j, k) - AT(cBFY, i - 1, j, k) * AT(cBY, i - 1, j, k))) * 1.0;
      AT(cJZ, i, j, k) = v * AT(cALZ, i, j, k);
    }
  });
}

// calc_Jcell (Current.cpp:203-243), owned cells.
__global__ void __launch_bounds__(kTileThreads) k_jcell(Dir D) {
  for_items<kCells>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
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
    const int64_t o = B.off(i, j, k);
    B.c(cJC)[o] = jx;
    B.c(cJC + 1)[o] = jy;
    B.c(cJC + 2)[o] = jz;
  });
}

// CFL time step of one cell and both species (Compute_Timestep,
// Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:8-141).
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
__device__ __forceinline__ double cell_dt(const V &B, const Consts &c, int i, int j, int k) {
  double dtl = 1e100;
  const double Vol = fabs(AT(cJAC, i, j, k));
  if (!(Vol > 0.0)) return dtl;
  const double Bx = AT(cBC, i, j, k), By = AT(cBC + 1, i, j, k), Bz = AT(cBC + 2, i, j, k);
  const double B2 = Bx * Bx + By * By + Bz * Bz;
  for (int s = 0; s < 2; ++s) {
    const int u0 = s ? cUN : cUH;
    const double rho = dmax(AT(u0, i, j, k), 1e-2);
    const double ux = AT(u0 + 1, i, j, k) / rho, uy = AT(u0 + 2, i, j, k) / rho, uz = AT(u0 + 3, i, j, k) / rho;
    const double E = AT(u0 + 4, i, j, k);
    const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
    const double pr = (c.gamma - 1.0) * (E - ke);
    const double cs2 = c.gamma * pr / rho;
    double den = 0.0;
    den += face_term(c, AT(cJDX, i, j, k), AT(cJDX + 1, i, j, k), AT(cJDX + 2, i, j, k), false, ux, uy, uz, Bx, By, Bz,
                     B2, rho, cs2);
    den += face_term(c, AT(cJDX, i + 1, j, k), AT(cJDX + 1, i + 1, j, k), AT(cJDX + 2, i + 1, j, k), true, ux, uy, uz, Bx,
                     By, Bz, B2, rho, cs2);
    den += face_term(c, AT(cJDY, i, j, k), AT(cJDY + 1, i, j, k), AT(cJDY + 2, i, j, k), false, ux, uy, uz, Bx, By, Bz,
                     B2, rho, cs2);
    den += face_term(c, AT(cJDY, i, j + 1, k), AT(cJDY + 1, i, j + 1, k), AT(cJDY + 2, i, j + 1, k), true, ux, uy, uz, Bx,
                     By, Bz, B2, rho, cs2);
    den += face_term(c, AT(cJDZ, i, j, k), AT(cJDZ + 1, i, j, k), AT(cJDZ + 2, i, j, k), false, ux, uy, uz, Bx, By, Bz,
                     B2, rho, cs2);
    den += face_term(c, AT(cJDZ, i, j, k + 1), AT(cJDZ + 1, i, j, k + 1), AT(cJDZ + 2, i, j, k + 1), true, ux, uy, uz, Bx,
                     By, Bz, B2, rho, cs2);
    if (den > 0.0) dtl = dmin(dtl, c.CFL * Vol / den);
  }
  return dtl;
}

// calc_PV + calc_Uplus (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:159-301) on the allocated
// cell range, the contravariant velocities UCON where the Jacobian exists
// ([-(g-1), n + g - 1)), and the next step's CFL dt on owned cells (CTA min,
// one atomicMin per tile on the positive-double bit pattern).
__global__ void __launch_bounds__(kTileThreads, 2) k_pv_uplus(Dir D) {
  __shared__ double red[kTileThreads / 32];
  for_items<kAlloc>(D, [&](const DevSolve &S, const V &B, const Item &it) {
    const Consts &c = S.c;
    const int i = it.i, j = it.j, k = it.k;
    double dtl = 1e100;
    if (it.in) {
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
        const int64_t o = B.off(i, j, k);
        B.c(pv0)[o] = u;
        B.c(pv0 + 1)[o] = v;
        B.c(pv0 + 2)[o] = w;
        B.c(pv0 + 3)[o] = pr;
        B.c(pv0 + 4)[o] = T;
        vel[s][0] = u;
        vel[s][1] = v;
        vel[s][2] = w;
      }
      const double rH = dmax(AT(cUH, i, j, k), 0.0), rN = dmax(AT(cUN, i, j, k), 0.0);
      const Num d = num_limiter(c, rH, rN);
      double up[3];
      for (int q = 0; q < 3; ++q) {
        const double uH = rH > 1e-20 ? vel[0][q] : 0.0;
        const double uN = rN > 1e-20 ? vel[1][q] : 0.0;
        up[q] = d.chiH * uH + d.chiNa * uN;
        AT(cUP + q, i, j, k) = up[q];
      }
      const int gm = c.nghost - 1;
      if (i >= -gm && i < B.n0 + gm && j >= -gm && j < B.n1 + gm && k >= -gm && k < B.n2 + gm) {
        const double inv_jac = 1.0 / (fabs(AT(cJAC, i, j, k)) + 1.0e-30);
        for (int axis = 0; axis < 3; ++axis) {
          int ip = i, jp = j, kp = k;
          shift1(axis, ip, jp, kp, 1);
          const int cm = axis == 0 ? cJDX : axis == 1 ? cJDY : cJDZ;
          const double kx = 0.5 * (AT(cm, i, j, k) + AT(cm, ip, jp, kp));
          const double ky = 0.5 * (AT(cm + 1, i, j, k) + AT(cm + 1, ip, jp, kp));
          const double kz = 0.5 * (AT(cm + 2, i, j, k) + AT(cm + 2, ip, jp, kp));
          AT(cUC + axis, i, j, k) = (kx * up[0] + ky * up[1] + kz * up[2]) * inv_jac;
        }
      }
      if (i >= 0 && i < B.n0 && j >= 0 && j < B.n1 && k >= 0 && k < B.n2) dtl = cell_dt(B, c, i, j, k);
    }
    for (int o = 16; o > 0; o >>= 1) dtl = dmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dtl;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < kTileThreads / 32 ? red[threadIdx.x] : 1e100;
      for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (threadIdx.x == 0 && v < 1e100)
        atomicMin(&D.state[it.s].dt_bits, (unsigned long long)__double_as_longlong(v));
    }
    __syncthreads();
  });
}

#undef AT

// ------------------------------------------------------------------ sync, alias, bookkeeping
__device__ __forceinline__ int find_solve(const int *prefix, int nsolves, int e) {
  int lo = 0, hi = nsolves;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ double *decode(const DevSolve &S, int cur, int64_t code) {
  const int blk = (int)(code >> 48);
  const int comp = (int)((code >> 40) & 0xff);
  const int64_t off = code & ((int64_t(1) << 40) - 1);
  const DevBlock &DB = S.blocks[blk];
  return comp < kNumUComps ? DB.U[cur] + (int64_t)comp * DB.total + off
                           : DB.M + (int64_t)(comp - kNumUComps) * DB.total + off;
}

// One sync phase (halo or owner copies) of group g for every active solve:
// dst <- sign * src (MercuryBoundary::Sync_, Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110).
__global__ void k_copy(Dir D, int g, int phase) {
  const int *pre = D.copy_prefix[g][phase];
  const int total = pre[D.nsolves];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int s = find_solve(pre, D.nsolves, e);
    if (!solve_active(D, s)) continue;
    const DevSolve &S = D.solves[s];
    const DevTable &T = phase ? S.owner[g] : S.halo[g];
    const int q = e - pre[s];
    const int cur = D.state[s].cur;
    *decode(S, cur, T.dst[q]) = T.sign[q] * *decode(S, cur, T.src[q]);
  }
}

// ReduceEdgeAliasCandidatesToOwners_ (Z4_Mercury/src/physics/MercurySolver_Current.cpp:3-57):
// one thread per class, members summed in stored order from 0.0.  which = 0: E, 1: J.
__global__ void k_alias(Dir D, int which) {
  const int *pre = which ? D.aliasJ_prefix : D.aliasE_prefix;
  const int total = pre[D.nsolves];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int s = find_solve(pre, D.nsolves, e);
    if (!solve_active(D, s)) continue;
    const DevSolve &S = D.solves[s];
    const DevAlias &A = which ? S.aliasJ : S.aliasE;
    const int q = e - pre[s];
    const int cur = D.state[s].cur;
    double sum = 0.0;
    for (int m = A.offset[q]; m < A.offset[q + 1]; ++m) sum += A.msign[m] * *decode(S, cur, A.member[m]);
    *decode(S, cur, A.owner[q]) = A.osign[q] * sum / (double)(A.offset[q + 1] - A.offset[q]);
  }
}

// After the updates: flip the state buffer, account time/step
// (Z4_Mercury/src/MercurySolver_Driver.cpp:40-45), record a dt failure (the
// reference's exit(-1), Timestep.cpp:129-140) and re-arm the dt reduction.
__global__ void k_flip(Dir D) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < D.nsolves; s += gridDim.x * blockDim.x) {
    SolveState &st = D.state[s];
    if (!st.remaining) continue;
    const double dt = __longlong_as_double((long long)st.dt_bits);
    if (!(dt >= 1e-7) || !isfinite(dt)) {
      st.status = MHD_ERR_DT;
      st.remaining = 0;
      continue;
    }
    st.cur ^= 1;
    st.dt = dt;
    st.time += dt;
    st.step += 1;
    st.dt_bits = (unsigned long long)__double_as_longlong(1e100);
  }
}

// End of a step: one step fewer to go (after every pass of the step has run).
__global__ void k_retire(Dir D) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < D.nsolves; s += gridDim.x * blockDim.x) {
    SolveState &st = D.state[s];
    if (st.remaining > 0) st.remaining -= 1;
  }
}

}  // namespace

// ------------------------------------------------------------------ launchers
static int g_grid_tiles = 0, g_grid_copy = 0;
static void grids() {
  if (g_grid_tiles) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  g_grid_tiles = sms * 8;  // persistent: up to 8 resident 256-thread CTAs per SM
  g_grid_copy = sms * 8;
}

void launch_step_kernel(StepKernel k, const Dir &D, cudaStream_t st, int arg0, int arg1) {
  grids();
  switch (k) {
    case SK_FACE_EMF: k_face_emf<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_EDGE_EMF: k_edge_emf<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_HALL_CELL: k_hall_cell<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_HALL_EDGE: k_hall_edge<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_ADD_HALL: k_add_hall<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_FLUID: k_fluid<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_BFACE: k_bface<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_BCELL_JEDGE: k_bcell_jedge<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_JCELL: k_jcell<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_PV_UPLUS: k_pv_uplus<<<g_grid_tiles, kTileThreads, 0, st>>>(D); break;
    case SK_COPY: k_copy<<<g_grid_copy, 256, 0, st>>>(D, arg0, arg1); break;
    case SK_ALIAS: k_alias<<<g_grid_copy, 128, 0, st>>>(D, arg0); break;
    case SK_FLIP: k_flip<<<1, 128, 0, st>>>(D); break;
    case SK_RETIRE: k_retire<<<1, 128, 0, st>>>(D); break;
    default: break;
  }
}

const char *step_kernel_name(StepKernel k) {
  static const char *names[] = {"k_face_emf", "k_edge_emf", "k_hall_cell", "k_hall_edge", "k_add_hall",
                                "k_fluid",    "k_bface",    "k_bcell_jedge", "k_jcell",   "k_pv_uplus",
                                "k_copy",     "k_alias",    "k_flip",        "k_retire"};
  return (k >= 0 && k < SK_COUNT) ? names[k] : "?";
}

}  // namespace mhd
