// Per-solve setup on the device: the static fields of one block computed
// from its node coordinates, with the reference's formulas in the operation
// order of the host setup (mpcns_mercury_b200/setup.py), which is pinned
// against the reference build:
//   cell centres (dual grid)      Block::calc_Dual_Grids    src/1_grid/1_MPCNS_Grid_GCL.cpp:6-21
//   face area vectors JD, Jac     compute_metric_fields     src/7_metric/Metric.cpp:108-326
//   |S|, |l*|, beta = |l*|/|S|    (faces)                   src/7_metric/Metric.cpp:398-474
//   |e|, |S*|, alpha = |e|/|S*|   (edges, dual-collapse cap) src/7_metric/Metric.cpp:476-669
//   edge vectors dr                                         src/7_metric/Metric.cpp:1261-1328
//   B_cell / J_cell weights       SetupCellReconstructionWeights_
//                                 Z4_Mercury/src/MercurySolver_ReconstructionSetup.cpp:29-193
//   photo-production rate         Initial_Na_And_PhotoRate_ Z4_Mercury/include/2_Initial.h:227-440
// Built with FMA contraction off and IEEE division and square root; the
// Jacobi rotations and the photo rate call the device's atan2 / sin / cos /
// acos / exp, so those fields can differ from the host's in the last bits.
// Each field is written over the range the host setup fills; the background
// field (no dipole, no IMF) is zero and the Hall radial taper is off (1 on
// the owned edges), as in the host setup of the periodic blocks.
#include <cmath>

#include "mhd_geometry.cuh"

namespace mhd {
namespace {

struct P3 {
  double v[3];
};

struct Geo {
  const double *X, *Y, *Z;
  GeoBox b;
  __device__ __forceinline__ int64_t off(int i, int j, int k) const {
    return (int64_t)(i + b.G) * b.si + (int64_t)(j + b.G) * b.sj + (k + b.G);
  }
  __device__ __forceinline__ P3 node(int i, int j, int k) const {
    const int64_t o = off(i, j, k);
    return P3{{X[o], Y[o], Z[o]}};
  }
  // dual point (I, J, K): the mean of the 8 nodes (I - 1 .. I) x ..., summed
  // in the order of Block::calc_Dual_Grids; the centre of cell (I-1, J-1, K-1)
  __device__ __forceinline__ P3 dual(int I, int J, int K) const {
    const P3 a = node(I, J, K), b1 = node(I - 1, J, K), c = node(I, J - 1, K), d = node(I - 1, J - 1, K),
             e = node(I, J, K - 1), f = node(I - 1, J, K - 1), g = node(I, J - 1, K - 1), h = node(I - 1, J - 1, K - 1);
    P3 r;
    for (int q = 0; q < 3; ++q)
      r.v[q] = 0.125 * (a.v[q] + b1.v[q] + c.v[q] + d.v[q] + e.v[q] + f.v[q] + g.v[q] + h.v[q]);
    return r;
  }
};

__device__ __forceinline__ P3 sub(const P3 &a, const P3 &b) { return P3{{a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]}}; }
__device__ __forceinline__ P3 cross(const P3 &a, const P3 &b) {
  return P3{{a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2], a.v[0] * b.v[1] - a.v[1] * b.v[0]}};
}
__device__ __forceinline__ double norm(const P3 &a) { return sqrt(a.v[0] * a.v[0] + a.v[1] * a.v[1] + a.v[2] * a.v[2]); }
__device__ __forceinline__ double vmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double vmin(double a, double b) { return b < a ? b : a; }

// Face area vector of face family `dir` at (i, j, k): half the sum of the
// cross products of its two diagonal frames (Metric.cpp:108-200).
__device__ P3 face_jd(const Geo &g, int dir, int i, int j, int k) {
  static constexpr int oxp[3][3] = {{0, 1, 0}, {0, 0, 1}, {1, 0, 0}};
  static constexpr int oyp[3][3] = {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}};
  static constexpr int oxy[3][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
  const P3 o = g.node(i, j, k);
  const P3 xp = g.node(i + oxp[dir][0], j + oxp[dir][1], k + oxp[dir][2]);
  const P3 yp = g.node(i + oyp[dir][0], j + oyp[dir][1], k + oyp[dir][2]);
  const P3 xyp = g.node(i + oxy[dir][0], j + oxy[dir][1], k + oxy[dir][2]);
  const P3 c1 = cross(sub(xp, o), sub(yp, o)), c2 = cross(sub(yp, xyp), sub(xp, xyp));
  P3 r;
  for (int q = 0; q < 3; ++q) r.v[q] = 0.5 * (c1.v[q] + c2.v[q]);
  return r;
}

// Pseudo-inverse of a symmetric 3x3 matrix by 18 sweeps of cyclic Jacobi
// rotations, dropping eigenvalues below 1e-10 of the largest
// (ReconstructionSetup.cpp:33-66,123-133).
__device__ void pinv_sym3(double A[3][3], double Minv[3][3]) {
  double V[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  for (int sweep = 0; sweep < 18; ++sweep)
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A[p][q];
        const bool skip = fabs(apq) <= 1.0e-16 * (fabs(A[p][p]) + fabs(A[q][q]) + 1.0);
        if (skip) continue;
        const double phi = 0.5 * atan2(2.0 * apq, A[q][q] - A[p][p]);
        const double c = cos(phi), s = sin(phi);
        const double app = A[p][p], aqq = A[q][q];
        const int r = 3 - p - q;
        const double akp = A[r][p], akq = A[r][q];
        A[r][p] = c * akp - s * akq;
        A[p][r] = A[r][p];
        A[r][q] = s * akp + c * akq;
        A[q][r] = A[r][q];
        A[p][p] = c * c * app - 2.0 * s * c * apq + s * s * aqq;
        A[q][q] = s * s * app + 2.0 * s * c * apq + c * c * aqq;
        A[p][q] = 0.0;
        A[q][p] = 0.0;
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  const double lam[3] = {A[0][0], A[1][1], A[2][2]};
  const double lmax = vmax(lam[0], vmax(lam[1], lam[2]));
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) Minv[a][c] = 0.0;
  for (int q = 0; q < 3; ++q) {
    const double inv = lam[q] > 1.0e-10 * lmax ? 1.0 / lam[q] : 0.0;
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) Minv[a][c] = Minv[a][c] + V[a][q] * inv * V[c][q];
  }
  if (lmax <= 1.0e-30)
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) Minv[a][c] = 0.0;
}

struct Out {
  void *const *p;
  bool fp32;
  int64_t o;
  __device__ __forceinline__ void put(int comp, double v) const {
    if (!p[comp]) return;  // a field the solve does not hold
    if (comp < kGeoMetric || !fp32) ((double *)p[comp])[o] = v;
    else ((float *)p[comp])[o] = (float)v;
  }
};

__device__ __forceinline__ bool in3(int i, int j, int k, const int lo[3], const int hi[3]) {
  return i >= lo[0] && i < hi[0] && j >= lo[1] && j < hi[1] && k >= lo[2] && k < hi[2];
}

__global__ void k_geometry(Geo g, void *const *outp, bool fp32, double L_ref) {
  const GeoBox &b = g.b;
  const int ei = b.n[0] + 1 + 2 * b.G, ej = b.n[1] + 1 + 2 * b.G, ek = b.n[2] + 1 + 2 * b.G;
  const int64_t npos = (int64_t)ei * ej * ek;
  const int gh = b.nghost;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npos; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % ek) - b.G, j = (int)((t / ek) % ej) - b.G, i = (int)(t / ((int64_t)ek * ej)) - b.G;
    const Out out{outp, fp32, g.off(i, j, k)};
    const int n[3] = {b.n[0], b.n[1], b.n[2]};
    // cell centres, cells [-g - 1, n + g)
    {
      const int lo[3] = {-gh - 1, -gh - 1, -gh - 1}, hi[3] = {n[0] + gh, n[1] + gh, n[2] + gh};
      if (in3(i, j, k, lo, hi)) {
        const P3 c = g.dual(i + 1, j + 1, k + 1);
        for (int q = 0; q < 3; ++q) out.put(GEO_CELL + q, c.v[q]);
      }
    }
    // face area vectors, faces [-g, n + stagger + g)
    for (int dir = 0; dir < 3; ++dir) {
      const int lo[3] = {-gh, -gh, -gh};
      const int hi[3] = {n[0] + gh + (dir == 0), n[1] + gh + (dir == 1), n[2] + gh + (dir == 2)};
      if (in3(i, j, k, lo, hi)) {
        const P3 a = face_jd(g, dir, i, j, k);
        for (int q = 0; q < 3; ++q) out.put(GEO_JD + 3 * dir + q, a.v[q]);
      }
    }
    // cell volume, cells [-(g - 1), n + g - 1): one third of the outward
    // flux of the position vector through the six faces (Metric.cpp:202-326)
    {
      const int lo[3] = {-(gh - 1), -(gh - 1), -(gh - 1)}, hi[3] = {n[0] + gh - 1, n[1] + gh - 1, n[2] + gh - 1};
      if (in3(i, j, k, lo, hi)) {
        const P3 xc = g.dual(i + 1, j + 1, k + 1);
        // (face family, +1 for the upper face, four corner offsets)
        static constexpr int fo[6][4][3] = {
            {{0, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}}, {{1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}},
            {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {1, 0, 1}}, {{0, 1, 0}, {1, 1, 0}, {0, 1, 1}, {1, 1, 1}},
            {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}}, {{0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}}};
        double V = 0.0;
        for (int f = 0; f < 6; ++f) {
          const int dir = f >> 1, up = f & 1;
          P3 Af = face_jd(g, dir, i + (dir == 0 ? up : 0), j + (dir == 1 ? up : 0), k + (dir == 2 ? up : 0));
          P3 nd[4];
          for (int c = 0; c < 4; ++c) nd[c] = g.node(i + fo[f][c][0], j + fo[f][c][1], k + fo[f][c][2]);
          double d[3];
          for (int q = 0; q < 3; ++q) {
            const double fc = 0.25 * (nd[0].v[q] + nd[1].v[q] + nd[2].v[q] + nd[3].v[q]);
            d[q] = fc - xc.v[q];
            if (!up) Af.v[q] = -Af.v[q];
          }
          V = V + (Af.v[0] * d[0] + Af.v[1] * d[1] + Af.v[2] * d[2]);
        }
        out.put(GEO_JAC, V / 3.0);
      }
    }
    // face area magnitude and Hodge ratio, faces [-(g - 1), n + stagger + g - 1)
    for (int dir = 0; dir < 3; ++dir) {
      const int lo[3] = {-(gh - 1), -(gh - 1), -(gh - 1)};
      const int hi[3] = {n[0] + gh - 1 + (dir == 0), n[1] + gh - 1 + (dir == 1), n[2] + gh - 1 + (dir == 2)};
      if (!in3(i, j, k, lo, hi)) continue;
      const double Smag = norm(face_jd(g, dir, i, j, k));
      const P3 cL = g.dual(i + (dir == 0 ? 0 : 1), j + (dir == 1 ? 0 : 1), k + (dir == 2 ? 0 : 1));
      const P3 cR = g.dual(i + 1, j + 1, k + 1);
      const double L = norm(sub(cR, cL));
      out.put(GEO_AREA + dir, Smag);
      out.put(GEO_BETA + dir, Smag < 1e-25 ? 0.0 : L / Smag);
    }
    // edge vectors, lengths and Hodge ratios, edges [-(g - 1), n + stagger + g - 1)
    for (int ax = 0; ax < 3; ++ax) {
      const int lo[3] = {-(gh - 1), -(gh - 1), -(gh - 1)};
      const int hi[3] = {n[0] + gh - 1 + (ax != 0), n[1] + gh - 1 + (ax != 1), n[2] + gh - 1 + (ax != 2)};
      if (!in3(i, j, k, lo, hi)) continue;
      // dual points around the edge: p00, p10, p01, p11 offsets
      static constexpr int od[3][4][3] = {{{1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}},
                                          {{0, 1, 0}, {1, 1, 0}, {0, 1, 1}, {1, 1, 1}},
                                          {{0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}}};
      const P3 r0 = g.node(i, j, k), r1 = g.node(i + (ax == 0), j + (ax == 1), k + (ax == 2));
      const P3 dr = sub(r1, r0);
      const double L = norm(dr);
      P3 pp[4];
      for (int c = 0; c < 4; ++c) pp[c] = g.dual(i + od[ax][c][0], j + od[ax][c][1], k + od[ax][c][2]);
      const P3 a0 = cross(sub(pp[1], pp[0]), sub(pp[2], pp[0]));
      const P3 a1 = cross(sub(pp[2], pp[3]), sub(pp[1], pp[3]));
      P3 Av;
      for (int q = 0; q < 3; ++q) Av.v[q] = 0.5 * (a0.v[q] + a1.v[q]);
      const double Amag = norm(Av);
      const double eps = 1e-25, ratio = 1e-3, abs_tol = 1e-12;
      const double raw = Amag < eps ? 0.0 : L / Amag;
      const double d00_10 = norm(sub(pp[1], pp[0])), d00_01 = norm(sub(pp[2], pp[0]));
      const double d10_11 = norm(sub(pp[3], pp[1])), d01_11 = norm(sub(pp[3], pp[2]));
      const double d00_11 = norm(sub(pp[3], pp[0])), d10_01 = norm(sub(pp[2], pp[1]));
      const double href = vmax(vmax(vmax(d00_10, d00_01), vmax(d10_11, d01_11)),
                               vmax(vmax(d00_11, d10_01), vmax(L, eps)));
      const double side_min = vmin(vmin(d00_10, d00_01), vmin(d10_11, d01_11));
      const double diag_min = vmin(d00_11, d10_01);
      const bool touch = (L < abs_tol) || (side_min < ratio * href) || (diag_min < ratio * href) ||
                         (Amag < ratio * href * href);
      out.put(GEO_DL + ax, L);
      for (int q = 0; q < 3; ++q) out.put(GEO_DR + 3 * ax + q, dr.v[q]);
      out.put(GEO_ALPHA + ax, touch ? 0.0 : raw);
    }
    // background field: zero on the faces [-g, n + stagger + g)
    for (int dir = 0; dir < 3; ++dir) {
      const int lo[3] = {-gh, -gh, -gh};
      const int hi[3] = {n[0] + gh + (dir == 0), n[1] + gh + (dir == 1), n[2] + gh + (dir == 2)};
      if (in3(i, j, k, lo, hi)) out.put(GEO_BADD + dir, 0.0);
    }
    // Hall radial taper (off): 1 on the owned edges, 0 on the rest of [-g, n + stagger + g)
    for (int ax = 0; ax < 3; ++ax) {
      const int lo[3] = {-gh, -gh, -gh};
      const int hi[3] = {n[0] + gh + (ax != 0), n[1] + gh + (ax != 1), n[2] + gh + (ax != 2)};
      if (!in3(i, j, k, lo, hi)) continue;
      const int olo[3] = {0, 0, 0}, ohi[3] = {n[0] + (ax != 0), n[1] + (ax != 1), n[2] + (ax != 2)};
      out.put(GEO_TAPER + ax, in3(i, j, k, olo, ohi) ? 1.0 : 0.0);
    }
    // cell range [-g, n + g): reconstruction weights (owned cells; zero on
    // the rest) and the photo-production rate
    const int clo[3] = {-gh, -gh, -gh}, chi[3] = {n[0] + gh, n[1] + gh, n[2] + gh};
    if (!in3(i, j, k, clo, chi)) continue;
    const int olo[3] = {0, 0, 0};
    out.put(GEO_TAPER_CELL, in3(i, j, k, olo, n) ? 1.0 : 0.0);  // the taper at cell centres (off)
    if (in3(i, j, k, olo, n)) {
      // B_cell weights from the six oriented face area vectors
      P3 s[6];
      for (int dir = 0; dir < 3; ++dir) {
        const P3 lo_f = face_jd(g, dir, i, j, k);
        const P3 hi_f = face_jd(g, dir, i + (dir == 0), j + (dir == 1), k + (dir == 2));
        for (int q = 0; q < 3; ++q) {
          s[2 * dir].v[q] = -lo_f.v[q];
          s[2 * dir + 1].v[q] = hi_f.v[q];
        }
      }
      static constexpr int n8[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                       {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
      P3 nd[8];
      for (int c = 0; c < 8; ++c) nd[c] = g.node(i + n8[c][0], j + n8[c][1], k + n8[c][2]);
      P3 xc;
      for (int q = 0; q < 3; ++q)
        xc.v[q] = 0.125 * (nd[0].v[q] + nd[1].v[q] + nd[2].v[q] + nd[3].v[q] + nd[4].v[q] + nd[5].v[q] +
                           nd[6].v[q] + nd[7].v[q]);
      static constexpr int fs[6][4] = {{0, 2, 4, 6}, {1, 3, 5, 7}, {0, 1, 4, 5}, {2, 3, 6, 7}, {0, 1, 2, 3}, {4, 5, 6, 7}};
      double mu[6], smag[6], sref = 0.0;
      for (int q = 0; q < 6; ++q) {
        P3 d;
        for (int a = 0; a < 3; ++a) {
          const double fc = 0.25 * (nd[fs[q][0]].v[a] + nd[fs[q][1]].v[a] + nd[fs[q][2]].v[a] + nd[fs[q][3]].v[a]);
          d.v[a] = fc - xc.v[a];
        }
        mu[q] = 1.0 / vmax(norm(d), 1.0e-14);
        smag[q] = norm(s[q]);
        sref = vmax(sref, smag[q]);
      }
      double M[3][3] = {}, Minv[3][3];
      for (int q = 0; q < 6; ++q) {
        const bool active = smag[q] > 1.0e-10 * sref;
        const double w = active ? mu[q] : 0.0;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) M[a][c] = M[a][c] + (active ? w * s[q].v[a] * s[q].v[c] : 0.0);
      }
      pinv_sym3(M, Minv);
      for (int q = 0; q < 6; ++q) {
        const bool active = smag[q] > 1.0e-10 * sref;
        for (int a = 0; a < 3; ++a) {
          const double val =
              mu[q] * (Minv[a][0] * s[q].v[0] + Minv[a][1] * s[q].v[1] + Minv[a][2] * s[q].v[2]);
          out.put(GEO_WB + 6 * a + q, active ? val : 0.0);
        }
      }
      // J_cell weights from the 12 edge vectors
      static constexpr int ed[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                        {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
      P3 l[12];
      double ln[12], lmax = 0.0;
      for (int q = 0; q < 12; ++q) {
        l[q] = sub(nd[ed[q][1]], nd[ed[q][0]]);
        ln[q] = norm(l[q]);
        lmax = vmax(lmax, ln[q]);
      }
      double MJ[3][3] = {}, MJinv[3][3];
      for (int q = 0; q < 12; ++q) {
        const bool active = ln[q] > 1.0e-10 * lmax;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) MJ[a][c] = MJ[a][c] + (active ? l[q].v[a] * l[q].v[c] : 0.0);
      }
      pinv_sym3(MJ, MJinv);
      for (int q = 0; q < 12; ++q) {
        const bool active = ln[q] > 1.0e-10 * lmax;
        for (int a = 0; a < 3; ++a) {
          const double val = MJinv[a][0] * l[q].v[0] + MJinv[a][1] * l[q].v[1] + MJinv[a][2] * l[q].v[2];
          out.put(GEO_WJ + 12 * a + q, active ? val : 0.0);
        }
      }
    } else {
      for (int q = 0; q < 18; ++q) out.put(GEO_WB + q, 0.0);
      for (int q = 0; q < 36; ++q) out.put(GEO_WJ + q, 0.0);
    }
    // neutral Na exosphere and Na+ photo-production rate at the cell centre
    {
      const P3 c = g.dual(i + 1, j + 1, k + 1);
      const double x = c.v[0], y = c.v[1], z = c.v[2];
      const double sk1 = 5.0e-5, sk2 = 1.0e-5;
      const double pi = acos(-1.0), deg = pi / 180.0;
      const double r = sqrt(x * x + y * y + z * z);
      const bool outside = (r > 1.0) && isfinite(r);
      const double rs = outside ? r : 2.0;
      const double inv_r = 1.0 / rs;
      const double rx = x * inv_r, ry = y * inv_r, rz = z * inv_r;
      const double drr = L_ref * rs - L_ref;
      const double r_factor = 1.0 / (rs * rs);
      auto delta = [&](double lat, double lon) {
        const double clat = cos(lat);
        const double px = clat * cos(lon), py = clat * sin(lon), pz = sin(lat);
        return acos(vmin(vmax(rx * px + ry * py + rz * pz, -1.0), 1.0));
      };
      auto gauss2 = [](double d, double H) {
        const double a = d / H;
        return exp(-(a * a));
      };
      const double n_miv = 7.84e6 * exp(-drr / 431.0e3);
      const double n_td = 8.86e9 * exp(-drr / 100.0e3) * gauss2(delta(0.0, 0.0), 15.0 * deg);
      const double rad_psd = 4.06e10 * exp(-drr / 232.0e3);
      const double n_psd = rad_psd * (gauss2(delta(50.0 * deg, 0.0), 20.0 * deg) + gauss2(delta(-50.0 * deg, 0.0), 20.0 * deg));
      const double rad_sp = 5.67e6 * exp(-drr / 748.0e3);
      const double n_sp_day = rad_sp * (gauss2(delta(80.0 * deg, 0.0), 15.0 * deg) + gauss2(delta(-80.0 * deg, 0.0), 15.0 * deg));
      const double n_sp_night = rad_sp * (gauss2(delta(15.0 * deg, pi), 10.0 * deg) + gauss2(delta(-15.0 * deg, pi), 10.0 * deg));
      double n_m3 = r_factor * (n_miv + n_td + n_psd + n_sp_day + n_sp_night);
      if (!(isfinite(n_m3) && n_m3 >= 0.0)) n_m3 = 0.0;
      const double n_cm3 = outside ? n_m3 * 1.0e-6 : 0.0;
      const bool shadow = (x < 0.0) && (sqrt(y * y + z * z) < 1.0);
      double q = (shadow ? sk2 : sk1) * n_cm3;
      if (!(isfinite(q) && q >= 0.0)) q = 0.0;
      out.put(GEO_PHOTO, q);
    }
  }
}

// The Hall radial taper at (x, y, z) (HallRadialTaper_,
// Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:6-13).
__device__ double hall_taper(const GeoBg &bg, double x, double y, double z) {
  const double r = sqrt(x * x + y * y + z * z);
  const double width = bg.hall_r_max - bg.hall_r_min;
  if (width <= 0.0) return (r >= bg.hall_r_min) ? 1.0 : 0.0;
  const double mid = 0.5 * (bg.hall_r_min + bg.hall_r_max);
  return 0.5 * (1.0 + tanh(2.0 * (r - mid) / width));
}

// Edge integrals of the dipoles' vector potential, A(midpoint) . dr, on the
// edges [-1, n + stagger] of every family (Build_Badd_FaceFlux step 1,
// Z4_Mercury/include/operators/Dipole.h:135-210, with A_of_dipole :26-43);
// the implicit resistivity and the Hall taper of the owned edges
// (ImplicitResistiveEtaAtEdge_, HallRadialTaperEdge_) and the taper at the
// owned cell centres.
__global__ void k_bg_edges(Geo g, void *const *outp, bool fp32, GeoBg bg, double *scratch) {
  const GeoBox &b = g.b;
  const int ei = b.n[0] + 1 + 2 * b.G, ej = b.n[1] + 1 + 2 * b.G, ek = b.n[2] + 1 + 2 * b.G;
  const int64_t npos = (int64_t)ei * ej * ek;
  const int gh = b.nghost;
  const int n[3] = {b.n[0], b.n[1], b.n[2]};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npos; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % ek) - b.G, j = (int)((t / ek) % ej) - b.G, i = (int)(t / ((int64_t)ek * ej)) - b.G;
    const Out out{outp, fp32, g.off(i, j, k)};
    for (int ax = 0; ax < 3; ++ax) {
      const int di = ax == 0, dj = ax == 1, dk = ax == 2;
      // A . dr on [-1, n + stagger]; taper and resistivity on [-g, n + stagger + g)
      const int alo[3] = {-1, -1, -1}, ahi[3] = {n[0] + 1 + (ax != 0), n[1] + 1 + (ax != 1), n[2] + 1 + (ax != 2)};
      const int elo[3] = {-gh, -gh, -gh}, ehi[3] = {n[0] + gh + (ax != 0), n[1] + gh + (ax != 1), n[2] + gh + (ax != 2)};
      const bool inA = in3(i, j, k, alo, ahi), inE = in3(i, j, k, elo, ehi);
      if (!inA && !inE) continue;  // (both ranges keep the edge's far node inside the box)
      const P3 x1 = g.node(i, j, k), x2 = g.node(i + di, j + dj, k + dk);
      P3 xm, dr;
      for (int q = 0; q < 3; ++q) {
        xm.v[q] = (x1.v[q] + x2.v[q]) * 0.5;
        dr.v[q] = x2.v[q] - x1.v[q];
      }
      if (inA) {
        double A[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < bg.nd; ++d) {
          double r[3];
          for (int q = 0; q < 3; ++q) r[q] = xm.v[q] - bg.r0[d][q];
          double f = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) + bg.a[d] * bg.a[d];
          f = sqrt(f) * f;
          const double *m = bg.m[d];
          const double c[3] = {m[1] * r[2] - m[2] * r[1], m[2] * r[0] - m[0] * r[2], m[0] * r[1] - m[1] * r[0]};
          for (int q = 0; q < 3; ++q) A[q] += c[q] / f;
        }
        scratch[ax * b.total + g.off(i, j, k)] = A[0] * dr.v[0] + A[1] * dr.v[1] + A[2] * dr.v[2];
      }
      // owned edges: the taper at the midpoint and the resistivity
      if (!inE) continue;
      const int olo[3] = {0, 0, 0}, ohi[3] = {n[0] + (ax != 0), n[1] + (ax != 1), n[2] + (ax != 2)};
      const bool own = in3(i, j, k, olo, ohi);
      // HallRadialTaperEdge_ averages as 0.5 * (x1 + x2)
      double hm[3];
      for (int q = 0; q < 3; ++q) hm[q] = 0.5 * (x1.v[q] + x2.v[q]);
      out.put(GEO_TAPER + ax, own ? hall_taper(bg, hm[0], hm[1], hm[2]) : 0.0);
      if (bg.inver_Rem > 0.0) {
        double eta = 0.0;
        if (own && !(fabs(norm(dr)) <= 1.0e-12)) {
          const double r = sqrt(hm[0] * hm[0] + hm[1] * hm[1] + hm[2] * hm[2]);
          double shape = 0.5 * (tanh((r - bg.eta_r0) / bg.eta_w) - tanh((r - bg.eta_r1) / bg.eta_w));
          shape = (!isfinite(shape) || shape <= 1.0e-10) ? 0.0 : (shape < 1.0 ? shape : 1.0);
          eta = bg.inver_Rem * shape;
        }
        out.put(GEO_ETA_RES + ax, eta);
      }
    }
    // the taper at the owned cell centres (the centre of cell (i, j, k) is dual point (i + 1, j + 1, k + 1))
    const int clo[3] = {-gh, -gh, -gh}, chi[3] = {n[0] + gh, n[1] + gh, n[2] + gh};
    if (in3(i, j, k, clo, chi)) {
      const int olo[3] = {0, 0, 0};
      double v = 0.0;
      if (in3(i, j, k, olo, n)) {
        const P3 c = g.dual(i + 1, j + 1, k + 1);
        v = hall_taper(bg, c.v[0], c.v[1], c.v[2]);
      }
      out.put(GEO_TAPER_CELL, v);
    }
  }
}

// The background field on the faces of [-g, n + stagger + g): the curl of
// the edge integrals where they reach (the faces [-1, n + stagger + 1)),
// plus B0 . JD (Build_Badd_FaceFlux steps 0, 2, 3, Dipole.h:93-123,213-361).
__global__ void k_bg_faces(Geo g, void *const *outp, bool fp32, GeoBg bg, const double *scratch) {
  const GeoBox &b = g.b;
  const int ei = b.n[0] + 1 + 2 * b.G, ej = b.n[1] + 1 + 2 * b.G, ek = b.n[2] + 1 + 2 * b.G;
  const int64_t npos = (int64_t)ei * ej * ek;
  const int gh = b.nghost;
  const int n[3] = {b.n[0], b.n[1], b.n[2]};
  const double *Ex = scratch, *Ey = scratch + b.total, *Ez = scratch + 2 * b.total;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npos; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % ek) - b.G, j = (int)((t / ek) % ej) - b.G, i = (int)(t / ((int64_t)ek * ej)) - b.G;
    const Out out{outp, fp32, g.off(i, j, k)};
    for (int dir = 0; dir < 3; ++dir) {
      const int lo[3] = {-gh, -gh, -gh};
      const int hi[3] = {n[0] + gh + (dir == 0), n[1] + gh + (dir == 1), n[2] + gh + (dir == 2)};
      if (!in3(i, j, k, lo, hi)) continue;
      const int clo[3] = {-1, -1, -1};
      const int chi[3] = {n[0] + 1 + (dir == 0), n[1] + 1 + (dir == 1), n[2] + 1 + (dir == 2)};
      double v = 0.0;
      if (in3(i, j, k, clo, chi)) {
        if (dir == 0)
          v = 1.0 * ((Ey[g.off(i, j, k)] - Ey[g.off(i, j, k + 1)]) + (Ez[g.off(i, j + 1, k)] - Ez[g.off(i, j, k)]));
        else if (dir == 1)
          v = 1.0 * ((Ex[g.off(i, j, k + 1)] - Ex[g.off(i, j, k)]) + (Ez[g.off(i, j, k)] - Ez[g.off(i + 1, j, k)]));
        else
          v = 1.0 * ((Ex[g.off(i, j, k)] - Ex[g.off(i, j + 1, k)]) + (Ey[g.off(i + 1, j, k)] - Ey[g.off(i, j, k)]));
      }
      const P3 a = face_jd(g, dir, i, j, k);
      v += (bg.B0[0] * a.v[0] + bg.B0[1] * a.v[1] + bg.B0[2] * a.v[2]);
      out.put(GEO_BADD + dir, v);
    }
  }
}

}  // namespace

cudaError_t launch_geometry(const double *nodes, const GeoBox &box, void *const *out, bool fp32, double L_ref,
                            const GeoBg *bg, double *scratch, cudaStream_t st) {
  Geo g{nodes, nodes + box.total, nodes + 2 * box.total, box};
  const int64_t npos = (int64_t)(box.n[0] + 1 + 2 * box.G) * (box.n[1] + 1 + 2 * box.G) * (box.n[2] + 1 + 2 * box.G);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (npos + 127) / 128;
  const int blocks = (int)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
  k_geometry<<<blocks > 0 ? blocks : 1, 128, 0, st>>>(g, out, fp32, L_ref);
  if (bg) {
    k_bg_edges<<<blocks > 0 ? blocks : 1, 128, 0, st>>>(g, out, fp32, *bg, scratch);
    k_bg_faces<<<blocks > 0 ? blocks : 1, 128, 0, st>>>(g, out, fp32, *bg, scratch);
  }
  return cudaGetLastError();
}

}  // namespace mhd
