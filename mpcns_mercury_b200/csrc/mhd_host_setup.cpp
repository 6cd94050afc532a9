// Host-side helpers of the case setup (no device work).
#include <cstdint>
#include <random>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_topology_impl.h"

// Seeded multiplicative-noise draws of the synthetic workloads: the engine is
// std::mt19937_64 seeded with `seed`, each uniform formed as (x >> 11) * 2^-53
// and mapped to U[-a, a] as -a + 2 a u, in draw order.
extern "C" int mhd_seeded_uniform(uint64_t seed, int64_t count, double a, double *out) {
  if (count < 0 || (count > 0 && !out)) return MHD_ERR_ARG;
  std::mt19937_64 g(seed);
  for (int64_t t = 0; t < count; ++t) {
    const double u = (double)(g() >> 11) * 0x1.0p-53;
    out[t] = -a + 2.0 * a * u;
  }
  return MHD_OK;
}

#include <cmath>

// Nodes of one panel of the 6-panel gnomonic (equiangular) cubed-sphere
// shell r in [1, r_out], na x na x nr cells, over the node range
// [-G, n + 1 + G) per axis (AoS x, y, z; k fastest).  Owned nodes: panel
// directions at the tangents of the equiangular angles (+-1 exactly on the
// panel edges), radius r_out^(k / nr) (1 and r_out exactly on the spheres),
// the same expressions the oracle's shell case writes; ghost nodes continue
// the same mapping past the panel and the spheres.
extern "C" int mhd_shell_nodes(int32_t na, int32_t nr, double r_out, int32_t panel, int32_t G, double *out) {
  if (na < 2 || nr < 2 || G < 0 || panel < 0 || panel > 5 || !out || !(r_out > 1.0)) return MHD_ERR_ARG;
  const double pi = std::acos(-1.0);
  auto tan_of = [&](int i) {
    const int q = 2 * i - na;
    if (q == na) return 1.0;
    if (q == -na) return -1.0;
    return std::tan(((double)q / (double)na) * (pi / 4.0));
  };
  const int e0 = na + 1 + 2 * G, e2 = nr + 1 + 2 * G;
  auto at = [&](int i, int j, int k) { return out + 3 * (((int64_t)(i + G) * e0 + (j + G)) * e2 + (k + G)); };
  // owned nodes: equiangular panel directions times r_k = r_out^(k / nr)
  for (int i = 0; i <= na; ++i)
    for (int j = 0; j <= na; ++j)
      for (int k = 0; k <= nr; ++k) {
        const double ta = tan_of(i), tb = tan_of(j);
        double d[3];
        switch (panel) {
          case 0: d[0] = 1.0; d[1] = ta; d[2] = tb; break;
          case 1: d[0] = -ta; d[1] = 1.0; d[2] = tb; break;
          case 2: d[0] = -1.0; d[1] = -ta; d[2] = tb; break;
          case 3: d[0] = ta; d[1] = -1.0; d[2] = tb; break;
          case 4: d[0] = -tb; d[1] = ta; d[2] = 1.0; break;
          default: d[0] = tb; d[1] = ta; d[2] = -1.0; break;
        }
        const double inv = 1.0 / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double r = (k == 0) ? 1.0 : (k == nr ? r_out : std::pow(r_out, (double)k / (double)nr));
        double *o = at(i, j, k);
        for (int a = 0; a < 3; ++a) o[a] = r * d[a] * inv;
      }
  // ghost nodes, one layer at a time as the reference grid reader adds them
  // (Block::Add_ghostmesh, src/1_grid/1_MPCNS_Grid.cpp:591-815): the faces
  // by point reflection through the boundary node, then the edge strips and
  // corners by the parallelogram rule, in its order
  const int m[3] = {na, na, nr};
  auto refl = [&](int i, int j, int k, int i0, int j0, int k0, int i1, int j1, int k1) {
    double *o = at(i, j, k);
    const double *a = at(i0, j0, k0), *b = at(i1, j1, k1);
    for (int c = 0; c < 3; ++c) o[c] = 2 * a[c] - b[c];
  };
  // o = p + q - r
  auto para = [&](int i, int j, int k, int pi_, int pj, int pk, int qi, int qj, int qk, int ri, int rj, int rk) {
    double *o = at(i, j, k);
    const double *p1 = at(pi_, pj, pk), *q1 = at(qi, qj, qk), *r1 = at(ri, rj, rk);
    for (int c = 0; c < 3; ++c) o[c] = p1[c] + q1[c] - r1[c];
  };
  for (int gh = 1; gh <= G; ++gh) {
    const int imin = -gh, imax = m[0] + gh, jmin = -gh, jmax = m[1] + gh, kmin = -gh, kmax = m[2] + gh;
    for (int j = jmin + 1; j < jmax; ++j)
      for (int k = kmin + 1; k < kmax; ++k) {
        refl(imin, j, k, 0, j, k, -imin, j, k);
        refl(imax, j, k, m[0], j, k, 2 * m[0] - imax, j, k);
      }
    for (int i = imin + 1; i < imax; ++i)
      for (int k = kmin + 1; k < kmax; ++k) {
        refl(i, jmin, k, i, 0, k, i, -jmin, k);
        refl(i, jmax, k, i, m[1], k, i, 2 * m[1] - jmax, k);
      }
    for (int i = imin + 1; i < imax; ++i)
      for (int j = jmin + 1; j < jmax; ++j) {
        refl(i, j, kmin, i, j, 0, i, j, -kmin);
        refl(i, j, kmax, i, j, m[2], i, j, 2 * m[2] - kmax);
      }
    for (int k = kmin + 1; k < kmax; ++k) {
      para(imin, jmin, k, imin + 1, jmin, k, imin, jmin + 1, k, imin + 1, jmin + 1, k);
      para(imax, jmin, k, imax - 1, jmin, k, imax, jmin + 1, k, imax - 1, jmin + 1, k);
      para(imin, jmax, k, imin + 1, jmax, k, imin, jmax - 1, k, imin + 1, jmax - 1, k);
      para(imax, jmax, k, imax - 1, jmax, k, imax, jmax - 1, k, imax - 1, jmax - 1, k);
    }
    for (int j = jmin + 1; j < jmax; ++j) {
      para(imin, j, kmin, imin + 1, j, kmin, imin, j, kmin + 1, imin + 1, j, kmin + 1);
      para(imax, j, kmin, imax - 1, j, kmin, imax, j, kmin + 1, imax - 1, j, kmin + 1);
      para(imin, j, kmax, imin + 1, j, kmax, imin, j, kmax - 1, imin + 1, j, kmax - 1);
      para(imax, j, kmax, imax - 1, j, kmax, imax, j, kmax - 1, imax - 1, j, kmax - 1);
    }
    for (int i = imin; i < imax + 1; ++i) {
      para(i, jmin, kmin, i, jmin + 1, kmin, i, jmin, kmin + 1, i, jmin + 1, kmin + 1);
      para(i, jmax, kmin, i, jmax - 1, kmin, i, jmax, kmin + 1, i, jmax - 1, kmin + 1);
      para(i, jmin, kmax, i, jmin + 1, kmax, i, jmin, kmax - 1, i, jmin + 1, kmax - 1);
      para(i, jmax, kmax, i, jmax - 1, kmax, i, jmax, kmax - 1, i, jmax - 1, kmax - 1);
    }
  }
  return MHD_OK;
}

// The Hall term's radial taper at n points (x, y, z AoS):
// 0.5 (1 + tanh(2 (r - mid) / width)) between r_min and r_max, a step at
// r_min when they coincide (HallRadialTaper_,
// Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:6-13).
extern "C" int mhd_hall_taper(double r_min, double r_max, int64_t n, const double *xyz, double *out) {
  if (n < 0 || (n > 0 && (!xyz || !out))) return MHD_ERR_ARG;
  const double width = r_max - r_min;
  const double mid = 0.5 * (r_min + r_max);
  for (int64_t t = 0; t < n; ++t) {
    const double x = xyz[3 * t], y = xyz[3 * t + 1], z = xyz[3 * t + 2];
    const double r = std::sqrt(x * x + y * y + z * z);
    out[t] = width <= 0.0 ? (r >= r_min ? 1.0 : 0.0) : 0.5 * (1.0 + std::tanh(2.0 * (r - mid) / width));
  }
  return MHD_OK;
}

// All six panels' nodes, ghost nodes as the reference's grid preprocessing
// leaves them on this grid (Grid::Grid_Preprocess, include/1_grid/1_MPCNS_Grid.h:151-224:
// Add_ghostmesh, then the inner-interface mesh transfer and the corner
// treatment, corner_treat 2): (1) every panel extrapolated alone
// (mhd_shell_nodes); (2) the ghost strips beside one panel edge (one of i, j
// outside the panel, any k) take the neighbour panel's nodes across that
// edge; (3) the corner columns (i and j outside) take, through the i-edge
// neighbour for the owned radii and through the j-edge neighbour for the
// radial ghost layers, the nodes step (2) left there.  Checked node for node
// against the reference's grid on shells with G <= na.
extern "C" int mhd_shell_grid(int32_t na, int32_t nr, double r_out, int32_t G, double *out) {
  if (!out || G < 0 || G > na) return MHD_ERR_ARG;
  const int e0 = na + 1 + 2 * G, e2 = nr + 1 + 2 * G;
  const int64_t per = (int64_t)e0 * e0 * e2 * 3;
  for (int p = 0; p < 6; ++p) {
    const int rc = mhd_shell_nodes(na, nr, r_out, p, G, out + p * per);
    if (rc) return rc;
  }
  std::vector<mhd_patch> fp;
  std::vector<mhd_physical_patch> phys;
  const int rc = mhd::cubed_sphere_patches(na, nr, &fp, &phys);
  if (rc) return rc;
  // the face patch of panel p in direction d (+-1, +-2)
  auto face_of = [&](int p, int d) -> const mhd_patch * {
    for (const auto &f : fp)
      if (f.this_block == p && f.direction == d) return &f;
    return nullptr;
  };
  auto idx = [&](int p, int i, int j, int k) {
    return p * per + 3 * (((int64_t)(i + G) * e0 + (j + G)) * e2 + (k + G));
  };
  std::vector<double> src(out, out + 6 * per);
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 2) src.assign(out, out + 6 * per);
    for (int p = 0; p < 6; ++p)
      for (int i = -G; i <= na + G; ++i)
        for (int j = -G; j <= na + G; ++j) {
          const bool oi = i >= 0 && i <= na, oj = j >= 0 && j <= na;
          if ((int)!oi + (int)!oj != stage) continue;
          const mhd_patch *fi = oi ? nullptr : face_of(p, i > na ? 1 : -1);
          const mhd_patch *fj = oj ? nullptr : face_of(p, j > na ? 2 : -2);
          for (int k = -G; k <= nr + G; ++k) {
            const mhd_patch *f = stage == 1 ? (fi ? fi : fj) : ((k >= 0 && k <= nr) ? fi : fj);
            if (!f) return MHD_ERR_ARG;
            const int q0[3] = {i, j, k};
            int q[3];
            for (int a = 0; a < 3; ++a) q[f->perm[a]] = f->sign[a] * q0[a] + f->offset[a];
            if (q[0] < -G || q[0] > na + G || q[1] < -G || q[1] > na + G || q[2] < -G || q[2] > nr + G)
              return MHD_ERR_ARG;
            const double *s = src.data() + idx(f->nb_block, q[0], q[1], q[2]);
            double *o = out + idx(p, i, j, k);
            for (int c = 0; c < 3; ++c) o[c] = s[c];
          }
        }
  }
  return MHD_OK;
}
