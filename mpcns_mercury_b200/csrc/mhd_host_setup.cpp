// Host-side helpers of the case setup (no device work).
#include <cstdint>
#include <random>

#include "mercury_mhd.h"

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
  if (2 * (na + 2 * G) >= 4 * na) return MHD_ERR_ARG;  // ghost angles must stay below 90 degrees
  const double pi = std::acos(-1.0);
  auto tan_of = [&](int i) {
    const int q = 2 * i - na;
    if (q == na) return 1.0;
    if (q == -na) return -1.0;
    return std::tan(((double)q / (double)na) * (pi / 4.0));
  };
  const int e0 = na + 1 + 2 * G, e2 = nr + 1 + 2 * G;
  for (int ii = 0; ii < e0; ++ii)
    for (int jj = 0; jj < e0; ++jj)
      for (int kk = 0; kk < e2; ++kk) {
        const int i = ii - G, j = jj - G, k = kk - G;
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
        double *o = out + 3 * (((int64_t)ii * e0 + jj) * e2 + kk);
        for (int a = 0; a < 3; ++a) o[a] = r * d[a] * inv;
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
