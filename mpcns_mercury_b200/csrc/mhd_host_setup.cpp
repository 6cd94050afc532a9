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
