// Device-side per-solve setup of the static fields the step reads, from a
// block's node coordinates (mhd_geometry.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace mhd {

// Output components, in the order of the pointer table the launcher takes.
// The first kGeoMetric are the metric (double in every precision); the rest
// are real-typed (float in mixed precision).
enum GeoOut {
  GEO_JAC = 0,
  GEO_JD = 1,       // 3 face families x 3 components
  GEO_AREA = 10,    // |JD| per face family
  GEO_BETA = 13,    // face Hodge ratio |l*| / |S|
  GEO_DL = 16,      // |e| per edge family
  GEO_DR = 19,      // edge vector, 3 families x 3 components
  GEO_ALPHA = 28,   // edge Hodge ratio |e| / |S*| (0 where the dual face collapses)
  GEO_WB = 31,      // 18 B_cell weights
  GEO_WJ = 49,      // 36 J_cell weights
  GEO_BADD = 85,    // background field face fluxes (zero: no dipole, no IMF)
  GEO_PHOTO = 88,   // Na+ photo-production rate
  GEO_CELL = 89,    // cell centres x, y, z
  GEO_TAPER = 92,   // Hall radial taper per edge family (off: 1 where read)
  GEO_COUNT = 95
};
constexpr int kGeoMetric = 10;

struct GeoBox {
  int n[3];        // cells per axis
  int G;           // box ghost width (nghost + 1)
  int nghost;
  int64_t si, sj;  // box strides (k contiguous)
  int64_t total;   // positions of the box
};

// nodes: 3 double arrays (x, y, z) over the box, node (i, j, k) at the box
// offset of (i, j, k); out: GEO_COUNT component base pointers (box layout).
cudaError_t launch_geometry(const double *nodes, const GeoBox &box, void *const *out, bool fp32, double L_ref,
                            cudaStream_t st);

}  // namespace mhd
