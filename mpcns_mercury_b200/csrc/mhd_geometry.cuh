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
  GEO_TAPER_CELL = 95,  // Hall radial taper at the owned cell centres (off: 1)
  GEO_ETA_RES = 96,     // implicit resistivity per owned edge family (null: the solve has none)
  GEO_COUNT = 99
};
constexpr int kGeoMetric = 10;

struct GeoBox {
  int n[3];        // cells per axis
  int G;           // box ghost width (nghost + 1)
  int nghost;
  int64_t si, sj;  // box strides (k contiguous)
  int64_t total;   // positions of the box
};

// A magnetosphere's background field, Hall taper and implicit resistivity,
// nondimensional (mhd_background after load_from_param's scaling).
constexpr int kGeoMaxDipoles = 4;
struct GeoBg {
  int nd;                                       // dipoles
  double r0[kGeoMaxDipoles][3], m[kGeoMaxDipoles][3], a[kGeoMaxDipoles];
  double B0[3];                                 // IMF
  double hall_r_min, hall_r_max;
  double inver_Rem, eta_r0, eta_r1, eta_w;      // inver_Rem <= 0: no resistivity written
};

// nodes: 3 double arrays (x, y, z) over the box, node (i, j, k) at the box
// offset of (i, j, k); out: GEO_COUNT component base pointers (box layout;
// the GEO_ETA_RES ones may be null).  bg (may be null): the background
// inputs, with `scratch` 3 double arrays over the box for the edge
// integrals of the dipoles' vector potential.
cudaError_t launch_geometry(const double *nodes, const GeoBox &box, void *const *out, bool fp32, double L_ref,
                            const GeoBg *bg, double *scratch, cudaStream_t st);

}  // namespace mhd
