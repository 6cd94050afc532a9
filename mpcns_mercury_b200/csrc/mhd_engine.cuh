// Batched execution engine of the MHD step: device-resident directory of
// solves, their blocks and their tile work-lists.
//
// Every step kernel is a persistent, grid-stride loop over work items of one
// "range kind" (cells, faces+edges, the extended face range of the ideal EMF,
// the allocated cell range).  A work item is a 32 (k) x 4 (j) x 2 (i) tile of
// one block of one solve; the directory maps the global item index to
// (solve, block, tile) through per-range prefix sums.  Grid sizes depend only
// on the SM count, so one CUDA graph captured once runs any set of solves:
// membership changes only rewrite the directory in device memory.
#pragma once
#include <cstdint>

#include "mhd_layout.cuh"

namespace mhd {

// The fluid kernel's tile variants: cells along k, j, i of one 256-thread
// CTA, and the resident CTAs per SM asked of the compiler (its register cap,
// 65536 / (256 n)).  The batch runs one of them (mhd_batch_fluid_tile),
// picked by timing (mhd_batch_time_fluid_tiles); variant 0 is the default:
// 16 x 4 x 4 wastes fewer lanes than 32 x 4 x 2 on k extents that are not
// multiples of 32 and needs 6% fewer face fluxes per tile (912 vs 968).
struct FluidTile {
  int k, j, i, min_ctas;
};
constexpr int kNumFluidTiles = MHD_NUM_FLUID_TILES;
__host__ __device__ constexpr FluidTile fluid_tile(int v) {
  return v == 1 ? FluidTile{8, 8, 4, 4} : v == 2 ? FluidTile{8, 8, 4, 3} : v == 3 ? FluidTile{16, 4, 4, 4}
         : v == 4 ? FluidTile{16, 4, 4, 2} : v == 5 ? FluidTile{8, 8, 4, 2} : FluidTile{16, 4, 4, 3};
}
// Variant 6 stages each tile's cell box (density and u, v, w, p of its
// species) with TMA tensor copies issued by a producer warp up to two tiles
// ahead of the compute threads (double-buffered, mbarrier-completed).  Its box: the 16 x 4 x 4
// tile and one cell beyond each side, the k window widened to whole 16-byte
// units from a 16-byte-aligned start.
__host__ __device__ constexpr bool fluid_tma(int v) { return v == 6; }
// Threads of a fluid CTA: 256 that compute (one per cell of the tile), and
// for the staged variant a producer warp that issues the copies.
__host__ __device__ constexpr int fluid_threads(int v) { return fluid_tma(v) ? 256 + 32 : 256; }
constexpr int kTmaBoxJI = 6;  // j and i extents of the staged box
__host__ __device__ constexpr int tma_box_k(int es) { return es == 4 ? 24 : 20; }
// Components of a block's real-valued M region that its tensor map spans
// (through the primitive variables of both species).
constexpr int kTmaMComps = kComp.first[MHD_PV_NA] + 5 - kNumUComps;
constexpr int kTileThreads = 256;
constexpr bool fluid_tiles_ok() {
  for (int v = 0; v < kNumFluidTiles; ++v)
    if (fluid_tile(v).k * fluid_tile(v).j * fluid_tile(v).i != kTileThreads) return false;
  return true;
}
static_assert(fluid_tiles_ok(), "fluid tiles of 256 cells");

// Range kinds of the work lists.
enum RangeKind : int {
  kCells = 0,    // owned cells [0, n)
  kBox = 1,      // [0, n + 1): owned faces and edges of all families
  kExt = 2,      // [-1, n + 2): face EMF candidates incl. one ghost layer
  kAlloc = 3,    // [-gs, n + gs), gs = min(nghost, kStepGhost): the ghost cells the step maintains
  kCells2 = 4,   // owned cells in fluid tiles of variant 0, two work items per tile (one per ion species)
  kFull = 5,     // [-(g + 1), n + g + 2): the whole box
  // owned cells in fluid tiles of variants 1 .. kNumFluidTiles - 1 (kinds 6 ..)
  // [0, n + 1) with k below the block's reskhi: the implicit substep's work
  // (its unknowns and the faces and edges they reach)
  kResK = 6 + kNumFluidTiles - 1,
  kNumRanges = kResK + 1
};
// The range kind of fluid tile variant v, and the variant of a range kind (-1: none).
__host__ __device__ constexpr int fluid_kind(int v) { return v == 0 ? (int)kCells2 : (int)kFull + v; }
__host__ __device__ constexpr int fluid_variant(int kind) {
  return kind == kCells2 ? 0 : (kind > kFull && kind < kResK ? kind - kFull : -1);
}

// Ghost depth the step keeps valid between its passes: the widest stencil
// reach of its kernels (face EMF candidates on [-1, n + 2) read contravariant
// velocities and face fluxes two layers out).  The step's halo copies stop at
// the depth each group's readers need (kHaloDepth); explicit syncs fill all
// ghost layers.
constexpr int kStepGhost = 2;

// Precision of a batch: every component array holds `real` values (double
// or float) except the metric (Jac and the face area vectors JD), which is
// always double.  In the FP64 path real = double throughout.
enum Precision : int { kFP64 = 0, kMixed = 1 };
constexpr int kMetricFirst = kComp.first[MHD_JAC];  // JAC, JDXI, JDET, JDZE are consecutive
constexpr int kNumMetric = kComp.first[MHD_JDZE] + 3 - kMetricFirst;
constexpr int kNumRComps = kNumComps - kNumUComps - kNumMetric;  // real-valued comps outside U
static_assert(kNumMetric == 10, "metric components");
// The work arrays of the implicit resistive substep are the last components;
// solves without the substep do not allocate them.
constexpr int kFirstResComp = kComp.first[MHD_RES_W];
constexpr int kNumResComps = kNumComps - kFirstResComp;
static_assert(MHD_RES_BSTAR == MHD_NUM_FIELDS - 1, "resistive work fields last");
__host__ __device__ constexpr bool is_metric(int comp) { return comp >= kMetricFirst && comp < kMetricFirst + kNumMetric; }
// Index of a non-U, non-metric component among the real-valued M arrays.
__host__ __device__ constexpr int rslot(int comp) {
  return comp - kNumUComps - (comp >= kMetricFirst + kNumMetric ? kNumMetric : 0);
}
static_assert(kTmaMComps == rslot(kComp.first[MHD_PV_NA] + 4) + 1 && kComp.first[MHD_PV_NA] < kMetricFirst,
              "the primitive variables lie in the first kTmaMComps real-valued M components");

// Per-block descriptor (device).  Block memory: U buffers of 10 real arrays
// each; M = [10 metric double arrays | kNumRComps real arrays].
struct DevBlock {
  void *U[2];         // U_H, U_Na components (10) of buffer 0 / 1
  char *M;
  // TMA tensor maps of the block (U buffer 0, U buffer 1, the real-valued M
  // components; 128 bytes each, 64-byte aligned), null where none could be
  // encoded: the staged fluid variant then loads that block's boxes itself
  const void *tmap;
  int64_t total, si, sj;
  int G, n[3];
  int solve;          // index of the owning solve in the directory
  int reskhi;         // the implicit substep's k bound (exclusive) of range kResK; n[2] + 1: the whole box
};

// Per-solve constants, as calc_physical_constant derives them
// (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48).
template <class T>
struct ConstsT {
  T gamma, M_H, M_Na, M_ref, T_ref, L_ref, U_ref, B_ref, n_ref, rho_ref, m_Na, k_Boltz, q_e, mu0;
  T state_coeff_H, state_coeff_Na, CFL, hall_coef, momentum_induce_coeff, momentum_hall_coeff;
  T inver_MA2, ne_hall_floor;
  T arti_eta_max, arti_J_start, arti_J_on;
  int ambipolar;
  int local_arti;
  int nghost;
  int resistive;
  T bc[MHD_NUM_BC];  // values of the physical boundary operations (mhd_bc_const)
};
using Consts = ConstsT<double>;
inline ConstsT<float> to_float(const Consts &c) {
  ConstsT<float> f{(float)c.gamma, (float)c.M_H, (float)c.M_Na, (float)c.M_ref, (float)c.T_ref,
                   (float)c.L_ref, (float)c.U_ref, (float)c.B_ref, (float)c.n_ref, (float)c.rho_ref,
                   (float)c.m_Na, (float)c.k_Boltz, (float)c.q_e, (float)c.mu0, (float)c.state_coeff_H,
                   (float)c.state_coeff_Na, (float)c.CFL, (float)c.hall_coef, (float)c.momentum_induce_coeff,
                   (float)c.momentum_hall_coeff, (float)c.inver_MA2, (float)c.ne_hall_floor,
                   (float)c.arti_eta_max, (float)c.arti_J_start, (float)c.arti_J_on, c.ambipolar,
                   c.local_arti, c.nghost, c.resistive, {}};
  for (int q = 0; q < MHD_NUM_BC; ++q) f.bc[q] = (float)c.bc[q];
  return f;
}

// Per-solve device state.
struct SolveState {
  unsigned long long dt_bits;  // running min of the next step's CFL dt (positive double bits)
  double dt, time;             // last dt used, simulated time
  long long step;              // steps taken
  long long remaining;         // steps still to take in the current request (0 = idle)
  int status;                  // sticky mhd_status
  int nonfinite;               // set when an owned cell's CFL dt came out non-finite (NaN/Inf state)
  int cur;                     // which U buffer holds the current state
  int mask;                    // selected for a targeted pass (Dir::mode == 1)
  unsigned long long divb_bits;  // max |div B| of the last mhd_div_b (non-negative double bits)
};

// Sync tables of one solve address DOFs by "codes": the byte offset from the
// solve's arena base (bits 0..54); bit 60 marks a U component, whose offset
// is taken in U buffer 0 and shifted by cur * ubuf bytes at run time.  All
// synced components are real-valued.
constexpr int64_t kCodeOffMask = (int64_t(1) << 55) - 1;
constexpr int64_t kCodeUFlag = int64_t(1) << 60;
// Copy segments: `reps` runs of `len` (1..32) consecutive destinations
// dst + r * stride .. <- sign * (src + r * stride) .. (consecutive sources),
// len * reps <= kSegElems, stored as three int64: the dst code with
// (len - 1) in bits 55..59 and a negative sign in bit 61; the src code;
// (reps - 1) in bits 0..15 and the byte stride in bits 16..63.
constexpr int kSegMax = 32;     // elements of one run
#ifndef MHD_SEG_ELEMS
#define MHD_SEG_ELEMS 32
#endif
constexpr int kSegElems = MHD_SEG_ELEMS;  // elements of one segment (a multiple of 8, at most 64)
static_assert(kSegElems % 8 == 0 && kSegElems <= 64, "segment size");
constexpr int kSegWords = 3;
constexpr int kSegLenShift = 55, kSegNegBit = 61, kSegStrideShift = 16;
struct DevTable {
  const int64_t *seg = nullptr;  // kSegWords * n
  int n = 0;                     // segments
};
// Edge alias classes: members member[offset[c] .. offset[c+1]) (codes and
// signs), written to owner[c]; processed 8 classes per lane group.
struct DevAlias {
  const int32_t *offset = nullptr;  // n + 1
  const int64_t *member = nullptr;
  const double *msign = nullptr;
  const int64_t *owner = nullptr;
  const double *osign = nullptr;
  int n = 0;                        // classes
};

constexpr int kMaxGroups = MHD_NUM_GROUPS;
// Copy phases of a group: 0 halo copies to the step's depth, 1 owner copies,
// 2 every halo copy, 3 staging <- sources the halo phase overwrites, 4
// destinations <- staging.
constexpr int kNumPhases = 5;
enum CopyPhase : int { kPhHalo = 0, kPhOwner = 1, kPhHaloFull = 2, kPhStash = 3, kPhUnstash = 4 };

// Physical boundary operations (mhd_phys_op) of one solve: per group, and
// the step's wall EMF as table kMaxGroups.  MHD_PHYS_SET operations are one
// word each: the destination code with the value index in bits 55..59; the
// others are DevPhysOp.
constexpr int kNumPhys = kMaxGroups + 1;
constexpr int kPhysArgShift = 55;
constexpr int kMaxWallGhosts = 8;
struct DevPhysOp {
  int64_t dst, src;                // codes of component 0 (WALL: cells; EFAR: the edge and its dr vector)
  int64_t cstride;                 // bytes between the components of dst / src
  int64_t ghost[kMaxWallGhosts];   // WALL: codes of the ghost cells it fills (component 0)
  int kind, nghost;
};
struct DevPhys {
  const int64_t *set = nullptr;  // nset segments of constant writes, two words each
  const DevPhysOp *op = nullptr;
  int nset = 0, nop = 0;
};
// Singular (valence-3) edges of one solve: owner edges (codes in E, E_Hall,
// J), aliases, incident cells and faces as (block, axis, i, j, k, sign)
// records, and the geometric data the prepare pass computes (per edge the
// canonical edge vector and the inverse Hodge star, per cell its weight).
struct DevSingular {
  int n = 0;
  const int64_t *owner = nullptr;   // 3 per edge
  const double *osign = nullptr;
  const int *aoff = nullptr, *alias = nullptr;  // 6 ints per alias: block axis i j k orient
  const int *coff = nullptr, *cell = nullptr;   // 6 ints per cell: block axis i j k orient
  const int *foff = nullptr, *face = nullptr;   // 6 ints per face: block axis i j k sign
  double *geo = nullptr;                        // 4 per edge: canonical vector, inverse Hodge star
  double *w = nullptr;                          // per incident cell
};

// Directory entry of one solve (device).
struct DevSolve {
  Consts c;
  ConstsT<float> cf;                  // the same, rounded (mixed precision)
  const DevBlock *blocks;             // this solve's blocks
  char *arena;                        // base of the sync codes
  int64_t ubuf;                       // bytes per U buffer
  int nblocks;
  const int *tile_prefix[kNumRanges]; // per range: nblocks + 1 prefix sums of tile counts
  DevTable tab[kMaxGroups][kNumPhases];
  DevAlias aliasE, aliasJ;
  DevPhys phys[kNumPhys];
  DevSingular sing;
  // a mixed-precision solve's FP64 companion (implicit substep): its blocks
  // and its state in the companion batch (null without one)
  const DevBlock *companion;
  SolveState *companion_state;
};

// The directory handed to every kernel (by value).
struct Dir {
  const DevSolve *solves;
  SolveState *state;
  int nsolves;
  int mode;  // 0: solves with remaining steps (the step); 1: solves with mask set (prepare, sync)
  const int *solve_tile_prefix[kNumRanges];  // nsolves + 1 per range
  // sync tables: per group and phase (0 halo to the step's depth, 1 owner,
  // 2 every halo copy) prefix sums over the solves of their segment counts;
  // alias tables: of their 8-class groups
  const int *copy_prefix[kMaxGroups][kNumPhases];
  const int *aliasE_prefix, *aliasJ_prefix;
  // physical operations (SET words, then the others) and singular edges:
  // prefix sums over the solves
  const int *phys_prefix[kNumPhys];
  const int *sing_prefix;
};

template <class R>
__device__ __forceinline__ const ConstsT<R> &consts_of(const DevSolve &S);
template <>
__device__ __forceinline__ const ConstsT<double> &consts_of<double>(const DevSolve &S) { return S.c; }
template <>
__device__ __forceinline__ const ConstsT<float> &consts_of<float>(const DevSolve &S) { return S.cf; }

__host__ __device__ inline bool solve_active(const Dir &D, int s) {
  return D.mode ? D.state[s].mask != 0 : D.state[s].remaining != 0;
}

// Tile grid of a block for a range kind.
struct RangeBox {
  int lo[3], hi[3];
};
__host__ __device__ inline RangeBox range_of(int kind, const int n[3], int g) {
  RangeBox r;
  for (int a = 0; a < 3; ++a) {
    switch (kind) {
      case kCells: r.lo[a] = 0; r.hi[a] = n[a]; break;
      case kBox:
      case kResK: r.lo[a] = 0; r.hi[a] = n[a] + 1; break;  // kResK: k clamped per block where it is used
      case kExt: r.lo[a] = -1; r.hi[a] = n[a] + 2; break;
      case kFull: r.lo[a] = -(g + 1); r.hi[a] = n[a] + g + 2; break;
      case kAlloc: {
        const int gs = g < kStepGhost ? g : kStepGhost;
        r.lo[a] = -gs;
        r.hi[a] = n[a] + gs;
        break;
      }
      default: r.lo[a] = 0; r.hi[a] = n[a]; break;  // the fluid kinds: owned cells
    }
  }
  return r;
}
// Work items of a block: the fluid kinds use 3-D tiles of their variant's
// shape (two work items per tile, one per species); every other range is
// cut into runs of kTileThreads consecutive positions of its box (k fastest),
// so no lane idles at the end of short k rows.
__host__ __device__ inline int tiles_of(const RangeBox &r, int kind) {
  const int v = fluid_variant(kind);
  if (v >= 0) {
    const FluidTile T = fluid_tile(v);
    const int tk = (r.hi[2] - r.lo[2] + T.k - 1) / T.k;
    const int tj = (r.hi[1] - r.lo[1] + T.j - 1) / T.j;
    const int ti = (r.hi[0] - r.lo[0] + T.i - 1) / T.i;
    return tk * tj * ti * 2;
  }
  const int64_t vol = (int64_t)(r.hi[0] - r.lo[0]) * (r.hi[1] - r.lo[1]) * (r.hi[2] - r.lo[2]);
  return (int)((vol + kTileThreads - 1) / kTileThreads);
}

}  // namespace mhd
