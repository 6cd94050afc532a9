// Engine host side and C ABI (include/mercury_mhd.h).
//
// A batch owns a fixed-capacity device directory of solve slots
// (mhd_engine.cuh), one CUDA stream and one CUDA graph of a full StepOnce over
// every active slot.  Every kernel reads the directory from device memory and
// runs a persistent grid, so the graph stays valid while solves join and
// leave: adding or removing a solve only rewrites directory entries with
// stream-ordered copies between graph launches.
//
// mhd_ctx (one solve) is a batch of capacity 1.
#include <cuda.h>  // CUtensorMap and the encoder's enums (the encoder itself is fetched from the driver)
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_engine.cuh"
#include "mhd_kernels.cuh"
#include "mhd_parallel.h"
#include "mhd_error.h"
#include "mhd_geometry.cuh"
#include "mhd_periodic.h"

using namespace mhd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

}  // namespace

int mhd::set_error(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

namespace {

#define CUDA_TRY(expr)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess) return fail(MHD_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

constexpr unsigned long long kDtUnset = 0x54B249AD2594C37DULL;  // bit pattern of 1e100

// AoS (FieldBlock) <-> SoA box scatter/gather for uploads and downloads; the
// device arrays hold doubles (fp32 = 0) or floats (fp32 = 1).
__global__ void k_scatter_aos(const double *__restrict__ aos, int lo0, int lo1, int lo2, int e0, int e1, int e2, int nc,
                              void *const *__restrict__ dst_comp, int ndst, int64_t si, int64_t sj, int G, int fp32) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npts = (int64_t)e0 * e1 * e2;
  if (t >= npts) return;
  const int k = (int)(t % e2), j = (int)((t / e2) % e1), i = (int)(t / ((int64_t)e1 * e2));
  const int64_t off = (int64_t)(i + lo0 + G) * si + (int64_t)(j + lo1 + G) * sj + (k + lo2 + G);
  for (int m = 0; m < nc; ++m) {
    const double v = aos[t * nc + m];
    for (int d = 0; d < ndst; ++d) {
      if (fp32)
        ((float *)dst_comp[d * nc + m])[off] = (float)v;
      else
        ((double *)dst_comp[d * nc + m])[off] = v;
    }
  }
}
// One value per component over a box range (mhd_batch_fill_field).
struct FillValues {
  double v[36];
};
__global__ void k_fill(FillValues val, int lo0, int lo1, int lo2, int e0, int e1, int e2, int nc,
                       void *const *__restrict__ dst_comp, int ndst, int64_t si, int64_t sj, int G, int fp32) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npts = (int64_t)e0 * e1 * e2;
  if (t >= npts) return;
  const int k = (int)(t % e2), j = (int)((t / e2) % e1), i = (int)(t / ((int64_t)e1 * e2));
  const int64_t off = (int64_t)(i + lo0 + G) * si + (int64_t)(j + lo1 + G) * sj + (k + lo2 + G);
  for (int m = 0; m < nc; ++m)
    for (int d = 0; d < ndst; ++d) {
      if (fp32)
        ((float *)dst_comp[d * nc + m])[off] = (float)val.v[m];
      else
        ((double *)dst_comp[d * nc + m])[off] = val.v[m];
    }
}
__global__ void k_gather_aos(double *__restrict__ aos, int lo0, int lo1, int lo2, int e0, int e1, int e2, int nc,
                             void *const *__restrict__ src_comp, int64_t si, int64_t sj, int G, int fp32) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npts = (int64_t)e0 * e1 * e2;
  if (t >= npts) return;
  const int k = (int)(t % e2), j = (int)((t / e2) % e1), i = (int)(t / ((int64_t)e1 * e2));
  const int64_t off = (int64_t)(i + lo0 + G) * si + (int64_t)(j + lo1 + G) * sj + (k + lo2 + G);
  for (int m = 0; m < nc; ++m)
    aos[t * nc + m] = fp32 ? (double)((const float *)src_comp[m])[off] : ((const double *)src_comp[m])[off];
}

template <class T>
int dev_upload(cudaMemPool_t pool, const std::vector<T> &h, T **d, cudaStream_t st) {
  *d = nullptr;
  if (h.empty()) return MHD_OK;
  CUDA_TRY(cudaMallocFromPoolAsync((void **)d, sizeof(T) * h.size(), pool, st));
  CUDA_TRY(cudaMemcpyAsync(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st));
  return MHD_OK;
}

// One solve: its arena, tables and its directory entry's pointees.  Arena
// bytes: [U buffer 0 | U buffer 1 | M of every block], per block U = 10 real
// arrays, M = 10 metric double arrays then kNumRComps real arrays.
// Device tables of a solve's topology (tile prefix sums, sync segments, alias
// classes).  Solves added with mhd_batch_add_like share their template's
// tables; the last user frees them.
struct Tables {
  int users = 0;
  int *dtile_prefix[kNumRanges] = {};
  int tiles[kNumRanges] = {};
  int64_t *tab_seg[kMaxGroups][kNumPhases] = {};
  int tab_n[kMaxGroups][kNumPhases] = {};  // segments per CopyPhase
  // physical boundary operations (per group, then the wall EMF)
  int64_t *ph_set[kNumPhys] = {};
  DevPhysOp *ph_op[kNumPhys] = {};
  int ph_nset[kNumPhys] = {}, ph_nop[kNumPhys] = {};
  // singular edges (the geometric data is per solve)
  int sg_n = 0, sg_ncell = 0;
  int64_t *sg_owner = nullptr;
  double *sg_osign = nullptr;
  int *sg_aoff = nullptr, *sg_alias = nullptr, *sg_coff = nullptr, *sg_cell = nullptr, *sg_foff = nullptr,
      *sg_face = nullptr;
  int32_t *al_off = nullptr;
  int64_t *al_memE = nullptr, *al_ownE = nullptr, *al_memJ = nullptr, *al_ownJ = nullptr;
  double *al_msign = nullptr, *al_osign = nullptr;
  int al_n = 0;
  int64_t table_bytes = 0;
  // The implicit substep's k bound: the largest source k of any E / dB / dJ
  // copy, alias or singular-edge record that carries a value to a lower k
  // (-1: every one keeps k or raises it; INT_MAX: unknown, no restriction)
  int res_kdown = INT_MAX;
  // Every halo, staged and physical write of Sync(Eres) and Sync(Jedge) lands
  // on a ghost position (res_light_syncs)
  bool res_ghost_writes_only = false;
};

struct Solve {
  int nblocks = 0, nghost = 0, es = 8;  // es: bytes per real
  cudaMemPool_t pool = nullptr;         // the batch's device memory pool
  bool prepared = false;
  std::vector<Box> boxes;
  std::vector<int64_t> ubase, mbase;  // bytes
  int64_t ubuf = 0, main_off = 0, arena_bytes = 0;
  int64_t staging_off = 0;  // the sync staging slots (real), after the fields
  int n_staging = 0;
  double *sg_geo = nullptr, *sg_w = nullptr;  // singular-edge geometry (k_sing_setup)
  char *arena = nullptr;
  DevBlock *dblocks = nullptr;
  void *dtmaps = nullptr;  // the blocks' TMA tensor maps (DevBlock::tmap)
  Tables *T = nullptr;
  double res_rtol = 0.0;
  int res_max_it = 0;
  int res_direct = 0;  // mixed precision: FP64 CG while the last substep took at most this many iterations
  // mixed precision with the implicit resistive substep: slot of the FP64
  // companion solve (same blocks and tables) in the batch's companion batch
  int shadow_slot = -1;
  // the last implicit resistive substep (mhd_info)
  double res_relres = 0.0;
  int res_iters = 0, res_refinements = 0;
  // the implicit substep's work range kResK (set at prepare): its tile
  // prefix over the blocks and count; null: the whole owned box (kBox)
  int *dres_prefix = nullptr;
  int res_tiles = 0;
  Consts consts{};

  int comp_bytes(int c) const { return is_metric(c) ? 8 : es; }
  // byte offset of component array c of block b (U comps in buffer `buf`)
  int64_t comp_base(int b, int c, int buf) const {
    const int64_t tot = boxes[b].total;
    if (c < kNumUComps) return (int64_t)buf * ubuf + ubase[b] + (int64_t)c * tot * es;
    if (is_metric(c)) return main_off + mbase[b] + (int64_t)(c - kMetricFirst) * tot * 8;
    return main_off + mbase[b] + (int64_t)kNumMetric * tot * 8 + (int64_t)rslot(c) * tot * es;
  }
  // Arena code of a DOF (kCodeOffMask / kCodeUFlag in mhd_engine.cuh).
  int64_t code(const mhd_dof &d, bool *ok) const {
    *ok = false;
    if (d.field == MHD_STAGING) {  // a staging slot
      if (d.i < 0 || d.i >= n_staging) return 0;
      *ok = true;
      return staging_off + (int64_t)d.i * es;
    }
    if (d.field < 0 || d.field >= MHD_NUM_FIELDS || d.block < 0 || d.block >= nblocks) return 0;
    if (d.comp < 0 || d.comp >= kFieldSpec[d.field].ncomp) return 0;
    const Box &bx = boxes[d.block];
    const int q[3] = {d.i, d.j, d.k};
    for (int a = 0; a < 3; ++a)
      if (q[a] < -bx.G || q[a] >= bx.n[a] + 1 + bx.G) return 0;
    const int64_t off = (int64_t)(d.i + bx.G) * bx.si + (int64_t)(d.j + bx.G) * bx.sj + (d.k + bx.G);
    const int c = kComp.first[d.field] + d.comp;
    if (is_metric(c)) return 0;  // the metric is static and never synced
    *ok = true;
    const int64_t code = comp_base(d.block, c, 0) + off * es;
    return c < kNumUComps ? (kCodeUFlag | code) : code;
  }
  void *comp_ptr(int b, int c, int buf) const { return arena + comp_base(b, c, buf); }
};

}  // namespace

struct mhd_batch {
  int capacity = 0;
  int precision = kFP64;
  cudaStream_t stream = nullptr;
  // Device memory of solves, tables and staging: the batch's own pool, which
  // keeps freed memory for the next solve instead of returning it to the
  // driver at every synchronisation (admitting a solve then maps no memory).
  cudaMemPool_t pool = nullptr;
  std::vector<Solve *> slots;
  // device directory (fixed addresses for the lifetime of the batch)
  DevSolve *dsolves = nullptr;
  SolveState *dstate = nullptr;
  int *dprefix_tiles[kNumRanges] = {};
  int *dprefix_copy[kMaxGroups][kNumPhases] = {};
  int *dprefix_phys[kNumPhys] = {};
  int *dprefix_sing = nullptr;
  int *dprefix_aliasE = nullptr, *dprefix_aliasJ = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaGraphExec_t graph_a = nullptr, graph_b = nullptr;  // the step split around implicit resistive solves
  cudaGraphExec_t graph_cg = nullptr;                   // the CG iteration loop of the masked solve
  // solves whose table of a group's copy phase has entries: sync phases
  // empty in every solve get no launch in the step (likewise the physical
  // operations and the singular edges)
  int live_tables[kMaxGroups][kNumPhases] = {};
  int live_phys[kNumPhys] = {};
  int live_sing = 0;
  int n_res = 0;                                        // slots whose solve has the implicit resistive substep
  int n_res_full = 0;                                   // of them, solves whose substep runs the full E / J syncs
  // FP64 batch of the companions of mixed-precision resistive solves, which
  // runs on this batch's stream and pool (borrowed = true in the companion)
  mhd_batch *shadow = nullptr;
  bool borrowed = false;
  ResScratch res{nullptr, nullptr};
  double *hres = nullptr;                               // pinned copy of res.result
  ResCG *hcg = nullptr;                                 // pinned copy of res.cg (one per slot)
  size_t tpart_elems = 0;                               // doubles allocated at res.tpartial
  bool cg_host_loop = false;                            // CG iterations launched one by one from the host
  // device time of the implicit substep: events around the last one, the sum and count so far
  cudaEvent_t res_ev[2] = {nullptr, nullptr};
  bool res_ev_pending = false;
  double res_ms = 0.0;
  int64_t res_steps = 0;
  int kernels_per_step = 0;
  double *staging = nullptr;
  size_t staging_elems = 0;
  void **comp_ptrs = nullptr;
  SolveState *hstate = nullptr;  // pinned mirror of dstate
  SolveState *hsnap[2] = {};     // pinned snapshots for mhd_batch_poll_async
  cudaEvent_t snap_ev[2] = {};
  int snap_next = 0;
  // eager profiling
  bool profiling = false;
  int fluid_tile = 0;  // the fluid kernel's tile variant (fluid_tile)
  std::vector<cudaEvent_t> prof_events;
  std::vector<const char *> prof_names;
  size_t prof_used = 0;

  Dir dir(int mode) const {
    Dir d;
    d.solves = dsolves;
    d.state = dstate;
    d.nsolves = capacity;
    d.mode = mode;
    for (int r = 0; r < kNumRanges; ++r) d.solve_tile_prefix[r] = dprefix_tiles[r];
    for (int g = 0; g < kMaxGroups; ++g)
      for (int p = 0; p < kNumPhases; ++p) d.copy_prefix[g][p] = dprefix_copy[g][p];
    d.aliasE_prefix = dprefix_aliasE;
    d.aliasJ_prefix = dprefix_aliasJ;
    for (int q = 0; q < kNumPhys; ++q) d.phys_prefix[q] = dprefix_phys[q];
    d.sing_prefix = dprefix_sing;
    return d;
  }
};

struct mhd_ctx {
  mhd_batch *batch = nullptr;
};

namespace {

void mark(mhd_batch *b, const char *name) {
  if (!b->profiling) return;
  if (b->prof_used == b->prof_events.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    b->prof_events.push_back(e);
    b->prof_names.push_back(name);
  }
  b->prof_names[b->prof_used] = name;
  cudaEventRecord(b->prof_events[b->prof_used++], b->stream);
}

void launch(mhd_batch *b, int mode, StepKernel k, int *nk, const SyncOps *ops = nullptr, int iarg = 0,
            double darg = 0.0) {
  launch_step_kernel(k, b->dir(mode), b->stream, ops, b->precision, iarg, darg, b->res);
  ++*nk;
  mark(b, step_kernel_name(k));
}

SyncOp copy_op(int g, int phase, int prev = 0, int mark = 0) { return SyncOp{SYNC_COPY, g, phase, prev, mark}; }
SyncOp alias_op(int which) { return SyncOp{SYNC_ALIAS, which, 0, 0, 0}; }

// A sync operation some solve of the batch has work for (a copy phase whose
// table is empty in every solve is left out: the depth-0 halos of E, E_Hall
// and the J edges, and the owner phases of cell fields, which have no alias
// DOFs).
bool op_live(const mhd_batch *b, const SyncOp &o) {
  return o.kind != SYNC_COPY || o.phase == kPhHaloFull || b->live_tables[o.arg][o.phase] > 0;
}

// One k_sync launch running one or two independent sync operations.
void sync1(mhd_batch *b, int mode, SyncOp a, int *nk) {
  if (!op_live(b, a)) return;
  SyncOps ops{{a, a}, 1};
  launch(b, mode, SK_SYNC, nk, &ops);
}
void sync2(mhd_batch *b, int mode, SyncOp a, SyncOp c, int *nk) {
  if (!op_live(b, a)) return sync1(b, mode, c, nk);
  if (!op_live(b, c)) return sync1(b, mode, a, nk);
  SyncOps ops{{a, c}, 2};
  launch(b, mode, SK_SYNC, nk, &ops);
}

// The physical boundary operations of table `which` (a group, or the wall
// EMF), when some solve has them.
void phys1(mhd_batch *b, int mode, int which, int *nk) {
  if (b->live_phys[which] > 0) launch(b, mode, SK_PHYS, nk, nullptr, which);
}
// Before a group's halo copies: its physical operations, then the staging of
// the sources its halo copies overwrite; after them: the staged copies.
// prev: the group's U ghosts hold their last synced values in the other
// buffer (Sync(U) right after the step's buffer flip).
void sync_pre(mhd_batch *b, int mode, int g, int *nk, int prev = 0) {
  phys1(b, mode, g, nk);
  sync1(b, mode, copy_op(g, kPhStash, prev), nk);
}
void sync_post(mhd_batch *b, int mode, int g, int *nk) { sync1(b, mode, copy_op(g, kPhUnstash), nk); }

// Adds (d = +1) or removes (d = -1) a solve's step tables from the batch's
// counts; true when a phase that no solve had entries for gains some (the
// step graphs, which leave that phase out, must be captured anew).
bool count_tables(mhd_batch *b, const Solve *S, int d);
void drop_graphs(mhd_batch *b);

// MercuryBoundary::Sync(group) (Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110):
// the group's physical operations, halo copies (staged where a source is
// overwritten by the same phase), then its owner copies.  full: every ghost
// layer (mhd_sync); otherwise the layers the step reads (kHaloDepth).
void enqueue_sync(mhd_batch *b, int mode, int g, int *nk, bool full = false) {
  sync_pre(b, mode, g, nk);
  sync1(b, mode, copy_op(g, full ? kPhHaloFull : kPhHalo), nk);
  sync_post(b, mode, g, nk);
  sync1(b, mode, copy_op(g, kPhOwner), nk);
}

// UpdateDerivedFields_ (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:309-321) plus the
// contravariant velocities and the next step's CFL dt.  Independent sync
// stages share a launch: Sync(B_cell) runs beside the J alias reduction and
// Sync(Jedge), in the same order per field as the reference; the singular
// edges' current replaces their owners' after the alias reduction
// (Calc_J_Edge, Z4_Mercury/src/physics/MercurySolver_Current.cpp:140-201).
void enqueue_derived(mhd_batch *b, int mode, int *nk) {
  launch(b, mode, SK_BCELL_JEDGE, nk);
  sync_pre(b, mode, MHD_SYNC_B_CELL, nk);
  sync2(b, mode, copy_op(MHD_SYNC_B_CELL, kPhHalo), alias_op(1), nk);
  sync_post(b, mode, MHD_SYNC_B_CELL, nk);
  if (b->live_sing > 0) launch(b, mode, SK_SING_J, nk);
  sync_pre(b, mode, MHD_SYNC_JEDGE, nk);
  sync2(b, mode, copy_op(MHD_SYNC_B_CELL, kPhOwner), copy_op(MHD_SYNC_JEDGE, kPhHalo), nk);
  sync_post(b, mode, MHD_SYNC_JEDGE, nk);
  sync1(b, mode, copy_op(MHD_SYNC_JEDGE, kPhOwner), nk);
  launch(b, mode, SK_JCELL, nk);
  enqueue_sync(b, mode, MHD_SYNC_J_CELL, nk);
  launch(b, mode, SK_PV_UPLUS, nk);
}

// StepOnce (Z4_Mercury/src/MercurySolver_Driver.cpp:21-61) for every active slot, in two
// parts: A up to the Euler update and Sync(U), Sync(B faces); B the derived
// refresh.  With implicit resistive solves, their substep
// (Driver.cpp:33-38) runs between A and B and B starts with Sync(B faces).
void enqueue_step_a(mhd_batch *b, int *nk) {
  const int m = 0;
  // AssembleRHS_Induction_CT_ (Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:90-171)
  launch(b, m, SK_FACE_EMF, nk);
  launch(b, m, SK_EDGE_EMF, nk);
  launch(b, m, SK_HALL_EDGE, nk);
  if (b->live_sing > 0 || b->live_phys[MHD_SYNC_EHALL] > 0 || b->live_tables[MHD_SYNC_EHALL][kPhStash] > 0) {
    // the E alias reduction, the singular edges' EMF and Hall EMF, Sync(Ehall)
    sync1(b, m, alias_op(0), nk);
    if (b->live_sing > 0) launch(b, m, SK_SING_EMF, nk);
    enqueue_sync(b, m, MHD_SYNC_EHALL, nk);
  } else {  // the E alias reduction and Sync(Ehall) touch different fields
    sync2(b, m, alias_op(0), copy_op(MHD_SYNC_EHALL, kPhHalo), nk);
    sync1(b, m, copy_op(MHD_SYNC_EHALL, kPhOwner), nk);
  }
  launch(b, m, SK_ADD_HALL, nk);
  phys1(b, m, kMaxGroups, nk);  // the wall EMF: E_t = 0 on solid-wall edges
  enqueue_sync(b, m, MHD_SYNC_EEDGE, nk);
  // AssembleRHS_Fluid_ + ApplyUpdate_Euler_ (state into the other buffer) and
  // the constrained-transport face update (Z4_Mercury/src/physics/MercurySolver_Advance.cpp:73-147)
  launch(b, m, SK_FLUID, nk, nullptr, b->fluid_tile);
  launch(b, m, SK_BFACE, nk);
  launch(b, m, SK_FLIP, nk);
  // the reference's Sync(Ucell) reads ghosts it does not overwrite first at
  // their values from the previous sync, which after the flip are in the
  // other buffer
  sync_pre(b, m, MHD_SYNC_UCELL, nk, 1);
  sync_pre(b, m, MHD_SYNC_BFACE, nk);
  sync2(b, m, copy_op(MHD_SYNC_UCELL, kPhHalo), copy_op(MHD_SYNC_BFACE, kPhHalo), nk);
  sync_post(b, m, MHD_SYNC_UCELL, nk);
  sync_post(b, m, MHD_SYNC_BFACE, nk);
  sync2(b, m, copy_op(MHD_SYNC_UCELL, kPhOwner), copy_op(MHD_SYNC_BFACE, kPhOwner), nk);
}
void enqueue_step_b(mhd_batch *b, int *nk, bool resync_b) {
  const int m = 0;
  if (resync_b) enqueue_sync(b, m, MHD_SYNC_BFACE, nk);
  enqueue_derived(b, m, nk);
  launch(b, m, SK_RETIRE, nk);
}
void enqueue_step(mhd_batch *b, int *nk) {
  enqueue_step_a(b, nk);
  enqueue_step_b(b, nk, false);
}

int ensure_staging(mhd_batch *b, size_t elems) {  // elems doubles
  if (elems <= b->staging_elems) return MHD_OK;
  if (b->staging) cudaFreeAsync(b->staging, b->stream);
  b->staging = nullptr;
  b->staging_elems = 0;
  if (cudaMallocFromPoolAsync((void **)&b->staging, sizeof(double) * elems, b->pool, b->stream) != cudaSuccess)
    return fail(MHD_ERR_OOM, "staging of %zu doubles", elems);
  b->staging_elems = elems;
  return MHD_OK;
}

// Rewrites the directory: per-range and per-table prefix sums over the slots
// and every slot's DevSolve (empty slots contribute no items).
int publish(mhd_batch *b) {
  const int C = b->capacity;
  std::vector<int> pre((size_t)C + 1);
  auto put = [&](int *dst, auto count) -> int {
    pre[0] = 0;
    for (int s = 0; s < C; ++s) pre[s + 1] = pre[s] + (b->slots[s] ? count(b->slots[s]) : 0);
    CUDA_TRY(cudaMemcpyAsync(dst, pre.data(), sizeof(int) * (C + 1), cudaMemcpyHostToDevice, b->stream));
    return MHD_OK;
  };
  int rc;
  for (int r = 0; r < kNumRanges; ++r)
    if ((rc = put(b->dprefix_tiles[r], [&](const Solve *S) {
           return r == kResK && S->dres_prefix ? S->res_tiles : S->T->tiles[r];
         })))
      return rc;
  for (int g = 0; g < kMaxGroups; ++g)
    for (int p = 0; p < kNumPhases; ++p)
      if ((rc = put(b->dprefix_copy[g][p], [&](const Solve *S) { return S->T->tab_n[g][p]; }))) return rc;
  if ((rc = put(b->dprefix_aliasE, [](const Solve *S) { return (S->T->al_n + 7) / 8; }))) return rc;
  if ((rc = put(b->dprefix_aliasJ, [](const Solve *S) { return (S->T->al_n + 7) / 8; }))) return rc;
  for (int q = 0; q < kNumPhys; ++q)
    if ((rc = put(b->dprefix_phys[q], [&](const Solve *S) { return S->T->ph_nset[q] + S->T->ph_nop[q]; }))) return rc;
  if ((rc = put(b->dprefix_sing, [](const Solve *S) { return S->T->sg_n; }))) return rc;
  std::vector<DevSolve> ds((size_t)C);
  for (int s = 0; s < C; ++s) {
    DevSolve &d = ds[s];
    d = DevSolve{};
    const Solve *S = b->slots[s];
    if (!S) continue;
    d.c = S->consts;
    d.cf = to_float(S->consts);
    d.blocks = S->dblocks;
    d.arena = S->arena;
    d.ubuf = S->ubuf;
    d.nblocks = S->nblocks;
    for (int r = 0; r < kNumRanges; ++r) d.tile_prefix[r] = S->T->dtile_prefix[r];
    if (S->dres_prefix) d.tile_prefix[kResK] = S->dres_prefix;
    for (int g = 0; g < kMaxGroups; ++g)
      for (int p = 0; p < kNumPhases; ++p) d.tab[g][p] = DevTable{S->T->tab_seg[g][p], S->T->tab_n[g][p]};
    for (int q = 0; q < kNumPhys; ++q)
      d.phys[q] = DevPhys{S->T->ph_set[q], S->T->ph_op[q], S->T->ph_nset[q], S->T->ph_nop[q]};
    const Tables &T = *S->T;
    d.sing = DevSingular{T.sg_n, T.sg_owner, T.sg_osign, T.sg_aoff, T.sg_alias, T.sg_coff, T.sg_cell, T.sg_foff,
                         T.sg_face, S->sg_geo, S->sg_w};
    d.aliasE = DevAlias{S->T->al_off, S->T->al_memE, S->T->al_msign, S->T->al_ownE, S->T->al_osign, S->T->al_n};
    d.aliasJ = DevAlias{S->T->al_off, S->T->al_memJ, S->T->al_msign, S->T->al_ownJ, S->T->al_osign, S->T->al_n};
    if (S->shadow_slot >= 0 && b->shadow && b->shadow->slots[S->shadow_slot]) {
      d.companion = b->shadow->slots[S->shadow_slot]->dblocks;
      d.companion_state = b->shadow->dstate + S->shadow_slot;
    }
  }
  CUDA_TRY(cudaMemcpyAsync(b->dsolves, ds.data(), sizeof(DevSolve) * C, cudaMemcpyHostToDevice, b->stream));
  return MHD_OK;
}

// Ghost depth each group's halo is filled to inside the step: the farthest
// ghost layer any kernel of the step reads it at (U and the face fluxes: the
// face EMF candidates and contravariant velocities two layers out; B_cell and
// J_cell: the Hall cell field one layer out; E, E_Hall and J edges are read
// only at owned and alias positions; in the implicit resistive substep E_res
// only there and dB one layer out).  Explicit syncs (mhd_sync) fill every
// layer.
constexpr int kHaloDepth[MHD_NUM_GROUPS] = {2, 2, 0, 0, 1, 0, 1, 0, 1, 0};

// Ghost depth of a DOF: how far outside its owned range [0, n + stagger) it lies.
int dof_depth(const Solve *S, const mhd_dof &d) {
  const Box &bx = S->boxes[d.block];
  const int *st = kStagger[kFieldSpec[d.field].loc];
  const int q[3] = {d.i, d.j, d.k};
  int depth = 0;
  for (int a = 0; a < 3; ++a) {
    const int hi = bx.n[a] + st[a];
    const int da = q[a] < 0 ? -q[a] : (q[a] >= hi ? q[a] - hi + 1 : 0);
    depth = da > depth ? da : depth;
  }
  return depth;
}

// A copy table encoded as arena codes (validated once, shared by the phases
// built from it).
struct Encoded {
  std::vector<int64_t> dst, src;
  std::vector<uint8_t> neg, depth;
  bool ascending = true;  // destinations strictly increasing in table order
};

constexpr int kEncodeChunk = 1 << 13;

// Encodes entries [t0, t1) of a table; records the first invalid entry of
// the chunk and whether its destinations ascend.
void encode_chunk(const Solve *S, const mhd_copy *tab, int t0, int t1, Encoded *e, int *bad, int *kind, char *asc) {
  *bad = -1;
  *asc = 1;
  for (int t = t0; t < t1; ++t) {
    bool o1, o2;
    const int64_t dc = S->code(tab[t].dst, &o1);
    const int64_t sc = S->code(tab[t].src, &o2);
    if (!o1 || !o2 || (tab[t].sign != 1.0 && tab[t].sign != -1.0)) {
      *bad = t;
      *kind = (!o1 || !o2) ? 1 : 2;
      return;
    }
    e->dst[t] = dc;
    e->src[t] = sc;
    e->neg[t] = tab[t].sign < 0.0;
    const int d = tab[t].dst.field == MHD_STAGING ? 0 : dof_depth(S, tab[t].dst);
    e->depth[t] = (uint8_t)(d > 255 ? 255 : d);
    if (t > t0 && dc <= e->dst[t - 1]) *asc = 0;
  }
}

// One phase's segments from an encoded table.  max_depth < 0: every entry;
// otherwise only entries whose destination lies at most max_depth ghost
// layers out.  A table already in ascending destination order (the periodic
// builder's) is segmented without a sort.  Entries sorted by destination (a
// destination written twice keeps the later entry, as sequential application
// would) form runs of up to kSegMax consecutive destinations with
// consecutive sources and one sign; runs of equal length, sign and
// source - destination offset whose destinations step by one stride are then
// merged into strided segments of up to kSegElems elements (the k ghosts of
// successive grid lines, the alias layer of a staggered axis).  Destinations
// of one phase are distinct and no copy of a phase reads a value the phase
// writes, so the order of application does not change the result.  Signs
// must be +1 or -1 (orientation flips).
std::vector<int64_t> build_segments(const Encoded &e, int es, int max_depth, const std::vector<char> *keep = nullptr) {
  const int n0 = (int)e.dst.size();
  std::vector<int> order;
  order.reserve(n0);
  for (int t = 0; t < n0; ++t)
    if (keep ? (*keep)[t] != 0 : (max_depth < 0 || e.depth[t] <= max_depth)) order.push_back(t);
  const int n = (int)order.size();
  if (!e.ascending)
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return e.dst[a] < e.dst[c]; });
  struct Run {
    int64_t dst, src;
    int len;
    bool neg;
  };
  std::vector<Run> runs;
  runs.reserve(n / 2 + 1);
  for (int u = 0; u < n; ++u) {
    const int t = order[u];
    if (u + 1 < n && e.dst[order[u + 1]] == e.dst[t]) continue;  // a later entry overwrites this destination
    if (!runs.empty()) {
      Run &r = runs.back();
      if (r.len < kSegMax && e.dst[t] == r.dst + (int64_t)r.len * es && e.src[t] == r.src + (int64_t)r.len * es &&
          (bool)e.neg[t] == r.neg) {
        ++r.len;
        continue;
      }
    }
    runs.push_back(Run{e.dst[t], e.src[t], 1, (bool)e.neg[t]});
  }
  // runs of one (len, sign, src - dst) class, each class in destination order
  // (classes are few: a hash of the key buckets the runs in one pass)
  std::vector<int> ro;
  ro.reserve(runs.size());
  {
    struct KeyHash {
      size_t operator()(const std::pair<int64_t, int> &k) const {
        return std::hash<int64_t>()(k.first) ^ (std::hash<int>()(k.second) * 0x9e3779b97f4a7c15ull);
      }
    };
    std::unordered_map<std::pair<int64_t, int>, int, KeyHash> cls;  // key -> class index
    std::vector<std::vector<int>> members;
    for (size_t q = 0; q < runs.size(); ++q) {
      const Run &r = runs[q];
      const std::pair<int64_t, int> key(r.src - r.dst, r.len * 2 + (r.neg ? 1 : 0));
      auto it = cls.find(key);
      if (it == cls.end()) {
        it = cls.emplace(key, (int)members.size()).first;
        members.emplace_back();
      }
      members[it->second].push_back((int)q);
    }
    for (auto &m : members) ro.insert(ro.end(), m.begin(), m.end());
  }
  std::vector<int64_t> seg;
  seg.reserve(kSegWords * runs.size());
  for (size_t u = 0; u < ro.size();) {
    const Run &r0 = runs[ro[u]];
    int reps = 1;
    int64_t stride = 0;
    while (u + reps < ro.size() && (reps + 1) * r0.len <= kSegElems && reps < 65536) {
      const Run &rn = runs[ro[u + reps]];
      if (rn.len != r0.len || rn.neg != r0.neg || rn.src - rn.dst != r0.src - r0.dst) break;
      const int64_t step = rn.dst - runs[ro[u + reps - 1]].dst;
      if (reps == 1) {
        if (step <= 0 || step >= (int64_t(1) << (63 - kSegStrideShift))) break;
        stride = step;
      } else if (step != stride) {
        break;
      }
      ++reps;
    }
    seg.push_back(r0.dst | ((int64_t)(r0.len - 1) << kSegLenShift) | ((int64_t)r0.neg << kSegNegBit));
    seg.push_back(r0.src);
    seg.push_back((int64_t)(reps - 1) | (stride << kSegStrideShift));
    u += reps;
  }
  return seg;
}

// The three phases of every group (pruned halo, owner, full halo) segmented
// on the host threads from the encoded halo (2 g) and owner (2 g + 1)
// tables, and uploaded.
// The halo copies the step keeps: those whose destination lies within the
// group's step depth, and (transitively) every halo copy that writes a
// source of a kept copy, of a staged copy or of an owner copy -- a ghost
// beyond the step depth that such a copy reads must hold its value from the
// previous sync, as in the reference.
std::vector<char> step_halo_mask(const Encoded &h, const Encoded *owner, const Encoded *stash, int max_depth) {
  const size_t n = h.dst.size();
  std::vector<char> keep(n, 0);
  std::unordered_map<int64_t, size_t> by_dst;
  by_dst.reserve(n * 2);
  for (size_t t = 0; t < n; ++t) by_dst[h.dst[t]] = t;  // the later entry wins a destination written twice
  std::vector<int64_t> todo;
  for (size_t t = 0; t < n; ++t)
    if (h.depth[t] <= max_depth) {
      keep[t] = 1;
      todo.push_back(h.src[t]);
    }
  for (const Encoded *o : {owner, stash})
    if (o) todo.insert(todo.end(), o->src.begin(), o->src.end());
  while (!todo.empty()) {
    const int64_t c = todo.back();
    todo.pop_back();
    auto it = by_dst.find(c);
    if (it == by_dst.end() || keep[it->second]) continue;
    keep[it->second] = 1;
    todo.push_back(h.src[it->second]);
  }
  return keep;
}

// Every group's phases (CopyPhase) segmented on the host threads from its
// encoded tables, enc[per_group * g + q]: q = 0 halo, 1 owner, 2 staging
// (per_group 4: the stash copies, then the copies from the staging slots).
int upload_encoded(Solve *S, const std::vector<Encoded> &enc, cudaStream_t st, int per_group = 2) {
  std::vector<std::vector<int64_t>> seg(kNumPhases * MHD_NUM_GROUPS);
  mhd::parallel_for(kNumPhases * MHD_NUM_GROUPS, [&](int q) {
    const int g = q / kNumPhases, phase = q % kNumPhases;
    const Encoded &h = enc[per_group * g], &o = enc[per_group * g + 1];
    const Encoded *stash = per_group > 2 ? &enc[per_group * g + 2] : nullptr;
    const Encoded *unstash = per_group > 2 ? &enc[per_group * g + 3] : nullptr;
    switch (phase) {
      case kPhHalo: {
        const std::vector<char> keep = step_halo_mask(h, &o, stash, kHaloDepth[g]);
        seg[q] = build_segments(h, S->es, -1, &keep);
        break;
      }
      case kPhOwner: seg[q] = build_segments(o, S->es, -1); break;
      case kPhHaloFull: seg[q] = build_segments(h, S->es, -1); break;
      case kPhStash: if (stash) seg[q] = build_segments(*stash, S->es, -1); break;
      default: if (unstash) seg[q] = build_segments(*unstash, S->es, -1); break;
    }
  });
  for (int q = 0; q < kNumPhases * MHD_NUM_GROUPS; ++q) {
    const int g = q / kNumPhases, phase = q % kNumPhases;
    S->T->tab_n[g][phase] = (int)(seg[q].size() / kSegWords);
    S->T->table_bytes += (int64_t)seg[q].size() * 8;
    const int rc = dev_upload(S->pool, seg[q], &S->T->tab_seg[g][phase], st);
    if (rc) return rc;
  }
  return MHD_OK;
}

// The encoded tables of a block periodic in every direction, straight from
// the periodic walks (mhd_periodic.h), without the explicit copy lists: one
// field component per host thread, a counting pass then a writing pass.
int upload_groups_periodic(Solve *S, cudaStream_t st) {
  using namespace mhd::periodic;
  const Box &bx = S->boxes[0];
  const int n[3] = {bx.n[0], bx.n[1], bx.n[2]}, g = S->nghost;
  struct Unit {
    const GroupSpec *gs;
    int field, m;
    size_t nh, no, oh, oo;
  };
  std::vector<Unit> units;
  for (const auto &gs : kGroups)
    for (int field : gs.fields)
      for (int m = 0; m < kFieldSpec[field].ncomp; ++m) units.push_back({&gs, field, m, 0, 0, 0, 0});
  const int nu = (int)units.size();
  mhd::parallel_for(nu, [&](int u) {
    Unit &U = units[u];
    walk_unit(*U.gs, U.field, U.m, n, g, [&](const mhd_copy &, bool own) { ++(own ? U.no : U.nh); });
  });
  std::vector<Encoded> enc(2 * MHD_NUM_GROUPS);
  size_t nh[MHD_NUM_GROUPS] = {}, no[MHD_NUM_GROUPS] = {};
  for (Unit &U : units) {
    U.oh = nh[U.gs->group];
    U.oo = no[U.gs->group];
    nh[U.gs->group] += U.nh;
    no[U.gs->group] += U.no;
  }
  for (int q = 0; q < MHD_NUM_GROUPS; ++q)
    for (int p = 0; p < 2; ++p) {
      Encoded &e = enc[2 * q + p];
      const size_t cnt = p ? no[q] : nh[q];
      e.dst.resize(cnt);
      e.src.resize(cnt);
      e.neg.assign(cnt, 0);
      e.depth.resize(cnt);
    }
  mhd::parallel_for(nu, [&](int u) {
    Unit &U = units[u];
    size_t ih = U.oh, io = U.oo;
    Encoded &eh = enc[2 * U.gs->group], &eo = enc[2 * U.gs->group + 1];
    // the arena code of (i, j, k) of this component: its array's base plus
    // the box offset (Solve::code for one block, without the lookups)
    const int c = kComp.first[U.field] + U.m;
    const int64_t base = S->comp_base(0, c, 0) | (c < kNumUComps ? kCodeUFlag : 0);
    const int64_t es = S->es, G = bx.G;
    const int *stg = kStagger[kFieldSpec[U.field].loc];
    auto code = [&](const mhd_dof &q) { return base + ((q.i + G) * bx.si + (q.j + G) * bx.sj + (q.k + G)) * es; };
    walk_unit(*U.gs, U.field, U.m, n, g, [&](const mhd_copy &cp, bool own) {
      Encoded &e = own ? eo : eh;
      const size_t t = own ? io++ : ih++;
      e.dst[t] = code(cp.dst);
      e.src[t] = code(cp.src);
      const int q[3] = {cp.dst.i, cp.dst.j, cp.dst.k};
      int depth = 0;
      for (int a = 0; a < 3; ++a) {
        const int hi = n[a] + stg[a];
        const int da = q[a] < 0 ? -q[a] : (q[a] >= hi ? q[a] - hi + 1 : 0);
        depth = da > depth ? da : depth;
      }
      e.depth[t] = (uint8_t)depth;
    });
  });
  for (Encoded &e : enc) {
    e.ascending = true;
    for (size_t t = 1; t < e.dst.size(); ++t)
      if (e.dst[t] <= e.dst[t - 1]) {
        e.ascending = false;
        break;
      }
  }
  // Sync(Eres) and Sync(dB) of a periodic block: the E edge and B face
  // copies (no physical boundary tells them apart)
  if (S->consts.resistive)
    for (int p = 0; p < 2; ++p) {
      enc[2 * MHD_SYNC_ERES + p] = enc[2 * MHD_SYNC_EEDGE + p];
      enc[2 * MHD_SYNC_DB + p] = enc[2 * MHD_SYNC_BFACE + p];
    }
  return upload_encoded(S, enc, st);
}

int upload_aliases(Solve *S, const mhd_alias_classes &a, cudaStream_t st);

// Edge alias classes of a periodic block (mhd_periodic.h).
int upload_aliases_periodic(Solve *S, cudaStream_t st) {
  const Box &bx = S->boxes[0];
  const int n[3] = {bx.n[0], bx.n[1], bx.n[2]};
  std::vector<int32_t> off;
  std::vector<mhd_dof> mem, own;
  std::vector<double> ms, os;
  mhd::periodic::alias_classes(n, off, mem, ms, own, os);
  mhd_alias_classes a{};
  a.n_classes = (int32_t)own.size();
  a.offset = off.data();
  a.member = mem.data();
  a.member_sign = ms.data();
  a.owner = own.data();
  a.owner_sign = os.data();
  return upload_aliases(S, a, st);
}

// Every group's explicit copy tables (the descriptor's) encoded on the host
// threads, then segmented and uploaded.
int upload_groups(Solve *S, const mhd_sync_group *groups, cudaStream_t st) {
  // every table's chunks on one pool of host threads
  // per group: halo, owner, staging in, staging out
  constexpr int NT = 4 * MHD_NUM_GROUPS;
  std::vector<Encoded> enc(NT);
  const mhd_copy *tabs[NT];
  int ntab[NT], first_chunk[NT + 1];
  first_chunk[0] = 0;
  for (int q = 0; q < NT; ++q) {
    const int g = q / 4, p = q % 4;
    const mhd_sync_group &G = groups[g];
    if (G.n_stash < 0 || (G.n_stash > 0 && !G.stash)) return fail(MHD_ERR_ARG, "group %d: bad staging table", g);
    tabs[q] = p == 0 ? G.halo : p == 1 ? G.owner : p == 2 ? G.stash : G.stash + G.n_stash;
    ntab[q] = p == 0 ? G.n_halo : p == 1 ? G.n_owner : G.n_stash;
    if (ntab[q] < 0 || (ntab[q] > 0 && !tabs[q])) return fail(MHD_ERR_ARG, "group %d phase %d: bad table", g, p);
    if ((g == MHD_SYNC_ERES || g == MHD_SYNC_DB) && !S->consts.resistive) ntab[q] = 0;  // only the implicit substep
    Encoded &e = enc[q];
    e.dst.resize(ntab[q]);
    e.src.resize(ntab[q]);
    e.neg.resize(ntab[q]);
    e.depth.resize(ntab[q]);
    first_chunk[q + 1] = first_chunk[q] + (ntab[q] + kEncodeChunk - 1) / kEncodeChunk;
  }
  const int nch = first_chunk[NT];
  std::vector<int> bad(nch), kind(nch, 0);
  std::vector<char> asc(nch);
  std::vector<int> chunk_table(nch);
  for (int q = 0; q < NT; ++q)
    for (int c = first_chunk[q]; c < first_chunk[q + 1]; ++c) chunk_table[c] = q;
  mhd::parallel_for(nch, [&](int c) {
    const int q = chunk_table[c];
    const int t0 = (c - first_chunk[q]) * kEncodeChunk, t1 = std::min(ntab[q], t0 + kEncodeChunk);
    encode_chunk(S, tabs[q], t0, t1, &enc[q], &bad[c], &kind[c], &asc[c]);
  });
  for (int q = 0; q < NT; ++q) {
    const int g = q / 4, p = q % 4;
    Encoded &e = enc[q];
    e.ascending = true;
    for (int c = first_chunk[q]; c < first_chunk[q + 1]; ++c) {
      if (bad[c] >= 0) {
        if (kind[c] == 1) return fail(MHD_ERR_ARG, "group %d phase %d: entry %d out of range", g, p, bad[c]);
        return fail(MHD_ERR_ARG, "group %d phase %d: entry %d has sign %g (must be +1 or -1)", g, p, bad[c],
                    tabs[q][bad[c]].sign);
      }
      const int t0 = (c - first_chunk[q]) * kEncodeChunk;
      if (!asc[c] || (t0 && e.dst[t0] <= e.dst[t0 - 1])) e.ascending = false;
    }
  }
  return upload_encoded(S, enc, st, 4);
}

int upload_aliases(Solve *S, const mhd_alias_classes &a, cudaStream_t st) {
  S->T->al_n = a.n_classes;
  if (a.n_classes <= 0) {
    S->T->al_n = 0;
    return MHD_OK;
  }
  if (!a.offset || !a.member || !a.member_sign || !a.owner || !a.owner_sign)
    return fail(MHD_ERR_ARG, "alias classes: null table");
  const int nm = a.offset[a.n_classes];
  std::vector<int64_t> mE(nm), mJ(nm), oE(a.n_classes), oJ(a.n_classes);
  const int ef[3] = {MHD_E_XI, MHD_E_ETA, MHD_E_ZETA}, jf[3] = {MHD_J_XI, MHD_J_ETA, MHD_J_ZETA};
  auto both = [&](mhd_dof d, int64_t *e, int64_t *j) {
    if (d.field < 0 || d.field > 2) return false;
    const int ax = d.field;
    bool o1, o2;
    d.field = ef[ax];
    *e = S->code(d, &o1);
    d.field = jf[ax];
    *j = S->code(d, &o2);
    return o1 && o2;
  };
  for (int q = 0; q < nm; ++q)
    if (!both(a.member[q], &mE[q], &mJ[q])) return fail(MHD_ERR_ARG, "alias member %d out of range", q);
  for (int c = 0; c < a.n_classes; ++c)
    if (!both(a.owner[c], &oE[c], &oJ[c])) return fail(MHD_ERR_ARG, "alias owner %d out of range", c);
  std::vector<int32_t> off(a.offset, a.offset + a.n_classes + 1);
  std::vector<double> ms(a.member_sign, a.member_sign + nm), os(a.owner_sign, a.owner_sign + a.n_classes);
  S->T->table_bytes += (int64_t)nm * 24 + (int64_t)a.n_classes * 28;
  int rc;
  if ((rc = dev_upload(S->pool, off, &S->T->al_off, st)) || (rc = dev_upload(S->pool, mE, &S->T->al_memE, st)) ||
      (rc = dev_upload(S->pool, mJ, &S->T->al_memJ, st)) || (rc = dev_upload(S->pool, oE, &S->T->al_ownE, st)) ||
      (rc = dev_upload(S->pool, oJ, &S->T->al_ownJ, st)) || (rc = dev_upload(S->pool, ms, &S->T->al_msign, st)) ||
      (rc = dev_upload(S->pool, os, &S->T->al_osign, st)))
    return rc;
  return MHD_OK;
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), null when the
// driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    cudaGetLastError();
  });
  return fn;
}

// TMA tensor maps of a solve's blocks for the staged fluid variant: per
// block U buffer 0 and U buffer 1 (4-D: k, j, i over the row pitch and the
// box extents, and the 10 U components; box tma_box_k x 6 x 6 x 1) and the
// real-valued M components through the primitive variables (box of 4
// components: u, v, w, p).  Copies that reach past the arrays read zeros.
// A block whose maps cannot be encoded keeps tmap null (the kernel then
// loads its boxes itself).
int upload_tmaps(Solve *S, std::vector<DevBlock> &blocks, cudaStream_t st) {
  for (DevBlock &d : blocks) d.tmap = nullptr;
  const auto enc = tmap_encoder();
  if (!enc) return MHD_OK;
  const int es = S->es;
  std::vector<CUtensorMap> maps(3 * blocks.size());
  std::vector<char> ok(blocks.size(), 0);
  for (size_t bi = 0; bi < blocks.size(); ++bi) {
    const Box &bx = S->boxes[bi];
    const cuuint64_t strides[3] = {(cuuint64_t)(bx.sj * es), (cuuint64_t)(bx.si * es), (cuuint64_t)(bx.total * es)};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    bool good = true;
    for (int q = 0; q < 3 && good; ++q) {
      void *base = q < 2 ? blocks[bi].U[q] : (void *)(blocks[bi].M + (int64_t)kNumMetric * bx.total * 8);
      const cuuint64_t dims[4] = {(cuuint64_t)bx.sj, (cuuint64_t)bx.ext[1], (cuuint64_t)bx.ext[0],
                                  (cuuint64_t)(q < 2 ? kNumUComps : kTmaMComps)};
      const cuuint32_t box[4] = {(cuuint32_t)tma_box_k(es), kTmaBoxJI, kTmaBoxJI, q < 2 ? 1u : 4u};
      good = enc(&maps[3 * bi + q], es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base,
                 dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    ok[bi] = good;
  }
  int rc;
  CUtensorMap *d = nullptr;
  if ((rc = dev_upload(S->pool, maps, &d, st))) return rc;
  S->dtmaps = d;
  if (((uintptr_t)d & 63) != 0) return MHD_OK;  // tensor maps in global memory must be 64-byte aligned
  for (size_t bi = 0; bi < blocks.size(); ++bi)
    if (ok[bi]) blocks[bi].tmap = d + 3 * bi;
  return MHD_OK;
}

void free_solve(Solve *S, cudaStream_t st) {
  if (!S) return;
  auto f = [&](void *p) {
    if (p) cudaFreeAsync(p, st);
  };
  f(S->arena);
  f(S->dblocks);
  f(S->dtmaps);
  f(S->sg_geo);
  f(S->sg_w);
  f(S->dres_prefix);
  Tables *T = S->T;
  if (T && --T->users == 0) {
    for (int r = 0; r < kNumRanges; ++r) f(T->dtile_prefix[r]);
    for (int g = 0; g < kMaxGroups; ++g)
      for (int p = 0; p < kNumPhases; ++p) f(T->tab_seg[g][p]);
    for (int q = 0; q < kNumPhys; ++q) {
      f(T->ph_set[q]);
      f(T->ph_op[q]);
    }
    for (void *p : {(void *)T->al_off, (void *)T->al_memE, (void *)T->al_ownE, (void *)T->al_memJ, (void *)T->al_ownJ,
                    (void *)T->al_msign, (void *)T->al_osign, (void *)T->sg_owner, (void *)T->sg_osign,
                    (void *)T->sg_aoff, (void *)T->sg_alias, (void *)T->sg_coff, (void *)T->sg_cell,
                    (void *)T->sg_foff, (void *)T->sg_face})
      f(p);
    delete T;
  }
  delete S;
}

int set_state_field(mhd_batch *b, int slot, size_t offset, const void *src, size_t bytes) {
  CUDA_TRY(cudaMemcpyAsync((char *)(b->dstate + slot) + offset, src, bytes, cudaMemcpyHostToDevice, b->stream));
  return MHD_OK;
}

int read_state(mhd_batch *b) {
  CUDA_TRY(cudaMemcpyAsync(b->hstate, b->dstate, sizeof(SolveState) * b->capacity, cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MHD_OK;
}

int slot_check(mhd_batch *b, int slot) {
  if (!b) return fail(MHD_ERR_ARG, "null batch");
  if (slot < 0 || slot >= b->capacity || !b->slots[slot]) return fail(MHD_ERR_ARG, "slot %d is not in use", slot);
  return MHD_OK;
}

// Runs `enqueue` over slot `slot` alone (the kernels' mode 1 selects slots by mask).
template <class F>
int targeted(mhd_batch *b, int slot, F &&enqueue) {
  const int one = 1, zero = 0;
  int rc = set_state_field(b, slot, offsetof(SolveState, mask), &one, sizeof one);
  if (rc) return rc;
  int nk = 0;
  enqueue(&nk);
  CUDA_TRY(cudaGetLastError());
  return set_state_field(b, slot, offsetof(SolveState, mask), &zero, sizeof zero);
}

template <class F>
int capture(mhd_batch *b, cudaGraphExec_t *out, int *nk_out, F &&enqueue) {
  if (*out) return MHD_OK;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int nk = 0;
  enqueue(&nk);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  if (nk_out) *nk_out = nk;
  return MHD_OK;
}

int build_graph(mhd_batch *b) {
  return capture(b, &b->graph, &b->kernels_per_step, [&](int *nk) { enqueue_step(b, nk); });
}

bool count_tables(mhd_batch *b, const Solve *S, int d) {
  bool grew = false;
  for (int g = 0; g < MHD_NUM_GROUPS; ++g)
    for (int p = 0; p < kNumPhases; ++p)
      if (S->T->tab_n[g][p] > 0) {
        grew = grew || (d > 0 && b->live_tables[g][p] == 0);
        b->live_tables[g][p] += d;
      }
  for (int q = 0; q < kNumPhys; ++q)
    if (S->T->ph_nset[q] + S->T->ph_nop[q] > 0) {
      grew = grew || (d > 0 && b->live_phys[q] == 0);
      b->live_phys[q] += d;
    }
  if (S->T->sg_n > 0) {
    grew = grew || (d > 0 && b->live_sing == 0);
    b->live_sing += d;
  }
  if (S->consts.resistive && !S->T->res_ghost_writes_only) {
    grew = grew || (d > 0 && b->n_res_full == 0);
    b->n_res_full += d;
  }
  return grew;
}

// The step graphs are captured again at the next run (call with no graph
// launch in flight).
void drop_graphs(mhd_batch *b) {
  for (cudaGraphExec_t *g : {&b->graph, &b->graph_a, &b->graph_b, &b->graph_cg})
    if (*g) {
      cudaGraphExecDestroy(*g);
      *g = nullptr;
    }
}

// Dot product of the CG (2 values) into b->hres.
int res_dot(mhd_batch *b) {
  int nk = 0;
  launch(b, 1, SK_RES_DOT, &nk);
  launch(b, 1, SK_RES_SUM, &nk);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(b->hres, b->res.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MHD_OK;
}

// q = A p (MatMultImplicitResistive_, Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:420-472):
// E_res from p, its owner copies, dB = -dt curl E_res, Sync(dB), dJ, its
// alias reduction and owner copies, q = E_res - eta dJ.
// On grids with physical boundaries or rotated seams the full Sync(Eres),
// Sync(dB) and Sync(dJ) run, in the reference's order, with the singular
// edges' current between the dJ alias reduction and its owner copies; the
// unknowns read only owned values (no copy of these groups writes an owned
// position from a ghost one), so of Sync(Eres) and Sync(dJ) only the owner
// copies change q, and dB is read one ghost layer out.
bool open_grids(const mhd_batch *b) {
  if (b->live_sing > 0) return true;
  for (int q = 0; q < kNumPhys; ++q)
    if (b->live_phys[q] > 0) return true;
  for (int g = 0; g < kMaxGroups; ++g)
    if (b->live_tables[g][kPhStash] > 0) return true;
  return false;
}
// Sync(group) after its owner copies already ran: the owner copies again
// only when the halo phase may have changed a source of them.
void sync_after_owner(mhd_batch *b, int mode, int g, int *nk) {
  if (b->live_phys[g] == 0 && b->live_tables[g][kPhHalo] == 0 && b->live_tables[g][kPhStash] == 0) return;
  enqueue_sync(b, mode, g, nk);
}
// With every solve's Sync(Eres) and Sync(Jedge) writing ghosts only (beyond
// their owner copies; res_ghost_writes_only), the substep runs the owner
// copies of E_res and the alias reduction of dJ and leaves out the rest of
// those two syncs: nothing it reads changes.
bool res_light_syncs(const mhd_batch *b) { return b->n_res_full == 0; }
void res_sync_eres(mhd_batch *b, int *nk) {
  sync1(b, 1, copy_op(MHD_SYNC_ERES, kPhOwner), nk);                  // HALO_OWNER::sync_edge_1form
  if (!res_light_syncs(b)) sync_after_owner(b, 1, MHD_SYNC_ERES, nk);  // Sync("Eres")
}
void res_sync_dj(mhd_batch *b, int *nk) {  // after the current's alias reduction and the singular edges
  if (res_light_syncs(b)) return;
  sync1(b, 1, copy_op(MHD_SYNC_JEDGE, kPhOwner), nk);
  sync_after_owner(b, 1, MHD_SYNC_JEDGE, nk);  // Sync("dJ")
}
void res_apply_core(mhd_batch *b, int *nk) {  // from E_res (set) to dJ (synced)
  res_sync_eres(b, nk);
  launch(b, 1, SK_RES_DB, nk);  // the ghost faces were cleared at the substep's start (res_step)
  enqueue_sync(b, 1, MHD_SYNC_DB, nk);
  launch(b, 1, SK_RES_DJ, nk);
  sync1(b, 1, alias_op(1), nk);
  if (b->live_sing > 0) launch(b, 1, SK_SING_J, nk);  // AssembleSingularEdgeCurrent_(dB, dJ)
  res_sync_dj(b, nk);
}
void res_apply(mhd_batch *b, int *nk) {
  launch(b, 1, SK_RES_VEC, nk, nullptr, RES_E_FROM_P);
  res_apply_core(b, nk);
  launch(b, 1, SK_RES_Q, nk);
}

// The CG iteration loop of every masked solve as one CUDA graph: k_res_cg
// and k_res_cg_sum (CG_INIT) set the loop condition, then a conditional
// WHILE node repeats the iteration (operator, q and (p.q)_W, the x / r update
// and the stop test, the direction update) while some solve's device CG
// state says it is still running; a solve whose loop ends leaves the mask.
// Captured once per batch (again after the tables or the partials change).
int build_cg_graph(mhd_batch *b) {
  if (b->graph_cg) return MHD_OK;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaGraphCreate(&g, 0));
  const bool prof = b->profiling;
  b->profiling = false;  // no event records inside the graph
  auto fin = [&](cudaError_t e, const char *what) {
    b->profiling = prof;
    b->res.in_graph = 0;
    cudaGraphDestroy(g);
    return fail(MHD_ERR_CUDA, "CG graph, %s: %s", what, cudaGetErrorString(e));
  };
  cudaGraphConditionalHandle h = 0;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return fin(e, "condition");
  b->res.handle = h;
  b->res.in_graph = 1;  // captured launches set the loop condition
  int nk = 0;
  if ((e = cudaStreamBeginCaptureToGraph(b->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return fin(e, "capture");
  launch(b, 1, SK_RES_CG, &nk, nullptr, CG_INIT);
  launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_INIT);
  if ((e = cudaStreamEndCapture(b->stream, &g)) != cudaSuccess) return fin(e, "capture");
  // the loop node follows the chain's last node
  cudaGraphNode_t nodes[2] = {};
  size_t n = 2;
  if ((e = cudaGraphGetNodes(g, nodes, &n)) != cudaSuccess || n != 2)
    return fin(e != cudaSuccess ? e : cudaErrorUnknown, "init nodes");
  cudaGraphNode_t init = nullptr;
  for (cudaGraphNode_t c : nodes) {
    size_t nd = 0;
    if ((e = cudaGraphNodeGetDependentNodes(c, nullptr, &nd)) != cudaSuccess) return fin(e, "init nodes");
    if (nd == 0) init = c;
  }
  if (!init) return fin(cudaErrorUnknown, "init nodes");
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t loop = nullptr;
  if ((e = cudaGraphAddNode(&loop, g, &init, 1, &p)) != cudaSuccess) return fin(e, "loop node");
  cudaGraph_t body = p.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return fin(e, "body capture");
  res_apply_core(b, &nk);
  launch(b, 1, SK_RES_CG, &nk, nullptr, CG_PQ);
  launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_PQ);
  launch(b, 1, SK_RES_CG, &nk, nullptr, CG_RR);
  launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_RR);
  launch(b, 1, SK_RES_PUPD_E, &nk);
  if ((e = cudaStreamEndCapture(b->stream, &body)) != cudaSuccess) return fin(e, "body capture");
  e = cudaGraphInstantiate(&b->graph_cg, g, 0);
  b->profiling = prof;
  b->res.in_graph = 0;
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->graph_cg = nullptr;
    return fail(MHD_ERR_CUDA, "CG graph instantiate: %s", cudaGetErrorString(e));
  }
  return MHD_OK;
}

// The per-warp tile partials of the batched CG: 2 doubles per warp of every
// kResK tile of the batch's solves (grown on demand; the loop graph holds the
// pointer, so a new buffer means a new graph).
int ensure_tpartial(mhd_batch *b) {
  size_t tiles = 0;
  for (int s = 0; s < b->capacity; ++s)
    if (const Solve *S = b->slots[s]) tiles += (size_t)(S->dres_prefix ? S->res_tiles : S->T->tiles[kResK]);
  const size_t need = std::max<size_t>(tiles, 1) * kWarpsPerTile * 2;
  if (need <= b->tpart_elems) return MHD_OK;
  CUDA_TRY(cudaStreamSynchronize(b->stream));  // no loop graph in flight
  if (b->graph_cg) {
    cudaGraphExecDestroy(b->graph_cg);
    b->graph_cg = nullptr;
  }
  cudaFree(b->res.tpartial);
  b->res.tpartial = nullptr;
  b->tpart_elems = 0;
  if (cudaMalloc(&b->res.tpartial, sizeof(double) * need) != cudaSuccess) {
    cudaGetLastError();
    return fail(MHD_ERR_OOM, "CG partials of %zu doubles", need);
  }
  b->tpart_elems = need;
  return MHD_OK;
}

// Sets every slot's mask (one strided copy of the mask fields).
int apply_masks(mhd_batch *b, const std::vector<int> &on) {
  CUDA_TRY(cudaMemcpy2DAsync((char *)b->dstate + offsetof(SolveState, mask), sizeof(SolveState), on.data(),
                             sizeof(int), sizeof(int), (size_t)b->capacity, cudaMemcpyHostToDevice, b->stream));
  return MHD_OK;
}

// One CG job of the batched loop: the slot, its stop factor and iteration cap.
struct CgJob {
  int slot;
  double tol_factor;
  int max_it;
};

// CG on every job's solve at once, each from x = 0 and p = r = its
// right-hand side (r already set), until ||r|| <= tol_factor ||r_0|| or max_it
// iterations, the loop on the device (build_cg_graph); the jobs' masks are
// set here and are all clear on return; one host round trip at the end.
// Each job's final state is in b->hcg[slot].
int res_cg_batch(mhd_batch *b, const std::vector<CgJob> &jobs) {
  int rc;
  if ((rc = ensure_tpartial(b)) || (!b->cg_host_loop && (rc = build_cg_graph(b)))) return rc;
  std::vector<int> on((size_t)b->capacity, 0);
  for (int s = 0; s < b->capacity; ++s) {
    b->hcg[s] = ResCG{};
    b->hcg[s].done = 1;
  }
  for (const CgJob &j : jobs) {
    ResCG &h = b->hcg[j.slot];
    h.done = 0;
    h.tol_factor = j.tol_factor;
    h.max_it = std::max(0, std::min(j.max_it, 100000));  // the loop runs on the device: a hard bound
    on[j.slot] = 1;
  }
  if ((rc = apply_masks(b, on))) return rc;
  CUDA_TRY(cudaMemcpyAsync(b->res.cg, b->hcg, sizeof(ResCG) * b->capacity, cudaMemcpyHostToDevice, b->stream));
  if (!b->cg_host_loop) {
    CUDA_TRY(cudaGraphLaunch(b->graph_cg, b->stream));
  } else {  // the same kernels launched from the host, the states read back after every iteration
    int nk = 0;
    launch(b, 1, SK_RES_CG, &nk, nullptr, CG_INIT);
    launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_INIT);
    for (;;) {
      CUDA_TRY(cudaMemcpyAsync(b->hcg, b->res.cg, sizeof(ResCG) * b->capacity, cudaMemcpyDeviceToHost, b->stream));
      CUDA_TRY(cudaStreamSynchronize(b->stream));
      bool running = false;
      for (int s = 0; s < b->capacity; ++s) running = running || !b->hcg[s].done;
      if (!running) break;  // every solve's loop ends by its own max_it at the latest
      res_apply_core(b, &nk);
      launch(b, 1, SK_RES_CG, &nk, nullptr, CG_PQ);
      launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_PQ);
      launch(b, 1, SK_RES_CG, &nk, nullptr, CG_RR);
      launch(b, 1, SK_RES_CGSUM, &nk, nullptr, CG_RR);
      launch(b, 1, SK_RES_PUPD_E, &nk);
    }
  }
  CUDA_TRY(cudaMemcpyAsync(b->hcg, b->res.cg, sizeof(ResCG) * b->capacity, cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  std::fill(on.begin(), on.end(), 0);
  return apply_masks(b, on);
}

// The mixed-precision solve of (I + dt eta alpha C^T beta C) E = b on the
// solve's FP64 companion (widened alpha, beta, eta, W; its own copies of the
// E / B / J syncs); b = eta J(B*) is the FP32 step's current (the state is
// FP32).  While the previous substep took at most res_direct iterations
// the companion runs the CG itself in FP64 (one host round trip); after a
// longer one, iterative refinement: the residual r = b - A x and its norms in
// FP64 on the companion, each correction A d = r solved by FP32 CG on the
// solve's own arrays to 1e-4 of ||r||, x += d in FP64 (half the bytes per
// iteration, two more round trips and an FP64 operator per refinement).  On
// return the solve's x holds the solution rounded to FP32.
constexpr int kDirectIters = 20;
int direct_iters(const mhd_constants &k) { return k.res_direct_iters == 0 ? kDirectIters : k.res_direct_iters; }

int res_refine(mhd_batch *b, int slot, Solve *S, bool *converged) {
  mhd_batch *sh = b->shadow;
  const int cs = S->shadow_slot;
  const Dir Dm = b->dir(1);
  cudaStream_t st = b->stream;
  constexpr int kMaxRefinements = 30;
  constexpr double kInnerRtol = 1e-4;
  int rc, nk = 0;
  std::vector<int> mb((size_t)b->capacity, 0), ms((size_t)sh->capacity, 0);
  mb[slot] = 1;
  ms[cs] = 1;
  if ((rc = apply_masks(b, mb)) || (rc = apply_masks(sh, ms))) return rc;
  // the companion's dt, b and x = 0; its dB ghost faces
  launch_res_cross(Dm, RES_X_SETUP, st);
  if (open_grids(sh)) launch(sh, 1, SK_RES_CLEARB, &nk);
  CUDA_TRY(cudaGetLastError());
  const double rtol = S->res_rtol > 0.0 ? S->res_rtol : 1e-10;
  if ((rc = res_dot(sh))) return rc;
  const double bnorm = std::sqrt(sh->hres[1]);
  double rn = bnorm;
  S->res_iters = 0;
  S->res_refinements = 0;
  for (;;) {
    if (S->res_refinements > 0) {  // r = b - A x in FP64
      launch(sh, 1, SK_RES_VEC, &nk, nullptr, RES_P_FROM_X);
      res_apply(sh, &nk);
      launch(sh, 1, SK_RES_VEC, &nk, nullptr, RES_RESID);
      if ((rc = res_dot(sh))) return rc;
      rn = std::sqrt(sh->hres[1]);
    }
    if (rn <= rtol * bnorm) {
      *converged = true;
      break;
    }
    if (S->res_refinements == kMaxRefinements || !(rn == rn)) break;
    // the correction: FP32 CG on r rounded to FP32, x += d in FP64
    launch_res_cross(Dm, RES_X_DEMOTE_R, st);
    if ((rc = res_cg_batch(b, {CgJob{slot, kInnerRtol, S->res_max_it}}))) return rc;
    if ((rc = apply_masks(b, mb))) return rc;  // the loop cleared it
    launch_res_cross(Dm, RES_X_ADD_X, st);
    S->res_iters += b->hcg[slot].it;
    ++S->res_refinements;
  }
  S->res_relres = bnorm > 0.0 ? rn / bnorm : 0.0;
  launch_res_cross(Dm, RES_X_DEMOTE_X, st);
  CUDA_TRY(cudaGetLastError());
  std::fill(ms.begin(), ms.end(), 0);
  return apply_masks(sh, ms);
}

// The implicit resistive substep (SolveImplicitResistiveDiffusion_,
// Mercury_ImplicitResistive.cpp:475-555) of every listed solve at once,
// after the explicit update and its Sync(B faces): B* snapshot, J(B*),
// b = eta J(B*), the solves (FP64: CG in the inner product weighted by
// 1 / (eta alpha), in which A is self-adjoint, all solves in one device
// loop; mixed precision: the short ones as FP64 CG on their companions in
// one loop, the others by res_refine), then B = B* - dt curl E_res.  The
// reference solves with GMRES; the solution is the same to the solvers'
// tolerance.  A solve that did not converge gets MHD_ERR_SOLVE.
int res_step(mhd_batch *b, const std::vector<int> &slots) {
  if (slots.empty()) return MHD_OK;
  cudaStream_t st = b->stream;
  std::vector<int> on((size_t)b->capacity, 0);
  for (int s : slots) on[s] = 1;
  int rc = apply_masks(b, on);
  if (rc) return rc;
  int nk = 0;
  launch(b, 1, SK_RES_COPYB, &nk, nullptr, RES_SNAPSHOT);
  // Calc_J_Edge on B* over the substep's range (the formula of k_bcell_jedge's
  // J part; B_cell is refreshed after the substep)
  launch(b, 1, SK_RES_DJ, &nk);
  sync1(b, 1, alias_op(1), &nk);
  if (b->live_sing > 0) launch(b, 1, SK_SING_J, &nk);  // reads B* around the singular edges
  res_sync_dj(b, &nk);
  launch(b, 1, SK_RES_VEC, &nk, nullptr, RES_INIT);
  // the B arrays turn into the operator's dB: its ghost faces start at zero
  // (restored with B* at the end)
  if (open_grids(b)) launch(b, 1, SK_RES_CLEARB, &nk);
  std::vector<char> conv((size_t)b->capacity, 0);
  auto take = [&](Solve *S, const ResCG &h, int s) {
    S->res_iters = h.it;
    S->res_refinements = 0;
    S->res_relres = h.r0 > 0.0 ? h.rnorm / h.r0 : 0.0;
    conv[s] = h.converged != 0;
  };
  if (b->precision != kMixed) {
    std::vector<CgJob> jobs;
    for (int s : slots) {
      const Solve *S = b->slots[s];
      jobs.push_back(CgJob{s, S->res_rtol > 0.0 ? S->res_rtol : 1e-13, S->res_max_it});
    }
    if ((rc = res_cg_batch(b, jobs))) return rc;
    for (int s : slots) take(b->slots[s], b->hcg[s], s);
  } else {
    mhd_batch *sh = b->shadow;
    std::vector<int> direct, refine;
    for (int s : slots) {
      const Solve *S = b->slots[s];
      (S->res_direct >= 0 && S->res_iters <= S->res_direct ? direct : refine).push_back(s);
    }
    if (!direct.empty()) {
      // FP64 CG on the companions of the short solves, from x = 0, p = r = b
      std::vector<int> mb((size_t)b->capacity, 0), ms((size_t)sh->capacity, 0);
      std::vector<CgJob> jobs;
      for (int s : direct) {
        const Solve *S = b->slots[s];
        mb[s] = 1;
        ms[S->shadow_slot] = 1;
        jobs.push_back(CgJob{S->shadow_slot, S->res_rtol > 0.0 ? S->res_rtol : 1e-10, S->res_max_it});
      }
      if ((rc = apply_masks(b, mb)) || (rc = apply_masks(sh, ms))) return rc;
      launch_res_cross(b->dir(1), RES_X_SETUP, st);
      if (open_grids(sh)) launch(sh, 1, SK_RES_CLEARB, &nk);  // the companions' dB ghost faces
      if ((rc = res_cg_batch(sh, jobs))) return rc;
      launch_res_cross(b->dir(1), RES_X_DEMOTE_X, st);
      CUDA_TRY(cudaGetLastError());
      for (int s : direct) take(b->slots[s], sh->hcg[b->slots[s]->shadow_slot], s);
    }
    for (int s : refine) {
      bool c = false;
      if ((rc = res_refine(b, s, b->slots[s], &c))) return rc;
      conv[s] = c;
    }
  }
  if ((rc = apply_masks(b, on))) return rc;  // the loops left their solves' masks clear
  for (int s : slots)
    if (!conv[s]) {
      const int e = MHD_ERR_SOLVE;
      if ((rc = set_state_field(b, s, offsetof(SolveState, status), &e, sizeof e))) return rc;
    }
  // E_res = x, its owner copies; B = B* + dt (-curl E_res) on the owned faces
  launch(b, 1, SK_RES_VEC, &nk, nullptr, RES_E_FROM_X);
  res_sync_eres(b, &nk);
  launch(b, 1, SK_RES_COPYB, &nk, nullptr, RES_RESTORE);
  launch(b, 1, SK_RES_BUPDATE, &nk);
  CUDA_TRY(cudaGetLastError());
  std::fill(on.begin(), on.end(), 0);
  return apply_masks(b, on);
}

int xfer(mhd_batch *b, int slot, int field, int block, const int32_t lo[3], const int32_t hi[3], int ncomp,
         Solve **S_out) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  Solve *S = b->slots[slot];
  if (field < 0 || field >= MHD_NUM_FIELDS || block < 0 || block >= S->nblocks || !lo || !hi)
    return fail(MHD_ERR_ARG, "transfer: bad arguments");
  if (ncomp != kFieldSpec[field].ncomp)
    return fail(MHD_ERR_ARG, "field %d has %d components, got %d", field, kFieldSpec[field].ncomp, ncomp);
  if (kComp.first[field] >= kFirstResComp && !S->consts.resistive)
    return fail(MHD_ERR_ARG, "field %d exists only in solves with the implicit resistive substep", field);
  const Box &bx = S->boxes[block];
  for (int a = 0; a < 3; ++a)
    if (lo[a] < -bx.G || hi[a] > bx.n[a] + 1 + bx.G || hi[a] <= lo[a])
      return fail(MHD_ERR_ARG, "transfer range [%d,%d) outside the block box on axis %d", lo[a], hi[a], a);
  *S_out = S;
  return MHD_OK;
}

}  // namespace

extern "C" {

const char *mhd_last_error(void) { return g_last_error.c_str(); }

int mhd_field_info(int field, int32_t *ncomp, int32_t *location) {
  if (field < 0 || field >= MHD_NUM_FIELDS) return fail(MHD_ERR_ARG, "field %d out of range", field);
  if (ncomp) *ncomp = kFieldSpec[field].ncomp;
  if (location) *location = kFieldSpec[field].loc;
  return MHD_OK;
}

// ------------------------------------------------------------------ batch API
int mhd_batch_create(int capacity, int precision, mhd_batch **out) {
  if (!out || capacity < 1 || capacity > 65536) return fail(MHD_ERR_ARG, "mhd_batch_create: capacity %d", capacity);
  if (precision != kFP64 && precision != kMixed) return fail(MHD_ERR_ARG, "mhd_batch_create: precision %d", precision);
  *out = nullptr;
  init_launch_grids();
  auto *b = new (std::nothrow) mhd_batch();
  if (!b) return fail(MHD_ERR_OOM, "host allocation");
  b->capacity = capacity;
  b->precision = precision;
  b->slots.assign(capacity, nullptr);
  auto bail = [&](int rc) {
    mhd_batch_destroy(b);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "stream create"));
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolCreate(&b->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
      b->pool = nullptr;
      return bail(fail(MHD_ERR_CUDA, "memory pool create"));
    }
  }
  const size_t C1 = (size_t)capacity + 1;
  if (cudaMalloc(&b->dsolves, sizeof(DevSolve) * capacity) != cudaSuccess ||
      cudaMalloc(&b->dstate, sizeof(SolveState) * capacity) != cudaSuccess ||
      cudaMalloc(&b->comp_ptrs, sizeof(void *) * 72) != cudaSuccess ||
      cudaMallocHost(&b->hstate, sizeof(SolveState) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->hsnap[0], sizeof(SolveState) * capacity) != cudaSuccess ||
      cudaMallocHost(&b->hsnap[1], sizeof(SolveState) * capacity) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->snap_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->snap_ev[1], cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(MHD_ERR_OOM, "directory of %d slots", capacity));
  for (int r = 0; r < kNumRanges; ++r)
    if (cudaMalloc(&b->dprefix_tiles[r], sizeof(int) * C1) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "prefix"));
  for (int g = 0; g < kMaxGroups; ++g)
    for (int p = 0; p < kNumPhases; ++p)
      if (cudaMalloc(&b->dprefix_copy[g][p], sizeof(int) * C1) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "prefix"));
  for (int q = 0; q < kNumPhys; ++q)
    if (cudaMalloc(&b->dprefix_phys[q], sizeof(int) * C1) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "prefix"));
  if (cudaMalloc(&b->dprefix_sing, sizeof(int) * C1) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "prefix"));
  if (cudaMalloc(&b->dprefix_aliasE, sizeof(int) * C1) != cudaSuccess ||
      cudaMalloc(&b->dprefix_aliasJ, sizeof(int) * C1) != cudaSuccess)
    return bail(fail(MHD_ERR_OOM, "prefix"));
  if (cudaMalloc(&b->res.partial, sizeof(double) * 2 * res_dot_grid()) != cudaSuccess ||
      cudaMalloc(&b->res.result, sizeof(double) * 2) != cudaSuccess ||
      cudaMalloc(&b->res.cg, sizeof(ResCG) * capacity) != cudaSuccess ||
      cudaMalloc(&b->res.ctl, sizeof(ResCtl)) != cudaSuccess ||
      cudaMemsetAsync(b->res.ctl, 0, sizeof(ResCtl), b->stream) != cudaSuccess ||
      cudaMalloc(&b->res.chunks, sizeof(double) * 2 * kCgChunks * capacity) != cudaSuccess ||
      cudaMalloc(&b->res.sarrivals, sizeof(unsigned int) * capacity) != cudaSuccess ||
      cudaMemsetAsync(b->res.sarrivals, 0, sizeof(unsigned int) * capacity, b->stream) != cudaSuccess ||
      cudaMallocHost(&b->hres, sizeof(double) * 2) != cudaSuccess ||
      cudaMallocHost(&b->hcg, sizeof(ResCG) * capacity) != cudaSuccess)
    return bail(fail(MHD_ERR_OOM, "solver scratch"));
  if (cudaMemsetAsync(b->dstate, 0, sizeof(SolveState) * capacity, b->stream) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "state init"));
  int rc = publish(b);
  if (rc) return bail(rc);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(fail(MHD_ERR_CUDA, "batch init"));
  *out = b;
  return MHD_OK;
}

int mhd_batch_destroy(mhd_batch *b) {
  if (!b) return MHD_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->shadow) mhd_batch_destroy(b->shadow);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->graph_a) cudaGraphExecDestroy(b->graph_a);
  if (b->graph_b) cudaGraphExecDestroy(b->graph_b);
  if (b->graph_cg) cudaGraphExecDestroy(b->graph_cg);
  for (cudaEvent_t e : b->res_ev)
    if (e) cudaEventDestroy(e);
  cudaFree(b->res.partial);
  cudaFree(b->res.result);
  cudaFree(b->res.cg);
  cudaFree(b->res.ctl);
  cudaFree(b->res.chunks);
  cudaFree(b->res.sarrivals);
  cudaFree(b->res.tpartial);
  if (b->hres) cudaFreeHost(b->hres);
  if (b->hcg) cudaFreeHost(b->hcg);
  for (auto *S : b->slots) free_solve(S, b->stream);
  if (b->staging) cudaFreeAsync(b->staging, b->stream);
  if (b->stream) cudaStreamSynchronize(b->stream);
  cudaFree(b->dsolves);
  cudaFree(b->dstate);
  cudaFree(b->comp_ptrs);
  if (b->hstate) cudaFreeHost(b->hstate);
  for (int q = 0; q < 2; ++q) {
    if (b->hsnap[q]) cudaFreeHost(b->hsnap[q]);
    if (b->snap_ev[q]) cudaEventDestroy(b->snap_ev[q]);
  }
  for (int r = 0; r < kNumRanges; ++r) cudaFree(b->dprefix_tiles[r]);
  for (int g = 0; g < kMaxGroups; ++g)
    for (int p = 0; p < kNumPhases; ++p) cudaFree(b->dprefix_copy[g][p]);
  for (int q = 0; q < kNumPhys; ++q) cudaFree(b->dprefix_phys[q]);
  cudaFree(b->dprefix_sing);
  cudaFree(b->dprefix_aliasE);
  cudaFree(b->dprefix_aliasJ);
  for (auto e : b->prof_events) cudaEventDestroy(e);
  if (b->stream && !b->borrowed) cudaStreamDestroy(b->stream);
  if (b->pool && !b->borrowed) cudaMemPoolDestroy(b->pool);  // every allocation from it was freed and the stream drained
  delete b;
  return MHD_OK;
}

int mhd_batch_reserve(mhd_batch *b, int64_t bytes) {
  if (!b || bytes < 0) return fail(MHD_ERR_ARG, "mhd_batch_reserve: bad arguments");
  if (bytes == 0) return MHD_OK;
  void *p = nullptr;
  if (cudaMallocFromPoolAsync(&p, (size_t)bytes, b->pool, b->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(MHD_ERR_OOM, "mhd_batch_reserve: %lld bytes", (long long)bytes);
  }
  CUDA_TRY(cudaFreeAsync(p, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MHD_OK;
}

int64_t mhd_desc_device_bytes(const mhd_desc *desc) {
  if (!desc || desc->n_blocks < 1 || !desc->cells || desc->nghost < 1) return -1;
  int64_t bytes = 0;
  for (int b = 0; b < desc->n_blocks; ++b) {
    const int n[3] = {desc->cells[3 * b], desc->cells[3 * b + 1], desc->cells[3 * b + 2]};
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) return -1;
    const Box bx = make_box(n, desc->nghost);
    const int64_t es = desc->precision == kMixed ? 4 : 8;
    const int64_t nr = kNumRComps - (desc->constants.resistive ? 0 : kNumResComps);
    bytes += ((int64_t)kNumMetric * 8 + (nr + 2 * kNumUComps) * es) * bx.total;
  }
  for (int g = 0; g < MHD_NUM_GROUPS; ++g)
    bytes += (int64_t)(desc->groups[g].n_halo + desc->groups[g].n_owner + 2 * desc->groups[g].n_stash) * 24 +
             (int64_t)desc->groups[g].n_phys * sizeof(DevPhysOp);
  bytes += (int64_t)desc->n_staging * (desc->precision == kMixed ? 4 : 8) + 256 +
           (int64_t)desc->n_wall * 8 + (int64_t)desc->singular.n_edges * 128;
  if (desc->edge_aliases.n_classes > 0 && desc->edge_aliases.offset)
    bytes += (int64_t)desc->edge_aliases.offset[desc->edge_aliases.n_classes] * 24 +
             (int64_t)desc->edge_aliases.n_classes * 28;
  if (desc->precision == kMixed && desc->constants.resistive) {  // the FP64 companion of the implicit substep
    mhd_desc d64 = *desc;
    d64.precision = kFP64;
    bytes += mhd_desc_device_bytes(&d64);
  }
  return bytes;
}

// The FP64 companion batch of a mixed-precision batch, made at its first
// resistive solve: same capacity, on the batch's own stream and pool.
static int ensure_shadow(mhd_batch *b) {
  if (b->shadow) return MHD_OK;
  mhd_batch *sh = nullptr;
  int rc = mhd_batch_create(b->capacity, kFP64, &sh);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(sh->stream));  // idle: its own stream and pool are replaced
  cudaStreamDestroy(sh->stream);
  cudaMemPoolDestroy(sh->pool);
  sh->stream = b->stream;
  sh->pool = b->pool;
  sh->borrowed = true;
  sh->cg_host_loop = b->cg_host_loop;
  b->shadow = sh;
  return MHD_OK;
}

// Per-solve constants from the descriptor's (calc_physical_constant values
// and the boundary-operation values).
static Consts make_consts(const mhd_constants &k, int nghost) {
  Consts c = Consts{k.gamma,         k.M_H,       k.M_Na,        k.M_ref,
                    k.T_ref,         k.L_ref,     k.U_ref,       k.B_ref,
                    k.n_ref,         k.rho_ref,   k.m_Na,        k.k_Boltz,
                    k.q_e,           k.mu0,       k.state_coeff_H, k.state_coeff_Na,
                    k.CFL,           k.hall_coef, k.momentum_induce_coeff, k.momentum_hall_coeff,
                    k.inver_MA2,     k.ne_hall_floor, k.arti_eta_max, k.arti_J_start, k.arti_J_on,
                    k.ambipolar,     k.local_arti, nghost, k.resistive, {}};
  for (int q = 0; q < MHD_NUM_BC; ++q) c.bc[q] = k.bc[q];
  return c;
}

// The physical boundary operations of every group and the wall EMF, encoded
// as arena codes (MHD_PHYS_SET: one word; the others DevPhysOp).
// The largest k whose value an E_res / dB / dJ copy (halo, owner, or staged
// through a slot), an edge alias class or a singular-edge record carries to a
// lower k; -1 when none does (the radial index of a shell: every copy keeps
// k, the inner boundary's copies reach k < 0 from the first layers).  The
// implicit substep then computes only k below this bound + 2 and below its
// unknowns' top + 2: no value it needs comes from above.
static int res_kdown(const mhd_desc *desc) {
  int m = -1;
  auto flow = [&](int src_k, int dst_k) {
    if (src_k > dst_k) m = std::max(m, src_k);
  };
  for (int g : {(int)MHD_SYNC_ERES, (int)MHD_SYNC_DB, (int)MHD_SYNC_JEDGE}) {
    const mhd_sync_group &G = desc->groups[g];
    for (int t = 0; t < G.n_halo; ++t) flow(G.halo[t].src.k, G.halo[t].dst.k);
    for (int t = 0; t < G.n_owner; ++t) flow(G.owner[t].src.k, G.owner[t].dst.k);
    if (G.n_stash > 0 && G.stash) {
      std::unordered_map<int, int> slot_k;  // staging slot -> the k it was filled from
      for (int t = 0; t < G.n_stash; ++t) slot_k[G.stash[t].dst.i] = G.stash[t].src.k;
      for (int t = 0; t < G.n_stash; ++t) {
        const mhd_copy &c = G.stash[G.n_stash + t];
        auto it = slot_k.find(c.src.i);
        if (it == slot_k.end()) return INT_MAX;
        flow(it->second, c.dst.k);
      }
    }
  }
  const mhd_alias_classes &a = desc->edge_aliases;
  if (a.n_classes > 0 && a.offset && a.member && a.owner)
    for (int c = 0; c < a.n_classes; ++c) {
      int lo = a.owner[c].k, hi = lo;
      for (int q = a.offset[c]; q < a.offset[c + 1]; ++q) {
        lo = std::min(lo, a.member[q].k);
        hi = std::max(hi, a.member[q].k);
      }
      flow(hi, lo);
    }
  const mhd_singular_edges &g = desc->singular;
  if (g.n_edges > 0 && g.owner && g.alias_offset && g.aliases && g.cell_offset && g.cells && g.face_offset && g.faces)
    for (int e = 0; e < g.n_edges; ++e) {
      const int k = g.owner[e].k;
      for (int q = g.alias_offset[e]; q < g.alias_offset[e + 1]; ++q) flow(g.aliases[q].edge.k, k);
      for (int q = g.cell_offset[e]; q < g.cell_offset[e + 1]; ++q) flow(g.cells[q].cell.k, k);
      for (int q = g.face_offset[e]; q < g.face_offset[e + 1]; ++q) flow(g.faces[q].face.k, k);
    }
  return m;
}

// Whether every halo, staged and physical write of Sync(Eres) and of
// Sync(Jedge) lands on a ghost position (outside the owned range of its
// field).  The substep reads E_res only at owned positions (the curl of the
// owned faces) and dJ only at its unknowns (owned owner positions), so then
// those syncs change nothing it reads beyond the owner copies of E_res and
// the alias reduction of dJ.
static bool res_ghost_writes_only(const Solve *S, const mhd_desc *desc) {
  auto ghost = [&](const mhd_dof &d) {
    if (d.field < 0 || d.field >= MHD_NUM_FIELDS || d.block < 0 || d.block >= S->nblocks) return false;
    const int *st = kStagger[kFieldSpec[d.field].loc];
    const int *nb = S->boxes[d.block].n;
    const int x[3] = {d.i, d.j, d.k};
    for (int a = 0; a < 3; ++a)
      if (x[a] < 0 || x[a] >= nb[a] + st[a]) return true;
    return false;
  };
  for (int g : {(int)MHD_SYNC_ERES, (int)MHD_SYNC_JEDGE}) {
    const mhd_sync_group &G = desc->groups[g];
    for (int t = 0; t < G.n_halo; ++t)
      if (!ghost(G.halo[t].dst)) return false;
    for (int t = 0; t < G.n_stash; ++t)  // the staged copies' destinations (the second half)
      if (!ghost(G.stash[G.n_stash + t].dst)) return false;
    for (int t = 0; t < G.n_phys; ++t)
      if (!ghost(G.phys[t].dst)) return false;
  }
  return true;
}

static int upload_phys(Solve *S, const mhd_desc *desc, cudaStream_t st) {
  for (int q = 0; q < kNumPhys; ++q) {
    const mhd_phys_op *ops = q < kMaxGroups ? desc->groups[q].phys : desc->wall;
    int n = q < kMaxGroups ? desc->groups[q].n_phys : desc->n_wall;
    if (n < 0 || (n > 0 && !ops)) return fail(MHD_ERR_ARG, "physical operations %d: bad table", q);
    if ((q == MHD_SYNC_ERES || q == MHD_SYNC_DB) && !S->consts.resistive) n = 0;  // the implicit substep's groups
    std::vector<int64_t> set;
    std::vector<DevPhysOp> other;
    for (int t = 0; t < n; ++t) {
      const mhd_phys_op &o = ops[t];
      bool ok1 = false, ok2 = true;
      const int64_t dc = S->code(o.dst, &ok1);
      if (!ok1) return fail(MHD_ERR_ARG, "physical operation %d of table %d: destination out of range", t, q);
      if (o.kind == MHD_PHYS_SET) {
        if (o.arg < 0 || o.arg >= MHD_NUM_BC) return fail(MHD_ERR_ARG, "physical operation %d: value index %d", t, o.arg);
        set.push_back(dc | ((int64_t)o.arg << kPhysArgShift));
        continue;
      }
      DevPhysOp d{};
      d.kind = o.kind;
      d.dst = dc;
      const Box &bx = S->boxes[o.dst.block];
      d.cstride = bx.total * S->es;
      if (o.kind == MHD_PHYS_WALL) {
        if (o.dst.field != MHD_U_H || o.dst.comp != 0 || o.src.field != MHD_U_H || o.src.block != o.dst.block)
          return fail(MHD_ERR_ARG, "wall operation %d: cells of U_H of one block", t);
        d.src = S->code(o.src, &ok2);
        const int ax = std::abs(o.arg) - 1, sg = o.arg > 0 ? 1 : -1;
        if (ax < 0 || ax > 2 || S->nghost > kMaxWallGhosts) return fail(MHD_ERR_ARG, "wall operation %d: direction", t);
        d.nghost = S->nghost;
        for (int g = 1; g <= S->nghost; ++g) {
          mhd_dof c = o.dst;
          int *q3[3] = {&c.i, &c.j, &c.k};
          *q3[ax] += g * sg;
          for (int a = 0; a < 3; ++a)  // clamped to the allocated cell range
            *q3[a] = std::min(std::max(*q3[a], -S->nghost), bx.n[a] + S->nghost - 1);
          bool okg = false;
          d.ghost[g - 1] = S->code(c, &okg);
          ok2 = ok2 && okg;
        }
      } else if (o.kind == MHD_PHYS_EFAR) {
        if (o.dst.field < MHD_E_XI || o.dst.field > MHD_E_ZETA) return fail(MHD_ERR_ARG, "farfield EMF %d: not an E edge", t);
        mhd_dof dr = o.dst;
        dr.field = MHD_DR_XI + (o.dst.field - MHD_E_XI);
        dr.comp = 0;
        d.src = S->code(dr, &ok2);
      } else {
        return fail(MHD_ERR_ARG, "physical operation %d: kind %d", t, o.kind);
      }
      if (!ok2) return fail(MHD_ERR_ARG, "physical operation %d of table %d: source out of range", t, q);
      other.push_back(d);
    }
    if (q == MHD_SYNC_DB && S->consts.resistive) {
      // The reference clears dB before every Sync(dB) (clear_triplet,
      // Mercury_ImplicitResistive.cpp:428); the substep clears the ghost
      // faces once and then, per sync, zeroes here the ghost faces its copies
      // read (the others keep their zeros or are rewritten by the sync)
      std::unordered_set<int64_t> written;
      for (int t = 0; t < n; ++t) {
        bool ok = false;
        written.insert(S->code(ops[t].dst, &ok));
      }
      const mhd_sync_group &G = desc->groups[q];
      auto ghost = [&](const mhd_dof &d) {
        if (d.field < MHD_B_XI || d.field > MHD_B_ZETA || d.block < 0 || d.block >= S->nblocks) return false;
        const int ax = d.field - MHD_B_XI;
        const int *nb = S->boxes[d.block].n;
        const int x[3] = {d.i, d.j, d.k};
        for (int a = 0; a < 3; ++a)
          if (x[a] < 0 || x[a] >= nb[a] + (a == ax ? 1 : 0)) return true;
        return false;
      };
      auto zero_src = [&](const mhd_copy *tab, int m) {
        for (int t = 0; t < m; ++t) {
          if (!ghost(tab[t].src)) continue;
          bool ok = false;
          const int64_t c = S->code(tab[t].src, &ok);
          if (ok && written.insert(c).second) set.push_back(c | ((int64_t)MHD_BC_ZERO << kPhysArgShift));
        }
      };
      zero_src(G.halo, G.n_halo);
      zero_src(G.owner, G.n_owner);
      if (G.n_stash > 0 && G.stash) zero_src(G.stash, G.n_stash);
    }
    // the constant writes as segments: runs of up to 32 consecutive
    // destinations of one value, runs of equal length and value whose starts
    // step by one stride merged up to 32 elements (the ghost rows of a
    // farfield slab); two words each (start | value index, shape)
    std::sort(set.begin(), set.end(), [](int64_t a, int64_t b) {
      const int64_t m = ~(int64_t(31) << kPhysArgShift);
      return (a & m) < (b & m);
    });
    std::vector<int64_t> segs;
    {
      const int64_t amask = int64_t(31) << kPhysArgShift, es = S->es;
      struct Run { int64_t start; int64_t arg; int len; };
      std::vector<Run> runs;
      for (int64_t w : set) {
        const int64_t c = w & ~amask, a = w & amask;
        if (!runs.empty()) {
          Run &r = runs.back();
          if (r.arg == a && r.len < 32 && c == r.start + r.len * es) {
            ++r.len;
            continue;
          }
        }
        runs.push_back(Run{c, a, 1});
      }
      for (size_t t = 0; t < runs.size();) {
        const Run &r0 = runs[t];
        size_t u = t + 1;
        int64_t stride = 0;
        while (u < runs.size() && (int)(u - t + 1) * r0.len <= 32 && runs[u].arg == r0.arg && runs[u].len == r0.len) {
          const int64_t d = runs[u].start - runs[u - 1].start;
          if (u == t + 1) {
            if (d <= 0 || d >= (int64_t(1) << 46)) break;
            stride = d;
          } else if (d != stride) {
            break;
          }
          ++u;
        }
        segs.push_back(r0.start | r0.arg);
        segs.push_back((int64_t)(r0.len - 1) | ((int64_t)(u - t - 1) << 8) | (stride << 16));
        t = u;
      }
    }
    set.swap(segs);
    S->T->ph_nset[q] = (int)set.size() / 2;
    S->T->ph_nop[q] = (int)other.size();
    S->T->table_bytes += (int64_t)set.size() * 8 + (int64_t)other.size() * sizeof(DevPhysOp);
    int rc;
    if ((rc = dev_upload(S->pool, set, &S->T->ph_set[q], st)) || (rc = dev_upload(S->pool, other, &S->T->ph_op[q], st)))
      return rc;
  }
  return MHD_OK;
}

// Per-solve geometric data of the singular edges (written by k_sing_setup).
static int alloc_singular_geo(Solve *S, cudaStream_t st) {
  if (S->T->sg_n <= 0) return MHD_OK;
  CUDA_TRY(cudaMallocFromPoolAsync((void **)&S->sg_geo, sizeof(double) * 4 * S->T->sg_n, S->pool, st));
  CUDA_TRY(cudaMallocFromPoolAsync((void **)&S->sg_w, sizeof(double) * std::max(1, S->T->sg_ncell), S->pool, st));
  CUDA_TRY(cudaMemsetAsync(S->sg_geo, 0, sizeof(double) * 4 * S->T->sg_n, st));
  CUDA_TRY(cudaMemsetAsync(S->sg_w, 0, sizeof(double) * std::max(1, S->T->sg_ncell), st));
  return MHD_OK;
}

// The singular-edge lists as device records (mhd_singular_edges).
static int upload_singular(Solve *S, const mhd_singular_edges &g, cudaStream_t st) {
  if (g.n_edges <= 0) return MHD_OK;
  if (!g.owner || !g.owner_sign || !g.alias_offset || !g.aliases || !g.cell_offset || !g.cells || !g.face_offset ||
      !g.faces)
    return fail(MHD_ERR_ARG, "singular edges: null table");
  const int n = g.n_edges;
  std::vector<int64_t> owner(3 * n);
  std::vector<double> osign(g.owner_sign, g.owner_sign + n);
  auto inside = [&](int field, int block, int i, int j, int k) {
    const mhd_dof d{field, block, i, j, k, 0};
    bool ok = false;
    S->code(d, &ok);
    return ok;
  };
  for (int e = 0; e < n; ++e) {
    const mhd_dof &o = g.owner[e];
    if (o.field < 0 || o.field > 2) return fail(MHD_ERR_ARG, "singular edge %d: owner axis %d", e, o.field);
    const int fl[3] = {MHD_E_XI + o.field, MHD_EHALL_XI + o.field, MHD_J_XI + o.field};
    for (int q = 0; q < 3; ++q) {
      mhd_dof d = o;
      d.field = fl[q];
      d.comp = 0;
      bool ok = false;
      owner[3 * e + q] = S->code(d, &ok);
      if (!ok) return fail(MHD_ERR_ARG, "singular edge %d: owner out of range", e);
    }
  }
  auto records = [&](const int32_t *off, auto get, int per, std::vector<int> &offs, std::vector<int> &rec,
                     const char *what) -> int {
    offs.assign(off, off + n + 1);
    for (int q = off[0]; q < off[n]; ++q) {
      int r[6];
      get(q, r);
      const int fld = per == 0 ? MHD_CELL : per;
      (void)fld;
      rec.insert(rec.end(), r, r + 6);
    }
    return MHD_OK;
    (void)what;
  };
  std::vector<int> aoff, alias, coff, cell, foff, face;
  records(g.alias_offset, [&](int q, int *r) {
    const mhd_singular_alias &a = g.aliases[q];
    r[0] = a.edge.block; r[1] = a.edge.field; r[2] = a.edge.i; r[3] = a.edge.j; r[4] = a.edge.k; r[5] = a.orient;
  }, 1, aoff, alias, "alias");
  records(g.cell_offset, [&](int q, int *r) {
    const mhd_singular_cell &c = g.cells[q];
    r[0] = c.cell.block; r[1] = c.axis; r[2] = c.cell.i; r[3] = c.cell.j; r[4] = c.cell.k; r[5] = c.orient;
  }, 0, coff, cell, "cell");
  records(g.face_offset, [&](int q, int *r) {
    const mhd_singular_face &f = g.faces[q];
    r[0] = f.face.block; r[1] = f.face.field; r[2] = f.face.i; r[3] = f.face.j; r[4] = f.face.k; r[5] = f.sign;
  }, 2, foff, face, "face");
  // every record inside its block's box (the kernels read +-1 cell around incident cells)
  for (size_t q = 0; q < alias.size(); q += 6)
    if (alias[q + 1] < 0 || alias[q + 1] > 2 || !inside(MHD_E_XI + alias[q + 1], alias[q], alias[q + 2], alias[q + 3], alias[q + 4]))
      return fail(MHD_ERR_ARG, "singular edges: alias %zu out of range", q / 6);
  for (size_t q = 0; q < cell.size(); q += 6) {
    if (cell[q + 1] < 0 || cell[q + 1] > 2 || cell[q] < 0 || cell[q] >= S->nblocks)
      return fail(MHD_ERR_ARG, "singular edges: cell %zu out of range", q / 6);
    const Box &bx = S->boxes[cell[q]];
    for (int a = 0; a < 3; ++a)
      if (cell[q + 2 + a] < 1 - bx.G || cell[q + 2 + a] >= bx.n[a] + bx.G)
        return fail(MHD_ERR_ARG, "singular edges: cell %zu out of range", q / 6);
  }
  for (size_t q = 0; q < face.size(); q += 6)
    if (face[q + 1] < 0 || face[q + 1] > 2 || !inside(MHD_B_XI + face[q + 1], face[q], face[q + 2], face[q + 3], face[q + 4]))
      return fail(MHD_ERR_ARG, "singular edges: face %zu out of range", q / 6);
  Tables &T = *S->T;
  T.sg_n = n;
  T.sg_ncell = (int)(cell.size() / 6);
  T.table_bytes += (int64_t)(owner.size() + osign.size()) * 8 + (int64_t)(alias.size() + cell.size() + face.size()) * 4;
  int rc;
  if ((rc = dev_upload(S->pool, owner, &T.sg_owner, st)) || (rc = dev_upload(S->pool, osign, &T.sg_osign, st)) ||
      (rc = dev_upload(S->pool, aoff, &T.sg_aoff, st)) || (rc = dev_upload(S->pool, alias, &T.sg_alias, st)) ||
      (rc = dev_upload(S->pool, coff, &T.sg_coff, st)) || (rc = dev_upload(S->pool, cell, &T.sg_cell, st)) ||
      (rc = dev_upload(S->pool, foff, &T.sg_foff, st)) || (rc = dev_upload(S->pool, face, &T.sg_face, st)))
    return rc;
  return MHD_OK;
}

static int add_solve(mhd_batch *b, const mhd_desc *desc, bool periodic, int *slot_out) {
  if (!b || !desc || !slot_out || desc->n_blocks < 1 || !desc->cells) return fail(MHD_ERR_ARG, "mhd_batch_add: bad descriptor");
  if (periodic && desc->n_blocks != 1) return fail(MHD_ERR_ARG, "mhd_batch_add_periodic: one block");
  if (desc->nghost < 2) return fail(MHD_ERR_ARG, "mhd_batch_add: nghost %d (the step's stencils need >= 2)", desc->nghost);
  if (desc->precision != b->precision)
    return fail(MHD_ERR_ARG, "solve precision %d differs from the batch's (%d)", desc->precision, b->precision);
  if (desc->n_blocks >= (1 << 15)) return fail(MHD_ERR_ARG, "too many blocks (%d)", desc->n_blocks);
  int slot = -1;
  for (int s = 0; s < b->capacity; ++s)
    if (!b->slots[s]) {
      slot = s;
      break;
    }
  if (slot < 0) return fail(MHD_ERR_OOM, "mhd_batch_add: all %d slots in use", b->capacity);
  auto *S = new (std::nothrow) Solve();
  if (!S) return fail(MHD_ERR_OOM, "host allocation");
  S->pool = b->pool;
  S->T = new (std::nothrow) Tables();
  if (!S->T) {
    delete S;
    return fail(MHD_ERR_OOM, "host allocation");
  }
  S->T->users = 1;
  cudaStream_t st = b->stream;
  auto bail = [&](int rc) {
    free_solve(S, st);
    return rc;
  };
  S->nblocks = desc->n_blocks;
  S->nghost = desc->nghost;
  S->es = b->precision == kMixed ? 4 : 8;
  int64_t u = 0, m = 0;
  std::vector<int> prefix[kNumRanges];
  for (int r = 0; r < kNumRanges; ++r) prefix[r].push_back(0);
  for (int bi = 0; bi < S->nblocks; ++bi) {
    const int n[3] = {desc->cells[3 * bi], desc->cells[3 * bi + 1], desc->cells[3 * bi + 2]};
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) return bail(fail(MHD_ERR_ARG, "block %d: cells %d %d %d", bi, n[0], n[1], n[2]));
    Box bx = make_box(n, desc->nghost);
    // kernels address a block's arrays with 32-bit element offsets
    if ((int64_t)(kNumComps + kNumUComps) * bx.total >= (int64_t(1) << 31))
      return bail(fail(MHD_ERR_ARG, "block %d too large (%lld cells with ghosts); split it into smaller blocks", bi,
                       (long long)bx.total));
    // the substep marks its unknowns by element offsets held in the real type
    if (desc->constants.resistive && S->es == 4 && bx.total > (int64_t(1) << 24))
      return bail(fail(MHD_ERR_ARG, "block %d: %lld cells with ghosts exceed 2^24 (mixed-precision implicit substep)",
                       bi, (long long)bx.total));
    S->boxes.push_back(bx);
    S->ubase.push_back(u);
    S->mbase.push_back(m);
    u += (int64_t)kNumUComps * bx.total * S->es;
    m += ((int64_t)kNumMetric * 8 + (int64_t)(kNumRComps - (desc->constants.resistive ? 0 : kNumResComps)) * S->es) *
         bx.total;
    for (int r = 0; r < kNumRanges; ++r)
      prefix[r].push_back(prefix[r].back() + tiles_of(range_of(r, n, desc->nghost), r));
  }
  S->ubuf = u;
  S->main_off = 2 * u;
  if (desc->n_staging < 0) return bail(fail(MHD_ERR_ARG, "n_staging %d", desc->n_staging));
  S->n_staging = periodic ? 0 : desc->n_staging;
  S->staging_off = 2 * u + m;
  S->arena_bytes = 2 * u + m + ((int64_t)S->n_staging * S->es + 255) / 256 * 256;
  const mhd_constants &k = desc->constants;
  S->consts = make_consts(k, desc->nghost);
  if (cudaMallocFromPoolAsync((void **)&S->arena, S->arena_bytes, b->pool, st) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MHD_ERR_OOM, "arena of %lld bytes", (long long)S->arena_bytes));
  }
  if (cudaMemsetAsync(S->arena, 0, S->arena_bytes, st) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "arena memset"));
  std::vector<DevBlock> blocks(S->nblocks);
  for (int bi = 0; bi < S->nblocks; ++bi) {
    const Box &bx = S->boxes[bi];
    DevBlock &d = blocks[bi];
    d.U[0] = S->arena + S->ubase[bi];
    d.U[1] = S->arena + S->ubuf + S->ubase[bi];
    d.M = S->arena + S->main_off + S->mbase[bi];
    d.total = bx.total;
    d.si = bx.si;
    d.sj = bx.sj;
    d.G = bx.G;
    for (int a = 0; a < 3; ++a) d.n[a] = bx.n[a];
    d.solve = slot;
    d.reskhi = bx.n[2] + 1;
  }
  int rc;
  if ((rc = upload_tmaps(S, blocks, st))) return bail(rc);
  if ((rc = dev_upload(S->pool, blocks, &S->dblocks, st))) return bail(rc);
  for (int r = 0; r < kNumRanges; ++r) {
    S->T->tiles[r] = prefix[r].back();
    if ((rc = dev_upload(S->pool, prefix[r], &S->T->dtile_prefix[r], st))) return bail(rc);
  }
  try {
    if (periodic) {
      if ((rc = upload_groups_periodic(S, st)) || (rc = upload_aliases_periodic(S, st))) return bail(rc);
    } else {
      if ((rc = upload_groups(S, desc->groups, st))) return bail(rc);
      if ((rc = upload_aliases(S, desc->edge_aliases, st))) return bail(rc);
      if ((rc = upload_phys(S, desc, st))) return bail(rc);
      if ((rc = upload_singular(S, desc->singular, st)) || (rc = alloc_singular_geo(S, st))) return bail(rc);
      if (S->consts.resistive) {
        S->T->res_kdown = res_kdown(desc);
        S->T->res_ghost_writes_only = res_ghost_writes_only(S, desc);
      }
    }
  } catch (...) {  // host allocation or thread creation failed
    return bail(fail(MHD_ERR_OOM, "host memory for the copy tables"));
  }
  SolveState s0{};
  s0.dt_bits = kDtUnset;
  if ((rc = set_state_field(b, slot, 0, &s0, sizeof s0))) return bail(rc);
  S->res_rtol = k.res_rtol;
  S->res_max_it = k.res_max_it;
  S->res_direct = direct_iters(k);
  b->slots[slot] = S;
  if (S->consts.resistive) ++b->n_res;
  const bool grew = count_tables(b, S, +1);
  if ((rc = publish(b))) return rc;
  // asynchronous: the host data went to the device through pageable copies,
  // staged before they returned; a step graph to capture anew waits for the
  // graphs in flight first
  if (grew) {
    CUDA_TRY(cudaStreamSynchronize(st));
    drop_graphs(b);
  }
  if (b->precision == kMixed && S->consts.resistive) {
    mhd_desc d64 = *desc;
    d64.precision = kFP64;
    int cs = -1;
    if ((rc = ensure_shadow(b)) || (rc = add_solve(b->shadow, &d64, periodic, &cs))) {
      mhd_batch_remove(b, slot);
      return rc;
    }
    S->shadow_slot = cs;
    if ((rc = publish(b))) return rc;  // the directory entry's companion
  }
  *slot_out = slot;
  return MHD_OK;
}

int mhd_batch_add(mhd_batch *b, const mhd_desc *desc, int *slot_out) { return add_solve(b, desc, false, slot_out); }

int mhd_batch_add_periodic(mhd_batch *b, const int32_t cells[3], int32_t nghost, const mhd_constants *constants,
                           int *slot_out) {
  if (!b || !cells || !constants) return fail(MHD_ERR_ARG, "mhd_batch_add_periodic: bad arguments");
  mhd_desc d{};
  d.n_blocks = 1;
  d.cells = cells;
  d.nghost = nghost;
  d.precision = b->precision;
  d.constants = *constants;
  return add_solve(b, &d, true, slot_out);
}

int mhd_batch_add_like(mhd_batch *b, int src_slot, const mhd_constants *constants, int copy_static, int *slot_out) {
  int rc = slot_check(b, src_slot);
  if (rc) return rc;
  if (!slot_out) return fail(MHD_ERR_ARG, "mhd_batch_add_like: null slot");
  if (constants && (constants->resistive != 0) != (b->slots[src_slot]->consts.resistive != 0))
    return fail(MHD_ERR_ARG, "mhd_batch_add_like: the implicit resistive substep must match the template's");
  int slot = -1;
  for (int s = 0; s < b->capacity; ++s)
    if (!b->slots[s]) {
      slot = s;
      break;
    }
  if (slot < 0) return fail(MHD_ERR_OOM, "mhd_batch_add_like: all %d slots in use", b->capacity);
  const Solve *src = b->slots[src_slot];
  auto *S = new (std::nothrow) Solve();
  if (!S) return fail(MHD_ERR_OOM, "host allocation");
  S->pool = b->pool;
  cudaStream_t st = b->stream;
  S->nblocks = src->nblocks;
  S->nghost = src->nghost;
  S->es = src->es;
  S->boxes = src->boxes;
  S->ubase = src->ubase;
  S->mbase = src->mbase;
  S->ubuf = src->ubuf;
  S->main_off = src->main_off;
  S->arena_bytes = src->arena_bytes;
  S->staging_off = src->staging_off;
  S->n_staging = src->n_staging;
  S->T = src->T;
  S->T->users += 1;
  S->consts = src->consts;
  if (constants) S->consts = make_consts(*constants, S->nghost);
  auto bail = [&](int code) {
    free_solve(S, st);
    return code;
  };
  if ((rc = alloc_singular_geo(S, st))) return bail(rc);
  if (cudaMallocFromPoolAsync((void **)&S->arena, S->arena_bytes, b->pool, st) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MHD_ERR_OOM, "arena of %lld bytes", (long long)S->arena_bytes));
  }
  // the template's fields (static geometry and sources, and its current
  // state, which the caller normally overwrites) or zeros
  const cudaError_t e = copy_static ? cudaMemcpyAsync(S->arena, src->arena, S->arena_bytes, cudaMemcpyDeviceToDevice, st)
                                    : cudaMemsetAsync(S->arena, 0, S->arena_bytes, st);
  if (e != cudaSuccess) return bail(fail(MHD_ERR_CUDA, "arena init: %s", cudaGetErrorString(e)));
  std::vector<DevBlock> blocks(S->nblocks);
  for (int bi = 0; bi < S->nblocks; ++bi) {
    const Box &bx = S->boxes[bi];
    DevBlock &d = blocks[bi];
    d.U[0] = S->arena + S->ubase[bi];
    d.U[1] = S->arena + S->ubuf + S->ubase[bi];
    d.M = S->arena + S->main_off + S->mbase[bi];
    d.total = bx.total;
    d.si = bx.si;
    d.sj = bx.sj;
    d.G = bx.G;
    for (int a = 0; a < 3; ++a) d.n[a] = bx.n[a];
    d.solve = slot;
    d.reskhi = bx.n[2] + 1;
  }
  if ((rc = upload_tmaps(S, blocks, st))) return bail(rc);
  if ((rc = dev_upload(S->pool, blocks, &S->dblocks, st))) return bail(rc);
  SolveState s0{};
  s0.dt_bits = kDtUnset;
  if ((rc = set_state_field(b, slot, 0, &s0, sizeof s0))) return bail(rc);
  S->res_rtol = constants ? constants->res_rtol : src->res_rtol;
  S->res_max_it = constants ? constants->res_max_it : src->res_max_it;
  S->res_direct = constants ? direct_iters(*constants) : src->res_direct;
  b->slots[slot] = S;
  if (S->consts.resistive) ++b->n_res;
  if (count_tables(b, S, +1)) {  // not reached while the template itself is in the batch
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
  }
  if ((rc = publish(b))) return rc;
  if (src->shadow_slot >= 0) {
    int cs = -1;
    if ((rc = mhd_batch_add_like(b->shadow, src->shadow_slot, nullptr, 0, &cs))) {
      mhd_batch_remove(b, slot);
      return rc;
    }
    S->shadow_slot = cs;
    if ((rc = publish(b))) return rc;  // the directory entry's companion
  }
  *slot_out = slot;  // asynchronous: stream-ordered with the batch's other work
  return MHD_OK;
}

int mhd_fluid_tile_shape(int variant, int32_t shape[4]) {
  if (variant < 0 || variant >= kNumFluidTiles || !shape) return fail(MHD_ERR_ARG, "fluid tile variant %d", variant);
  const FluidTile T = fluid_tile(variant);
  shape[0] = T.k;
  shape[1] = T.j;
  shape[2] = T.i;
  shape[3] = T.min_ctas;
  return MHD_OK;
}

int mhd_batch_fluid_tile(mhd_batch *b, int variant) {
  if (!b || variant < 0 || variant >= kNumFluidTiles) return fail(MHD_ERR_ARG, "mhd_batch_fluid_tile: bad arguments");
  if (variant == b->fluid_tile) return MHD_OK;
  CUDA_TRY(cudaStreamSynchronize(b->stream));  // no step graph in flight
  b->fluid_tile = variant;
  drop_graphs(b);
  return MHD_OK;
}

int mhd_batch_time_fluid_tiles(mhd_batch *b, int reps, float ms[MHD_NUM_FLUID_TILES]) {
  if (!b || reps < 1 || !ms) return fail(MHD_ERR_ARG, "mhd_batch_time_fluid_tiles: bad arguments");
  int rc = read_state(b);
  if (rc) return rc;
  bool any = false;
  for (int s = 0; s < b->capacity; ++s)
    any = any || (b->slots[s] && b->hstate[s].remaining != 0 && b->hstate[s].status == 0);
  if (!any) return fail(MHD_ERR_STATE, "mhd_batch_time_fluid_tiles: no solve has steps requested");
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int nk = 0;
  for (int v = 0; v < kNumFluidTiles; ++v) {
    // the fluid pass alone writes only the next state buffer, which the next
    // step rewrites with the same values: the solves are unchanged
    launch(b, 0, SK_FLUID, &nk, nullptr, v);  // untimed
    cudaEventRecord(e0, b->stream);
    for (int r = 0; r < reps; ++r) launch(b, 0, SK_FLUID, &nk, nullptr, v);
    cudaEventRecord(e1, b->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(MHD_ERR_CUDA, "mhd_batch_time_fluid_tiles: %s", cudaGetErrorString(cudaGetLastError()));
    }
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    ms[v] = t / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CUDA_TRY(cudaGetLastError());
  return MHD_OK;
}

int mhd_batch_set_constants(mhd_batch *b, int slot, const mhd_constants *constants) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  if (!constants) return fail(MHD_ERR_ARG, "mhd_batch_set_constants: null constants");
  Solve *S = b->slots[slot];
  if ((constants->resistive != 0) != (S->consts.resistive != 0))
    return fail(MHD_ERR_ARG, "mhd_batch_set_constants: the implicit resistive substep cannot be switched");
  S->consts = make_consts(*constants, S->nghost);
  S->res_rtol = constants->res_rtol;
  S->res_max_it = constants->res_max_it;
  S->res_direct = direct_iters(*constants);
  S->prepared = false;
  if ((rc = publish(b))) return rc;
  if (S->shadow_slot >= 0 && b->shadow) return mhd_batch_set_constants(b->shadow, S->shadow_slot, constants);
  return MHD_OK;
}

int mhd_batch_remove(mhd_batch *b, int slot) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  Solve *S = b->slots[slot];
  if (S->shadow_slot >= 0 && (rc = mhd_batch_remove(b->shadow, S->shadow_slot))) return rc;
  b->slots[slot] = nullptr;
  if (S->consts.resistive) --b->n_res;
  count_tables(b, S, -1);
  SolveState s0{};
  if ((rc = set_state_field(b, slot, 0, &s0, sizeof s0))) return rc;
  if ((rc = publish(b))) return rc;
  free_solve(S, b->stream);
  return MHD_OK;
}

int mhd_batch_upload_field(mhd_batch *b, int slot, int field, int block, const double *data, const int32_t lo[3],
                           const int32_t hi[3], int ncomp) {
  Solve *S = nullptr;
  int rc = xfer(b, slot, field, block, lo, hi, ncomp, &S);
  if (rc) return rc;
  if (!data) return fail(MHD_ERR_ARG, "upload: null data");
  const int e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  if ((rc = ensure_staging(b, npts * ncomp))) return rc;
  CUDA_TRY(cudaMemcpyAsync(b->staging, data, sizeof(double) * npts * ncomp, cudaMemcpyHostToDevice, b->stream));
  // U components go to both buffers: ghost corners the step never writes must
  // be identical in both.
  const int c0 = kComp.first[field];
  const int ndst = c0 < kNumUComps ? 2 : 1;
  void *ptrs[72];
  for (int d = 0; d < ndst; ++d)
    for (int m = 0; m < ncomp; ++m) ptrs[d * ncomp + m] = S->comp_ptr(block, c0 + m, d);
  CUDA_TRY(cudaMemcpyAsync(b->comp_ptrs, ptrs, sizeof(void *) * ndst * ncomp, cudaMemcpyHostToDevice, b->stream));
  const Box &bx = S->boxes[block];
  k_scatter_aos<<<(unsigned)((npts + 255) / 256), 256, 0, b->stream>>>(b->staging, lo[0], lo[1], lo[2], e[0], e[1], e[2],
                                                                       ncomp, b->comp_ptrs, ndst, bx.si, bx.sj, bx.G,
                                                                       S->comp_bytes(c0) == 4);
  CUDA_TRY(cudaGetLastError());
  // A copy from pageable memory is staged by CUDA before
  // cudaMemcpyAsync returns; page-locked memory is read by the DMA later, so
  // wait for it before the caller may reuse the buffer.
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, data) != cudaSuccess) {
    cudaGetLastError();
    pa.type = cudaMemoryTypeHost;
  }
  if (pa.type != cudaMemoryTypeUnregistered) CUDA_TRY(cudaStreamSynchronize(b->stream));
  S->prepared = false;
  return MHD_OK;
}

int mhd_batch_fill_field(mhd_batch *b, int slot, int field, int block, const double *values, const int32_t lo[3],
                         const int32_t hi[3], int ncomp) {
  Solve *S = nullptr;
  int rc = xfer(b, slot, field, block, lo, hi, ncomp, &S);
  if (rc) return rc;
  if (!values || ncomp > 36) return fail(MHD_ERR_ARG, "fill: bad values");
  FillValues val{};
  for (int m = 0; m < ncomp; ++m) val.v[m] = values[m];
  const int e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  const int c0 = kComp.first[field];
  const int ndst = c0 < kNumUComps ? 2 : 1;  // U: both buffers, as an upload
  void *ptrs[72];
  for (int d = 0; d < ndst; ++d)
    for (int m = 0; m < ncomp; ++m) ptrs[d * ncomp + m] = S->comp_ptr(block, c0 + m, d);
  CUDA_TRY(cudaMemcpyAsync(b->comp_ptrs, ptrs, sizeof(void *) * ndst * ncomp, cudaMemcpyHostToDevice, b->stream));
  const Box &bx = S->boxes[block];
  k_fill<<<(unsigned)((npts + 255) / 256), 256, 0, b->stream>>>(val, lo[0], lo[1], lo[2], e[0], e[1], e[2], ncomp,
                                                                b->comp_ptrs, ndst, bx.si, bx.sj, bx.G,
                                                                S->comp_bytes(c0) == 4);
  CUDA_TRY(cudaGetLastError());
  // the pointer table is pageable: staged before the copy returned
  S->prepared = false;
  return MHD_OK;
}

int mhd_batch_download_field(mhd_batch *b, int slot, int field, int block, double *data, const int32_t lo[3],
                             const int32_t hi[3], int ncomp) {
  Solve *S = nullptr;
  int rc = xfer(b, slot, field, block, lo, hi, ncomp, &S);
  if (rc) return rc;
  if (!data) return fail(MHD_ERR_ARG, "download: null data");
  if ((rc = read_state(b))) return rc;
  const int cur = b->hstate[slot].cur;
  const int e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  if ((rc = ensure_staging(b, npts * ncomp))) return rc;
  const int c0 = kComp.first[field];
  void *ptrs[36];
  for (int m = 0; m < ncomp; ++m) ptrs[m] = S->comp_ptr(block, c0 + m, cur);
  CUDA_TRY(cudaMemcpyAsync(b->comp_ptrs, ptrs, sizeof(void *) * ncomp, cudaMemcpyHostToDevice, b->stream));
  const Box &bx = S->boxes[block];
  k_gather_aos<<<(unsigned)((npts + 255) / 256), 256, 0, b->stream>>>(b->staging, lo[0], lo[1], lo[2], e[0], e[1], e[2],
                                                                      ncomp, b->comp_ptrs, bx.si, bx.sj, bx.G,
                                                                      S->comp_bytes(c0) == 4);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(data, b->staging, sizeof(double) * npts * ncomp, cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MHD_OK;
}

int mhd_batch_sync(mhd_batch *b, int slot, int group) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  if (group < 0 || group >= MHD_NUM_GROUPS) return fail(MHD_ERR_ARG, "mhd_sync: bad group %d", group);
  return targeted(b, slot, [&](int *nk) { enqueue_sync(b, 1, group, nk, true); });  // asynchronous
}

// The implicit substep's work range of one solve (kResK), after its
// unknowns are marked: per block k < min(n_k + 1, R), R = 2 + the larger of
// the unknowns' top k (over the blocks) and the tables' k bound (res_kdown).
// Every value the substep computes for its unknowns then lies in the range,
// bit for bit as over the whole box; above it E_res stays 0 and B does not
// change.  The FP64 companion of a mixed solve takes the same range.  One
// host round trip (the unknowns are known on the device only).
static int apply_res_range(mhd_batch *b, Solve *S, const std::vector<int> &hi) {
  bool whole = true;
  for (int bi = 0; bi < S->nblocks; ++bi) whole = whole && hi[bi] == S->boxes[bi].n[2] + 1;
  cudaStream_t st = b->stream;
  if (S->dres_prefix) {
    CUDA_TRY(cudaFreeAsync(S->dres_prefix, st));
    S->dres_prefix = nullptr;
  }
  S->res_tiles = 0;
  std::vector<int> prefix(1, 0);
  for (int bi = 0; bi < S->nblocks; ++bi) {
    CUDA_TRY(cudaMemcpyAsync(&S->dblocks[bi].reskhi, &hi[bi], sizeof(int), cudaMemcpyHostToDevice, st));
    RangeBox r = range_of(kResK, S->boxes[bi].n, S->nghost);
    r.hi[2] = hi[bi];
    prefix.push_back(prefix.back() + tiles_of(r, kResK));
  }
  if (!whole) {
    int rc = dev_upload(S->pool, prefix, &S->dres_prefix, st);
    if (rc) return rc;
    S->res_tiles = prefix.back();
  }
  CUDA_TRY(cudaStreamSynchronize(st));  // the host values above are staged
  return publish(b);
}

static int res_range(mhd_batch *b, int slot) {
  Solve *S = b->slots[slot];
  int *dk = nullptr;
  CUDA_TRY(cudaMallocFromPoolAsync((void **)&dk, sizeof(int) * S->nblocks, b->pool, b->stream));
  CUDA_TRY(cudaMemsetAsync(dk, 0xff, sizeof(int) * S->nblocks, b->stream));  // -1
  const int one = 1, zero = 0;
  int rc = set_state_field(b, slot, offsetof(SolveState, mask), &one, sizeof one);
  if (rc) return rc;
  launch_res_kmax(b->dir(1), b->precision, dk, b->stream);
  CUDA_TRY(cudaGetLastError());
  if ((rc = set_state_field(b, slot, offsetof(SolveState, mask), &zero, sizeof zero))) return rc;
  std::vector<int> kmax(S->nblocks, -1);
  CUDA_TRY(cudaMemcpyAsync(kmax.data(), dk, sizeof(int) * S->nblocks, cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaFreeAsync(dk, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  int top = -1;
  for (int k : kmax) top = std::max(top, k);
  const int kd = S->T->res_kdown;
  const int64_t R = kd == INT_MAX ? INT64_MAX : (int64_t)std::max(top, kd) + 2;
  std::vector<int> hi(S->nblocks);
  for (int bi = 0; bi < S->nblocks; ++bi) hi[bi] = (int)std::min<int64_t>(S->boxes[bi].n[2] + 1, R);
  if ((rc = apply_res_range(b, S, hi))) return rc;
  if (S->shadow_slot >= 0 && b->shadow) return apply_res_range(b->shadow, b->shadow->slots[S->shadow_slot], hi);
  return MHD_OK;
}

int mhd_batch_prepare(mhd_batch *b, int slot, double time, int64_t step) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  SolveState s0{};
  s0.dt_bits = kDtUnset;
  s0.time = time;
  s0.step = step;
  // reset everything before the buffer index (dt, time, step, remaining, status); keep cur
  if ((rc = set_state_field(b, slot, 0, &s0, offsetof(SolveState, cur)))) return rc;
  const bool res = b->slots[slot]->consts.resistive != 0;
  const bool sing = b->slots[slot]->T->sg_n > 0;
  rc = targeted(b, slot, [&](int *nk) {
    if (sing) launch(b, 1, SK_SING_SETUP, nk);  // before anything reads the edge Hodge field it updates
    launch(b, 1, SK_FACE_NORMALS, nk);
    if (res) {  // unknowns of the implicit resistive substep: W = 1 / (eta alpha) on them
      launch(b, 1, SK_RES_SEED, nk);
      sync1(b, 1, copy_op(MHD_SYNC_ERES, kPhOwner, 0, 1), nk);  // zero the non-owner aliases
      launch(b, 1, SK_RES_W, nk);
    }
    enqueue_derived(b, 1, nk);
  });
  if (rc) return rc;
  if (res && (rc = res_range(b, slot))) return rc;
  const Solve *S = b->slots[slot];
  if (res && S->shadow_slot >= 0) {
    if (S->T->sg_n > 0)  // the singular edges' geometry, FP64 in both
      CUDA_TRY(cudaMemcpyAsync(b->shadow->slots[S->shadow_slot]->sg_geo, S->sg_geo, sizeof(double) * 4 * S->T->sg_n,
                               cudaMemcpyDeviceToDevice, b->stream));
    // the operator's coefficients (alpha, beta, eta, W), widened into the companion once
    if ((rc = targeted(b, slot, [&](int *) { launch_res_cross(b->dir(1), RES_X_STATIC, b->stream); }))) return rc;
  }
  b->slots[slot]->prepared = true;  // asynchronous: stream-ordered with the batch's other work
  return MHD_OK;
}

int mhd_batch_save_restart(mhd_batch *b, int slot, const char *path) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  if (!path) return fail(MHD_ERR_ARG, "mhd_batch_save_restart: null path");
  const Solve *S = b->slots[slot];
  // every ghost layer of the state fields, as the reference's checkpoint holds them
  if ((rc = mhd_batch_sync(b, slot, MHD_SYNC_UCELL)) || (rc = mhd_batch_sync(b, slot, MHD_SYNC_BFACE))) return rc;
  if ((rc = read_state(b))) return rc;
  std::vector<int32_t> cells;
  for (const Box &bx : S->boxes)
    for (int a = 0; a < 3; ++a) cells.push_back(bx.n[a]);
  mhd_restart_image img{};
  img.step = (int32_t)b->hstate[slot].step;
  img.time = b->hstate[slot].time;
  img.n_blocks = S->nblocks;
  img.cells = cells.data();
  img.nghost = S->nghost;
  const int fields[MHD_RESTART_FIELDS] = {MHD_U_H, MHD_U_NA, MHD_B_XI, MHD_B_ETA, MHD_B_ZETA};
  std::vector<double> buf[MHD_RESTART_FIELDS];
  for (int f = 0; f < MHD_RESTART_FIELDS; ++f) {
    buf[f].resize((size_t)mhd_restart_values(&img, f));
    img.data[f] = buf[f].data();
    double *d = buf[f].data();
    const int *st = kStagger[kFieldSpec[fields[f]].loc];
    const int nc = kFieldSpec[fields[f]].ncomp;
    for (int blk = 0; blk < S->nblocks; ++blk) {
      int32_t lo[3], hi[3];
      int64_t n = nc;
      for (int a = 0; a < 3; ++a) {
        lo[a] = -S->nghost;
        hi[a] = S->boxes[blk].n[a] + st[a] + S->nghost;
        n *= hi[a] - lo[a];
      }
      if ((rc = mhd_batch_download_field(b, slot, fields[f], blk, d, lo, hi, nc))) return rc;
      d += n;
    }
  }
  return mhd_restart_write(path, &img);
}

int mhd_batch_load_restart(mhd_batch *b, int slot, const char *path, int32_t *step, double *time) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  if (!path) return fail(MHD_ERR_ARG, "mhd_batch_load_restart: null path");
  const Solve *S = b->slots[slot];
  std::vector<int32_t> cells;
  for (const Box &bx : S->boxes)
    for (int a = 0; a < 3; ++a) cells.push_back(bx.n[a]);
  mhd_restart_image img{};
  img.n_blocks = S->nblocks;
  img.cells = cells.data();
  img.nghost = S->nghost;
  std::vector<double> buf[MHD_RESTART_FIELDS];
  for (int f = 0; f < MHD_RESTART_FIELDS; ++f) {
    buf[f].resize((size_t)mhd_restart_values(&img, f));
    img.data[f] = buf[f].data();
  }
  if ((rc = mhd_restart_read(path, &img))) return rc;
  const int fields[MHD_RESTART_FIELDS] = {MHD_U_H, MHD_U_NA, MHD_B_XI, MHD_B_ETA, MHD_B_ZETA};
  for (int f = 0; f < MHD_RESTART_FIELDS; ++f) {
    if (!(img.loaded & (1u << f))) continue;  // not in the file: the solve keeps its values
    const double *d = buf[f].data();
    const int *st = kStagger[kFieldSpec[fields[f]].loc];
    const int nc = kFieldSpec[fields[f]].ncomp;
    for (int blk = 0; blk < S->nblocks; ++blk) {
      int32_t lo[3], hi[3];
      int64_t n = nc;
      for (int a = 0; a < 3; ++a) {
        lo[a] = -S->nghost;
        hi[a] = S->boxes[blk].n[a] + st[a] + S->nghost;
        n *= hi[a] - lo[a];
      }
      if ((rc = mhd_batch_upload_field(b, slot, fields[f], blk, d, lo, hi, nc))) return rc;
      d += n;
    }
  }
  // the reference synchronises the restored fields before its first derived
  // refresh (Z4_Mercury/src/MercurySolver.cpp:133-145)
  if ((rc = mhd_batch_sync(b, slot, MHD_SYNC_UCELL)) || (rc = mhd_batch_sync(b, slot, MHD_SYNC_BFACE)) ||
      (rc = mhd_batch_prepare(b, slot, img.time, img.step)))
    return rc;
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (step) *step = img.step;
  if (time) *time = img.time;
  return MHD_OK;
}

// The background inputs nondimensionalised as DipoleField::load_from_param
// (Z4_Mercury/include/operators/Dipole.h:46-86) and Build_Badd_FaceFlux's IMF
// (:323-325) do it.
static bool geo_background(const mhd_background &in, GeoBg *out) {
  if (in.n_dipoles < 0 || in.n_dipoles > MHD_MAX_DIPOLES || !(in.L_ref > 0.0) || !(in.B_ref > 0.0) ||
      !(in.mu_mag > 0.0))
    return false;
  if (in.inver_Rem > 0.0 && !(in.eta_width > 0.0)) return false;
  GeoBg g{};
  g.nd = in.n_dipoles;
  double inver_m = 4 * 3.1415926535 * in.B_ref * in.L_ref * in.L_ref * in.L_ref / in.mu_mag;
  inver_m = 1.0 / inver_m;
  for (int d = 0; d < in.n_dipoles; ++d) {
    for (int q = 0; q < 3; ++q) {
      g.r0[d][q] = in.dipole[d][q] / in.L_ref;
      g.m[d][q] = in.dipole[d][3 + q] * inver_m;
    }
    g.a[d] = in.dipole[d][6] / in.L_ref;
  }
  for (int q = 0; q < 3; ++q) g.B0[q] = in.B_imf[q] / in.B_ref;
  g.hall_r_min = in.hall_r_min;
  g.hall_r_max = in.hall_r_max;
  g.inver_Rem = in.inver_Rem;
  g.eta_r0 = in.eta_r_inner;
  g.eta_r1 = in.eta_r_outer;
  g.eta_w = in.eta_width;
  *out = g;
  return true;
}

int mhd_batch_setup_geometry(mhd_batch *b, int slot, int block, const double *nodes, double L_ref) {
  return mhd_batch_setup_geometry_bg(b, slot, block, nodes, L_ref, nullptr);
}

int mhd_batch_setup_geometry_bg(mhd_batch *b, int slot, int block, const double *nodes, double L_ref,
                                const mhd_background *bgp) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  Solve *S = b->slots[slot];
  if (block < 0 || block >= S->nblocks || !nodes) return fail(MHD_ERR_ARG, "mhd_batch_setup_geometry: bad arguments");
  GeoBg bg{};
  if (bgp && !geo_background(*bgp, &bg)) return fail(MHD_ERR_ARG, "mhd_batch_setup_geometry_bg: bad background");
  const Box &bx = S->boxes[block];
  cudaStream_t st = b->stream;
  // the nodes (x, y, z over the whole box) into a temporary device array
  const int e[3] = {bx.n[0] + 1 + 2 * bx.G, bx.n[1] + 1 + 2 * bx.G, bx.n[2] + 1 + 2 * bx.G};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  double *dn = nullptr;
  void **dtab = nullptr;
  auto release = [&]() {
    if (dn) cudaFreeAsync(dn, st);
    if (dtab) cudaFreeAsync(dtab, st);
  };
  // with a background: 3 more arrays for the edge integrals of A
  if (cudaMallocFromPoolAsync((void **)&dn, sizeof(double) * (bgp ? 6 : 3) * (size_t)bx.total, b->pool, st) !=
          cudaSuccess ||
      cudaMallocFromPoolAsync((void **)&dtab, sizeof(void *) * GEO_COUNT, b->pool, st) != cudaSuccess) {
    cudaGetLastError();
    release();
    return fail(MHD_ERR_OOM, "mhd_batch_setup_geometry: temporary arrays");
  }
  if ((rc = ensure_staging(b, npts * 3))) {
    release();
    return rc;
  }
  void *node_ptrs[3] = {dn, dn + bx.total, dn + 2 * bx.total};
  // every output component of the block, in GeoOut order
  std::vector<void *> tab;
  auto add = [&](int field, int ncomp) {
    for (int m = 0; m < ncomp; ++m) tab.push_back(S->comp_ptr(block, kComp.first[field] + m, 0));
  };
  add(MHD_JAC, 1);
  add(MHD_JDXI, 3);
  add(MHD_JDET, 3);
  add(MHD_JDZE, 3);
  for (int f : {MHD_AREA_XI, MHD_AREA_ETA, MHD_AREA_ZETA, MHD_HODGE_FACE_XI, MHD_HODGE_FACE_ETA, MHD_HODGE_FACE_ZETA,
                MHD_DL_XI, MHD_DL_ETA, MHD_DL_ZETA})
    add(f, 1);
  for (int f : {MHD_DR_XI, MHD_DR_ETA, MHD_DR_ZETA}) add(f, 3);
  for (int f : {MHD_HODGE_EDGE_XI, MHD_HODGE_EDGE_ETA, MHD_HODGE_EDGE_ZETA}) add(f, 1);
  add(MHD_BCELL_W, 18);
  add(MHD_JCELL_W, 36);
  for (int f : {MHD_BADD_XI, MHD_BADD_ETA, MHD_BADD_ZETA, MHD_PHOTO, MHD_CELL_X, MHD_CELL_Y, MHD_CELL_Z, MHD_TAPER_XI,
                MHD_TAPER_ETA, MHD_TAPER_ZETA, MHD_TAPER_CELL})
    add(f, 1);
  for (int f : {MHD_ETA_RES_XI, MHD_ETA_RES_ETA, MHD_ETA_RES_ZETA}) {  // only solves with the implicit substep hold it
    if (S->consts.resistive) add(f, 1);
    else tab.push_back(nullptr);
  }
  if ((int)tab.size() != GEO_COUNT) {
    release();
    return fail(MHD_ERR_ARG, "mhd_batch_setup_geometry: output table of %d components", (int)tab.size());
  }
  GeoBox gb;
  for (int a = 0; a < 3; ++a) gb.n[a] = bx.n[a];
  gb.G = bx.G;
  gb.nghost = S->nghost;
  gb.si = bx.si;
  gb.sj = bx.sj;
  gb.total = bx.total;
  cudaError_t ce;
  if ((ce = cudaMemcpyAsync(b->staging, nodes, sizeof(double) * 3 * npts, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(b->comp_ptrs, node_ptrs, sizeof node_ptrs, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(dtab, tab.data(), sizeof(void *) * GEO_COUNT, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
    release();
    return fail(MHD_ERR_CUDA, "mhd_batch_setup_geometry: %s", cudaGetErrorString(ce));
  }
  k_scatter_aos<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(b->staging, -bx.G, -bx.G, -bx.G, e[0], e[1], e[2], 3,
                                                                 b->comp_ptrs, 1, bx.si, bx.sj, bx.G, 0);
  if ((ce = cudaGetLastError()) != cudaSuccess ||
      (ce = launch_geometry(dn, gb, dtab, S->es == 4, L_ref, bgp ? &bg : nullptr, dn + 3 * bx.total, st)) !=
          cudaSuccess) {
    release();
    return fail(MHD_ERR_CUDA, "mhd_batch_setup_geometry: %s", cudaGetErrorString(ce));
  }
  release();
  // page-locked nodes are read by the DMA later: wait before the caller may
  // reuse them (pageable ones were staged before the copy returned)
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, nodes) != cudaSuccess) {
    cudaGetLastError();
    pa.type = cudaMemoryTypeHost;
  }
  if (pa.type != cudaMemoryTypeUnregistered) CUDA_TRY(cudaStreamSynchronize(st));
  S->prepared = false;
  return MHD_OK;
}

int mhd_batch_div_b(mhd_batch *b, int slot, double *max_abs) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  const unsigned long long zero = 0;
  if ((rc = set_state_field(b, slot, offsetof(SolveState, divb_bits), &zero, sizeof zero))) return rc;
  rc = targeted(b, slot, [&](int *nk) { launch(b, 1, SK_DIVB, nk); });
  if (rc) return rc;
  if ((rc = read_state(b))) return rc;
  unsigned long long bits = b->hstate[slot].divb_bits;
  double v;
  std::memcpy(&v, &bits, sizeof v);
  if (max_abs) *max_abs = v;
  return MHD_OK;
}

int mhd_batch_request(mhd_batch *b, int slot, int64_t nsteps) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  if (nsteps < 0) return fail(MHD_ERR_ARG, "nsteps %lld", (long long)nsteps);
  if (nsteps > 0 && !b->slots[slot]->prepared) return fail(MHD_ERR_STATE, "steps requested before prepare");
  const long long n = nsteps;
  return set_state_field(b, slot, offsetof(SolveState, remaining), &n, sizeof n);
}

// Adds the last substep's event time to the batch's sum (its events have
// completed: the caller synchronised the stream after them).
static void fold_substep_time(mhd_batch *b) {
  if (!b->res_ev_pending) return;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, b->res_ev[0], b->res_ev[1]) == cudaSuccess) {
    b->res_ms += ms;
    ++b->res_steps;
  } else {
    cudaGetLastError();
  }
  b->res_ev_pending = false;
}

int mhd_batch_cg_host_loop(mhd_batch *b, int on) {
  if (!b) return fail(MHD_ERR_ARG, "mhd_batch_cg_host_loop: null batch");
  b->cg_host_loop = on != 0;
  if (b->shadow) b->shadow->cg_host_loop = on != 0;
  return MHD_OK;
}

int mhd_batch_substep_ms(mhd_batch *b, double *ms_per_step) {
  if (!b || !ms_per_step) return fail(MHD_ERR_ARG, "mhd_batch_substep_ms: bad arguments");
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  fold_substep_time(b);
  *ms_per_step = b->res_steps > 0 ? b->res_ms / (double)b->res_steps : 0.0;
  b->res_ms = 0.0;
  b->res_steps = 0;
  return MHD_OK;
}

int mhd_batch_run(mhd_batch *b, int nsteps) {
  if (!b || nsteps < 0) return fail(MHD_ERR_ARG, "mhd_batch_run: bad arguments");
  int rc;
  if (b->n_res == 0) {
    if ((rc = build_graph(b))) return rc;
    for (int s = 0; s < nsteps; ++s) CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    return MHD_OK;
  }
  // with implicit resistive solves: part A, their substep (all at once, host-driven), part B
  if ((rc = capture(b, &b->graph_a, nullptr, [&](int *nk) { enqueue_step_a(b, nk); }))) return rc;
  if ((rc = capture(b, &b->graph_b, nullptr, [&](int *nk) { enqueue_step_b(b, nk, true); }))) return rc;
  if (!b->res_ev[0]) {
    CUDA_TRY(cudaEventCreate(&b->res_ev[0]));
    CUDA_TRY(cudaEventCreate(&b->res_ev[1]));
  }
  std::vector<int> slots;
  for (int s = 0; s < nsteps; ++s) {
    CUDA_TRY(cudaGraphLaunch(b->graph_a, b->stream));
    if ((rc = read_state(b))) return rc;
    fold_substep_time(b);  // the previous step's substep is complete
    slots.clear();
    for (int q = 0; q < b->capacity; ++q) {
      const Solve *S = b->slots[q];
      if (S && S->consts.resistive && b->hstate[q].remaining > 0 && b->hstate[q].status == 0) slots.push_back(q);
    }
    if (!slots.empty()) CUDA_TRY(cudaEventRecord(b->res_ev[0], b->stream));
    if ((rc = res_step(b, slots))) return rc;
    if (!slots.empty()) {
      CUDA_TRY(cudaEventRecord(b->res_ev[1], b->stream));
      b->res_ev_pending = true;
    }
    CUDA_TRY(cudaGraphLaunch(b->graph_b, b->stream));
  }
  return MHD_OK;
}

// Host-side fields of a slot's mhd_info: device bytes (with an FP64
// companion's) and the last implicit substep's figures.
static void fill_solve_info(const mhd_batch *b, int s, mhd_info *info) {
  const Solve *S = b->slots[s];
  if (!S) return;
  info->device_bytes = S->arena_bytes + S->T->table_bytes;
  if (S->shadow_slot >= 0) {
    const Solve *C = b->shadow->slots[S->shadow_slot];
    info->device_bytes += C->arena_bytes + C->T->table_bytes;
  }
  info->res_relres = S->res_relres;
  info->res_iters = S->res_iters;
  info->res_refinements = S->res_refinements;
}

int mhd_batch_poll(mhd_batch *b, mhd_info *infos) {
  if (!b || !infos) return fail(MHD_ERR_ARG, "mhd_batch_poll: bad arguments");
  int rc = read_state(b);
  if (rc) return rc;
  for (int s = 0; s < b->capacity; ++s) {
    const SolveState &st = b->hstate[s];
    std::memset(&infos[s], 0, sizeof(mhd_info));
    infos[s].time = st.time;
    infos[s].dt = st.dt;
    infos[s].step = st.step;
    infos[s].status = st.status;
    infos[s].remaining = st.remaining;
    fill_solve_info(b, s, &infos[s]);
  }
  return MHD_OK;
}

static void fill_infos(mhd_batch *b, const SolveState *hs, mhd_info *infos) {
  for (int s = 0; s < b->capacity; ++s) {
    const SolveState &st = hs[s];
    std::memset(&infos[s], 0, sizeof(mhd_info));
    infos[s].time = st.time;
    infos[s].dt = st.dt;
    infos[s].step = st.step;
    infos[s].status = st.status;
    infos[s].remaining = st.remaining;
    fill_solve_info(b, s, &infos[s]);
  }
}

int mhd_batch_poll_async(mhd_batch *b, int *ticket) {
  if (!b || !ticket) return fail(MHD_ERR_ARG, "mhd_batch_poll_async: bad arguments");
  const int t = b->snap_next;
  b->snap_next ^= 1;
  CUDA_TRY(cudaMemcpyAsync(b->hsnap[t], b->dstate, sizeof(SolveState) * b->capacity, cudaMemcpyDeviceToHost,
                           b->stream));
  CUDA_TRY(cudaEventRecord(b->snap_ev[t], b->stream));
  *ticket = t;
  return MHD_OK;
}

int mhd_batch_poll_wait(mhd_batch *b, int ticket, mhd_info *infos) {
  if (!b || !infos || ticket < 0 || ticket > 1) return fail(MHD_ERR_ARG, "mhd_batch_poll_wait: bad arguments");
  CUDA_TRY(cudaEventSynchronize(b->snap_ev[ticket]));
  fill_infos(b, b->hsnap[ticket], infos);
  return MHD_OK;
}

void *mhd_batch_stream(mhd_batch *b) { return b ? (void *)b->stream : nullptr; }

int mhd_batch_kernels_per_step(mhd_batch *b) {
  if (!b) return -1;
  if (build_graph(b) != MHD_OK) return -1;
  return b->kernels_per_step;
}

int mhd_batch_step_profiled(mhd_batch *b, int nsteps, int max_kernels, float *kernel_ms, const char **kernel_names,
                            int *n_kernels) {
  if (!b || nsteps < 1 || !kernel_ms || !n_kernels) return fail(MHD_ERR_ARG, "mhd_step_profiled: bad arguments");
  std::vector<float> acc;
  int per_step = 0;
  for (int s = 0; s < nsteps; ++s) {
    b->profiling = true;
    b->prof_used = 0;
    mark(b, "start");
    int nk = 0;
    enqueue_step(b, &nk);
    b->profiling = false;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    per_step = (int)b->prof_used - 1;
    if (acc.empty()) acc.assign(per_step, 0.0f);
    for (int q = 0; q < per_step; ++q) {
      float ms = 0.0f;
      CUDA_TRY(cudaEventElapsedTime(&ms, b->prof_events[q], b->prof_events[q + 1]));
      acc[q] += ms;
    }
  }
  const int n = per_step < max_kernels ? per_step : max_kernels;
  for (int q = 0; q < n; ++q) {
    kernel_ms[q] = acc[q] / (float)nsteps;
    if (kernel_names) kernel_names[q] = b->prof_names[q + 1];
  }
  *n_kernels = n;
  return MHD_OK;
}

int mhd_batch_device_view(mhd_batch *b, int slot, int field, int block, int comp, double **base, int32_t *G,
                          int64_t *si, int64_t *sj, int32_t ext[3]) {
  int rc = slot_check(b, slot);
  if (rc) return rc;
  Solve *S = b->slots[slot];
  if (field < 0 || field >= MHD_NUM_FIELDS || block < 0 || block >= S->nblocks || comp < 0 ||
      comp >= kFieldSpec[field].ncomp)
    return fail(MHD_ERR_ARG, "mhd_device_view: bad arguments");
  if ((rc = read_state(b))) return rc;
  const Box &bx = S->boxes[block];
  if (base) *base = (double *)S->comp_ptr(block, kComp.first[field] + comp, b->hstate[slot].cur);
  if (G) *G = bx.G;
  if (si) *si = bx.si;
  if (sj) *sj = bx.sj;
  if (ext)
    for (int a = 0; a < 3; ++a) ext[a] = bx.ext[a];
  return MHD_OK;
}

// ------------------------------------------------------------------ single solve
int mhd_ctx_create(const mhd_desc *desc, mhd_ctx **out) {
  if (!desc || !out) return fail(MHD_ERR_ARG, "mhd_ctx_create: bad descriptor");
  auto *ctx = new (std::nothrow) mhd_ctx();
  if (!ctx) return fail(MHD_ERR_OOM, "host allocation");
  const int prec = desc->precision == kMixed ? kMixed : kFP64;
  int rc = mhd_batch_create(1, prec, &ctx->batch);
  if (rc) {
    delete ctx;
    return rc;
  }
  int slot = -1;
  if ((rc = mhd_batch_add(ctx->batch, desc, &slot))) {
    const std::string err = g_last_error;
    mhd_batch_destroy(ctx->batch);
    delete ctx;
    g_last_error = err;
    return rc;
  }
  *out = ctx;
  return MHD_OK;
}

int mhd_ctx_destroy(mhd_ctx *ctx) {
  if (!ctx) return MHD_OK;
  mhd_batch_destroy(ctx->batch);
  delete ctx;
  return MHD_OK;
}

int mhd_upload_field(mhd_ctx *ctx, int field, int block, const double *data, const int32_t lo[3], const int32_t hi[3],
                     int ncomp) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_upload_field(ctx->batch, 0, field, block, data, lo, hi, ncomp);
}

int mhd_fluid_tile(mhd_ctx *ctx, int variant) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_fluid_tile(ctx->batch, variant);
}

int mhd_set_constants(mhd_ctx *ctx, const mhd_constants *constants) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_set_constants(ctx->batch, 0, constants);
}

int mhd_fill_field(mhd_ctx *ctx, int field, int block, const double *values, const int32_t lo[3], const int32_t hi[3],
                   int ncomp) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_fill_field(ctx->batch, 0, field, block, values, lo, hi, ncomp);
}

int mhd_download_field(mhd_ctx *ctx, int field, int block, double *data, const int32_t lo[3], const int32_t hi[3],
                       int ncomp) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_download_field(ctx->batch, 0, field, block, data, lo, hi, ncomp);
}

int mhd_prepare(mhd_ctx *ctx, double time, int64_t step) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_prepare(ctx->batch, 0, time, step);
}

int mhd_step_async(mhd_ctx *ctx, int nsteps) {
  if (!ctx || nsteps < 0) return fail(MHD_ERR_ARG, "mhd_step: bad arguments");
  int rc = mhd_batch_request(ctx->batch, 0, nsteps);
  if (rc) return rc;
  return mhd_batch_run(ctx->batch, nsteps);
}

int mhd_synchronize(mhd_ctx *ctx) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  int rc = read_state(ctx->batch);
  if (rc) return rc;
  const SolveState &s = ctx->batch->hstate[0];
  if (s.status) return fail(s.status, "device status %d at step %lld", s.status, s.step);
  return MHD_OK;
}

int mhd_step(mhd_ctx *ctx, int nsteps, double *dt_out) {
  int rc = mhd_step_async(ctx, nsteps);
  if (rc) return rc;
  if ((rc = mhd_synchronize(ctx))) return rc;
  if (dt_out) *dt_out = ctx->batch->hstate[0].dt;
  return MHD_OK;
}

int mhd_step_profiled(mhd_ctx *ctx, int nsteps, int max_kernels, float *kernel_ms, const char **kernel_names,
                      int *n_kernels) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  if (nsteps < 1) return fail(MHD_ERR_ARG, "mhd_step_profiled: bad arguments");
  int rc = mhd_batch_request(ctx->batch, 0, nsteps);
  if (rc) return rc;
  rc = mhd_batch_step_profiled(ctx->batch, nsteps, max_kernels, kernel_ms, kernel_names, n_kernels);
  if (rc) return rc;
  return mhd_synchronize(ctx);
}

int mhd_div_b(mhd_ctx *ctx, double *max_abs) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_div_b(ctx->batch, 0, max_abs);
}

int mhd_setup_geometry(mhd_ctx *ctx, int block, const double *nodes, double L_ref) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_setup_geometry(ctx->batch, 0, block, nodes, L_ref);
}

int mhd_setup_geometry_bg(mhd_ctx *ctx, int block, const double *nodes, double L_ref, const mhd_background *bg) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_setup_geometry_bg(ctx->batch, 0, block, nodes, L_ref, bg);
}

int mhd_save_restart(mhd_ctx *ctx, const char *path) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_save_restart(ctx->batch, 0, path);
}

int mhd_load_restart(mhd_ctx *ctx, const char *path, int32_t *step, double *time) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_load_restart(ctx->batch, 0, path, step, time);
}

int mhd_sync(mhd_ctx *ctx, int group) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_sync(ctx->batch, 0, group);
}

int mhd_get_info(mhd_ctx *ctx, mhd_info *info) {
  if (!ctx || !info) return fail(MHD_ERR_ARG, "mhd_get_info: bad arguments");
  return mhd_batch_poll(ctx->batch, info);
}

int mhd_get_status(mhd_ctx *ctx, int32_t *status) {
  if (!ctx || !status) return fail(MHD_ERR_ARG, "mhd_get_status: bad arguments");
  const int rc = read_state(ctx->batch);
  if (rc) return rc;
  *status = ctx->batch->hstate[0].status;
  return MHD_OK;
}

void *mhd_stream(mhd_ctx *ctx) { return ctx ? mhd_batch_stream(ctx->batch) : nullptr; }

int mhd_kernels_per_step(mhd_ctx *ctx) { return ctx ? mhd_batch_kernels_per_step(ctx->batch) : -1; }

int mhd_device_view(mhd_ctx *ctx, int field, int block, int comp, double **base, int32_t *G, int64_t *si, int64_t *sj,
                    int32_t ext[3]) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  return mhd_batch_device_view(ctx->batch, 0, field, block, comp, base, G, si, sj, ext);
}

}  // extern "C"
