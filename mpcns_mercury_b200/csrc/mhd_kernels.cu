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
#include <mutex>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <type_traits>

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
constexpr int cDIVB = kComp.first[MHD_DIVB];
constexpr int cETAR = kComp.first[MHD_ETA_RES_XI];  // ETA_RES_ETA, ETA_RES_ZETA follow
constexpr int cRW = kComp.first[MHD_RES_W], cRX = kComp.first[MHD_RES_X], cRR = kComp.first[MHD_RES_R],
              cRP = kComp.first[MHD_RES_P], cRQ = kComp.first[MHD_RES_Q], cRBS = kComp.first[MHD_RES_BSTAR];
constexpr int cFNX = kComp.first[MHD_FNORM_XI], cFNY = kComp.first[MHD_FNORM_ETA], cFNZ = kComp.first[MHD_FNORM_ZETA];
constexpr int cPEN = kComp.first[MHD_PE_NODE], cAMB = kComp.first[MHD_AMBI_COEF], cDPE = kComp.first[MHD_DPE];
constexpr int cUCK = kComp.first[MHD_UCON_COEF];
constexpr int cIHX = kComp.first[MHD_HALL_IH_XI], cIHY = kComp.first[MHD_HALL_IH_ETA], cIHZ = kComp.first[MHD_HALL_IH_ZETA];
constexpr int cFM = kComp.first[MHD_FLUX_METRIC];
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
static_assert(cBFY == cBFX + 1 && cBFZ == cBFX + 2 && cALY == cALX + 1 && cALZ == cALX + 2, "xi, eta, zeta consecutive");
constexpr int cBAX = kComp.first[MHD_BADD_XI], cBAY = kComp.first[MHD_BADD_ETA], cBAZ = kComp.first[MHD_BADD_ZETA];
constexpr int cPHOTO = kComp.first[MHD_PHOTO], cCX = kComp.first[MHD_CELL_X];  // CELL_Y, CELL_Z follow
constexpr int cTPX = kComp.first[MHD_TAPER_XI], cTPY = kComp.first[MHD_TAPER_ETA], cTPZ = kComp.first[MHD_TAPER_ZETA];
constexpr int cTPC = kComp.first[MHD_TAPER_CELL];
constexpr int cLEX = kComp.first[MHD_LOCAL_ETA_XI];  // LOCAL_ETA_ETA, LOCAL_ETA_ZETA follow

// std::max / std::min semantics (first argument wins ties, incl. signed zeros).
template <class R>
__device__ __forceinline__ R dmax(R a, R b) { return (a < b) ? b : a; }
template <class R>
__device__ __forceinline__ R dmin(R a, R b) { return (b < a) ? b : a; }

// One block's fields for the current step: U = current buffer, M = metric
// (double) then the other real-valued components (mhd_engine.cuh).
// Element offsets inside a block are 32-bit (mhd_batch_add keeps every
// block's component arrays below 2^31 elements in total).
template <class R>
struct V {
  R *U, *Un;
  char *M;
  int total, si, sj;
  int G, n0, n1, n2;
  // real-valued component (U or M)
  __device__ __forceinline__ R *c(int comp) const {
    return comp < kNumUComps ? U + comp * total : (R *)(M + (int64_t)kNumMetric * total * 8) + rslot(comp) * total;
  }
  // metric component (JAC, JD*), double in every precision
  __device__ __forceinline__ double *m(int comp) const { return (double *)M + (comp - kMetricFirst) * total; }
  __device__ __forceinline__ int off(int i, int j, int k) const { return (i + G) * si + (j + G) * sj + (k + G); }
};
#define AT(cc, i, j, k) (B.c(cc)[B.off((i), (j), (k))])
#define ATM(cc, i, j, k) (B.m(cc)[B.off((i), (j), (k))])
// Reads of an array the kernel does not write, through the read-only path:
// the compiler may then move them ahead of the kernel's stores (it cannot
// prove that plain loads and stores into one arena do not alias).  Used by
// the primitive-variable pass, where it measured faster; elsewhere it did not.
#define LD(cc, i, j, k) __ldg(B.c(cc) + B.off((i), (j), (k)))
#define LDM(cc, i, j, k) __ldg(B.m(cc) + B.off((i), (j), (k)))

struct Item {
  int s;       // solve
  int blk;     // block of the solve
  int species; // kCells2 only
  int i, j, k;
  bool in;     // inside the kernel's range
  int o[3];    // tile origin (i, j, k)
  int hi[3];   // range upper bounds (exclusive)
  int lo[3];   // range lower bounds
};

struct NoTileEnd {
  __device__ void operator()(int) const {}
};

// The solve s, its block b and the block's tile t of work item w of range
// KIND (two binary searches over the directory's prefix sums).
template <int KIND>
__device__ __forceinline__ void lookup_item(const Dir &D, int w, int &s, int &b, int &t) {
  const int *sp = D.solve_tile_prefix[KIND];
  int lo = 0, hi = D.nsolves;  // largest s with sp[s] <= w
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (sp[mid] <= w) lo = mid; else hi = mid;
  }
  s = lo;
  const int lw = w - sp[s];
  const int *bp = D.solves[s].tile_prefix[KIND];
  int blo = 0, bhi = D.solves[s].nblocks;
  while (bhi - blo > 1) {
    const int mid = (blo + bhi) >> 1;
    if (bp[mid] <= lw) blo = mid; else bhi = mid;
  }
  b = blo;
  t = lw - bp[blo];
}

// Origin (i, j, k) and species of tile t of a fluid range over range box r.
template <int KIND>
__device__ __forceinline__ void fluid_tile_origin(const RangeBox &r, int t, int o[3], int &species) {
  constexpr FluidTile T = fluid_tile(fluid_variant(KIND));
  species = t & 1;
  t >>= 1;
  const int tk = (r.hi[2] - r.lo[2] + T.k - 1) / T.k;
  const int tj = (r.hi[1] - r.lo[1] + T.j - 1) / T.j;
  const int bk = t % tk, bj = (t / tk) % tj, bi = t / (tk * tj);
  o[0] = r.lo[0] + bi * T.i;
  o[1] = r.lo[1] + bj * T.j;
  o[2] = r.lo[2] + bk * T.k;
}

// The work item (s, b, t) of range KIND as this thread sees it, and the
// block's fields of the current step.
template <class R, int KIND>
__device__ __forceinline__ void build_item(const Dir &D, int s, int b, int t, Item &it, V<R> &B) {
  const int tid = threadIdx.x;
  const DevSolve &S = D.solves[s];
  const DevBlock &DB = S.blocks[b];
  RangeBox r = range_of(KIND, DB.n, S.c.nghost);
  if constexpr (KIND == kResK) r.hi[2] = DB.reskhi;
  it.s = s;
  it.blk = b;
  it.species = 0;
  for (int a = 0; a < 3; ++a) {
    it.hi[a] = r.hi[a];
    it.lo[a] = r.lo[a];
  }
  if constexpr (fluid_variant(KIND) >= 0) {  // a fluid tile, one species
    constexpr FluidTile T = fluid_tile(fluid_variant(KIND));
    fluid_tile_origin<KIND>(r, t, it.o, it.species);
    it.k = it.o[2] + (tid % T.k);
    it.j = it.o[1] + ((tid / T.k) % T.j);
    it.i = it.o[0] + (tid / (T.k * T.j));
    it.in = it.i < r.hi[0] && it.j < r.hi[1] && it.k < r.hi[2];
  } else {  // a run of kTileThreads consecutive positions of the range box (k fastest)
    const int ek = r.hi[2] - r.lo[2], ej = r.hi[1] - r.lo[1];
    const int L = t * kTileThreads + tid;
    const int rest = L / ek;
    it.k = r.lo[2] + (L - rest * ek);
    it.j = r.lo[1] + rest % ej;
    it.i = r.lo[0] + rest / ej;
    it.in = L < ek * ej * (r.hi[0] - r.lo[0]);
    it.o[0] = it.o[1] = it.o[2] = 0;
  }
  const int cur = D.state[s].cur;
  B.U = (R *)DB.U[cur];
  B.Un = (R *)DB.U[cur ^ 1];
  B.M = DB.M;
  B.total = (int)DB.total;
  B.si = (int)DB.si;
  B.sj = (int)DB.sj;
  B.G = DB.G;
  B.n0 = DB.n[0];
  B.n1 = DB.n[1];
  B.n2 = DB.n[2];
}

// Work-item loop: for every tile of range `KIND` of every active solve, call
// f(S, B, item), then end(w) with the tile's index w over all solves (every
// thread of the CTA).  Tile lookup by thread 0, broadcast through shared
// memory.
template <class R, int KIND, class F, class E = NoTileEnd>
__device__ __forceinline__ void for_items(const Dir &D, F &&f, E &&end = E{}) {
  __shared__ int sh[3];
  const int total = D.solve_tile_prefix[KIND][D.nsolves];
  const int tid = threadIdx.x;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    if (tid == 0) lookup_item<KIND>(D, w, sh[0], sh[1], sh[2]);
    __syncthreads();
    const int s = sh[0], b = sh[1], t = sh[2];
    __syncthreads();
    if (!solve_active(D, s)) continue;  // inactive solve (the whole CTA agrees)
    Item it;
    V<R> B;
    build_item<R, KIND>(D, s, b, t, it, B);
    f(D.solves[s], B, it);
    end(w);
  }
}

// ------------------------------------------------------------------ TMA staging
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for phase `parity` of the barrier to complete, at most about a
// second: false when it did not (the caller records MHD_ERR_TIMEOUT).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (int n = 0; n < (1 << 24); ++n) {
    if (mbar_try_wait(bar, parity)) return true;
    if (n >= 16) __nanosleep(64);
  }
  return false;
}
// One 4-D tiled tensor copy (no multicast) of the box at coordinates
// (c0 .. c3) into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void *dst, const void *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// The staged variant's 256 compute threads synchronise among themselves
// (named barrier 1; its producer warp takes no part).
__device__ __forceinline__ void compute_bar() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
__device__ __forceinline__ bool compute_and(bool v) {
  uint32_t r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, 256, p;\n selp.u32 %0, 1, 0, q;\n}"
               : "=r"(r)
               : "r"((uint32_t)v)
               : "memory");
  return r != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Work-item loop of the TMA-staged fluid variant, warp-specialised: the
// CTA's 256 compute threads run f(S, B, item, box) for its items, while its
// ninth warp (one lane) looks the items up and stages each one's box
// (density, then u, v, w, p of its species; k window of
// tma_box_k(sizeof(R)) from the 16-byte unit holding k = o - 1, j and i
// windows of 6 from o - 1) with TMA tensor copies into one of two stages,
// running up to two items ahead.  bars[0..1]: a stage is full (the item's
// record, and its copies complete); bars[2..3]: the compute threads are done
// reading it (f arrives once its face fluxes are built).  A block without
// tensor maps has its box loaded by the compute threads instead.  A wait that
// does not end within its bound records MHD_ERR_TIMEOUT on the solve of the
// item waited for and ends the CTA's loop.
template <class R, int KIND, class F>
__device__ __forceinline__ void for_fluid_items_tma(const Dir &D, R *stage, uint64_t *bars, F &&f) {
  constexpr int W = tma_box_k(sizeof(R)), BV = W * kTmaBoxJI * kTmaBoxJI;
  constexpr int kAlign = 16 / (int)sizeof(R);
  __shared__ int sh[2][4];  // per stage: solve, block, tile, copy state (0 inactive, 1 TMA, 2 by the threads)
  const int total = D.solve_tile_prefix[KIND][D.nsolves];
  const int tid = threadIdx.x;
  // the box's coordinates in the block's arrays (k, j, i including the ghost offset)
  auto box_at = [&](const DevBlock &DB, int s, int t, int c[3], int &species) {
    const DevSolve &S = D.solves[s];
    const RangeBox r = range_of(KIND, DB.n, S.c.nghost);
    int o[3];
    fluid_tile_origin<KIND>(r, t, o, species);
    c[0] = (o[2] + DB.G - 1) & ~(kAlign - 1);
    c[1] = o[1] - 1 + DB.G;
    c[2] = o[0] - 1 + DB.G;
  };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], kTileThreads);
    mbar_init(&bars[3], kTileThreads);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid >= kTileThreads) {  // the producer warp
    if (tid != kTileThreads) return;
    uint32_t n = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x, ++n) {
      const int st = n & 1;
      int s, b, t;
      lookup_item<KIND>(D, w, s, b, t);
      if (n >= 2 && !mbar_wait_bounded(&bars[2 + st], ((n >> 1) - 1) & 1u)) {
        atomicCAS(&D.state[s].status, 0, (int)MHD_ERR_TIMEOUT);
        return;
      }
      sh[st][0] = s;
      sh[st][1] = b;
      sh[st][2] = t;
      const DevBlock &DB = D.solves[s].blocks[b];
      if (!solve_active(D, s) || !DB.tmap) {
        sh[st][3] = solve_active(D, s) ? 2 : 0;
        mbar_arrive(&bars[st]);
        continue;
      }
      sh[st][3] = 1;
      int c[3], species;
      box_at(DB, s, t, c, species);
      const char *maps = (const char *)DB.tmap;
      R *dst = stage + st * 5 * BV;
      const int cur = D.state[s].cur;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the stage's earlier reads, then the copies
      mbar_expect_tx(&bars[st], (uint32_t)(5 * BV * sizeof(R)));
      tma_load_4d(dst, maps + 128 * cur, c[0], c[1], c[2], species ? 5 : 0, &bars[st]);
      tma_load_4d(dst + BV, maps + 256, c[0], c[1], c[2], rslot(species ? cPVN : cPVH), &bars[st]);
    }
    return;
  }
  uint32_t n = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x, ++n) {
    const int st = n & 1;
    const bool ok = mbar_wait_bounded(&bars[st], (n >> 1) & 1u);
    if (!compute_and(ok)) {
      if (tid == 0) atomicCAS(&D.state[sh[st][0]].status, 0, (int)MHD_ERR_TIMEOUT);
      return;
    }
    const int s = sh[st][0], b = sh[st][1], t = sh[st][2], how = sh[st][3];
    R *box = stage + st * 5 * BV;
    if (how == 0) {  // inactive solve (every compute thread agrees)
      mbar_arrive(&bars[2 + st]);
      continue;
    }
    if (how == 2) {  // no tensor maps: the same box by plain loads (zeros outside the block's arrays)
      const DevBlock &DB = D.solves[s].blocks[b];
      int c[3], species;
      box_at(DB, s, t, c, species);
      const int cur = D.state[s].cur;
      const R *u0p = (const R *)DB.U[cur] + (species ? 5 : 0) * DB.total;
      const R *pvp = (const R *)(DB.M + (int64_t)kNumMetric * DB.total * 8) +
                     (int64_t)rslot(species ? cPVN : cPVH) * DB.total;
      const int ext1 = DB.n[1] + 1 + 2 * DB.G, ext0 = DB.n[0] + 1 + 2 * DB.G;
      for (int q = tid; q < 5 * BV; q += kTileThreads) {
        const int m = q / BV, e = q % BV;
        const int x = c[0] + e % W, y = c[1] + (e / W) % kTmaBoxJI, z = c[2] + e / (W * kTmaBoxJI);
        const R *src = m == 0 ? u0p : pvp + (int64_t)(m - 1) * DB.total;
        box[q] = (x < DB.sj && y < ext1 && z < ext0) ? src[(int64_t)z * DB.si + (int64_t)y * DB.sj + x] : R(0.0);
      }
      compute_bar();
    }
    Item it;
    V<R> B;
    build_item<R, KIND>(D, s, b, t, it, B);
    f(D.solves[s], B, it, (const R *)box);
  }
}

template <class R>
struct Num {
  R nH, nNa, ne_eff, chiH, chiNa, wH, wNa;
};

// Hall_Num_Limiter (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:111-157)
template <class R>
__device__ __forceinline__ Num<R> num_limiter(const ConstsT<R> &c, R rhoH, R rhoNa) {
  Num<R> d;
  const R rH = dmax(rhoH, R(0.0)), rN = dmax(rhoNa, R(0.0));
  d.nH = rH / c.M_H * c.M_ref;
  d.nNa = rN / c.M_Na * c.M_ref;
  const R ne_true = d.nH + d.nNa;
  d.ne_eff = sqrt(ne_true * ne_true + c.ne_hall_floor * c.ne_hall_floor);
  if ((double)ne_true > 1.0e-300) {
    d.chiH = d.nH / ne_true;
    d.chiNa = d.nNa / ne_true;
  } else {
    d.chiH = R(1.0);
    d.chiNa = R(0.0);
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
template <class R>
__device__ __forceinline__ R face_tot(const V<R> &B, int axis, int i, int j, int k) {
  return AT(bcomp(axis), i, j, k) + AT(bacomp(axis), i, j, k);
}
template <class R>
__device__ __forceinline__ R cell_beta_ind(const V<R> &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return R(0.5) * (AT(bcomp(axis), i, j, k) + AT(bcomp(axis), ip, jp, kp));
}
template <class R>
__device__ __forceinline__ R cell_beta_tot(const V<R> &B, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, ip, jp, kp, 1);
  return R(0.5) * (face_tot(B, axis, i, j, k) + face_tot(B, axis, ip, jp, kp));
}
template <class R>
__device__ __forceinline__ R ucon(const V<R> &B, int axis, int i, int j, int k) { return AT(cUC + axis, i, j, k); }

// flux() of AssembleOneDirectionEMF_ (Ideal.cpp:517-536).  The right cell's
// cell-averaged total and induced B (btR[ba], biR[ba]) and contravariant
// velocities (uR[a]) are evaluated once per cell by the caller: every face
// family of the cell shares that cell.
template <class R>
__device__ __forceinline__ R emf_flux(const V<R> &B, int ba, int fa, int iL, int jL, int kL, const R btR[3],
                                      const R biR[3], const R uR[3], R bff) {
  const R btL = cell_beta_tot(B, ba, iL, jL, kL);
  const R biL = cell_beta_ind(B, ba, iL, jL, kL);
  const R ufL = ucon(B, fa, iL, jL, kL), ufR = uR[fa];
  const R ubL = ucon(B, ba, iL, jL, kL), ubR = uR[ba];
  const R GL = ufL * btL - ubL * bff, GR = ufR * btR[ba] - ubR * bff;
  const R r = dmax(fabs(ufL), fabs(ufR));
  return R(0.5) * (GL + GR) - R(0.5) * r * (biR[ba] - biL);
}

// Electron pressure at node (i, j, k): the mean of p_H + p_Na over the 8
// cells around it, summed in the order of AddAmbipolarEdgeEMF_
// (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ambipo.cpp:3-143).
template <class R>
__device__ __forceinline__ R pe_node(const V<R> &B, int i, int j, int k) {
  R sum = R(0.0);
  for (int di = -1; di <= 0; ++di)
    for (int dj = -1; dj <= 0; ++dj)
      for (int dk = -1; dk <= 0; ++dk)
        sum += AT(cPVH + 3, i + di, j + dj, k + dk) + AT(cPVN + 3, i + di, j + dj, k + dk);
  return R(0.125) * sum;
}

// AssembleOneDirectionEMF_ (Ideal.cpp:433-594) for all three face families on
// [-1, inner_hi + 1) (the one locally evaluated ghost layer, Ideal.cpp:548-555),
// and, with the ambipolar term on, the node electron pressure on [0, n + 1)
// that the edge EMFs of the owned edges read (each node is shared by six
// edges) and the grad p_e source term of the owned cells that the fluid
// update of both species reads.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_face_emf(Dir D) {
  for_items<R, kExt>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const int q[3] = {i, j, k}, n[3] = {B.n0, B.n1, B.n2};
    if (consts_of<R>(S).ambipolar && i >= 0 && j >= 0 && k >= 0 && i <= n[0] && j <= n[1] && k <= n[2]) {
      AT(cPEN, i, j, k) = pe_node(B, i, j, k);
      if (i < n[0] && j < n[1] && k < n[2]) {
        // grad p_e term of the ion momentum sources of an owned cell, the
        // same for both species (AddSourceToRHS_Fluid, FluidRHS.cpp:206-527)
        const R pip = AT(cPVH + 3, i + 1, j, k) + AT(cPVN + 3, i + 1, j, k);
        const R pim = AT(cPVH + 3, i - 1, j, k) + AT(cPVN + 3, i - 1, j, k);
        const R pjp = AT(cPVH + 3, i, j + 1, k) + AT(cPVN + 3, i, j + 1, k);
        const R pjm = AT(cPVH + 3, i, j - 1, k) + AT(cPVN + 3, i, j - 1, k);
        const R pkp = AT(cPVH + 3, i, j, k + 1) + AT(cPVN + 3, i, j, k + 1);
        const R pkm = AT(cPVH + 3, i, j, k - 1) + AT(cPVN + 3, i, j, k - 1);
        const R ax = AT(cAMB, i, j, k), ay = AT(cAMB + 1, i, j, k), az = AT(cAMB + 2, i, j, k);
        const R bx = AT(cAMB + 3, i, j, k), by = AT(cAMB + 4, i, j, k), bz = AT(cAMB + 5, i, j, k);
        const R cxm = AT(cAMB + 6, i, j, k), cym = AT(cAMB + 7, i, j, k), czm = AT(cAMB + 8, i, j, k);
        AT(cDPE, i, j, k) = R(0.5) * (ax * (pip - pim) + bx * (pjp - pjm) + cxm * (pkp - pkm));
        AT(cDPE + 1, i, j, k) = R(0.5) * (ay * (pip - pim) + by * (pjp - pjm) + cym * (pkp - pkm));
        AT(cDPE + 2, i, j, k) = R(0.5) * (az * (pip - pim) + bz * (pjp - pjm) + czm * (pkp - pkm));
      }
    }
    // this cell is the right cell of its three faces
    R btR[3], biR[3], uR[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      btR[a] = cell_beta_tot(B, a, i, j, k);
      biR[a] = cell_beta_ind(B, a, i, j, k);
      uR[a] = ucon(B, a, i, j, k);
    }
#pragma unroll 1
    for (int fa = 0; fa < 3; ++fa) {
      bool in = true;
      for (int a = 0; a < 3; ++a) in = in && q[a] < n[a] + (a == fa ? 1 : 0) + 1;
      if (!in) continue;
      int iL = i, jL = j, kL = k;
      shift1(fa, iL, jL, kL, -1);
      const R bff = face_tot(B, fa, i, j, k);
      R e0 = R(0.0), e1 = R(0.0), e2 = R(0.0);
      if (fa == 0) {
        const R Ge = emf_flux(B, 1, 0, iL, jL, kL, btR, biR, uR, bff);
        const R Gz = emf_flux(B, 2, 0, iL, jL, kL, btR, biR, uR, bff);
        e1 = Gz;
        e2 = -Ge;
      } else if (fa == 1) {
        const R Gx = emf_flux(B, 0, 1, iL, jL, kL, btR, biR, uR, bff);
        const R Gz = emf_flux(B, 2, 1, iL, jL, kL, btR, biR, uR, bff);
        e0 = -Gz;
        e2 = Gx;
      } else {
        const R Gx = emf_flux(B, 0, 2, iL, jL, kL, btR, biR, uR, bff);
        const R Ge = emf_flux(B, 1, 2, iL, jL, kL, btR, biR, uR, bff);
        e0 = Ge;
        e1 = -Gx;
      }
      const int ce = fa == 0 ? cEFX : fa == 1 ? cEFY : cEFZ;
      const int o = B.off(i, j, k);
      B.c(ce)[o] = e0;
      B.c(ce + 1)[o] = e1;
      B.c(ce + 2)[o] = e2;
    }
  });
}

template <class R>
__device__ __forceinline__ R max_abs_u4(const V<R> &B, int axis, int i0, int j0, int k0, int i1, int j1, int k1,
                                             int i2, int j2, int k2, int i3, int j3, int k3) {
  R a = R(0.0);
  a = dmax(a, fabs(ucon(B, axis, i0, j0, k0)));
  a = dmax(a, fabs(ucon(B, axis, i1, j1, k1)));
  a = dmax(a, fabs(ucon(B, axis, i2, j2, k2)));
  a = dmax(a, fabs(ucon(B, axis, i3, j3, k3)));
  return a;
}

// AddArtificialResistivityToEdgeEMF_ and AddLocalArtificialResistivityToEdgeEMF_
// (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Resis.cpp:6-64, 66-185) on one owned edge of
// family `axis`: E += eta_art(|J| / |dr|) J, then E += eta_local J.
template <class R>
__device__ __forceinline__ R add_artificial(const V<R> &B, const ConstsT<R> &c, int axis, int i, int j, int k, R e) {
  const int cj = axis == 0 ? cJX : axis == 1 ? cJY : cJZ;
  if (c.arti_eta_max > R(0.0)) {
    const int cd = axis == 0 ? cDRX : axis == 1 ? cDRY : cDRZ;
    const R J1 = AT(cj, i, j, k);
    const R dx = AT(cd, i, j, k), dy = AT(cd + 1, i, j, k), dz = AT(cd + 2, i, j, k);
    const R dr_len = sqrt(dx * dx + dy * dy + dz * dz);
    const R Jmag = fabs(J1) / dmax(dr_len, R(1.0e-30));
    R eta;
    if (c.arti_J_on <= c.arti_J_start) {
      eta = (Jmag > c.arti_J_start) ? c.arti_eta_max : R(0.0);
    } else {
      R q = (Jmag - c.arti_J_start) / (c.arti_J_on - c.arti_J_start);
      q = dmax(R(0.0), dmin(R(1.0), q));
      const R S = q * q * (R(3.0) - R(2.0) * q);
      eta = c.arti_eta_max * S;
    }
    e += eta * J1;
  }
  if (c.local_arti) e += AT(cLEX + axis, i, j, k) * AT(cj, i, j, k);
  return e;
}

// AssembleEdgeEMF_FromFaceE_Ideal_ (Ideal.cpp:138-372) + AddAmbipolarEdgeEMF_
// (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ambipo.cpp:3-143) on the owned edges.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_edge_emf(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const ConstsT<R> &c = consts_of<R>(S);
    const int i = it.i, j = it.j, k = it.k;
    const R Cuct = R(0.5);
    const R pc = (c.rho_ref * c.U_ref) / (c.q_e * c.L_ref * c.B_ref * c.n_ref);
    if (i < B.n0) {
      const R Ec = R(0.25) * (AT(cEFY, i, j, k) + AT(cEFY, i, j, k - 1) + AT(cEFZ, i, j, k) + AT(cEFZ, i, j - 1, k));
      const R ae = max_abs_u4(B, 1, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
      const R az = max_abs_u4(B, 2, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
      const R d1 = AT(cBZ, i, j, k) - AT(cBZ, i, j - 1, k);
      const R d2 = AT(cBY, i, j, k) - AT(cBY, i, j, k - 1);
      R e = Ec + Cuct * (R(0.5) * ae * d1 - R(0.5) * az * d2);
      if (c.ambipolar) {
        const R p0 = AT(cPEN, i, j, k), p1 = AT(cPEN, i + 1, j, k);
        R rH = R(0.0), rN = R(0.0);
        for (int dj = -1; dj <= 0; ++dj)
          for (int dk = -1; dk <= 0; ++dk) {
            rH += AT(cUH, i, j + dj, k + dk);
            rN += AT(cUN, i, j + dj, k + dk);
          }
        e -= pc * (p1 - p0) / num_limiter(c, R(0.25) * rH, R(0.25) * rN).ne_eff;
      }
      AT(cEX, i, j, k) = add_artificial(B, c, 0, i, j, k, e);
    }
    if (j < B.n1) {
      const R Ec = R(0.25) * (AT(cEFX + 1, i, j, k) + AT(cEFX + 1, i, j, k - 1) + AT(cEFZ + 1, i, j, k) +
                                AT(cEFZ + 1, i - 1, j, k));
      const R az = max_abs_u4(B, 2, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
      const R ax = max_abs_u4(B, 0, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
      const R d1 = AT(cBX, i, j, k) - AT(cBX, i, j, k - 1);
      const R d2 = AT(cBZ, i, j, k) - AT(cBZ, i - 1, j, k);
      R e = Ec + Cuct * (R(0.5) * az * d1 - R(0.5) * ax * d2);
      if (c.ambipolar) {
        const R p0 = AT(cPEN, i, j, k), p1 = AT(cPEN, i, j + 1, k);
        R rH = R(0.0), rN = R(0.0);
        for (int di = -1; di <= 0; ++di)
          for (int dk = -1; dk <= 0; ++dk) {
            rH += AT(cUH, i + di, j, k + dk);
            rN += AT(cUN, i + di, j, k + dk);
          }
        e -= pc * (p1 - p0) / num_limiter(c, R(0.25) * rH, R(0.25) * rN).ne_eff;
      }
      AT(cEY, i, j, k) = add_artificial(B, c, 1, i, j, k, e);
    }
    if (k < B.n2) {
      const R Ec = R(0.25) * (AT(cEFX + 2, i, j, k) + AT(cEFX + 2, i, j - 1, k) + AT(cEFY + 2, i, j, k) +
                                AT(cEFY + 2, i - 1, j, k));
      const R ax = max_abs_u4(B, 0, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
      const R ae = max_abs_u4(B, 1, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
      const R d1 = AT(cBY, i, j, k) - AT(cBY, i - 1, j, k);
      const R d2 = AT(cBX, i, j, k) - AT(cBX, i, j - 1, k);
      R e = Ec + Cuct * (R(0.5) * ax * d1 - R(0.5) * ae * d2);
      if (c.ambipolar) {
        const R p0 = AT(cPEN, i, j, k), p1 = AT(cPEN, i, j, k + 1);
        R rH = R(0.0), rN = R(0.0);
        for (int di = -1; di <= 0; ++di)
          for (int dj = -1; dj <= 0; ++dj) {
            rH += AT(cUH, i + di, j + dj, k);
            rN += AT(cUN, i + di, j + dj, k);
          }
        e -= pc * (p1 - p0) / num_limiter(c, R(0.25) * rH, R(0.25) * rN).ne_eff;
      }
      AT(cEZ, i, j, k) = add_artificial(B, c, 2, i, j, k, e);
    }
  });
}

// ------------------------------------------------------------------ Hall EMF
// BuildHallFaceEMF_Rusanov_diff_ steps 2-4 (Hall.cpp:148-400).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_hall_edge(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const R Cwh = R(0.1);
    if (i < B.n0) {
      R Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = R(0.25) * (AT(cEHC + q, i, j - 1, k - 1) + AT(cEHC + q, i, j - 1, k) + AT(cEHC + q, i, j, k - 1) +
                        AT(cEHC + q, i, j, k));
      const R Ecen = Ec[0] * AT(cDRX, i, j, k) + Ec[1] * AT(cDRX + 1, i, j, k) + Ec[2] * AT(cDRX + 2, i, j, k);
      const R be =
          dmax(dmax(AT(cHB, i, j - 1, k - 1), AT(cHB, i, j - 1, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
      const R ihe = AT(cIHX, i, j, k), ihz = AT(cIHX + 1, i, j, k);
      const R mue = Cwh * be * ihe * ihe;
      const R muz = Cwh * be * ihz * ihz;
      const R d1 = AT(cBZ, i, j, k) - AT(cBZ, i, j - 1, k);
      const R d2 = AT(cBY, i, j, k) - AT(cBY, i, j, k - 1);
      AT(cHX, i, j, k) = AT(cTPX, i, j, k) * (Ecen + R(0.5) * mue * d1 - R(0.5) * muz * d2);
    }
    if (j < B.n1) {
      R Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = R(0.25) * (AT(cEHC + q, i - 1, j, k - 1) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j, k - 1) +
                        AT(cEHC + q, i, j, k));
      const R Ecen = Ec[0] * AT(cDRY, i, j, k) + Ec[1] * AT(cDRY + 1, i, j, k) + Ec[2] * AT(cDRY + 2, i, j, k);
      const R be =
          dmax(dmax(AT(cHB, i - 1, j, k - 1), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j, k - 1), AT(cHB, i, j, k)));
      const R ihz = AT(cIHY, i, j, k), ihx = AT(cIHY + 1, i, j, k);
      const R muz = Cwh * be * ihz * ihz;
      const R mux = Cwh * be * ihx * ihx;
      const R d1 = AT(cBX, i, j, k) - AT(cBX, i, j, k - 1);
      const R d2 = AT(cBZ, i, j, k) - AT(cBZ, i - 1, j, k);
      AT(cHY, i, j, k) = AT(cTPY, i, j, k) * (Ecen + R(0.5) * muz * d1 - R(0.5) * mux * d2);
    }
    if (k < B.n2) {
      R Ec[3];
      for (int q = 0; q < 3; ++q)
        Ec[q] = R(0.25) * (AT(cEHC + q, i - 1, j - 1, k) + AT(cEHC + q, i - 1, j, k) + AT(cEHC + q, i, j - 1, k) +
                        AT(cEHC + q, i, j, k));
      const R Ecen = Ec[0] * AT(cDRZ, i, j, k) + Ec[1] * AT(cDRZ + 1, i, j, k) + Ec[2] * AT(cDRZ + 2, i, j, k);
      const R be =
          dmax(dmax(AT(cHB, i - 1, j - 1, k), AT(cHB, i - 1, j, k)), dmax(AT(cHB, i, j - 1, k), AT(cHB, i, j, k)));
      const R ihx = AT(cIHZ, i, j, k), ihe = AT(cIHZ + 1, i, j, k);
      const R mux = Cwh * be * ihx * ihx;
      const R mue = Cwh * be * ihe * ihe;
      const R d1 = AT(cBY, i, j, k) - AT(cBY, i - 1, j, k);
      const R d2 = AT(cBX, i, j, k) - AT(cBX, i, j - 1, k);
      AT(cHZ, i, j, k) = AT(cTPZ, i, j, k) * (Ecen + R(0.5) * mux * d1 - R(0.5) * mue * d2);
    }
  });
}

// E += Ehall on owned edges (Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:135-147).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_add_hall(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    if (it.i < B.n0) B.c(cEX)[o] += B.c(cHX)[o];
    if (it.j < B.n1) B.c(cEY)[o] += B.c(cHY)[o];
    if (it.k < B.n2) B.c(cEZ)[o] += B.c(cHZ)[o];
  });
}

// ------------------------------------------------------------------ fluid update
// Rusanov face flux of Scheme_U_ (Z4_Mercury/src/physics/MercurySolver_FluidRHS.cpp:36-104)
// from the two cells' staged quantities (rho, u, v, w, p and
// the per-cell terms re = p / (g - 1) + rho |u|^2 / 2, c = sqrt(g p / rho),
// which Scheme_U_ evaluates per face with the same operations on the same
// cell values, so staging them once per cell keeps the result bit for bit).
template <class R>
__device__ __forceinline__ void rusanov_staged(const R *L, const R *Rr, R k1, R k2, R k3, R sk, R out[5]) {
  const R rhoL = L[0], uL = L[1], vL = L[2], wL = L[3], pL = L[4], reL = L[5], cL = L[6];
  const R rhoR = Rr[0], uR = Rr[1], vR = Rr[2], wR = Rr[3], pR = Rr[4], reR = Rr[5], cR = Rr[6];
  const R uvwL = k1 * uL + k2 * vL + k3 * wL, uvwR = k1 * uR + k2 * vR + k3 * wR;
  const R rad = dmax(fabs(uvwL) + cL * sk, fabs(uvwR) + cR * sk);
  out[0] = R(0.5) * (rhoL * uvwL + rhoR * uvwR) - R(0.5) * rad * (rhoR - rhoL);
  out[1] = R(0.5) * ((rhoL * uvwL * uL + k1 * pL) + (rhoR * uvwR * uR + k1 * pR)) - R(0.5) * rad * (rhoR * uR - rhoL * uL);
  out[2] = R(0.5) * ((rhoL * uvwL * vL + k2 * pL) + (rhoR * uvwR * vR + k2 * pR)) - R(0.5) * rad * (rhoR * vR - rhoL * vL);
  out[3] = R(0.5) * ((rhoL * uvwL * wL + k3 * pL) + (rhoR * uvwR * wR + k3 * pR)) - R(0.5) * rad * (rhoR * wR - rhoL * wL);
  out[4] = R(0.5) * (uvwL * (reL + pL) + uvwR * (reR + pR)) - R(0.5) * rad * (reR - reL);
}

// A tile's faces per direction and in all (variant V).
template <int VT>
struct TileFaces {
  static constexpr FluidTile T = fluid_tile(VT);
  static constexpr int n0 = (T.i + 1) * T.j * T.k, n1 = T.i * (T.j + 1) * T.k, n2 = T.i * T.j * (T.k + 1);
  static constexpr int all = n0 + n1 + n2;
};

// Shared memory of the fluid kernel's tile (variant VT): the staged
// quantities of the tile's cells and their face neighbours (7 values per cell
// of the tile padded by one layer) and the tile's face fluxes (5 per face).
// The TMA-staged variant instead holds two stages of its box (5 components
// each), re and c over the box, the face fluxes, and 128 bytes to align the
// stages to 128 bytes.
template <class R, int VT>
struct FluidSmem {
  static constexpr FluidTile T = fluid_tile(VT);
  static constexpr int PK = T.k + 2, PJ = T.j + 2, PI = T.i + 2, cells = PK * PJ * PI;
  static constexpr int BV = tma_box_k(sizeof(R)) * kTmaBoxJI * kTmaBoxJI;  // elements of one component's box
  static constexpr size_t bytes =
      fluid_tma(VT) ? 128 + sizeof(R) * (size_t)(2 * 5 * BV + 2 * BV + 5 * TileFaces<VT>::all)
                    : sizeof(R) * (size_t)(7 * cells + 5 * TileFaces<VT>::all);
  static_assert(!fluid_tma(VT) || (T.k == 16 && T.j == 4 && T.i == 4), "the staged box assumes a 16 x 4 x 4 tile");
  static_assert((BV * sizeof(R)) % 128 == 0, "stages stay 128-byte aligned");
};

// ZeroRHS_ + Scheme_U_ + AddSourceToRHS_Fluid (FluidRHS.cpp:206-527) +
// ApplyUpdate_Euler_ (Z4_Mercury/src/physics/MercurySolver_Advance.cpp:73-147)
// for one tile of owned cells and one ion species; the state goes to the
// other buffer.  Per direction, the tile's face fluxes are computed once into
// shared memory (a face's flux has the same inputs and operation order for
// both cells that share it), then every cell accumulates
// r[m] -= (F+ - F-) / J, the per-component order of Scheme_U_'s divergence.
// Minimum resident CTAs per SM asked of the compiler for the primitive pass
// (caps registers at 65536 / (256 * n)); the fluid kernel's is its tile variant's.
#ifndef MHD_MIN_CTAS_PV
#define MHD_MIN_CTAS_PV 4
#endif
template <class R, int VT>
__global__ void __launch_bounds__(fluid_threads(VT), (sizeof(R) == 8 && fluid_tma(VT)) ? 2 : fluid_tile(VT).min_ctas)
    k_fluid(Dir D) {
  constexpr FluidTile T = fluid_tile(VT);
  constexpr int kNF0 = TileFaces<VT>::n0, kNF1 = TileFaces<VT>::n1, kTileFaces = TileFaces<VT>::all;
  constexpr int kTileK = T.k, kTileJ = T.j;
  constexpr int PK = FluidSmem<R, VT>::PK, PJ = FluidSmem<R, VT>::PJ, NP = FluidSmem<R, VT>::cells;
  constexpr bool kTma = fluid_tma(VT);
  constexpr int W = tma_box_k(sizeof(R)), BV = FluidSmem<R, VT>::BV;
  extern __shared__ __align__(16) unsigned char fluid_smem[];
  unsigned char *sbase = fluid_smem;
  if constexpr (kTma) sbase += (128 - (smem_u32(fluid_smem) & 127)) & 127;
  // the staged variant: [2 stages][5][BV] | RC [2][BV] (re, c) | F
  R *stage = reinterpret_cast<R *>(sbase);
  R(*RC)[BV] = reinterpret_cast<R(*)[BV]>(sbase + sizeof(R) * 10 * BV);
  R(*C)[NP] = reinterpret_cast<R(*)[NP]>(sbase);  // [7][NP]
  R(*F)[kTileFaces] =
      reinterpret_cast<R(*)[kTileFaces]>(sbase + sizeof(R) * (kTma ? 12 * BV : 7 * NP));  // [5][faces]
  __shared__ uint64_t bars[4];
  auto cta_sync = [] {
    if constexpr (kTma) compute_bar();
    else __syncthreads();
  };
  auto body = [&](const DevSolve &S, const V<R> &B, const Item &it, const R *box) {
    const ConstsT<R> &c = consts_of<R>(S);
    const R dt = __longlong_as_double((long long)D.state[it.s].dt_bits);
    // the reference aborts; k_flip records the status (and a solve with a
    // non-finite cell is not advanced)
    const bool dt_ok = (dt >= R(1e-7)) && isfinite(dt) && !D.state[it.s].nonfinite;
    const int i = it.i, j = it.j, k = it.k, s = it.species;
    const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
    const R g = c.gamma;
    const int tid = threadIdx.x;
    const int li = tid / (kTileK * kTileJ), lj = (tid / kTileK) % kTileJ, lk = tid % kTileK;
    R r[5] = {R(0.0), R(0.0), R(0.0), R(0.0), R(0.0)};
    // The cell values the source terms and the update read: cen(q) loads
    // value q; in FP32 all of them are loaded before the flux passes into
    // registers (their latency hides behind the passes), in FP64 at their use.
    auto cen = [&](int q) -> R {
      switch (q) {
        case 0: case 1: case 2: return AT(cUP + q, i, j, k);
        case 3: case 4: case 5: return AT(cBC + (q - 3), i, j, k);
        case 6: case 7: case 8: return AT(cJC + (q - 6), i, j, k);
        case 9: return AT(cUH, i, j, k);
        case 10: return AT(cUN, i, j, k);
        case 11: return AT(pv0 + 4, i, j, k);
        case 12: case 13: case 14: case 15: case 16: return AT(u0 + (q - 12), i, j, k);
        case 17: return AT(cPHOTO, i, j, k);
        case 18: case 19: case 20: return AT(cCX + (q - 18), i, j, k);
        default: return AT(pv0 + (q - 21), i, j, k);  // 21..23: u, v, w
      }
    };
    constexpr int kCen = sizeof(R) == 4 ? 24 : 1;
    R cvals[kCen];
    if constexpr (sizeof(R) == 4) {
      if (it.in && dt_ok) {
#pragma unroll
        for (int q = 0; q < 24; ++q) cvals[q] = cen(q);
      }
    }
    auto CV = [&](int q) -> R {
      if constexpr (sizeof(R) == 4) return cvals[q];
      else return cen(q);
    };
    // 1/J of this cell (the same value every direction divides by)
    R invJ = R(0.0);
    if (it.in && dt_ok) {
      if constexpr (sizeof(R) == 4) invJ = AT(cFM + 9, i, j, k);  // R(1) / R(Jac), from k_face_normals
      else invJ = R(1.0) / R(ATM(cJAC, i, j, k));
    }
    // Stage the cells the tile's faces read (the tile and one layer beyond
    // each of its six sides, inside the owned range widened by one): rho,
    // u, v, w, p and the per-cell terms re and c.
    // the staged variant: the box of this item holds the cells; re and c of
    // the cells the faces read go to RC (box indexing, k shifted by koff)
    const int koff = kTma ? (it.o[2] + B.G - 1) & (16 / (int)sizeof(R) - 1) : 0;
#pragma unroll 1
    for (int q = tid; q < NP; q += kTileThreads) {
      const int ck = q % PK, cj = (q / PK) % PJ, ci = q / (PK * PJ);
      const int x0 = it.o[0] - 1 + ci, x1 = it.o[1] - 1 + cj, x2 = it.o[2] - 1 + ck;
      const int out = (ci == 0 || ci == T.i + 1) + (cj == 0 || cj == T.j + 1) + (ck == 0 || ck == T.k + 1);
      if (!dt_ok || out > 1 || x0 < it.lo[0] - 1 || x0 > it.hi[0] || x1 < it.lo[1] - 1 || x1 > it.hi[1] ||
          x2 < it.lo[2] - 1 || x2 > it.hi[2])
        continue;
      if constexpr (kTma) {
        const int e = (ci * kTmaBoxJI + cj) * W + ck + koff;
        const R rho = box[e], u = box[BV + e], v = box[2 * BV + e], w = box[3 * BV + e], p = box[4 * BV + e];
        RC[0][e] = p / (g - R(1.0)) + R(0.5) * rho * (u * u + v * v + w * w);
        RC[1][e] = sqrt(dmax(R(0.0), g * p / dmax(rho, R(1e-30))));
        continue;
      }
      const R rho = AT(u0, x0, x1, x2), u = AT(pv0, x0, x1, x2), v = AT(pv0 + 1, x0, x1, x2),
              w = AT(pv0 + 2, x0, x1, x2), p = AT(pv0 + 3, x0, x1, x2);
      C[0][q] = rho;
      C[1][q] = u;
      C[2][q] = v;
      C[3][q] = w;
      C[4][q] = p;
      C[5][q] = p / (g - R(1.0)) + R(0.5) * rho * (u * u + v * v + w * w);
      C[6][q] = sqrt(dmax(R(0.0), g * p / dmax(rho, R(1e-30))));
    }
    cta_sync();
    // one face of direction dir (index f among that direction's faces, the
    // slot gf of the tile's face array): the direction is a compile-time
    // constant in each of the three instantiations, so the face grid's
    // extents divide as constants
    auto face = [&](auto dirc, int f, int gf) {
      constexpr int dir = decltype(dirc)::value;
      constexpr int ej = kTileJ + (dir == 1), ek = kTileK + (dir == 2);
      // the face's JD: FP32 reads the real-typed copy (k_face_normals), FP64
      // the metric itself (the same values; faster there)
      constexpr int cm = sizeof(R) == 4 ? cFM + 3 * dir : dir == 0 ? cJDX : dir == 1 ? cJDY : cJDZ;
      constexpr int cn = dir == 0 ? cFNX : dir == 1 ? cFNY : cFNZ;
      const int fk = f % ek, fj = (f / ek) % ej, fi = f / (ek * ej);
      const int x[3] = {it.o[0] + fi, it.o[1] + fj, it.o[2] + fk};
      bool need = dt_ok;
#pragma unroll
      for (int a = 0; a < 3; ++a) need = need && x[a] >= it.lo[a] && x[a] < it.hi[a] + (a == dir);
      if (!need) return;
      R k1, k2, k3;
      if constexpr (sizeof(R) == 4) {
        k1 = AT(cm, x[0], x[1], x[2]);
        k2 = AT(cm + 1, x[0], x[1], x[2]);
        k3 = AT(cm + 2, x[0], x[1], x[2]);
      } else {
        k1 = ATM(cm, x[0], x[1], x[2]);
        k2 = ATM(cm + 1, x[0], x[1], x[2]);
        k3 = ATM(cm + 2, x[0], x[1], x[2]);
      }
      // the face's right cell is (fi, fj, fk) of the tile, its left one step back along dir
      R Lv[7], Rv[7];
      if constexpr (kTma) {
        const int er = ((fi + 1) * kTmaBoxJI + (fj + 1)) * W + (fk + 1) + koff;
        const int el = er - (dir == 0 ? kTmaBoxJI * W : dir == 1 ? W : 1);
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          Lv[m] = box[m * BV + el];
          Rv[m] = box[m * BV + er];
        }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          Lv[5 + m] = RC[m][el];
          Rv[5 + m] = RC[m][er];
        }
      } else {
        const int qr = ((fi + 1) * PJ + (fj + 1)) * PK + (fk + 1);
        const int ql = qr - (dir == 0 ? PJ * PK : dir == 1 ? PK : 1);
#pragma unroll
        for (int m = 0; m < 7; ++m) {
          Lv[m] = C[m][ql];
          Rv[m] = C[m][qr];
        }
      }
      R Fl[5];
      rusanov_staged(Lv, Rv, k1, k2, k3, AT(cn + 3, x[0], x[1], x[2]), Fl);
#pragma unroll
      for (int m = 0; m < 5; ++m) F[m][gf] = Fl[m];
    };
    // The tile's face fluxes of all three directions in one pass, dealt
    // round-robin over the threads (912 faces of a 16 x 4 x 4 tile take four
    // rounds of 256; a warp straddles a direction change at most twice), then
    // every cell takes its six faces' differences direction by direction, in
    // Scheme_U_'s order.
#pragma unroll 1
    for (int gf = tid; gf < kTileFaces; gf += kTileThreads) {
      if (gf < kNF0) face(std::integral_constant<int, 0>{}, gf, gf);
      else if (gf < kNF0 + kNF1) face(std::integral_constant<int, 1>{}, gf - kNF0, gf);
      else face(std::integral_constant<int, 2>{}, gf - kNF0 - kNF1, gf);
    }
    cta_sync();
    if constexpr (kTma) mbar_arrive(&bars[2 + (box == stage ? 0 : 1)]);  // this stage's box is no longer read
    if (it.in && dt_ok) {
      auto take = [&](auto dirc) {
        constexpr int dir = decltype(dirc)::value;
        constexpr int base = dir == 0 ? 0 : dir == 1 ? kNF0 : kNF0 + kNF1;
        constexpr int ej = kTileJ + (dir == 1), ek = kTileK + (dir == 2);
        const int fm = base + (li * ej + lj) * ek + lk;
        const int fp = fm + (dir == 0 ? ej * ek : dir == 1 ? ek : 1);
#pragma unroll
        for (int m = 0; m < 5; ++m) r[m] -= (F[m][fp] - F[m][fm]) * invJ;
      };
      take(std::integral_constant<int, 0>{});
      take(std::integral_constant<int, 1>{});
      take(std::integral_constant<int, 2>{});
    }
    cta_sync();  // F is rewritten by the next tile
    if (!it.in || !dt_ok) return;
    // sources (FluidRHS.cpp:206-527)
    const R Tn0 = R(1000.0), sk1 = R(5.0e-5), sk2 = R(1.0e-5);
    const R a4 = (c.L_ref / c.U_ref);
    const R a5 = (R(3.0) * c.L_ref * c.k_Boltz * c.n_ref) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref);
    const R upx = CV(0), upy = CV(1), upz = CV(2);
    const R Bx = CV(3), By = CV(4), Bz = CV(5);
    const R Jx = CV(6), Jy = CV(7), Jz = CV(8);
    const R sjbx = Jy * Bz - Jz * By, sjby = Jz * Bx - Jx * Bz, sjbz = Jx * By - Jy * Bx;
    const Num<R> num = num_limiter(c, CV(9), CV(10));
    R dpex = R(0.0), dpey = R(0.0), dpez = R(0.0);
    if (c.ambipolar) {  // grad p_e term, once per cell (k_face_emf)
      dpex = AT(cDPE, i, j, k);
      dpey = AT(cDPE + 1, i, j, k);
      dpez = AT(cDPE + 2, i, j, k);
    }
    const R x = CV(18), y = CV(19), z = CV(20);
    const R rho_cyl = sqrt(y * y + z * z);
    const R vst = (x < R(0.0) && rho_cyl < R(1.0)) ? sk2 : sk1;
    const R nS = s ? num.nNa : num.nH;
    const R chi = s ? num.wNa : num.wH;
    const R rho = dmax(CV(12), R(0.0));
    const R u = CV(21), v = CV(22), w = CV(23);
    const R u2 = u * u + v * v + w * w;
    const R subx = (v - upy) * Bz - (w - upz) * By;
    const R suby = (w - upz) * Bx - (u - upx) * Bz;
    const R subz = (u - upx) * By - (v - upy) * Bx;
    const R subu = subx * u + suby * v + subz * w;
    const R sjbu = sjbx * u + sjby * v + sjbz * w;
    const R dpeu = dpex * u + dpey * v + dpez * w;
    const R Ts0 = CV(11) * c.T_ref;
    R b1, b2;
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
      const R a1_Na = (c.L_ref / c.U_ref) * (c.m_Na / c.rho_ref) * R(1e6);
      const R a6 = (R(1.0e6) * c.L_ref * c.k_Boltz) / (c.rho_ref * c.U_ref * c.U_ref * c.U_ref * (c.gamma - R(1.0)));
      const R sss = CV(17);
      r[0] += a1_Na * sss;
      r[4] += a6 * sss * Tn0;
    }
    r[1] -= a4 * rho * u * vst;
    r[2] -= a4 * rho * v * vst;
    r[3] -= a4 * rho * w * vst;
    r[4] -= a4 * rho * u2 * vst;
    r[4] += a5 * nS * b1;
    r[4] += a4 * rho * u2 * b2;
    const int o = B.off(i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m) B.Un[(u0 + m) * B.total + o] = CV(12 + m) + dt * r[m];
  };
  if constexpr (kTma) {
    for_fluid_items_tma<R, fluid_kind(VT)>(D, stage, bars, body);
  } else {
    for_items<R, fluid_kind(VT)>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) { body(S, B, it, nullptr); });
  }
}

// B_face += dt * (-curl E) on the owned faces (CTOperators.cpp:6-56 with multiplier -1).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_bface(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const R dt = __longlong_as_double((long long)D.state[it.s].dt_bits);
    if (!(dt >= R(1e-7)) || !isfinite(dt) || D.state[it.s].nonfinite) return;  // k_flip records the status
    const int i = it.i, j = it.j, k = it.k;
    if (j < B.n1 && k < B.n2) {
      const R rb = -R(1.0) * ((AT(cEY, i, j, k) - AT(cEY, i, j, k + 1)) + (AT(cEZ, i, j + 1, k) - AT(cEZ, i, j, k)));
      AT(cBX, i, j, k) += dt * rb;
    }
    if (i < B.n0 && k < B.n2) {
      const R rb = -R(1.0) * ((AT(cEX, i, j, k + 1) - AT(cEX, i, j, k)) + (AT(cEZ, i, j, k) - AT(cEZ, i + 1, j, k)));
      AT(cBY, i, j, k) += dt * rb;
    }
    if (i < B.n0 && j < B.n1) {
      const R rb = -R(1.0) * ((AT(cEX, i, j, k) - AT(cEX, i, j + 1, k)) + (AT(cEY, i + 1, j, k) - AT(cEY, i, j, k)));
      AT(cBZ, i, j, k) += dt * rb;
    }
  });
}

// ------------------------------------------------------------------ derived fields
// calc_Bcell (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:3-90) on owned cells and
// CurlAdjFaceToEdge + alpha scaling of Calc_J_Edge (CTOperators.cpp:59-110,
// Z4_Mercury/src/physics/MercurySolver_Current.cpp:140-190) on owned edges.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_bcell_jedge(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    if (i < B.n0 && j < B.n1 && k < B.n2) {
      const R pt[6] = {-AT(cBX, i, j, k) - AT(cBAX, i, j, k), AT(cBX, i + 1, j, k) + AT(cBAX, i + 1, j, k),
                            -AT(cBY, i, j, k) - AT(cBAY, i, j, k), AT(cBY, i, j + 1, k) + AT(cBAY, i, j + 1, k),
                            -AT(cBZ, i, j, k) - AT(cBAZ, i, j, k), AT(cBZ, i, j, k + 1) + AT(cBAZ, i, j, k + 1)};
      const R pi_[6] = {-AT(cBX, i, j, k), AT(cBX, i + 1, j, k), -AT(cBY, i, j, k),
                             AT(cBY, i, j + 1, k), -AT(cBZ, i, j, k), AT(cBZ, i, j, k + 1)};
      R bxt = 0, byt = 0, bzt = 0, bxi = 0, byi = 0, bzi = 0;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const R wx = AT(cWB + q, i, j, k), wy = AT(cWB + 6 + q, i, j, k), wz = AT(cWB + 12 + q, i, j, k);
        bxt += wx * pt[q];
        byt += wy * pt[q];
        bzt += wz * pt[q];
        bxi += wx * pi_[q];
        byi += wy * pi_[q];
        bzi += wz * pi_[q];
      }
      const int o = B.off(i, j, k);
      B.c(cBC)[o] = bxt;
      B.c(cBC + 1)[o] = byt;
      B.c(cBC + 2)[o] = bzt;
      B.c(cBIC)[o] = bxi;
      B.c(cBIC + 1)[o] = byi;
      B.c(cBIC + 2)[o] = bzi;
    }
    if (i < B.n0) {
      const R v = ((AT(cBFY, i, j, k - 1) * AT(cBY, i, j, k - 1) - AT(cBFY, i, j, k) * AT(cBY, i, j, k)) +
                        (AT(cBFZ, i, j, k) * AT(cBZ, i, j, k) - AT(cBFZ, i, j - 1, k) * AT(cBZ, i, j - 1, k))) * R(1.0);
      AT(cJX, i, j, k) = v * AT(cALX, i, j, k);
    }
    if (j < B.n1) {
      const R v = ((AT(cBFX, i, j, k) * AT(cBX, i, j, k) - AT(cBFX, i, j, k - 1) * AT(cBX, i, j, k - 1)) +
                        (AT(cBFZ, i - 1, j, k) * AT(cBZ, i - 1, j, k) - AT(cBFZ, i, j, k) * AT(cBZ, i, j, k))) * R(1.0);
      AT(cJY, i, j, k) = v * AT(cALY, i, j, k);
    }
    if (k < B.n2) {
      const R v = ((AT(cBFX, i, j - 1, k) * AT(cBX, i, j - 1, k) - AT(cBFX, i, j, k) * AT(cBX, i, j, k)) +
                        (AT(cBFY, i, j, k) * AT(cBY, i, j, k) - AT(cBFY, i - 1, j, k) * AT(cBY, i - 1, j, k))) * R(1.0);
      AT(cJZ, i, j, k) = v * AT(cALZ, i, j, k);
    }
  });
}

// calc_Jcell (Current.cpp:203-243), owned cells.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_jcell(Dir D) {
  for_items<R, kCells>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const R s[12] = {AT(cJX, i, j, k),         AT(cJX, i, j + 1, k),     AT(cJX, i, j, k + 1),
                          AT(cJX, i, j + 1, k + 1), AT(cJY, i, j, k),         AT(cJY, i + 1, j, k),
                          AT(cJY, i, j, k + 1),     AT(cJY, i + 1, j, k + 1), AT(cJZ, i, j, k),
                          AT(cJZ, i + 1, j, k),     AT(cJZ, i, j + 1, k),     AT(cJZ, i + 1, j + 1, k)};
    R jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      jx += AT(cWJ + q, i, j, k) * s[q];
      jy += AT(cWJ + 12 + q, i, j, k) * s[q];
      jz += AT(cWJ + 24 + q, i, j, k) * s[q];
    }
    const int o = B.off(i, j, k);
    B.c(cJC)[o] = jx;
    B.c(cJC + 1)[o] = jy;
    B.c(cJC + 2)[o] = jz;
  });
}

// CFL time step of one cell and both species (Compute_Timestep,
// Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:8-141).
template <class R>
__device__ __forceinline__ R fast_cf(R cs2, R vA2, R vAn2) {
  const R term = cs2 + vA2;
  R disc = term * term - R(4.0) * cs2 * vAn2;
  if (disc < R(0.0)) disc = R(0.0);
  return sqrt(R(0.5) * (term + sqrt(disc)));
}
// One face's term of the CFL denominator.  (nx, ny, nz, An) are the face's
// precomputed a / |a| and |a| (k_face_normals: the same operations as the
// reference evaluates per face); vA2 = inver_MA2 * B2 / rho is the same for
// all faces of a cell and species.
template <class R>
__device__ __forceinline__ R face_term(const ConstsT<R> &c, R nx, R ny, R nz, R An,
                                            bool outward_plus, R ux, R uy, R uz, R Bx, R By,
                                            R Bz, R vA2, R rho, R cs2) {
  if (An <= R(0.0)) return R(0.0);
  if (!outward_plus) {
    nx = -nx;
    ny = -ny;
    nz = -nz;
  }
  const R un = ux * nx + uy * ny + uz * nz;
  const R Bn = Bx * nx + By * ny + Bz * nz;
  const R vAn2 = c.inver_MA2 * (Bn * Bn) / rho;
  return (fabs(un) + fast_cf(cs2, vA2, vAn2)) * An;
}
template <class R>
__device__ __forceinline__ R cell_dt(const V<R> &B, const ConstsT<R> &c, int i, int j, int k) {
  R dtl = R(1e100);
  const R Vol = fabs(R(LDM(cJAC, i, j, k)));
  if (!(Vol > R(0.0))) return dtl;
  const R Bx = LD(cBC, i, j, k), By = LD(cBC + 1, i, j, k), Bz = LD(cBC + 2, i, j, k);
  const R B2 = Bx * Bx + By * By + Bz * Bz;
  if constexpr (sizeof(R) == 4) {
    // FP32: the six faces' unit normals and |a| and both species' states are
    // loaded once, up front (xi-, xi+, eta-, eta+, zeta-, zeta+: the
    // reference's summation order)
    R fn[6][4];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int a = f >> 1, up = f & 1;
      const int cn = a == 0 ? cFNX : a == 1 ? cFNY : cFNZ;
      int fi = i, fj = j, fk = k;
      shift1(a, fi, fj, fk, up);
#pragma unroll
      for (int q = 0; q < 4; ++q) fn[f][q] = LD(cn + q, fi, fj, fk);
    }
    R Us[2][5];
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int q = 0; q < 5; ++q) Us[s][q] = LD((s ? cUN : cUH) + q, i, j, k);
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      const R rho = dmax(Us[s][0], R(1e-2));
      const R ux = Us[s][1] / rho, uy = Us[s][2] / rho, uz = Us[s][3] / rho;
      const R E = Us[s][4];
      const R ke = R(0.5) * rho * (ux * ux + uy * uy + uz * uz);
      const R pr = (c.gamma - R(1.0)) * (E - ke);
      const R cs2 = c.gamma * pr / rho;
      const R vA2 = c.inver_MA2 * B2 / rho;
      R den = R(0.0);
#pragma unroll
      for (int f = 0; f < 6; ++f)
        den += face_term(c, fn[f][0], fn[f][1], fn[f][2], fn[f][3], (f & 1) != 0, ux, uy, uz, Bx, By, Bz, vA2, rho, cs2);
      if (den > R(0.0)) dtl = dmin(dtl, c.CFL * Vol / den);
    }
  } else {
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      const int u0 = s ? cUN : cUH;
      const R rho = dmax(LD(u0, i, j, k), R(1e-2));
      const R ux = LD(u0 + 1, i, j, k) / rho, uy = LD(u0 + 2, i, j, k) / rho, uz = LD(u0 + 3, i, j, k) / rho;
      const R E = LD(u0 + 4, i, j, k);
      const R ke = R(0.5) * rho * (ux * ux + uy * uy + uz * uz);
      const R pr = (c.gamma - R(1.0)) * (E - ke);
      const R cs2 = c.gamma * pr / rho;
      const R vA2 = c.inver_MA2 * B2 / rho;
      R den = R(0.0);
      // faces xi-, xi+, eta-, eta+, zeta-, zeta+ (the reference's summation order)
#pragma unroll 1
      for (int f = 0; f < 6; ++f) {
        const int a = f >> 1, up = f & 1;
        const int cn = a == 0 ? cFNX : a == 1 ? cFNY : cFNZ;
        int fi = i, fj = j, fk = k;
        shift1(a, fi, fj, fk, up);
        den += face_term(c, LD(cn, fi, fj, fk), LD(cn + 1, fi, fj, fk), LD(cn + 2, fi, fj, fk), LD(cn + 3, fi, fj, fk),
                         up != 0, ux, uy, uz, Bx, By, Bz, vA2, rho, cs2);
      }
      if (den > R(0.0)) dtl = dmin(dtl, c.CFL * Vol / den);
    }
  }
  return dtl;
}

// calc_divB (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:186-193) on the owned cells,
// and max |div B| per solve (atomicMax on the bits of the non-negative double).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_div_b(Dir D) {
  for_items<R, kCells>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    R v = R(0.0);
    if (it.in) {
      const int i = it.i, j = it.j, k = it.k;
      v = (AT(cBX, i + 1, j, k) - AT(cBX, i, j, k) + AT(cBY, i, j + 1, k) - AT(cBY, i, j, k) + AT(cBZ, i, j, k + 1) -
           AT(cBZ, i, j, k)) /
          R(ATM(cJAC, i, j, k));
      AT(cDIVB, i, j, k) = v;
    }
    double a = fabs((double)v);
    if (!(a == a)) a = __longlong_as_double(0x7ff0000000000000LL);  // NaN counts as infinite
    for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&D.state[it.s].divb_bits, (unsigned long long)__double_as_longlong(a));
  });
}

// ------------------------------------------------------------------ implicit resistive substep
// SolveImplicitResistiveDiffusion_ (Z4_Mercury/src/implicit/Mercury_ImplicitResistive.cpp:475-575):
// (I + dt eta alpha C^T beta C) E = eta J(B*) on the owned edges with eta > 0.
// The operator is self-adjoint in the inner product weighted by
// W = 1 / (eta alpha), so CG runs in that inner product; the edge, face and J
// fields of the explicit step are the operator's scratch (E: E_res, B: dB,
// J: dJ), with the step's own E / B / J sync and alias tables.

// Owned-range test of an edge of family a at (i, j, k).
__device__ __forceinline__ bool edge_owned(int a, int i, int j, int k, int n0, int n1, int n2) {
  return a == 0 ? (i < n0 && j <= n1 && k <= n2) : a == 1 ? (i <= n0 && j < n1 && k <= n2) : (i <= n0 && j <= n1 && k < n2);
}

// E = 1 on every edge of the owned range; the owner phase of Sync(E_res)
// run in mark mode then zeros its destinations, the non-owner aliases, so
// an edge still at 1 is its own unknown.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_seed(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) B.c(cEX + a)[o] = R(1.0);
  });
}

// W = 1 / (eta alpha) on the unknowns (owned, not a non-owner alias, eta > 0,
// alpha > 0: BuildImplicitResistiveEdgeDofMap_, Mercury_ImplicitResistive.cpp:168-226), 0 elsewhere.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_w(Dir D) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      R w = R(0.0);
      if (edge_owned(a, it.i, it.j, it.k, B.n0, B.n1, B.n2) && B.c(cEX + a)[o] != R(0.0)) {
        const R eta = B.c(cETAR + a)[o], alpha = B.c(cALX + a)[o];
        if (eta > R(0.0) && alpha > R(0.0)) w = R(1.0) / (eta * alpha);
      }
      B.c(cRW + a)[o] = w;
    }
  });
}

// Per block of the masked solve: the largest k of an edge with W > 0 (out
// starts at -1).  The substep's work range kResK ends two layers above it:
// the faces below the unknowns' top layer read E_res one layer up, the
// current on the unknowns reads those faces.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_kmax(Dir D, int *out) {
  for_items<R, kBox>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    const int o = it.in ? B.off(it.i, it.j, it.k) : 0;
    const bool dof = it.in && (B.c(cRW)[o] > R(0.0) || B.c(cRW + 1)[o] > R(0.0) || B.c(cRW + 2)[o] > R(0.0));
    int k = dof ? it.k : -1;
    for (int of = 16; of > 0; of >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, of));
    if ((threadIdx.x & 31) == 0 && k >= 0) atomicMax(out + it.blk, k);
  });
}

// Vector operations of the CG on the unknowns (W > 0); other entries stay 0.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_vec(Dir D, int op) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      const bool dof = B.c(cRW + a)[o] > R(0.0);
      R *x = B.c(cRX + a) + o, *r = B.c(cRR + a) + o, *p = B.c(cRP + a) + o;
      switch (op) {
        case RES_INIT:  // r = b = eta J (PackImplicitJedgeToVec_, :395-418); the CG's start sets x and p
          *r = dof ? R(0.0) + B.c(cETAR + a)[o] * B.c(cJX + a)[o] : R(0.0);
          break;
        case RES_E_FROM_P: B.c(cEX + a)[o] = dof ? *p : R(0.0); break;  // UnpackVecToImplicitEres_ (:294-312)
        case RES_E_FROM_X: B.c(cEX + a)[o] = dof ? *x : R(0.0); break;
        case RES_P_FROM_X: *p = dof ? *x : R(0.0); break;
        case RES_RESID:  // r = b - q, b kept in the B* snapshot arrays (FP64 companion of a mixed solve)
          *r = dof ? B.c(cRBS + a)[o] - B.c(cRQ + a)[o] : R(0.0);
          break;
        default: break;
      }
    }
  });
}

// dB = -dt curl E on the owned faces (CurlEdgeToFace with multiplier -dt,
// Z4_Mercury/src/operators/CTOperators.cpp:6-56; MatMultImplicitResistive_, :420-445).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_db(Dir D) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const R m = R(-D.state[it.s].dt);
    const int i = it.i, j = it.j, k = it.k;
    if (j < B.n1 && k < B.n2)
      AT(cBX, i, j, k) = m * ((AT(cEY, i, j, k) - AT(cEY, i, j, k + 1)) + (AT(cEZ, i, j + 1, k) - AT(cEZ, i, j, k)));
    if (i < B.n0 && k < B.n2)
      AT(cBY, i, j, k) = m * ((AT(cEX, i, j, k + 1) - AT(cEX, i, j, k)) + (AT(cEZ, i, j, k) - AT(cEZ, i + 1, j, k)));
    if (i < B.n0 && j < B.n1)
      AT(cBZ, i, j, k) = m * ((AT(cEX, i, j, k) - AT(cEX, i, j + 1, k)) + (AT(cEY, i + 1, j, k) - AT(cEY, i, j, k)));
  });
}

// dJ = alpha CurlAdjFaceToEdge(beta dB) on the owned edges (CalcImplicitDeltaJedgeFromDeltaB_,
// Mercury_ImplicitResistive.cpp:314-393; CTOperators.cpp:59-110).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_dj(Dir D) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    if (i < B.n0) {
      const R v = ((AT(cBFY, i, j, k - 1) * AT(cBY, i, j, k - 1) - AT(cBFY, i, j, k) * AT(cBY, i, j, k)) +
                   (AT(cBFZ, i, j, k) * AT(cBZ, i, j, k) - AT(cBFZ, i, j - 1, k) * AT(cBZ, i, j - 1, k))) * R(1.0);
      AT(cJX, i, j, k) = v * AT(cALX, i, j, k);
    }
    if (j < B.n1) {
      const R v = ((AT(cBFX, i, j, k) * AT(cBX, i, j, k) - AT(cBFX, i, j, k - 1) * AT(cBX, i, j, k - 1)) +
                   (AT(cBFZ, i - 1, j, k) * AT(cBZ, i - 1, j, k) - AT(cBFZ, i, j, k) * AT(cBZ, i, j, k))) * R(1.0);
      AT(cJY, i, j, k) = v * AT(cALY, i, j, k);
    }
    if (k < B.n2) {
      const R v = ((AT(cBFX, i, j - 1, k) * AT(cBX, i, j - 1, k) - AT(cBFX, i, j, k) * AT(cBX, i, j, k)) +
                   (AT(cBFY, i, j, k) * AT(cBY, i, j, k) - AT(cBFY, i - 1, j, k) * AT(cBY, i - 1, j, k))) * R(1.0);
      AT(cJZ, i, j, k) = v * AT(cALZ, i, j, k);
    }
  });
}

// dB = 0 on every face of the block outside the owned range: the reference
// clears dB before the curl (clear_triplet, Mercury_ImplicitResistive.cpp:428),
// so Sync(dB) starts from zero ghosts; a Coupled-Solid boundary leaves them
// at zero and the halo copies of a rotated seam can read them.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_clearb(Dir D) {
  for_items<R, kFull>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int i = it.i, j = it.j, k = it.k;
    const bool ci = i >= 0 && i < B.n0, cj = j >= 0 && j < B.n1, ck = k >= 0 && k < B.n2;
    const int o = B.off(i, j, k);
    if (!(i >= 0 && i <= B.n0 && cj && ck)) B.c(cBX)[o] = R(0.0);
    if (!(ci && j >= 0 && j <= B.n1 && ck)) B.c(cBY)[o] = R(0.0);
    if (!(ci && cj && k >= 0 && k <= B.n2)) B.c(cBZ)[o] = R(0.0);
  });
}

// q = A p = E_res - eta dJ on the unknowns (MatMultImplicitResistive_, :446-468).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_q(Dir D) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      const bool dof = B.c(cRW + a)[o] > R(0.0);
      B.c(cRQ + a)[o] = dof ? B.c(cEX + a)[o] - B.c(cETAR + a)[o] * B.c(cJX + a)[o] : R(0.0);
    }
  });
}

// Dot products of r on the unknowns of the masked solve: (sum W r r, sum r r).  Per-CTA partial sums in a fixed order (deterministic).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_dot(Dir D, double *partial) {
  __shared__ double sh[2][kTileThreads / 32];
  double acc0 = 0.0, acc1 = 0.0;
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      const double w = (double)B.c(cRW + a)[o];
      if (!(w > 0.0)) continue;
      const double r = (double)B.c(cRR + a)[o];
      acc0 += w * r * r;
      acc1 += r * r;
    }
  });
  for (int of = 16; of > 0; of >>= 1) {
    acc0 += __shfl_xor_sync(0xffffffffu, acc0, of);
    acc1 += __shfl_xor_sync(0xffffffffu, acc1, of);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = acc0;
    sh[1][threadIdx.x >> 5] = acc1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < kTileThreads / 32; ++w) {
      s0 += sh[0][w];
      s1 += sh[1][w];
    }
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
}
__global__ void k_res_sum(const double *partial, int n, double *result) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int q = 0; q < n; ++q) {
      s0 += partial[2 * q];
      s1 += partial[2 * q + 1];
    }
    result[0] = s0;
    result[1] = s1;
  }
}

// One step of the CG iteration of every masked solve with its dot products:
// each warp writes its sums over each tile to its own slot of tpart (2
// doubles per warp and tile), k_res_cg_sum then adds a solve's slots in a
// fixed order (deterministic) and updates its scalars.  CG_PQ first clears
// the loop condition, so a loop whose stop test did not run ends.  Both
// kernels write the condition of the loop graph they belong to
// (build_cg_graph) only when launched inside it (in_graph; the host-driven
// loop of res_cg_batch reads the states instead).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_cg(Dir D, int op, double *tpart, const ResCG *cg,
                                                         cudaGraphConditionalHandle handle, int in_graph) {
  if (in_graph && op == CG_PQ && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
  double acc0 = 0.0, acc1 = 0.0;
  for_items<R, kResK>(
      D,
      [&](const DevSolve &S, const V<R> &B, const Item &it) {
        if (!it.in) return;
        const R alpha = R(cg[it.s].alpha);
        const int o = B.off(it.i, it.j, it.k);
        for (int a = 0; a < 3; ++a) {
          const R wr = B.c(cRW + a)[o];
          const bool dof = wr > R(0.0);
          const double w = (double)wr;
          R *x = B.c(cRX + a) + o, *r = B.c(cRR + a) + o, *p = B.c(cRP + a) + o, *q = B.c(cRQ + a) + o;
          if (op == CG_INIT) {  // x = 0, p = r (the start), E_res = p
            const R pv = dof ? *r : R(0.0);
            *x = R(0.0);
            *p = pv;
            B.c(cEX + a)[o] = pv;
            if (w > 0.0) {
              const double rv = (double)*r;
              acc0 += w * rv * rv;
              acc1 += rv * rv;
            }
          } else if (op == CG_PQ) {
            const R qv = dof ? B.c(cEX + a)[o] - B.c(cETAR + a)[o] * B.c(cJX + a)[o] : R(0.0);
            *q = qv;
            if (w > 0.0) acc0 += w * (double)*p * (double)qv;
          } else {
            if (dof) {
              *x += alpha * *p;
              *r -= alpha * *q;
            }
            if (w > 0.0) {
              const double rv = (double)*r;
              acc0 += w * rv * rv;
              acc1 += rv * rv;
            }
          }
        }
      },
      [&](int w) {  // the warp's sums over this tile
        for (int of = 16; of > 0; of >>= 1) {
          acc0 += __shfl_xor_sync(0xffffffffu, acc0, of);
          acc1 += __shfl_xor_sync(0xffffffffu, acc1, of);
        }
        if ((threadIdx.x & 31) == 0) {
          const int64_t slot = (int64_t)w * kWarpsPerTile + (threadIdx.x >> 5);
          tpart[2 * slot] = acc0;
          tpart[2 * slot + 1] = acc1;
        }
        acc0 = acc1 = 0.0;
      });
}

// The per-solve end of a k_res_cg step: kCgChunks CTAs per slot, CTA c of
// solve s adds chunk c of the solve's tile partials (threads stride over it,
// then a fixed tree); the last of them (atomic ticket per solve) adds the
// chunks in order and updates the solve's state; a solve whose loop ends
// (converged, max_it, breakdown) leaves the mask, so the following kernels
// skip it.  The last slot to report (atomic ticket) sets the loop condition
// after CG_INIT and CG_RR: some solve still running.  Every sum has fixed
// bounds and order (deterministic, and the same for a solve alone or in a
// batch).
__global__ void __launch_bounds__(kTileThreads) k_res_cg_sum(Dir D, int op, const double *tpart, ResCG *cg,
                                                             ResCtl *ctl, double *chunks, unsigned int *sarr,
                                                             cudaGraphConditionalHandle handle, int in_graph) {
  __shared__ double sh[2][kWarpsPerTile];
  const int s = blockIdx.x / kCgChunks, c = blockIdx.x % kCgChunks;
  const bool act = s < D.nsolves && solve_active(D, s);  // the whole CTA agrees
  bool last_of_solve = false;
  if (act) {
    const int *sp = D.solve_tile_prefix[kResK];
    const int64_t a0 = (int64_t)sp[s] * kWarpsPerTile, n = (int64_t)(sp[s + 1] - sp[s]) * kWarpsPerTile;
    const int64_t len = (n + kCgChunks - 1) / kCgChunks;
    const int64_t a = a0 + min(n, (int64_t)c * len), e = a0 + min(n, (int64_t)(c + 1) * len);
    double u0 = 0.0, u1 = 0.0;
    for (int64_t q = a + threadIdx.x; q < e; q += kTileThreads) {
      u0 += tpart[2 * q];
      u1 += tpart[2 * q + 1];
    }
    for (int of = 16; of > 0; of >>= 1) {
      u0 += __shfl_xor_sync(0xffffffffu, u0, of);
      u1 += __shfl_xor_sync(0xffffffffu, u1, of);
    }
    if ((threadIdx.x & 31) == 0) {
      sh[0][threadIdx.x >> 5] = u0;
      sh[1][threadIdx.x >> 5] = u1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t0 = 0.0, t1 = 0.0;
      for (int w = 0; w < kWarpsPerTile; ++w) {
        t0 += sh[0][w];
        t1 += sh[1][w];
      }
      chunks[2 * (s * kCgChunks + c)] = t0;
      chunks[2 * (s * kCgChunks + c) + 1] = t1;
      __threadfence();
      last_of_solve = atomicAdd(&sarr[s], 1u) == kCgChunks - 1;
    }
  }
  if (threadIdx.x != 0) return;
  if (act ? !last_of_solve : c != 0) return;  // one report per slot: its last chunk, or chunk 0 of an idle slot
  if (act) {  // every chunk of solve s is in
    __threadfence();
    sarr[s] = 0;
    double t0 = 0.0, t1 = 0.0;
    for (int q = 0; q < kCgChunks; ++q) {
      t0 += __ldcg(chunks + 2 * (s * kCgChunks + q));
      t1 += __ldcg(chunks + 2 * (s * kCgChunks + q) + 1);
    }
    ResCG &cs = cg[s];
    if (op == CG_INIT) {
      cs.rho = t0;
      cs.r0 = cs.rnorm = sqrt(t1);
      cs.tol = cs.tol_factor * cs.r0;
      cs.it = 0;
      cs.converged = cs.rnorm <= cs.tol;
      cs.done = cs.converged || cs.max_it <= 0;
    } else if (op == CG_PQ) {
      if (!(t0 > 0.0)) cs.done = 1;  // breakdown: not positive definite on these unknowns
      else cs.alpha = cs.rho / t0;
    } else {
      cs.it += 1;
      cs.rnorm = sqrt(t1);
      if (cs.rnorm <= cs.tol) cs.converged = cs.done = 1;
      else if (cs.it >= cs.max_it) cs.done = 1;
      cs.beta = t0 / cs.rho;
      cs.rho = t0;
    }
    if (cs.done) D.state[s].mask = 0;
    else atomicAdd(&ctl->running, 1);
  }
  __threadfence();
  if (atomicAdd(&ctl->arrivals, 1u) != (unsigned)(gridDim.x / kCgChunks) - 1) return;  // the last slot to report
  __threadfence();
  const int running = atomicAdd(&ctl->running, 0);
  ctl->arrivals = 0;
  ctl->running = 0;
  if (in_graph && op != CG_PQ) cudaGraphSetConditional(handle, running > 0 ? 1u : 0u);
}

// p = r + beta p and E_res = p on the unknowns (the next iteration's
// operator input) of every solve still iterating (in the mask).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_pupd_e(Dir D, const ResCG *cg) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const R beta = R(cg[it.s].beta);
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      const bool dof = B.c(cRW + a)[o] > R(0.0);
      R *p = B.c(cRP + a) + o;
      if (dof) *p = B.c(cRR + a)[o] + beta * *p;
      B.c(cEX + a)[o] = dof ? *p : R(0.0);
    }
  });
}

// B* snapshot / restore over the whole box (SnapshotImplicitResistiveBstar_,
// RestoreImplicitResistiveBstar_, :260-292).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_copyb(Dir D, int op) {
  for_items<R, kFull>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const int o = B.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      if (op == RES_SNAPSHOT) B.c(cRBS + a)[o] = B.c(cBX + a)[o];
      else B.c(cBX + a)[o] = B.c(cRBS + a)[o];
    }
  });
}

// B += dt (-curl E_res) on the owned faces (ApplyImplicitResistiveUpdate_, :557-575;
// ApplyUpdate_Euler_BfaceOnly_, Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:435-473).
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_res_bupdate(Dir D) {
  for_items<R, kResK>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    const R dt = R(D.state[it.s].dt);
    const int i = it.i, j = it.j, k = it.k;
    // the faces whose edges E_res covers (k + 1 below the range's bound);
    // above them E_res is 0 and B does not change
    if (j < B.n1 && k + 1 < it.hi[2]) {
      const R rb = R(-1.0) * ((AT(cEY, i, j, k) - AT(cEY, i, j, k + 1)) + (AT(cEZ, i, j + 1, k) - AT(cEZ, i, j, k)));
      AT(cBX, i, j, k) += dt * rb;
    }
    if (i < B.n0 && k + 1 < it.hi[2]) {
      const R rb = R(-1.0) * ((AT(cEX, i, j, k + 1) - AT(cEX, i, j, k)) + (AT(cEZ, i, j, k) - AT(cEZ, i + 1, j, k)));
      AT(cBY, i, j, k) += dt * rb;
    }
    if (i < B.n0 && j < B.n1) {
      const R rb = R(-1.0) * ((AT(cEX, i, j, k) - AT(cEX, i, j + 1, k)) + (AT(cEY, i + 1, j, k) - AT(cEY, i, j, k)));
      AT(cBZ, i, j, k) += dt * rb;
    }
  });
}

// Static per-face terms of the CFL time step and the Rusanov wave speed, once
// per solve (run by mhd_prepare): |a| = sqrt(ax ax + ay ay + az az) and
// a / |a| of the face area vectors JD, the operations and order
// Per-solve static terms, evaluated once at prepare with the reference's
// expressions: the face normals and |JD| that Compute_Timestep
// (Timestep.cpp:15-16,78-93) and calc_Jac_radius_GCL (FluidRHS.cpp:5-14) apply
// every step (owned faces and one more layer), the ambipolar gradient
// coefficients (owned cells), the contravariant-velocity coefficients (the
// cells k_pv_uplus refreshes), the Hall diffusion ratios (owned edges) and
// the fluid fluxes' face JD and 1 / Jac in the real type.
template <class R>
__global__ void __launch_bounds__(kTileThreads) k_face_normals(Dir D) {
  for_items<R, kAlloc>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    if (!it.in) return;
    {
      // Coefficients of the contravariant velocities (calc_Uplus,
      // Tools.cpp:159-301) on the cells k_pv_uplus refreshes them on: the
      // face JD of each axis averaged to the cell, and 1 / (|Jac| + 1e-30).
      const int i = it.i, j = it.j, k = it.k;
      const int gm = min(consts_of<R>(S).nghost - 1, kStepGhost);
      if (i >= -gm && i < B.n0 + gm && j >= -gm && j < B.n1 + gm && k >= -gm && k < B.n2 + gm) {
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
          int ip = i, jp = j, kp = k;
          shift1(axis, ip, jp, kp, 1);
          const int cm = axis == 0 ? cJDX : axis == 1 ? cJDY : cJDZ;
#pragma unroll
          for (int q = 0; q < 3; ++q)
            AT(cUCK + 3 * axis + q, i, j, k) = R(0.5) * (R(ATM(cm + q, i, j, k)) + R(ATM(cm + q, ip, jp, kp)));
        }
        AT(cUCK + 9, i, j, k) = R(1.0) / (fabs(R(ATM(cJAC, i, j, k))) + R(1.0e-30));
      }
    }
    if (it.i < 0 || it.j < 0 || it.k < 0 || it.i > B.n0 || it.j > B.n1 || it.k > B.n2) return;  // [0, n + 1) below
    {
      // the face JD the fluid fluxes read and the cell's 1 / Jac, converted
      // to the real type once (the values the fluid kernel would form)
      const int i = it.i, j = it.j, k = it.k;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        AT(cFM + q, i, j, k) = R(ATM(cJDX + q, i, j, k));
        AT(cFM + 3 + q, i, j, k) = R(ATM(cJDY + q, i, j, k));
        AT(cFM + 6 + q, i, j, k) = R(ATM(cJDZ + q, i, j, k));
      }
      AT(cFM + 9, i, j, k) = R(1.0) / R(ATM(cJAC, i, j, k));
    }
    {
      // Hall diffusion ratios of the owned edges (BuildHallFaceEMF_Rusanov_diff_
      // step 3, Hall.cpp:148-400): edge length over the face area averaged
      // to the edge, both floored at 1e-14, per transverse direction.
      const int i = it.i, j = it.j, k = it.k;
      const R eps = R(1e-14);
      if (i < B.n0) {
        const R L = dmax(AT(cDLX, i, j, k), eps);
        const R Abz = R(0.5) * (AT(cAZ, i, j, k) + AT(cAZ, i, j - 1, k));
        const R Abe = R(0.5) * (AT(cAY, i, j, k) + AT(cAY, i, j, k - 1));
        AT(cIHX, i, j, k) = L / dmax(Abz, eps);
        AT(cIHX + 1, i, j, k) = L / dmax(Abe, eps);
      }
      if (j < B.n1) {
        const R L = dmax(AT(cDLY, i, j, k), eps);
        const R Abx = R(0.5) * (AT(cAX, i, j, k) + AT(cAX, i, j, k - 1));
        const R Abz = R(0.5) * (AT(cAZ, i, j, k) + AT(cAZ, i - 1, j, k));
        AT(cIHY, i, j, k) = L / dmax(Abx, eps);
        AT(cIHY + 1, i, j, k) = L / dmax(Abz, eps);
      }
      if (k < B.n2) {
        const R L = dmax(AT(cDLZ, i, j, k), eps);
        const R Abe = R(0.5) * (AT(cAY, i, j, k) + AT(cAY, i - 1, j, k));
        const R Abx = R(0.5) * (AT(cAX, i, j, k) + AT(cAX, i, j - 1, k));
        AT(cIHZ, i, j, k) = L / dmax(Abe, eps);
        AT(cIHZ + 1, i, j, k) = L / dmax(Abx, eps);
      }
    }
    {
      // Ambipolar pressure-gradient coefficients of an owned cell
      // (AddSourceToRHS_Fluid, FluidRHS.cpp:206-527): face JD averaged to the
      // cell and divided by |Jac| (zero where |Jac| is not positive).
      const int i = it.i, j = it.j, k = it.k;
      if (consts_of<R>(S).ambipolar && i < B.n0 && j < B.n1 && k < B.n2) {
        const R Vol = fabs(R(ATM(cJAC, i, j, k)));
        R a[9] = {R(0.0), R(0.0), R(0.0), R(0.0), R(0.0), R(0.0), R(0.0), R(0.0), R(0.0)};
        if (Vol > R(0.0)) {
          a[0] = R(0.5) * (R(ATM(cJDX, i - 1, j, k)) + R(ATM(cJDX, i, j, k))) / Vol;
          a[1] = R(0.5) * (R(ATM(cJDX + 1, i - 1, j, k)) + R(ATM(cJDX + 1, i, j, k))) / Vol;
          a[2] = R(0.5) * (R(ATM(cJDX + 2, i - 1, j, k)) + R(ATM(cJDX + 2, i, j, k))) / Vol;
          a[3] = R(0.5) * (R(ATM(cJDY, i, j - 1, k)) + R(ATM(cJDY, i, j, k))) / Vol;
          a[4] = R(0.5) * (R(ATM(cJDY + 1, i, j - 1, k)) + R(ATM(cJDY + 1, i, j, k))) / Vol;
          a[5] = R(0.5) * (R(ATM(cJDY + 2, i, j - 1, k)) + R(ATM(cJDY + 2, i, j, k))) / Vol;
          a[6] = R(0.5) * (R(ATM(cJDZ, i, j, k - 1)) + R(ATM(cJDZ, i, j, k))) / Vol;
          a[7] = R(0.5) * (R(ATM(cJDZ + 1, i, j, k - 1)) + R(ATM(cJDZ + 1, i, j, k))) / Vol;
          a[8] = R(0.5) * (R(ATM(cJDZ + 2, i, j, k - 1)) + R(ATM(cJDZ + 2, i, j, k))) / Vol;
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) AT(cAMB + q, i, j, k) = a[q];
      }
    }
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
      const int cm = a == 0 ? cJDX : a == 1 ? cJDY : cJDZ;
      const int cn = a == 0 ? cFNX : a == 1 ? cFNY : cFNZ;
      const int o = B.off(it.i, it.j, it.k);
      const double ax = B.m(cm)[o], ay = B.m(cm + 1)[o], az = B.m(cm + 2)[o];
      const double An = sqrt(ax * ax + ay * ay + az * az);
      B.c(cn)[o] = R(ax / An);
      B.c(cn + 1)[o] = R(ay / An);
      B.c(cn + 2)[o] = R(az / An);
      B.c(cn + 3)[o] = R(An);
    }
  });
}

// calc_PV + calc_Uplus (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:159-301) on the allocated
// cell range the step keeps, the contravariant velocities UCON and the next
// step's Hall cell field there, and the next step's CFL dt on owned cells (warp min, one atomicMin per warp on
// the bit pattern of the positive double).
template <class R>
__global__ void __launch_bounds__(kTileThreads, MHD_MIN_CTAS_PV) k_pv_uplus(Dir D) {
  for_items<R, kAlloc>(D, [&](const DevSolve &S, const V<R> &B, const Item &it) {
    const ConstsT<R> &c = consts_of<R>(S);
    const int i = it.i, j = it.j, k = it.k;
    R dtl = R(1e100);
    bool bad = false;
    if (it.in) {
      R vel[2][3];
      R chk = R(0.0);  // sum of the conserved components: non-finite if any of them is
      for (int s = 0; s < 2; ++s) {
        const int u0 = s ? cUN : cUH, pv0 = s ? cPVN : cPVH;
        const R coeff = s ? c.state_coeff_Na : c.state_coeff_H;
        const R r0 = LD(u0, i, j, k), m1 = LD(u0 + 1, i, j, k), m2 = LD(u0 + 2, i, j, k), m3 = LD(u0 + 3, i, j, k);
        const R rho = dmax(r0, R(1e-12));
        const R u = m1 / rho, v = m2 / rho, w = m3 / rho;
        const R E = LD(u0 + 4, i, j, k);
        chk += ((r0 + m1) + (m2 + m3)) + E;
        const R ke = R(0.5) * rho * (u * u + v * v + w * w);
        R eint = E - ke;
        if (eint < R(0.0)) eint = R(0.0);
        R pr = (c.gamma - R(1.0)) * eint;
        pr = dmax(pr, R(1e-12));
        const R T = pr / (rho * coeff);
        const int o = B.off(i, j, k);
        B.c(pv0)[o] = u;
        B.c(pv0 + 1)[o] = v;
        B.c(pv0 + 2)[o] = w;
        B.c(pv0 + 3)[o] = pr;
        B.c(pv0 + 4)[o] = T;
        vel[s][0] = u;
        vel[s][1] = v;
        vel[s][2] = w;
      }
      const R rH = dmax(LD(cUH, i, j, k), R(0.0)), rN = dmax(LD(cUN, i, j, k), R(0.0));
      const Num<R> d = num_limiter(c, rH, rN);
      {
        // the next step's Hall cell field, BuildHallFaceEMF_Rusanov_diff_ step 1
        // (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:110-146): its inputs (J_cell,
        // B_cell, the densities) are final here (num_limiter clamps the
        // densities at zero itself, so d is the limiter of the raw densities)
        const R alpha = c.hall_coef / d.ne_eff;
        const R Jx = LD(cJC, i, j, k), Jy = LD(cJC + 1, i, j, k), Jz = LD(cJC + 2, i, j, k);
        const R Bx = LD(cBC, i, j, k), By = LD(cBC + 1, i, j, k), Bz = LD(cBC + 2, i, j, k);
        AT(cEHC, i, j, k) = alpha * (Jy * Bz - Jz * By);
        AT(cEHC + 1, i, j, k) = alpha * (Jz * Bx - Jx * Bz);
        AT(cEHC + 2, i, j, k) = alpha * (Jx * By - Jy * Bx);
        AT(cHB, i, j, k) = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
      }
      R up[3];
      for (int q = 0; q < 3; ++q) {
        const R uH = rH > R(1e-20) ? vel[0][q] : R(0.0);
        const R uN = rN > R(1e-20) ? vel[1][q] : R(0.0);
        up[q] = d.chiH * uH + d.chiNa * uN;
        AT(cUP + q, i, j, k) = up[q];
      }
      const int gm = min(c.nghost - 1, kStepGhost);
      if (i >= -gm && i < B.n0 + gm && j >= -gm && j < B.n1 + gm && k >= -gm && k < B.n2 + gm) {
        // coefficients (cell-averaged JD, 1 / (|Jac| + 1e-30)) from k_face_normals
        const R inv_jac = LD(cUCK + 9, i, j, k);
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
          const R kx = LD(cUCK + 3 * axis, i, j, k), ky = LD(cUCK + 3 * axis + 1, i, j, k),
                  kz = LD(cUCK + 3 * axis + 2, i, j, k);
          AT(cUC + axis, i, j, k) = (kx * up[0] + ky * up[1] + kz * up[2]) * inv_jac;
        }
      }
      if (i >= 0 && i < B.n0 && j >= 0 && j < B.n1 && k >= 0 && k < B.n2) {
        dtl = cell_dt(B, c, i, j, k);
        // a NaN drops out of the minimum below (and the pressure floors can
        // hide a non-finite energy from it): record it instead
        bad = !isfinite(dtl) || !isfinite(chk);
      }
    }
    // warp minimum, one atomicMin per warp (min is exact in any order)
    for (int o = 16; o > 0; o >>= 1) dtl = dmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
    if ((threadIdx.x & 31) == 0 && dtl < R(1e100))
      atomicMin(&D.state[it.s].dt_bits, (unsigned long long)__double_as_longlong(dtl));
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(&D.state[it.s].nonfinite, 1);
  });
}

#undef AT
#undef LD
#undef LDM

// ------------------------------------------------------------------ sync, alias, bookkeeping
__device__ __forceinline__ int find_solve(const int *prefix, int nsolves, int e) {
  int lo = 0, hi = nsolves;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}
template <class R>
__device__ __forceinline__ R *at_code(const DevSolve &S, int cur, int64_t code) {
  return (R *)(S.arena + (code & kCodeOffMask) + ((code & kCodeUFlag) ? (int64_t)cur * S.ubuf : int64_t(0)));
}
__device__ __forceinline__ const int *op_prefix(const Dir &D, const SyncOp &op) {
  if (op.kind == SYNC_COPY) return D.copy_prefix[op.arg][op.phase];
  return op.arg ? D.aliasJ_prefix : D.aliasE_prefix;
}

// MercuryBoundary::Sync_ stages (Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110) and
// ReduceEdgeAliasCandidatesToOwners_ (Z4_Mercury/src/physics/MercurySolver_Current.cpp:3-57)
// for every active solve, up to two independent operations per launch.
// Work unit: a group of 8 lanes.  A copy phase gives each group one segment
// (dst <- sign * src on up to kSegElems elements: reps strided runs of len
// consecutive elements); an alias reduction gives each lane one class, whose
// members are summed in stored order from 0.0 and written to the owner as
// owner_sign * sum / count.
template <class R>
__global__ void __launch_bounds__(256) k_sync(Dir D, SyncOps ops) {
  const int lane = threadIdx.x & 7;
  const int stride = (gridDim.x * blockDim.x) >> 3;
  const int *pre0 = op_prefix(D, ops.op[0]);
  const int *pre1 = ops.n > 1 ? op_prefix(D, ops.op[1]) : nullptr;
  const int t0 = pre0[D.nsolves];
  const int total = t0 + (pre1 ? pre1[D.nsolves] : 0);
  for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 3; g < total; g += stride) {
    const bool second = g >= t0;
    const SyncOp &op = second ? ops.op[1] : ops.op[0];
    const int *pre = second ? pre1 : pre0;
    const int e = second ? g - t0 : g;
    const int s = find_solve(pre, D.nsolves, e);
    if (!solve_active(D, s)) continue;
    const DevSolve &S = D.solves[s];
    const int q = e - pre[s];
    const int cur = D.state[s].cur;
    if (op.kind == SYNC_COPY) {
      const DevTable &T = S.tab[op.arg][op.phase];
      const int64_t *w = T.seg + kSegWords * (int64_t)q;
      const int64_t dcode = w[0], scode = w[1], rw = w[2];
      const int len = (int)((dcode >> kSegLenShift) & 31) + 1;
      const int n = len * ((int)(rw & 0xffff) + 1);
      const int64_t stride = rw >> kSegStrideShift;  // bytes between runs
      const bool neg = (dcode >> kSegNegBit) & 1;
      const char *src = (const char *)at_code<R>(S, cur ^ op.prev, scode);
      char *dst = (char *)at_code<R>(S, cur, dcode);
      // element e of the segment: run e / len, offset e % len (e < 64, so
      // e * ceil(2^16 / len) >> 16 is the exact quotient)
      const int inv = (65536 + len - 1) / len;
      R v[kSegElems / 8];
      int64_t off[kSegElems / 8];
#pragma unroll
      for (int u = 0; u < kSegElems / 8; ++u) {
        const int e = lane + 8 * u;
        const int r = (e * inv) >> 16;
        off[u] = r * stride + (int64_t)(e - r * len) * (int64_t)sizeof(R);
        if (e < n) v[u] = *(const R *)(src + off[u]);
      }
#pragma unroll
      for (int u = 0; u < kSegElems / 8; ++u)
        if (lane + 8 * u < n) *(R *)(dst + off[u]) = op.mark ? R(0.0) : (neg ? -v[u] : v[u]);
    } else {
      const DevAlias &A = op.arg ? S.aliasJ : S.aliasE;
      const int c = q * 8 + lane;
      if (c < A.n) {
        R sum = R(0.0);
        for (int m = A.offset[c]; m < A.offset[c + 1]; ++m) sum += R(A.msign[m]) * *at_code<R>(S, cur, A.member[m]);
        *at_code<R>(S, cur, A.owner[c]) = R(A.osign[c]) * sum / (R)(A.offset[c + 1] - A.offset[c]);
      }
    }
  }
}

#define AT(cc, i, j, k) (B.c(cc)[B.off((i), (j), (k))])
#define ATM(cc, i, j, k) (B.m(cc)[B.off((i), (j), (k))])

// A block's view outside the tile loop (the singular-edge passes).
template <class R>
__device__ __forceinline__ V<R> block_view(const Dir &D, int s, int b) {
  const DevBlock &DB = D.solves[s].blocks[b];
  V<R> B;
  const int cur = D.state[s].cur;
  B.U = (R *)DB.U[cur];
  B.Un = (R *)DB.U[cur ^ 1];
  B.M = DB.M;
  B.total = (int)DB.total;
  B.si = (int)DB.si;
  B.sj = (int)DB.sj;
  B.G = DB.G;
  B.n0 = DB.n[0];
  B.n1 = DB.n[1];
  B.n2 = DB.n[2];
  return B;
}

// Physical boundary operations of table `which` (a sync group, or the wall
// EMF) for every active solve (mhd_phys_op; BoundaryCore::ApplyPhysical with
// MercuryBoundary's handlers, Z4_Mercury/src/boundary/Boundary_Build.cpp:5-300).
// The operations of one table write distinct DOFs and read none another
// writes, so they run in any order.
template <class R>
__global__ void __launch_bounds__(256) k_phys(Dir D, int which) {
  const int *pre = D.phys_prefix[which];
  const int total = pre[D.nsolves];
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  // a warp takes 32 consecutive operations, one per lane; the constant
  // segments among them are then written by the whole warp, one element per
  // lane (consecutive destinations to consecutive lanes)
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < total; base += nwarps * 32) {
    const int e = base + lane;
    unsigned long long seg_p = 0;  // the segment's first destination (0: not a segment)
    int64_t seg_w = 0;
    R seg_v = R(0.0);
    const DevPhysOp *opp = nullptr;
    const DevSolve *Sp = nullptr;
    int cur = 0;
    if (e < total) {
      const int s = find_solve(pre, D.nsolves, e);
      if (solve_active(D, s)) {
        Sp = &D.solves[s];
        const DevPhys &P = Sp->phys[which];
        cur = D.state[s].cur;
        const int q = e - pre[s];
        if (q < P.nset) {  // destinations <- bc[arg]: nr runs of len elements, stride bytes apart
          const int64_t w0 = P.set[2 * q];
          seg_w = P.set[2 * q + 1];
          seg_v = consts_of<R>(*Sp).bc[(int)((w0 >> kPhysArgShift) & 31)];
          seg_p = (unsigned long long)at_code<R>(*Sp, cur, w0 & ~(int64_t(31) << kPhysArgShift));
        } else {
          opp = &P.op[q - P.nset];
        }
      }
    }
    for (unsigned m = __ballot_sync(0xffffffffu, seg_p != 0); m; m &= m - 1) {
      const int src = __ffs(m) - 1;
      char *p0 = (char *)__shfl_sync(0xffffffffu, seg_p, src);
      const int64_t w1 = __shfl_sync(0xffffffffu, seg_w, src);
      const R v = __shfl_sync(0xffffffffu, seg_v, src);
      const int len = (int)(w1 & 255) + 1, nr = (int)((w1 >> 8) & 255) + 1;
      const int64_t stride = w1 >> 16;
      if (lane < len * nr) {
        const int r = lane / len;
        *(R *)(p0 + r * stride + (int64_t)(lane - r * len) * (int64_t)sizeof(R)) = v;
      }
    }
    if (!opp) continue;
    const DevSolve &S = *Sp;
    const ConstsT<R> &c = consts_of<R>(S);
    const DevPhysOp &op = *opp;
    if (op.kind == MHD_PHYS_WALL) {
      // BC_Solid_Surface_ (Z4_Mercury/src/boundary/Boundary_Condition_Fluid.cpp:37-259), H+:
      // the boundary cell from the cell one deeper (density floor 2.5e-3,
      // no-slip, pressure from the conserved state with its floors), then
      // the ghost cells from the boundary cell's new state
      const R floor = R(2.5e-3), g1 = c.gamma - R(1.0);
      auto wall = [&](const R *U, R *out) {
        const R rho_r = dmax(U[0], floor);
        const R rho = dmax(rho_r, floor);
        const R ke = R(0.5) * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rho;
        R eint = U[4] - ke;
        if (eint < R(0.0)) eint = R(0.0);
        const R p = dmax(g1 * eint, R(1.0e-12));
        out[0] = rho_r;
        out[1] = out[2] = out[3] = rho_r * R(0.0);
        out[4] = p / g1 + R(0.5) * rho_r * R(0.0);
      };
      R u[5], w1[5], w2[5];
      for (int m = 0; m < 5; ++m) u[m] = *at_code<R>(S, cur, op.src + m * op.cstride);
      wall(u, w1);
      wall(w1, w2);
      for (int m = 0; m < 5; ++m) *at_code<R>(S, cur, op.dst + m * op.cstride) = w1[m];
      for (int g = 0; g < op.nghost; ++g)
        for (int m = 0; m < 5; ++m) *at_code<R>(S, cur, op.ghost[g] + m * op.cstride) = w2[m];
    } else {
      // BC_Farfield_Eedge_set_zerocurl (Z4_Mercury/src/boundary/Boundary_Condition.cpp:573-624):
      // E = E_inf . dr with E_inf = -u_inf x B_imf
      const R *u = c.bc + MHD_BC_UINF, *Bi = c.bc + MHD_BC_BIMF;
      const R E0 = Bi[1] * u[2] - Bi[2] * u[1], E1 = Bi[2] * u[0] - Bi[0] * u[2], E2 = Bi[0] * u[1] - Bi[1] * u[0];
      const R d0 = *at_code<R>(S, cur, op.src), d1 = *at_code<R>(S, cur, op.src + op.cstride),
              d2 = *at_code<R>(S, cur, op.src + 2 * op.cstride);
      *at_code<R>(S, cur, op.dst) = E0 * d0 + E1 * d1 + E2 * d2;
    }
  }
}

// One thread per singular edge of every active solve.
template <class F>
__device__ __forceinline__ void for_singular(const Dir &D, F &&f) {
  const int total = D.sing_prefix[D.nsolves];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int s = find_solve(D.sing_prefix, D.nsolves, e);
    if (!solve_active(D, s)) continue;
    f(s, D.solves[s].sing, e - D.sing_prefix[s]);
  }
}

// The geometric data of the singular edges (SingularEdgeRegistry::build,
// src/7_metric/SingularEdgeRegistry.cpp:78-300) from the uploaded geometry,
// in the reference's operation order: the mean primal length and the
// canonical edge vector over the aliases, the |Jac| weights of the incident
// cells, the dual polygon through their centres (sorted by angle about the
// edge) and its area, the inverse Hodge star, which also replaces the edge
// Hodge field of every alias.  Computed in FP64 from the double metric and
// the real-typed edge fields.
template <class R>
__global__ void k_sing_setup(Dir D) {
  for_singular(D, [&](int s, const DevSingular &G, int e) {
    double len = 0.0, dr[3] = {0.0, 0.0, 0.0};
    int nlen = 0;
    for (int a = G.aoff[e]; a < G.aoff[e + 1]; ++a) {
      const int *r = G.alias + 6 * a;
      const V<R> B = block_view<R>(D, s, r[0]);
      const int ax = r[1];
      const double L = (double)AT(cDLX + ax, r[2], r[3], r[4]);
      if (isfinite(L) && L > 0.0) {
        len += L;
        ++nlen;
      }
      for (int q = 0; q < 3; ++q) dr[q] += r[5] * (double)AT((ax == 0 ? cDRX : ax == 1 ? cDRY : cDRZ) + q, r[2], r[3], r[4]);
    }
    double gv = 0.0;
    constexpr int kMaxCells = 16;
    double pts[kMaxCells][3];
    int np = 0;
    for (int q = G.coff[e]; q < G.coff[e + 1]; ++q) {
      const int *r = G.cell + 6 * q;
      const V<R> B = block_view<R>(D, s, r[0]);
      const double v = fabs(ATM(cJAC, r[2], r[3], r[4]));
      if (isfinite(v) && v > 1.e-30) {
        gv += v;
        if (np < kMaxCells) {
          for (int c = 0; c < 3; ++c) pts[np][c] = (double)AT(cCX + c, r[2], r[3], r[4]);
          ++np;
        }
      }
    }
    for (int q = G.coff[e]; q < G.coff[e + 1]; ++q) {
      const int *r = G.cell + 6 * q;
      const V<R> B = block_view<R>(D, s, r[0]);
      const double v = fabs(ATM(cJAC, r[2], r[3], r[4]));
      G.w[q] = (isfinite(v) && v > 1.e-30 && gv > 0.0) ? v / gv : 0.0;
    }
    const double primal = nlen ? len / nlen : 0.0;
    double dual = 0.0;
    if (np >= 3) {
      double cen[3] = {0.0, 0.0, 0.0};
      for (int n = 0; n < np; ++n)
        for (int c = 0; c < 3; ++c) cen[c] += pts[n][c];
      for (int c = 0; c < 3; ++c) cen[c] /= np;
      double t[3] = {dr[0], dr[1], dr[2]};
      const double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      if (tn > 0.0)
        for (double &x : t) x /= tn;
      const double ref[3] = {fabs(t[0]) < 0.9 ? 1.0 : 0.0, fabs(t[0]) < 0.9 ? 0.0 : 1.0, 0.0};
      double u[3] = {t[1] * ref[2] - t[2] * ref[1], t[2] * ref[0] - t[0] * ref[2], t[0] * ref[1] - t[1] * ref[0]};
      const double un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      if (un > 0.0)
        for (double &x : u) x /= un;
      const double v[3] = {t[1] * u[2] - t[2] * u[1], t[2] * u[0] - t[0] * u[2], t[0] * u[1] - t[1] * u[0]};
      double ang[kMaxCells];
      for (int n = 0; n < np; ++n) {
        double du = 0.0, dv = 0.0;
        for (int c = 0; c < 3; ++c) {
          du += (pts[n][c] - cen[c]) * u[c];
          dv += (pts[n][c] - cen[c]) * v[c];
        }
        ang[n] = atan2(dv, du);
      }
      int ord[kMaxCells];
      for (int n = 0; n < np; ++n) ord[n] = n;
      for (int n = 1; n < np; ++n)  // insertion sort by angle (the points are few and their angles distinct)
        for (int m = n; m > 0 && ang[ord[m]] < ang[ord[m - 1]]; --m) {
          const int tmp = ord[m];
          ord[m] = ord[m - 1];
          ord[m - 1] = tmp;
        }
      double av[3] = {0.0, 0.0, 0.0};
      for (int n = 0; n < np; ++n) {
        const double *a = pts[ord[n]], *b = pts[ord[(n + 1) % np]];
        av[0] += a[1] * b[2] - a[2] * b[1];
        av[1] += a[2] * b[0] - a[0] * b[2];
        av[2] += a[0] * b[1] - a[1] * b[0];
      }
      dual = 0.5 * sqrt(av[0] * av[0] + av[1] * av[1] + av[2] * av[2]);
    }
    if (!(dual > 0.0)) dual = primal > 0.0 ? gv / primal : 0.0;
    const double ih = dual > 0.0 ? primal / dual : 0.0;
    double *geo = G.geo + 4 * e;
    for (int q = 0; q < 3; ++q) geo[q] = nlen > 0 ? dr[q] / nlen : 0.0;
    geo[3] = ih;
    for (int a = G.aoff[e]; a < G.aoff[e + 1]; ++a) {  // the registry publishes it to every alias
      const int *r = G.alias + 6 * a;
      const V<R> B = block_view<R>(D, s, r[0]);
      AT(cALX + r[1], r[2], r[3], r[4]) = (R)ih;
    }
  });
}

// The EMF and the Hall EMF of the singular edges' owners:
// AssembleSingularEdgeEMF_NonHall_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ideal.cpp:57-130) and
// AssembleSingularEdgeEMF_HallExplicit_ (MercurySolver_MagExplicit_Hall.cpp:32-56): the |Jac|-weighted
// sum over the incident cells of the cell field projected on the canonical
// edge vector, times the owner's orientation.  (The local artificial
// resistivity term of the non-Hall EMF is not included.)
template <class R>
__global__ void k_sing_emf(Dir D) {
  for_singular(D, [&](int s, const DevSingular &G, int e) {
    const ConstsT<R> &c = consts_of<R>(D.solves[s]);
    const double *geo = G.geo + 4 * e;
    const R cv[3] = {(R)geo[0], (R)geo[1], (R)geo[2]};
    R sumE = R(0.0), sumH = R(0.0);
    for (int q = G.coff[e]; q < G.coff[e + 1]; ++q) {
      const int *r = G.cell + 6 * q;
      const V<R> B = block_view<R>(D, s, r[0]);
      const int i = r[2], j = r[3], k = r[4];
      const R u0 = AT(cUP, i, j, k), u1 = AT(cUP + 1, i, j, k), u2 = AT(cUP + 2, i, j, k);
      const R b0 = AT(cBC, i, j, k), b1 = AT(cBC + 1, i, j, k), b2 = AT(cBC + 2, i, j, k);
      const R ex = -(u1 * b2 - u2 * b1), ey = -(u2 * b0 - u0 * b2), ez = -(u0 * b1 - u1 * b0);
      R emf = ex * cv[0] + ey * cv[1] + ez * cv[2];
      const Num<R> num = num_limiter<R>(c, AT(cUH, i, j, k), AT(cUN, i, j, k));
      if (c.ambipolar) {
        const int ax = r[1];
        const int im = i - (ax == 0), jm = j - (ax == 1), km = k - (ax == 2);
        const int ip = i + (ax == 0), jp = j + (ax == 1), kp = k + (ax == 2);
        const R dp = R(0.5) * ((AT(cPVH + 3, ip, jp, kp) + AT(cPVN + 3, ip, jp, kp)) -
                               (AT(cPVH + 3, im, jm, km) + AT(cPVN + 3, im, jm, km)));
        const R pressure_coef = (c.rho_ref * c.U_ref) / (c.q_e * c.L_ref * c.B_ref * c.n_ref);
        emf -= pressure_coef * R(r[5]) * dp / num.ne_eff;
      }
      const R j0 = AT(cJC, i, j, k), j1 = AT(cJC + 1, i, j, k), j2 = AT(cJC + 2, i, j, k);
      if (c.arti_eta_max > R(0.0)) {
        const R jedge = j0 * cv[0] + j1 * cv[1] + j2 * cv[2];
        const R jmag = sqrt(j0 * j0 + j1 * j1 + j2 * j2);
        R qq = (jmag - c.arti_J_start) / dmax(c.arti_J_on - c.arti_J_start, R(1.e-30));
        qq = dmax(R(0.0), dmin(R(1.0), qq));
        emf += c.arti_eta_max * qq * qq * (R(3.0) - R(2.0) * qq) * jedge;
      }
      const R w = (R)G.w[q];
      sumE += w * emf;
      // Hall: alpha (J x B) at the cell, times the radial taper at its centre
      const R alpha = c.hall_coef / num.ne_eff;
      const R hx = alpha * (j1 * b2 - j2 * b1), hy = alpha * (j2 * b0 - j0 * b2), hz = alpha * (j0 * b1 - j1 * b0);
      sumH += w * (AT(cTPC, i, j, k) * (hx * cv[0] + hy * cv[1] + hz * cv[2]));
    }
    const R os = (R)G.osign[e];
    *at_code<R>(D.solves[s], D.state[s].cur, G.owner[3 * e]) = os * sumE;
    *at_code<R>(D.solves[s], D.state[s].cur, G.owner[3 * e + 1]) = os * sumH;
  });
}

// The current of the singular edges' owners (AssembleSingularEdgeCurrent_,
// Z4_Mercury/src/physics/MercurySolver_Current.cpp:59-138): the inverse Hodge star times the sum
// over the incident owner faces of the signed beta B, times the owner's
// orientation.
template <class R>
__global__ void k_sing_j(Dir D) {
  for_singular(D, [&](int s, const DevSingular &G, int e) {
    const R ih = (R)G.geo[4 * e + 3];
    R sum = R(0.0);
    for (int q = G.foff[e]; q < G.foff[e + 1]; ++q) {
      const int *r = G.face + 6 * q;
      if (r[5] == 0) continue;
      const V<R> B = block_view<R>(D, s, r[0]);
      const int ax = r[1];
      sum += ih * R(r[5]) * AT(cBFX + ax, r[2], r[3], r[4]) * AT((ax == 0 ? cBX : ax == 1 ? cBY : cBZ), r[2], r[3], r[4]);
    }
    *at_code<R>(D.solves[s], D.state[s].cur, G.owner[3 * e + 2]) = R(G.osign[e]) * sum;
  });
}

#undef AT
#undef ATM

// After the updates: flip the state buffer, account time/step
// (Z4_Mercury/src/MercurySolver_Driver.cpp:40-45), record a dt failure (the
// reference's exit(-1), Timestep.cpp:129-140) and re-arm the dt reduction.
__global__ void k_flip(Dir D) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < D.nsolves; s += gridDim.x * blockDim.x) {
    SolveState &st = D.state[s];
    if (!st.remaining) continue;
    if (st.nonfinite) {  // a NaN/Inf cell: retire the solve, the others go on
      st.status = MHD_ERR_NONFINITE;
      st.remaining = 0;
      continue;
    }
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
// Every range kernel is persistent (grid-stride over tiles): its grid is the
// SM count times the CTAs of it that fit on one SM (at most 8), so all CTAs
// are resident at once and none starts in a late partial wave.  The
// residual-dot kernel keeps a fixed grid: its partial sums are indexed by CTA.
static int g_grid_tiles = 0;
static int g_grid_kernel[SK_COUNT];
static int g_grid_fluid[kNumFluidTiles];  // the fluid kernel's, per tile variant

template <class R>
static const void *fluid_fn(int v) {
  switch (v) {
    case 1: return (const void *)k_fluid<R, 1>;
    case 2: return (const void *)k_fluid<R, 2>;
    case 3: return (const void *)k_fluid<R, 3>;
    case 4: return (const void *)k_fluid<R, 4>;
    case 5: return (const void *)k_fluid<R, 5>;
    case 6: return (const void *)k_fluid<R, 6>;
    default: return (const void *)k_fluid<R, 0>;
  }
}
static_assert(kNumFluidTiles == 7, "fluid_fn and launch_fluid list every variant");
template <class R>
static size_t fluid_smem(int v) {
  switch (v) {
    case 1: return FluidSmem<R, 1>::bytes;
    case 2: return FluidSmem<R, 2>::bytes;
    case 3: return FluidSmem<R, 3>::bytes;
    case 4: return FluidSmem<R, 4>::bytes;
    case 5: return FluidSmem<R, 5>::bytes;
    case 6: return FluidSmem<R, 6>::bytes;
    default: return FluidSmem<R, 0>::bytes;
  }
}
template <class R>
static void launch_fluid(int v, const Dir &D, cudaStream_t st) {
  const int G = g_grid_fluid[(v >= 0 && v < kNumFluidTiles) ? v : 0];
  switch (v) {
    case 1: k_fluid<R, 1><<<G, kTileThreads, FluidSmem<R, 1>::bytes, st>>>(D); break;
    case 2: k_fluid<R, 2><<<G, kTileThreads, FluidSmem<R, 2>::bytes, st>>>(D); break;
    case 3: k_fluid<R, 3><<<G, kTileThreads, FluidSmem<R, 3>::bytes, st>>>(D); break;
    case 4: k_fluid<R, 4><<<G, kTileThreads, FluidSmem<R, 4>::bytes, st>>>(D); break;
    case 5: k_fluid<R, 5><<<G, kTileThreads, FluidSmem<R, 5>::bytes, st>>>(D); break;
    case 6: k_fluid<R, 6><<<G, fluid_threads(6), FluidSmem<R, 6>::bytes, st>>>(D); break;
    default: k_fluid<R, 0><<<G, kTileThreads, FluidSmem<R, 0>::bytes, st>>>(D); break;
  }
}

template <class R>
static const void *kernel_fn(StepKernel k) {
  switch (k) {
    case SK_FACE_EMF: return (const void *)k_face_emf<R>;
    case SK_EDGE_EMF: return (const void *)k_edge_emf<R>;
    case SK_HALL_EDGE: return (const void *)k_hall_edge<R>;
    case SK_ADD_HALL: return (const void *)k_add_hall<R>;
    case SK_FLUID: return fluid_fn<R>(0);
    case SK_BFACE: return (const void *)k_bface<R>;
    case SK_BCELL_JEDGE: return (const void *)k_bcell_jedge<R>;
    case SK_JCELL: return (const void *)k_jcell<R>;
    case SK_PV_UPLUS: return (const void *)k_pv_uplus<R>;
    case SK_SYNC: return (const void *)k_sync<R>;
    case SK_FACE_NORMALS: return (const void *)k_face_normals<R>;
    case SK_DIVB: return (const void *)k_div_b<R>;
    case SK_RES_SEED: return (const void *)k_res_seed<R>;
    case SK_RES_W: return (const void *)k_res_w<R>;
    case SK_RES_VEC: return (const void *)k_res_vec<R>;
    case SK_RES_DB: return (const void *)k_res_db<R>;
    case SK_RES_DJ: return (const void *)k_res_dj<R>;
    case SK_RES_Q: return (const void *)k_res_q<R>;
    case SK_RES_COPYB: return (const void *)k_res_copyb<R>;
    case SK_RES_BUPDATE: return (const void *)k_res_bupdate<R>;
    case SK_RES_CG: return (const void *)k_res_cg<R>;
    case SK_RES_PUPD_E: return (const void *)k_res_pupd_e<R>;
    case SK_PHYS: return (const void *)k_phys<R>;
    case SK_RES_CLEARB: return (const void *)k_res_clearb<R>;
    case SK_RES_CGSUM: return (const void *)k_res_cg_sum;
    default: return nullptr;
  }
}

static std::once_flag g_grids_once;

template <class R>
static void grids_init() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  for (int k = 0; k < SK_COUNT; ++k) {
    int per_sm = 8;
    const void *fn = kernel_fn<R>((StepKernel)k);
    if (fn && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kTileThreads, 0) != cudaSuccess ||
               per_sm < 1)) {
      cudaGetLastError();
      per_sm = 1;
    }
    g_grid_kernel[k] = sms * (per_sm < 8 ? per_sm : 8);
  }
  for (int v = 0; v < kNumFluidTiles; ++v) {
    int per_sm = 8;
    // the staged cells and face fluxes are dynamic shared memory (above the
    // 48 KB default in FP64)
    cudaFuncSetAttribute(fluid_fn<R>(v), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fluid_smem<R>(v));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fluid_fn<R>(v), fluid_threads(v), fluid_smem<R>(v)) !=
            cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    g_grid_fluid[v] = sms * (per_sm < 8 ? per_sm : 8);
  }
  g_grid_tiles = sms * 8;
}

template <class R>
static void grids() {
  std::call_once(g_grids_once, grids_init<R>);
}

template <class R>
static void launch_as(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int iarg, double darg,
                      ResScratch rs) {
  const int G = g_grid_kernel[k];
  switch (k) {
    case SK_FACE_EMF: k_face_emf<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_EDGE_EMF: k_edge_emf<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_HALL_EDGE: k_hall_edge<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_ADD_HALL: k_add_hall<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_FLUID: launch_fluid<R>(iarg, D, st); break;  // iarg: the tile variant
    case SK_BFACE: k_bface<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_BCELL_JEDGE: k_bcell_jedge<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_JCELL: k_jcell<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_PV_UPLUS: k_pv_uplus<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_SYNC: k_sync<R><<<G, kTileThreads, 0, st>>>(D, *ops); break;
    case SK_FACE_NORMALS: k_face_normals<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_DIVB: k_div_b<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_SEED: k_res_seed<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_W: k_res_w<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_VEC: k_res_vec<R><<<G, kTileThreads, 0, st>>>(D, iarg); break;
    case SK_RES_DB: k_res_db<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_DJ: k_res_dj<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_Q: k_res_q<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_DOT: k_res_dot<R><<<g_grid_tiles, kTileThreads, 0, st>>>(D, rs.partial); break;
    case SK_RES_SUM: k_res_sum<<<1, 32, 0, st>>>(rs.partial, g_grid_tiles, rs.result); break;
    case SK_RES_COPYB: k_res_copyb<R><<<G, kTileThreads, 0, st>>>(D, iarg); break;
    case SK_RES_BUPDATE: k_res_bupdate<R><<<G, kTileThreads, 0, st>>>(D); break;
    case SK_RES_CG:
      k_res_cg<R><<<g_grid_tiles, kTileThreads, 0, st>>>(D, iarg, rs.tpartial, rs.cg, rs.handle, rs.in_graph);
      break;
    case SK_RES_CGSUM:
      k_res_cg_sum<<<D.nsolves * kCgChunks, kTileThreads, 0, st>>>(D, iarg, rs.tpartial, rs.cg, rs.ctl, rs.chunks,
                                                                   rs.sarrivals, rs.handle, rs.in_graph);
      break;
    case SK_RES_PUPD_E: k_res_pupd_e<R><<<G, kTileThreads, 0, st>>>(D, rs.cg); break;
    case SK_FLIP: k_flip<<<1, 128, 0, st>>>(D); break;
    case SK_RETIRE: k_retire<<<1, 128, 0, st>>>(D); break;
    case SK_PHYS: k_phys<R><<<G, 256, 0, st>>>(D, iarg); break;
    // one thread per singular edge (8 radial lines of nr edges per shell)
    case SK_SING_SETUP: k_sing_setup<R><<<g_grid_tiles / 2, 64, 0, st>>>(D); break;
    case SK_SING_EMF: k_sing_emf<R><<<g_grid_tiles / 2, 64, 0, st>>>(D); break;
    case SK_SING_J: k_sing_j<R><<<g_grid_tiles / 2, 64, 0, st>>>(D); break;
    case SK_RES_CLEARB: k_res_clearb<R><<<G, kTileThreads, 0, st>>>(D); break;
    default: break;
  }
}

// The FP32 instantiations are compiled in their own translation unit (this
// file built with MHD_KERNELS_F32 and FP32 fast-math flags: FMA contraction,
// approximate division and square root); the FP64 one keeps the bit-exact
// flags.
#if MHD_KERNELS_F32
// Vectors of the mixed-precision implicit substep between a solve's FP32
// arena (every masked solve of D) and its FP64 companion (DevSolve::companion:
// the companion's blocks, the same boxes):
// RES_X_STATIC (the whole box, once at prepare): companion alpha, beta, eta,
//   W = the solve's (widened).
// The others over the substep's range (kResK), where its unknowns are:
// RES_X_SETUP: the companion's b (B* snapshot arrays) and r = the solve's r
//   (the FP32 right-hand side eta J(B*)); companion x = 0; the companion's
//   dt = the step's.
// RES_X_DEMOTE_R: r = (float) companion r (the next correction's right-hand side).
// RES_X_ADD_X: companion x += x (the correction).
// RES_X_DEMOTE_X: x = (float) companion x (the solution).
template <int KIND>
__global__ void __launch_bounds__(kTileThreads) k_res_cross(Dir D, int op) {
  for_items<float, KIND>(D, [&](const DevSolve &S, const V<float> &B, const Item &it) {
    if (!it.in) return;
    const DevBlock &CB = S.companion[it.blk];
    if (op == RES_X_SETUP && it.blk == 0 && it.i == it.lo[0] && it.j == it.lo[1] && it.k == it.lo[2]) {
      S.companion_state->dt = D.state[it.s].dt;  // the step's dt, once per solve
      S.companion_state->dt_bits = D.state[it.s].dt_bits;
    }
    V<double> C;
    C.U = C.Un = nullptr;
    C.M = CB.M;
    C.total = (int)CB.total;
    C.si = (int)CB.si;
    C.sj = (int)CB.sj;
    C.G = CB.G;
    C.n0 = CB.n[0];
    C.n1 = CB.n[1];
    C.n2 = CB.n[2];
    const int o = B.off(it.i, it.j, it.k), oc = C.off(it.i, it.j, it.k);
    for (int a = 0; a < 3; ++a) {
      switch (op) {
        case RES_X_STATIC:
          for (int c : {cALX, cBFX, cETAR, cRW}) C.c(c + a)[oc] = (double)B.c(c + a)[o];
          break;
        case RES_X_SETUP:
          C.c(cRBS + a)[oc] = C.c(cRR + a)[oc] = (double)B.c(cRR + a)[o];
          C.c(cRX + a)[oc] = 0.0;
          break;
        case RES_X_DEMOTE_R: B.c(cRR + a)[o] = (float)C.c(cRR + a)[oc]; break;
        case RES_X_ADD_X: C.c(cRX + a)[oc] += (double)B.c(cRX + a)[o]; break;
        default: B.c(cRX + a)[o] = (float)C.c(cRX + a)[oc]; break;  // RES_X_DEMOTE_X
      }
    }
  });
}

void launch_res_cross(const Dir &D, int op, cudaStream_t st) {
  grids<float>();
  if (op == RES_X_STATIC) k_res_cross<kFull><<<g_grid_tiles, kTileThreads, 0, st>>>(D, op);
  else k_res_cross<kResK><<<g_grid_tiles, kTileThreads, 0, st>>>(D, op);
}

void launch_step_kernel_f32(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int iarg, double darg,
                            ResScratch rs) {
  grids<float>();
  launch_as<float>(k, D, st, ops, iarg, darg, rs);
}

void init_launch_grids_f32() { grids<float>(); }

void launch_res_kmax_f32(const Dir &D, int *out, cudaStream_t st) {
  grids<float>();
  k_res_kmax<float><<<g_grid_tiles, kTileThreads, 0, st>>>(D, out);
}
#else
void launch_res_kmax_f32(const Dir &D, int *out, cudaStream_t st);

void launch_res_kmax(const Dir &D, int precision, int *out, cudaStream_t st) {
  if (precision == kMixed) {
    launch_res_kmax_f32(D, out, st);
  } else {
    grids<double>();
    k_res_kmax<double><<<g_grid_tiles, kTileThreads, 0, st>>>(D, out);
  }
}

void launch_step_kernel_f32(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int iarg, double darg,
                            ResScratch rs);

void launch_step_kernel(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int precision, int iarg,
                        double darg, ResScratch rs) {
  if (precision == kMixed) {
    launch_step_kernel_f32(k, D, st, ops, iarg, darg, rs);
  } else {
    grids<double>();
    launch_as<double>(k, D, st, ops, iarg, darg, rs);
  }
}

void init_launch_grids_f32();

void init_launch_grids() {
  grids<double>();
  init_launch_grids_f32();
}

int res_dot_grid() {
  grids<double>();
  return g_grid_tiles;
}

const char *step_kernel_name(StepKernel k) {
  static const char *names[] = {"k_face_emf", "k_edge_emf", "k_hall_edge", "k_add_hall",
                                "k_fluid",    "k_bface",    "k_bcell_jedge", "k_jcell",   "k_pv_uplus",
                                "k_sync",     "k_flip",     "k_retire",      "k_face_normals", "k_div_b",
                                "k_res_seed", "k_res_w",    "k_res_vec",     "k_res_db",   "k_res_dj",
                                "k_res_q",    "k_res_dot",  "k_res_sum",     "k_res_copyb", "k_res_bupdate",
                                "k_res_cg",   "k_res_pupd_e", "k_phys",      "k_sing_setup", "k_sing_emf",
                                "k_sing_j",   "k_res_clearb", "k_res_cg_sum"};
  static_assert(sizeof(names) / sizeof(names[0]) == SK_COUNT, "a name per kernel");
  return (k >= 0 && k < SK_COUNT) ? names[k] : "?";
}
#endif  // MHD_KERNELS_F32

}  // namespace mhd
