// Context, device arena and C ABI of the MHD step (include/mercury_mhd.h).
//
// One context = one solve on one GPU: a device arena holding every field
// component of every block (layout in mhd_layout.cuh), the flattened sync and
// alias tables translated to arena offsets, a CUDA stream, and two CUDA graphs
// (one per parity of the double-buffered conserved state) that each replay one
// full StepOnce.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_layout.cuh"
#include "mhd_step.cuh"

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

#define CUDA_TRY(expr)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess) return fail(MHD_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

struct DevTable {
  int64_t *dst = nullptr, *src = nullptr;
  double *sign = nullptr;
  int n = 0;
};
struct DevAlias {
  int32_t *offset = nullptr;
  int64_t *member = nullptr, *owner = nullptr;
  double *msign = nullptr, *osign = nullptr;
  int n = 0;
};

constexpr int64_t kUFlag = int64_t(1) << 62;

// AoS (FieldBlock) <-> SoA box scatter/gather for uploads and downloads.
__global__ void k_scatter_aos(const double *__restrict__ aos, int lo0, int lo1, int lo2, int e0, int e1, int e2, int nc,
                              double *const *__restrict__ dst_comp, int ndst, int64_t si, int64_t sj, int G) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npts = (int64_t)e0 * e1 * e2;
  if (t >= npts) return;
  const int k = (int)(t % e2), j = (int)((t / e2) % e1), i = (int)(t / ((int64_t)e1 * e2));
  const int64_t off = (int64_t)(i + lo0 + G) * si + (int64_t)(j + lo1 + G) * sj + (k + lo2 + G);
  for (int m = 0; m < nc; ++m) {
    const double v = aos[t * nc + m];
    for (int d = 0; d < ndst; ++d) dst_comp[d * nc + m][off] = v;
  }
}
__global__ void k_gather_aos(double *__restrict__ aos, int lo0, int lo1, int lo2, int e0, int e1, int e2, int nc,
                             double *const *__restrict__ src_comp, int64_t si, int64_t sj, int G) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npts = (int64_t)e0 * e1 * e2;
  if (t >= npts) return;
  const int k = (int)(t % e2), j = (int)((t / e2) % e1), i = (int)(t / ((int64_t)e1 * e2));
  const int64_t off = (int64_t)(i + lo0 + G) * si + (int64_t)(j + lo1 + G) * sj + (k + lo2 + G);
  for (int m = 0; m < nc; ++m) aos[t * nc + m] = src_comp[m][off];
}

}  // namespace

struct mhd_ctx {
  int nblocks = 0, nghost = 0;
  std::vector<Box> boxes;
  std::vector<int64_t> ubase, mbase;  // per-block offsets inside the U regions / main region
  int64_t ubuf = 0;                   // elements of one U region (all blocks)
  int64_t main_off = 0;               // element offset of the main region
  int64_t arena_elems = 0;
  double *arena = nullptr;
  Scalars *S = nullptr;
  Consts consts{};
  cudaStream_t stream = nullptr;
  DevTable halo[MHD_NUM_GROUPS], owner[MHD_NUM_GROUPS];
  DevAlias aliasE, aliasJ;
  int ucur = 0;
  bool prepared = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double *staging = nullptr;  // upload / download staging (device)
  size_t staging_elems = 0;
  double **comp_ptrs = nullptr;  // device array of component pointers for scatter/gather
  int kernels_per_step = 0;
  // eager profiling: an event after every launch, labelled by kernel name
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;
  std::vector<const char *> prof_names;
  size_t prof_used = 0;

  BlockView view(int b, int cur) const {
    BlockView v;
    const Box &bx = boxes[b];
    v.U = arena + (int64_t)cur * ubuf + ubase[b];
    v.Unext = arena + (int64_t)(cur ^ 1) * ubuf + ubase[b];
    v.M = arena + main_off + mbase[b];
    v.total = bx.total;
    v.si = bx.si;
    v.sj = bx.sj;
    v.G = bx.G;
    for (int a = 0; a < 3; ++a) v.n[a] = bx.n[a];
    return v;
  }
  // Arena offset of a DOF; U components relative to the U region with the flag bit.
  int64_t dof_offset(const mhd_dof &d, bool *ok) const {
    *ok = false;
    if (d.field < 0 || d.field >= MHD_NUM_FIELDS || d.block < 0 || d.block >= nblocks) return 0;
    if (d.comp < 0 || d.comp >= kFieldSpec[d.field].ncomp) return 0;
    const Box &bx = boxes[d.block];
    const int q[3] = {d.i, d.j, d.k};
    for (int a = 0; a < 3; ++a)
      if (q[a] < -bx.G || q[a] >= bx.n[a] + 1 + bx.G) return 0;
    const int64_t off = (int64_t)(d.i + bx.G) * bx.si + (int64_t)(d.j + bx.G) * bx.sj + (d.k + bx.G);
    const int c = kComp.first[d.field] + d.comp;
    *ok = true;
    if (c < kNumUComps) return (ubase[d.block] + (int64_t)c * bx.total + off) | kUFlag;
    return main_off + mbase[d.block] + (int64_t)(c - kNumUComps) * bx.total + off;
  }
  double *comp_ptr(int b, int c, int cur) const {
    if (c < kNumUComps) return arena + (int64_t)cur * ubuf + ubase[b] + (int64_t)c * boxes[b].total;
    return arena + main_off + mbase[b] + (int64_t)(c - kNumUComps) * boxes[b].total;
  }
};

namespace {

// After a launch: in profiling mode record an event labelled `name`.
void mark(mhd_ctx *ctx, const char *name) {
  if (!ctx->profiling) return;
  if (ctx->prof_used == ctx->prof_events.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->prof_events.push_back(e);
    ctx->prof_names.push_back(name);
  }
  ctx->prof_names[ctx->prof_used] = name;
  cudaEventRecord(ctx->prof_events[ctx->prof_used++], ctx->stream);
}

int upload_table(const mhd_copy *tab, int n, const mhd_ctx *ctx, DevTable *out) {
  out->n = n;
  if (n <= 0) return MHD_OK;
  std::vector<int64_t> dst(n), src(n);
  std::vector<double> sign(n);
  for (int t = 0; t < n; ++t) {
    bool ok1, ok2;
    dst[t] = ctx->dof_offset(tab[t].dst, &ok1);
    src[t] = ctx->dof_offset(tab[t].src, &ok2);
    if (!ok1 || !ok2) return fail(MHD_ERR_ARG, "sync table entry %d out of range", t);
    sign[t] = tab[t].sign;
  }
  CUDA_TRY(cudaMalloc(&out->dst, sizeof(int64_t) * n));
  CUDA_TRY(cudaMalloc(&out->src, sizeof(int64_t) * n));
  CUDA_TRY(cudaMalloc(&out->sign, sizeof(double) * n));
  CUDA_TRY(cudaMemcpy(out->dst, dst.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->src, src.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->sign, sign.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  return MHD_OK;
}

int upload_alias(const mhd_alias_classes &a, const int fields[3], const mhd_ctx *ctx, DevAlias *out) {
  out->n = a.n_classes;
  if (a.n_classes <= 0) return MHD_OK;
  const int nm = a.offset[a.n_classes];
  std::vector<int64_t> mem(nm), own(a.n_classes);
  for (int q = 0; q < nm; ++q) {
    mhd_dof d = a.member[q];
    if (d.field < 0 || d.field > 2) return fail(MHD_ERR_ARG, "alias member %d: axis %d", q, d.field);
    d.field = fields[d.field];
    bool ok;
    mem[q] = ctx->dof_offset(d, &ok);
    if (!ok || (mem[q] & kUFlag)) return fail(MHD_ERR_ARG, "alias member %d out of range", q);
  }
  for (int c = 0; c < a.n_classes; ++c) {
    mhd_dof d = a.owner[c];
    if (d.field < 0 || d.field > 2) return fail(MHD_ERR_ARG, "alias owner %d: axis %d", c, d.field);
    d.field = fields[d.field];
    bool ok;
    own[c] = ctx->dof_offset(d, &ok);
    if (!ok) return fail(MHD_ERR_ARG, "alias owner %d out of range", c);
  }
  CUDA_TRY(cudaMalloc(&out->offset, sizeof(int32_t) * (a.n_classes + 1)));
  CUDA_TRY(cudaMalloc(&out->member, sizeof(int64_t) * nm));
  CUDA_TRY(cudaMalloc(&out->msign, sizeof(double) * nm));
  CUDA_TRY(cudaMalloc(&out->owner, sizeof(int64_t) * a.n_classes));
  CUDA_TRY(cudaMalloc(&out->osign, sizeof(double) * a.n_classes));
  CUDA_TRY(cudaMemcpy(out->offset, a.offset, sizeof(int32_t) * (a.n_classes + 1), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->member, mem.data(), sizeof(int64_t) * nm, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->msign, a.member_sign, sizeof(double) * nm, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->owner, own.data(), sizeof(int64_t) * a.n_classes, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(out->osign, a.owner_sign, sizeof(double) * a.n_classes, cudaMemcpyHostToDevice));
  return MHD_OK;
}

void free_table(DevTable &t) {
  cudaFree(t.dst);
  cudaFree(t.src);
  cudaFree(t.sign);
  t = DevTable{};
}
void free_alias(DevAlias &a) {
  cudaFree(a.offset);
  cudaFree(a.member);
  cudaFree(a.msign);
  cudaFree(a.owner);
  cudaFree(a.osign);
  a = DevAlias{};
}

// MercuryBoundary::Sync(group): halo copies then owner copies.
int enqueue_sync(mhd_ctx *ctx, int g, int cur, int *nk) {
  const int64_t ucur_off = (int64_t)cur * ctx->ubuf;
  if (ctx->halo[g].n) {
    launch_copy(ctx->halo[g].dst, ctx->halo[g].src, ctx->halo[g].sign, ctx->halo[g].n, ctx->arena, ucur_off, ctx->stream);
    mark(ctx, "k_copy(halo)");
    ++*nk;
  }
  if (ctx->owner[g].n) {
    launch_copy(ctx->owner[g].dst, ctx->owner[g].src, ctx->owner[g].sign, ctx->owner[g].n, ctx->arena, ucur_off,
                ctx->stream);
    mark(ctx, "k_copy(owner)");
    ++*nk;
  }
  return MHD_OK;
}

// UpdateDerivedFields_ (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:309-321) on buffer `cur`.
void enqueue_derived(mhd_ctx *ctx, int cur, int *nk) {
  cudaStream_t st = ctx->stream;
  for (int b = 0; b < ctx->nblocks; ++b, ++*nk) {
    launch_bcell(ctx->view(b, cur), ctx->S, b == 0, st);
    mark(ctx, "k_bcell");
  }
  enqueue_sync(ctx, MHD_SYNC_B_CELL, cur, nk);
  for (int b = 0; b < ctx->nblocks; ++b, ++*nk) {
    launch_jedge(ctx->view(b, cur), st);
    mark(ctx, "k_jedge");
  }
  if (ctx->aliasJ.n) {
    launch_alias(ctx->aliasJ.offset, ctx->aliasJ.member, ctx->aliasJ.msign, ctx->aliasJ.owner, ctx->aliasJ.osign,
                 ctx->aliasJ.n, ctx->arena, st);
    mark(ctx, "k_alias(J)");
    ++*nk;
  }
  enqueue_sync(ctx, MHD_SYNC_JEDGE, cur, nk);
  for (int b = 0; b < ctx->nblocks; ++b, ++*nk) {
    launch_jcell(ctx->view(b, cur), st);
    mark(ctx, "k_jcell");
  }
  enqueue_sync(ctx, MHD_SYNC_J_CELL, cur, nk);
  for (int b = 0; b < ctx->nblocks; ++b, ++*nk) {
    launch_pv_uplus(ctx->view(b, cur), ctx->consts, ctx->nghost, st);
    mark(ctx, "k_pv_uplus");
  }
}

// StepOnce (Z4_Mercury/src/MercurySolver_Driver.cpp:21-61), state in buffer `cur`
// on entry and in buffer cur^1 on exit.
void enqueue_step(mhd_ctx *ctx, int cur, int *nk) {
  cudaStream_t st = ctx->stream;
  const int nb = ctx->nblocks;
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_timestep(ctx->view(b, cur), ctx->consts, ctx->S, st);
    mark(ctx, "k_timestep");
  }
  // AssembleRHS_Induction_CT_ (Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:90-171)
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_face_emf(ctx->view(b, cur), st);
    mark(ctx, "k_face_emf");
  }
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_edge_emf(ctx->view(b, cur), ctx->consts, st);
    mark(ctx, "k_edge_emf");
  }
  if (ctx->aliasE.n) {
    launch_alias(ctx->aliasE.offset, ctx->aliasE.member, ctx->aliasE.msign, ctx->aliasE.owner, ctx->aliasE.osign,
                 ctx->aliasE.n, ctx->arena, st);
    mark(ctx, "k_alias(E)");
    ++*nk;
  }
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_hall_cell(ctx->view(b, cur), ctx->consts, ctx->nghost, st);
    mark(ctx, "k_hall_cell");
  }
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_hall_edge(ctx->view(b, cur), st);
    mark(ctx, "k_hall_edge");
  }
  enqueue_sync(ctx, MHD_SYNC_EHALL, cur, nk);
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_add_hall(ctx->view(b, cur), st);
    mark(ctx, "k_add_hall");
  }
  enqueue_sync(ctx, MHD_SYNC_EEDGE, cur, nk);
  // fluid RHS + Euler update into the other buffer, B_face update in place
  for (int b = 0; b < nb; ++b, ++*nk) {
    launch_update(ctx->view(b, cur), ctx->consts, ctx->S, b == 0, st);
    mark(ctx, "k_update");
  }
  const int nxt = cur ^ 1;
  enqueue_sync(ctx, MHD_SYNC_UCELL, nxt, nk);
  enqueue_sync(ctx, MHD_SYNC_BFACE, nxt, nk);
  enqueue_derived(ctx, nxt, nk);
}

int check_status(mhd_ctx *ctx) {
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, ctx->S, sizeof s, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (s.status) return fail(s.status, "device status %d at step %lld (dt=%g)", s.status, s.step, s.dt);
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

int mhd_ctx_create(const mhd_desc *desc, mhd_ctx **out) {
  if (!desc || !out || desc->n_blocks < 1 || !desc->cells || desc->nghost < 1)
    return fail(MHD_ERR_ARG, "mhd_ctx_create: bad descriptor");
  if (desc->precision != 0) return fail(MHD_ERR_ARG, "mhd_ctx_create: precision %d not available", desc->precision);
  auto *ctx = new (std::nothrow) mhd_ctx();
  if (!ctx) return fail(MHD_ERR_OOM, "host allocation");
  ctx->nblocks = desc->n_blocks;
  ctx->nghost = desc->nghost;
  int64_t u = 0, m = 0;
  for (int b = 0; b < ctx->nblocks; ++b) {
    const int n[3] = {desc->cells[3 * b], desc->cells[3 * b + 1], desc->cells[3 * b + 2]};
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) {
      delete ctx;
      return fail(MHD_ERR_ARG, "block %d: cells %d %d %d", b, n[0], n[1], n[2]);
    }
    Box bx = make_box(n, desc->nghost);
    ctx->boxes.push_back(bx);
    ctx->ubase.push_back(u);
    ctx->mbase.push_back(m);
    u += (int64_t)kNumUComps * bx.total;
    m += (int64_t)(kNumComps - kNumUComps) * bx.total;
  }
  ctx->ubuf = u;
  ctx->main_off = 2 * u;
  ctx->arena_elems = 2 * u + m;
  const mhd_constants &k = desc->constants;
  ctx->consts = Consts{k.gamma,  k.M_H,           k.M_Na,          k.M_ref, k.T_ref, k.L_ref, k.U_ref, k.B_ref,
                       k.n_ref,  k.rho_ref,       k.m_Na,          k.k_Boltz, k.q_e, k.mu0, k.state_coeff_H,
                       k.state_coeff_Na, k.CFL,   k.hall_coef,     k.momentum_induce_coeff, k.momentum_hall_coeff,
                       k.inver_MA2, k.ne_hall_floor, k.ambipolar};
  int rc = MHD_OK;
  auto bail = [&](int code) {
    mhd_ctx_destroy(ctx);
    return code;
  };
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "stream create"));
  if (cudaMalloc(&ctx->arena, sizeof(double) * ctx->arena_elems) != cudaSuccess)
    return bail(fail(MHD_ERR_OOM, "arena of %lld doubles", (long long)ctx->arena_elems));
  if (cudaMemset(ctx->arena, 0, sizeof(double) * ctx->arena_elems) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "arena memset"));
  if (cudaMalloc(&ctx->S, sizeof(Scalars)) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "scalars"));
  Scalars s0{};
  s0.dt_bits = 0;
  if (cudaMemcpy(ctx->S, &s0, sizeof s0, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(MHD_ERR_CUDA, "scalars init"));
  if (cudaMalloc(&ctx->comp_ptrs, sizeof(double *) * 2 * 36) != cudaSuccess) return bail(fail(MHD_ERR_OOM, "ptrs"));
  for (int g = 0; g < MHD_NUM_GROUPS; ++g) {
    if ((rc = upload_table(desc->groups[g].halo, desc->groups[g].n_halo, ctx, &ctx->halo[g])) != MHD_OK) return bail(rc);
    if ((rc = upload_table(desc->groups[g].owner, desc->groups[g].n_owner, ctx, &ctx->owner[g])) != MHD_OK)
      return bail(rc);
  }
  const int ef[3] = {MHD_E_XI, MHD_E_ETA, MHD_E_ZETA}, jf[3] = {MHD_J_XI, MHD_J_ETA, MHD_J_ZETA};
  if ((rc = upload_alias(desc->edge_aliases, ef, ctx, &ctx->aliasE)) != MHD_OK) return bail(rc);
  if ((rc = upload_alias(desc->edge_aliases, jf, ctx, &ctx->aliasJ)) != MHD_OK) return bail(rc);
  *out = ctx;
  return MHD_OK;
}

int mhd_ctx_destroy(mhd_ctx *ctx) {
  if (!ctx) return MHD_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &g : ctx->graph)
    if (g) cudaGraphExecDestroy(g);
  for (int g = 0; g < MHD_NUM_GROUPS; ++g) {
    free_table(ctx->halo[g]);
    free_table(ctx->owner[g]);
  }
  free_alias(ctx->aliasE);
  free_alias(ctx->aliasJ);
  for (auto e : ctx->prof_events) cudaEventDestroy(e);
  cudaFree(ctx->arena);
  cudaFree(ctx->S);
  cudaFree(ctx->staging);
  cudaFree(ctx->comp_ptrs);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MHD_OK;
}

static int xfer_check(mhd_ctx *ctx, int field, int block, const int32_t lo[3], const int32_t hi[3], int ncomp) {
  if (!ctx || field < 0 || field >= MHD_NUM_FIELDS || block < 0 || block >= ctx->nblocks || !lo || !hi)
    return fail(MHD_ERR_ARG, "transfer: bad arguments");
  if (ncomp != kFieldSpec[field].ncomp) return fail(MHD_ERR_ARG, "field %d has %d components, got %d", field,
                                                    kFieldSpec[field].ncomp, ncomp);
  const Box &bx = ctx->boxes[block];
  for (int a = 0; a < 3; ++a)
    if (lo[a] < -bx.G || hi[a] > bx.n[a] + 1 + bx.G || hi[a] <= lo[a])
      return fail(MHD_ERR_ARG, "transfer range [%d,%d) outside the block box on axis %d", lo[a], hi[a], a);
  return MHD_OK;
}

static int ensure_staging(mhd_ctx *ctx, size_t elems) {
  if (elems <= ctx->staging_elems) return MHD_OK;
  cudaFree(ctx->staging);
  ctx->staging = nullptr;
  ctx->staging_elems = 0;
  if (cudaMalloc(&ctx->staging, sizeof(double) * elems) != cudaSuccess)
    return fail(MHD_ERR_OOM, "staging of %zu doubles", elems);
  ctx->staging_elems = elems;
  return MHD_OK;
}

int mhd_upload_field(mhd_ctx *ctx, int field, int block, const double *data, const int32_t lo[3], const int32_t hi[3],
                     int ncomp) {
  int rc = xfer_check(ctx, field, block, lo, hi, ncomp);
  if (rc) return rc;
  if (!data) return fail(MHD_ERR_ARG, "upload: null data");
  const int e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  if ((rc = ensure_staging(ctx, npts * ncomp))) return rc;
  CUDA_TRY(cudaMemcpyAsync(ctx->staging, data, sizeof(double) * npts * ncomp, cudaMemcpyHostToDevice, ctx->stream));
  // U components go to both buffers (ghost corners never written by the step
  // must be identical in both).
  const int c0 = kComp.first[field];
  const int ndst = c0 < kNumUComps ? 2 : 1;
  double *ptrs[72];
  for (int d = 0; d < ndst; ++d)
    for (int m = 0; m < ncomp; ++m) ptrs[d * ncomp + m] = ctx->comp_ptr(block, c0 + m, d == 0 ? ctx->ucur : ctx->ucur ^ 1);
  CUDA_TRY(cudaMemcpyAsync(ctx->comp_ptrs, ptrs, sizeof(double *) * ndst * ncomp, cudaMemcpyHostToDevice, ctx->stream));
  const Box &bx = ctx->boxes[block];
  k_scatter_aos<<<(unsigned)((npts + 255) / 256), 256, 0, ctx->stream>>>(ctx->staging, lo[0], lo[1], lo[2], e[0], e[1],
                                                                         e[2], ncomp, ctx->comp_ptrs, ndst, bx.si, bx.sj,
                                                                         bx.G);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->prepared = false;
  return MHD_OK;
}

int mhd_download_field(mhd_ctx *ctx, int field, int block, double *data, const int32_t lo[3], const int32_t hi[3],
                       int ncomp) {
  int rc = xfer_check(ctx, field, block, lo, hi, ncomp);
  if (rc) return rc;
  if (!data) return fail(MHD_ERR_ARG, "download: null data");
  const int e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const size_t npts = (size_t)e[0] * e[1] * e[2];
  if ((rc = ensure_staging(ctx, npts * ncomp))) return rc;
  const int c0 = kComp.first[field];
  double *ptrs[36];
  for (int m = 0; m < ncomp; ++m) ptrs[m] = ctx->comp_ptr(block, c0 + m, ctx->ucur);
  CUDA_TRY(cudaMemcpyAsync(ctx->comp_ptrs, ptrs, sizeof(double *) * ncomp, cudaMemcpyHostToDevice, ctx->stream));
  const Box &bx = ctx->boxes[block];
  k_gather_aos<<<(unsigned)((npts + 255) / 256), 256, 0, ctx->stream>>>(ctx->staging, lo[0], lo[1], lo[2], e[0], e[1],
                                                                        e[2], ncomp, ctx->comp_ptrs, bx.si, bx.sj, bx.G);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(data, ctx->staging, sizeof(double) * npts * ncomp, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MHD_OK;
}

int mhd_prepare(mhd_ctx *ctx, double time, int64_t step) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  Scalars s0{};
  s0.dt_bits = (unsigned long long)0;
  s0.time = time;
  s0.step = step;
  CUDA_TRY(cudaMemcpyAsync(ctx->S, &s0, sizeof s0, cudaMemcpyHostToDevice, ctx->stream));
  int nk = 0;
  enqueue_derived(ctx, ctx->ucur, &nk);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->prepared = true;
  return MHD_OK;
}

static int build_graph(mhd_ctx *ctx, int cur) {
  if (ctx->graph[cur]) return MHD_OK;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int nk = 0;
  enqueue_step(ctx, cur, &nk);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&ctx->graph[cur], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  ctx->kernels_per_step = nk;
  return MHD_OK;
}

int mhd_step_async(mhd_ctx *ctx, int nsteps) {
  if (!ctx || nsteps < 0) return fail(MHD_ERR_ARG, "mhd_step: bad arguments");
  if (!ctx->prepared) return fail(MHD_ERR_STATE, "mhd_step before mhd_prepare");
  int rc;
  for (int s = 0; s < nsteps; ++s) {
    if ((rc = build_graph(ctx, ctx->ucur))) return rc;
    CUDA_TRY(cudaGraphLaunch(ctx->graph[ctx->ucur], ctx->stream));
    ctx->ucur ^= 1;
  }
  return MHD_OK;
}

int mhd_synchronize(mhd_ctx *ctx) {
  if (!ctx) return fail(MHD_ERR_ARG, "null ctx");
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return check_status(ctx);
}

int mhd_step(mhd_ctx *ctx, int nsteps, double *dt_out) {
  int rc = mhd_step_async(ctx, nsteps);
  if (rc) return rc;
  if ((rc = mhd_synchronize(ctx))) return rc;
  if (dt_out) {
    Scalars s;
    CUDA_TRY(cudaMemcpy(&s, ctx->S, sizeof s, cudaMemcpyDeviceToHost));
    *dt_out = s.dt;
  }
  return MHD_OK;
}

int mhd_step_profiled(mhd_ctx *ctx, int nsteps, int max_kernels, float *kernel_ms, const char **kernel_names,
                      int *n_kernels) {
  if (!ctx || nsteps < 1 || !kernel_ms || !n_kernels) return fail(MHD_ERR_ARG, "mhd_step_profiled: bad arguments");
  if (!ctx->prepared) return fail(MHD_ERR_STATE, "mhd_step_profiled before mhd_prepare");
  std::vector<float> acc;
  int per_step = 0;
  for (int s = 0; s < nsteps; ++s) {
    ctx->profiling = true;
    ctx->prof_used = 0;
    mark(ctx, "start");
    int nk = 0;
    enqueue_step(ctx, ctx->ucur, &nk);
    ctx->profiling = false;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->ucur ^= 1;
    per_step = (int)ctx->prof_used - 1;
    if (acc.empty()) acc.assign(per_step, 0.0f);
    for (int q = 0; q < per_step; ++q) {
      float ms = 0.0f;
      CUDA_TRY(cudaEventElapsedTime(&ms, ctx->prof_events[q], ctx->prof_events[q + 1]));
      acc[q] += ms;
    }
  }
  const int n = per_step < max_kernels ? per_step : max_kernels;
  for (int q = 0; q < n; ++q) {
    kernel_ms[q] = acc[q] / (float)nsteps;
    if (kernel_names) kernel_names[q] = ctx->prof_names[q + 1];
  }
  *n_kernels = n;
  return check_status(ctx);
}

int mhd_sync(mhd_ctx *ctx, int group) {
  if (!ctx || group < 0 || group >= MHD_NUM_GROUPS) return fail(MHD_ERR_ARG, "mhd_sync: bad arguments");
  int nk = 0;
  enqueue_sync(ctx, group, ctx->ucur, &nk);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MHD_OK;
}

int mhd_get_info(mhd_ctx *ctx, mhd_info *info) {
  if (!ctx || !info) return fail(MHD_ERR_ARG, "mhd_get_info: bad arguments");
  Scalars s;
  CUDA_TRY(cudaMemcpyAsync(&s, ctx->S, sizeof s, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  info->time = s.time;
  info->dt = s.dt;
  info->step = s.step;
  info->status = s.status;
  info->device_bytes = (int64_t)(ctx->arena_elems * sizeof(double));
  return MHD_OK;
}

void *mhd_stream(mhd_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int mhd_kernels_per_step(mhd_ctx *ctx) {
  if (!ctx) return -1;
  if (!ctx->kernels_per_step && build_graph(ctx, ctx->ucur) != MHD_OK) return -1;
  return ctx->kernels_per_step;
}

int mhd_device_view(mhd_ctx *ctx, int field, int block, int comp, double **base, int32_t *G, int64_t *si, int64_t *sj,
                    int32_t ext[3]) {
  if (!ctx || field < 0 || field >= MHD_NUM_FIELDS || block < 0 || block >= ctx->nblocks || comp < 0 ||
      comp >= kFieldSpec[field].ncomp)
    return fail(MHD_ERR_ARG, "mhd_device_view: bad arguments");
  const Box &bx = ctx->boxes[block];
  if (base) *base = ctx->comp_ptr(block, kComp.first[field] + comp, ctx->ucur);
  if (G) *G = bx.G;
  if (si) *si = bx.si;
  if (sj) *sj = bx.sj;
  if (ext)
    for (int a = 0; a < 3; ++a) ext[a] = bx.ext[a];
  return MHD_OK;
}

}  // extern "C"
