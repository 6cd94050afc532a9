// Launch interface of the engine's step kernels (mhd_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "mhd_engine.cuh"

namespace mhd {

enum StepKernel {
  SK_FACE_EMF = 0, SK_EDGE_EMF, SK_HALL_EDGE, SK_ADD_HALL, SK_FLUID, SK_BFACE, SK_BCELL_JEDGE,
  SK_JCELL, SK_PV_UPLUS, SK_SYNC, SK_FLIP, SK_RETIRE, SK_FACE_NORMALS, SK_DIVB,
  // implicit resistive substep
  SK_RES_SEED, SK_RES_W, SK_RES_VEC, SK_RES_DB, SK_RES_DJ, SK_RES_Q, SK_RES_DOT, SK_RES_SUM, SK_RES_COPYB,
  SK_RES_BUPDATE, SK_RES_CG, SK_RES_PUPD_E,
  // grids with physical boundaries and singular edges
  SK_PHYS, SK_SING_SETUP, SK_SING_EMF, SK_SING_J,
  // implicit resistive substep on grids with physical boundaries: zero the ghost faces of dB
  SK_RES_CLEARB,
  // the batched CG's per-solve sums
  SK_RES_CGSUM, SK_COUNT
};

// One launch of k_sync runs up to two independent sync operations: a copy
// phase of a group (halo or owner copies) or an edge alias reduction.
enum SyncKind { SYNC_COPY = 0, SYNC_ALIAS = 1 };
struct SyncOp {
  int kind;   // SyncKind
  int arg;    // SYNC_COPY: group; SYNC_ALIAS: 0 = E, 1 = J
  int phase;  // SYNC_COPY: a CopyPhase (mhd_engine.cuh)
  int prev;   // SYNC_COPY: read U components from the other buffer (1) -- the staged
              // ghosts of Sync(U) inside the step, whose last synced values are there
  int mark;   // SYNC_COPY: write 0 to every destination instead of the copy (marks
              // the phase's destinations, e.g. the non-owner aliases of an owner phase)
};
struct SyncOps {
  SyncOp op[2];
  int n;
};

// Operations of SK_RES_VEC / SK_RES_DOT / SK_RES_COPYB (the arg of the launch).
enum ResVecOp { RES_INIT = 0, RES_E_FROM_P, RES_E_FROM_X, RES_P_FROM_X, RES_RESID };
enum ResCopyOp { RES_SNAPSHOT = 0, RES_RESTORE };

// CG state of one solve on the device (one per slot), for the iteration
// loop run as a CUDA graph over every masked solve at once (k_res_cg,
// k_res_cg_sum, k_res_pupd_e): the host sets tol_factor and max_it (and
// zeros the rest) before the graph and reads it back after.
struct ResCG {
  double rho, alpha, beta;  // W-weighted r.r, step length, direction update
  double r0, rnorm, tol;    // ||r|| at the start and now, stop when rnorm <= tol = tol_factor * r0
  double tol_factor;
  int it, max_it;           // iterations taken, at most max_it
  int done, converged;      // loop over (converged, max_it reached, or breakdown)
};
// The loop's shared counters: slots of k_res_cg_sum reported, solves still iterating.
struct ResCtl {
  unsigned int arrivals;
  int running;
};
// Steps of k_res_cg: CG_INIT: x = 0, p = r, E = p, (r.r)_W and r.r, sets rho, r0, tol;
// CG_PQ: q = A p (its last part, E - eta dJ) and (p.q)_W, sets alpha;
// CG_RR: x += alpha p, r -= alpha q, (r.r)_W and r.r, the stop test and beta.
// k_res_cg writes one partial pair per warp and tile; k_res_cg_sum
// (kCgChunks CTAs per slot) sums a solve's pairs in fixed chunks and a fixed
// order and updates its state; a solve whose loop is over leaves the mask.
enum ResCgOp { CG_INIT = 0, CG_PQ, CG_RR };
constexpr int kWarpsPerTile = kTileThreads / 32;
constexpr int kCgChunks = 32;

// Scratch of the CG dot products: per-CTA partial sums and the two results
// (k_res_dot, one masked solve); the per-slot CG states, the per-warp tile
// partials of the batched loop, its counters and the graph's loop condition.
struct ResScratch {
  double *partial;  // 2 * grid
  double *result;   // 2
  ResCG *cg = nullptr;
  double *tpartial = nullptr;  // 2 per warp of every kResK tile
  ResCtl *ctl = nullptr;
  double *chunks = nullptr;           // 2 per chunk of every slot (k_res_cg_sum)
  unsigned int *sarrivals = nullptr;  // per slot: its chunks summed so far
  unsigned long long handle = 0;  // cudaGraphConditionalHandle of the loop
  int in_graph = 0;               // the CG kernels set the loop condition (launched inside the loop graph)
};

// Launch one engine kernel over the directory D (ops: SK_SYNC only) in the
// batch's precision (Precision); iarg / darg: the operation and scalar of the
// implicit resistive kernels.
void launch_step_kernel(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int precision, int iarg = 0,
                        double darg = 0.0, ResScratch rs = ResScratch{nullptr, nullptr});
int res_dot_grid();
// Mixed-precision implicit substep: moves its coefficients (RES_X_STATIC, at
// prepare) and vectors between every masked solve of the FP32 directory D and
// its FP64 companion (DevSolve::companion; RES_X_SETUP also hands over the
// step's dt) (k_res_cross, FP32 translation unit).
enum ResCrossOp { RES_X_SETUP = 0, RES_X_DEMOTE_R, RES_X_ADD_X, RES_X_DEMOTE_X, RES_X_STATIC };
void launch_res_cross(const Dir &D, int op, cudaStream_t st);
// Per block of the masked solve of D: the largest k of an unknown of the
// implicit substep into out[block] (atomic max; out starts at -1).
void launch_res_kmax(const Dir &D, int precision, int *out, cudaStream_t st);
// Queries every kernel's resident CTAs per SM once (call before any stream capture).
void init_launch_grids();
const char *step_kernel_name(StepKernel k);

}  // namespace mhd
