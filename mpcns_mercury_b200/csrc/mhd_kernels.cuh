// Launch interface of the engine's step kernels (mhd_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "mhd_engine.cuh"

namespace mhd {

enum StepKernel {
  SK_FACE_EMF = 0, SK_EDGE_EMF, SK_HALL_CELL, SK_HALL_EDGE, SK_ADD_HALL, SK_FLUID, SK_BFACE, SK_BCELL_JEDGE,
  SK_JCELL, SK_PV_UPLUS, SK_SYNC, SK_FLIP, SK_RETIRE, SK_FACE_NORMALS, SK_DIVB, SK_COUNT
};

// One launch of k_sync runs up to two independent sync operations: a copy
// phase of a group (halo or owner copies) or an edge alias reduction.
enum SyncKind { SYNC_COPY = 0, SYNC_ALIAS = 1 };
struct SyncOp {
  int kind;   // SyncKind
  int arg;    // SYNC_COPY: group; SYNC_ALIAS: 0 = E, 1 = J
  int phase;  // SYNC_COPY: 0 halo copies to the step's depth, 1 owner copies, 2 every halo copy
};
struct SyncOps {
  SyncOp op[2];
  int n;
};

// Launch one engine kernel over the directory D (ops: SK_SYNC only) in the
// batch's precision (Precision).
void launch_step_kernel(StepKernel k, const Dir &D, cudaStream_t st, const SyncOps *ops, int precision);
const char *step_kernel_name(StepKernel k);

}  // namespace mhd
