// Launch interface of the engine's step kernels (mhd_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "mhd_engine.cuh"

namespace mhd {

enum StepKernel {
  SK_FACE_EMF = 0, SK_EDGE_EMF, SK_HALL_CELL, SK_HALL_EDGE, SK_ADD_HALL, SK_FLUID, SK_BFACE, SK_BCELL_JEDGE,
  SK_JCELL, SK_PV_UPLUS, SK_COPY, SK_ALIAS, SK_FLIP, SK_RETIRE, SK_COUNT
};

// Launch one engine kernel over the directory D.  SK_COPY: arg0 = group,
// arg1 = phase (0 halo, 1 owner); SK_ALIAS: arg0 = 0 (E) or 1 (J).
void launch_step_kernel(StepKernel k, const Dir &D, cudaStream_t st, int arg0 = 0, int arg1 = 0);
const char *step_kernel_name(StepKernel k);

}  // namespace mhd
