// Launch interface of the FP64 step kernels (mhd_step.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mhd_layout.cuh"

namespace mhd {

// Constants of the step, as calc_physical_constant derives them
// (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48).
struct Consts {
  double gamma, M_H, M_Na, M_ref, T_ref, L_ref, U_ref, B_ref, n_ref, rho_ref, m_Na, k_Boltz, q_e, mu0;
  double state_coeff_H, state_coeff_Na, CFL, hall_coef, momentum_induce_coeff, momentum_hall_coeff;
  double inver_MA2, ne_hall_floor;
  int ambipolar;
};

// Device scalars of one context.
struct Scalars {
  unsigned long long dt_bits;  // running min of the CFL dt (positive double bit pattern)
  double dt, time;
  long long step;
  int status;
  int pad;
};

void launch_timestep(const BlockView &B, const Consts &c, Scalars *S, cudaStream_t st);
void launch_face_emf(const BlockView &B, cudaStream_t st);
void launch_edge_emf(const BlockView &B, const Consts &c, cudaStream_t st);
void launch_hall_cell(const BlockView &B, const Consts &c, int g, cudaStream_t st);
void launch_hall_edge(const BlockView &B, cudaStream_t st);
void launch_add_hall(const BlockView &B, cudaStream_t st);
void launch_update(const BlockView &B, const Consts &c, Scalars *S, int account, cudaStream_t st);
void launch_bcell(const BlockView &B, Scalars *S, int rearm, cudaStream_t st);
void launch_jedge(const BlockView &B, cudaStream_t st);
void launch_jcell(const BlockView &B, cudaStream_t st);
void launch_pv_uplus(const BlockView &B, const Consts &c, int g, cudaStream_t st);
void launch_copy(const int64_t *dst, const int64_t *src, const double *sign, int n, double *arena, int64_t ucur_off,
                 cudaStream_t st);
void launch_alias(const int32_t *offset, const int64_t *member, const double *msign, const int64_t *owner,
                  const double *osign, int n_classes, double *arena, cudaStream_t st);

}  // namespace mhd
