// Hall edge EMF with library-owned static scratch: an entry point that
// allocates no device memory.
//
// Who needs it: callers that are not allowed to call cudaMalloc / cudaFree
// themselves — for example a host framework that reserves the whole device
// memory for its own pool at start-up and hands out only pointers into that
// pool, or a latency-bound request loop that must not allocate per call
// because cudaMalloc can synchronise the device and can fail once memory is
// fragmented.  Such a caller owns its input and output buffers (any device
// pointers it can obtain) and calls mhd_hall_emf_static_scratch; the only
// intermediate the computation needs, the cell-centred Hall field
// alpha (J x B) and the diffusivity scale |alpha||B| on the cells around the
// owned edges, lives in a file-scope __device__ array of fixed size instead
// of being allocated.
//
// The arithmetic is the same as the context path (the Hall cell field of
// k_pv_uplus and k_hall_edge in mhd_kernels.cu, i.e. BuildHallFaceEMF_Rusanov_diff_ of the reference,
// Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:58-400), in the
// same operation order, so the two agree bitwise on the edges both write.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "mercury_mhd.h"
#include "mhd_error.h"

namespace {

// Scratch: 4 doubles (Ehc x, y, z and beta) per cell of the range the edge
// pass reads, [-1, n]^3 (n + 2 cells per axis), at most
// MHD_HALL_SCRATCH_MAX_CELLS cells (32 MiB).
// Every GPU that loads the library holds this array until the process exits.
__device__ __align__(256) double g_hall_scratch[4 * (size_t)MHD_HALL_SCRATCH_MAX_CELLS];

constexpr int kMaxDevices = 64;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

struct View {
  int n0, n1, n2, G;
  int64_t si, sj;
  int e1, e2;  // extents of the scratch cell range [-1, n] along j and k
  __device__ __forceinline__ int64_t off(int i, int j, int k) const {
    return (int64_t)(i + G) * si + (int64_t)(j + G) * sj + (k + G);
  }
  // compact scratch index of cell (i, j, k) in [-1, n]^3
  __device__ __forceinline__ int64_t soff(int i, int j, int k) const {
    return ((int64_t)(i + 1) * e1 + (j + 1)) * e2 + (k + 1);
  }
};

// Pass 1: alpha (J x B) and |alpha||B| on every cell of [-1, n]^3, the cells
// around the owned edges.
__global__ void k_hall_cell_static(mhd_hall_block in, View v, double *scratch, int64_t ncell) {
  const int k = -1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = -1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int i = -1 + (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i > v.n0 || j > v.n1 || k > v.n2) return;
  const int64_t o = v.off(i, j, k);
  // Hall_Num_Limiter (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:111-157): only ne_eff is needed
  const double rH = dmax(in.rho_H[o], 0.0), rN = dmax(in.rho_Na[o], 0.0);
  const double nH = rH / in.M_H * in.M_ref;
  const double nNa = rN / in.M_Na * in.M_ref;
  const double ne_true = nH + nNa;
  const double ne_eff = sqrt(ne_true * ne_true + in.ne_hall_floor * in.ne_hall_floor);
  const double alpha = in.hall_coef / ne_eff;
  const double Jx = in.J_cell[0][o], Jy = in.J_cell[1][o], Jz = in.J_cell[2][o];
  const double Bx = in.B_cell[0][o], By = in.B_cell[1][o], Bz = in.B_cell[2][o];
  const int64_t s = v.soff(i, j, k);
  scratch[s] = alpha * (Jy * Bz - Jz * By);
  scratch[ncell + s] = alpha * (Jz * Bx - Jx * Bz);
  scratch[2 * ncell + s] = alpha * (Jx * By - Jy * Bx);
  scratch[3 * ncell + s] = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
}

// Pass 2: Hall edge EMF with whistler-LLF diffusion (C_wh = 0.1) and the
// per-edge taper, on the owned edges of all three families.
__global__ void k_hall_edge_static(mhd_hall_block in, View v, const double *scratch, int64_t ncell,
                                   double *out_xi, double *out_eta, double *out_zeta) {
  const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int i = (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i > v.n0 || j > v.n1 || k > v.n2) return;
  const double eps = 1e-14, Cwh = 0.1;
  const int64_t o = v.off(i, j, k);
#define EHC(q, a, b, c) scratch[(int64_t)(q) * ncell + v.soff((a), (b), (c))]
#define HB(a, b, c) scratch[3 * ncell + v.soff((a), (b), (c))]
#define F(p, a, b, c) (p)[v.off((a), (b), (c))]
  if (i < v.n0) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (EHC(q, i, j - 1, k - 1) + EHC(q, i, j - 1, k) + EHC(q, i, j, k - 1) + EHC(q, i, j, k));
    const double Ecen = Ec[0] * in.dr_xi[0][o] + Ec[1] * in.dr_xi[1][o] + Ec[2] * in.dr_xi[2][o];
    const double be = dmax(dmax(HB(i, j - 1, k - 1), HB(i, j - 1, k)), dmax(HB(i, j, k - 1), HB(i, j, k)));
    const double L = dmax(in.dl[0][o], eps);
    const double Abz = 0.5 * (F(in.area[2], i, j, k) + F(in.area[2], i, j - 1, k));
    const double ihe = L / dmax(Abz, eps);
    const double mue = Cwh * be * ihe * ihe;
    const double Abe = 0.5 * (F(in.area[1], i, j, k) + F(in.area[1], i, j, k - 1));
    const double ihz = L / dmax(Abe, eps);
    const double muz = Cwh * be * ihz * ihz;
    const double d1 = F(in.B_face[2], i, j, k) - F(in.B_face[2], i, j - 1, k);
    const double d2 = F(in.B_face[1], i, j, k) - F(in.B_face[1], i, j, k - 1);
    out_xi[o] = in.taper[0][o] * (Ecen + 0.5 * mue * d1 - 0.5 * muz * d2);
  }
  if (j < v.n1) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (EHC(q, i - 1, j, k - 1) + EHC(q, i - 1, j, k) + EHC(q, i, j, k - 1) + EHC(q, i, j, k));
    const double Ecen = Ec[0] * in.dr_eta[0][o] + Ec[1] * in.dr_eta[1][o] + Ec[2] * in.dr_eta[2][o];
    const double be = dmax(dmax(HB(i - 1, j, k - 1), HB(i - 1, j, k)), dmax(HB(i, j, k - 1), HB(i, j, k)));
    const double L = dmax(in.dl[1][o], eps);
    const double Abx = 0.5 * (F(in.area[0], i, j, k) + F(in.area[0], i, j, k - 1));
    const double ihz = L / dmax(Abx, eps);
    const double muz = Cwh * be * ihz * ihz;
    const double Abz = 0.5 * (F(in.area[2], i, j, k) + F(in.area[2], i - 1, j, k));
    const double ihx = L / dmax(Abz, eps);
    const double mux = Cwh * be * ihx * ihx;
    const double d1 = F(in.B_face[0], i, j, k) - F(in.B_face[0], i, j, k - 1);
    const double d2 = F(in.B_face[2], i, j, k) - F(in.B_face[2], i - 1, j, k);
    out_eta[o] = in.taper[1][o] * (Ecen + 0.5 * muz * d1 - 0.5 * mux * d2);
  }
  if (k < v.n2) {
    double Ec[3];
    for (int q = 0; q < 3; ++q)
      Ec[q] = 0.25 * (EHC(q, i - 1, j - 1, k) + EHC(q, i - 1, j, k) + EHC(q, i, j - 1, k) + EHC(q, i, j, k));
    const double Ecen = Ec[0] * in.dr_zeta[0][o] + Ec[1] * in.dr_zeta[1][o] + Ec[2] * in.dr_zeta[2][o];
    const double be = dmax(dmax(HB(i - 1, j - 1, k), HB(i - 1, j, k)), dmax(HB(i, j - 1, k), HB(i, j, k)));
    const double L = dmax(in.dl[2][o], eps);
    const double Abe = 0.5 * (F(in.area[1], i, j, k) + F(in.area[1], i - 1, j, k));
    const double ihx = L / dmax(Abe, eps);
    const double mux = Cwh * be * ihx * ihx;
    const double Abx = 0.5 * (F(in.area[0], i, j, k) + F(in.area[0], i, j - 1, k));
    const double ihe = L / dmax(Abx, eps);
    const double mue = Cwh * be * ihe * ihe;
    const double d1 = F(in.B_face[1], i, j, k) - F(in.B_face[1], i - 1, j, k);
    const double d2 = F(in.B_face[0], i, j, k) - F(in.B_face[0], i, j - 1, k);
    out_zeta[o] = in.taper[2][o] * (Ecen + 0.5 * mux * d1 - 0.5 * mue * d2);
  }
#undef EHC
#undef HB
#undef F
}

// Device address of the static scratch on the current device: looked up
// once per device (cudaGetSymbolAddress, with that device current) and cached.
int scratch_for_current_device(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MHD_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_hall_scratch) != cudaSuccess || !p) return MHD_ERR_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return MHD_OK;
}

}  // namespace

extern "C" int mhd_hall_emf_static_scratch(const mhd_hall_block *in, double *out_xi, double *out_eta,
                                           double *out_zeta, void *stream) {
  using mhd::set_error;
  if (!in || !out_xi || !out_eta || !out_zeta)
    return set_error(MHD_ERR_ARG, "mhd_hall_emf_static_scratch: null block description or output pointer");
  if (in->n[0] < 1 || in->n[1] < 1 || in->n[2] < 1 || in->nghost < 1 || in->G < in->nghost + 1)
    return set_error(MHD_ERR_ARG, "mhd_hall_emf_static_scratch: need n >= 1 per axis, nghost >= 1, G >= nghost + 1");
  // the box layout of mhd_device_view: [-G, n + 1 + G) per axis, k contiguous
  const int64_t bj = (int64_t)in->n[2] + 1 + 2 * (int64_t)in->G, bi = (int64_t)in->n[1] + 1 + 2 * (int64_t)in->G;
  if (in->sj < bj || in->si < in->sj * bi)
    return set_error(MHD_ERR_ARG,
                     "mhd_hall_emf_static_scratch: strides sj=%lld si=%lld smaller than the box (need sj >= %lld, "
                     "si >= sj * %lld)", (long long)in->sj, (long long)in->si, (long long)bj, (long long)bi);
  if (!in->rho_H || !in->rho_Na)
    return set_error(MHD_ERR_ARG, "mhd_hall_emf_static_scratch: null density pointer");
  for (int a = 0; a < 3; ++a)
    if (!in->J_cell[a] || !in->B_cell[a] || !in->B_face[a] || !in->area[a] || !in->dl[a] || !in->taper[a] ||
        !in->dr_xi[a] || !in->dr_eta[a] || !in->dr_zeta[a])
      return set_error(MHD_ERR_ARG, "mhd_hall_emf_static_scratch: null input pointer (component %d)", a);
  const int64_t e0 = (int64_t)in->n[0] + 2, e1 = (int64_t)in->n[1] + 2, e2 = (int64_t)in->n[2] + 2;
  const int64_t ncell = e0 * e1 * e2;
  if (ncell > (int64_t)MHD_HALL_SCRATCH_MAX_CELLS)
    return set_error(MHD_ERR_ARG,
                     "mhd_hall_emf_static_scratch: block of %dx%dx%d cells needs %lld scratch cells ((n + 2) per "
                     "axis), more than the static array's %d", in->n[0], in->n[1], in->n[2], (long long)ncell,
                     MHD_HALL_SCRATCH_MAX_CELLS);
  double *scratch = nullptr;
  if (scratch_for_current_device(&scratch) != MHD_OK)
    return set_error(MHD_ERR_CUDA, "mhd_hall_emf_static_scratch: device address of the static scratch not found "
                                   "(cudaGetDevice / cudaGetSymbolAddress failed)");
  View v;
  v.n0 = in->n[0];
  v.n1 = in->n[1];
  v.n2 = in->n[2];
  v.G = in->G;
  v.si = in->si;
  v.sj = in->sj;
  v.e1 = (int)e1;
  v.e2 = (int)e2;
  cudaStream_t st = (cudaStream_t)stream;
  mhd_hall_block blk = *in;
  const dim3 b3(32, 4, 2);
  // each launch's own status (an earlier, unrelated launch error of the
  // caller is neither reported nor cleared here)
  const dim3 gc((unsigned)((e2 + 31) / 32), (unsigned)((e1 + 3) / 4), (unsigned)((e0 + 1) / 2));
  void *cell_args[] = {&blk, &v, &scratch, (void *)&ncell};
  cudaError_t err = cudaLaunchKernel((const void *)k_hall_cell_static, gc, b3, cell_args, 0, st);
  if (err != cudaSuccess)
    return set_error(MHD_ERR_CUDA, "mhd_hall_emf_static_scratch: cell pass launch: %s", cudaGetErrorString(err));
  const dim3 ge((unsigned)((in->n[2] + 1 + 31) / 32), (unsigned)((in->n[1] + 1 + 3) / 4),
                (unsigned)((in->n[0] + 1 + 1) / 2));
  const double *cscratch = scratch;
  void *edge_args[] = {&blk, &v, (void *)&cscratch, (void *)&ncell, &out_xi, &out_eta, &out_zeta};
  err = cudaLaunchKernel((const void *)k_hall_edge_static, ge, b3, edge_args, 0, st);
  if (err != cudaSuccess)
    return set_error(MHD_ERR_CUDA, "mhd_hall_emf_static_scratch: edge pass launch: %s", cudaGetErrorString(err));
  return MHD_OK;
}
