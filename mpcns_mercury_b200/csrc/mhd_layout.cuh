// Device layout of the MHD step.
//
// Every field component of a block lives in its own array over one uniform
// box of logical indices [-G, n_a + 1 + G) per axis, G = nghost + 1, k
// contiguous (rows padded to 8 doubles = 64 B).  All stagger locations share
// the box, so one (i, j, k) offset addresses the cell, its three lower faces
// and its three lower edges at once, which is what lets stencils of different
// fields fuse.  Each reference FieldBlock (include/3_field/FieldBlock.cpp:5-62)
// is a sub-box of it.
//
// Arena: [U buffer 0 | U buffer 1 | all other components], each region laid
// out block after block.  The conserved states U_H, U_Na are double-buffered so
// the fluid update U^{n+1} = U^n + dt RHS(U^n) is fused with its RHS.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

#include "mercury_mhd.h"

namespace mhd {

constexpr int kNumUComps = 10;  // U_H (5) + U_Na (5)

struct FieldSpec {
  int ncomp;
  int loc;  // mhd_location
};

// ncomp and location of every mhd_field (same order as the enum).
constexpr FieldSpec kFieldSpec[MHD_NUM_FIELDS] = {
    {5, MHD_CELL},      {5, MHD_CELL},      {1, MHD_FACE_XI},   {1, MHD_FACE_ETA},  {1, MHD_FACE_ZETA},
    {5, MHD_CELL},      {5, MHD_CELL},      {3, MHD_CELL},      {3, MHD_CELL},      {3, MHD_CELL},
    {3, MHD_CELL},      {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA}, {1, MHD_EDGE_XI},
    {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA}, {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA},
    {3, MHD_FACE_XI},   {3, MHD_FACE_ETA},  {3, MHD_FACE_ZETA}, {3, MHD_CELL},      {1, MHD_CELL},
    {3, MHD_CELL} /* UCON */, {1, MHD_CELL} /* DIVB */,
    {4, MHD_FACE_XI},   {4, MHD_FACE_ETA},  {4, MHD_FACE_ZETA} /* FNORM */, {1, MHD_NODE} /* PE_NODE */, {9, MHD_CELL} /* AMBI_COEF */,
    {3, MHD_CELL} /* DPE */, {10, MHD_CELL} /* UCON_COEF */,
    {2, MHD_EDGE_XI},   {2, MHD_EDGE_ETA},  {2, MHD_EDGE_ZETA} /* HALL_IH */, {10, MHD_CELL} /* FLUX_METRIC */,
    {1, MHD_CELL},      {3, MHD_FACE_XI},   {3, MHD_FACE_ETA},  {3, MHD_FACE_ZETA}, {1, MHD_FACE_XI},
    {1, MHD_FACE_ETA},  {1, MHD_FACE_ZETA}, {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA},
    {3, MHD_EDGE_XI},   {3, MHD_EDGE_ETA},  {3, MHD_EDGE_ZETA}, {1, MHD_FACE_XI},   {1, MHD_FACE_ETA},
    {1, MHD_FACE_ZETA}, {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA}, {18, MHD_CELL},
    {36, MHD_CELL},     {1, MHD_FACE_XI},   {1, MHD_FACE_ETA},  {1, MHD_FACE_ZETA}, {1, MHD_CELL},
    {1, MHD_CELL},      {1, MHD_CELL},      {1, MHD_CELL},      {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},
    {1, MHD_EDGE_ZETA}, {1, MHD_CELL} /* TAPER_CELL */,
    {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA} /* LOCAL_ETA */,
    {1, MHD_EDGE_XI},   {1, MHD_EDGE_ETA},  {1, MHD_EDGE_ZETA} /* ETA_RES */,
    {3, MHD_EDGE_XI},   {3, MHD_EDGE_XI},   {3, MHD_EDGE_XI},   {3, MHD_EDGE_XI},   {3, MHD_EDGE_XI},
    {3, MHD_FACE_XI} /* RES_W, RES_X, RES_R, RES_P, RES_Q, RES_BSTAR */};

// Stagger: 1 where the location is node-like (n + 1 owned DOFs) along an axis.
constexpr int kStagger[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};

// First component index of each field in the component numbering
// (U_H, U_Na occupy 0..9; everything else follows).
struct CompTable {
  int first[MHD_NUM_FIELDS + 1];
  constexpr CompTable() : first() {
    int c = 0;
    for (int f = 0; f < MHD_NUM_FIELDS; ++f) {
      first[f] = c;
      c += kFieldSpec[f].ncomp;
    }
    first[MHD_NUM_FIELDS] = c;
  }
};
constexpr CompTable kComp{};
constexpr int kNumComps = kComp.first[MHD_NUM_FIELDS];

// One block's box geometry.
struct Box {
  int n[3];   // cells per axis
  int G;      // box ghost width (nghost + 1)
  int ext[3]; // n + 1 + 2G
  int64_t sj, si, total;
};

inline Box make_box(const int n[3], int nghost) {
  Box b;
  b.G = nghost + 1;
  for (int a = 0; a < 3; ++a) {
    b.n[a] = n[a];
    b.ext[a] = n[a] + 1 + 2 * b.G;
  }
  b.sj = (b.ext[2] + 7) / 8 * 8;
  b.si = b.sj * b.ext[1];
  b.total = b.si * b.ext[0];
  return b;
}

// Device view of one block: U (current), Unext (other buffer), M (component
// 10 onward), all with the block's box strides.
struct BlockView {
  double *U;      // 10 components, current buffer
  double *Unext;  // 10 components, other buffer
  double *M;      // components kNumUComps.. of this block
  int64_t total, si, sj;
  int G;
  int n[3];
  __host__ __device__ inline int64_t off(int i, int j, int k) const {
    return (int64_t)(i + G) * si + (int64_t)(j + G) * sj + (k + G);
  }
  // pointer to component `c` (global component numbering) of field data
  __host__ __device__ inline double *comp(int c) const {
    return c < kNumUComps ? U + (int64_t)c * total : M + (int64_t)(c - kNumUComps) * total;
  }
};

}  // namespace mhd
