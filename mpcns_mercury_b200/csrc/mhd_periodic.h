// The sync connectivity of one block that is periodic in every direction,
// as walks shared by the explicit copy-table builder (mhd_topology.cpp) and
// the engine's direct table compiler (mhd_batch_add_periodic).
//
// The reference builds the same connectivity from periodic inner patches
// (negative block ids, src/1_grid/1_MPCNS_Grid.cpp:455-464) through its
// topology and halo builders (src/2_topology/TopologyBuilder.cpp:436,
// src/4_halo/core/HaloBuild.cpp:382-540).  On a periodic block those compose
// to the following map, which the unique-code probe of the reference
// reproduces DOF for DOF:
//   halo  : a ghost DOF copies the DOF reached by wrapping every out-of-range
//           index by +-n; along a node-like (staggered) axis the alias layer
//           n is an owned DOF and is kept.  Corner1D groups (Ucell) fill only
//           ghosts that are out of range along exactly one axis.
//   owner : an owned alias DOF (node-like index == n) takes its owner's value
//           (index 0), after the halo copies.
// Edge alias classes (ReduceEdgeAliasCandidatesToOwners_,
// Z4_Mercury/src/physics/MercurySolver_Current.cpp:3-57) group the 2 or 4
// periodic images of a boundary edge; the owner is the image with all
// node-like indices in [0, n) and members are listed in lexicographic (i, j, k)
// order, the order the reference's topology stores them in.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_layout.cuh"

namespace mhd {
namespace periodic {

struct GroupSpec {
  int group;
  int corner1d;
  std::vector<int> fields;
};

inline const GroupSpec kGroups[] = {
    {MHD_SYNC_UCELL, 1, {MHD_U_H, MHD_U_NA}},
    {MHD_SYNC_BFACE, 0, {MHD_B_XI, MHD_B_ETA, MHD_B_ZETA}},
    {MHD_SYNC_EHALL, 0, {MHD_EHALL_XI, MHD_EHALL_ETA, MHD_EHALL_ZETA}},
    {MHD_SYNC_EEDGE, 0, {MHD_E_XI, MHD_E_ETA, MHD_E_ZETA}},
    {MHD_SYNC_B_CELL, 0, {MHD_B_CELL, MHD_BIND_CELL}},
    {MHD_SYNC_JEDGE, 0, {MHD_J_XI, MHD_J_ETA, MHD_J_ZETA}},
    {MHD_SYNC_J_CELL, 0, {MHD_J_CELL}},
};

// One field component of a group: its halo and owner copies are emitted in
// (i, j, k) order, the order of the engine's arena, so the compiled tables
// need no sort.  emit(copy, is_owner) receives every entry.
template <class Emit>
inline void walk_unit(const GroupSpec &gs, int field, int m, const int n[3], int g, Emit &&emit) {
  const int *st = mhd::kStagger[mhd::kFieldSpec[field].loc];
  for (int i = -g; i < n[0] + st[0] + g; ++i)
    for (int j = -g; j < n[1] + st[1] + g; ++j) {
      // (i, j) owned and not an alias index: positions k in [0, n) copy nothing
      const bool ij_in = i >= 0 && i < n[0] + st[0] && j >= 0 && j < n[1] + st[1];
      const bool ij_alias = (st[0] && i == n[0]) || (st[1] && j == n[1]);
      const bool skip_interior = ij_in && !ij_alias;
      for (int k = -g; k < n[2] + st[2] + g; ++k) {
        if (skip_interior && k == 0) k = n[2];
        const int idx[3] = {i, j, k};
        int src[3];
        int nout = 0;
        for (int a = 0; a < 3; ++a) nout += !(idx[a] >= 0 && idx[a] < n[a] + st[a]);
        bool is_owner_copy = false;
        if (nout == 0) {
          bool alias = false;
          for (int a = 0; a < 3; ++a) {
            const bool al = st[a] && idx[a] == n[a];
            src[a] = al ? 0 : idx[a];
            alias = alias || al;
          }
          if (!alias) continue;
          is_owner_copy = true;
        } else {
          if (gs.corner1d && nout > 1) continue;
          for (int a = 0; a < 3; ++a) {
            int v = idx[a];
            if (st[a]) {
              if (v < 0) v += n[a];
              else if (v > n[a]) v -= n[a];
            } else {
              v = ((v % n[a]) + n[a]) % n[a];
            }
            src[a] = v;
          }
        }
        mhd_copy c;
        c.dst = {field, 0, i, j, k, m};
        c.src = {field, 0, src[0], src[1], src[2], m};
        c.sign = 1.0;
        emit(c, is_owner_copy);
      }
    }
}

// Edge alias classes: offsets into the member list, members and owners
// (edge family in mhd_dof.field: 0 xi, 1 eta, 2 zeta) with unit signs.
inline void alias_classes(const int n[3], std::vector<int32_t> &offset, std::vector<mhd_dof> &member,
                          std::vector<double> &member_sign, std::vector<mhd_dof> &owner, std::vector<double> &owner_sign) {
  offset.push_back(0);
  const int locs[3] = {MHD_EDGE_XI, MHD_EDGE_ETA, MHD_EDGE_ZETA};
  for (int axis = 0; axis < 3; ++axis) {
    const int *st = mhd::kStagger[locs[axis]];
    for (int i = 0; i < n[0] + st[0]; ++i)
      for (int j = 0; j < n[1] + st[1]; ++j)
        for (int k = 0; k < n[2] + st[2]; ++k) {
          const int idx[3] = {i, j, k};
          bool ok = true, dup = false;
          int axes[3], na = 0;
          for (int a = 0; a < 3; ++a) {
            if (st[a] && idx[a] == n[a]) ok = false;
            if (st[a] && idx[a] == 0) {
              dup = true;
              axes[na++] = a;
            }
          }
          if (!ok || !dup) continue;
          for (int c = 0; c < (1 << na); ++c) {
            int p[3] = {i, j, k};
            for (int b = 0; b < na; ++b)
              if (c & (1 << (na - 1 - b))) p[axes[b]] = n[axes[b]];
            member.push_back({axis, 0, p[0], p[1], p[2], 0});
            member_sign.push_back(1.0);
          }
          owner.push_back({axis, 0, i, j, k, 0});
          owner_sign.push_back(1.0);
          offset.push_back((int32_t)member.size());
        }
  }
}


// A periodic box cut into nb[0] x nb[1] x nb[2] aligned blocks of n cells
// each (block id (p * nb[1] + q) * nb[2] + r at lattice position (p, q, r)),
// joined face to face by inner patches.  The reference composes its
// face/edge/vertex halo stages on such a lattice to the single-block map
// above with the wrap replaced by a step to the neighbouring block (the
// unique-code probe of the reference reproduces it DOF for DOF):
//   halo  : an index below 0 reads index + n of the block before it along
//           that axis, an index past the owned range reads index - n of the
//           block after it; a node-like index n is kept (the same block's
//           alias DOF); corner ghosts read the diagonal neighbour.
//   owner : an owned DOF on a block boundary plane (node-like index 0 or n)
//           takes the value of its owner among its images in the blocks it
//           touches, the image with the smallest (block, i, j, k).
//   edge alias classes: the same images and owner, members in (block, i, j,
//   k) order.
struct Lattice {
  int nb[3];
  int id(const int pos[3]) const { return (pos[0] * nb[1] + pos[1]) * nb[2] + pos[2]; }
  void pos(int b, int out[3]) const {
    out[2] = b % nb[2];
    out[1] = (b / nb[2]) % nb[1];
    out[0] = b / (nb[1] * nb[2]);
  }
  // the block reached from b by step[a] in {-1, 0, 1} along each axis (wrapping)
  int step(int b, const int d[3]) const {
    int q[3];
    pos(b, q);
    for (int a = 0; a < 3; ++a) q[a] = ((q[a] + d[a]) % nb[a] + nb[a]) % nb[a];
    return id(q);
  }
  int blocks() const { return nb[0] * nb[1] * nb[2]; }
  // The images of owned DOF idx of block b (stagger st): along each
  // node-like axis where idx is 0 (or n) the same DOF is index n (or 0) of
  // the block before (or after); all combinations, as (block, i, j, k).
  int images(int b, const int idx[3], const int *st, const int n[3], int out[8][4]) const {
    int axes[3], na = 0;
    for (int a = 0; a < 3; ++a)
      if (st[a] && (idx[a] == 0 || idx[a] == n[a])) axes[na++] = a;
    for (int c = 0; c < (1 << na); ++c) {
      int p[3] = {idx[0], idx[1], idx[2]}, d[3] = {0, 0, 0};
      for (int q = 0; q < na; ++q)
        if (c & (1 << (na - 1 - q))) {
          const int a = axes[q];
          d[a] = idx[a] == 0 ? -1 : 1;
          p[a] = idx[a] == 0 ? n[a] : 0;
        }
      out[c][0] = step(b, d);
      out[c][1] = p[0];
      out[c][2] = p[1];
      out[c][3] = p[2];
    }
    return 1 << na;
  }
  // The owner of a shared DOF is its image with the smallest (block, i, j,
  // k); true (and the owner in *ob, src) when that is not (b, idx) itself.
  bool owner_of(int b, const int idx[3], const int *st, const int n[3], int *ob, int src[3]) const {
    int im[8][4];
    const int ni = images(b, idx, st, n, im);
    int best = 0;
    for (int c = 1; c < ni; ++c)
      for (int f = 0; f < 4; ++f) {
        if (im[c][f] != im[best][f]) {
          if (im[c][f] < im[best][f]) best = c;
          break;
        }
      }
    const bool self = im[best][0] == b && im[best][1] == idx[0] && im[best][2] == idx[1] && im[best][3] == idx[2];
    *ob = im[best][0];
    for (int a = 0; a < 3; ++a) src[a] = im[best][1 + a];
    return !self;
  }
};

// walk_unit for block blk of a lattice (the same entries for a 1 x 1 x 1
// lattice).  An owned DOF shared with other block positions takes the value
// of its owner, the image with the smallest (block, i, j, k): across a
// periodic wrap that is index 0 (as on one block), across an inner patch the
// block with the smaller id, which is what the reference's probe shows.
template <class Emit>
inline void walk_lattice(const GroupSpec &gs, int field, int m, const int n[3], const Lattice &L, int blk, int g,
                         Emit &&emit) {
  const int *st = mhd::kStagger[mhd::kFieldSpec[field].loc];
  for (int i = -g; i < n[0] + st[0] + g; ++i)
    for (int j = -g; j < n[1] + st[1] + g; ++j) {
      // (i, j) owned and off every block boundary plane: the positions k
      // strictly inside the block copy nothing (index 0 of a node-like axis
      // is shared with the block before)
      const bool ij_in = i >= 0 && i < n[0] + st[0] && j >= 0 && j < n[1] + st[1];
      const bool ij_shared = (st[0] && (i == 0 || i == n[0])) || (st[1] && (j == 0 || j == n[1]));
      const bool skip_interior = ij_in && !ij_shared;
      const int k_first = st[2] ? 1 : 0;
      for (int k = -g; k < n[2] + st[2] + g; ++k) {
        if (skip_interior && k == k_first) k = n[2];
        const int idx[3] = {i, j, k};
        int src[3], d[3] = {0, 0, 0};
        int nout = 0;
        for (int a = 0; a < 3; ++a) nout += !(idx[a] >= 0 && idx[a] < n[a] + st[a]);
        if (nout == 0) {
          // an owned DOF on a block's boundary planes: its owner among its images
          int ob = blk;
          if (!L.owner_of(blk, idx, st, n, &ob, src)) continue;
          mhd_copy c;
          c.dst = {field, blk, i, j, k, m};
          c.src = {field, ob, src[0], src[1], src[2], m};
          c.sign = 1.0;
          emit(c, true);
          continue;
        } else {
          if (gs.corner1d && nout > 1) continue;
          for (int a = 0; a < 3; ++a) {
            int v = idx[a];
            if (v < 0) {
              v += n[a];
              d[a] = -1;
            } else if (v > n[a] || (!st[a] && v == n[a])) {
              v -= n[a];
              d[a] = 1;
            }
            src[a] = v;
          }
        }
        mhd_copy c;
        c.dst = {field, blk, i, j, k, m};
        c.src = {field, L.step(blk, d), src[0], src[1], src[2], m};
        c.sign = 1.0;
        emit(c, false);
      }
    }
}

// alias_classes for every block of a lattice: a class for every edge shared
// by more than one block position, listed once (from its owner), members in
// (block, i, j, k) order.
inline void alias_classes_lattice(const int n[3], const Lattice &L, std::vector<int32_t> &offset,
                                  std::vector<mhd_dof> &member, std::vector<double> &member_sign,
                                  std::vector<mhd_dof> &owner, std::vector<double> &owner_sign) {
  offset.push_back(0);
  const int locs[3] = {MHD_EDGE_XI, MHD_EDGE_ETA, MHD_EDGE_ZETA};
  for (int blk = 0; blk < L.blocks(); ++blk)
    for (int axis = 0; axis < 3; ++axis) {
      const int *st = mhd::kStagger[locs[axis]];
      for (int i = 0; i < n[0] + st[0]; ++i)
        for (int j = 0; j < n[1] + st[1]; ++j)
          for (int k = 0; k < n[2] + st[2]; ++k) {
            const int idx[3] = {i, j, k};
            int im[8][4], ob, src[3];
            const int ni = L.images(blk, idx, st, n, im);
            if (ni < 2 || L.owner_of(blk, idx, st, n, &ob, src)) continue;
            int order[8];
            for (int c = 0; c < ni; ++c) order[c] = c;
            std::sort(order, order + ni, [&](int x, int y) {
              return std::lexicographical_compare(im[x], im[x] + 4, im[y], im[y] + 4);
            });
            for (int c = 0; c < ni; ++c) {
              const int *q = im[order[c]];
              member.push_back({axis, q[0], q[1], q[2], q[3], 0});
              member_sign.push_back(1.0);
            }
            owner.push_back({axis, blk, i, j, k, 0});
            owner_sign.push_back(1.0);
            offset.push_back((int32_t)member.size());
          }
    }
}

}  // namespace periodic
}  // namespace mhd
