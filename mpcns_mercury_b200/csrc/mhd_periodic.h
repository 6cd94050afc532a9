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


}  // namespace periodic
}  // namespace mhd
