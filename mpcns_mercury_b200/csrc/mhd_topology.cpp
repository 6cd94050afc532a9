// Host-side topology builder: flattened sync tables and edge alias classes
// for one block that is periodic in every direction.
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
#include <cstdint>
#include <memory>
#include <new>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_layout.cuh"
#include "mhd_parallel.h"

// A copy table whose entries are written once, by the building threads (no
// zero-fill of a freshly allocated table).
struct CopyTable {
  std::unique_ptr<mhd_copy[]> p;
  size_t n = 0;
  void allocate(size_t count) {
    p.reset(count ? new mhd_copy[count] : nullptr);
    n = count;
  }
  mhd_copy *data() const { return p.get(); }
  size_t size() const { return n; }
};

struct mhd_topology {
  CopyTable halo[MHD_NUM_GROUPS], owner[MHD_NUM_GROUPS];
  std::vector<int32_t> alias_offset;
  std::vector<mhd_dof> alias_member, alias_owner;
  std::vector<double> alias_msign, alias_osign;
};

namespace {

struct GroupSpec {
  int group;
  int corner1d;
  std::vector<int> fields;
};

const GroupSpec kGroups[] = {
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
void walk_unit(const GroupSpec &gs, int field, int m, const int n[3], int g, Emit &&emit) {
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

// Every group's tables, one field component per task: a counting pass sizes
// the tables, a second pass writes each component's entries at its offset.
void build_groups(mhd_topology *t, const int n[3], int g) {
  struct Unit {
    const GroupSpec *gs;
    int field, m;
    size_t nh, no, oh, oo;  // counts and offsets in the group's tables
  };
  std::vector<Unit> units;
  for (const auto &gs : kGroups)
    for (int field : gs.fields)
      for (int m = 0; m < mhd::kFieldSpec[field].ncomp; ++m) units.push_back({&gs, field, m, 0, 0, 0, 0});
  const int nu = (int)units.size();
  mhd::parallel_for(nu, [&](int u) {
    Unit &U = units[u];
    walk_unit(*U.gs, U.field, U.m, n, g, [&](const mhd_copy &, bool own) { ++(own ? U.no : U.nh); });
  });
  size_t nh[MHD_NUM_GROUPS] = {}, no[MHD_NUM_GROUPS] = {};
  for (Unit &U : units) {
    U.oh = nh[U.gs->group];
    U.oo = no[U.gs->group];
    nh[U.gs->group] += U.nh;
    no[U.gs->group] += U.no;
  }
  for (int q = 0; q < MHD_NUM_GROUPS; ++q) {
    t->halo[q].allocate(nh[q]);
    t->owner[q].allocate(no[q]);
  }
  mhd::parallel_for(nu, [&](int u) {
    const Unit &U = units[u];
    mhd_copy *h = t->halo[U.gs->group].data() + U.oh, *o = t->owner[U.gs->group].data() + U.oo;
    walk_unit(*U.gs, U.field, U.m, n, g, [&](const mhd_copy &c, bool own) { *(own ? o++ : h++) = c; });
  });
}

void build_alias(mhd_topology *t, const int n[3]) {
  t->alias_offset.push_back(0);
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
            t->alias_member.push_back({axis, 0, p[0], p[1], p[2], 0});
            t->alias_msign.push_back(1.0);
          }
          t->alias_owner.push_back({axis, 0, i, j, k, 0});
          t->alias_osign.push_back(1.0);
          t->alias_offset.push_back((int32_t)t->alias_member.size());
        }
  }
}

}  // namespace

extern "C" int mhd_topology_periodic_block(const int32_t cells[3], int32_t nghost, mhd_topology **out) {
  if (!cells || !out || nghost < 1) return MHD_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (cells[a] < 2) return MHD_ERR_ARG;
  auto *t = new (std::nothrow) mhd_topology();
  if (!t) return MHD_ERR_OOM;
  const int n[3] = {cells[0], cells[1], cells[2]};
  try {
    build_groups(t, n, nghost);
    build_alias(t, n);
  } catch (...) {  // allocation or thread creation failed
    delete t;
    return MHD_ERR_OOM;
  }
  *out = t;
  return MHD_OK;
}

extern "C" int mhd_topology_fill_desc(const mhd_topology *t, mhd_desc *d) {
  if (!t || !d) return MHD_ERR_ARG;
  for (int g = 0; g < MHD_NUM_GROUPS; ++g) {
    d->groups[g].n_halo = (int32_t)t->halo[g].size();
    d->groups[g].halo = t->halo[g].data();
    d->groups[g].n_owner = (int32_t)t->owner[g].size();
    d->groups[g].owner = t->owner[g].data();
  }
  d->edge_aliases.n_classes = (int32_t)t->alias_owner.size();
  d->edge_aliases.offset = t->alias_offset.data();
  d->edge_aliases.member = t->alias_member.data();
  d->edge_aliases.member_sign = t->alias_msign.data();
  d->edge_aliases.owner = t->alias_owner.data();
  d->edge_aliases.owner_sign = t->alias_osign.data();
  return MHD_OK;
}

extern "C" int mhd_topology_destroy(mhd_topology *t) {
  delete t;
  return MHD_OK;
}
