// Host-side topology builder: flattened sync tables (explicit copy lists,
// the reference's format) and edge alias classes for one block that is
// periodic in every direction, or for a periodic box cut into a lattice of
// aligned blocks, from the walks of mhd_periodic.h.
#include <cstdint>
#include <new>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_layout.cuh"
#include "mhd_parallel.h"
#include "mhd_periodic.h"

#include "mhd_topology_impl.h"

namespace {

using namespace mhd::periodic;

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
  mhd::periodic::alias_classes(n, t->alias_offset, t->alias_member, t->alias_msign, t->alias_owner, t->alias_osign);
}

// The lattice's tables: one task per (block, field component), counted and
// then written in place, as build_groups.
void build_lattice_groups(mhd_topology *t, const int n[3], const Lattice &L, int g) {
  struct Unit {
    const GroupSpec *gs;
    int field, m, blk;
    size_t nh, no, oh, oo;
  };
  std::vector<Unit> units;
  for (int blk = 0; blk < L.blocks(); ++blk)
    for (const auto &gs : kGroups)
      for (int field : gs.fields)
        for (int m = 0; m < mhd::kFieldSpec[field].ncomp; ++m) units.push_back({&gs, field, m, blk, 0, 0, 0, 0});
  const int nu = (int)units.size();
  mhd::parallel_for(nu, [&](int u) {
    Unit &U = units[u];
    walk_lattice(*U.gs, U.field, U.m, n, L, U.blk, g, [&](const mhd_copy &, bool own) { ++(own ? U.no : U.nh); });
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
    walk_lattice(*U.gs, U.field, U.m, n, L, U.blk, g, [&](const mhd_copy &c, bool own) { *(own ? o++ : h++) = c; });
  });
}

}  // namespace

extern "C" int mhd_topology_periodic_block(const int32_t cells[3], int32_t nghost, mhd_topology **out) {
  if (!cells || !out || nghost < 1) return MHD_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (cells[a] < 2) return MHD_ERR_ARG;
  auto *t = new (std::nothrow) mhd_topology();
  if (!t) return MHD_ERR_OOM;
  const int n[3] = {cells[0], cells[1], cells[2]};
  t->res_groups_alias = true;
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

extern "C" int mhd_topology_periodic_lattice(const int32_t cells[3], const int32_t blocks[3], int32_t nghost,
                                             mhd_topology **out) {
  if (!cells || !blocks || !out || nghost < 1) return MHD_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (cells[a] < 2 || blocks[a] < 1) return MHD_ERR_ARG;
  // a block's ghost layers come from its neighbours' owned DOFs, one block away
  for (int a = 0; a < 3; ++a)
    if (cells[a] < nghost) return MHD_ERR_ARG;
  if ((int64_t)blocks[0] * blocks[1] * blocks[2] >= (1 << 15)) return MHD_ERR_ARG;
  auto *t = new (std::nothrow) mhd_topology();
  if (!t) return MHD_ERR_OOM;
  const int n[3] = {cells[0], cells[1], cells[2]};
  const Lattice L{{blocks[0], blocks[1], blocks[2]}};
  t->res_groups_alias = true;
  try {
    build_lattice_groups(t, n, L, nghost);
    alias_classes_lattice(n, L, t->alias_offset, t->alias_member, t->alias_msign, t->alias_owner, t->alias_osign);
  } catch (...) {
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
    d->groups[g].n_phys = (int32_t)t->phys[g].size();
    d->groups[g].phys = t->phys[g].data();
    d->groups[g].n_stash = (int32_t)(t->stash[g].size() / 2);
    d->groups[g].stash = t->stash[g].data();
  }
  if (t->res_groups_alias) {
    d->groups[MHD_SYNC_ERES] = d->groups[MHD_SYNC_EEDGE];
    d->groups[MHD_SYNC_DB] = d->groups[MHD_SYNC_BFACE];
  }
  d->n_staging = t->n_staging;
  d->n_wall = (int32_t)t->wall.size();
  d->wall = t->wall.data();
  mhd_singular_edges &s = d->singular;
  s.n_edges = (int32_t)t->sing_owner.size();
  s.owner = t->sing_owner.data();
  s.owner_sign = t->sing_owner_sign.data();
  s.alias_offset = t->sing_alias_offset.data();
  s.aliases = t->sing_aliases.data();
  s.cell_offset = t->sing_cell_offset.data();
  s.cells = t->sing_cells.data();
  s.face_offset = t->sing_face_offset.data();
  s.faces = t->sing_faces.data();
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
