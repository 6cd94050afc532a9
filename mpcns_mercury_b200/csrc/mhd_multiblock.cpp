// Host-side table builder for general multi-block grids with physical
// boundaries (the cubed-sphere shell): from the blocks, their inner face
// patches and their physical patches it derives what the reference's
// topology and halo layers derive (edge and vertex patches, the halo regions
// of every stage, the face/edge equivalence classes) and then replays every
// sync group of MercuryBoundary::Sync (Z4_Mercury/src/boundary/Boundary_Sync_.cpp:4-110)
// on symbolic DOF values.  Each DOF starts holding its own identity; the
// physical handlers, the halo stages (with the reference's exchange rules:
// a component copy packs every source of a stage before it writes, the form
// triplets write one region after another) and the owner-to-alias copies move
// identities (with orientation signs) exactly as the reference moves values.
// The identity a DOF ends with is the value it must receive, which flattens
// into the descriptor's tables:
//   physical operations   values computed by a handler (farfield states, the
//                         solid-wall state, the farfield EMF)
//   halo copies           ghost <- (sign) source, every source read before any
//                         write of the phase; a copy whose source the phase
//                         overwrites goes through a staging slot
//   owner copies          owned alias <- (sign) owner
// The reference's index mapping is reproduced as it is, including where its
// node-index transform lands a ghost on the neighbour's ghost (face pairs of
// equal orientation on the cubed sphere): such ghosts keep, or exchange, the
// values they held, as in the reference.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <new>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_error.h"
#include "mhd_layout.cuh"
#include "mhd_parallel.h"
#include "mhd_topology_impl.h"

namespace {

// ------------------------------------------------------------------ boxes, transforms
struct IBox {
  int lo[3], hi[3];
  bool empty() const {
    for (int a = 0; a < 3; ++a)
      if (hi[a] <= lo[a]) return true;
    return false;
  }
  bool contains(const int p[3]) const {
    for (int a = 0; a < 3; ++a)
      if (p[a] < lo[a] || p[a] >= hi[a]) return false;
    return true;
  }
  int64_t volume() const {
    return empty() ? 0 : (int64_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
  }
};
IBox intersect(const IBox &a, const IBox &b) {
  IBox r;
  for (int q = 0; q < 3; ++q) {
    r.lo[q] = std::max(a.lo[q], b.lo[q]);
    r.hi[q] = std::min(a.hi[q], b.hi[q]);
  }
  return r;
}

// Node index map this -> nb: nb[perm[a]] = sign[a] * this[a] + off[a]
// (TOPO::IndexTransform, include/2_topology/TopologyTypes.h:92-100).
struct Tr {
  int perm[3], sign[3], off[3];
};
void fwd(const Tr &t, const int p[3], int q[3]) {
  for (int a = 0; a < 3; ++a) q[t.perm[a]] = t.sign[a] * p[a] + t.off[a];
}
void inv(const Tr &t, const int q[3], int p[3]) {
  for (int a = 0; a < 3; ++a) p[a] = t.sign[a] * (q[t.perm[a]] - t.off[a]);
}
// transform_node_box (src/2_topology/TopologyOps.cpp:91-116)
IBox transform_node_box(const IBox &b, const Tr &t) {
  if (b.empty()) return b;
  int p0[3] = {b.lo[0], b.lo[1], b.lo[2]}, p1[3] = {b.hi[0] - 1, b.hi[1] - 1, b.hi[2] - 1}, q0[3], q1[3];
  fwd(t, p0, q0);
  fwd(t, p1, q1);
  IBox r;
  for (int a = 0; a < 3; ++a) {
    r.lo[a] = std::min(q0[a], q1[a]);
    r.hi[a] = std::max(q0[a], q1[a]) + 1;
  }
  return r;
}

int axis_of(int dir) { return std::abs(dir) - 1; }

// LAYOUT::dof_delta (src/0_basic/LayoutTraits.cpp): 1 along the axes where a
// location has one DOF fewer than nodes.
void dof_delta(int loc, int d[3]) {
  for (int a = 0; a < 3; ++a) d[a] = 1 - mhd::kStagger[loc][a];
}
IBox node_box_to_dof_box(int loc, const IBox &nb) {
  int d[3];
  dof_delta(loc, d);
  IBox r = nb;
  for (int a = 0; a < 3; ++a) r.hi[a] = nb.hi[a] - d[a];
  return r;
}
// apply_ghost_strip: a low direction takes [-g, 0), a high one [hi, hi + g)
void ghost_strip(IBox &b, int dir, int g) {
  const int a = axis_of(dir);
  if (dir < 0) {
    b.lo[a] = -g;
    b.hi[a] = 0;
  } else {
    b.lo[a] = b.hi[a];
    b.hi[a] = b.hi[a] + g;
  }
}

// ------------------------------------------------------------------ grid
struct Face {  // an inner face patch (Topology::inner_patches)
  int tb, nb, dir, ndir;
  IBox tbox, nbox;
  Tr tr;
};
struct Edge {  // an edge patch (inner, or physical when nb < 0)
  int tb, nb;
  IBox tbox, nbox;
  Tr tr;
  int d1, d2;
  bool inner;
};
struct Vert {
  int tb, nb;
  IBox tbox, nbox;
  Tr tr;
  int d1, d2, d3;
  bool inner;
};
struct Phys {
  int b, dir, bc;
  IBox box;
};

struct Grid {
  int nb = 0, g = 0;
  std::vector<std::array<int, 3>> n;  // cells per block
  std::vector<Face> faces;
  std::vector<Phys> phys;
  std::vector<Edge> edges, pedges;    // inner, physical edge patches
  std::vector<Vert> verts, pverts;

  // owned DOF box of a location: [0, nodes - delta)
  IBox owned(int b, int loc) const {
    int d[3];
    dof_delta(loc, d);
    IBox r;
    for (int a = 0; a < 3; ++a) {
      r.lo[a] = 0;
      r.hi[a] = n[b][a] + 1 - d[a];
    }
    return r;
  }
  IBox alloc(int b, int loc) const {
    IBox r = owned(b, loc);
    for (int a = 0; a < 3; ++a) {
      r.lo[a] -= g;
      r.hi[a] += g;
    }
    return r;
  }
};

// patch_priority: inner 3 > physical 1 (src/2_topology/TopologyOps.cpp:218-240)
// build_edge_patches (src/2_topology/TopologyEdge.cpp:45-196): every pair of
// face patches of a block on distinct axes whose node boxes meet gives an
// edge patch owned by the higher-priority face (the first on ties).
void build_edge_patches(Grid &G) {
  struct FOB {
    bool inner;
    int tb, nb, dir;
    IBox tbox;
    Tr tr;
  };
  std::map<int, std::vector<FOB>> fob;
  for (const Face &f : G.faces) fob[f.tb].push_back({true, f.tb, f.nb, f.dir, f.tbox, f.tr});
  for (const Phys &p : G.phys) fob[p.b].push_back({false, p.b, -1, p.dir, p.box, Tr{{0, 1, 2}, {1, 1, 1}, {0, 0, 0}}});
  for (auto &kv : fob) {
    auto &fl = kv.second;
    for (size_t i = 0; i < fl.size(); ++i)
      for (size_t j = i + 1; j < fl.size(); ++j) {
        const FOB &f1 = fl[i], &f2 = fl[j];
        if (axis_of(f1.dir) == axis_of(f2.dir)) continue;
        const IBox e = intersect(f1.tbox, f2.tbox);
        if (e.empty()) continue;
        const FOB *own = &f1;
        if ((f2.inner ? 3 : 1) > (f1.inner ? 3 : 1)) own = &f2;
        Edge ep;
        ep.tb = own->tb;
        ep.nb = own->nb;
        ep.tbox = e;
        ep.inner = own->inner;
        if (own->inner) {
          ep.nbox = transform_node_box(e, own->tr);
          ep.tr = own->tr;
        } else {
          ep.nbox = IBox{{0, 0, 0}, {0, 0, 0}};
          ep.tr = Tr{{0, 1, 2}, {1, 1, 1}, {0, 0, 0}};
        }
        ep.d1 = f1.dir;
        ep.d2 = f2.dir;
        if (ep.d1 != own->dir) std::swap(ep.d1, ep.d2);  // order_edge_dirs_by_owner
        (ep.inner ? G.edges : G.pedges).push_back(ep);
      }
  }
}

// build_vertex_patches (src/2_topology/TopologyEdge.cpp:198-345)
void build_vertex_patches(Grid &G) {
  std::map<int, std::vector<const Edge *>> eob;
  for (const Edge &e : G.edges) eob[e.tb].push_back(&e);
  for (const Edge &e : G.pedges) eob[e.tb].push_back(&e);
  auto edge_axis = [](int d1, int d2) {  // the axis (1..3) neither face direction uses
    bool used[4] = {false, false, false, false};
    used[std::abs(d1)] = used[std::abs(d2)] = true;
    return !used[1] ? 1 : !used[2] ? 2 : 3;
  };
  for (auto &kv : eob) {
    auto &el = kv.second;
    if (el.size() < 2) continue;
    std::vector<std::array<int, 3>> used_nodes;
    for (size_t i = 0; i < el.size(); ++i)
      for (size_t j = i + 1; j < el.size(); ++j) {
        const Edge &e1 = *el[i], &e2 = *el[j];
        if (edge_axis(e1.d1, e1.d2) == edge_axis(e2.d1, e2.d2)) continue;
        const IBox v = intersect(e1.tbox, e2.tbox);
        if (v.empty()) continue;
        if (v.hi[0] - v.lo[0] != 1 || v.hi[1] - v.lo[1] != 1 || v.hi[2] - v.lo[2] != 1) continue;
        const std::array<int, 3> node = {v.lo[0], v.lo[1], v.lo[2]};
        if (std::find(used_nodes.begin(), used_nodes.end(), node) != used_nodes.end()) continue;
        used_nodes.push_back(node);
        std::vector<const Edge *> cand = {&e1, &e2};
        for (size_t k = 0; k < el.size(); ++k) {
          if (el[k] == &e1 || el[k] == &e2) continue;
          if (!intersect(el[k]->tbox, v).empty()) cand.push_back(el[k]);
        }
        const Edge *own = cand[0];
        for (size_t k = 1; k < cand.size(); ++k)
          if ((cand[k]->inner ? 3 : 1) > (own->inner ? 3 : 1)) own = cand[k];
        Vert vp;
        vp.tb = own->tb;
        vp.nb = own->nb;
        vp.tbox = v;
        vp.inner = own->inner;
        if (own->inner) {
          vp.nbox = transform_node_box(v, own->tr);
          vp.tr = own->tr;
        } else {
          vp.nbox = IBox{{0, 0, 0}, {0, 0, 0}};
          vp.tr = Tr{{0, 1, 2}, {1, 1, 1}, {0, 0, 0}};
        }
        int by_axis[4] = {0, 0, 0, 0};
        for (const Edge *c : cand)
          for (int d : {c->d1, c->d2})
            if (by_axis[std::abs(d)] == 0) by_axis[std::abs(d)] = d;
        vp.d1 = by_axis[1];
        vp.d2 = by_axis[2];
        vp.d3 = by_axis[3];
        // order_vertex_dirs_by_owner
        const int od = own->d1;
        if (vp.d2 == od) std::swap(vp.d1, vp.d2);
        else if (vp.d3 == od) std::swap(vp.d1, vp.d3);
        (vp.inner ? G.verts : G.pverts).push_back(vp);
      }
  }
}

// number of block-boundary node planes a node box lies on (HaloBuildEdge.cpp:8-25)
int boundary_dir_count(const IBox &b, const std::array<int, 3> &n) {
  int c = 0;
  for (int a = 0; a < 3; ++a) {
    if (b.lo[a] == 0 && b.hi[a] == 1) ++c;
    if (b.lo[a] == n[a] && b.hi[a] == n[a] + 1) ++c;
  }
  return c;
}
// detect_face_direction (src/4_halo/build/HaloBuildTools.cpp:12-37)
int face_direction(const IBox &b, const std::array<int, 3> &n) {
  for (int a = 0; a < 3; ++a) {
    if (b.lo[a] == 0 && b.hi[a] == 1) return -(a + 1);
    if (b.lo[a] == n[a] && b.hi[a] == n[a] + 1) return a + 1;
  }
  throw std::runtime_error("face patch box is not on a block boundary");
}

// A halo region: recv box on block rb, values from block sb through the
// transform (stage 1: the recv block is the patch's neighbour and sources are
// found with the inverse transform; stages 2 and 3: the recv block is the
// patch's own and sources are found with the forward transform).
struct Region {
  int rb, sb;
  Tr tr;
  IBox recv;
};
// The regions of one stage for one location, in patch order.
std::vector<Region> regions(const Grid &G, int stage, int loc) {
  std::vector<Region> out;
  if (stage == 1) {
    for (const Face &f : G.faces) {
      IBox r = node_box_to_dof_box(loc, f.nbox);
      ghost_strip(r, face_direction(f.nbox, G.n[f.nb]), G.g);
      out.push_back({f.nb, f.tb, f.tr, r});
    }
  } else if (stage == 2) {
    for (const Edge &e : G.edges) {
      if (boundary_dir_count(e.tbox, G.n[e.tb]) != 2 || boundary_dir_count(e.nbox, G.n[e.nb]) != 2) continue;
      IBox r = node_box_to_dof_box(loc, e.tbox);
      ghost_strip(r, e.d1, G.g);
      ghost_strip(r, e.d2, G.g);
      out.push_back({e.tb, e.nb, e.tr, r});
    }
  } else {
    for (const Vert &v : G.verts) {
      if (boundary_dir_count(v.tbox, G.n[v.tb]) != 3 || boundary_dir_count(v.nbox, G.n[v.nb]) != 3) continue;
      IBox r = node_box_to_dof_box(loc, v.tbox);
      ghost_strip(r, v.d1, G.g);
      ghost_strip(r, v.d2, G.g);
      ghost_strip(r, v.d3, G.g);
      out.push_back({v.tb, v.nb, v.tr, r});
    }
  }
  return out;
}

// ------------------------------------------------------------------ symbolic values
// A value: the identity of the DOF whose value it is (id), whether it is that
// DOF's value after the physical handlers of the sync (phys) and a sign.
constexpr int64_t kPhysBit = 1;
constexpr int64_t kNegBit = 2;
inline int64_t sym(int64_t id, bool phys, bool neg) { return (id << 2) | (phys ? kPhysBit : 0) | (neg ? kNegBit : 0); }
inline int64_t sym_id(int64_t v) { return v >> 2; }
inline int64_t negate(int64_t v) { return v ^ kNegBit; }

// Value kinds of the group's fields (FieldValueKind of the catalog,
// Z4_Mercury/include/0_MercuryFieldCatalog.h:70-202) and their halo level.
enum Kind { kComponent, kFace2, kEdge1 };
struct GroupDef {
  int group;
  Kind kind;
  int level;                 // highest halo stage (1, 2 or 3)
  std::vector<int> fields;   // in the group's order
  bool owner;                // owner-to-alias sync after the halo stages
};
const GroupDef kGroupDefs[MHD_NUM_GROUPS] = {
    {MHD_SYNC_UCELL, kComponent, 1, {MHD_U_H, MHD_U_NA}, false},
    {MHD_SYNC_BFACE, kFace2, 3, {MHD_B_XI, MHD_B_ETA, MHD_B_ZETA}, true},
    {MHD_SYNC_EHALL, kEdge1, 3, {MHD_EHALL_XI, MHD_EHALL_ETA, MHD_EHALL_ZETA}, true},
    {MHD_SYNC_EEDGE, kEdge1, 3, {MHD_E_XI, MHD_E_ETA, MHD_E_ZETA}, true},
    {MHD_SYNC_B_CELL, kComponent, 3, {MHD_B_CELL, MHD_BIND_CELL}, false},
    {MHD_SYNC_JEDGE, kEdge1, 3, {MHD_J_XI, MHD_J_ETA, MHD_J_ZETA}, true},
    {MHD_SYNC_J_CELL, kComponent, 3, {MHD_J_CELL}, false},
    // the implicit substep's E_res and dB, kept in the E edge and B face arrays
    {MHD_SYNC_ERES, kEdge1, 3, {MHD_E_XI, MHD_E_ETA, MHD_E_ZETA}, true},
    {MHD_SYNC_DB, kFace2, 3, {MHD_B_XI, MHD_B_ETA, MHD_B_ZETA}, true},
    // the background field, synced once after its setup
    {MHD_SYNC_BADD, kFace2, 3, {MHD_BADD_XI, MHD_BADD_ETA, MHD_BADD_ZETA}, true},
};

// The physical handlers MercuryBoundary::InstallHandlers registers for the
// fields of these groups (Z4_Mercury/src/boundary/Boundary_Build.cpp:5-300).
enum Handler { hNop, hCopy, hFarU_H, hFarU_Na, hWallU_H, hWallU_Na, hFarE, hFarBcell, hFarBind, hWallJcell };
Handler handler(int group, int field, int bc, bool resistive) {
  const bool far = bc == MHD_BC_FARFIELD;
  // Eres_*, dB_*, dJ_*: the defaults (Farfield and Pole copy, Coupled-Solid
  // nothing); BC_Farfield_Eedge_set_zerocurl, registered for Eres_* on
  // Farfield, falls back to the copy for every field not named E_*
  if (group == MHD_SYNC_ERES || group == MHD_SYNC_DB) return far ? hCopy : hNop;
  if (group == MHD_SYNC_BADD) return far ? hCopy : hNop;  // Badd_*: the defaults
  switch (field) {
    case MHD_U_H: return far ? hFarU_H : hWallU_H;
    case MHD_U_NA: return far ? hFarU_Na : hWallU_Na;
    case MHD_B_XI: case MHD_B_ETA: case MHD_B_ZETA: return hNop;
    case MHD_E_XI: case MHD_E_ETA: case MHD_E_ZETA: return far ? hFarE : hNop;
    case MHD_B_CELL: return far ? hFarBcell : hNop;
    case MHD_BIND_CELL: return far ? hFarBind : hNop;
    case MHD_J_CELL: return far ? hCopy : (resistive ? hNop : hWallJcell);
    default: return far ? hCopy : hNop;  // E_Hall, J edges
  }
}

struct Replay {
  const Grid &G;
  const GroupDef &gd;
  // one array per (field slot, block, component) over the allocated box
  struct Arr {
    int field, fslot, block, comp, loc;
    IBox box;
    int64_t base;  // identity of its first element
    std::vector<int64_t> v;
    int64_t index(const int p[3]) const {
      return ((int64_t)(p[0] - box.lo[0]) * (box.hi[1] - box.lo[1]) + (p[1] - box.lo[1])) * (box.hi[2] - box.lo[2]) +
             (p[2] - box.lo[2]);
    }
  };
  std::vector<Arr> arrs;
  std::vector<int> first;  // first array of each (fslot, block): first[fslot * nb + b], comps consecutive
  std::vector<mhd_phys_op> phys;
  std::unordered_set<int64_t> phys_written;  // identities a physical operation wrote

  Replay(const Grid &g, const GroupDef &d) : G(g), gd(d) {
    int64_t base = 0;
    first.resize(gd.fields.size() * G.nb);
    for (size_t fs = 0; fs < gd.fields.size(); ++fs)
      for (int b = 0; b < G.nb; ++b) {
        const int f = gd.fields[fs];
        const int loc = mhd::kFieldSpec[f].loc;
        first[fs * G.nb + b] = (int)arrs.size();
        for (int m = 0; m < mhd::kFieldSpec[f].ncomp; ++m) {
          Arr a;
          a.field = f;
          a.fslot = (int)fs;
          a.block = b;
          a.comp = m;
          a.loc = loc;
          a.box = G.alloc(b, loc);
          a.base = base;
          const int64_t vol = a.box.volume();
          a.v.resize(vol);
          for (int64_t q = 0; q < vol; ++q) a.v[q] = sym(base + q, false, false);
          base += vol;
          arrs.push_back(std::move(a));
        }
      }
  }
  Arr &arr(int fslot, int b, int m) { return arrs[first[fslot * G.nb + b] + m]; }
  int ncomp(int fslot) const { return mhd::kFieldSpec[gd.fields[fslot]].ncomp; }

  // identity -> DOF
  mhd_dof dof_of(int64_t id) const {
    size_t lo = 0, hi = arrs.size();
    while (hi - lo > 1) {
      const size_t mid = (lo + hi) / 2;
      if (arrs[mid].base <= id) lo = mid; else hi = mid;
    }
    const Arr &a = arrs[lo];
    int64_t q = id - a.base;
    const int e1 = a.box.hi[1] - a.box.lo[1], e2 = a.box.hi[2] - a.box.lo[2];
    mhd_dof d;
    d.field = a.field;
    d.block = a.block;
    d.comp = a.comp;
    d.k = (int)(q % e2) + a.box.lo[2];
    q /= e2;
    d.j = (int)(q % e1) + a.box.lo[1];
    d.i = (int)(q / e1) + a.box.lo[0];
    return d;
  }

  // ---- physical handlers (BoundaryCore::ApplyPhysical, src/5_boundary/Boundary_Physical.cpp:158-186)
  void set_phys(Arr &a, const int p[3], int kind, int arg, const int src[3] = nullptr) {
    const int64_t q = a.index(p);
    const int64_t id = a.base + q;
    a.v[q] = sym(id, true, false);
    phys_written.insert(id);
    if (kind < 0) return;  // written by an operation recorded elsewhere
    mhd_phys_op op;
    op.kind = kind;
    op.arg = arg;
    op.dst = mhd_dof{a.field, a.block, p[0], p[1], p[2], a.comp};
    op.src = src ? mhd_dof{a.field, a.block, src[0], src[1], src[2], 0} : op.dst;
    phys.push_back(op);
  }
  // LAYOUT::boundary_inner_slab_one_layer_from_cells (src/0_basic/LayoutTraits.cpp:406-433)
  IBox inner_slab(int b, int loc, const IBox &node, int dir) const {
    const int ax = axis_of(dir);
    int d[3];
    dof_delta(loc, d);
    const IBox own = G.owned(b, loc);
    IBox r;
    for (int a = 0; a < 3; ++a) {
      r.lo[a] = node.lo[a];
      r.hi[a] = d[a] == 0 ? node.hi[a] : node.hi[a] - 1;
    }
    if (dir < 0) {
      r.lo[ax] = 0;
      r.hi[ax] = 1;
    } else {
      r.lo[ax] = own.hi[ax] - 1;
      r.hi[ax] = own.hi[ax];
    }
    return r;
  }
  // LAYOUT::ghost_slab_from_inner (src/0_basic/LayoutTraits.cpp:435-451)
  IBox ghost_slab(const IBox &in, int dir) const {
    const int ax = axis_of(dir);
    IBox r = in;
    if (dir < 0) {
      r.lo[ax] = in.lo[ax] - G.g;
      r.hi[ax] = in.lo[ax];
    } else {
      r.lo[ax] = in.hi[ax];
      r.hi[ax] = in.hi[ax] + G.g;
    }
    return r;
  }
  template <class F>
  static void each(const IBox &b, F &&f) {
    int p[3];
    for (p[0] = b.lo[0]; p[0] < b.hi[0]; ++p[0])
      for (p[1] = b.lo[1]; p[1] < b.hi[1]; ++p[1])
        for (p[2] = b.lo[2]; p[2] < b.hi[2]; ++p[2]) f(p);
  }
  // BoundaryCore::DefaultPhysicalCopy (src/5_boundary/Boundary_Physical.cpp:280-315)
  void default_copy(int fs, int b, const IBox &in, int dir) {
    const int ax = axis_of(dir);
    const int ref = dir < 0 ? in.lo[ax] : in.hi[ax] - 1;
    const IBox gs = ghost_slab(in, dir);
    each(gs, [&](const int p[3]) {
      int s[3] = {p[0], p[1], p[2]};
      s[ax] = ref;
      for (int m = 0; m < ncomp(fs); ++m) {
        Arr &a = arr(fs, b, m);
        a.v[a.index(p)] = a.v[a.index(s)];
      }
    });
  }
  void apply_physical(bool resistive) {
    for (size_t fs = 0; fs < gd.fields.size(); ++fs)
      for (const Phys &pp : G.phys) {
        const int f = gd.fields[fs], b = pp.b, loc = mhd::kFieldSpec[f].loc;
        const IBox in = inner_slab(b, loc, pp.box, pp.dir);
        const int ax = axis_of(pp.dir), sgn = pp.dir > 0 ? 1 : -1;
        switch (handler(gd.group, f, pp.bc, resistive)) {
          case hNop: break;
          case hCopy: default_copy((int)fs, b, in, pp.dir); break;
          case hFarU_H:
          case hFarU_Na: {  // BC_UH_Farfield_H_ / _Na_ (Boundary_Condition_Fluid.cpp:3-34)
            const int base = f == MHD_U_H ? MHD_BC_QINF : MHD_BC_QINFS;
            each(ghost_slab(in, pp.dir), [&](const int p[3]) {
              for (int m = 0; m < 5; ++m) set_phys(arr((int)fs, b, m), p, MHD_PHYS_SET, base + m);
            });
            break;
          }
          case hWallU_H: {  // BC_Solid_Surface_, H+: the boundary cell and its ghosts from the cell one deeper
            const IBox al = G.alloc(b, loc);
            auto clamp = [&](int p[3]) {
              for (int a = 0; a < 3; ++a) p[a] = std::min(std::max(p[a], al.lo[a]), al.hi[a] - 1);
            };
            each(in, [&](const int p[3]) {
              int r[3] = {p[0], p[1], p[2]};
              r[ax] -= sgn;
              clamp(r);
              set_phys(arr((int)fs, b, 0), p, MHD_PHYS_WALL, pp.dir, r);
              for (int m = 1; m < 5; ++m) set_phys(arr((int)fs, b, m), p, -1, 0);
              for (int ng = 1; ng <= G.g; ++ng) {
                int q[3] = {p[0], p[1], p[2]};
                q[ax] += ng * sgn;
                clamp(q);
                for (int m = 0; m < 5; ++m) set_phys(arr((int)fs, b, m), q, -1, 0);
              }
            });
            break;
          }
          case hWallU_Na: {  // BC_Solid_Surface_, Na+: floor state in the ghosts
            const IBox al = G.alloc(b, loc);
            each(in, [&](const int p[3]) {
              for (int ng = 1; ng <= G.g; ++ng) {
                int q[3] = {p[0], p[1], p[2]};
                q[ax] += ng * sgn;
                for (int a = 0; a < 3; ++a) q[a] = std::min(std::max(q[a], al.lo[a]), al.hi[a] - 1);
                set_phys(arr((int)fs, b, 0), q, MHD_PHYS_SET, MHD_BC_NA_RHO_FLOOR);
                for (int m = 1; m < 4; ++m) set_phys(arr((int)fs, b, m), q, MHD_PHYS_SET, MHD_BC_ZERO);
                set_phys(arr((int)fs, b, 4), q, MHD_PHYS_SET, MHD_BC_NA_E_FLOOR);
              }
            });
            break;
          }
          case hFarE:  // BC_Farfield_Eedge_set_zerocurl: boundary edges, then the ghost copy
            each(in, [&](const int p[3]) { set_phys(arr((int)fs, b, 0), p, MHD_PHYS_EFAR, 0); });
            default_copy((int)fs, b, in, pp.dir);
            break;
          case hFarBcell:  // BC_Farfield_Bface on B_cell: the IMF
          case hFarBind:   // and zero on Bind_cell
            each(ghost_slab(in, pp.dir), [&](const int p[3]) {
              for (int m = 0; m < 3; ++m)
                set_phys(arr((int)fs, b, m), p, MHD_PHYS_SET,
                         handler(gd.group, f, pp.bc, resistive) == hFarBcell ? MHD_BC_BIMF + m : MHD_BC_ZERO);
            });
            break;
          case hWallJcell:  // BC_Solid_Surface_Jcell: zero the boundary layer and the next inward, copy out
            each(in, [&](const int p[3]) {
              int q[3] = {p[0], p[1], p[2]};
              q[ax] -= sgn;
              for (int m = 0; m < 3; ++m) set_phys(arr((int)fs, b, m), p, MHD_PHYS_SET, MHD_BC_ZERO);
              for (int m = 0; m < 3; ++m) set_phys(arr((int)fs, b, m), q, MHD_PHYS_SET, MHD_BC_ZERO);
            });
            default_copy((int)fs, b, in, pp.dir);
            break;
        }
      }
  }

  // ---- halo stages
  // component copy (HaloExchangeInner.cpp:176-247): all sources of a stage are
  // packed before any destination is written
  void stage_component(int fs, int stage) {
    const int loc = mhd::kFieldSpec[gd.fields[fs]].loc;
    struct Pending {
      int b;
      int p[3];
      std::vector<int64_t> val;
    };
    std::vector<Pending> pend;
    for (const Region &r : regions(G, stage, loc)) {
      const IBox sbox = G.alloc(r.sb, loc);
      each(r.recv, [&](const int p[3]) {
        int s[3];
        if (stage == 1) inv(r.tr, p, s); else fwd(r.tr, p, s);
        if (!sbox.contains(s)) return;
        Pending pe{r.rb, {p[0], p[1], p[2]}, {}};
        for (int m = 0; m < ncomp(fs); ++m) {
          Arr &a = arr(fs, r.sb, m);
          pe.val.push_back(a.v[a.index(s)]);
        }
        pend.push_back(std::move(pe));
      });
    }
    for (const Pending &pe : pend) {
      const IBox rbox = G.alloc(pe.b, loc);
      if (!rbox.contains(pe.p)) continue;
      for (int m = 0; m < ncomp(fs); ++m) {
        Arr &a = arr(fs, pe.b, m);
        a.v[a.index(pe.p)] = pe.val[m];
      }
    }
  }
  // form triplets (src/4_halo/forms/HaloTriplet.cpp:355-830): one region after
  // another, writing as they go; the component of a destination axis comes
  // from the corresponding axis of the source block with an orientation sign
  void stage_triplet(int stage) {
    const bool face = gd.kind == kFace2;
    auto loc_of = [&](int axis) { return face ? MHD_FACE_XI + axis : MHD_EDGE_XI + axis; };
    for (int dst = 0; dst < 3; ++dst) {
      const std::vector<Region> rd = regions(G, stage, loc_of(dst));
      for (size_t ir = 0; ir < rd.size(); ++ir) {
        const Region &r = rd[ir];
        int src;
        int factor;
        if (stage == 1 || face) {  // inverse_perm_axis(trans, dst_axis)
          src = 0;
          for (int a = 0; a < 3; ++a)
            if (r.tr.perm[a] == dst) src = a;
        } else {
          src = r.tr.perm[dst];
        }
        if (face) {  // face_2form_orientation_sign: det(sign) * sign[source axis]
          factor = r.tr.sign[0] * r.tr.sign[1] * r.tr.sign[2] * r.tr.sign[src] >= 0 ? 1 : -1;
        } else {
          factor = stage == 1 ? r.tr.sign[src] : r.tr.sign[dst];
        }
        const IBox sbox = G.alloc(r.sb, loc_of(src));
        Arr &from = arr(src, r.sb, 0);
        Arr &to = arr(dst, r.rb, 0);
        each(r.recv, [&](const int p[3]) {
          int s[3];
          if (stage == 1) inv(r.tr, p, s); else fwd(r.tr, p, s);
          if (!sbox.contains(s)) return;
          const int64_t v = from.v[from.index(s)];
          to.v[to.index(p)] = factor < 0 ? negate(v) : v;
        });
      }
    }
  }
  void halo(int stage) {
    if (stage > gd.level) return;
    if (gd.kind == kComponent) {
      for (size_t fs = 0; fs < gd.fields.size(); ++fs) stage_component((int)fs, stage);
    } else {
      stage_triplet(stage);
    }
  }
};

// ------------------------------------------------------------------ equivalence classes
struct NodeKey {
  int b, i, j, k;
  bool operator<(const NodeKey &o) const {
    if (b != o.b) return b < o.b;
    if (i != o.i) return i < o.i;
    if (j != o.j) return j < o.j;
    return k < o.k;
  }
  bool operator==(const NodeKey &o) const { return b == o.b && i == o.i && j == o.j && k == o.k; }
};

// Node representatives: nodes joined by the face patches' node maps; the
// representative of a class is its smallest (block, i, j, k)
// (src/2_topology/TopologyNode.cpp:150-235).
struct Nodes {
  const Grid &G;
  std::vector<int64_t> base;
  std::vector<int64_t> parent;
  std::vector<NodeKey> rep;
  explicit Nodes(const Grid &g) : G(g) {
    int64_t t = 0;
    for (int b = 0; b < G.nb; ++b) {
      base.push_back(t);
      t += (int64_t)(G.n[b][0] + 1) * (G.n[b][1] + 1) * (G.n[b][2] + 1);
    }
    parent.resize(t);
    for (int64_t q = 0; q < t; ++q) parent[q] = q;
    for (const Face &f : G.faces)
      Replay::each(f.tbox, [&](const int p[3]) {
        int q[3];
        fwd(f.tr, p, q);
        unite(id(f.tb, p), id(f.nb, q));
      });
    rep.resize(t);
    std::vector<int64_t> best(t, -1);
    for (int64_t q = 0; q < t; ++q) {
      const int64_t r = find(q);
      if (best[r] < 0 || key(q) < key(best[r])) best[r] = q;
    }
    for (int64_t q = 0; q < t; ++q) rep[q] = key(best[find(q)]);
  }
  int64_t id(int b, const int p[3]) const {
    return base[b] + ((int64_t)p[0] * (G.n[b][1] + 1) + p[1]) * (G.n[b][2] + 1) + p[2];
  }
  NodeKey key(int64_t q) const {
    int b = (int)(std::upper_bound(base.begin(), base.end(), q) - base.begin()) - 1;
    int64_t r = q - base[b];
    const int e2 = G.n[b][2] + 1, e1 = G.n[b][1] + 1;
    NodeKey k{b, 0, 0, 0};
    k.k = (int)(r % e2);
    r /= e2;
    k.j = (int)(r % e1);
    k.i = (int)(r / e1);
    return k;
  }
  int64_t find(int64_t q) {
    while (parent[q] != q) q = parent[q] = parent[parent[q]];
    return q;
  }
  void unite(int64_t a, int64_t b) {
    a = find(a);
    b = find(b);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
  NodeKey rep_of(int b, int i, int j, int k) const {
    const int p[3] = {i, j, k};
    return rep[id(b, p)];
  }
};

// A member of a class: (block, i, j, k, axis) with its sign to the canonical
// orientation.
struct Member {
  int b, i, j, k, axis, sign;
  bool operator<(const Member &o) const {
    if (b != o.b) return b < o.b;
    if (i != o.i) return i < o.i;
    if (j != o.j) return j < o.j;
    if (k != o.k) return k < o.k;
    return axis < o.axis;
  }
};
struct Classes {
  std::vector<std::vector<Member>> cls;  // members sorted; owner = first
};

// Edge classes: the two endpoint representatives, canonical orientation from
// the smaller to the larger (TOPO::make_edge_key).
Classes edge_classes(const Grid &G, const Nodes &N) {
  std::map<std::pair<NodeKey, NodeKey>, std::vector<Member>> m;
  for (int b = 0; b < G.nb; ++b)
    for (int ax = 0; ax < 3; ++ax) {
      const IBox own = G.owned(b, MHD_EDGE_XI + ax);
      Replay::each(own, [&](const int p[3]) {
        // only an edge on the block's boundary (in a face plane across
        // another axis) has nodes another block shares; the rest are classes
        // of one, which are dropped
        bool on = false;
        for (int c = 0; c < 3; ++c)
          if (c != ax && (p[c] == 0 || p[c] == G.n[b][c])) on = true;
        if (!on) return;
        int q[3] = {p[0], p[1], p[2]};
        q[ax] += 1;
        const NodeKey a = N.rep_of(b, p[0], p[1], p[2]), c = N.rep_of(b, q[0], q[1], q[2]);
        const bool fw = a < c;
        m[fw ? std::make_pair(a, c) : std::make_pair(c, a)].push_back({b, p[0], p[1], p[2], ax, fw ? 1 : -1});
      });
    }
  Classes out;
  for (auto &kv : m)
    if (kv.second.size() > 1) {
      std::sort(kv.second.begin(), kv.second.end());
      out.cls.push_back(kv.second);
    }
  // the reference numbers classes by their owners' order
  std::sort(out.cls.begin(), out.cls.end(), [](const auto &x, const auto &y) { return x[0] < y[0]; });
  return out;
}

// The oriented boundary of a face as a map from edge keys (their two node
// representatives, ascending) to the incidence sign times the edge's
// canonical sign (boundary_of_face, include/2_topology/LocalIncidence.h:44-80;
// face_boundary_stencil_to_canonical_edges, src/2_topology/TopologyFaceEquiv.cpp:195-228).
std::map<std::pair<NodeKey, NodeKey>, int> face_stencil(const Nodes &N, const Member &f) {
  struct E {
    int di, dj, dk, axis, sign;
  };
  std::vector<E> el;
  if (f.axis == 0) el = {{0, 0, 0, 1, +1}, {0, 1, 0, 2, +1}, {0, 0, 1, 1, -1}, {0, 0, 0, 2, -1}};
  else if (f.axis == 1) el = {{0, 0, 0, 2, +1}, {0, 0, 1, 0, +1}, {1, 0, 0, 2, -1}, {0, 0, 0, 0, -1}};
  else el = {{0, 0, 0, 0, +1}, {1, 0, 0, 1, +1}, {0, 1, 0, 0, -1}, {0, 0, 0, 1, -1}};
  std::map<std::pair<NodeKey, NodeKey>, int> st;
  for (const E &e : el) {
    int p[3] = {f.i + e.di, f.j + e.dj, f.k + e.dk}, q[3] = {p[0], p[1], p[2]};
    q[e.axis] += 1;
    const NodeKey a = N.rep_of(f.b, p[0], p[1], p[2]), c = N.rep_of(f.b, q[0], q[1], q[2]);
    const bool fw = a < c;
    st[fw ? std::make_pair(a, c) : std::make_pair(c, a)] += e.sign * (fw ? 1 : -1);
  }
  return st;
}

// Face classes: faces with the same four corner representatives; the
// owner's sign is +1 and a member's is +1 when its oriented boundary equals
// the owner's, -1 when it is the opposite (orient_face_members_to_owner,
// src/2_topology/TopologyFaceEquiv.cpp:305-345).
Classes face_classes(const Grid &G, const Nodes &N) {
  std::map<std::array<NodeKey, 4>, std::vector<Member>> m;
  for (int b = 0; b < G.nb; ++b)
    for (int ax = 0; ax < 3; ++ax) {
      const IBox own = G.owned(b, MHD_FACE_XI + ax);
      const int u = ax == 0 ? 1 : 0, w = ax == 2 ? 1 : 2;  // the face's two in-plane axes (corners order)
      Replay::each(own, [&](const int p[3]) {
        if (p[ax] != 0 && p[ax] != G.n[b][ax]) return;  // an interior face is a class of one
        std::array<NodeKey, 4> c;
        for (int n = 0; n < 4; ++n) {
          int q[3] = {p[0], p[1], p[2]};
          if (n == 1 || n == 3) q[u] += 1;
          if (n == 2 || n == 3) q[w] += 1;
          c[n] = N.rep_of(b, q[0], q[1], q[2]);
        }
        auto s = c;
        std::sort(s.begin(), s.end());
        int inv_ = 0;
        for (int x = 0; x < 4; ++x)
          for (int y = x + 1; y < 4; ++y)
            if (c[y] < c[x]) ++inv_;
        m[s].push_back({b, p[0], p[1], p[2], ax, inv_ % 2 == 0 ? 1 : -1});
      });
    }
  Classes out;
  for (auto &kv : m)
    if (kv.second.size() > 1) {
      auto &c = kv.second;
      std::sort(c.begin(), c.end());
      const auto own = face_stencil(N, c[0]);
      c[0].sign = 1;
      for (size_t q = 1; q < c.size(); ++q) {
        const auto st = face_stencil(N, c[q]);
        bool same = st.size() == own.size(), opposite = same;
        for (const auto &e : st) {
          auto it = own.find(e.first);
          same = same && it != own.end() && it->second == e.second;
          opposite = opposite && it != own.end() && it->second == -e.second;
        }
        if (!same && !opposite) throw std::runtime_error("a face's boundary does not match its class owner's");
        c[q].sign = same ? 1 : -1;
      }
      out.cls.push_back(c);
    }
  std::sort(out.cls.begin(), out.cls.end(), [](const auto &x, const auto &y) { return x[0] < y[0]; });
  return out;
}

// ------------------------------------------------------------------ flattening
struct GroupTables {
  std::vector<mhd_phys_op> phys;
  std::vector<mhd_copy> halo, owner, stash;
  int n_stash = 0;
  int n_staging = 0;  // staging slots, numbered from 0
};

bool in_owned(const Grid &G, const mhd_dof &d) {
  const IBox o = G.owned(d.block, mhd::kFieldSpec[d.field].loc);
  const int p[3] = {d.i, d.j, d.k};
  return o.contains(p);
}


// The group's tables; its staging slots are numbered from 0 (n_staging of
// them): the caller shifts them past the other groups'.
GroupTables replay_group(const Grid &G, const GroupDef &gd, const Classes &fcls, const Classes &ecls, bool resistive) {
  Replay R(G, gd);
  // stage 1: physical handlers, then the face halo; stages 2 and 3: the edge
  // and vertex halos (the grid has no physical edge or vertex patches, so the
  // corner defaults do nothing; checked by the caller)
  R.apply_physical(resistive);
  for (int stage = 1; stage <= 3; ++stage) R.halo(stage);
  if (gd.owner) {
    // owner-to-alias copies (Halo::sync_owner_alias_group): alias <- owner
    // times the product of their canonical signs
    const Classes &C = gd.kind == kFace2 ? fcls : ecls;
    for (const auto &cls : C.cls) {
      const Member &o = cls[0];
      for (size_t q = 1; q < cls.size(); ++q) {
        const Member &a = cls[q];
        Replay::Arr &to = R.arr(a.axis, a.b, 0);
        Replay::Arr &from = R.arr(o.axis, o.b, 0);
        const int pa[3] = {a.i, a.j, a.k}, po[3] = {o.i, o.j, o.k};
        const int64_t v = from.v[from.index(po)];
        to.v[to.index(pa)] = a.sign * o.sign < 0 ? negate(v) : v;
      }
    }
  }
  GroupTables T;
  T.phys = R.phys;
  // every DOF whose value changed: a copy from its source, unless a physical
  // operation computed it; halo copies as (destination, source) identities
  const int64_t nsym = R.arrs.empty() ? 0 : R.arrs.back().base + (int64_t)R.arrs.back().v.size();
  std::vector<char> phys_w(nsym, 0);
  for (int64_t id : R.phys_written) phys_w[id] = 1;
  std::vector<int64_t> hdst, hsrc;
  std::vector<char> hneg;
  for (const auto &a : R.arrs)
    for (int64_t q = 0; q < (int64_t)a.v.size(); ++q) {
      const int64_t v = a.v[q], self = a.base + q;
      if (v == sym(self, false, false)) continue;
      if (v == sym(self, true, false)) continue;  // kept the value its handler computed
      const int64_t sid = sym_id(v);
      if (!(v & kPhysBit) && phys_w[sid]) throw std::runtime_error("a copy reads a value the physical handlers overwrite");
      const bool neg = (v & kNegBit) != 0;
      if (sid == self && !neg) continue;
      const mhd_dof d = R.dof_of(self);
      if (in_owned(G, d)) {
        T.owner.push_back(mhd_copy{d, R.dof_of(sid), neg ? -1.0 : 1.0});
      } else {
        hdst.push_back(self);
        hsrc.push_back(sid);
        hneg.push_back(neg);
      }
    }
  // copies whose source the halo phase itself overwrites go through staging
  std::vector<char> is_dst(nsym, 0);
  for (int64_t id : hdst) is_dst[id] = 1;
  std::vector<mhd_copy> unstash;
  int slots = 0;
  for (size_t t = 0; t < hdst.size(); ++t) {
    const mhd_dof d = R.dof_of(hdst[t]), src = R.dof_of(hsrc[t]);
    const double sign = hneg[t] ? -1.0 : 1.0;
    if (!is_dst[hsrc[t]]) {
      T.halo.push_back(mhd_copy{d, src, sign});
      continue;
    }
    const mhd_dof st{MHD_STAGING, 0, slots++, 0, 0, 0};
    T.stash.push_back(mhd_copy{st, src, 1.0});
    unstash.push_back(mhd_copy{d, st, sign});
  }
  T.n_stash = (int)unstash.size();
  T.n_staging = slots;
  T.stash.insert(T.stash.end(), unstash.begin(), unstash.end());
  return T;
}

// ------------------------------------------------------------------ singular edges
// Classes of three or more edge aliases whose incident owner faces number
// three (SingularEdgeRegistry::build, src/7_metric/SingularEdgeRegistry.cpp:78-200).
void singular_edges(const Grid &G, const Classes &ecls, const Classes &fcls, mhd_topology *t) {
  // owner faces, as (axis, block, i, j, k)
  std::set<std::array<int, 5>> member_faces, owner_faces;
  for (const auto &c : fcls.cls)
    for (size_t q = 0; q < c.size(); ++q) {
      member_faces.insert({c[q].axis, c[q].b, c[q].i, c[q].j, c[q].k});
      if (q == 0) owner_faces.insert({c[q].axis, c[q].b, c[q].i, c[q].j, c[q].k});
    }
  auto is_owner_face = [&](int ax, int b, int i, int j, int k) {
    const std::array<int, 5> f = {ax, b, i, j, k};
    if (owner_faces.count(f)) return true;
    if (member_faces.count(f)) return false;
    return true;  // a face of one block only is its own owner
  };
  auto face_in_owned = [&](int ax, int b, int i, int j, int k) {
    const int p[3] = {i, j, k};
    return G.owned(b, MHD_FACE_XI + ax).contains(p);
  };
  t->sing_alias_offset.push_back(0);
  t->sing_cell_offset.push_back(0);
  t->sing_face_offset.push_back(0);
  for (const auto &c : ecls.cls) {
    if (c.size() < 3) continue;
    std::vector<mhd_singular_cell> cells;
    std::vector<mhd_singular_face> faces;
    std::set<std::array<int, 4>> seen_cells;
    std::set<std::array<int, 5>> seen_faces;
    int nfaces = 0;
    for (const Member &a : c) {
      // incident cells in the order (-1, -1), (-1, 0), (0, -1), (0, 0) of the transverse axes
      for (int s0 : {-1, 0})
        for (int s1 : {-1, 0}) {
          int p[3] = {a.i, a.j, a.k};
          if (a.axis == 0) { p[1] += s0; p[2] += s1; }
          if (a.axis == 1) { p[0] += s0; p[2] += s1; }
          if (a.axis == 2) { p[0] += s0; p[1] += s1; }
          if (!seen_cells.insert({a.b, p[0], p[1], p[2]}).second) continue;
          if (!G.owned(a.b, MHD_CELL).contains(p)) continue;
          cells.push_back({mhd_dof{MHD_CELL, a.b, p[0], p[1], p[2], 0}, a.axis, a.sign});
        }
      // incident faces (incident_faces, SingularEdgeRegistry.cpp:43-68) with
      // the incidence sign of AssembleSingularEdgeCurrent_
      // (Z4_Mercury/src/physics/MercurySolver_Current.cpp:59-112)
      struct F {
        int ax, di, dj, dk, sign;
      };
      std::vector<F> fl;
      if (a.axis == 0) fl = {{1, 0, 0, 0, -1}, {1, 0, 0, -1, +1}, {2, 0, 0, 0, +1}, {2, 0, -1, 0, -1}};
      else if (a.axis == 1) fl = {{0, 0, 0, 0, +1}, {0, 0, 0, -1, -1}, {2, 0, 0, 0, -1}, {2, -1, 0, 0, +1}};
      else fl = {{0, 0, 0, 0, -1}, {0, 0, -1, 0, +1}, {1, 0, 0, 0, +1}, {1, -1, 0, 0, -1}};
      for (const F &f : fl) {
        const int i = a.i + f.di, j = a.j + f.dj, k = a.k + f.dk;
        if (!seen_faces.insert({f.ax, a.b, i, j, k}).second) continue;
        if (!face_in_owned(f.ax, a.b, i, j, k)) continue;
        if (!is_owner_face(f.ax, a.b, i, j, k)) continue;
        ++nfaces;
        faces.push_back({mhd_dof{f.ax, a.b, i, j, k, 0}, f.sign * a.sign, 0});
      }
    }
    if (nfaces != 3 && nfaces <= 4) continue;  // valence 4 (regular) or a boundary edge
    t->sing_owner.push_back(mhd_dof{c[0].axis, c[0].b, c[0].i, c[0].j, c[0].k, 0});
    t->sing_owner_sign.push_back(c[0].sign);
    for (const Member &a : c) t->sing_aliases.push_back({mhd_dof{a.axis, a.b, a.i, a.j, a.k, 0}, a.sign, 0});
    t->sing_cells.insert(t->sing_cells.end(), cells.begin(), cells.end());
    t->sing_faces.insert(t->sing_faces.end(), faces.begin(), faces.end());
    t->sing_alias_offset.push_back((int32_t)t->sing_aliases.size());
    t->sing_cell_offset.push_back((int32_t)t->sing_cells.size());
    t->sing_face_offset.push_back((int32_t)t->sing_faces.size());
  }
}

// The wall EMF edges (ApplyStationaryWallNonResistiveEMF_,
// Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:5-88): the tangential
// edges of every solid-wall patch, within the owned range.
void wall_edges(const Grid &G, mhd_topology *t) {
  for (const Phys &p : G.phys) {
    if (p.bc != MHD_BC_SOLID) continue;
    const int na = axis_of(p.dir);
    for (int ax = 0; ax < 3; ++ax) {
      if (ax == na) continue;
      const int loc = MHD_EDGE_XI + ax;
      const IBox e = intersect(node_box_to_dof_box(loc, p.box), G.owned(p.b, loc));
      Replay::each(e, [&](const int q[3]) {
        mhd_phys_op op;
        op.kind = MHD_PHYS_SET;
        op.arg = MHD_BC_ZERO;
        op.dst = mhd_dof{MHD_E_XI + ax, p.b, q[0], q[1], q[2], 0};
        op.src = op.dst;
        t->wall.push_back(op);
      });
    }
  }
}

mhd_patch to_patch(int tb, int nb, int d1, int d2, int d3, const IBox &tbox, const IBox &nbox, const Tr &tr) {
  mhd_patch p;
  p.this_block = tb;
  p.nb_block = nb;
  p.direction = d1;
  p.nb_direction = d2;
  p.dir3 = d3;
  for (int a = 0; a < 3; ++a) {
    p.this_lo[a] = tbox.lo[a];
    p.this_hi[a] = tbox.hi[a];
    p.nb_lo[a] = nbox.lo[a];
    p.nb_hi[a] = nbox.hi[a];
    p.perm[a] = tr.perm[a];
    p.sign[a] = tr.sign[a];
    p.offset[a] = tr.off[a];
  }
  return p;
}

int build(Grid &G, bool resistive, mhd_topology **out) {
  auto *t = new (std::nothrow) mhd_topology();
  if (!t) return MHD_ERR_OOM;
  try {
    build_edge_patches(G);
    build_vertex_patches(G);
    if (!G.pedges.empty() || !G.pverts.empty())
      throw std::runtime_error("physical patches that meet each other (physical corners) are not supported");
    const Nodes N(G);
    const Classes ecls = edge_classes(G, N), fcls = face_classes(G, N);
    // the groups replayed on the host threads, their staging slots then
    // numbered group after group
    std::vector<int> todo;
    for (int q = 0; q < MHD_NUM_GROUPS; ++q)
      if (!((q == MHD_SYNC_ERES || q == MHD_SYNC_DB) && !resistive)) todo.push_back(q);  // implicit substep only
    std::vector<GroupTables> tabs(MHD_NUM_GROUPS);
    std::vector<std::string> errs(MHD_NUM_GROUPS);
    mhd::parallel_for((int)todo.size(), [&](int u) {
      const int q = todo[u];
      try {
        tabs[q] = replay_group(G, kGroupDefs[q], fcls, ecls, resistive);
      } catch (const std::exception &e) {
        errs[q] = e.what();
      }
    });
    for (const std::string &e : errs)
      if (!e.empty()) throw std::runtime_error(e);
    int staging = 0;
    for (int q : todo) {
      GroupTables &T = tabs[q];
      for (mhd_copy &c : T.stash) {
        if (c.dst.field == MHD_STAGING) c.dst.i += staging;
        if (c.src.field == MHD_STAGING) c.src.i += staging;
      }
      staging += T.n_staging;
      t->halo[q].assign(T.halo);
      t->owner[q].assign(T.owner);
      t->phys[q] = std::move(T.phys);
      t->stash[q] = std::move(T.stash);
    }
    t->n_staging = staging;
    // edge alias classes of the E and J reductions
    t->alias_offset.push_back(0);
    for (const auto &c : ecls.cls) {
      for (const Member &m : c) {
        t->alias_member.push_back(mhd_dof{m.axis, m.b, m.i, m.j, m.k, 0});
        t->alias_msign.push_back(m.sign);
      }
      t->alias_owner.push_back(mhd_dof{c[0].axis, c[0].b, c[0].i, c[0].j, c[0].k, 0});
      t->alias_osign.push_back(c[0].sign);
      t->alias_offset.push_back((int32_t)t->alias_member.size());
    }
    singular_edges(G, ecls, fcls, t);
    wall_edges(G, t);
    for (const Face &f : G.faces) t->faces.push_back(to_patch(f.tb, f.nb, f.dir, f.ndir, 0, f.tbox, f.nbox, f.tr));
    for (const Edge &e : G.edges) t->edges.push_back(to_patch(e.tb, e.nb, e.d1, e.d2, 0, e.tbox, e.nbox, e.tr));
    for (const Vert &v : G.verts) t->vertices.push_back(to_patch(v.tb, v.nb, v.d1, v.d2, v.d3, v.tbox, v.nbox, v.tr));
    for (const Phys &p : G.phys) {
      mhd_physical_patch pp{};
      pp.block = p.b;
      pp.direction = p.dir;
      pp.bc = p.bc;
      for (int a = 0; a < 3; ++a) {
        pp.lo[a] = p.box.lo[a];
        pp.hi[a] = p.box.hi[a];
      }
      t->physical.push_back(pp);
    }
  } catch (const std::bad_alloc &) {
    delete t;
    return mhd::set_error(MHD_ERR_OOM, "multi-block topology: host memory");
  } catch (const std::exception &e) {
    delete t;
    return mhd::set_error(MHD_ERR_ARG, "multi-block topology: %s", e.what());
  }
  *out = t;
  return MHD_OK;
}

// ------------------------------------------------------------------ the cubed-sphere shell
// Panel p's outward directions at tangent coordinates (ta, tb) of its two
// angular axes: the oracle's shell case (panel 0 +x, 1 +y, 2 -x, 3 -y,
// 4 +z, 5 -z).  Only the combinatorics matter here: two panel edges are
// joined when their nodes coincide.
void shell_dir(int p, double ta, double tb, double d[3]) {
  switch (p) {
    case 0: d[0] = 1.0; d[1] = ta; d[2] = tb; break;
    case 1: d[0] = -ta; d[1] = 1.0; d[2] = tb; break;
    case 2: d[0] = -1.0; d[1] = -ta; d[2] = tb; break;
    case 3: d[0] = ta; d[1] = -1.0; d[2] = tb; break;
    case 4: d[0] = -tb; d[1] = ta; d[2] = 1.0; break;
    default: d[0] = tb; d[1] = ta; d[2] = -1.0; break;
  }
}

}  // namespace

extern "C" int mhd_topology_multiblock(int32_t n_blocks, const int32_t *cells, int32_t nghost, int32_t n_faces,
                                       const mhd_patch *faces, int32_t n_physical, const mhd_physical_patch *physical,
                                       int32_t resistive, mhd_topology **out) {
  if (n_blocks < 1 || !cells || nghost < 1 || n_faces < 0 || (n_faces && !faces) || n_physical < 0 ||
      (n_physical && !physical) || !out)
    return mhd::set_error(MHD_ERR_ARG, "mhd_topology_multiblock: invalid arguments");
  Grid G;
  G.nb = n_blocks;
  G.g = nghost;
  for (int b = 0; b < n_blocks; ++b) {
    if (cells[3 * b] < 1 || cells[3 * b + 1] < 1 || cells[3 * b + 2] < 1)
      return mhd::set_error(MHD_ERR_ARG, "mhd_topology_multiblock: block %d has no cells", b);
    G.n.push_back({cells[3 * b], cells[3 * b + 1], cells[3 * b + 2]});
  }
  for (int q = 0; q < n_faces; ++q) {
    const mhd_patch &p = faces[q];
    if (p.this_block < 0 || p.this_block >= n_blocks || p.nb_block < 0 || p.nb_block >= n_blocks)
      return mhd::set_error(MHD_ERR_ARG, "mhd_topology_multiblock: face patch %d: block out of range", q);
    Face f;
    f.tb = p.this_block;
    f.nb = p.nb_block;
    f.dir = p.direction;
    f.ndir = p.nb_direction;
    for (int a = 0; a < 3; ++a) {
      f.tbox.lo[a] = p.this_lo[a];
      f.tbox.hi[a] = p.this_hi[a];
      f.nbox.lo[a] = p.nb_lo[a];
      f.nbox.hi[a] = p.nb_hi[a];
      f.tr.perm[a] = p.perm[a];
      f.tr.sign[a] = p.sign[a];
      f.tr.off[a] = p.offset[a];
    }
    G.faces.push_back(f);
  }
  for (int q = 0; q < n_physical; ++q) {
    const mhd_physical_patch &p = physical[q];
    if (p.block < 0 || p.block >= n_blocks || (p.bc != MHD_BC_FARFIELD && p.bc != MHD_BC_SOLID))
      return mhd::set_error(MHD_ERR_ARG, "mhd_topology_multiblock: physical patch %d: bad block or kind", q);
    Phys ph;
    ph.b = p.block;
    ph.dir = p.direction;
    ph.bc = p.bc;
    for (int a = 0; a < 3; ++a) {
      ph.box.lo[a] = p.lo[a];
      ph.box.hi[a] = p.hi[a];
    }
    G.phys.push_back(ph);
  }
  return build(G, resistive != 0, out);
}

// The shell's face patches and physical patches (mhd_topology_cubed_sphere).
int mhd::cubed_sphere_patches(int na, int nr, std::vector<mhd_patch> *faces_out,
                              std::vector<mhd_physical_patch> *phys_out) {
  if (na < 2 || nr < 2) return mhd::set_error(MHD_ERR_ARG, "cubed sphere: need na, nr >= 2");
  // panel edges e: 0 i = 0, 1 i = na, 2 j = 0, 3 j = na; partners found by
  // matching the directions of the edge nodes (tangents of the equiangular
  // grid, +-1 exactly at the panel edges)
  auto tan_of = [&](int i) {
    const int q = 2 * i - na;
    if (q == na) return 1.0;
    if (q == -na) return -1.0;
    return std::tan(((double)q / (double)na) * (std::acos(-1.0) / 4.0));
  };
  auto edge_pt = [&](int p, int e, int t, double d[3]) {
    const int i = e == 0 ? 0 : e == 1 ? na : t;
    const int j = e == 2 ? 0 : e == 3 ? na : t;
    shell_dir(p, tan_of(i), tan_of(j), d);
  };
  struct Conn {
    int q, f;
    bool rev;
  };
  Conn conn[6][4];
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e) {
      bool found = false;
      for (int q = 0; q < 6 && !found; ++q)
        for (int f = 0; f < 4 && !found; ++f) {
          if (q == p) continue;
          for (int rev = 0; rev < 2 && !found; ++rev) {
            bool ok = true;
            for (int t = 0; t <= na && ok; ++t) {
              double a[3], b[3];
              edge_pt(p, e, t, a);
              edge_pt(q, f, rev ? na - t : t, b);
              ok = a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
            }
            if (ok) {
              conn[p][e] = {q, f, rev != 0};
              found = true;
            }
          }
        }
      if (!found) return mhd::set_error(MHD_ERR_ARG, "mhd_topology_cubed_sphere: panel %d edge %d has no partner", p, e);
    }
  // the node boxes and index maps the reference derives from the shell's
  // inner-patch file (Inner_Boundary::Pre_process, include/1_grid/Grid_Boundary.h:244-330;
  // make_index_transform_from_boundary_arrays, src/2_topology/TopologyOps.cpp:118-215):
  // normal axis to normal axis (sign -1 when both faces are low or both high),
  // angular tangent to angular tangent (sign -1 on a reversed join), radius to radius
  std::vector<mhd_patch> faces;
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e) {
      const Conn &c = conn[p][e];
      const int an = e < 2 ? 0 : 1, bn = c.f < 2 ? 0 : 1;
      const int dir = (e % 2 == 0 ? -1 : 1) * (an + 1), ndir = (c.f % 2 == 0 ? -1 : 1) * (bn + 1);
      const int my_n = e % 2 == 0 ? 0 : na, tar_n = c.f % 2 == 0 ? 0 : na;
      mhd_patch fp{};
      fp.this_block = p;
      fp.nb_block = c.q;
      fp.direction = dir;
      fp.nb_direction = ndir;
      fp.perm[an] = bn;
      fp.sign[an] = dir * ndir > 0 ? -1 : 1;
      fp.offset[an] = -fp.sign[an] * my_n + tar_n;
      fp.perm[1 - an] = 1 - bn;
      fp.sign[1 - an] = c.rev ? -1 : 1;
      fp.offset[1 - an] = c.rev ? na : 0;
      fp.perm[2] = 2;
      fp.sign[2] = 1;
      fp.offset[2] = 0;
      for (int a = 0; a < 2; ++a) {
        fp.this_lo[a] = a == an ? my_n : 0;
        fp.this_hi[a] = a == an ? my_n + 1 : na + 1;
        fp.nb_lo[a] = a == bn ? tar_n : 0;
        fp.nb_hi[a] = a == bn ? tar_n + 1 : na + 1;
      }
      fp.this_lo[2] = fp.nb_lo[2] = 0;
      fp.this_hi[2] = fp.nb_hi[2] = nr + 1;
      faces.push_back(fp);
    }
  // physical patches in the reference's order: every panel's inner sphere,
  // then every panel's outer sphere
  std::vector<mhd_physical_patch> phys;
  for (int side = 0; side < 2; ++side)
    for (int p = 0; p < 6; ++p) {
      mhd_physical_patch pp{};
      pp.block = p;
      pp.direction = side ? 3 : -3;
      pp.bc = side ? MHD_BC_FARFIELD : MHD_BC_SOLID;
      pp.lo[0] = pp.lo[1] = 0;
      pp.hi[0] = pp.hi[1] = na + 1;
      pp.lo[2] = side ? nr : 0;
      pp.hi[2] = pp.lo[2] + 1;
      phys.push_back(pp);
    }
  *faces_out = std::move(faces);
  *phys_out = std::move(phys);
  return MHD_OK;
}

extern "C" int mhd_topology_cubed_sphere(int32_t na, int32_t nr, int32_t nghost, int32_t resistive,
                                         mhd_topology **out) {
  if (na < 2 || nr < 2 || nghost < 1 || !out)
    return mhd::set_error(MHD_ERR_ARG, "mhd_topology_cubed_sphere: need na, nr >= 2 and nghost >= 1");
  std::vector<mhd_patch> faces;
  std::vector<mhd_physical_patch> phys;
  const int rc = mhd::cubed_sphere_patches(na, nr, &faces, &phys);
  if (rc) return rc;
  std::vector<int32_t> cells;
  for (int p = 0; p < 6; ++p) cells.insert(cells.end(), {na, na, nr});
  return mhd_topology_multiblock(6, cells.data(), nghost, (int32_t)faces.size(), faces.data(), (int32_t)phys.size(),
                                 phys.data(), resistive, out);
}

extern "C" int mhd_topology_patches(const mhd_topology *t, int32_t which, const mhd_patch **patches, int32_t *n) {
  if (!t || !patches || !n || which < 0 || which > 2) return MHD_ERR_ARG;
  const std::vector<mhd_patch> &v = which == 0 ? t->faces : which == 1 ? t->edges : t->vertices;
  *patches = v.data();
  *n = (int32_t)v.size();
  return MHD_OK;
}

extern "C" int mhd_topology_physical(const mhd_topology *t, const mhd_physical_patch **patches, int32_t *n) {
  if (!t || !patches || !n) return MHD_ERR_ARG;
  *patches = t->physical.data();
  *n = (int32_t)t->physical.size();
  return MHD_OK;
}
