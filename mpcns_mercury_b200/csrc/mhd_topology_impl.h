// The host topology object behind the opaque mhd_topology of the C ABI: the
// flattened sync tables, edge alias classes and (multi-block grids with
// physical boundaries) the boundary operations and singular-edge lists a
// builder produced.  Shared by the builders (mhd_topology.cpp,
// mhd_multiblock.cpp).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "mercury_mhd.h"

// A copy table whose entries are written once, by the building threads (no
// zero-fill of a freshly allocated table).
struct CopyTable {
  std::unique_ptr<mhd_copy[]> p;
  size_t n = 0;
  void allocate(size_t count) {
    p.reset(count ? new mhd_copy[count] : nullptr);
    n = count;
  }
  void assign(const std::vector<mhd_copy> &v) {
    allocate(v.size());
    for (size_t q = 0; q < v.size(); ++q) p[q] = v[q];
  }
  mhd_copy *data() const { return p.get(); }
  size_t size() const { return n; }
};

struct mhd_topology {
  CopyTable halo[MHD_NUM_GROUPS], owner[MHD_NUM_GROUPS];
  std::vector<int32_t> alias_offset;
  std::vector<mhd_dof> alias_member, alias_owner;
  std::vector<double> alias_msign, alias_osign;
  // multi-block grids with physical boundaries (empty otherwise)
  std::vector<mhd_phys_op> phys[MHD_NUM_GROUPS];
  std::vector<mhd_copy> stash[MHD_NUM_GROUPS];  // n_stash copies into staging slots, then n_stash back
  std::vector<mhd_phys_op> wall;                 // the step's wall EMF (E_t = 0 on solid-wall edges)
  int32_t n_staging = 0;
  std::vector<int32_t> sing_cell_offset, sing_face_offset;
  std::vector<mhd_dof> sing_owner;
  std::vector<double> sing_owner_sign;
  std::vector<mhd_singular_cell> sing_cells;
  std::vector<mhd_singular_face> sing_faces;
  std::vector<mhd_singular_alias> sing_aliases;
  std::vector<int32_t> sing_alias_offset;
  // the grid's patches as the builder derived them (for inspection)
  std::vector<mhd_patch> faces, edges, vertices;
  std::vector<mhd_physical_patch> physical;
  // periodic blocks and lattices: Sync(Eres) and Sync(dB) are the E edge and
  // B face groups' copies (no physical boundary tells them apart)
  bool res_groups_alias = false;
};

namespace mhd {
// The 6-panel cubed-sphere shell's face patches (index maps between panels)
// and physical patches, in the order mhd_topology_cubed_sphere builds from.
int cubed_sphere_patches(int na, int nr, std::vector<mhd_patch> *faces, std::vector<mhd_physical_patch> *phys);
}  // namespace mhd
