"""The multi-block table builder on the 6-panel cubed-sphere shell against
the reference itself (oracle/_ref, built from its own sources):

- the face, edge, vertex and physical patches it derives equal the
  reference's topology (TOPO::build_topology) patch for patch, in order;
- every sync group's tables (physical boundary operations, staged and plain
  halo copies, owner copies), applied to the reference's unique-code probe
  state, give exactly the state the reference's own MercuryBoundary::Sync
  leaves (every DOF bit for bit, NaN where the reference leaves a ghost
  unfilled) -- the halo known-answer method of
  Z0_NULL/test/halo_comm/Z0_HaloCommTest.cpp:361-398;
- the edge alias classes (owners, member order, orientation signs up to the
  class's common sign) equal the reference's."""
import ctypes

import numpy as np
import pytest

from shell_sync import GROUPS, probe_and_apply, shell_topology

SIZES = [(4, 4), (5, 6)]


def _ref_patches(ref_oracle, na, nr):
    d = ref_oracle.run_job(dict(case="shell", na=na, nr=nr, mode="topology", steps=0))

    def rows(name, w):
        a = d[(name, -1)].data.ravel().astype(int)
        return [] if (len(a) == 1 and a[0] == -1) else [tuple(r) for r in a.reshape(-1, w)]

    return d, rows


@pytest.mark.parametrize("na,nr", SIZES)
def test_shell_patches_match_reference(ref_oracle, na, nr):
    from mpcns_mercury_b200 import capi

    d, rows = _ref_patches(ref_oracle, na, nr)
    L, t, _ = shell_topology(na, nr)
    try:
        def ours(which):
            p = ctypes.POINTER(capi.MhdPatch)()
            n = ctypes.c_int32()
            capi.check(L.mhd_topology_patches(t, which, ctypes.byref(p), ctypes.byref(n)), "patches")
            return [p[q] for q in range(n.value)]

        faces = [(x.this_block, x.nb_block, x.direction, x.nb_direction, 0, *x.this_lo, *x.this_hi, *x.nb_lo,
                  *x.nb_hi, *x.perm, *x.sign, *x.offset) for x in ours(0)]
        assert faces == rows("topo_faces", 26)
        edges = [(x.this_block, x.nb_block, x.direction, x.nb_direction, 0, *x.this_lo, *x.this_hi, *x.nb_lo,
                  *x.nb_hi, *x.perm, *x.sign, *x.offset) for x in ours(1)]
        assert edges == rows("topo_edges", 26)
        verts = [(x.this_block, x.nb_block, x.direction, x.nb_direction, x.dir3, 0, *x.this_lo, *x.this_hi,
                  *x.nb_lo, *x.nb_hi, *x.perm, *x.sign, *x.offset) for x in ours(2)]
        assert verts == rows("topo_vertices", 27)
        p = ctypes.POINTER(capi.MhdPhysicalPatch)()
        n = ctypes.c_int32()
        capi.check(L.mhd_topology_physical(t, ctypes.byref(p), ctypes.byref(n)), "physical")
        bc_id = {capi.BC_SOLID: 17, capi.BC_FARFIELD: 4}  # the case's boundary-name ids
        phys = [(p[q].block, p[q].direction, bc_id[p[q].bc], *p[q].lo, *p[q].hi) for q in range(n.value)]
        assert phys == rows("topo_physical", 9)
        assert rows("topo_phys_edges", 9) == [] and rows("topo_phys_vertices", 10) == []
    finally:
        L.mhd_topology_destroy(t)


@pytest.mark.parametrize("na,nr", SIZES)
@pytest.mark.parametrize("group", list(GROUPS))
def test_shell_sync_tables_match_reference_probe(ref_oracle, group, na, nr):
    from shell_sync import field_key

    dump, arrays, fields = probe_and_apply(ref_oracle, group, na, nr)
    for f in fields:
        for b in range(6):
            got = arrays[(field_key(f), b)]
            want = dump[("after:" + f, b)].data
            assert np.array_equal(np.isnan(got), np.isnan(want)), (f, b)
            m = ~np.isnan(want)
            assert np.array_equal(got[m], want[m]), (f, b)


@pytest.mark.parametrize("na,nr", SIZES)
def test_shell_edge_classes_match_reference(ref_oracle, na, nr):
    d, _ = _ref_patches(ref_oracle, na, nr)
    buf = d[("edge_alias_classes", -1)].data.ravel().astype(np.int64)
    ref = []
    p = 0
    while p < len(buf):
        nm = int(buf[p + 1])
        own = (int(buf[p + 2]), int(buf[p + 7]), *[int(v) for v in buf[p + 3:p + 6]])
        osign = int(buf[p + 6])
        mem = []
        for q in range(nm):
            r = buf[p + 8 + 6 * q:p + 14 + 6 * q]
            mem.append((int(r[0]), int(r[5]), int(r[1]), int(r[2]), int(r[3]), int(r[4]) * osign))
        ref.append((own, tuple(mem)))
        p += 8 + 6 * nm
    L, t, desc = shell_topology(na, nr)
    try:
        a = desc.edge_aliases
        ours = []
        for c in range(a.n_classes):
            o = a.owner[c]
            os_ = int(a.owner_sign[c])
            mem = tuple((a.member[q].field, a.member[q].block, a.member[q].i, a.member[q].j, a.member[q].k,
                         int(a.member_sign[q]) * os_) for q in range(a.offset[c], a.offset[c + 1]))
            ours.append(((o.field, o.block, o.i, o.j, o.k), mem))
        # same classes in the same (owner) order, members in stored order,
        # signs relative to the owner's
        assert ours == ref
    finally:
        L.mhd_topology_destroy(t)


def test_shell_singular_edges_are_the_eight_radial_lines():
    """Valence-3 edges: the radial edges of the eight cube-corner lines."""
    L, t, desc = shell_topology(4, 6)
    try:
        s = desc.singular
        assert s.n_edges == 8 * 6
        for e in range(s.n_edges):
            assert s.owner[e].field == 2  # zeta (radial) edges
            assert s.alias_offset[e + 1] - s.alias_offset[e] == 3
            assert s.cell_offset[e + 1] - s.cell_offset[e] == 3  # one owned cell per sector
            assert s.face_offset[e + 1] - s.face_offset[e] == 3  # three seam faces, one owner each
    finally:
        L.mhd_topology_destroy(t)


@pytest.mark.parametrize("na,nr", [(5, 6), (6, 8), (8, 12)])
def test_shell_grid_matches_reference_grid(ref_oracle, na, nr):
    """mhd_shell_grid: the owned nodes of the shell case and every ghost node
    as the reference's grid preprocessing leaves it (extrapolation, interface
    transfer, corner treatment), bit for bit over the whole node range; and
    mhd_shell_nodes alone: the owned nodes and the radial ghost layers above
    the panel (the extrapolation, which no transfer overwrites)."""
    from mpcns_mercury_b200 import capi

    d = ref_oracle.shell_run(na=na, nr=nr, steps=0, dump_at=[0], extra={"dump_fields": "U_H"})
    G = -d[("node_x", 0)].lo[0]
    grid = capi.shell_grid(na, nr, r_out=8.0, G=G)
    for b in range(6):
        alone = capi.shell_nodes(na, nr, b, r_out=8.0, G=G)
        for a, ax in enumerate("xyz"):
            want = d[("node_" + ax, b)].data[..., 0]
            assert want.shape == grid.shape[1:4], (want.shape, grid.shape)
            assert np.array_equal(grid[b, ..., a], want), (b, ax, float(np.abs(grid[b, ..., a] - want).max()))
            o = slice(G, G + na + 1)
            assert np.array_equal(alone[o, o, :, a], want[o, o, :]), (b, ax)
