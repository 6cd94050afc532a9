"""Halo/owner sync tables and edge alias classes built by the library's host
topology builder (mhd_topology_periodic_block) against the reference itself:
the reference's own MercuryBoundary::Sync is probed with unique codes (the
method of Z0_NULL/test/halo_comm/Z0_HaloCommTest.cpp:361-398) and every DOF's
final code must match what the tables produce — bit-exact."""
import ctypes

import numpy as np
import pytest

GROUPS = {
    "UCELL": ("Ucell", ["U_H", "U_Na"]),
    "BFACE": ("Bface", ["B_xi", "B_eta", "B_zeta"]),
    "EHALL": ("Ehall", ["Ehall_xi", "Ehall_eta", "Ehall_zeta"]),
    "EEDGE": ("Eedge", ["E_xi", "E_eta", "E_zeta"]),
    "B_CELL": ("B_cell", ["B_cell", "Bind_cell"]),
    "JEDGE": ("Jedge", ["J_xi", "J_eta", "J_zeta"]),
    "J_CELL": ("J_cell", ["J_cell"]),
}


def _tables(n, nghost=4):
    from mpcns_mercury_b200 import capi

    L = capi.lib()
    t = ctypes.c_void_p()
    capi.check(L.mhd_topology_periodic_block(capi._i3([n, n, n]), nghost, ctypes.byref(t)), "topology")
    d = capi.MhdDesc()
    capi.check(L.mhd_topology_fill_desc(t, ctypes.byref(d)), "fill")
    return L, t, d


def _apply(arrays, recs, copies, n_copies):
    """dst <- sign * src over the pre-phase snapshot (numpy stand-in of k_copy)."""
    snap = {k: v.copy() for k, v in arrays.items()}
    for q in range(n_copies):
        c = copies[q]
        fd, fs = c.dst, c.src
        rd, rs = recs[fd.field], recs[fs.field]
        arrays[fd.field][fd.i - rd.lo[0], fd.j - rd.lo[1], fd.k - rd.lo[2], fd.comp] = \
            c.sign * snap[fs.field][fs.i - rs.lo[0], fs.j - rs.lo[1], fs.k - rs.lo[2], fs.comp]


@pytest.mark.parametrize("n", [4, 5])
@pytest.mark.parametrize("group", list(GROUPS))
def test_sync_tables_match_reference_probe(ref_oracle, n, group):
    from mpcns_mercury_b200.capi import FIELD_ID, REF_FIELD, GROUPS as GORDER

    ref_group, fields = GROUPS[group]
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=n, mode="probe", probe_group=ref_group, probe_fields=" ".join(fields), steps=0)
    d = ref_oracle.run_job(job)
    L, t, desc = _tables(n)
    try:
        g = desc.groups[GORDER.index(group)]
        recs = {FIELD_ID[REF_FIELD[f]]: d[("before:" + f, 0)] for f in fields}
        arrays = {k: r.data.copy() for k, r in recs.items()}
        _apply(arrays, recs, g.halo, g.n_halo)
        _apply(arrays, recs, g.owner, g.n_owner)
        for f in fields:
            got = arrays[FIELD_ID[REF_FIELD[f]]]
            want = d[("after:" + f, 0)].data
            assert np.array_equal(np.isnan(got), np.isnan(want)), f
            m = ~np.isnan(want)
            assert np.array_equal(got[m], want[m]), f
    finally:
        L.mhd_topology_destroy(t)


@pytest.mark.parametrize("n", [4, 6])
def test_alias_classes_match_reference(ref_oracle, n):
    job = dict(ref_oracle.CUBE_JOB)
    job.update(n=n, mode="classes", steps=0)
    buf = ref_oracle.run_job(job)[("edge_alias_classes", -1)].data.ravel().astype(np.int64)
    ref = []
    p = 0
    while p < len(buf):
        nm = int(buf[p + 1])
        own = tuple(buf[p + 2:p + 6])
        mem = [tuple(buf[p + 8 + 6 * q:p + 8 + 6 * q + 4]) for q in range(nm)]
        ref.append((own, mem))
        p += 8 + 6 * nm
    L, t, d = _tables(n)
    try:
        a = d.edge_aliases
        ours = []
        for c in range(a.n_classes):
            o = a.owner[c]
            mem = [(a.member[q].field, a.member[q].i, a.member[q].j, a.member[q].k)
                   for q in range(a.offset[c], a.offset[c + 1])]
            ours.append(((o.field, o.i, o.j, o.k), mem))
        # same classes, same owners, same member order (the summation order)
        assert sorted(ref) == sorted(ours)
    finally:
        L.mhd_topology_destroy(t)


# Periodic boxes cut into aligned blocks: cells per block and blocks per axis
# (the reference's "lattice" case: inner patches between blocks, periodic
# ones where a patch wraps around the box).
LATTICES = [(4, (2, 2, 2)), (4, (2, 1, 3)), (5, (1, 2, 2))]


def _lattice_tables(n, nb, nghost=4):
    from mpcns_mercury_b200 import capi

    L = capi.lib()
    t = ctypes.c_void_p()
    capi.check(L.mhd_topology_periodic_lattice(capi._i3([n, n, n]), capi._i3(list(nb)), nghost, ctypes.byref(t)),
               "lattice topology")
    d = capi.MhdDesc()
    capi.check(L.mhd_topology_fill_desc(t, ctypes.byref(d)), "fill")
    return L, t, d


def _apply_blocks(arrays, recs, copies, n_copies):
    """dst <- sign * src over the pre-phase snapshot, arrays keyed by (field, block)."""
    snap = {k: v.copy() for k, v in arrays.items()}
    for q in range(n_copies):
        c = copies[q]
        fd, fs = c.dst, c.src
        rd, rs = recs[(fd.field, fd.block)], recs[(fs.field, fs.block)]
        arrays[(fd.field, fd.block)][fd.i - rd.lo[0], fd.j - rd.lo[1], fd.k - rd.lo[2], fd.comp] = \
            c.sign * snap[(fs.field, fs.block)][fs.i - rs.lo[0], fs.j - rs.lo[1], fs.k - rs.lo[2], fs.comp]


@pytest.mark.parametrize("n,nb", LATTICES)
@pytest.mark.parametrize("group", list(GROUPS))
def test_lattice_tables_match_reference_probe(ref_oracle, n, nb, group):
    from mpcns_mercury_b200.capi import FIELD_ID, REF_FIELD, GROUPS as GORDER

    ref_group, fields = GROUPS[group]
    job = dict(ref_oracle.CUBE_JOB)
    job.update(case="lattice", n=n, nb=" ".join(map(str, nb)), mode="probe", probe_group=ref_group,
               probe_fields=" ".join(fields), steps=0)
    d = ref_oracle.run_job(job)
    nblock = nb[0] * nb[1] * nb[2]
    L, t, desc = _lattice_tables(n, nb)
    try:
        g = desc.groups[GORDER.index(group)]
        recs = {(FIELD_ID[REF_FIELD[f]], b): d[("before:" + f, b)] for f in fields for b in range(nblock)}
        arrays = {k: r.data.copy() for k, r in recs.items()}
        _apply_blocks(arrays, recs, g.halo, g.n_halo)
        _apply_blocks(arrays, recs, g.owner, g.n_owner)
        for f in fields:
            for b in range(nblock):
                got = arrays[(FIELD_ID[REF_FIELD[f]], b)]
                want = d[("after:" + f, b)].data
                assert np.array_equal(np.isnan(got), np.isnan(want)), (f, b)
                m = ~np.isnan(want)
                assert np.array_equal(got[m], want[m]), (f, b)
    finally:
        L.mhd_topology_destroy(t)


@pytest.mark.parametrize("n,nb", LATTICES)
def test_lattice_alias_classes_match_reference(ref_oracle, n, nb):
    job = dict(ref_oracle.CUBE_JOB)
    job.update(case="lattice", n=n, nb=" ".join(map(str, nb)), mode="classes", steps=0)
    buf = ref_oracle.run_job(job)[("edge_alias_classes", -1)].data.ravel().astype(np.int64)
    ref = []
    p = 0
    while p < len(buf):
        nm = int(buf[p + 1])
        own = tuple(int(v) for v in buf[p + 2:p + 6]) + (int(buf[p + 7]),)
        mem = [tuple(int(v) for v in buf[p + 8 + 6 * q:p + 8 + 6 * q + 4]) + (int(buf[p + 8 + 6 * q + 5]),)
               for q in range(nm)]
        # aligned blocks: one orientation sign per class (the reference stores
        # some classes with all signs -1, its canonical edge orientation); the
        # reduction sign * sum(sign * v) / count is then the all +1 one, bitwise
        signs = {int(buf[p + 6])} | {int(buf[p + 8 + 6 * q + 4]) for q in range(nm)}
        assert len(signs) == 1
        ref.append((own, mem))
        p += 8 + 6 * nm
    L, t, d = _lattice_tables(n, nb)
    try:
        a = d.edge_aliases
        ours = []
        for c in range(a.n_classes):
            o = a.owner[c]
            mem = [(a.member[q].field, a.member[q].i, a.member[q].j, a.member[q].k, a.member[q].block)
                   for q in range(a.offset[c], a.offset[c + 1])]
            ours.append(((o.field, o.i, o.j, o.k, o.block), mem))
        assert sorted(ref) == sorted(ours)
    finally:
        L.mhd_topology_destroy(t)


def test_one_block_lattice_is_the_periodic_block():
    """A 1 x 1 x 1 lattice has the single periodic block's tables and classes."""
    L, t1, d1 = _tables(6)
    _, t2, d2 = _lattice_tables(6, (1, 1, 1))

    def entries(copies, n):
        return sorted((c.dst.field, c.dst.block, c.dst.i, c.dst.j, c.dst.k, c.dst.comp,
                       c.src.field, c.src.block, c.src.i, c.src.j, c.src.k, c.src.comp, c.sign) for c in copies[:n])

    try:
        for g in range(len(d1.groups)):
            a, b = d1.groups[g], d2.groups[g]
            assert entries(a.halo, a.n_halo) == entries(b.halo, b.n_halo)
            assert entries(a.owner, a.n_owner) == entries(b.owner, b.n_owner)
        e1, e2 = d1.edge_aliases, d2.edge_aliases
        assert e1.n_classes == e2.n_classes

        def classes(e):
            return sorted(((e.owner[c].field, e.owner[c].i, e.owner[c].j, e.owner[c].k),
                           tuple((e.member[q].field, e.member[q].i, e.member[q].j, e.member[q].k)
                                 for q in range(e.offset[c], e.offset[c + 1]))) for c in range(e.n_classes))

        assert classes(e1) == classes(e2)
    finally:
        L.mhd_topology_destroy(t1)
        L.mhd_topology_destroy(t2)


@pytest.mark.parametrize("cells,blocks,nghost", [((3, 4, 4), (2, 2, 2), 4), ((4, 4, 4), (0, 2, 2), 4),
                                                 ((4, 4, 4), (2, 2, 2), 0), ((1, 4, 4), (1, 1, 1), 1)])
def test_lattice_rejects_bad_arguments(cells, blocks, nghost):
    """Blocks thinner than the ghost depth, empty lattices, no ghosts: MHD_ERR_ARG."""
    from mpcns_mercury_b200 import capi

    t = ctypes.c_void_p()
    rc = capi.lib().mhd_topology_periodic_lattice(capi._i3(list(cells)), capi._i3(list(blocks)), nghost,
                                                  ctypes.byref(t))
    assert rc == 1 and not t.value  # MHD_ERR_ARG, nothing allocated
