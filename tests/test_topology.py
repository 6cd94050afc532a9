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
