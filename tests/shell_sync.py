"""Test helper: applies a multi-block descriptor's sync tables (physical
operations, staging, halo and owner copies) to field arrays in numpy, the way
the device applies them, so that they can be compared with the reference's own
MercuryBoundary::Sync on unique-code probes (the method of
Z0_NULL/test/halo_comm/Z0_HaloCommTest.cpp:361-398)."""
import ctypes
import math

import numpy as np

from mpcns_mercury_b200 import capi
from mpcns_mercury_b200.capi import FIELD_ID, REF_FIELD

GROUPS = {"UCELL": ("Ucell", ["U_H", "U_Na"]), "BFACE": ("Bface", ["B_xi", "B_eta", "B_zeta"]),
          "EHALL": ("Ehall", ["Ehall_xi", "Ehall_eta", "Ehall_zeta"]), "EEDGE": ("Eedge", ["E_xi", "E_eta", "E_zeta"]),
          "B_CELL": ("B_cell", ["B_cell", "Bind_cell"]), "JEDGE": ("Jedge", ["J_xi", "J_eta", "J_zeta"]),
          "J_CELL": ("J_cell", ["J_cell"]),
          # the implicit resistive substep's groups (a resistive run); the
          # engine keeps E_res, dB and dJ in the E, B and J arrays, and dJ
          # uses the J edge group's tables
          "ERES": ("Eres", ["Eres_xi", "Eres_eta", "Eres_zeta"]), "DB": ("dB", ["dB_xi", "dB_eta", "dB_zeta"]),
          "DJ": ("dJ", ["dJ_xi", "dJ_eta", "dJ_zeta"])}
RESISTIVE_GROUPS = {"ERES", "DB", "DJ"}
TABLES = {"DJ": "JEDGE"}  # probe group -> the descriptor group whose tables apply
_ARRAY_OF = {"Eres": "E", "dB": "B", "dJ": "J"}


def field_key(f):
    """The mhd_field id whose arrays hold the reference field f."""
    head, _, tail = f.partition("_")
    if head in _ARRAY_OF:
        f = _ARRAY_OF[head] + "_" + tail
    return FIELD_ID[REF_FIELD[f]]
# the oracle harness's default upstream (INITIAL list, SI): U T n M c_y c_z Bx By Bz
INITIAL = (4.03112887e5, 1.7407e5, 4e7, 0.001, 1.240347346e-1, 0.0, -1.52e-8, 8.4e-9, -8.5e-9)
GAMMA = 1.6667


def shell_topology(na, nr, nghost=4, resistive=0):
    L = capi.lib()
    t = ctypes.c_void_p()
    capi.check(L.mhd_topology_cubed_sphere(na, nr, nghost, resistive, ctypes.byref(t)), "mhd_topology_cubed_sphere")
    d = capi.MhdDesc()
    capi.check(L.mhd_topology_fill_desc(t, ctypes.byref(d)), "mhd_topology_fill_desc")
    return L, t, d


def _std_max(x, f):  # std::max(x, f) = (x < f) ? f : x
    return f if x < f else x


def _wall_state(U, gamma):
    """BC_Solid_Surface_'s state for a cell whose reference cell holds U
    (Z4_Mercury/src/boundary/Boundary_Condition_Fluid.cpp:37-259)."""
    floor = 2.5e-3
    rho_r = _std_max(U[0], floor)
    rho = _std_max(rho_r, floor)
    ke = 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rho
    eint = U[4] - ke
    if eint < 0.0:
        eint = 0.0
    p = _std_max((gamma - 1.0) * eint, 1e-12)
    return [rho_r, rho_r * 0.0, rho_r * 0.0, rho_r * 0.0, p / (gamma - 1.0) + 0.5 * rho_r * 0.0]


def apply_group(desc, gi, arrays, recs, nodes, bc, gamma=GAMMA):
    """The group's sync on arrays {(field id, block): data[i, j, k, comp]}
    (logical origin recs[...].lo); nodes {block: (x, y, z) records} give the
    edge vectors of the farfield EMF."""
    g = desc.groups[gi]
    stage = {}

    def at(dof):
        r = recs[(dof.field, dof.block)]
        return arrays[(dof.field, dof.block)], (dof.i - r.lo[0], dof.j - r.lo[1], dof.k - r.lo[2], dof.comp)

    def get(dof, src=None):
        if dof.field == capi.MHD_STAGING:
            return stage[dof.i]
        a, ix = at(dof)
        if src is not None:
            a = src[(dof.field, dof.block)]
        return a[ix]

    def put(dof, v):
        if dof.field == capi.MHD_STAGING:
            stage[dof.i] = v
            return
        a, ix = at(dof)
        a[ix] = v

    for q in range(g.n_phys):
        op = g.phys[q]
        if op.kind == capi.PHYS_SET:
            put(op.dst, bc[op.arg])
        elif op.kind == capi.PHYS_EFAR:
            ax = op.dst.field - FIELD_ID["E_XI"]
            u, B = bc[16:19], bc[10:13]
            E = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
            p = [op.dst.i, op.dst.j, op.dst.k]
            pr = list(p)
            pr[ax] += 1
            xs = nodes[op.dst.block]
            g0 = [-v for v in xs[0].lo]

            def X(rec, pp):
                return rec.data[pp[0] + g0[0], pp[1] + g0[1], pp[2] + g0[2], 0]

            put(op.dst, E[0] * (X(xs[0], pr) - X(xs[0], p)) + E[1] * (X(xs[1], pr) - X(xs[1], p)) +
                E[2] * (X(xs[2], pr) - X(xs[2], p)))
        elif op.kind == capi.PHYS_WALL:
            a, ix = at(op.src)
            first = _wall_state([a[ix[0], ix[1], ix[2], m] for m in range(5)], gamma)
            b, jx = at(op.dst)
            for m in range(5):
                b[jx[0], jx[1], jx[2], m] = first[m]
            ghost = _wall_state(first, gamma)
            r = recs[(op.dst.field, op.dst.block)]
            ax, sg = abs(op.arg) - 1, (1 if op.arg > 0 else -1)
            for ng in range(1, -r.lo[0] + 1):
                q3 = [op.dst.i, op.dst.j, op.dst.k]
                q3[ax] += ng * sg
                q3 = [min(max(q3[c], r.lo[c]), r.hi[c] - 1) for c in range(3)]
                for m in range(5):
                    b[q3[0] - r.lo[0], q3[1] - r.lo[1], q3[2] - r.lo[2], m] = ghost[m]
    for q in range(g.n_stash):
        c = g.stash[q]
        put(c.dst, c.sign * get(c.src))
    snap = {k: v.copy() for k, v in arrays.items()}
    for q in range(g.n_halo):
        c = g.halo[q]
        put(c.dst, c.sign * get(c.src, snap))
    for q in range(g.n_stash):
        c = g.stash[g.n_stash + q]
        put(c.dst, c.sign * get(c.src))
    snap = {k: v.copy() for k, v in arrays.items()}
    for q in range(g.n_owner):
        c = g.owner[q]
        put(c.dst, c.sign * get(c.src, snap))


def probe_and_apply(ref_oracle, group, na, nr):
    """The reference's probe of one group on the na x na x nr shell and the
    same sync applied with the builder's tables: (dump, arrays)."""
    from mpcns_mercury_b200.capi import GROUPS as GORDER
    from mpcns_mercury_b200.constants import reference_constants

    ref_group, fields = GROUPS[group]
    res = 1 if group in RESISTIVE_GROUPS else 0
    job = dict(case="shell", na=na, nr=nr, mode="probe", probe_group=ref_group, probe_fields=" ".join(fields),
               steps=0, dump_grid=1, initial_line=" ".join(repr(v) for v in INITIAL), resistive=res)
    dump = ref_oracle.run_job(job)
    L, t, desc = shell_topology(na, nr, resistive=res)
    try:
        recs = {(field_key(f), b): dump[("before:" + f, b)] for f in fields for b in range(6)}
        arrays = {k: r.data.copy() for k, r in recs.items()}
        nodes = {b: (dump[("node_x", b)], dump[("node_y", b)], dump[("node_z", b)]) for b in range(6)}
        c = reference_constants(initial=INITIAL)
        apply_group(desc, GORDER.index(TABLES.get(group, group)), arrays, recs, nodes, [c.bc[q] for q in range(19)])
    finally:
        L.mhd_topology_destroy(t)
    return dump, arrays, fields
