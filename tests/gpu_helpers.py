"""Shared helpers of the GPU parity tests: build a device solve from a
reference dump and compare fields."""
import numpy as np

import mercury_oracle as mo
from mpcns_mercury_b200 import Context, reference_constants
from mpcns_mercury_b200.capi import REF_FIELD

NGHOST = 4


def n_blocks(dump):
    """Blocks of a dump (records of block -1 are global)."""
    return 1 + max(b for (_, b) in dump)


def upload_from_dump(upload, dump, tag="step0:"):
    """upload(field, data, lo, hi[, block]) of the reference's state at ``tag``
    and its static inputs, for every block of the dump."""
    for b in range(n_blocks(dump)):
        up = (lambda f, a, lo, hi: upload(f, a, lo, hi)) if b == 0 else \
            (lambda f, a, lo, hi, b=b: upload(f, a, lo, hi, block=b))
        for name in mo.STATE_FIELDS:
            r = dump[(tag + name, b)]
            up(REF_FIELD[name], r.data, r.lo, r.hi)
        for name in mo.STATIC_FIELDS + ["taper_xi", "taper_eta", "taper_zeta"]:
            r = dump[("static:" + name, b)]
            up(REF_FIELD[name], r.data, r.lo, r.hi)
        if ("static:taper_cell", b) in dump:
            r = dump[("static:taper_cell", b)]
            up("TAPER_CELL", r.data, r.lo, r.hi)
        for name in ("local_arti_eta_xi", "local_arti_eta_eta", "local_arti_eta_zeta", "eta_res_xi", "eta_res_eta",
                     "eta_res_zeta"):
            if ("static:" + name, b) in dump:
                r = dump[("static:" + name, b)]
                up(REF_FIELD[name], r.data, r.lo, r.hi)
        # cell centres: the reference reads dual_x(i+1, j+1, k+1) for cell (i, j, k)
        for ax, fld in zip("xyz", ("CELL_X", "CELL_Y", "CELL_Z")):
            r = dump[("dual_" + ax, b)]
            lo = tuple(v - 1 for v in r.lo)
            hi = tuple(v - 1 for v in r.hi)
            up(fld, r.data, lo, hi)


def cells3(n):
    """Cells per axis of a block: an int (cube) or three per-axis counts."""
    return (n, n, n) if isinstance(n, int) else tuple(int(v) for v in n)


def context_from_dump(dump, n, tag="step0:", cfl=0.4, precision=0, constants=None, lattice=None):
    """Upload the reference's step-0 state and static inputs into a new
    context: one periodic block of n cells (an int or per-axis counts), or a
    periodic box cut into ``lattice`` = (bx, by, bz) blocks of n cells each."""
    nb = 1 if lattice is None else lattice[0] * lattice[1] * lattice[2]
    ctx = Context([cells3(n)] * nb, NGHOST, constants or reference_constants(cfl=cfl), precision=precision,
                  lattice=lattice)
    upload_from_dump(ctx.upload, dump, tag)
    return ctx


def owned(rec):
    g = [-v for v in rec.lo]
    return rec.data[g[0]:rec.hi[0], g[1]:rec.hi[1], g[2]:rec.hi[2]]


def compare(ctx, dump, tag, names, tol):
    """Max relative L2 over ``names`` (owned DOFs) of device vs dump."""
    worst = {}
    for name in names:
        for b in range(n_blocks(dump)):
            r = dump[(tag + name, b)]
            dev = ctx.download(REF_FIELD[name], r.lo, r.hi, block=b)
            g = [-v for v in r.lo]
            sl = (slice(g[0], r.hi[0]), slice(g[1], r.hi[1]), slice(g[2], r.hi[2]))
            key = name if b == 0 else f"{name}[{b}]"
            worst[key] = mo.rel_l2(dev[sl], r.data[sl])
    bad = {k: v for k, v in worst.items() if not v <= tol}
    return worst, bad


def div_b(ctx, n):
    """max |sum of outward face fluxes| / max |B face| over the owned cells."""
    g = NGHOST
    lo = (-g, -g, -g)
    B = []
    for ax, name in enumerate(("B_XI", "B_ETA", "B_ZETA")):
        hi = [n + g] * 3
        hi[ax] += 1
        B.append(ctx.download(name, lo, tuple(hi))[..., 0])
    o = slice(g, g + n)
    p = slice(g + 1, g + n + 1)
    d = (B[0][p, o, o] - B[0][o, o, o]) + (B[1][o, p, o] - B[1][o, o, o]) + (B[2][o, o, p] - B[2][o, o, o])
    scale = max(float(np.abs(b[o, o, o]).max()) for b in B)
    return float(np.abs(d).max()) / scale


def shell_constants(precision=0, **kw):
    """The shell case's constants: the reference's REF list with the shell
    job's upstream (INITIAL list), as the oracle harness writes them; kw:
    further reference_constants arguments (resistive, res_rtol, ...)."""
    from mpcns_mercury_b200 import reference_constants

    initial = tuple(float(v) for v in mo.SHELL_UPSTREAM.split())
    return reference_constants(cfl=mo.SHELL_JOB["cfl"], initial=initial, **kw)


def shell_context(dump, na, nr, precision=0, constants=None):
    """A context of the 6-panel shell (tables from mhd_topology_cubed_sphere)
    with the reference's step-0 state and static inputs uploaded."""
    import ctypes

    from mpcns_mercury_b200 import capi

    constants = constants or shell_constants()
    t = ctypes.c_void_p()
    capi.check(capi.lib().mhd_topology_cubed_sphere(na, nr, NGHOST, int(bool(constants.resistive)), ctypes.byref(t)),
               "mhd_topology_cubed_sphere")
    ctx = Context([(na, na, nr)] * 6, NGHOST, constants, topology=t, precision=precision)
    upload_from_dump(ctx.upload, dump)
    return ctx
