"""mhd_hall_emf_static_scratch: the Hall edge EMF for callers that may not
allocate device memory (their memory belongs to another allocator or pool, or
they must not pay cudaMalloc inside a request).  The entry point takes the
caller's input and output device pointers and keeps its only intermediate in
a library-owned static device array.

Checked through the C ABI against the existing entry point (the Hall EMF the
context's mhd_step computes) on two calls in a row, each on a new state, so
that values left in the shared static scratch by the first call cannot leak
into the second.  This file is collected last (test_zz_*)."""
import ctypes

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 parity tolerance of the other GPU tests


def _view(ctx, field, comp=0):
    from mpcns_mercury_b200 import capi

    base, G, si, sj = ctypes.c_void_p(), ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
    ext = (ctypes.c_int32 * 3)()
    capi.check(capi.lib().mhd_device_view(ctx.ctx, capi.FIELD_ID[field], 0, comp, ctypes.byref(base),
                                          ctypes.byref(G), ctypes.byref(si), ctypes.byref(sj), ext), "view")
    return base.value, G.value, si.value, sj.value, tuple(ext)


class HallBlock(ctypes.Structure):
    P = ctypes.c_void_p
    _fields_ = [("n", ctypes.c_int32 * 3), ("nghost", ctypes.c_int32), ("G", ctypes.c_int32),
                ("pad_", ctypes.c_int32), ("si", ctypes.c_int64), ("sj", ctypes.c_int64),
                ("rho_H", P), ("rho_Na", P), ("J_cell", P * 3), ("B_cell", P * 3), ("B_face", P * 3),
                ("area", P * 3), ("dl", P * 3), ("dr_xi", P * 3), ("dr_eta", P * 3), ("dr_zeta", P * 3),
                ("taper", P * 3), ("hall_coef", ctypes.c_double), ("M_H", ctypes.c_double),
                ("M_Na", ctypes.c_double), ("M_ref", ctypes.c_double), ("ne_hall_floor", ctypes.c_double)]


def _block(ctx, cells, consts):
    blk = HallBlock()
    blk.n[:] = list(cells)
    blk.nghost = 4
    _, G, si, sj, _ = _view(ctx, "U_H")
    blk.G, blk.si, blk.sj = G, si, sj
    blk.rho_H = _view(ctx, "U_H", 0)[0]
    blk.rho_Na = _view(ctx, "U_NA", 0)[0]
    for a, ax in enumerate(("XI", "ETA", "ZETA")):
        blk.J_cell[a] = _view(ctx, "J_CELL", a)[0]
        blk.B_cell[a] = _view(ctx, "B_CELL", a)[0]
        blk.B_face[a] = _view(ctx, "B_" + ax)[0]
        blk.area[a] = _view(ctx, "AREA_" + ax)[0]
        blk.dl[a] = _view(ctx, "DL_" + ax)[0]
        blk.taper[a] = _view(ctx, "TAPER_" + ax)[0]
        blk.dr_xi[a] = _view(ctx, "DR_XI", a)[0]
        blk.dr_eta[a] = _view(ctx, "DR_ETA", a)[0]
        blk.dr_zeta[a] = _view(ctx, "DR_ZETA", a)[0]
    blk.hall_coef, blk.M_H, blk.M_Na = consts.hall_coef, consts.M_H, consts.M_Na
    blk.M_ref, blk.ne_hall_floor = consts.M_ref, consts.ne_hall_floor
    return blk, G, si, sj


@pytest.mark.parametrize("cells", [(16, 16, 16), (12, 16, 20)], ids=["cube16", "box12x16x20"])
def test_static_scratch_hall_emf_matches_step(cells):
    """A cube and a block with three different extents (a swapped axis in the
    scratch or launch indexing would still pass on a cube)."""
    if not has_gpu():
        pytest.skip("no GPU")
    import torch

    from bench import make_context
    from mpcns_mercury_b200 import capi, reference_constants
    from mpcns_mercury_b200 import setup as S

    L = capi.lib()
    L.mhd_hall_emf_static_scratch.argtypes = [ctypes.POINTER(HallBlock), ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]
    L.mhd_last_error.restype = ctypes.c_char_p
    _, fields = S.cube_case(cells)
    ctx, _ = make_context([cells], [fields])
    consts = reference_constants(cfl=0.4)
    try:
        _, G, si, sj, ext = _view(ctx, "U_H")
        for call in range(2):
            blk, G, si, sj = _block(ctx, cells, consts)
            # the caller's own output buffers (memory the caller already owns)
            outs = [torch.full((ext[0] * si,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
            torch.cuda.synchronize()
            rc = L.mhd_hall_emf_static_scratch(ctypes.byref(blk), outs[0].data_ptr(), outs[1].data_ptr(),
                                               outs[2].data_ptr(), ctx.stream())
            assert rc == 0, L.mhd_last_error()
            ctx.synchronize()
            ctx.step(1)  # the existing entry point computes the same Hall EMF inside the step
            for a, (fld, stag) in enumerate((("EHALL_XI", (0, 1, 1)), ("EHALL_ETA", (1, 0, 1)),
                                             ("EHALL_ZETA", (1, 1, 0)))):
                hi = tuple(c + s for c, s in zip(cells, stag))
                want = ctx.download(fld, (0, 0, 0), hi)[..., 0]
                box = outs[a].cpu().numpy().reshape(ext[0], ext[1], sj)
                got = box[G:G + hi[0], G:G + hi[1], G:G + hi[2]]
                # owned edges that are not periodic aliases (alias edges take
                # their owner's value in the step's Ehall sync)
                sl = tuple(slice(0, c) for c in cells)
                g, w = got[sl], want[sl]
                assert np.all(np.isfinite(g)), (call, fld)
                err = np.linalg.norm((g - w).ravel()) / np.linalg.norm(w.ravel())
                assert err <= TOL, (call, fld, err)
    finally:
        ctx.close()


def test_rejects_blocks_beyond_the_static_scratch():
    if not has_gpu():
        pytest.skip("no GPU")
    from mpcns_mercury_b200 import capi

    L = capi.lib()
    L.mhd_hall_emf_static_scratch.argtypes = [ctypes.POINTER(HallBlock), ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]
    blk = HallBlock()
    blk.n[:] = [200, 200, 200]  # (200 + 2)^3 scratch cells > MHD_HALL_SCRATCH_MAX_CELLS
    blk.nghost, blk.G = 4, 5
    blk.sj = 200 + 1 + 2 * 5
    blk.si = blk.sj * (200 + 1 + 2 * 5)
    dummy = 16  # non-null placeholders: rejected before any device access
    for name in ("rho_H", "rho_Na"):
        setattr(blk, name, dummy)
    for name in ("J_cell", "B_cell", "B_face", "area", "dl", "dr_xi", "dr_eta", "dr_zeta", "taper"):
        arr = getattr(blk, name)
        for a in range(3):
            arr[a] = dummy
    assert L.mhd_hall_emf_static_scratch(ctypes.byref(blk), dummy, dummy, dummy, None) == 1  # MHD_ERR_ARG
    # a block that fits, with strides smaller than its box (k extent
    # n + 1 + 2G, j extent n + 1 + 2G): rejected, nothing touches the device
    blk.n[:] = [10, 12, 14]
    blk.sj, blk.si = 14 + 1 + 2 * 5 - 1, (14 + 1 + 2 * 5) * (12 + 1 + 2 * 5)
    assert L.mhd_hall_emf_static_scratch(ctypes.byref(blk), dummy, dummy, dummy, None) == 1
    blk.sj = 14 + 1 + 2 * 5
    blk.si = blk.sj * (12 + 1 + 2 * 5) - 1
    assert L.mhd_hall_emf_static_scratch(ctypes.byref(blk), dummy, dummy, dummy, None) == 1
