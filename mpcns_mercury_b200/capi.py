"""ctypes binding of the C ABI in include/mercury_mhd.h (libmercury_mhd.so).

The structures mirror the header one for one.  The library is loaded from the
package directory; there is no fallback: a missing or unloadable library is
an error.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# MERCURY_MHD_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = os.environ.get("MERCURY_MHD_LIB") or os.path.join(HERE, "libmercury_mhd.so")

# enum mhd_field, in header order
FIELDS = [
    "U_H", "U_NA", "B_XI", "B_ETA", "B_ZETA",
    "PV_H", "PV_NA", "U_PLUS", "B_CELL", "BIND_CELL", "J_CELL", "J_XI", "J_ETA", "J_ZETA",
    "E_XI", "E_ETA", "E_ZETA", "EHALL_XI", "EHALL_ETA", "EHALL_ZETA",
    "EFACE_XI", "EFACE_ETA", "EFACE_ZETA", "EHC", "HALL_BETA", "UCON", "DIVB", "FNORM_XI", "FNORM_ETA", "FNORM_ZETA", "PE_NODE", "AMBI_COEF",
    "DPE", "UCON_COEF", "HALL_IH_XI", "HALL_IH_ETA", "HALL_IH_ZETA", "FLUX_METRIC",
    "JAC", "JDXI", "JDET", "JDZE", "AREA_XI", "AREA_ETA", "AREA_ZETA",
    "DL_XI", "DL_ETA", "DL_ZETA", "DR_XI", "DR_ETA", "DR_ZETA",
    "HODGE_FACE_XI", "HODGE_FACE_ETA", "HODGE_FACE_ZETA",
    "HODGE_EDGE_XI", "HODGE_EDGE_ETA", "HODGE_EDGE_ZETA",
    "BCELL_W", "JCELL_W", "BADD_XI", "BADD_ETA", "BADD_ZETA", "PHOTO",
    "CELL_X", "CELL_Y", "CELL_Z", "TAPER_XI", "TAPER_ETA", "TAPER_ZETA", "TAPER_CELL",
    "LOCAL_ETA_XI", "LOCAL_ETA_ETA", "LOCAL_ETA_ZETA", "ETA_RES_XI", "ETA_RES_ETA", "ETA_RES_ZETA",
    "RES_W", "RES_X", "RES_R", "RES_P", "RES_Q", "RES_BSTAR",
]
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}

# Reference catalog name -> mhd_field (Z4_Mercury/include/0_MercuryFieldCatalog.h,
# src/7_metric/Metric.cpp:14-73)
REF_FIELD = {
    "U_H": "U_H", "U_Na": "U_NA", "B_xi": "B_XI", "B_eta": "B_ETA", "B_zeta": "B_ZETA",
    "PV_H": "PV_H", "PV_Na": "PV_NA", "U_plus": "U_PLUS", "B_cell": "B_CELL", "Bind_cell": "BIND_CELL",
    "J_cell": "J_CELL", "J_xi": "J_XI", "J_eta": "J_ETA", "J_zeta": "J_ZETA",
    "E_xi": "E_XI", "E_eta": "E_ETA", "E_zeta": "E_ZETA",
    "Ehall_xi": "EHALL_XI", "Ehall_eta": "EHALL_ETA", "Ehall_zeta": "EHALL_ZETA",
    "Eface_xi": "EFACE_XI", "Eface_eta": "EFACE_ETA", "Eface_zeta": "EFACE_ZETA",
    "Jac": "JAC", "JDxi": "JDXI", "JDet": "JDET", "JDze": "JDZE",
    "Area_xi": "AREA_XI", "Area_eta": "AREA_ETA", "Area_zeta": "AREA_ZETA",
    "dl_xi": "DL_XI", "dl_eta": "DL_ETA", "dl_zeta": "DL_ZETA",
    "dr_xi": "DR_XI", "dr_eta": "DR_ETA", "dr_zeta": "DR_ZETA",
    "Hodge_star_2form_to_1form_face_xi_lumped": "HODGE_FACE_XI",
    "Hodge_star_2form_to_1form_face_eta_lumped": "HODGE_FACE_ETA",
    "Hodge_star_2form_to_1form_face_zeta_lumped": "HODGE_FACE_ZETA",
    "Hodge_star_inverse_2form_to_1form_edge_xi_lumped": "HODGE_EDGE_XI",
    "Hodge_star_inverse_2form_to_1form_edge_eta_lumped": "HODGE_EDGE_ETA",
    "Hodge_star_inverse_2form_to_1form_edge_zeta_lumped": "HODGE_EDGE_ZETA",
    "Bcell_from_Bface_w": "BCELL_W", "Jcell_from_Jedge_w": "JCELL_W",
    "Badd_xi": "BADD_XI", "Badd_eta": "BADD_ETA", "Badd_zeta": "BADD_ZETA", "Photo_rate": "PHOTO",
    "divB": "DIVB", "taper_xi": "TAPER_XI", "taper_eta": "TAPER_ETA", "taper_zeta": "TAPER_ZETA",
    "taper_cell": "TAPER_CELL",
    "eta_res_xi": "ETA_RES_XI", "eta_res_eta": "ETA_RES_ETA", "eta_res_zeta": "ETA_RES_ZETA",
    "local_arti_eta_xi": "LOCAL_ETA_XI", "local_arti_eta_eta": "LOCAL_ETA_ETA", "local_arti_eta_zeta": "LOCAL_ETA_ZETA",
}

GROUPS = ["UCELL", "BFACE", "EHALL", "EEDGE", "B_CELL", "JEDGE", "J_CELL", "ERES", "DB", "BADD"]
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_OOM", 4: "ERR_DT", 5: "ERR_NONFINITE", 6: "ERR_SOLVE",
          7: "ERR_STATE", 8: "ERR_TIMEOUT"}


class MhdConstants(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "gamma", "M_H", "M_Na", "M_ref", "T_ref", "L_ref", "U_ref", "B_ref", "n_ref", "rho_ref", "m_Na",
        "k_Boltz", "q_e", "mu0", "state_coeff_H", "state_coeff_Na", "CFL", "hall_coef",
        "momentum_induce_coeff", "momentum_hall_coeff", "inver_MA2", "ne_hall_floor",
        "arti_eta_max", "arti_J_start", "arti_J_on")] + [
        ("ambipolar", ctypes.c_int32), ("local_arti", ctypes.c_int32), ("res_rtol", ctypes.c_double),
        ("resistive", ctypes.c_int32), ("res_max_it", ctypes.c_int32), ("bc", ctypes.c_double * 19),
        ("res_direct_iters", ctypes.c_int32), ("pad_", ctypes.c_int32)]


# indices into MhdConstants.bc (enum mhd_bc_const)
BC_QINF, BC_QINFS, BC_BIMF, BC_ZERO, BC_NA_RHO_FLOOR, BC_NA_E_FLOOR, BC_UINF = 0, 5, 10, 13, 14, 15, 16
MHD_STAGING = 1000  # pseudo field of a staging slot in MhdDof
PHYS_SET, PHYS_WALL, PHYS_EFAR = 0, 1, 2
BC_FARFIELD, BC_SOLID = 0, 1


class MhdDof(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("field", "block", "i", "j", "k", "comp")]


class MhdCopy(ctypes.Structure):
    _fields_ = [("dst", MhdDof), ("src", MhdDof), ("sign", ctypes.c_double)]


class MhdPhysOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("arg", ctypes.c_int32), ("dst", MhdDof), ("src", MhdDof)]


class MhdSyncGroup(ctypes.Structure):
    _fields_ = [("n_halo", ctypes.c_int32), ("n_owner", ctypes.c_int32),
                ("halo", ctypes.POINTER(MhdCopy)), ("owner", ctypes.POINTER(MhdCopy)),
                ("n_phys", ctypes.c_int32), ("n_stash", ctypes.c_int32),
                ("phys", ctypes.POINTER(MhdPhysOp)), ("stash", ctypes.POINTER(MhdCopy))]


class MhdAliasClasses(ctypes.Structure):
    _fields_ = [("n_classes", ctypes.c_int32), ("offset", ctypes.POINTER(ctypes.c_int32)),
                ("member", ctypes.POINTER(MhdDof)), ("member_sign", ctypes.POINTER(ctypes.c_double)),
                ("owner", ctypes.POINTER(MhdDof)), ("owner_sign", ctypes.POINTER(ctypes.c_double))]


class MhdSingularAlias(ctypes.Structure):
    _fields_ = [("edge", MhdDof), ("orient", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class MhdSingularCell(ctypes.Structure):
    _fields_ = [("cell", MhdDof), ("axis", ctypes.c_int32), ("orient", ctypes.c_int32)]


class MhdSingularFace(ctypes.Structure):
    _fields_ = [("face", MhdDof), ("sign", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class MhdSingularEdges(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_int32), ("owner", ctypes.POINTER(MhdDof)),
                ("owner_sign", ctypes.POINTER(ctypes.c_double)), ("alias_offset", ctypes.POINTER(ctypes.c_int32)),
                ("aliases", ctypes.POINTER(MhdSingularAlias)), ("cell_offset", ctypes.POINTER(ctypes.c_int32)),
                ("cells", ctypes.POINTER(MhdSingularCell)), ("face_offset", ctypes.POINTER(ctypes.c_int32)),
                ("faces", ctypes.POINTER(MhdSingularFace))]


class MhdBackground(ctypes.Structure):
    """mhd_background: dipoles (x0 y0 z0 mx my mz a, SI), IMF [T], units,
    Hall taper radii, implicit resistivity window."""
    _fields_ = [("n_dipoles", ctypes.c_int32), ("pad_", ctypes.c_int32), ("dipole", (ctypes.c_double * 7) * 4),
                ("B_imf", ctypes.c_double * 3), ("L_ref", ctypes.c_double), ("B_ref", ctypes.c_double),
                ("mu_mag", ctypes.c_double), ("hall_r_min", ctypes.c_double), ("hall_r_max", ctypes.c_double),
                ("inver_Rem", ctypes.c_double), ("eta_r_inner", ctypes.c_double), ("eta_r_outer", ctypes.c_double),
                ("eta_width", ctypes.c_double)]


class MhdDesc(ctypes.Structure):
    _fields_ = [("n_blocks", ctypes.c_int32), ("cells", ctypes.POINTER(ctypes.c_int32)),
                ("nghost", ctypes.c_int32), ("precision", ctypes.c_int32), ("constants", MhdConstants),
                ("groups", MhdSyncGroup * len(GROUPS)), ("edge_aliases", MhdAliasClasses),
                ("n_staging", ctypes.c_int32), ("n_wall", ctypes.c_int32), ("wall", ctypes.POINTER(MhdPhysOp)),
                ("singular", MhdSingularEdges)]


class MhdPatch(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("this_block", "nb_block", "direction", "nb_direction")] + [
        (n, ctypes.c_int32 * 3) for n in ("this_lo", "this_hi", "nb_lo", "nb_hi", "perm", "sign", "offset")] + [
        ("dir3", ctypes.c_int32)]


class MhdPhysicalPatch(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("block", "direction", "bc", "pad_")] + [
        ("lo", ctypes.c_int32 * 3), ("hi", ctypes.c_int32 * 3)]


class MhdInfo(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("dt", ctypes.c_double), ("step", ctypes.c_int64),
                ("status", ctypes.c_int32), ("pad_", ctypes.c_int32), ("device_bytes", ctypes.c_int64),
                ("remaining", ctypes.c_int64), ("res_relres", ctypes.c_double), ("res_iters", ctypes.c_int32),
                ("res_refinements", ctypes.c_int32)]


RESTART_FIELDS = ["U_H", "U_Na", "B_xi", "B_eta", "B_zeta"]  # MPCNSRST field list, in file order
RESTART_CAPI = ["U_H", "U_NA", "B_XI", "B_ETA", "B_ZETA"]


class MhdRestartImage(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int32), ("time", ctypes.c_double), ("n_blocks", ctypes.c_int32),
                ("cells", ctypes.POINTER(ctypes.c_int32)), ("nghost", ctypes.c_int32),
                ("data", ctypes.POINTER(ctypes.c_double) * 5), ("loaded", ctypes.c_uint32)]


TECPLOT_FIELDS = ["PV_H", "PV_Na", "B_cell", "Bind_cell", "Na", "J_cell"]  # mhd_tecplot_image.cell order
_DPP = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))


class MhdTecplotImage(ctypes.Structure):
    _fields_ = [("n_blocks", ctypes.c_int32), ("cells", ctypes.POINTER(ctypes.c_int32)),
                ("block_names", ctypes.POINTER(ctypes.c_char_p)), ("time", ctypes.c_double),
                ("nodes", _DPP), ("jac", _DPP), ("jac_ghost", ctypes.c_int32),
                ("cell", _DPP * 6), ("cell_ghost", ctypes.c_int32)]


EXPORTS = [
    "mhd_ctx_create", "mhd_ctx_destroy", "mhd_upload_field", "mhd_download_field", "mhd_prepare", "mhd_step",
    "mhd_step_async", "mhd_synchronize", "mhd_sync", "mhd_get_info", "mhd_get_status", "mhd_field_info", "mhd_stream",
    "mhd_kernels_per_step", "mhd_device_view", "mhd_last_error", "mhd_topology_periodic_block", "mhd_topology_periodic_lattice",
    "mhd_topology_multiblock", "mhd_topology_cubed_sphere", "mhd_topology_patches", "mhd_topology_physical",
    "mhd_topology_fill_desc", "mhd_topology_destroy", "mhd_batch_create", "mhd_batch_destroy", "mhd_batch_reserve",
    "mhd_div_b", "mhd_batch_div_b", "mhd_setup_geometry", "mhd_batch_setup_geometry", "mhd_restart_values", "mhd_restart_write", "mhd_restart_read",
    "mhd_save_restart", "mhd_load_restart", "mhd_tecplot_write", "mhd_rundata_write", "mhd_rundata_read", "mhd_batch_save_restart", "mhd_batch_load_restart", "mhd_desc_device_bytes", "mhd_batch_add", "mhd_batch_add_periodic", "mhd_batch_add_like", "mhd_batch_remove", "mhd_batch_upload_field",
    "mhd_batch_download_field", "mhd_batch_sync", "mhd_batch_prepare", "mhd_batch_request", "mhd_batch_run", "mhd_batch_substep_ms", "mhd_batch_cg_host_loop",
    "mhd_batch_poll", "mhd_batch_poll_async", "mhd_batch_poll_wait", "mhd_batch_stream", "mhd_batch_kernels_per_step", "mhd_batch_step_profiled",
    "mhd_batch_device_view", "mhd_shell_nodes", "mhd_shell_grid", "mhd_hall_taper", "mhd_setup_geometry_bg",
    "mhd_batch_setup_geometry_bg", "mhd_fill_field", "mhd_batch_fill_field", "mhd_set_constants",
    "mhd_batch_set_constants", "mhd_fluid_tile_shape", "mhd_batch_fluid_tile", "mhd_batch_time_fluid_tiles",
    "mhd_fluid_tile",
]

_lib = None


class MhdError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        msg = _lib.mhd_last_error().decode() if _lib is not None else ""
        super().__init__(f"{where}: {STATUS.get(code, code)} {msg}")


def lib() -> ctypes.CDLL:
    """Load libmercury_mhd.so (building it first if it is missing and nvcc is
    present).  Raises if the library cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.mhd_ctx_create.argtypes = [ctypes.POINTER(MhdDesc), ctypes.POINTER(P)]
    L.mhd_ctx_destroy.argtypes = [P]
    L.mhd_upload_field.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, i32p, i32p, ctypes.c_int]
    L.mhd_download_field.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, i32p, i32p, ctypes.c_int]
    L.mhd_prepare.argtypes = [P, ctypes.c_double, ctypes.c_int64]
    L.mhd_step.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.mhd_step_async.argtypes = [P, ctypes.c_int]
    L.mhd_synchronize.argtypes = [P]
    L.mhd_sync.argtypes = [P, ctypes.c_int]
    L.mhd_get_info.argtypes = [P, ctypes.POINTER(MhdInfo)]
    L.mhd_get_status.argtypes = [P, ctypes.POINTER(ctypes.c_int32)]
    L.mhd_field_info.argtypes = [ctypes.c_int, i32p, i32p]
    L.mhd_stream.argtypes = [P]
    L.mhd_stream.restype = ctypes.c_void_p
    L.mhd_kernels_per_step.argtypes = [P]
    L.mhd_device_view.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                  i32p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), i32p]
    L.mhd_last_error.restype = ctypes.c_char_p
    L.mhd_topology_cubed_sphere.argtypes = [ctypes.c_int32] * 4 + [ctypes.POINTER(P)]
    L.mhd_topology_multiblock.argtypes = [ctypes.c_int32, i32p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.POINTER(MhdPatch), ctypes.c_int32, ctypes.POINTER(MhdPhysicalPatch),
                                          ctypes.c_int32, ctypes.POINTER(P)]
    L.mhd_topology_patches.argtypes = [P, ctypes.c_int32, ctypes.POINTER(ctypes.POINTER(MhdPatch)),
                                       ctypes.POINTER(ctypes.c_int32)]
    L.mhd_topology_physical.argtypes = [P, ctypes.POINTER(ctypes.POINTER(MhdPhysicalPatch)),
                                        ctypes.POINTER(ctypes.c_int32)]
    L.mhd_topology_periodic_block.argtypes = [i32p, ctypes.c_int32, ctypes.POINTER(P)]
    L.mhd_topology_periodic_lattice.argtypes = [i32p, i32p, ctypes.c_int32, ctypes.POINTER(P)]
    L.mhd_topology_fill_desc.argtypes = [P, ctypes.POINTER(MhdDesc)]
    L.mhd_topology_destroy.argtypes = [P]
    L.mhd_batch_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
    L.mhd_div_b.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
    L.mhd_setup_geometry.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_double]
    L.mhd_shell_nodes.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                  ctypes.c_void_p]
    L.mhd_fluid_tile_shape.argtypes = [ctypes.c_int, i32p]
    L.mhd_batch_fluid_tile.argtypes = [P, ctypes.c_int]
    L.mhd_fluid_tile.argtypes = [P, ctypes.c_int]
    L.mhd_batch_time_fluid_tiles.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.mhd_set_constants.argtypes = [P, ctypes.POINTER(MhdConstants)]
    L.mhd_batch_set_constants.argtypes = [P, ctypes.c_int, ctypes.POINTER(MhdConstants)]
    L.mhd_fill_field.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, i32p, i32p, ctypes.c_int]
    L.mhd_batch_fill_field.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, i32p, i32p,
                                       ctypes.c_int]
    L.mhd_setup_geometry_bg.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_double,
                                        ctypes.POINTER(MhdBackground)]
    L.mhd_batch_setup_geometry_bg.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_double,
                                              ctypes.POINTER(MhdBackground)]
    L.mhd_shell_grid.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p]
    L.mhd_hall_taper.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    L.mhd_batch_setup_geometry.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_double]
    RI = ctypes.POINTER(MhdRestartImage)
    L.mhd_restart_values.argtypes = [RI, ctypes.c_int32]
    L.mhd_restart_values.restype = ctypes.c_int64
    L.mhd_restart_write.argtypes = [ctypes.c_char_p, RI]
    L.mhd_tecplot_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(MhdTecplotImage)]
    L.mhd_rundata_write.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double), ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int32)]
    L.mhd_rundata_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    L.mhd_restart_read.argtypes = [ctypes.c_char_p, RI]
    L.mhd_save_restart.argtypes = [P, ctypes.c_char_p]
    L.mhd_load_restart.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)]
    L.mhd_batch_save_restart.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
    L.mhd_batch_load_restart.argtypes = [P, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32),
                                         ctypes.POINTER(ctypes.c_double)]
    L.mhd_batch_div_b.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.mhd_batch_destroy.argtypes = [P]
    L.mhd_batch_reserve.argtypes = [P, ctypes.c_int64]
    L.mhd_batch_add_periodic.argtypes = [P, i32p, ctypes.c_int32, ctypes.POINTER(MhdConstants), ctypes.POINTER(ctypes.c_int)]
    L.mhd_desc_device_bytes.argtypes = [ctypes.POINTER(MhdDesc)]
    L.mhd_desc_device_bytes.restype = ctypes.c_int64
    L.mhd_batch_add.argtypes = [P, ctypes.POINTER(MhdDesc), ctypes.POINTER(ctypes.c_int)]
    L.mhd_batch_add_like.argtypes = [P, ctypes.c_int, ctypes.POINTER(MhdConstants), ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int)]
    L.mhd_batch_remove.argtypes = [P, ctypes.c_int]
    L.mhd_batch_upload_field.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, i32p, i32p,
                                         ctypes.c_int]
    L.mhd_batch_download_field.argtypes = L.mhd_batch_upload_field.argtypes
    L.mhd_batch_sync.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.mhd_batch_prepare.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_int64]
    L.mhd_batch_request.argtypes = [P, ctypes.c_int, ctypes.c_int64]
    L.mhd_batch_run.argtypes = [P, ctypes.c_int]
    L.mhd_batch_substep_ms.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
    L.mhd_batch_cg_host_loop.argtypes = [P, ctypes.c_int]
    L.mhd_batch_poll.argtypes = [P, ctypes.POINTER(MhdInfo)]
    L.mhd_batch_poll_async.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
    L.mhd_batch_poll_wait.argtypes = [P, ctypes.c_int, ctypes.POINTER(MhdInfo)]
    L.mhd_batch_stream.argtypes = [P]
    L.mhd_batch_stream.restype = ctypes.c_void_p
    L.mhd_batch_kernels_per_step.argtypes = [P]
    L.mhd_batch_step_profiled.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int)]
    L.mhd_batch_device_view.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p), i32p, ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_int64), i32p]
    _lib = L
    return L


def check(rc, where):
    if rc != 0:
        raise MhdError(rc, where)


def field_info(field: str):
    nc, loc = ctypes.c_int32(), ctypes.c_int32()
    check(lib().mhd_field_info(FIELD_ID[field], ctypes.byref(nc), ctypes.byref(loc)), "mhd_field_info")
    return nc.value, loc.value


def _i3(v):
    return (ctypes.c_int32 * 3)(*[int(x) for x in v])


def _restart_shapes(cells, nghost):
    """Per state field, per block: the (ni, nj, nk, ncomp) FieldBlock shape."""
    stag = {"U_H": (0, 0, 0, 5), "U_Na": (0, 0, 0, 5), "B_xi": (1, 0, 0, 1), "B_eta": (0, 1, 0, 1),
            "B_zeta": (0, 0, 1, 1)}
    return {f: [tuple(n[a] + stag[f][a] + 2 * nghost for a in range(3)) + (stag[f][3],) for n in cells]
            for f in RESTART_FIELDS}


def restart_read(path, cells, nghost: int):
    """Read an MPCNSRST restart file (mhd_restart_read) for blocks of `cells`
    with `nghost` ghost layers: returns (step, time, {field: [array per block]})
    with only the fields the file holds; arrays are (ni, nj, nk, ncomp) over
    the FieldBlock range [-nghost, n + stagger + nghost)."""
    import numpy as np
    shapes = _restart_shapes(cells, nghost)
    bufs = {f: np.zeros(sum(int(np.prod(sh)) for sh in shapes[f])) for f in RESTART_FIELDS}
    cc = (ctypes.c_int32 * (3 * len(cells)))(*[int(x) for b in cells for x in b])
    img = MhdRestartImage(0, 0.0, len(cells), cc, nghost)
    for q, f in enumerate(RESTART_FIELDS):
        img.data[q] = bufs[f].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    check(lib().mhd_restart_read(os.fsencode(path), ctypes.byref(img)), "mhd_restart_read")
    out = {}
    for q, f in enumerate(RESTART_FIELDS):
        if img.loaded & (1 << q):
            arrs, off = [], 0
            for sh in shapes[f]:
                n = int(np.prod(sh))
                arrs.append(bufs[f][off:off + n].reshape(sh).copy())
                off += n
            out[f] = arrs
    return img.step, img.time, out


def restart_write(path, step: int, time: float, cells, nghost: int, fields):
    """Write an MPCNSRST restart file (mhd_restart_write); `fields` maps each
    of RESTART_FIELDS to a list of per-block arrays shaped as restart_read
    returns them."""
    import numpy as np
    shapes = _restart_shapes(cells, nghost)
    bufs = {}
    for f in RESTART_FIELDS:
        parts = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)).reshape(sh) for a, sh in zip(fields[f], shapes[f])]
        bufs[f] = np.concatenate([a.ravel() for a in parts])
    cc = (ctypes.c_int32 * (3 * len(cells)))(*[int(x) for b in cells for x in b])
    img = MhdRestartImage(int(step), float(time), len(cells), cc, nghost)
    for q, f in enumerate(RESTART_FIELDS):
        img.data[q] = bufs[f].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    check(lib().mhd_restart_write(os.fsencode(path), ctypes.byref(img)), "mhd_restart_write")


def tecplot_write(path, cells, block_names, time: float, nodes, jac, jac_ghost: int, fields, cell_ghost: int):
    """Write the checkpoint plot file (mhd_tecplot_write).  nodes: per block
    an array (n+1, n+1, n+1, 3) of node x, y, z; jac: per block Jac over
    [-jac_ghost, n + jac_ghost); fields: each of TECPLOT_FIELDS mapped to per
    block arrays over [-cell_ghost, n + cell_ghost) (FieldBlock layout)."""
    import numpy as np

    nb = len(cells)
    keep = []

    def ptrs(arrays):
        arr = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in arrays]
        keep.append(arr)
        return (ctypes.POINTER(ctypes.c_double) * nb)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in arr])

    cc = (ctypes.c_int32 * (3 * nb))(*[int(x) for b in cells for x in b])
    names = (ctypes.c_char_p * nb)(*[str(n).encode() for n in block_names])
    img = MhdTecplotImage()
    img.n_blocks = nb
    img.cells = cc
    img.block_names = names
    img.time = float(time)
    pn, pj = ptrs(nodes), ptrs(jac)
    img.nodes = ctypes.cast(pn, _DPP)
    img.jac = ctypes.cast(pj, _DPP)
    img.jac_ghost = int(jac_ghost)
    pf = [ptrs(fields[f]) for f in TECPLOT_FIELDS]
    for q in range(6):
        img.cell[q] = ctypes.cast(pf[q], _DPP)
    img.cell_ghost = int(cell_ghost)
    check(lib().mhd_tecplot_write(os.fsencode(path), ctypes.byref(img)), "mhd_tecplot_write")


MERCURY_NRES = 13  # residual references of the Mercury solver's run-data file


def rundata_write(path, step: int, time: float, dt: float, residual_ref=(1.0,) * MERCURY_NRES,
                  residual_max: float = 0.0, monitors_d=None, monitors_i=None):
    """Write the run-data file (mhd_rundata_write); monitors_d / monitors_i:
    {key: value} of double / int32 monitors."""
    ref = (ctypes.c_double * len(residual_ref))(*[float(v) for v in residual_ref])
    md, mi = dict(monitors_d or {}), dict(monitors_i or {})
    dk = (ctypes.c_char_p * max(1, len(md)))(*[k.encode() for k in md])
    dv = (ctypes.c_double * max(1, len(md)))(*[float(v) for v in md.values()])
    ik = (ctypes.c_char_p * max(1, len(mi)))(*[k.encode() for k in mi])
    iv = (ctypes.c_int32 * max(1, len(mi)))(*[int(v) for v in mi.values()])
    check(lib().mhd_rundata_write(os.fsencode(path), int(step), float(time), float(dt), len(residual_ref), ref,
                                  float(residual_max), len(md), dk, dv, len(mi), ik, iv), "mhd_rundata_write")


def rundata_read(path):
    """(step, time, dt) of a run-data file (mhd_rundata_read)."""
    st, t, dt = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
    check(lib().mhd_rundata_read(os.fsencode(path), ctypes.byref(st), ctypes.byref(t), ctypes.byref(dt)),
          "mhd_rundata_read")
    return st.value, t.value, dt.value


class Context:
    """One device-resident solve behind the C ABI (mhd_ctx)."""

    def __init__(self, cells, nghost: int, constants: MhdConstants, topology=None, precision: int = 0,
                 lattice=None, keep_topology: bool = False):
        """cells: cells per block; one block is periodic in every direction,
        lattice=(bx, by, bz) makes bx * by * bz equal blocks tile a periodic
        box (mhd_topology_periodic_lattice).  topology: a topology handle
        (mhd_topology_*) the context destroys at close, unless keep_topology
        (the caller shares it between solves of one grid)."""
        L = lib()
        self._cells = (ctypes.c_int32 * (3 * len(cells)))(*[int(x) for b in cells for x in b])
        self.desc = MhdDesc()
        self.desc.n_blocks = len(cells)
        self.desc.cells = self._cells
        self.desc.nghost = nghost
        self.desc.precision = precision
        self.desc.constants = constants
        self._topo = ctypes.c_void_p()
        self._owns_topo = topology is None or not keep_topology
        if topology is not None:  # a topology handle (mhd_topology_*) that fills the descriptor's tables
            self._topo = topology
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")
        elif lattice is not None:
            if len(cells) != lattice[0] * lattice[1] * lattice[2] or any(tuple(c) != tuple(cells[0]) for c in cells):
                raise ValueError("a lattice has bx * by * bz blocks of equal cells")
            check(L.mhd_topology_periodic_lattice(_i3(cells[0]), _i3(lattice), nghost, ctypes.byref(self._topo)),
                  "mhd_topology_periodic_lattice")
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")
        elif len(cells) == 1:
            check(L.mhd_topology_periodic_block(_i3(cells[0]), nghost, ctypes.byref(self._topo)),
                  "mhd_topology_periodic_block")
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")
        self.ctx = ctypes.c_void_p()
        check(L.mhd_ctx_create(ctypes.byref(self.desc), ctypes.byref(self.ctx)), "mhd_ctx_create")

    def upload(self, field: str, array: np.ndarray, lo, hi, block: int = 0):
        a = np.ascontiguousarray(array, dtype=np.float64)
        check(lib().mhd_upload_field(self.ctx, FIELD_ID[field], block, a.ctypes.data_as(ctypes.c_void_p),
                                     _i3(lo), _i3(hi), a.shape[-1]), f"upload {field}")

    def fluid_tile(self, variant: int):
        """Run the fluid kernel's tile variant `variant` (mhd_fluid_tile)."""
        check(lib().mhd_fluid_tile(self.ctx, int(variant)), "mhd_fluid_tile")

    def set_constants(self, constants: MhdConstants):
        """A new upstream state on the same grid (mhd_set_constants); prepare must follow."""
        self.constants = constants
        check(lib().mhd_set_constants(self.ctx, ctypes.byref(constants)), "mhd_set_constants")

    def fill(self, field: str, values, lo, hi, block: int = 0):
        """Every position of [lo, hi) set to values (one per component) on the device."""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(lib().mhd_fill_field(self.ctx, FIELD_ID[field], block, v.ctypes.data, _i3(lo), _i3(hi), v.size),
              f"fill {field}")

    def download(self, field: str, lo, hi, block: int = 0) -> np.ndarray:
        nc, _ = field_info(field)
        out = np.empty((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], nc), dtype=np.float64)
        check(lib().mhd_download_field(self.ctx, FIELD_ID[field], block, out.ctypes.data_as(ctypes.c_void_p),
                                       _i3(lo), _i3(hi), nc), f"download {field}")
        return out

    def prepare(self, time: float = 0.0, step: int = 0):
        check(lib().mhd_prepare(self.ctx, time, step), "mhd_prepare")

    def step(self, n: int = 1) -> float:
        dt = ctypes.c_double()
        check(lib().mhd_step(self.ctx, n, ctypes.byref(dt)), "mhd_step")
        return dt.value

    def step_async(self, n: int = 1):
        check(lib().mhd_step_async(self.ctx, n), "mhd_step_async")

    def synchronize(self):
        check(lib().mhd_synchronize(self.ctx), "mhd_synchronize")

    def sync(self, group: str):
        check(lib().mhd_sync(self.ctx, GROUPS.index(group)), f"mhd_sync {group}")

    def info(self) -> MhdInfo:
        inf = MhdInfo()
        check(lib().mhd_get_info(self.ctx, ctypes.byref(inf)), "mhd_get_info")
        return inf

    def status(self) -> int:
        """The sticky device status (0 = MHD_OK) after the queued work."""
        st = ctypes.c_int32()
        check(lib().mhd_get_status(self.ctx, ctypes.byref(st)), "mhd_get_status")
        return st.value

    def kernels_per_step(self) -> int:
        return lib().mhd_kernels_per_step(self.ctx)

    def div_b(self) -> float:
        """max |div B| over the owned cells (MHD_DIVB holds the field)."""
        v = ctypes.c_double()
        check(lib().mhd_div_b(self.ctx, ctypes.byref(v)), "mhd_div_b")
        return v.value

    def setup_geometry(self, nodes, block: int = 0, L_ref: float = 2.44e6):
        """Compute the block's static fields on the device from its nodes
        (mhd_setup_geometry); nodes: (ni, nj, nk, 3) over the node range."""
        import numpy as np
        a = np.ascontiguousarray(nodes, dtype=np.float64)
        check(lib().mhd_setup_geometry(self.ctx, block, a.ctypes.data, float(L_ref)), "mhd_setup_geometry")

    def setup_background(self, nodes, background, block: int = 0, L_ref: float = 2.44e6):
        """setup_geometry plus the background field, Hall taper and implicit
        resistivity of an MhdBackground (mhd_setup_geometry_bg); sync("BADD")
        once every block is set."""
        a = np.ascontiguousarray(nodes, dtype=np.float64)
        check(lib().mhd_setup_geometry_bg(self.ctx, block, a.ctypes.data, float(L_ref), ctypes.byref(background)),
              "mhd_setup_geometry_bg")

    def save_restart(self, path):
        """Write the state as an MPCNSRST restart file (mhd_save_restart)."""
        check(lib().mhd_save_restart(self.ctx, os.fsencode(path)), "mhd_save_restart")

    def load_restart(self, path):
        """Load an MPCNSRST restart file and prepare the solve at its step and
        time (mhd_load_restart); returns (step, time)."""
        st, t = ctypes.c_int32(), ctypes.c_double()
        check(lib().mhd_load_restart(self.ctx, os.fsencode(path), ctypes.byref(st), ctypes.byref(t)),
              "mhd_load_restart")
        return st.value, t.value

    def stream(self) -> int:
        return lib().mhd_stream(self.ctx)

    def close(self):
        if getattr(self, "ctx", None):
            lib().mhd_ctx_destroy(self.ctx)
            self.ctx = None
        if getattr(self, "_topo", None) and getattr(self, "_owns_topo", True):
            lib().mhd_topology_destroy(self._topo)
        self._topo = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolveDesc:
    """A solve descriptor (mhd_desc) with the storage it points to kept alive."""

    def __init__(self, cells, nghost: int, constants: MhdConstants, precision: int = 0, lattice=None, topology=None):
        """cells: cells per block.  One block: periodic in every direction.
        lattice=(bx, by, bz): the blocks (bx * by * bz equal ones, in the
        order of mhd_topology_periodic_lattice) tile a periodic box.
        topology: a topology handle (mhd_topology_*) whose tables fill the
        descriptor; the caller keeps it (and may share it between solves of
        one grid) and destroys it after the solves are added."""
        L = lib()
        self._cells = (ctypes.c_int32 * (3 * len(cells)))(*[int(x) for b in cells for x in b])
        self.desc = MhdDesc()
        self.desc.n_blocks = len(cells)
        self.desc.cells = self._cells
        self.desc.nghost = nghost
        self.desc.precision = precision
        self.desc.constants = constants
        self._topo = ctypes.c_void_p()
        self._owns_topo = topology is None
        if topology is not None:
            self._topo = topology
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")
        elif lattice is not None:
            if len(cells) != lattice[0] * lattice[1] * lattice[2] or any(tuple(c) != tuple(cells[0]) for c in cells):
                raise ValueError("a lattice has bx * by * bz blocks of equal cells")
            check(L.mhd_topology_periodic_lattice(_i3(cells[0]), _i3(lattice), nghost, ctypes.byref(self._topo)),
                  "mhd_topology_periodic_lattice")
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")
        elif len(cells) == 1:
            check(L.mhd_topology_periodic_block(_i3(cells[0]), nghost, ctypes.byref(self._topo)),
                  "mhd_topology_periodic_block")
            check(L.mhd_topology_fill_desc(self._topo, ctypes.byref(self.desc)), "mhd_topology_fill_desc")

    def device_bytes(self) -> int:
        return int(lib().mhd_desc_device_bytes(ctypes.byref(self.desc)))

    def close(self):
        if getattr(self, "_topo", None) and getattr(self, "_owns_topo", True):
            lib().mhd_topology_destroy(self._topo)
        self._topo = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent solves advanced together by one CUDA graph per step (mhd_batch)."""

    def __init__(self, capacity: int, precision: int = 0):
        self.capacity = capacity
        self.precision = precision
        self.b = ctypes.c_void_p()
        check(lib().mhd_batch_create(capacity, precision, ctypes.byref(self.b)), "mhd_batch_create")

    def add(self, desc: SolveDesc) -> int:
        slot = ctypes.c_int()
        check(lib().mhd_batch_add(self.b, ctypes.byref(desc.desc), ctypes.byref(slot)), "mhd_batch_add")
        return slot.value

    def add_like(self, src_slot: int, constants=None, copy_static: bool = True) -> int:
        slot = ctypes.c_int()
        cp = ctypes.byref(constants) if constants is not None else None
        check(lib().mhd_batch_add_like(self.b, src_slot, cp, int(copy_static), ctypes.byref(slot)),
              "mhd_batch_add_like")
        return slot.value

    def remove(self, slot: int):
        check(lib().mhd_batch_remove(self.b, slot), "mhd_batch_remove")

    def upload(self, slot: int, field: str, array: np.ndarray, lo, hi, block: int = 0):
        a = np.ascontiguousarray(array, dtype=np.float64)
        check(lib().mhd_batch_upload_field(self.b, slot, FIELD_ID[field], block, a.ctypes.data_as(ctypes.c_void_p),
                                           _i3(lo), _i3(hi), a.shape[-1]), f"upload {field}")

    def fill(self, slot: int, field: str, values, lo, hi, block: int = 0):
        """Every position of [lo, hi) of a solve set to values on the device (mhd_batch_fill_field)."""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(lib().mhd_batch_fill_field(self.b, slot, FIELD_ID[field], block, v.ctypes.data, _i3(lo), _i3(hi),
                                         v.size), f"fill {field}")

    def download(self, slot: int, field: str, lo, hi, block: int = 0) -> np.ndarray:
        nc, _ = field_info(field)
        out = np.empty((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], nc), dtype=np.float64)
        check(lib().mhd_batch_download_field(self.b, slot, FIELD_ID[field], block,
                                             out.ctypes.data_as(ctypes.c_void_p), _i3(lo), _i3(hi), nc),
              f"download {field}")
        return out

    def sync(self, slot: int, group: str):
        check(lib().mhd_batch_sync(self.b, slot, GROUPS.index(group)), f"mhd_batch_sync {group}")

    def prepare(self, slot: int, time: float = 0.0, step: int = 0):
        check(lib().mhd_batch_prepare(self.b, slot, time, step), "mhd_batch_prepare")

    def request(self, slot: int, nsteps: int):
        check(lib().mhd_batch_request(self.b, slot, nsteps), "mhd_batch_request")

    def run(self, nsteps: int):
        check(lib().mhd_batch_run(self.b, nsteps), "mhd_batch_run")

    def cg_host_loop(self, on: bool = True):
        """Launch the substep's CG iterations from the host (for profilers)."""
        check(lib().mhd_batch_cg_host_loop(self.b, int(bool(on))), "mhd_batch_cg_host_loop")

    def substep_ms(self) -> float:
        """Mean device ms per step of the implicit substep since the last call."""
        v = ctypes.c_double()
        check(lib().mhd_batch_substep_ms(self.b, ctypes.byref(v)), "mhd_batch_substep_ms")
        return v.value

    def poll(self):
        infos = (MhdInfo * self.capacity)()
        check(lib().mhd_batch_poll(self.b, infos), "mhd_batch_poll")
        return list(infos)

    def poll_async(self) -> int:
        t = ctypes.c_int()
        check(lib().mhd_batch_poll_async(self.b, ctypes.byref(t)), "mhd_batch_poll_async")
        return t.value

    def poll_wait(self, ticket: int):
        infos = (MhdInfo * self.capacity)()
        check(lib().mhd_batch_poll_wait(self.b, ticket, infos), "mhd_batch_poll_wait")
        return list(infos)

    def stream(self) -> int:
        return lib().mhd_batch_stream(self.b)

    def kernels_per_step(self) -> int:
        return lib().mhd_batch_kernels_per_step(self.b)

    def reserve(self, nbytes: int):
        """Grow the batch's device memory pool ahead of the solves (mhd_batch_reserve)."""
        check(lib().mhd_batch_reserve(self.b, int(nbytes)), "mhd_batch_reserve")

    def setup_geometry(self, slot: int, nodes, block: int = 0, L_ref: float = 2.44e6):
        """Compute a solve's static fields on the device from a block's nodes
        (mhd_batch_setup_geometry)."""
        import numpy as np
        a = np.ascontiguousarray(nodes, dtype=np.float64)
        check(lib().mhd_batch_setup_geometry(self.b, slot, block, a.ctypes.data, float(L_ref)),
              "mhd_batch_setup_geometry")

    def fluid_tile(self, variant: int):
        """Run the fluid kernel's tile variant `variant` (mhd_batch_fluid_tile)."""
        check(lib().mhd_batch_fluid_tile(self.b, int(variant)), "mhd_batch_fluid_tile")

    def time_fluid_tiles(self, reps: int = 5):
        """ms per fluid pass of every tile variant on the active solves (mhd_batch_time_fluid_tiles)."""
        ms = (ctypes.c_float * NUM_FLUID_TILES)()
        check(lib().mhd_batch_time_fluid_tiles(self.b, int(reps), ms), "mhd_batch_time_fluid_tiles")
        return [float(v) for v in ms]

    def setup_background(self, slot: int, nodes, background, block: int = 0, L_ref: float = 2.44e6):
        """setup_geometry plus an MhdBackground (mhd_batch_setup_geometry_bg);
        sync(slot, "BADD") once every block of the solve is set."""
        a = np.ascontiguousarray(nodes, dtype=np.float64)
        check(lib().mhd_batch_setup_geometry_bg(self.b, slot, block, a.ctypes.data, float(L_ref),
                                                ctypes.byref(background)), "mhd_batch_setup_geometry_bg")

    def save_restart(self, slot: int, path):
        """Write a solve's state as an MPCNSRST restart file (mhd_batch_save_restart)."""
        check(lib().mhd_batch_save_restart(self.b, slot, os.fsencode(path)), "mhd_batch_save_restart")

    def load_restart(self, slot: int, path):
        """Load an MPCNSRST restart file into a solve and prepare it
        (mhd_batch_load_restart); returns (step, time)."""
        st, t = ctypes.c_int32(), ctypes.c_double()
        check(lib().mhd_batch_load_restart(self.b, slot, os.fsencode(path), ctypes.byref(st), ctypes.byref(t)),
              "mhd_batch_load_restart")
        return st.value, t.value

    def add_periodic(self, cells, nghost: int, constants) -> int:
        """Add a one-block periodic solve with its tables compiled directly
        (mhd_batch_add_periodic); returns its slot."""
        slot = ctypes.c_int()
        check(lib().mhd_batch_add_periodic(self.b, _i3(cells), nghost, ctypes.byref(constants), ctypes.byref(slot)),
              "mhd_batch_add_periodic")
        return slot.value

    def close(self):
        if getattr(self, "b", None):
            lib().mhd_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NUM_FLUID_TILES = 7  # MHD_NUM_FLUID_TILES


def fluid_tile_shape(variant: int):
    """(k, j, i, CTAs per SM) of a fluid tile variant (mhd_fluid_tile_shape)."""
    out = (ctypes.c_int32 * 4)()
    check(lib().mhd_fluid_tile_shape(int(variant), out), "mhd_fluid_tile_shape")
    return tuple(int(v) for v in out)


def shell_nodes(na: int, nr: int, panel: int, r_out: float = 8.0, G: int = 5) -> np.ndarray:
    """Nodes of one panel of the cubed-sphere shell over [-G, n + 1 + G) per
    axis, (ni, nj, nk, 3) (mhd_shell_nodes)."""
    e0, e2 = na + 1 + 2 * G, nr + 1 + 2 * G
    out = np.empty((e0, e0, e2, 3), dtype=np.float64)
    check(lib().mhd_shell_nodes(na, nr, float(r_out), panel, G, out.ctypes.data), "mhd_shell_nodes")
    return out


def shell_grid(na: int, nr: int, r_out: float = 8.0, G: int = 5) -> np.ndarray:
    """All six panels' nodes with the ghost nodes of the reference's grid
    preprocessing, (6, ni, nj, nk, 3) (mhd_shell_grid)."""
    e0, e2 = na + 1 + 2 * G, nr + 1 + 2 * G
    out = np.empty((6, e0, e0, e2, 3), dtype=np.float64)
    check(lib().mhd_shell_grid(na, nr, float(r_out), G, out.ctypes.data), "mhd_shell_grid")
    return out


def hall_taper(r_min: float, r_max: float, xyz) -> np.ndarray:
    """The Hall radial taper at points xyz (..., 3) (mhd_hall_taper)."""
    a = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.empty(a.shape[:-1], dtype=np.float64)
    check(lib().mhd_hall_taper(float(r_min), float(r_max), out.size, a.ctypes.data, out.ctypes.data), "mhd_hall_taper")
    return out
