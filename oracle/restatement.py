"""ctypes front end of the C restatement ``oracle/mhd_oracle.c`` (test
infrastructure: the oracle).  Builds ``oracle/_build/libmhd_oracle.so`` on
first use with gcc (no FMA contraction, matching the reference's x86-64
build) and runs the restated step on numpy arrays in the reference's
FieldBlock layout."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mhd_oracle.c")
LIB = os.path.join(HERE, "_build", "libmhd_oracle.so")

# Slot order of the ofld members of struct octx (mhd_oracle.c).
SLOTS = (
    "U_H U_Na B_xi B_eta B_zeta "
    "PV_H PV_Na U_plus B_cell Bind_cell J_cell J_xi J_eta J_zeta "
    "RHS_H RHS_Na F_xi F_eta F_zeta RHS_B_xi RHS_B_eta RHS_B_zeta E_xi E_eta E_zeta "
    "Ehall_xi Ehall_eta Ehall_zeta Eface_xi Eface_eta Eface_zeta Ehc hall_beta "
    "Jac JDxi JDet JDze Area_xi Area_eta Area_zeta dl_xi dl_eta dl_zeta dr_xi dr_eta dr_zeta "
    "beta_xi beta_eta beta_zeta alpha_xi alpha_eta alpha_zeta Bcell_from_Bface_w Jcell_from_Jedge_w "
    "Badd_xi Badd_eta Badd_zeta Photo_rate dual_x dual_y dual_z taper_xi taper_eta taper_zeta"
).split()

# Reference field names of the static inputs that are stored under a different slot name.
REF_NAME = {
    "beta_xi": "Hodge_star_2form_to_1form_face_xi_lumped",
    "beta_eta": "Hodge_star_2form_to_1form_face_eta_lumped",
    "beta_zeta": "Hodge_star_2form_to_1form_face_zeta_lumped",
    "alpha_xi": "Hodge_star_inverse_2form_to_1form_edge_xi_lumped",
    "alpha_eta": "Hodge_star_inverse_2form_to_1form_edge_eta_lumped",
    "alpha_zeta": "Hodge_star_inverse_2form_to_1form_edge_zeta_lumped",
}

# Raw normalisation inputs, in the order oracle_create() reads them: the
# reference's production constants and REF list (Z4_Mercury/9999setup/
# 0_General_Setting.txt, 1_Initial_condition.txt) and the CFL number.
def raw_constants(cfl: float = 0.4):
    return [1.6667, 6.02e23, 8.314, 1.256637061e-6, 1.602e-19,
            4.031e5, 1.7407e5, 4e7, 0.001, 1e-9, 2.44e6,
            0.001, 0.023, cfl]


def build() -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                               "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.oracle_create.restype = ctypes.c_void_p
        _lib.oracle_create.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int]
        _lib.oracle_bind.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        for fn in ("oracle_step", "oracle_get_dt", "oracle_get_time"):
            getattr(_lib, fn).restype = ctypes.c_double
            getattr(_lib, fn).argtypes = [ctypes.c_void_p]
        _lib.oracle_update_derived.argtypes = [ctypes.c_void_p]
        _lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    return _lib


class Restatement:
    """One periodic block stepped by the C restatement.

    ``arrays`` maps slot names to (lo, hi, ndarray[ni, nj, nk, nc]) in the
    reference's FieldBlock index space; work and derived slots missing from it
    are allocated like the reference's catalog does.
    """

    def __init__(self, n: int, arrays: dict, cfl: float = 0.4, ambipolar: bool = True):
        L = lib()
        raw = (ctypes.c_double * 14)(*raw_constants(cfl))
        self.ctx = L.oracle_create(raw, n, int(ambipolar))
        self.arrays = {}
        for slot_id, name in enumerate(SLOTS):
            lo, hi, arr = arrays[name]
            arr = np.ascontiguousarray(arr, dtype=np.float64)
            self.arrays[name] = (lo, hi, arr)
            L.oracle_bind(self.ctx, slot_id, arr.ctypes.data_as(ctypes.c_void_p),
                          (ctypes.c_int * 3)(*lo), (ctypes.c_int * 3)(*hi), arr.shape[3])

    def update_derived(self):
        lib().oracle_update_derived(self.ctx)

    def step(self) -> float:
        return lib().oracle_step(self.ctx)

    def __getitem__(self, name):
        return self.arrays[name][2]

    def __del__(self):
        if getattr(self, "ctx", None):
            lib().oracle_destroy(self.ctx)
            self.ctx = None


# Extents of the derived and work fields, as the reference's catalog allocates
# them (Z4_Mercury/include/0_MercuryFieldCatalog.h:70-202): (stagger, ncomp, nghost)
_WORK = {
    "PV_H": ((0, 0, 0), 5, 4), "PV_Na": ((0, 0, 0), 5, 4), "U_plus": ((0, 0, 0), 3, 4),
    "B_cell": ((0, 0, 0), 3, 4), "Bind_cell": ((0, 0, 0), 3, 4), "J_cell": ((0, 0, 0), 3, 4),
    "J_xi": ((0, 1, 1), 1, 4), "J_eta": ((1, 0, 1), 1, 4), "J_zeta": ((1, 1, 0), 1, 4),
    "RHS_H": ((0, 0, 0), 5, 0), "RHS_Na": ((0, 0, 0), 5, 0),
    "F_xi": ((1, 0, 0), 5, 0), "F_eta": ((0, 1, 0), 5, 0), "F_zeta": ((0, 0, 1), 5, 0),
    "RHS_B_xi": ((1, 0, 0), 1, 0), "RHS_B_eta": ((0, 1, 0), 1, 0), "RHS_B_zeta": ((0, 0, 1), 1, 0),
    "E_xi": ((0, 1, 1), 1, 4), "E_eta": ((1, 0, 1), 1, 4), "E_zeta": ((1, 1, 0), 1, 4),
    "Ehall_xi": ((0, 1, 1), 1, 4), "Ehall_eta": ((1, 0, 1), 1, 4), "Ehall_zeta": ((1, 1, 0), 1, 4),
    "Eface_xi": ((1, 0, 0), 3, 4), "Eface_eta": ((0, 1, 0), 3, 4), "Eface_zeta": ((0, 0, 1), 3, 4),
    "Ehc": ((0, 0, 0), 3, 4), "hall_beta": ((0, 0, 0), 1, 4),
}
_SETUP_NAME = {"dual_x": None, "dual_y": None, "dual_z": None}


def inputs_from_fields(n: int, fields: dict):
    """Restatement slots from a case built by the package's host setup
    ({reference field name: (lo, hi, data)} plus cell_x/y/z cell centres)."""
    out = {}
    for slot in SLOTS:
        if slot in _WORK:
            st, nc, g = _WORK[slot]
            lo = (-g, -g, -g)
            hi = tuple(n + st[a] + g for a in range(3))
            out[slot] = (lo, hi, np.zeros(tuple(hi[a] - lo[a] for a in range(3)) + (nc,)))
        elif slot in ("dual_x", "dual_y", "dual_z"):
            lo, hi, data = fields["cell_" + slot[-1]]
            # dual(i+1, j+1, k+1) is the centre of cell (i, j, k)
            out[slot] = (tuple(v + 1 for v in lo), tuple(v + 1 for v in hi), data)
        else:
            out[slot] = fields[slot]
    return out


def sync_state(r: "Restatement"):
    L = lib()
    L.oracle_sync_state.argtypes = [ctypes.c_void_p]
    L.oracle_sync_state(r.ctx)
