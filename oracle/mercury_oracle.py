"""Driver for the reference-built CPU oracle (test infrastructure only).

``oracle/_ref/mercury_ref`` is the reference solver compiled from its own,
unmodified sources (``oracle/Makefile``) plus ``oracle/ref_harness.cpp``.
This module writes the harness job file, runs it, and reads the field dumps.
Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
use it; the product never does.
"""
from __future__ import annotations

import os
import struct
import shutil
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "mercury_ref")


def available() -> bool:
    return os.path.isfile(REF_BIN) and os.access(REF_BIN, os.X_OK)


@dataclass
class Record:
    name: str
    block: int
    lo: tuple
    hi: tuple
    ncomp: int
    data: np.ndarray  # shape (ni, nj, nk, ncomp), reference (i, j, k, m) order

    def at(self, i, j, k, m=0):
        return self.data[i - self.lo[0], j - self.lo[1], k - self.lo[2], m]

    def inner(self):
        """Owned DOFs: logical [0, hi - g) per axis, g = -lo (FieldBlock.h:34-35)."""
        g = [-x for x in self.lo]
        return self.data[g[0] : self.hi[0], g[1] : self.hi[1], g[2] : self.hi[2]]


def read_dump(path: str) -> dict:
    """Read an ``MHDDUMP1`` file into {(name, block): Record}."""
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"MHDDUMP1":
            raise ValueError(f"{path}: not an oracle dump")
        (nrec,) = struct.unpack("<i", f.read(4))
        for _ in range(nrec):
            (ln,) = struct.unpack("<i", f.read(4))
            name = f.read(ln).decode()
            block, l0, l1, l2, h0, h1, h2, nc = struct.unpack("<8i", f.read(32))
            shape = (h0 - l0, h1 - l1, h2 - l2, nc)
            n = shape[0] * shape[1] * shape[2] * nc
            data = np.frombuffer(f.read(8 * n), dtype="<f8").reshape(shape).copy()
            out[(name, block)] = Record(name, block, (l0, l1, l2), (h0, h1, h2), nc, data)
    return out


def run_job(job: dict, timeout: float = 3600.0, workdir: str | None = None) -> dict:
    """Run the reference harness with ``job`` (key -> value) and return its dump."""
    if not available():
        raise FileNotFoundError(f"{REF_BIN} is not built (make -C oracle REF=<reference sources>)")
    own = workdir is None
    if own:  # a fresh folder under the oracle's own (git-ignored) build directory, removed afterwards
        jobs = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "jobs")
        os.makedirs(jobs, exist_ok=True)
        workdir = tempfile.mkdtemp(prefix="job_", dir=jobs)
    tmp = workdir
    os.makedirs(tmp, exist_ok=True)
    dump = os.path.join(tmp, "dump.bin")
    jobfile = os.path.join(tmp, "job.txt")
    lines = dict(job)
    lines.setdefault("out", dump)
    lines.setdefault("workdir", os.path.join(tmp, "work"))
    with open(jobfile, "w") as f:
        for k, v in lines.items():
            f.write(f"{k} {v}\n")
    try:
        proc = subprocess.run([REF_BIN, jobfile], capture_output=True, text=True, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"oracle failed ({proc.returncode}):\n{proc.stdout[-4000:]}\n{proc.stderr[-4000:]}")
        return read_dump(lines["out"])
    finally:
        if own:
            shutil.rmtree(tmp, ignore_errors=True)


# The cube case: periodic curvilinear unit cube, Orszag-Tang vortex, two ion
# fluids, Hall + electron pressure on, resistivity off, CFL 0.4.  The IMF is
# zero so the background field Badd vanishes and B is the vortex field alone.
CUBE_JOB = {
    "case": "cube",
    "n": 32,
    "amp": 0.05,
    "cfl": 0.4,
    "steps": 100,
    "resistive": 0,
    "ambipolar": 1,
    "hall_r_min": 0.0,
    "hall_r_max": 0.0,
    "noise": 1e-3,
    "solve_id": 0,
    "initial_line": "4.03112887E5 1.7407E5 4E7 0.001 1.240347346E-1 0.0 0.0 0.0 0.0",
}

STATE_FIELDS = ["U_H", "U_Na", "B_xi", "B_eta", "B_zeta"]
DERIVED_FIELDS = ["PV_H", "PV_Na", "U_plus", "B_cell", "Bind_cell", "J_cell", "J_xi", "J_eta", "J_zeta"]
WORK_FIELDS = ["RHS_H", "RHS_Na", "F_xi", "F_eta", "F_zeta", "RHS_B_xi", "RHS_B_eta", "RHS_B_zeta",
               "E_xi", "E_eta", "E_zeta", "Ehall_xi", "Ehall_eta", "Ehall_zeta",
               "Eface_xi", "Eface_eta", "Eface_zeta"]
STATIC_FIELDS = ["Jac", "JDxi", "JDet", "JDze", "Area_xi", "Area_eta", "Area_zeta",
                 "dl_xi", "dl_eta", "dl_zeta", "dr_xi", "dr_eta", "dr_zeta",
                 "Hodge_star_2form_to_1form_face_xi_lumped", "Hodge_star_2form_to_1form_face_eta_lumped",
                 "Hodge_star_2form_to_1form_face_zeta_lumped",
                 "Hodge_star_inverse_2form_to_1form_edge_xi_lumped",
                 "Hodge_star_inverse_2form_to_1form_edge_eta_lumped",
                 "Hodge_star_inverse_2form_to_1form_edge_zeta_lumped",
                 "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Badd_xi", "Badd_eta", "Badd_zeta", "Photo_rate"]


def cube_run(n=32, steps=100, dump_at=None, extra=None, workdir=None):
    """Run the periodic curvilinear Orszag-Tang cube (32^3, or another n) on the reference build.

    Returns the dump: ``static:<name>`` (block 0) for the static inputs and the
    Hall taper, grid arrays, and ``step<k>:<name>`` for state + derived + work
    fields at each requested step (0 = the initial state after the reference's
    Sync/UpdateDerivedFields_ preamble)."""
    job = dict(CUBE_JOB)
    job.update(n=n, steps=steps, dump_grid=1, dump_taper=1,
               dump_static=" ".join(STATIC_FIELDS),
               dump_fields=" ".join(STATE_FIELDS + DERIVED_FIELDS + WORK_FIELDS),
               dump_at=" ".join(str(s) for s in (dump_at or [0, steps])))
    if extra:
        job.update(extra)
    return run_job(job, workdir=workdir)


def restatement_inputs(dump, tag="step0:"):
    """Map a reference dump onto the restatement's slots (lo, hi, array)."""
    from restatement import SLOTS, REF_NAME  # noqa: E402  (oracle-local module)

    out = {}
    for slot in SLOTS:
        if slot in ("Ehc", "hall_beta"):
            r = dump[(tag + "B_cell", 0)]
            nc = 3 if slot == "Ehc" else 1
            out[slot] = (r.lo, r.hi, np.zeros(r.data.shape[:3] + (nc,)))
            continue
        if slot in ("dual_x", "dual_y", "dual_z"):
            r = dump[(slot, 0)]
        elif (tag + slot, 0) in dump:
            r = dump[(tag + slot, 0)]
        else:
            r = dump[("static:" + REF_NAME.get(slot, slot), 0)]
        out[slot] = (r.lo, r.hi, r.data.copy())
    return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


# The shell case: 6-panel cubed-sphere shell r in [1, 8], 48x48x96 cells per
# panel (r_k = 8^(k/96)), inner wall (the reference's Coupled-Solid handlers),
# outer Farfield; upstream v = (-4, 0, 0), n = 1, p = 0.1, IMF (0, 0, -0.2);
# centred dipole, tilt 0, |B| = 1 at the surface equator (moment in A m^2 with
# the reference's own nondimensionalisation, operators/Dipole.h:46-80);
# two ion fluids, Na+ at 1e-3 number fraction; Hall on (the reference's
# production taper r_min 1.1, r_max 1.2); CFL 0.4.
SHELL_UPSTREAM = "1612400.0 1954409.5501563628 4E7 0.001 0.0 0.0 0.0 0.0 -2.0000000000000003e-10"
SHELL_JOB = {
    "case": "shell",
    "na": 48,
    "nr": 96,
    "r_out": 8.0,
    "cfl": 0.4,
    "steps": 200,
    "resistive": 0,
    "ambipolar": 1,
    "hall_r_min": 1.1,
    "hall_r_max": 1.2,
    "init": "na_fraction",
    "na_fraction": 1e-3,
    "num_of_dipole": 1,
    "dipole_line": "0.0 0.0 0.0 0.0 0.0 -1.452678400462402e+17 0.0",
    "initial_line": SHELL_UPSTREAM,
    "farfield_line": "1612400.0 1954409.5501563628 4E7 0.0 0.0",
}


def shell_run(na=8, nr=16, steps=5, dump_at=None, extra=None, workdir=None):
    """Run the cubed-sphere shell case (SHELL_JOB with na x na x nr cells per
    panel) on the reference build; returns the dump with the static inputs,
    the Hall taper (edges and cell centres), the grid and the state, derived
    and work fields at the requested steps (0 = after the preamble)."""
    job = dict(SHELL_JOB)
    job.update(na=na, nr=nr, steps=steps, dump_grid=1, dump_taper=1,
               dump_static=" ".join(STATIC_FIELDS),
               dump_fields=" ".join(STATE_FIELDS + DERIVED_FIELDS + WORK_FIELDS),
               dump_at=" ".join(str(s) for s in (dump_at or [0, steps])))
    if extra:
        job.update(extra)
    return run_job(job, workdir=workdir)
