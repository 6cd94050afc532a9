"""The magnetosphere case: a 6-panel cubed-sphere shell around a planet,
set up on the device from its parameters, with nothing uploaded but the
node coordinates and the initial state.

Parameters follow the reference's parameter lists: the INITIAL list (upstream
U [m/s], T [K], n [1/m^3], M, the flow direction cosines c_y, c_z and the IMF
Bx, By, Bz [T]), the Dipole<n> lists (x0 y0 z0 [m], mx my mz [A m^2], a [m]),
the Hall taper radii r_min, r_max and the implicit resistivity window
(mercury_eta_r_inner/_outer/_width, eta_max_mercury).

The grid is the shell of mhd_shell_grid: panels of na x na x nr cells,
r in [1, r_out] with r_k = r_out^(k / nr), inner sphere a solid wall
(Coupled-Solid), outer sphere Farfield; its ghost nodes are the ones the
reference's grid preprocessing leaves there, so the static fields computed on
the device from them are the reference's.  The initial state is the
reference's Common_Initial (Z4_Mercury/include/2_Initial.h:134-215) for H+,
U_H = the upstream state, with Na+ at a number-density fraction f of it at
the same velocity and temperature, and B (induced) = 0; then Sync(Ucell),
Sync(Bface) as the reference does before its first derived refresh
(Z4_Mercury/src/MercurySolver.cpp:133-145).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .constants import reference_constants

NGHOST = 4

# the INITIAL list of the magnetosphere workload: U T n M c_y c_z Bx By Bz
UPSTREAM = (1612400.0, 1954409.5501563628, 4e7, 0.001, 0.0, 0.0, 0.0, 0.0, -2.0000000000000003e-10)
# a centred dipole along -z (x0 y0 z0 mx my mz a)
DIPOLE = (0.0, 0.0, 0.0, 0.0, 0.0, -1.452678400462402e+17, 0.0)


# The configuration's implicit resistivity, eta = 1e-3 exp(-(r - 1) / 0.2) in
# units of mu0 U_ref L_ref (r in planet radii), written in the reference's one
# radial profile, the tanh window eta_max (tanh((r - r_in) / w) -
# tanh((r - r_out) / w)) / 2 (MercurySolver.cpp:173-181 reads its parameters):
# r_out = 1 and w = 0.4 make its outer flank exp(-2 (r - 1) / 0.4) =
# exp(-(r - 1) / 0.2) for r - 1 >> 0.2 (half of eta_max at the surface);
# r_in = 0 puts the inner flank inside the planet.  Solved to 1e-10.
ETA_CONFIG = dict(eta_max=1e-3 * 1.256637061e-6 * 4.031e5 * 2.44e6, eta_r_inner=0.0, eta_r_outer=1.0,
                  eta_width=0.4, res_rtol=1e-10, res_max_it=2000)


@dataclass
class ShellCase:
    na: int = 48                 # cells per panel along each angle
    nr: int = 96                 # cells along the radius
    r_out: float = 8.0           # outer radius (planet radii)
    upstream: tuple = UPSTREAM   # INITIAL list
    na_fraction: float = 1e-3    # Na+ number-density fraction
    dipoles: list = field(default_factory=lambda: [DIPOLE])
    hall_r_min: float = 1.1
    hall_r_max: float = 1.2
    cfl: float = 0.4
    resistive: bool = False
    eta_max: float = 1.25e7      # eta_max_mercury
    eta_r_inner: float = 0.84
    eta_r_outer: float = 1.04
    eta_width: float = 0.02
    res_rtol: float = 1e-13
    res_max_it: int = 500

    @property
    def cells(self):
        return [(self.na, self.na, self.nr)] * 6

    def cell_count(self) -> int:
        return 6 * self.na * self.na * self.nr


def constants(case: ShellCase):
    """The solve's mhd_constants (calc_physical_constant and the boundary
    values of the upstream state)."""
    return reference_constants(cfl=case.cfl, initial=tuple(case.upstream), resistive=case.resistive,
                               res_rtol=case.res_rtol, res_max_it=case.res_max_it)


def background(case: ShellCase, k=None) -> capi.MhdBackground:
    """The case's mhd_background: dipoles and IMF in SI, units of the REF
    list, the Hall taper radii and (with the implicit substep) the
    resistivity window with inver_Rem = eta_max / (mu_mag U_ref L_ref)."""
    k = k if k is not None else constants(case)
    bg = capi.MhdBackground()
    bg.n_dipoles = len(case.dipoles)
    for d, dip in enumerate(case.dipoles):
        for q in range(7):
            bg.dipole[d][q] = float(dip[q])
    for q in range(3):
        bg.B_imf[q] = float(case.upstream[6 + q])
    bg.L_ref, bg.B_ref, bg.mu_mag = k.L_ref, k.B_ref, k.mu0
    bg.hall_r_min, bg.hall_r_max = case.hall_r_min, case.hall_r_max
    if case.resistive:
        bg.inver_Rem = case.eta_max / (k.mu0 * k.U_ref * k.L_ref)
        bg.eta_r_inner, bg.eta_r_outer, bg.eta_width = case.eta_r_inner, case.eta_r_outer, case.eta_width
    return bg


def initial_state(case: ShellCase, k=None):
    """(U_H, U_Na) per cell: the upstream H+ state and Na+ at the number
    fraction f with the same velocity and temperature:
    rho_Na = f (M_Na / M_H) rho_H, p_Na = f p_H."""
    k = k if k is not None else constants(case)
    uh = np.array([k.bc[q] for q in range(5)], dtype=np.float64)
    g = k.gamma
    rho = uh[0]
    u, v, w = uh[1] / rho, uh[2] / rho, uh[3] / rho
    p = (g - 1.0) * (uh[4] - 0.5 * rho * (u * u + v * v + w * w))
    f = case.na_fraction
    rn, pn = f * (k.M_Na / k.M_H) * rho, f * p
    un = np.array([rn, rn * u, rn * v, rn * w, pn / (g - 1.0) + 0.5 * rn * (u * u + v * v + w * w)])
    return uh, un


def topology(case: ShellCase):
    """The shell's sync tables (mhd_topology_cubed_sphere); the caller owns
    the handle (a Context takes it over unless keep_topology)."""
    t = ctypes.c_void_p()
    capi.check(capi.lib().mhd_topology_cubed_sphere(case.na, case.nr, NGHOST, int(case.resistive), ctypes.byref(t)),
               "mhd_topology_cubed_sphere")
    return t


class TopologyCache:
    """Topologies shared by the solves of one grid: they depend only on
    (na, nr, resistive), not on the upstream parameters."""

    def __init__(self):
        self._t = {}

    def get(self, case: ShellCase):
        key = (case.na, case.nr, bool(case.resistive))
        if key not in self._t:
            self._t[key] = topology(case)
        return self._t[key]

    def close(self):
        for t in self._t.values():
            capi.lib().mhd_topology_destroy(t)
        self._t = {}


def set_up(target, case: ShellCase, slot=None, nodes=None, k=None) -> int:
    """Static fields, background and initial state of the case on the device
    of `target` (a Context, or a Batch with `slot`); the caller prepares.
    nodes: mhd_shell_grid's nodes (computed when None).  Returns the bytes
    sent to the device."""
    k = k if k is not None else constants(case)
    G = NGHOST + 1
    nodes = nodes if nodes is not None else capi.shell_grid(case.na, case.nr, case.r_out, G)
    bg = background(case, k)
    batch = slot is not None
    nbytes = 0
    for b in range(6):
        if batch:
            target.setup_background(slot, nodes[b], bg, block=b, L_ref=k.L_ref)
        else:
            target.setup_background(nodes[b], bg, block=b, L_ref=k.L_ref)
        nbytes += nodes[b].nbytes
    sync = (lambda g: target.sync(slot, g)) if batch else target.sync
    sync("BADD")
    uh, un = initial_state(case, k)
    n = (case.na, case.na, case.nr)
    lo = (-NGHOST, -NGHOST, -NGHOST)
    hi = tuple(c + NGHOST for c in n)
    fill = (lambda *a, **kw: target.fill(slot, *a, **kw)) if batch else target.fill
    for b in range(6):  # uniform values: filled on the device, nothing but 10 numbers sent
        fill("U_H", uh, lo, hi, block=b)
        fill("U_NA", un, lo, hi, block=b)
        for ax, fld in enumerate(("B_XI", "B_ETA", "B_ZETA")):
            fhi = list(hi)
            fhi[ax] += 1
            fill(fld, [0.0], lo, tuple(fhi), block=b)
        nbytes += 13 * 8
    sync("UCELL")
    sync("BFACE")
    return nbytes


def context(case: ShellCase, precision: int = 0, k=None, topologies: TopologyCache | None = None, nodes=None):
    """A Context holding the case, set up on the device and prepared
    (topologies: a cache to take the grid's tables from)."""
    k = k if k is not None else constants(case)
    if topologies is not None:
        ctx = capi.Context(case.cells, NGHOST, k, topology=topologies.get(case), precision=precision,
                           keep_topology=True)
    else:
        ctx = capi.Context(case.cells, NGHOST, k, topology=topology(case), precision=precision)
    set_up(ctx, case, k=k, nodes=nodes)
    ctx.prepare()
    return ctx


def ensemble(nsolves: int, stream: int = 300000, resistive: bool = True):
    """The magnetosphere ensemble: per solve, cells per panel axis drawn
    log-uniform (na in [24, 64], nr in [24, 128]: blocks of 24^3 to
    64 x 64 x 128 cells) and the upstream drawn uniform: speed |v| in [2, 6]
    and density n in [0.5, 3] (units of the REF list's U and n), IMF Bz in
    [-0.4, 0.4] (units of B_ref), Na+ fraction in [1e-4, 1e-2]; flow along
    the INITIAL list's axis, T and M of the base upstream; the implicit
    resistivity ETA_CONFIG (unless resistive is False).  Seeded draws
    (mhd_seeded_uniform's generator, solve_id = stream), computed without
    the CUDA library."""
    import math

    from .setup import host_uniform_sym

    u = host_uniform_sym(stream, 0.5, 6 * nsolves) + 0.5
    U_ref, n_ref, B_ref = 4.031e5, 4e7, 1e-9
    la, ha, hr = math.log(24.0), math.log(64.0), math.log(128.0)
    out = []
    for s in range(nsolves):
        a, b, c, d, e, f = u[6 * s:6 * s + 6]
        na = int(round(math.exp(la + a * (ha - la))))
        nr = int(round(math.exp(la + b * (hr - la))))
        v = 2.0 + 4.0 * c
        n = 0.5 + 2.5 * d
        bz = -0.4 + 0.8 * e
        frac = 1e-4 + (1e-2 - 1e-4) * f
        up = (v * U_ref, UPSTREAM[1], n * n_ref, UPSTREAM[3], 0.0, 0.0, 0.0, 0.0, bz * B_ref)
        out.append(ShellCase(na=na, nr=nr, upstream=up, na_fraction=frac, **_res(resistive)))
    return out


def _res(resistive: bool) -> dict:
    return dict(resistive=True, **ETA_CONFIG) if resistive else dict(resistive=False)


def request_stream(nreq: int, rate: float, shapes: int = 16, na_max: int = 96, nr_max: int = 192,
                   steps_min: int = 50, steps_max: int = 500, stream: int = 500000, resistive: bool = True):
    """A seeded Poisson stream of magnetosphere requests: [(arrival_s,
    ShellCase, steps)].  The grids come from a pool of ``shapes`` sizes drawn
    log-uniform (na in [24, na_max], nr in [24, nr_max]); each request has
    its own upstream conditions (the ensemble's ranges and resistivity),
    exponential inter-arrival times of mean 1 / rate and steps uniform in
    [steps_min, steps_max]."""
    import math

    from .setup import host_uniform_sym

    u = host_uniform_sym(stream, 0.5, 2 * shapes + 7 * nreq) + 0.5
    la = math.log(24.0)
    grid = [(int(round(math.exp(la + u[2 * g] * (math.log(na_max) - la)))),
             int(round(math.exp(la + u[2 * g + 1] * (math.log(nr_max) - la))))) for g in range(shapes)]
    U_ref, n_ref, B_ref = 4.031e5, 4e7, 1e-9
    out, t = [], 0.0
    for q in range(nreq):
        a, b, c, d, e, f, h = u[2 * shapes + 7 * q:2 * shapes + 7 * q + 7]
        t += -math.log(1.0 - a) / rate
        na, nr = grid[min(int(b * shapes), shapes - 1)]
        up = (float((2.0 + 4.0 * c) * U_ref), UPSTREAM[1], float((0.5 + 2.5 * d) * n_ref), UPSTREAM[3], 0.0, 0.0,
              0.0, 0.0, float((-0.4 + 0.8 * e) * B_ref))
        case = ShellCase(na=na, nr=nr, upstream=up, na_fraction=float(1e-4 + (1e-2 - 1e-4) * f), **_res(resistive))
        steps = steps_min + min(int(h * (steps_max - steps_min + 1)), steps_max - steps_min)
        out.append((t, case, steps))
    return out
