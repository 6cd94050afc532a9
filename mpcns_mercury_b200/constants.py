"""Physical constants of the step, derived as the reference's
calc_physical_constant does (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48),
in the same arithmetic order, from the reference's production parameter values
(Z4_Mercury/9999setup/0_General_Setting.txt: constant list, mole masses;
1_Initial_condition.txt: REF list)."""
from __future__ import annotations

from .capi import MhdConstants


def reference_constants(cfl: float = 0.4, ambipolar: bool = True, gamma: float = 1.6667, NA: float = 6.02e23,
                        R_uni: float = 8.314, mu_mag: float = 1.256637061e-6, q_e: float = 1.602e-19,
                        U_ref: float = 4.031e5, T_ref: float = 1.7407e5, n_ref: float = 4e7,
                        M_ref: float = 0.001, B_ref: float = 1e-9, L_ref: float = 2.44e6,
                        M_H: float = 0.001, M_Na: float = 0.023, arti_eta_max: float = 0.0,
                        arti_J_start: float = 800.0, arti_J_on: float = 3000.0,
                        local_arti: bool = False, resistive: bool = False, res_rtol: float = 1e-13,
                        res_max_it: int = 500, res_direct_iters: int = 0, initial=None) -> MhdConstants:
    if initial is None:
        initial = DEFAULT_INITIAL
    c = MhdConstants()
    c.gamma = gamma
    c.q_e = q_e
    c.k_Boltz = R_uni / NA
    c.mu0 = mu_mag
    c.U_ref = U_ref
    c.L_ref = L_ref
    c.B_ref = B_ref
    c.T_ref = T_ref
    c.n_ref = n_ref
    c.M_ref = M_ref
    c.rho_ref = M_ref * n_ref / NA
    c.M_H = M_H
    c.M_Na = M_Na
    c.m_Na = M_Na / NA
    c.state_coeff_H = (R_uni * T_ref) / (M_H * U_ref * U_ref)
    c.state_coeff_Na = (R_uni * T_ref) / (M_Na * U_ref * U_ref)
    c.CFL = cfl
    c.hall_coef = B_ref * M_ref / (U_ref * q_e * L_ref * mu_mag * c.rho_ref * NA)
    c.momentum_induce_coeff = (q_e * L_ref * B_ref * n_ref) / (c.rho_ref * U_ref)
    c.momentum_hall_coeff = (B_ref * B_ref) / (mu_mag * c.rho_ref * U_ref * U_ref)
    c.inver_MA2 = B_ref * B_ref / (U_ref * U_ref * mu_mag * c.rho_ref)
    c.ne_hall_floor = 0.01
    c.ambipolar = 1 if ambipolar else 0
    # artificial resistivity (arti_eta_max, J_range_start, J_range_on,
    # is_local_artificial_resistivity of the MHD control file)
    c.arti_eta_max = arti_eta_max
    c.arti_J_start = arti_J_start
    c.arti_J_on = arti_J_on
    c.local_arti = 1 if local_arti else 0
    # implicit resistive substep (is_Mercury_resistance; the per-edge eta is a field)
    c.resistive = 1 if resistive else 0
    c.res_rtol = res_rtol
    c.res_max_it = res_max_it
    # mixed precision: FP64 CG while the last substep took at most this many
    # iterations (0: 20), iterative refinement after a longer one (negative: always)
    c.res_direct_iters = res_direct_iters
    set_boundary(c, gamma=gamma, NA=NA, R_uni=R_uni, U_ref=U_ref, T_ref=T_ref, n_ref=n_ref, M_ref=M_ref,
                 B_ref=B_ref, initial=initial)
    return c


# The reference's default INITIAL list (Z4_Mercury/9999setup/1_Initial_condition.txt):
# U, T, n, Molecular_mass, c_y, c_z, Bx, By, Bz (SI)
DEFAULT_INITIAL = (4.03112887e5, 1.7407e5, 4e7, 0.001, 1.240347346e-1, 0.0, 0.0, 0.0, 0.0)


def set_boundary(c, gamma=1.6667, NA=6.02e23, R_uni=8.314, U_ref=4.031e5, T_ref=1.7407e5, n_ref=4e7,
                 M_ref=0.001, B_ref=1e-9, initial=DEFAULT_INITIAL, rho_small=1e-6):
    """The values of the physical boundary operations (mhd_constants.bc):
    the upstream states of both species, the IMF and the upstream velocity as
    BuildMercuryBackgroundState derives them from the INITIAL and REF lists
    (Z4_Mercury/include/0_BackgroundState.h:18-85), zero, and the Na+ floor
    state of the solid wall (Z4_Mercury/src/boundary/Boundary_Condition_Fluid.cpp:59-170)."""
    import math

    U, T, n, Mm, c_y, c_z, Bx, By, Bz = initial
    k_B = R_uni / NA
    rho_ref = M_ref / NA * n_ref
    rho0 = (n / n_ref) * (Mm / M_ref)
    c_x = -math.sqrt(1.0 - c_y * c_y - c_z * c_z)
    u0, v0, w0 = c_x * U / U_ref, c_y * U / U_ref, c_z * U / U_ref
    p0 = n * k_B * T / (rho_ref * U_ref * U_ref)
    qinf = [rho0, rho0 * u0, rho0 * v0, rho0 * w0, 0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 / (gamma - 1.0)]
    pN = p0 * rho_small / 23.0
    rhoN = rho_small * rho0
    qinfs = [rhoN, 0.0, 0.0, 0.0, pN / (gamma - 1.0) + 0.5 * rhoN * (0.0 * 0.0 + 0.0 * 0.0 + 0.0 * 0.0)]
    vals = qinf + qinfs + [Bx / B_ref, By / B_ref, Bz / B_ref, 0.0, 1.0e-12, 1.0e-12 / (gamma - 1.0), u0, v0, w0]
    for q, v in enumerate(vals):
        c.bc[q] = v
    return c
