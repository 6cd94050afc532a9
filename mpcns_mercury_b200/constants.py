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
                        res_max_it: int = 500) -> MhdConstants:
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
    return c
