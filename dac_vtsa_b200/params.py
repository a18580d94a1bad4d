"""Per-step constants for the device kernels (the C struct dv_step_params of include/dacvtsa.h).

Everything TVSAModel.__init__ derives on the host in the reference (core/residual.py:41-123 and
the physics-module constructors it calls) is computed here with the same expressions and handed
to the kernels in one struct, plus three small per-step arrays (feed flux and nominal flux over
(Nr, Nth), jacket coverage over (Nth, Nz)).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import host
from ._lib import (BEDCOND, COADS, DISP, DV_MAX_NR, END_KIND, LIMITER, WALLHTC, DvStepParams)


def _set(arr, values):
    for i, v in enumerate(values):
        arr[i] = float(v)


def build_params(cfg, grid, props, step, P_start, T_jacket_prev=None):
    """Return (DvStepParams, feed_flux (Nr,Nth), n_nom (Nr,Nth), coverage (Nth,Nz), extras dict)."""
    if not cfg.components.water:
        raise NotImplementedError("components.water = false: the reference's own dry model raises at "
                                  "physics/isotherms.py:118; only the humid (CO2/H2O/N2) model is supported")
    if grid.Nr > DV_MAX_NR:
        raise NotImplementedError(f"Nr > {DV_MAX_NR} is not supported by the kernels")
    g = grid
    p = DvStepParams()
    p.Nr, p.Nth, p.Nz = g.Nr, g.Nth, g.Nz
    wall = cfg.wall
    p.wall_on = int(bool(wall.enabled))
    p.dz, p.dth, p.half_dr_outer = g.dz, g.dth, g.half_dr_outer
    p.A_wall_in, p.A_wall_out = g.A_wall_in, g.A_wall_out
    p.wall_C = wall.density * wall.cp * g.V_wall                             # physics/energy.py:93
    p.wall_kz = wall.conductivity * g.A_wall_axial / g.dz                    # physics/energy.py:101
    p.wall_kt = wall.conductivity * g.wall_thickness * g.dz / (g.R_wall_mid * g.dth)   # :106
    _set(p.Az, g.Az[:, 0])
    _set(p.V, g.V[:, 0, 0])
    _set(p.Ath, g.Ath[:, 0, 0])
    _set(p.arc, g.arc[:, 0, 0])
    if g.Nr > 1:
        _set(p.Ar, g.Ar[:, 0, 0])
        _set(p.drc, g.drc[:, 0, 0])
    so, tr, th = cfg.sorbent, cfg.transport, cfg.thermo
    p.eps_b, p.eps_t, p.rho_b = so.bed_voidage, so.total_voidage, cfg.derived.bulk_density
    p.cp_s, p.dp, p.T_ref = so.cp_solid, so.particle_diameter, th.T_ref
    _set(p.cpg, props.cp)
    _set(p.cpa, [th.cp_ads_co2, th.cp_ads_h2o])
    _set(p.dH, [th.dH_ads_co2, th.dH_ads_h2o])
    _set(p.M, props.M)
    for s, terms in enumerate(props.mu_terms()):
        p.mu_nt[s] = len(terms)
        for t, (w, a, b) in enumerate(terms):
            p.mu_w[s][t], p.mu_D[s][t], p.mu_E[s][t] = w, a, b
    for s, terms in enumerate(props.k_terms()):
        p.k_nt[s] = len(terms)
        for t, (w, k0, e) in enumerate(terms):
            p.k_w[s][t], p.k_0[s][t], p.k_n[s][t] = w, k0, e
    for i in range(3):
        for j in range(3):
            p.mass_q[i][j] = props.mass_q[i, j]
            p.wilke_den[i][j] = props.wilke_den[i, j]
    for q, (a, b) in enumerate((("CO2", "AIR"), ("CO2", "H2O"))):
        Ma, Mb = host.MOLAR_MASS_G[a], host.MOLAR_MASS_G[b]
        Mab = 2.0 / (1.0 / Ma + 1.0 / Mb)
        p.fuller_sqrtM[q] = float(np.sqrt(Mab))
        p.fuller_s[q] = host.DIFF_VOLUME[a] ** (1 / 3) + host.DIFF_VOLUME[b] ** (1 / 3)
    iso = cfg.isotherm
    c2, hw, co = iso.co2, iso.h2o, iso.coadsorption
    p.co2_q_inf0, p.co2_chi, p.co2_b0, p.co2_dH0 = c2.q_inf0, c2.chi, c2.b0, c2.dH0
    p.co2_tau0, p.co2_alpha, p.co2_T0, p.p_reg = c2.tau0, c2.alpha, c2.T0, c2.p_regularization
    p.h2o_q_m, p.h2o_C, p.h2o_D, p.h2o_F, p.h2o_G = hw.q_m, hw.C, hw.D, hw.F, hw.G
    p.h2o_E10_slope, p.h2o_E10_intercept, p.rh_cap = hw.E10_slope, hw.E10_intercept, hw.rh_cap
    wd, me, sb = co.wadst, co.mechanistic, co.stampi_bombelli
    p.wadst_b0, p.wadst_q_inf0, p.wadst_tau0, p.wadst_chi = wd.b0_wet, wd.q_inf0_wet, wd.tau0_wet, wd.chi_wet
    p.wadst_alpha, p.wadst_dH, p.wadst_A = wd.alpha_wet, wd.dH_wet, wd.A
    p.mech_f_blocked_max, p.mech_k, p.mech_phi_dry = me.f_blocked_max, me.k, me.phi_dry
    p.mech_A, p.mech_dH_wet, p.mech_n = me.A, me.dH_wet, me.n
    p.sb_gamma, p.sb_beta = sb.gamma, sb.beta
    p.coads = COADS[co.model]
    p.basis_state = int(co.water_loading_basis == "state")
    kin = cfg.kinetics
    _set(p.k_ldf, [kin.k_ldf_co2, kin.k_ldf_h2o])
    _set(p.Ea, [kin.Ea_co2, kin.Ea_h2o])
    p.T_ref_kin = kin.T_ref
    p.ea_zero = int(kin.Ea_co2 == 0.0 and kin.Ea_h2o == 0.0)
    eps = so.bed_voidage
    p.ka = tr.ergun_A * (1.0 - eps) ** 2 / (eps ** 3 * so.particle_diameter ** 2)    # physics/pressure.py:32-34
    p.kb = tr.ergun_B * (1.0 - eps) / (eps ** 3 * so.particle_diameter)
    p.disp_model = DISP[tr.dispersion_model]
    p.g1, p.g2, p.er_beta, p.Pe_T = tr.er_gamma1, tr.er_gamma2, tr.er_beta, tr.Pe_mass_radial_inf
    p.bed_model = BEDCOND[tr.bed_conductivity_model]
    p.lam_const, p.lam_s = tr.bed_conductivity_constant, so.particle_conductivity
    p.zs_B = tr.zs_shape_factor * ((1.0 - eps) / eps) ** (10.0 / 9.0)              # heat_transfer.py:25
    p.zs_s = float(np.sqrt(1.0 - eps))
    p.Pe_r, p.Pe_z = tr.Pe_heat_radial_inf, tr.Pe_heat_axial_inf
    p.htc_model = WALLHTC[tr.wall_htc_model]
    p.alpha_const = tr.wall_htc_constant
    p.N_ratio = 2.0 * cfg.geometry.bed_radius / so.particle_diameter
    p.lumped = int(tr.heat_transfer_mode == "lumped")
    p.U_lumped = tr.lumped_U
    p.limiter = LIMITER[cfg.solver.limiter]
    # ---- ends (valves/valve_logic.py:71-109), feed (:112-148), nominal flux (core/residual.py:75-85)
    conds = host.end_conditions(cfg, step, list(props.species), props)
    for e, end in enumerate(("top", "bottom")):
        c = conds[end]
        E = p.ends[e]
        E.kind = END_KIND[c.kind]
        E.valve = -1 if c.valve is None else int(c.valve[1]) - 1
        E.check_valve, E.is_vacuum, E.is_feed = int(c.check_valve), int(c.is_vacuum), int(c.is_feed)
        E.P_target, E.T_ext, E.speed = c.P_target, c.T_ext, c.speed
        E.P_start = float(P_start[end])
        if c.y_ext is not None:
            _set(E.y_ext, c.y_ext)
    p.tau_valve = cfg.operation.valve_time_constant
    prof = host.feed_profile(cfg, g)
    feed_flux = host.feed_molar_flux(cfg) * prof * g.Az
    has_feed = any(c.kind == "feed" for c in conds.values())
    p.u_nom = cfg.feed.velocity if has_feed else 0.0
    n_nom = (host.feed_molar_flux(cfg) * prof) if has_feed else np.zeros((g.Nr, g.Nth))
    # ---- jacket / exchanger / energy accounting (core/residual.py:87-108)
    jk = step["jacket"]
    p.jacket_on = int(jk["mode"] == "temperature")
    T_set = jk.get("T", cfg.ambient.T)
    p.T_jac_set = T_set
    p.T_jac_prev = T_set if T_jacket_prev is None else T_jacket_prev
    p.jac_tau, p.h_jac, p.h_amb = cfg.jacket.ramp_time, cfg.jacket.h_jacket, cfg.jacket.h_ambient
    p.T_amb, p.P_amb = cfg.ambient.T, cfg.ambient.P
    p.hx_on = int(bool(cfg.internal_hx.enabled) and p.jacket_on)
    p.hA_v = cfg.internal_hx.hA_per_volume
    en = cfg.energy
    p.gam, p.eta_vac, p.eta_bl = en.gamma_gas, en.eta_vacuum, en.eta_blower
    p.vac_krishnamurthy = int(en.vacuum_efficiency_model == "krishnamurthy")
    p.pump_water = int(bool(en.pump_handles_water))
    # ---- solver constants (core/residual.py:135-144, core/jacobian.py:39-48)
    s = cfg.solver
    rho_cp = p.rho_b * so.cp_solid
    _set(p.atol, [s.atol_c_co2, s.atol_c_h2o, s.atol_c_inert, s.atol_q, s.atol_q, rho_cp * s.atol_T, s.atol_T])
    _set(p.typ, [1e-3, 1e-2, 1.0, 1e-3, 1e-3, rho_cp, 1.0])
    cov = g.coverage_fraction(cfg.jacket.theta_coverage_deg, cfg.jacket.z_coverage)
    extras = {"conds": conds, "has_feed": has_feed, "T_jac_set": T_set}
    return (p, np.ascontiguousarray(feed_flux, dtype=np.float64), np.ascontiguousarray(n_nom, dtype=np.float64),
            np.ascontiguousarray(cov, dtype=np.float64), extras)


def params_bytes(p: DvStepParams) -> bytes:
    return C.string_at(C.addressof(p), C.sizeof(p))
