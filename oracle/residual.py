"""Oracle: semi-discrete right-hand side f(t, y) of one cycle step (numpy restatement).

Follows core/residual.py:40-482 of the reference and the closures it calls:
physics/energy.py (Thermo 31-78, Wall 86-113, enthalpy_flux 81-83),
physics/isotherms.py (toth 50-56, gab 59-67, smooth_cap 70-80, equilibrium 108-153),
physics/kinetics.py:29-39, physics/pressure.py:36-56, physics/dispersion.py:32-47,
physics/heat_transfer.py:23-76, physics/mass.py:23-74, numerics/stencils.py:45-101,
boundaries/conditions.py:43-160, properties/ideal_gas_backend.py:48-137, utils/diffusion.py:19-26.

Layout of y: [c_1..c_ng | q_1..q_na | e | Tw], each block C-ordered over (Nr, Nth, Nz)
(walls: (Nth, Nz)) -- core/residual.py:110-118.
"""
from __future__ import annotations

import numpy as np

from dac_vtsa_b200.host import (R_GAS, end_conditions, feed_molar_flux, feed_profile,
                                humid_air_composition)

U_SMOOTH = 1e-4            # numerics/stencils.py:45
VALVE_DP = 0.2             # boundaries/conditions.py:43


def _nxt(a):               # periodic theta neighbour j+1 (axis -2), physics/mass.py:23-26
    return np.roll(a, -1, axis=-2)


def _prv(a):               # periodic theta neighbour j-1, physics/mass.py:29-31
    return np.roll(a, 1, axis=-2)


def _upw(u):               # numerics/stencils.py:48-56
    return 0.5 * (1.0 + np.tanh(u / U_SMOOTH))


def _softplus(x, width):   # boundaries/conditions.py:46-49
    return width * np.logaddexp(0.0, x / width)


def _ergun_u(g, a, b):     # physics/pressure.py:40-42
    return -2.0 * g / (a + np.sqrt(a * a + 4.0 * b * np.abs(g)))


def _slope(dm, dp, limiter):   # numerics/stencils.py:59-76
    if limiter == "upwind":
        return np.zeros_like(dm)
    prod = dm * dp
    if limiter == "van_albada":
        return prod * (dm + dp) / (dm * dm + dp * dp + 1e-300)
    if limiter == "van_albada_tvd":
        return np.where(prod > 0.0, prod * (dm + dp) / (dm * dm + dp * dp + 1e-300), 0.0)
    if limiter == "van_leer":
        return np.where(prod > 0.0, 2.0 * prod / (dm + dp + 1e-300), 0.0)
    if limiter == "minmod":
        return np.where(prod > 0.0, np.sign(dm) * np.minimum(np.abs(dm), np.abs(dp)), 0.0)
    raise ValueError(limiter)


def _muscl_z(phi, u, limiter):  # numerics/stencils.py:79-95 (boundary-adjacent cells: zero slope)
    w = _upw(u)
    nz = phi.shape[-1]
    if nz < 3 or limiter == "upwind":
        return w * phi[..., :-1] + (1.0 - w) * phi[..., 1:]
    d = phi[..., 1:] - phi[..., :-1]
    s = np.zeros_like(phi)
    s[..., 1:-1] = _slope(d[..., :-1], d[..., 1:], limiter)
    return w * (phi[..., :-1] + 0.5 * s[..., :-1]) + (1.0 - w) * (phi[..., 1:] - 0.5 * s[..., 1:])


def _wsum(w, a):            # physics/energy.py:70-75
    out = w[0] * a[0]
    for k in range(1, len(w)):
        out = out + w[k] * a[k]
    return out


def _toth(p, T, q_inf0, chi, b0, dH0, tau0, alpha, T0):   # physics/isotherms.py:50-56
    p = np.maximum(p, 0.0)
    qinf = q_inf0 * np.exp(chi * (1.0 - T / T0))
    b = b0 * np.exp(-dH0 / (R_GAS * T))
    tau = tau0 + alpha * (1.0 - T0 / T)
    bp = b * p
    return qinf * bp / (1.0 + bp ** tau) ** (1.0 / tau)


def _gab(x, T, q_m, C, D, F, G, E10_slope, E10_intercept):   # physics/isotherms.py:59-67
    E1 = C - np.exp(D * T)
    E29 = F + G * T
    E10 = E10_slope * T + E10_intercept
    RT = R_GAS * T
    c = np.exp((E1 - E10) / RT)
    k = np.exp((E29 - E10) / RT)
    kx = k * x
    return q_m * c * kx / ((1.0 - kx) * (1.0 + (c - 1.0) * kx))


def _smooth_cap(x, cap, width=0.02):   # physics/isotherms.py:70-80
    x = np.maximum(x, -0.2)
    lo = cap - width
    over = np.maximum(x - lo, 0.0)
    blend = lo + over - over ** 2 / (4.0 * width)
    return np.where(x <= lo, x, np.where(over >= 2.0 * width, cap, blend))


class OracleModel:
    """Numpy twin of the reference TVSAModel for one cycle step (core/residual.py:40-123)."""

    def __init__(self, cfg, grid, props, step, state0, T_jacket_prev=None):
        g = grid
        self.cfg, self.grid, self.props, self.step = cfg, grid, props, step
        self.species = list(props.species)
        self.ng = len(self.species)
        self.water = bool(cfg.components.water)
        self.adsorbed = ["CO2", "H2O"] if self.water else ["CO2"]
        self.na = len(self.adsorbed)
        self.i_co2 = self.species.index("CO2")
        self.i_h2o = self.species.index("H2O") if self.water else None
        self.ads_to_gas = [self.species.index(s) for s in self.adsorbed]
        so, tr, th = cfg.sorbent, cfg.transport, cfg.thermo
        self.eps_b, self.eps_t, self.rho_b = so.bed_voidage, so.total_voidage, cfg.derived.bulk_density
        self.cp_s, self.dp = so.cp_solid, so.particle_diameter
        self.cpg = np.asarray(props.cp, dtype=float)
        self.cpa = np.array([th.cp_ads_co2, th.cp_ads_h2o] if self.water else [th.cp_ads_co2])
        self.dH = np.array([th.dH_ads_co2, th.dH_ads_h2o] if self.water else [th.dH_ads_co2])
        self.T_ref = th.T_ref
        self.limiter = cfg.solver.limiter
        self.lumped = tr.heat_transfer_mode == "lumped"
        eps = self.eps_b
        self.ka = tr.ergun_A * (1.0 - eps) ** 2 / (eps ** 3 * self.dp ** 2)      # physics/pressure.py:32-34
        self.kb = tr.ergun_B * (1.0 - eps) / (eps ** 3 * self.dp)
        self.conds = end_conditions(cfg, step, self.species, props)
        self.tau_valve = cfg.operation.valve_time_constant
        P0 = state0.P
        self.P_start = {"top": float(np.mean(P0[:, :, 0])), "bottom": float(np.mean(P0[:, :, -1]))}
        prof = feed_profile(cfg, g)
        self.feed_flux = feed_molar_flux(cfg) * prof * g.Az
        has_feed = any(c.kind == "feed" for c in self.conds.values())
        self.u_nom = cfg.feed.velocity if has_feed else 0.0
        self.N_nom = (feed_molar_flux(cfg) * prof)[..., None] if has_feed else np.zeros(g.Az.shape + (1,))
        jk = step["jacket"]
        self.jacket_on = jk["mode"] == "temperature"
        self.T_jac_set = jk.get("T", cfg.ambient.T)
        self.T_jac_prev = self.T_jac_set if T_jacket_prev is None else T_jacket_prev
        self.jac_tau, self.h_jac, self.h_amb = cfg.jacket.ramp_time, cfg.jacket.h_jacket, cfg.jacket.h_ambient
        self.T_amb, self.P_amb = cfg.ambient.T, cfg.ambient.P
        self.cov = g.coverage_fraction(cfg.jacket.theta_coverage_deg, cfg.jacket.z_coverage)
        self.hx_on = bool(cfg.internal_hx.enabled) and self.jacket_on
        self.hA_v, self.U_lumped = cfg.internal_hx.hA_per_volume, tr.lumped_U
        w = cfg.wall
        self.wall_on = bool(w.enabled)
        self.wall_C = w.density * w.cp * g.V_wall
        self.wall_lam = w.conductivity
        en = cfg.energy
        self.gam, self.eta_vac, self.vac_model = en.gamma_gas, en.eta_vacuum, en.vacuum_efficiency_model
        self.eta_bl, self.pump_water = en.eta_blower, bool(en.pump_handles_water)
        n = g.ncell
        self.n_c, self.n_q = self.ng * n, self.na * n
        self.off_q, self.off_e = self.n_c, self.n_c + self.n_q
        self.off_w = self.off_e + n
        self.n_w = g.Nth * g.Nz if self.wall_on else 0
        self.n_core = self.off_w + self.n_w
        names = []
        for v in ("V1", "V2", "V3"):
            names += [f"n_in_{v}_{s}" for s in self.species] + [f"n_out_{v}_{s}" for s in self.species]
            names += [f"H_in_{v}", f"H_out_{v}", f"W_pump_{v}", f"W_fan_{v}"]
        names += ["Q_jac_pos", "Q_jac_neg", "Q_amb", "Q_wb", "Q_hx_pos", "Q_hx_neg"]
        self.acc_names = names
        self.n_acc = len(names)
        self.acc_index = {nm: i for i, nm in enumerate(names)}
        s = cfg.solver
        tol_c = {"CO2": s.atol_c_co2, "H2O": s.atol_c_h2o, "N2": s.atol_c_inert}
        parts = [np.full(n, tol_c[sp]) for sp in self.species] + [np.full(n, s.atol_q)] * self.na
        parts.append(np.full(n, self.rho_b * self.cp_s * s.atol_T))
        if self.n_w:
            parts.append(np.full(self.n_w, s.atol_T))
        self.atol = np.concatenate(parts)                      # core/residual.py:135-144
        self.nfev = 0

    # ---------------------------------------------------------------- thermo (physics/energy.py:39-52)
    def _AB(self, c, q):
        Cg = c[0] + c[1] if len(c) == 2 else c[0] + c[1] + c[2]
        A = self.eps_t * _wsum(self.cpg, c) + self.rho_b * (self.cp_s + _wsum(self.cpa, q))
        return A, self.eps_t * R_GAS * Cg, self.rho_b * _wsum(self.dH, q)

    def temperature(self, e, c, q):
        A, B, Hq = self._AB(c, q)
        return (e - Hq + A * self.T_ref) / (A - B)

    def energy(self, T, c, q):
        A, B, Hq = self._AB(c, q)
        return A * (T - self.T_ref) - B * T + Hq

    def pack(self, st):
        parts = [st.c.ravel(), st.q.ravel(), self.energy(st.T, st.c, st.q).ravel()]
        if self.n_w:
            parts.append(st.Tw.ravel())
        return np.concatenate(parts)

    def unpack(self, y):
        g = self.grid
        c = y[:self.n_c].reshape((self.ng,) + g.shape)
        q = y[self.off_q:self.off_e].reshape((self.na,) + g.shape)
        e = y[self.off_e:self.off_w].reshape(g.shape)
        Tw = y[self.off_w:self.n_core].reshape(g.wall_shape) if self.n_w else None
        return c, q, e, Tw

    def T_jacket(self, t):                          # core/residual.py:199-202
        if self.jac_tau <= 0:
            return self.T_jac_set
        return self.T_jac_set + (self.T_jac_prev - self.T_jac_set) * np.exp(-t / self.jac_tau)

    # ---------------------------------------------------------------- gas properties
    def _mu_k(self, T, y):      # properties/ideal_gas_backend.py:94-113, 148-166
        p = self.props
        mu = np.stack([sum(f * (a * T + b) for f, a, b in terms) if len(terms) > 1 else terms[0][1] * T + terms[0][2]
                       for terms in p.mu_terms()])
        kk = np.stack([sum(f * k0 * (T / 300.0) ** e for f, k0, e in terms) if len(terms) > 1
                       else terms[0][1] * (T / 300.0) ** terms[0][2] for terms in p.k_terms()])
        sq = np.sqrt(mu)
        mu_m = 0.0
        k_m = 0.0
        for i in range(self.ng):
            den = 0.0
            for j in range(self.ng):
                if i == j:
                    den = den + y[j]
                else:
                    den = den + y[j] * ((1.0 + (sq[i] / sq[j]) * p.mass_q[i, j]) ** 2 / p.wilke_den[i, j])
            den = np.maximum(den, 1e-30)
            mu_m = mu_m + y[i] * mu[i] / den
            k_m = k_m + y[i] * kk[i] / den
        return mu_m, k_m

    def _fuller(self, T, P, a, b):   # utils/diffusion.py:19-26
        from dac_vtsa_b200.host import DIFF_VOLUME, MOLAR_MASS_G
        Ma, Mb = MOLAR_MASS_G[a], MOLAR_MASS_G[b]
        Mab = 2.0 / (1.0 / Ma + 1.0 / Mb)
        s = DIFF_VOLUME[a] ** (1 / 3) + DIFF_VOLUME[b] ** (1 / 3)
        P = np.maximum(P, 1.0)
        return 1.43e-7 * T ** 1.75 / ((P / 1e5) * np.sqrt(Mab) * s * s)

    def _Dm(self, T, P, y):     # properties/ideal_gas_backend.py:127-137
        D_ca = self._fuller(T, P, "CO2", "AIR")
        yi = y[self.species.index("N2")]
        if self.i_h2o is None:
            return D_ca
        D_cw = self._fuller(T, P, "CO2", "H2O")
        yw = y[self.i_h2o]
        return (yi + yw + 1e-9) / (yi / D_ca + yw / D_cw + 1e-9 / D_ca)

    def _stagnant(self, lam_g):  # physics/heat_transfer.py:23-31, 51-56
        tr = self.cfg.transport
        if tr.bed_conductivity_model == "constant":
            return tr.bed_conductivity_constant * np.ones_like(lam_g)
        lam_s, eps = self.cfg.sorbent.particle_conductivity, self.eps_b
        if tr.bed_conductivity_model == "parallel":
            return eps * lam_g + (1.0 - eps) * lam_s
        kap = lam_s / lam_g
        B = tr.zs_shape_factor * ((1.0 - eps) / eps) ** (10.0 / 9.0)
        s = np.sqrt(1.0 - eps)
        one_m = 1.0 - B / kap
        kc = (2.0 / one_m) * ((1.0 - 1.0 / kap) * B / one_m ** 2 * np.log(kap / B)
                              - 0.5 * (B + 1.0) - (B - 1.0) / one_m)
        return lam_g * (1.0 - s + s * kc)

    # ---------------------------------------------------------------- isotherms (physics/isotherms.py:98-153)
    def _iso(self):
        return self.cfg.isotherm

    def q_h2o(self, p_w, T, p_sat):
        h = self._iso().h2o
        x = _smooth_cap(p_w / p_sat, h.rh_cap)
        return _gab(x, T, h.q_m, h.C, h.D, h.F, h.G, h.E10_slope, h.E10_intercept)

    def _co2_pars(self):
        c = self._iso().co2
        return dict(q_inf0=c.q_inf0, chi=c.chi, b0=c.b0, dH0=c.dH0, tau0=c.tau0, alpha=c.alpha, T0=c.T0)

    def q_co2_dry(self, p, T):
        return _toth(p, T, **self._co2_pars())

    def q_co2(self, p, T, qw):
        iso = self._iso()
        pp = np.maximum(p, 0.0)
        model = iso.coadsorption.model if self.water else "none"
        co = self._co2_pars()
        if model == "none":
            raw = _toth(pp, T, **co)
        else:
            qw = np.maximum(qw, 1e-12)
            if model == "wadst":
                wd = iso.coadsorption.wadst
                w = np.exp(-wd.A / qw)
                q_wet = _toth(pp, T, wd.q_inf0_wet, wd.chi_wet, wd.b0_wet, wd.dH_wet, wd.tau0_wet,
                              wd.alpha_wet, co["T0"])
                raw = (1.0 - w) * _toth(pp, T, **co) + w * q_wet
            elif model == "mechanistic":
                m = iso.coadsorption.mechanistic
                w = np.exp(-m.A / qw)
                f_bl = m.f_blocked_max * (1.0 - np.exp(-(m.k * qw) ** m.n))
                phi = m.phi_dry + ((1.0 - f_bl) - m.phi_dry) * w
                pars = dict(co)
                pars["dH0"] = (1.0 - w) * co["dH0"] + w * m.dH_wet
                raw = (phi / m.phi_dry) * _toth(pp, T, **pars)
            elif model == "stampi_bombelli":
                sb = iso.coadsorption.stampi_bombelli
                pars = dict(co)
                pars["q_inf0"] = co["q_inf0"] / (1.0 - sb.gamma * qw)
                pars["b0"] = co["b0"] * (1.0 + sb.beta * qw)
                raw = _toth(pp, T, **pars)
            else:
                raise ValueError(model)
        return raw * (pp / (pp + iso.co2.p_regularization))

    # ---------------------------------------------------------------- boundary faces
    def _end(self, cond, t, P_start, c, T, P, mu, rho, Az, half_dz):   # boundaries/conditions.py:75-160
        cpg, Tr = self.cpg, self.T_ref
        if cond.kind == "closed":
            z = np.zeros_like(T)
            return {"F_in": np.zeros_like(c), "H_in": z, "u_out": z.copy(), "P_face": P.copy()}
        a, b = self.ka * mu, self.kb * rho
        yx = None if cond.y_ext is None else cond.y_ext.reshape(-1, 1, 1) if c.ndim == 3 else cond.y_ext.reshape(-1, 1)
        C_cell = np.maximum(c.sum(axis=0), 1e-12)
        if cond.kind == "feed":
            F_in = self.feed_flux[None] * yx
            H_in = np.tensordot(cpg, F_in, axes=(0, 0)) * (cond.T_ext - Tr)
            u_in = self.feed_flux / (Az * C_cell)
            return {"F_in": F_in, "H_in": H_in, "u_out": -u_in, "P_face": P + (a * u_in + b * u_in * u_in) * half_dz}
        if cond.kind == "pump":
            dp = P - cond.P_target
            y_cell = c / C_cell
            if cond.check_valve:
                dp = _softplus(dp, 1.0)
                w_out = np.ones_like(dp)
            else:
                w_out = 0.5 * (1.0 + np.tanh(dp / VALVE_DP))
            N_out = cond.speed * dp / (R_GAS * T)
            F_out = (N_out * Az)[None] * (w_out[None] * y_cell + (1.0 - w_out[None]) * yx)
            T_up = w_out * T + (1.0 - w_out) * cond.T_ext
            H_out = np.tensordot(cpg, F_out, axes=(0, 0)) * (T_up - Tr)
            u_out = N_out / C_cell
            return {"F_in": -F_out, "H_in": -H_out, "u_out": u_out,
                    "P_face": P - (a * u_out + b * np.abs(u_out) * u_out) * half_dz}
        if cond.kind == "valve":
            tau = self.tau_valve
            P_res = (cond.P_target + (P_start - cond.P_target) * np.exp(-t / tau)) if tau > 0 else cond.P_target
            dp = P_res - P
            N_in = cond.speed * _softplus(dp, VALVE_DP) / (R_GAS * cond.T_ext)
            N_out = cond.speed * _softplus(-dp, VALVE_DP) / (R_GAS * T)
            F_inp = (N_in * Az)[None] * yx
            F_outp = (N_out * Az)[None] * (c / C_cell)
            H_inp = np.tensordot(cpg, F_inp, axes=(0, 0)) * (cond.T_ext - Tr)
            H_outp = np.tensordot(cpg, F_outp, axes=(0, 0)) * (T - Tr)
            u_out = -(N_in - N_out) / C_cell
            return {"F_in": F_inp - F_outp, "H_in": H_inp - H_outp, "u_out": u_out,
                    "P_face": P - (a * u_out + b * np.abs(u_out) * u_out) * half_dz,
                    "F_inpart": F_inp, "F_outpart": F_outp, "H_inpart": H_inp, "H_outpart": H_outp}
        tau = self.tau_valve
        P_face = (cond.P_target + (P_start - cond.P_target) * np.exp(-t / tau)) * np.ones_like(P)
        u_out = _ergun_u((P_face - P) / half_dz, a, b)
        if cond.check_valve:
            u_out = 0.5 * (u_out + np.sqrt(u_out * u_out + 1e-14)) - 0.5e-7
        c_ext = yx * P_face[None] / (R_GAS * cond.T_ext)
        w = _upw(u_out)
        F_out = u_out[None] * Az[None] * (w[None] * c + (1.0 - w[None]) * c_ext)
        T_up = w * T + (1.0 - w) * cond.T_ext
        H_out = np.tensordot(cpg, F_out, axes=(0, 0)) * (T_up - Tr)
        return {"F_in": -F_out, "H_in": -H_out, "u_out": u_out, "P_face": P_face}

    # ---------------------------------------------------------------- RHS (core/residual.py:211-417)
    def rhs(self, t, y, want_acc=True, diag=False):
        self.nfev += 1
        g, cfg = self.grid, self.cfg
        tr = cfg.transport
        c, q, e, Tw = self.unpack(y)
        Ctot = c.sum(axis=0)
        T = self.temperature(e, c, q)
        P = Ctot * R_GAS * T
        Tp = np.clip(T, 150.0, 1500.0)
        Cpos = np.maximum(Ctot, 1e-9)
        yk = c / Cpos
        ycl = np.clip(yk, 0.0, 1.0)
        mu, kg = self._mu_k(Tp, ycl)
        rho = Cpos * _wsum(self.props.M, ycl)
        cpm = _wsum(self.props.cp, ycl)
        Dm = self._Dm(Tp, np.maximum(P, 1.0), ycl)
        lam0 = self._stagnant(kg)
        pk = c * R_GAS * Tp
        psat = self.props.p_sat(Tp)
        if self.water:
            qw_eq = self.q_h2o(pk[self.i_h2o], Tp, psat)
            basis = q[1] if cfg.isotherm.coadsorption.water_loading_basis == "state" else qw_eq
            qstar = np.stack([self.q_co2(pk[self.i_co2], Tp, basis), qw_eq])
        else:
            qstar = self.q_co2(pk[self.i_co2], Tp, None)[None]
        kin = cfg.kinetics
        kr = np.array([kin.k_ldf_co2, kin.k_ldf_h2o] if self.water else [kin.k_ldf_co2])
        Ea = np.array([kin.Ea_co2, kin.Ea_h2o] if self.water else [kin.Ea_co2])
        shp = (self.na,) + (1,) * Tp.ndim
        if np.all(Ea == 0.0):
            kk = kr.reshape(shp) * np.ones_like(Tp)
        else:
            kk = kr.reshape(shp) * np.exp(-Ea.reshape(shp) / R_GAS * (1.0 / Tp - 1.0 / kin.T_ref))
        rate = kk * (qstar - q)                                          # physics/kinetics.py:38-39
        # ---- Ergun face velocities
        mu_z = 0.5 * (mu[..., 1:] + mu[..., :-1])
        rho_z = 0.5 * (rho[..., 1:] + rho[..., :-1])
        uz = _ergun_u((P[..., 1:] - P[..., :-1]) / g.dz, self.ka * mu_z, self.kb * rho_z)
        ur = uth = None
        if g.Nr > 1:
            ur = _ergun_u((P[1:] - P[:-1]) / g.drc, self.ka * (0.5 * (mu[1:] + mu[:-1])),
                          self.kb * (0.5 * (rho[1:] + rho[:-1])))
        if g.Nth > 1:
            uth = _ergun_u((_nxt(P) - P) / g.arc, self.ka * (0.5 * (mu + _nxt(mu))), self.kb * (0.5 * (rho + _nxt(rho))))
        bnd = {}
        for end, k in (("top", 0), ("bottom", -1)):
            bnd[end] = self._end(self.conds[end], t, self.P_start[end], c[..., k], T[..., k], P[..., k],
                                 mu[..., k], rho[..., k], g.Az, 0.5 * g.dz)
        # ---- species fluxes (physics/mass.py)
        eb = self.eps_b
        disp = tr
        Cz = 0.5 * (Cpos[..., 1:] + Cpos[..., :-1])
        u_disp = self.N_nom / Cz
        Dz = self._axial_D(0.5 * (Dm[..., 1:] + Dm[..., :-1]), u_disp, rho_z, mu_z)
        Az3 = g.Az[:, :, None]
        Fz_conv = uz * Az3 * _muscl_z(c, uz, self.limiter)
        Jz = -eb * Dz * Cz * (yk[..., 1:] - yk[..., :-1]) / g.dz * Az3
        Fz = np.concatenate([bnd["top"]["F_in"][..., None], Fz_conv + Jz, -bnd["bottom"]["F_in"][..., None]], axis=-1)
        Fr = Ft = Fr_conv = Jr = Ft_conv = Jt = None
        if ur is not None:
            Cr = 0.5 * (Cpos[1:] + Cpos[:-1])
            Dr = disp.er_gamma1 * (0.5 * (Dm[1:] + Dm[:-1])) + self.dp * (abs(self.u_nom) / eb) / disp.Pe_mass_radial_inf
            wr = _upw(ur)
            Fr_conv = ur * g.Ar * (wr * c[:, :-1] + (1.0 - wr) * c[:, 1:])
            Jr = -eb * Dr * Cr * (yk[:, 1:] - yk[:, :-1]) / g.drc * g.Ar
            Fr = Fr_conv + Jr
        if uth is not None:
            Ct = 0.5 * (Cpos + _nxt(Cpos))
            Dt = disp.er_gamma1 * (0.5 * (Dm + _nxt(Dm))) + self.dp * (abs(self.u_nom) / eb) / disp.Pe_mass_radial_inf
            wt = _upw(uth)
            Ft_conv = uth * g.Ath * (wt * c + (1.0 - wt) * _nxt(c))
            Jt = -eb * Dt * Ct * (_nxt(yk) - yk) / g.arc * g.Ath
            Ft = Ft_conv + Jt
        div_c = self._div(Fz, Fr, Ft)
        sink = np.zeros_like(c)
        for j, kgas in enumerate(self.ads_to_gas):
            sink[kgas] = rate[j]
        dcdt = -div_c / (self.eps_t * g.V) - (self.rho_b / self.eps_t) * sink
        # ---- energy fluxes (core/residual.py:300-326)
        cpg, Tr = self.cpg, self.T_ref
        Tz_f = _muscl_z(T, uz, self.limiter)
        lam_z = self._lam(0.5 * (lam0[..., 1:] + lam0[..., :-1]), Cz, 0.5 * (cpm[..., 1:] + cpm[..., :-1]),
                          u_disp, tr.Pe_heat_axial_inf)
        Hz_int = (_wsum(cpg, Fz_conv) * (Tz_f - Tr) + _wsum(cpg, Jz) * (0.5 * (T[..., 1:] + T[..., :-1]) - Tr)
                  - lam_z * (T[..., 1:] - T[..., :-1]) / g.dz * Az3)
        Hz = np.concatenate([bnd["top"]["H_in"][..., None], Hz_int, -bnd["bottom"]["H_in"][..., None]], axis=-1)
        Hr = Ht = None
        if ur is not None:
            wr = _upw(ur)
            lam_r = self._lam(0.5 * (lam0[1:] + lam0[:-1]), Cr, 0.5 * (cpm[1:] + cpm[:-1]), self.u_nom,
                              tr.Pe_heat_radial_inf)
            Hr = (_wsum(cpg, Fr_conv) * ((wr * T[:-1] + (1.0 - wr) * T[1:]) - Tr)
                  + _wsum(cpg, Jr) * (0.5 * (T[1:] + T[:-1]) - Tr) - lam_r * (T[1:] - T[:-1]) / g.drc * g.Ar)
        if uth is not None:
            Tn = _nxt(T)
            wt = _upw(uth)
            lam_t = self._lam(0.5 * (lam0 + _nxt(lam0)), Ct, 0.5 * (cpm + _nxt(cpm)), self.u_nom, tr.Pe_heat_radial_inf)
            Ht = (_wsum(cpg, Ft_conv) * ((wt * T + (1.0 - wt) * Tn) - Tr) + _wsum(cpg, Jt) * (0.5 * (T + Tn) - Tr)
                  - lam_t * (Tn - T) / g.arc * g.Ath)
        div_e = self._div(Hz, Hr, Ht)
        # ---- wall / jacket / exchanger (core/residual.py:328-359)
        To = T[-1]
        lam_out = self._lam(lam0[-1], Cpos[-1], cpm[-1], self.u_nom, tr.Pe_heat_radial_inf)
        if self.lumped:
            R_bed = 1.0 / self.U_lumped
        else:
            aw = self._alpha_w(lam0[-1], kg[-1], rho[-1], mu[-1], cpm[-1] / np.maximum(rho[-1] / Cpos[-1], 1e-6))
            R_bed = 1.0 / aw + g.half_dr_outer / lam_out
        Tj = self.T_jacket(t)
        dTw = None
        if self.wall_on:
            Q_jac = self.cov * self.h_jac * g.A_wall_out * (Tj - Tw) if self.jacket_on else np.zeros_like(Tw)
            Q_amb = (1.0 - self.cov) * self.h_amb * g.A_wall_out * (self.T_amb - Tw)
            Q_wb = g.A_wall_in * (Tw - To) / R_bed
            dTw = (Q_jac + Q_amb - Q_wb + self._wall_cond(Tw)) / self.wall_C
        else:
            if self.jacket_on and self.h_jac > 0:
                R_j = R_bed if self.lumped else R_bed + 1.0 / self.h_jac
                Q_jac = self.cov * g.A_wall_in * (Tj - To) / R_j
            else:
                Q_jac = np.zeros_like(To)
            Q_amb = ((1.0 - self.cov) * g.A_wall_in * (self.T_amb - To) / (R_bed + 1.0 / self.h_amb)
                     if self.h_amb > 0 else np.zeros_like(To))
            Q_wb = Q_jac + Q_amb
        src = np.zeros_like(T)
        src[-1] += Q_wb
        Q_hx = None
        if self.hx_on:
            Q_hx = self.hA_v * g.V * (Tj - T)
            src += Q_hx
        dedt = (-div_e + src) / g.V
        parts = [dcdt.ravel(), rate.ravel(), dedt.ravel()] + ([dTw.ravel()] if dTw is not None else [])
        f = np.concatenate(parts)
        if diag:
            return {"T": T, "P": P, "y": yk, "qstar": qstar, "uz": uz, "ur": ur, "uth": uth, "bnd": bnd,
                    "Q_jac": Q_jac, "Q_wb": Q_wb, "Q_amb": Q_amb, "Q_hx": Q_hx, "R_bed": R_bed}
        if not want_acc:
            return f, None
        return f, self._accumulators(bnd, T, Q_jac, Q_amb, Q_wb, Q_hx)

    def _axial_D(self, Dm, u_s, rho, mu):     # physics/dispersion.py:32-43
        tr = self.cfg.transport
        v = np.abs(u_s) / self.eps_b
        dp = self.dp
        if tr.dispersion_model == "edwards_richardson":
            return tr.er_gamma1 * Dm + tr.er_gamma2 * dp * v / (1.0 + tr.er_beta * tr.er_gamma1 * Dm / (dp * v + 1e-30))
        if tr.dispersion_model == "young2021":
            return 0.7 * Dm + 0.5 * dp * v
        Re = rho * np.abs(u_s) * dp / mu
        Sc = mu / (rho * Dm)
        return Dm / self.eps_b * (20.0 + 0.5 * Re * Sc)

    def _lam(self, lam0, C, cp, u, Pe):       # physics/heat_transfer.py:58-62
        return lam0 + C * cp * np.abs(u) * self.dp / Pe

    def _alpha_w(self, lam0, lam_g, rho, mu, cp_mass):   # physics/heat_transfer.py:64-76
        tr = self.cfg.transport
        if tr.wall_htc_model == "constant":
            return tr.wall_htc_constant * np.ones_like(lam0)
        N = 2.0 * self.cfg.geometry.bed_radius / self.dp
        Re = rho * np.abs(self.u_nom) * self.dp / mu
        Pr = cp_mass * mu / lam_g
        nu0 = (1.3 + 5.0 / N) * lam0 / lam_g
        if np.all(Re <= 0):
            dyn = 0.0
        else:
            a = 0.3 * Pr ** (1.0 / 3.0) * np.maximum(Re, 1e-12) ** 0.75
            b = 0.054 * Pr * np.maximum(Re, 1e-12)
            dyn = 1.0 / (1.0 / a + 1.0 / b)
        return (nu0 + dyn) * lam_g / self.dp

    def _wall_cond(self, Tw):                 # physics/energy.py:98-113
        g = self.grid
        out = np.zeros_like(Tw)
        if g.Nz > 1:
            fz = self.wall_lam * g.A_wall_axial / g.dz * (Tw[:, 1:] - Tw[:, :-1])
            out[:, :-1] += fz
            out[:, 1:] -= fz
        if g.Nth > 1:
            kt = self.wall_lam * g.wall_thickness * g.dz / (g.R_wall_mid * g.dth)
            ft = kt * (np.roll(Tw, -1, axis=0) - Tw)
            out += ft
            out -= np.roll(ft, 1, axis=0)
        return out

    def _div(self, Fz, Fr, Ft):               # physics/mass.py:61-74
        out = Fz[..., 1:] - Fz[..., :-1]
        if Fr is not None and Fr.shape[-3] > 0:
            out[..., :-1, :, :] += Fr
            out[..., 1:, :, :] -= Fr
        if Ft is not None and self.grid.Nth > 1:
            out += Ft - _prv(Ft)
        return out

    def eta_vacuum(self, P):                  # core/residual.py:204-208
        if self.vac_model == "krishnamurthy":
            pb = P / 1e5
            return np.maximum(0.8 * 19.55 * pb / (1.0 + 19.55 * pb), 1e-3)
        return self.eta_vac

    def _accumulators(self, bnd, T, Q_jac, Q_amb, Q_wb, Q_hx):   # core/residual.py:371-417
        acc = np.zeros(self.n_acc)
        ai = self.acc_index
        ex = (self.gam - 1.0) / self.gam
        pre = self.gam / (self.gam - 1.0) * R_GAS
        for end in ("top", "bottom"):
            cond = self.conds[end]
            if cond.valve is None:
                continue
            v, b = cond.valve, bnd[end]
            inflow = b["u_out"] < 0.0
            Fin = b["F_in"]
            if "F_inpart" in b:
                for k, s in enumerate(self.species):
                    acc[ai[f"n_in_{v}_{s}"]] = np.sum(b["F_inpart"][k])
                    acc[ai[f"n_out_{v}_{s}"]] = np.sum(b["F_outpart"][k])
                acc[ai[f"H_in_{v}"]] = np.sum(b["H_inpart"])
                acc[ai[f"H_out_{v}"]] = np.sum(b["H_outpart"])
            else:
                for k, s in enumerate(self.species):
                    acc[ai[f"n_in_{v}_{s}"]] = np.sum(np.where(inflow, Fin[k], 0.0))
                    acc[ai[f"n_out_{v}_{s}"]] = np.sum(np.where(inflow, 0.0, -Fin[k]))
                acc[ai[f"H_in_{v}"]] = np.sum(np.where(inflow, b["H_in"], 0.0))
                acc[ai[f"H_out_{v}"]] = np.sum(np.where(inflow, 0.0, -b["H_in"]))
            if cond.is_vacuum:
                Fout = np.where(inflow, 0.0, -Fin)
                if not self.pump_water and self.i_h2o is not None:
                    Fout = np.delete(Fout, self.i_h2o, axis=0)
                ratio = np.maximum(self.P_amb / np.maximum(b["P_face"], 1.0), 1.0)
                T_lay = T[..., 0] if end == "top" else T[..., -1]
                acc[ai[f"W_pump_{v}"]] = np.sum(pre * T_lay * Fout.sum(axis=0) * (ratio ** ex - 1.0)
                                                / self.eta_vacuum(b["P_face"]))
            if cond.is_feed:
                Ftot = b["F_inpart"].sum(axis=0) if "F_inpart" in b else np.where(inflow, Fin, 0.0).sum(axis=0)
                ratio = np.maximum(b["P_face"] / self.P_amb, 1.0)
                acc[ai[f"W_fan_{v}"]] = np.sum(pre * cond.T_ext * Ftot * (ratio ** ex - 1.0) / self.eta_bl)
        acc[ai["Q_jac_pos"]] = np.sum(np.maximum(Q_jac, 0.0))
        acc[ai["Q_jac_neg"]] = np.sum(np.minimum(Q_jac, 0.0))
        acc[ai["Q_amb"]] = np.sum(Q_amb)
        acc[ai["Q_wb"]] = np.sum(Q_wb)
        if Q_hx is not None:
            acc[ai["Q_hx_pos"]] = np.sum(np.maximum(Q_hx, 0.0))
            acc[ai["Q_hx_neg"]] = np.sum(np.minimum(Q_hx, 0.0))
        return acc

    # ---------------------------------------------------------------- solver helpers
    def stage_residual(self, t, y, gamma_h, rhs_known):      # core/residual.py:420-423
        f, _ = self.rhs(t, y, want_acc=False)
        return y - gamma_h * f - rhs_known

    def conservation_matrix(self):                            # core/residual.py:146-168
        import scipy.sparse as sp
        g = self.grid
        n = g.ncell
        Vc = np.broadcast_to(g.V, g.shape).ravel()
        rows, cols, vals = [], [], []
        for k, s in enumerate(self.species):
            rows.append(np.full(n, k)); cols.append(np.arange(k * n, (k + 1) * n)); vals.append(self.eps_t * Vc)
            if s in self.adsorbed:
                j = self.adsorbed.index(s)
                rows.append(np.full(n, k)); cols.append(self.off_q + np.arange(j * n, (j + 1) * n))
                vals.append(self.rho_b * Vc)
        rows.append(np.full(n, self.ng)); cols.append(self.off_e + np.arange(n)); vals.append(Vc)
        if self.n_w:
            rows.append(np.full(self.n_w, self.ng)); cols.append(self.off_w + np.arange(self.n_w))
            vals.append(np.full(self.n_w, self.wall_C))
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(self.ng + 1, self.n_core))

    def inventories(self, y):                                 # core/residual.py:426-443
        g = self.grid
        c, q, e, Tw = self.unpack(y)
        out = {}
        for k, s in enumerate(self.species):
            gas = float(np.sum(self.eps_t * c[k] * g.V))
            ads = float(np.sum(self.rho_b * q[self.adsorbed.index(s)] * g.V)) if s in self.adsorbed else 0.0
            out[f"gas_{s}"], out[f"ads_{s}"], out[f"tot_{s}"] = gas, ads, gas + ads
        out["E_bed"] = float(np.sum(e * g.V))
        out["E_wall"] = float(np.sum(self.wall_C * (Tw - self.T_ref))) if Tw is not None else 0.0
        out["E_total"] = out["E_bed"] + out["E_wall"]
        return out

    def q_feed_eq(self):                                      # core/residual.py:471-482
        cfg = self.cfg
        T = cfg.feed.T
        psat = float(self.props.p_sat(T))
        yv = humid_air_composition(self.species, cfg.feed.P, T, cfg.feed.RH if self.water else 0.0,
                                   cfg.feed.y_co2_dry, psat)
        p = yv * cfg.feed.P
        if self.water:
            return float(self.q_co2(p[self.i_co2], T, self.q_h2o(p[self.i_h2o], T, psat)))
        return float(self.q_co2_dry(p[self.i_co2], T))
