// dv_physics.cuh -- FP64 device closures of the finite-volume residual, one cell at a time.
//
// Every formula follows the reference's numpy code with the same operation order (the
// translation unit is compiled with -fmad=false, so +,-,*,/ and sqrt round exactly as numpy
// does; only the transcendental functions differ, by an ulp or so):
//   thermo             physics/energy.py:39-52        gas data   properties/ideal_gas_backend.py:48-137
//   diffusion          utils/diffusion.py:19-26       isotherms  physics/isotherms.py:34-153
//   LDF                physics/kinetics.py:29-39      Ergun      physics/pressure.py:36-56
//   dispersion         physics/dispersion.py:32-47    heat       physics/heat_transfer.py:23-76
//   stencils           numerics/stencils.py:45-101    fluxes     physics/mass.py:34-74
//   end faces          boundaries/conditions.py:43-160
//   residual assembly  core/residual.py:211-365
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "dacvtsa.h"

#define DV_R 8.314462618
#define DV_U_SMOOTH 1e-4
#define DV_VALVE_DP 0.2

namespace dv {

// numpy semantics: NaN propagates through maximum/minimum/clip
static __device__ __forceinline__ double npmax(double a, double b) { return (a >= b || a != a) ? a : b; }
static __device__ __forceinline__ double npmin(double a, double b) { return (a <= b || a != a) ? a : b; }
static __device__ __forceinline__ double npclip(double x, double lo, double hi) { return npmin(npmax(x, lo), hi); }

// np.logaddexp(0, x) (numpy npymath logaddexp)
static __device__ __forceinline__ double logaddexp0(double x) {
    if (x == 0.0) return 0.6931471805599453;   // log(2)
    double tmp = -x;
    if (tmp > 0.0) return log1p(exp(-tmp));
    if (tmp <= 0.0) return x + log1p(exp(tmp));
    return tmp;                                // NaN
}
static __device__ __forceinline__ double softplus(double x, double w) { return w * logaddexp0(x / w); }
static __device__ __forceinline__ double upw(double u) { return 0.5 * (1.0 + tanh(u / DV_U_SMOOTH)); }
static __device__ __forceinline__ double ergun_u(double g, double a, double b) {
    return -2.0 * g / (a + sqrt(a * a + 4.0 * b * fabs(g)));
}

struct Cell {           // raw unknowns of one cell
    double c[DV_NG], q[DV_NA], e;
};

struct Props {          // per-cell derived quantities used by fluxes (core/residual.py:219-238)
    double T, P, Tp, Cpos, y[DV_NG], mu, kg, rho, cpm, Dm, lam0;
};

static __device__ __forceinline__ double wsum3(const double w[3], const double a[3]) {
    double o = w[0] * a[0];
    o = o + w[1] * a[1];
    o = o + w[2] * a[2];
    return o;
}
static __device__ __forceinline__ double wsum2(const double w[2], const double a[2]) {
    double o = w[0] * a[0];
    o = o + w[1] * a[1];
    return o;
}

// T from (e, c, q): physics/energy.py:39-52
static __device__ __forceinline__ double cell_T(const dv_step_params& p, const Cell& s) {
    double Cg = s.c[0] + s.c[1] + s.c[2];
    double A = p.eps_t * wsum3(p.cpg, s.c) + p.rho_b * (p.cp_s + wsum2(p.cpa, s.q));
    double B = p.eps_t * DV_R * Cg;
    double Hq = p.rho_b * wsum2(p.dH, s.q);
    return (s.e - Hq + A * p.T_ref) / (A - B);
}

static __device__ __forceinline__ double fuller(const dv_step_params& p, int pair, double T, double P) {
    P = npmax(P, 1.0);
    return 1.43e-7 * pow(T, 1.75) / ((P / 1e5) * p.fuller_sqrtM[pair] * p.fuller_s[pair] * p.fuller_s[pair]);
}

static __device__ __forceinline__ double stagnant(const dv_step_params& p, double lam_g) {   // heat_transfer.py:23-56
    if (p.bed_model == DV_BED_CONSTANT) return p.lam_const * 1.0;
    if (p.bed_model == DV_BED_PARALLEL) return p.eps_b * lam_g + (1.0 - p.eps_b) * p.lam_s;
    double kap = p.lam_s / lam_g;
    double B = p.zs_B, s = p.zs_s;
    double one_m = 1.0 - B / kap;
    double kc = (2.0 / one_m) * ((1.0 - 1.0 / kap) * B / (one_m * one_m) * log(kap / B)
                                 - 0.5 * (B + 1.0) - (B - 1.0) / one_m);
    return lam_g * (1.0 - s + s * kc);
}

// The state part of the cell properties: T, P, clipped T, positive total concentration, mole
// fractions and their clipped copies.
static __device__ __forceinline__ void props_state(const dv_step_params& p, const Cell& s, Props& o, double ycl[DV_NG]) {
    double Ctot = s.c[0] + s.c[1] + s.c[2];
    o.T = cell_T(p, s);
    o.P = Ctot * DV_R * o.T;
    o.Tp = npclip(o.T, 150.0, 1500.0);
    o.Cpos = npmax(Ctot, 1e-9);
#pragma unroll
    for (int k = 0; k < DV_NG; ++k) {
        o.y[k] = s.c[k] / o.Cpos;
        ycl[k] = npclip(o.y[k], 0.0, 1.0);
    }
}

// pure-gas viscosity and conductivity of gas s2 (ideal_gas_backend.py:94-113,148-166); T3 = T / 300
static __device__ __forceinline__ double gas_mu(const dv_step_params& p, int s2, double T) {
    if (p.mu_nt[s2] == 1) return p.mu_D[s2][0] * T + p.mu_E[s2][0];
    return p.mu_w[s2][0] * (p.mu_D[s2][0] * T + p.mu_E[s2][0]) + p.mu_w[s2][1] * (p.mu_D[s2][1] * T + p.mu_E[s2][1]);
}
static __device__ __forceinline__ double gas_k(const dv_step_params& p, int s2, double T3) {
    if (p.k_nt[s2] == 1) return p.k_0[s2][0] * pow(T3, p.k_n[s2][0]);
    return p.k_w[s2][0] * p.k_0[s2][0] * pow(T3, p.k_n[s2][0]) + p.k_w[s2][1] * p.k_0[s2][1] * pow(T3, p.k_n[s2][1]);
}

// Wilke & Mason-Saxena mixing of the pure-gas viscosities and conductivities
static __device__ __forceinline__ void wilke_mix(const dv_step_params& p, const double ycl[DV_NG], const double mu[DV_NG],
                                                 const double kk[DV_NG], const double sq[DV_NG], double& mu_m, double& k_m) {
    mu_m = 0.0;
    k_m = 0.0;
#pragma unroll
    for (int i = 0; i < DV_NG; ++i) {
        double den = 0.0;
#pragma unroll
        for (int j = 0; j < DV_NG; ++j) {
            if (i == j) {
                den = den + ycl[j];
            } else {
                double t1 = 1.0 + (sq[i] / sq[j]) * p.mass_q[i][j];
                den = den + ycl[j] * ((t1 * t1) / p.wilke_den[i][j]);
            }
        }
        den = npmax(den, 1e-30);
        mu_m = mu_m + ycl[i] * mu[i] / den;
        k_m = k_m + ycl[i] * kk[i] / den;
    }
}

// Blanc CO2 diffusivity over air and water (ideal_gas_backend.py:127-137) from the two Fuller values
static __device__ __forceinline__ double blanc_Dm(const double ycl[DV_NG], double D_ca, double D_cw) {
    double yi = ycl[2], yw = ycl[1];
    return (yi + yw + 1e-9) / (yi / D_ca + yw / D_cw + 1e-9 / D_ca);
}

static __device__ void cell_props(const dv_step_params& p, const Cell& s, Props& o) {
    double ycl[DV_NG];
    props_state(p, s, o, ycl);
    const double T = o.Tp;
    double mu[DV_NG], kk[DV_NG], sq[DV_NG];
    const double T3 = T / 300.0;
#pragma unroll
    for (int s2 = 0; s2 < DV_NG; ++s2) {
        mu[s2] = gas_mu(p, s2, T);
        kk[s2] = gas_k(p, s2, T3);
        sq[s2] = sqrt(mu[s2]);
    }
    double mu_m, k_m;
    wilke_mix(p, ycl, mu, kk, sq, mu_m, k_m);
    o.mu = mu_m;
    o.kg = k_m;
    o.rho = o.Cpos * wsum3(p.M, ycl);
    o.cpm = wsum3(p.cpg, ycl);
    double Pc = npmax(o.P, 1.0);
    o.Dm = blanc_Dm(ycl, fuller(p, 0, T, Pc), fuller(p, 1, T, Pc));
    o.lam0 = stagnant(p, o.kg);
}

// ---------------------------------------------------------------- isotherms + LDF
static __device__ __forceinline__ double toth(double pr, double T, double q_inf0, double chi, double b0, double dH0,
                                       double tau0, double alpha, double T0) {   // isotherms.py:50-56
    pr = npmax(pr, 0.0);
    double qinf = q_inf0 * exp(chi * (1.0 - T / T0));
    double b = b0 * exp(-dH0 / (DV_R * T));
    double tau = tau0 + alpha * (1.0 - T0 / T);
    double bp = b * pr;
    return qinf * bp / pow(1.0 + pow(bp, tau), 1.0 / tau);
}

static __device__ __forceinline__ double smooth_cap(double x, double cap) {   // isotherms.py:70-80
    const double width = 0.02;
    x = npmax(x, -0.2);
    double lo = cap - width;
    double over = npmax(x - lo, 0.0);
    double blend = lo + over - (over * over) / (4.0 * width);
    return (x <= lo) ? x : ((over >= 2.0 * width) ? cap : blend);
}

static __device__ __forceinline__ double q_h2o(const dv_step_params& p, double pw, double T, double psat) {  // gab
    double x = smooth_cap(pw / psat, p.rh_cap);
    double E1 = p.h2o_C - exp(p.h2o_D * T);
    double E29 = p.h2o_F + p.h2o_G * T;
    double E10 = p.h2o_E10_slope * T + p.h2o_E10_intercept;
    double RT = DV_R * T;
    double c = exp((E1 - E10) / RT);
    double k = exp((E29 - E10) / RT);
    double kx = k * x;
    return p.h2o_q_m * c * kx / ((1.0 - kx) * (1.0 + (c - 1.0) * kx));
}

// The Toth terms of the CO2 isotherm that do not depend on the water loading: the dry one (models
// none and wadst) and the wet one (wadst); pp = max(p_CO2, 0).
static __device__ __forceinline__ double co2_toth_dry(const dv_step_params& p, double pp, double T) {
    return toth(pp, T, p.co2_q_inf0, p.co2_chi, p.co2_b0, p.co2_dH0, p.co2_tau0, p.co2_alpha, p.co2_T0);
}
static __device__ __forceinline__ double co2_toth_wet(const dv_step_params& p, double pp, double T) {
    return toth(pp, T, p.wadst_q_inf0, p.wadst_chi, p.wadst_b0, p.wadst_dH, p.wadst_tau0, p.wadst_alpha, p.co2_T0);
}
// WADST blend of the two Toth terms by the water loading qw (already floored at 1e-12)
static __device__ __forceinline__ double wadst_blend(const dv_step_params& p, double qw, double q_dry, double q_wet) {
    double w = exp(-p.wadst_A / qw);
    return (1.0 - w) * q_dry + w * q_wet;
}
// the co-adsorption models whose Toth terms need the water loading first
static __device__ __forceinline__ bool co2_needs_qw(const dv_step_params& p) {
    return p.coads != DV_COADS_NONE && p.coads != DV_COADS_WADST;
}

// CO2 loading before the low-pressure regularisation (isotherms.py:108-143); pp = max(p_CO2, 0).
// q_dry / q_wet: the Toth terms when already evaluated (models none and wadst), else NaN.
static __device__ double q_co2_raw(const dv_step_params& p, double pp, double T, double qw, double q_dry, double q_wet) {
    if (p.coads == DV_COADS_NONE) return (q_dry == q_dry) ? q_dry : co2_toth_dry(p, pp, T);
    qw = npmax(qw, 1e-12);
    if (p.coads == DV_COADS_WADST) {
        if (q_wet != q_wet) q_wet = co2_toth_wet(p, pp, T);
        if (q_dry != q_dry) q_dry = co2_toth_dry(p, pp, T);
        return wadst_blend(p, qw, q_dry, q_wet);
    }
    if (p.coads == DV_COADS_MECHANISTIC) {
        double w = exp(-p.mech_A / qw);
        double f_bl = p.mech_f_blocked_max * (1.0 - exp(-pow(p.mech_k * qw, p.mech_n)));
        double phi_av = 1.0 - f_bl;
        double phi = p.mech_phi_dry + (phi_av - p.mech_phi_dry) * w;
        double dH_ave = (1.0 - w) * p.co2_dH0 + w * p.mech_dH_wet;
        return (phi / p.mech_phi_dry) * toth(pp, T, p.co2_q_inf0, p.co2_chi, p.co2_b0, dH_ave, p.co2_tau0,
                                             p.co2_alpha, p.co2_T0);
    }
    double qi = p.co2_q_inf0 / (1.0 - p.sb_gamma * qw);
    double b0 = p.co2_b0 * (1.0 + p.sb_beta * qw);
    return toth(pp, T, qi, p.co2_chi, b0, p.co2_dH0, p.co2_tau0, p.co2_alpha, p.co2_T0);
}

static __device__ __forceinline__ double q_co2(const dv_step_params& p, double pc, double T, double qw) {
    double pp = npmax(pc, 0.0);
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    return q_co2_raw(p, pp, T, qw, nan, nan) * (pp / (pp + p.p_reg));
}

// saturation pressure of water (Arden Buck) at the clipped temperature
static __device__ __forceinline__ double psat_h2o(double Tp) {
    double Tc = Tp - 273.15;
    return 611.21 * exp((18.678 - Tc / 234.5) * (Tc / (257.14 + Tc)));
}

// LDF rates from the equilibrium loadings (core/residual.py:232-238)
static __device__ __forceinline__ void ldf_rates(const dv_step_params& p, const Cell& s, double Tp,
                                                 const double qstar[DV_NA], double rate[DV_NA]) {
#pragma unroll
    for (int j = 0; j < DV_NA; ++j) {
        double k = p.k_ldf[j];
        if (!p.ea_zero) k = p.k_ldf[j] * exp(-p.Ea[j] / DV_R * (1.0 / Tp - 1.0 / p.T_ref_kin));
        else k = k * 1.0;
        rate[j] = k * (qstar[j] - s.q[j]);
    }
}

// LDF rates (na) and equilibrium loadings of one cell (core/residual.py:232-238)
static __device__ void uptake(const dv_step_params& p, const Cell& s, const Props& o, double rate[DV_NA], double qstar[DV_NA]) {
    const double Tp = o.Tp;
    double pk0 = s.c[0] * DV_R * Tp;
    double pk1 = s.c[1] * DV_R * Tp;
    double psat = psat_h2o(Tp);
    double qw_eq = q_h2o(p, pk1, Tp, psat);
    double basis = p.basis_state ? s.q[1] : qw_eq;
    qstar[0] = q_co2(p, pk0, Tp, basis);
    qstar[1] = qw_eq;
    ldf_rates(p, s, Tp, qstar, rate);
}

// ---------------------------------------------------------------- faces
static __device__ __forceinline__ double limited_slope(int lim, double dm, double dp) {   // stencils.py:59-76
    if (lim == DV_LIM_UPWIND) return 0.0;
    double prod = dm * dp;
    if (lim == DV_LIM_VAN_ALBADA) return prod * (dm + dp) / (dm * dm + dp * dp + 1e-300);
    if (lim == DV_LIM_VAN_ALBADA_TVD) return (prod > 0.0) ? prod * (dm + dp) / (dm * dm + dp * dp + 1e-300) : 0.0;
    if (lim == DV_LIM_VAN_LEER) return (prod > 0.0) ? 2.0 * prod / (dm + dp + 1e-300) : 0.0;
    if (prod > 0.0) {
        double sg = (dm > 0.0) ? 1.0 : ((dm < 0.0) ? -1.0 : 0.0);
        return sg * npmin(fabs(dm), fabs(dp));
    }
    return 0.0;
}

static __device__ __forceinline__ double enth(const dv_step_params& p, const double F[DV_NG], double Tf) {
    return wsum3(p.cpg, F) * (Tf - p.T_ref);     // physics/energy.py:81-83
}

struct Flux { double F[DV_NG]; double H; };

// Interior z-face between cells L (k) and R (k+1) of column (i, j).
// phiL/phiR limited slopes sL/sR (index 0..2 species, 3 = T); N_nom: nominal column flux.
static __device__ void zface(const dv_step_params& p, int i, const Props& L, const Props& R, const Cell& cL, const Cell& cR,
                      const double sL[4], const double sR[4], bool muscl, double N_nom, Flux& out, double* uz_out) {
    double mu_z = 0.5 * (R.mu + L.mu), rho_z = 0.5 * (R.rho + L.rho);
    double uz = ergun_u((R.P - L.P) / p.dz, p.ka * mu_z, p.kb * rho_z);
    if (uz_out) *uz_out = uz;
    double w = upw(uz);
    double Cz = 0.5 * (R.Cpos + L.Cpos);
    double u_disp = N_nom / Cz;
    double Dmf = 0.5 * (R.Dm + L.Dm);
    double v = fabs(u_disp) / p.eps_b;
    double Dz;
    if (p.disp_model == DV_DISP_EDWARDS_RICHARDSON)
        Dz = p.g1 * Dmf + p.g2 * p.dp * v / (1.0 + p.er_beta * p.g1 * Dmf / (p.dp * v + 1e-30));
    else if (p.disp_model == DV_DISP_YOUNG2021)
        Dz = 0.7 * Dmf + 0.5 * p.dp * v;
    else {
        double Re = rho_z * fabs(u_disp) * p.dp / mu_z;
        double Sc = mu_z / (rho_z * Dmf);
        Dz = Dmf / p.eps_b * (20.0 + 0.5 * Re * Sc);
    }
    const double Az = p.Az[i];
    double Fconv[DV_NG], J[DV_NG];
#pragma unroll
    for (int k = 0; k < DV_NG; ++k) {
        double fv = muscl ? (w * (cL.c[k] + 0.5 * sL[k]) + (1.0 - w) * (cR.c[k] - 0.5 * sR[k]))
                          : (w * cL.c[k] + (1.0 - w) * cR.c[k]);
        Fconv[k] = uz * Az * fv;
        J[k] = -p.eps_b * Dz * Cz * (R.y[k] - L.y[k]) / p.dz * Az;
        out.F[k] = Fconv[k] + J[k];
    }
    double Tf = muscl ? (w * (L.T + 0.5 * sL[3]) + (1.0 - w) * (R.T - 0.5 * sR[3])) : (w * L.T + (1.0 - w) * R.T);
    double cpz = 0.5 * (R.cpm + L.cpm);
    double lam_z = 0.5 * (R.lam0 + L.lam0) + Cz * cpz * fabs(u_disp) * p.dp / p.Pe_z;
    out.H = enth(p, Fconv, Tf) + enth(p, J, 0.5 * (R.T + L.T)) - lam_z * (R.T - L.T) / p.dz * Az;
}

// Transverse (r or theta) face between cells A (minus side) and B (plus side):
// dist = drc (r) or arc (theta), area = Ar or Ath.
static __device__ void tface(const dv_step_params& p, const Props& A, const Props& B, const Cell& cA, const Cell& cB,
                      double dist, double area, Flux& out, double* u_out) {
    double mu_f = 0.5 * (B.mu + A.mu), rho_f = 0.5 * (B.rho + A.rho);
    double u = ergun_u((B.P - A.P) / dist, p.ka * mu_f, p.kb * rho_f);
    if (u_out) *u_out = u;
    double w = upw(u);
    double Cf = 0.5 * (A.Cpos + B.Cpos);
    double vn = fabs(p.u_nom) / p.eps_b;
    double Df = p.g1 * (0.5 * (A.Dm + B.Dm)) + p.dp * vn / p.Pe_T;
    double Fconv[DV_NG], J[DV_NG];
#pragma unroll
    for (int k = 0; k < DV_NG; ++k) {
        Fconv[k] = u * area * (w * cA.c[k] + (1.0 - w) * cB.c[k]);
        J[k] = -p.eps_b * Df * Cf * (B.y[k] - A.y[k]) / dist * area;
        out.F[k] = Fconv[k] + J[k];
    }
    double lam = 0.5 * (A.lam0 + B.lam0) + Cf * (0.5 * (A.cpm + B.cpm)) * fabs(p.u_nom) * p.dp / p.Pe_r;
    out.H = enth(p, Fconv, w * A.T + (1.0 - w) * B.T) + enth(p, J, 0.5 * (A.T + B.T)) - lam * (B.T - A.T) / dist * area;
}

// Boundary record of one end face (accumulators / diagnostics), 16 doubles.
enum { BR_FIN = 0, BR_HIN = 3, BR_UOUT = 4, BR_PFACE = 5, BR_FINP = 6, BR_FOUTP = 9, BR_HINP = 12, BR_HOUTP = 13,
       BR_TLAY = 14, BR_N = 16 };

// End-face flux INTO the bed (boundaries/conditions.py:75-160); rec (16 fields, stride rs) optional.
static __device__ void end_face(const dv_step_params& p, const dv_end& e, double t, int i, const Cell& s, const Props& o,
                         double feed_flux, double F_in[DV_NG], double& H_in, double* rec, int64_t rs) {
    const double Az = p.Az[i];
    const double half_dz = 0.5 * p.dz;
    double u_out = 0.0, P_face = o.P;
    double Fip[DV_NG] = {0.0, 0.0, 0.0}, Fop[DV_NG] = {0.0, 0.0, 0.0}, Hip = 0.0, Hop = 0.0;
    if (e.kind == DV_END_CLOSED) {
#pragma unroll
        for (int k = 0; k < DV_NG; ++k) F_in[k] = 0.0;
        H_in = 0.0;
    } else {
        double a = p.ka * o.mu, b = p.kb * o.rho;
        double C_cell = npmax(s.c[0] + s.c[1] + s.c[2], 1e-12);
        if (e.kind == DV_END_FEED) {
#pragma unroll
            for (int k = 0; k < DV_NG; ++k) F_in[k] = feed_flux * e.y_ext[k];
            H_in = wsum3(p.cpg, F_in) * (e.T_ext - p.T_ref);
            double u_in = feed_flux / (Az * C_cell);
            u_out = -u_in;
            P_face = o.P + (a * u_in + b * u_in * u_in) * half_dz;
        } else if (e.kind == DV_END_PUMP) {
            double dp = o.P - e.P_target;
            double w_out;
            if (e.check_valve) {
                dp = softplus(dp, 1.0);
                w_out = 1.0;
            } else {
                w_out = 0.5 * (1.0 + tanh(dp / DV_VALVE_DP));
            }
            double N_out = e.speed * dp / (DV_R * o.T);
            double F_out[DV_NG];
#pragma unroll
            for (int k = 0; k < DV_NG; ++k) {
                double y_use = w_out * (s.c[k] / C_cell) + (1.0 - w_out) * e.y_ext[k];
                F_out[k] = N_out * Az * y_use;
                F_in[k] = -F_out[k];
            }
            double T_up = w_out * o.T + (1.0 - w_out) * e.T_ext;
            H_in = -(wsum3(p.cpg, F_out) * (T_up - p.T_ref));
            u_out = N_out / C_cell;
            P_face = o.P - (a * u_out + b * fabs(u_out) * u_out) * half_dz;
        } else if (e.kind == DV_END_VALVE) {
            double P_res = (p.tau_valve > 0.0) ? e.P_target + (e.P_start - e.P_target) * exp(-t / p.tau_valve) : e.P_target;
            double dp = P_res - o.P;
            double N_in = e.speed * softplus(dp, DV_VALVE_DP) / (DV_R * e.T_ext);
            double N_out = e.speed * softplus(-dp, DV_VALVE_DP) / (DV_R * o.T);
#pragma unroll
            for (int k = 0; k < DV_NG; ++k) {
                Fip[k] = N_in * Az * e.y_ext[k];
                Fop[k] = N_out * Az * (s.c[k] / C_cell);
                F_in[k] = Fip[k] - Fop[k];
            }
            Hip = wsum3(p.cpg, Fip) * (e.T_ext - p.T_ref);
            Hop = wsum3(p.cpg, Fop) * (o.T - p.T_ref);
            H_in = Hip - Hop;
            double N_net = N_in - N_out;
            u_out = -N_net / C_cell;
            P_face = o.P - (a * u_out + b * fabs(u_out) * u_out) * half_dz;
        } else {   // Dirichlet pressure ramp port
            P_face = (e.P_target + (e.P_start - e.P_target) * exp(-t / p.tau_valve)) * 1.0;
            double uo = ergun_u((P_face - o.P) / half_dz, a, b);
            if (e.check_valve) uo = 0.5 * (uo + sqrt(uo * uo + 1e-7 * 1e-7)) - 0.5 * 1e-7;
            double w = upw(uo);
            double F_out[DV_NG];
#pragma unroll
            for (int k = 0; k < DV_NG; ++k) {
                double c_ext = e.y_ext[k] * P_face / (DV_R * e.T_ext);
                F_out[k] = uo * Az * (w * s.c[k] + (1.0 - w) * c_ext);
                F_in[k] = -F_out[k];
            }
            double T_up = w * o.T + (1.0 - w) * e.T_ext;
            H_in = -(wsum3(p.cpg, F_out) * (T_up - p.T_ref));
            u_out = uo;
        }
    }
    if (rec) {
#pragma unroll
        for (int k = 0; k < DV_NG; ++k) {
            rec[(BR_FIN + k) * rs] = F_in[k];
            rec[(BR_FINP + k) * rs] = Fip[k];
            rec[(BR_FOUTP + k) * rs] = Fop[k];
        }
        rec[BR_HIN * rs] = H_in;
        rec[BR_UOUT * rs] = u_out;
        rec[BR_PFACE * rs] = P_face;
        rec[BR_HINP * rs] = Hip;
        rec[BR_HOUTP * rs] = Hop;
        rec[BR_TLAY * rs] = o.T;
        rec[15 * rs] = 0.0;
    }
}

// Bed-side wall resistance of an outer-ring cell (core/residual.py:329-335)
static __device__ __forceinline__ double wall_R_bed(const dv_step_params& p, const Props& o) {
    if (p.lumped) return 1.0 / p.U_lumped;
    double lam_out = o.lam0 + o.Cpos * o.cpm * fabs(p.u_nom) * p.dp / p.Pe_r;
    double aw;
    if (p.htc_model == DV_HTC_CONSTANT) {
        aw = p.alpha_const * 1.0;
    } else {
        double cp_mass = o.cpm / npmax(o.rho / o.Cpos, 1e-6);
        double Re = o.rho * fabs(p.u_nom) * p.dp / o.mu;
        double Pr = cp_mass * o.mu / o.kg;
        double nu0 = (1.3 + 5.0 / p.N_ratio) * o.lam0 / o.kg;
        double dyn = 0.0;
        if (p.u_nom != 0.0) {     // reference: np.all(Re <= 0) -> 0 (Re = 0 exactly when u_nom = 0)
            double Rm = npmax(Re, 1e-12);
            double a = 0.3 * pow(Pr, 1.0 / 3.0) * pow(Rm, 0.75);
            double b = 0.054 * Pr * Rm;
            dyn = 1.0 / (1.0 / a + 1.0 / b);
        }
        aw = (nu0 + dyn) * o.kg / p.dp;
    }
    return 1.0 / aw + p.half_dr_outer / lam_out;
}

static __device__ __forceinline__ double jacket_T(const dv_step_params& p, double t) {   // core/residual.py:199-202
    if (p.jac_tau <= 0.0) return p.T_jac_set;
    return p.T_jac_set + (p.T_jac_prev - p.T_jac_set) * exp(-t / p.jac_tau);
}

}  // namespace dv
