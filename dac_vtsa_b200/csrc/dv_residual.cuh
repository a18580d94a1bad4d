// dv_residual.cuh -- residual of one cell (core/residual.py:211-365) from the raw state of its
// stencil, shared by the rhs / stage-residual / matvec kernels and the FD Jacobian kernel.
#pragma once
#include "dv_physics.cuh"

namespace dv {

struct Aux {                   // per-step device arrays
    const double* feed_flux;   // (Nr, Nth) mol/s per inlet face
    const double* n_nom;       // (Nr, Nth) nominal column flux mol/m2/s
    const double* cov;         // (Nth, Nz) jacket coverage
};

struct Rec {                   // optional per-face / per-wall records (accumulators, diagnostics)
    double* bnd;               // [2][BR_N][Nr*Nth]
    double* Qj;                // [Nth*Nz] Q_jac
    double* Qa;                // Q_amb
    double* Qw;                // Q_wb
    double* Rb;                // R_bed
    double* Qhx;               // [ncell]
    double* uz;                // [Nr*Nth*(Nz-1)]
    double* ur;                // [(Nr-1)*Nth*Nz]
    double* uth;               // [ncell]
    double* T;                 // [ncell]
    double* P;
    double* y;                 // [3][ncell]
    double* qstar;             // [2][ncell]
};

struct LoadPlain {
    const double* y;
    __device__ __forceinline__ double operator()(int64_t i) const { return y[i]; }
};
struct LoadPert {              // y with one column perturbed: yp = y; yp[col] += h (core/jacobian.py:79-82)
    const double* y;
    int64_t col;
    double h;
    __device__ __forceinline__ double operator()(int64_t i) const {
        double v = y[i];
        return (i == col) ? v + h : v;
    }
};
struct LoadDir {               // z + sig * (u * s): the finite-difference matvec point (core/solver.py:196-203)
    const double* z;
    const double* u;
    const double* s;
    double sig;
    __device__ __forceinline__ double operator()(int64_t i) const { return z[i] + sig * (u[i] * s[i]); }
};

template <class L>
static __device__ __forceinline__ void load_cell(const L& ld, int64_t nc, int64_t c, Cell& s) {
    s.c[0] = ld(c);
    s.c[1] = ld(nc + c);
    s.c[2] = ld(2 * nc + c);
    s.q[0] = ld(3 * nc + c);
    s.q[1] = ld(4 * nc + c);
    s.e = ld(5 * nc + c);
}

static __device__ __forceinline__ void slope4(int lim, const Cell& m, const double Tm, const Cell& o, const double To,
                                       const Cell& pl, const double Tp, double s[4]) {
#pragma unroll
    for (int k = 0; k < DV_NG; ++k) s[k] = limited_slope(lim, o.c[k] - m.c[k], pl.c[k] - o.c[k]);
    s[3] = limited_slope(lim, To - Tm, Tp - To);
}

// Divergence of the face fluxes, sorption sinks, wall / jacket / exchanger terms and records of
// cell (i,j,k) (core/residual.py:298-365): f[0..5]; *fw = dTw/dt of its wall node.  Shared by the
// thread-per-cell residual and the split residual's assembly, so both add in the same order.
template <class L>
static __device__ __forceinline__ void cell_tail(const dv_step_params& p, const Aux& aux, const L& ld, double t, int i,
                                                 int j, int k, const Props& P0, const double rate[DV_NA],
                                                 const double qstar[DV_NA], const Flux& Fzm, const Flux& Fzp,
                                                 const Flux& Frm, const Flux& Frp, const Flux& Ftm, const Flux& Ftp,
                                                 double f[DV_NV], double* fw, const Rec* rec) {
    const int Nr = p.Nr, Nth = p.Nth, Nz = p.Nz;
    const int64_t nc = (int64_t)Nr * Nth * Nz;
    const int64_t c0 = ((int64_t)i * Nth + j) * Nz + k;
    const int64_t off_w = (int64_t)DV_NV * nc;
    // ---------------- divergence (physics/mass.py:61-74) and species balance
    const double V = p.V[i];
#pragma unroll
    for (int q = 0; q < DV_NG; ++q) {
        double d = Fzp.F[q] - Fzm.F[q];
        if (Nr > 1) {
            if (i < Nr - 1) d = d + Frp.F[q];
            if (i > 0) d = d - Frm.F[q];
        }
        if (Nth > 1) d = d + (Ftp.F[q] - Ftm.F[q]);
        double sink = (q < DV_NA) ? rate[q] : 0.0;
        f[q] = -d / (p.eps_t * V) - (p.rho_b / p.eps_t) * sink;
    }
    f[3] = rate[0];
    f[4] = rate[1];
    double de = Fzp.H - Fzm.H;
    if (Nr > 1) {
        if (i < Nr - 1) de = de + Frp.H;
        if (i > 0) de = de - Frm.H;
    }
    if (Nth > 1) de = de + (Ftp.H - Ftm.H);
    // ---------------- wall / jacket / exchanger (core/residual.py:328-359)
    double src = 0.0;
    const double Tj = jacket_T(p, t);
    if (i == Nr - 1) {
        const int64_t wn = (int64_t)j * Nz + k;
        const double cov = aux.cov[wn];
        const double To = P0.T;
        const double R_bed = wall_R_bed(p, P0);
        double Q_jac, Q_amb, Q_wb;
        if (p.wall_on) {
            const double Tw = ld(off_w + wn);
            Q_jac = p.jacket_on ? cov * p.h_jac * p.A_wall_out * (Tj - Tw) : 0.0;
            Q_amb = (1.0 - cov) * p.h_amb * p.A_wall_out * (p.T_amb - Tw);
            Q_wb = p.A_wall_in * (Tw - To) / R_bed;
            double cond = 0.0;
            if (Nz > 1) {
                if (k < Nz - 1) cond = cond + p.wall_kz * (ld(off_w + wn + 1) - Tw);
                if (k > 0) cond = cond - p.wall_kz * (Tw - ld(off_w + wn - 1));
            }
            if (Nth > 1) {
                const int jm = (j == 0) ? Nth - 1 : j - 1;
                const int jp = (j == Nth - 1) ? 0 : j + 1;
                const double Twp = ld(off_w + (int64_t)jp * Nz + k);
                const double Twm = ld(off_w + (int64_t)jm * Nz + k);
                cond = cond + p.wall_kt * (Twp - Tw);
                cond = cond - p.wall_kt * (Tw - Twm);
            }
            if (fw) *fw = (Q_jac + Q_amb - Q_wb + cond) / p.wall_C;
        } else {
            if (p.jacket_on && p.h_jac > 0.0) {
                double R_j = p.lumped ? R_bed : R_bed + 1.0 / p.h_jac;
                Q_jac = cov * p.A_wall_in * (Tj - To) / R_j;
            } else {
                Q_jac = 0.0;
            }
            Q_amb = (p.h_amb > 0.0) ? (1.0 - cov) * p.A_wall_in * (p.T_amb - To) / (R_bed + 1.0 / p.h_amb) : 0.0;
            Q_wb = Q_jac + Q_amb;
        }
        src = src + Q_wb;
        if (rec) {
            rec->Qj[wn] = Q_jac;
            rec->Qa[wn] = Q_amb;
            rec->Qw[wn] = Q_wb;
            rec->Rb[wn] = R_bed;
        }
    }
    double Q_hx = 0.0;
    if (p.hx_on) {
        Q_hx = p.hA_v * V * (Tj - P0.T);
        src = src + Q_hx;
    }
    f[5] = (-de + src) / V;
    if (rec) {
        rec->Qhx[c0] = Q_hx;
        rec->T[c0] = P0.T;
        rec->P[c0] = P0.P;
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) rec->y[q * nc + c0] = P0.y[q];
        rec->qstar[c0] = qstar[0];
        rec->qstar[nc + c0] = qstar[1];
    }
}

// f[0..5] = d(c, q, e)/dt of cell (i,j,k); *fw = dTw/dt of its wall node (outer ring, wall on).
template <class L>
static __device__ void cell_eval(const dv_step_params& p, const Aux& aux, const L& ld, double t, int i, int j, int k,
                          double f[DV_NV], double* fw, const Rec* rec) {
    const int Nr = p.Nr, Nth = p.Nth, Nz = p.Nz;
    const int64_t nc = (int64_t)Nr * Nth * Nz;
    const int64_t c0 = ((int64_t)i * Nth + j) * Nz + k;
    Cell s0;
    load_cell(ld, nc, c0, s0);
    Props P0;
    cell_props(p, s0, P0);
    double rate[DV_NA], qstar[DV_NA];
    uptake(p, s0, P0, rate, qstar);
    const bool muscl = (Nz >= 3 && p.limiter != DV_LIM_UPWIND);
    const int lim = p.limiter;
    const int col = i * Nth + j;
    const double N_nom = aux.n_nom[col];

    // ---------------- axial faces k-1/2 and k+1/2 (flux in +z)
    Flux Fzm, Fzp;
    double s_k[4] = {0.0, 0.0, 0.0, 0.0};
    Cell sm1, sp1, sm2, sp2;
    double Tm1 = 0.0, Tp1 = 0.0, Tm2 = 0.0, Tp2 = 0.0;
    if (k > 0) { load_cell(ld, nc, c0 - 1, sm1); Tm1 = cell_T(p, sm1); }
    if (k < Nz - 1) { load_cell(ld, nc, c0 + 1, sp1); Tp1 = cell_T(p, sp1); }
    if (muscl && k >= 1 && k <= Nz - 2) slope4(lim, sm1, Tm1, s0, P0.T, sp1, Tp1, s_k);
    if (k > 0) {
        double s_m[4] = {0.0, 0.0, 0.0, 0.0};
        if (muscl && k - 1 >= 1) {
            load_cell(ld, nc, c0 - 2, sm2);
            Tm2 = cell_T(p, sm2);
            slope4(lim, sm2, Tm2, sm1, Tm1, s0, P0.T, s_m);
        }
        Props Pm;
        cell_props(p, sm1, Pm);
        zface(p, i, Pm, P0, sm1, s0, s_m, s_k, muscl, N_nom, Fzm, nullptr);
    } else {
        double F_in[DV_NG], H_in;
        end_face(p, p.ends[0], t, i, s0, P0, aux.feed_flux[col], F_in, H_in,
                 rec ? rec->bnd + (int64_t)col : nullptr, (int64_t)Nr * Nth);
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) Fzm.F[q] = F_in[q];
        Fzm.H = H_in;
    }
    if (k < Nz - 1) {
        double s_p[4] = {0.0, 0.0, 0.0, 0.0};
        if (muscl && k + 1 <= Nz - 2) {
            load_cell(ld, nc, c0 + 2, sp2);
            Tp2 = cell_T(p, sp2);
            slope4(lim, s0, P0.T, sp1, Tp1, sp2, Tp2, s_p);
        }
        Props Pp;
        cell_props(p, sp1, Pp);
        double uz;
        zface(p, i, P0, Pp, s0, sp1, s_k, s_p, muscl, N_nom, Fzp, &uz);
        if (rec) rec->uz[(int64_t)col * (Nz - 1) + k] = uz;
    } else {
        double F_in[DV_NG], H_in;
        end_face(p, p.ends[1], t, i, s0, P0, aux.feed_flux[col], F_in, H_in,
                 rec ? rec->bnd + (int64_t)BR_N * Nr * Nth + col : nullptr, (int64_t)Nr * Nth);
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) Fzp.F[q] = -F_in[q];
        Fzp.H = -H_in;
    }
    // ---------------- radial faces
    Flux Frm, Frp;
    if (Nr > 1) {
        if (i > 0) {
            Cell sa;
            load_cell(ld, nc, c0 - (int64_t)Nth * Nz, sa);
            Props Pa;
            cell_props(p, sa, Pa);
            tface(p, Pa, P0, sa, s0, p.drc[i - 1], p.Ar[i - 1], Frm, nullptr);
        }
        if (i < Nr - 1) {
            Cell sb;
            load_cell(ld, nc, c0 + (int64_t)Nth * Nz, sb);
            Props Pb;
            cell_props(p, sb, Pb);
            double ur;
            tface(p, P0, Pb, s0, sb, p.drc[i], p.Ar[i], Frp, &ur);
            if (rec) rec->ur[c0] = ur;
        }
    }
    // ---------------- angular faces (periodic)
    Flux Ftm, Ftp;
    if (Nth > 1) {
        const int jm = (j == 0) ? Nth - 1 : j - 1;
        const int jp = (j == Nth - 1) ? 0 : j + 1;
        Cell sa, sb;
        load_cell(ld, nc, ((int64_t)i * Nth + jm) * Nz + k, sa);
        load_cell(ld, nc, ((int64_t)i * Nth + jp) * Nz + k, sb);
        Props Pa, Pb;
        cell_props(p, sa, Pa);
        cell_props(p, sb, Pb);
        tface(p, Pa, P0, sa, s0, p.arc[i], p.Ath[i], Ftm, nullptr);
        double ut;
        tface(p, P0, Pb, s0, sb, p.arc[i], p.Ath[i], Ftp, &ut);
        if (rec) rec->uth[c0] = ut;
    }
    cell_tail(p, aux, ld, t, i, j, k, P0, rate, qstar, Fzm, Fzp, Frm, Frp, Ftm, Ftp, f, fw, rec);
}

}  // namespace dv
