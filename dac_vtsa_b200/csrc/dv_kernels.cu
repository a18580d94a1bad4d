// dv_kernels.cu -- residual, matvec, diagnostics, accumulator and FD-Jacobian kernels.
// Compiled with -fmad=false (see dv_physics.cuh).
#include "dv_internal.h"
#include "dv_residual.cuh"

#include <algorithm>
#include <mutex>
#include <utility>

namespace dv {

RecLayout rec_layout(const dv_step_params& p) {
    RecLayout r;
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz, nf = (int64_t)p.Nr * p.Nth, nw = (int64_t)p.Nth * p.Nz;
    int64_t o = 0;
    r.T = o; o += nc;
    r.P = o; o += nc;
    r.y = o; o += 3 * nc;
    r.qstar = o; o += 2 * nc;
    r.uz = o; o += nf * (p.Nz - 1);
    r.ur = o; o += (int64_t)(p.Nr - 1) * p.Nth * p.Nz;
    r.uth = o; o += nc;
    r.bnd = o; o += 2 * BR_N * nf;
    r.Qj = o; o += nw;
    r.Qa = o; o += nw;
    r.Qw = o; o += nw;
    r.Rb = o; o += nw;
    r.Qhx = o; o += nc;
    r.total = o;
    return r;
}

static Rec make_rec(const RecLayout& l, double* base) {
    Rec r;
    r.T = base + l.T;
    r.P = base + l.P;
    r.y = base + l.y;
    r.qstar = base + l.qstar;
    r.uz = base + l.uz;
    r.ur = base + l.ur;
    r.uth = base + l.uth;
    r.bnd = base + l.bnd;
    r.Qj = base + l.Qj;
    r.Qa = base + l.Qa;
    r.Qw = base + l.Qw;
    r.Rb = base + l.Rb;
    r.Qhx = base + l.Qhx;
    return r;
}

static __device__ __forceinline__ void cell_ijk(const dv_step_params& p, int64_t c, int& i, int& j, int& k) {
    k = (int)(c % p.Nz);
    int64_t r = c / p.Nz;
    j = (int)(r % p.Nth);
    i = (int)(r / p.Nth);
}

enum { M_RHS = 0, M_STAGE = 1, M_MATVEC = 2 };

// One thread per cell.  MODE selects the epilogue:
//  M_RHS    out = f                                   (core/residual.py:361-365)
//  M_STAGE  out = y - gh f - rhs_known                (core/residual.py:420-423)
//  M_MATVEC out = (v - dh (f(z+sig v) - f0)/sig)/s    (core/solver.py:196-203)
template <int MODE, bool REC>
__global__ void __launch_bounds__(128) k_cells(dv_step_params p, Aux aux, Rec rec, double t, const double* __restrict__ y,
                                               const double* __restrict__ u, const double* __restrict__ sc,
                                               const double* __restrict__ f0, const double* __restrict__ scal,
                                               double gh, double* __restrict__ out) {
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    int i, j, k;
    cell_ijk(p, c, i, j, k);
    double f[DV_NV], fw = 0.0;
    const bool outer_wall = (i == p.Nr - 1) && p.wall_on;
    const int64_t iw = (int64_t)DV_NV * nc + (int64_t)j * p.Nz + k;
    if (MODE == M_MATVEC) {
        const double un = scal[0];
        if (un == 0.0) {            // matvec of a zero direction is zero
#pragma unroll
            for (int v = 0; v < DV_NV; ++v) out[v * nc + c] = 0.0;
            if (outer_wall) out[iw] = 0.0;
            return;
        }
        const double sig = 1.4901161193847656e-08 * scal[1] / un;
        LoadDir ld{y, u, sc, sig};
        cell_eval(p, aux, ld, t, i, j, k, f, outer_wall ? &fw : nullptr, REC ? &rec : nullptr);
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) {
            const int64_t ix = v * nc + c;
            const double vv = u[ix] * sc[ix];
            out[ix] = (vv - gh * (f[v] - f0[ix]) / sig) / sc[ix];
        }
        if (outer_wall) {
            const double vv = u[iw] * sc[iw];
            out[iw] = (vv - gh * (fw - f0[iw]) / sig) / sc[iw];
        }
        return;
    }
    LoadPlain ld{y};
    cell_eval(p, aux, ld, t, i, j, k, f, outer_wall ? &fw : nullptr, REC ? &rec : nullptr);
    if (MODE == M_RHS) {
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) out[v * nc + c] = f[v];
        if (outer_wall) out[iw] = fw;
    } else {
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) {
            const int64_t ix = v * nc + c;
            out[ix] = y[ix] - gh * f[v] - u[ix];
        }
        if (outer_wall) out[iw] = y[iw] - gh * fw - u[iw];
    }
}

// Deterministic block sum (fixed blockDim = 256).
__device__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// The 36 accumulator rates from the end-face and wall records (core/residual.py:371-417).
__global__ void __launch_bounds__(256) k_accumulators(dv_step_params p, const double* __restrict__ rec_bnd,
                                                      const double* __restrict__ Qj, const double* __restrict__ Qa,
                                                      const double* __restrict__ Qw, const double* __restrict__ Qhx,
                                                      double* __restrict__ acc) {
    __shared__ double sh[256];
    const int t = threadIdx.x;
    const int nf = p.Nr * p.Nth, nw = p.Nth * p.Nz;
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz;
    double a[DV_NACC];
    for (int q = 0; q < DV_NACC; ++q) a[q] = 0.0;
    const double ex = (p.gam - 1.0) / p.gam;
    const double pre = p.gam / (p.gam - 1.0) * DV_R;
    for (int e = 0; e < 2; ++e) {
        const dv_end& E = p.ends[e];
        if (E.valve < 0) continue;
        const double* b = rec_bnd + (int64_t)e * BR_N * nf;
        const bool parts = (E.kind == DV_END_VALVE);
        const int base = E.valve * (2 * DV_NG + 4);
        double s_in[DV_NG] = {0, 0, 0}, s_out[DV_NG] = {0, 0, 0}, h_in = 0, h_out = 0, wp = 0, wf = 0;
        for (int f = t; f < nf; f += blockDim.x) {
            const bool inflow = b[BR_UOUT * nf + f] < 0.0;
            double Fin[DV_NG];
            for (int q = 0; q < DV_NG; ++q) {
                Fin[q] = b[(BR_FIN + q) * nf + f];
                s_in[q] += parts ? b[(BR_FINP + q) * nf + f] : (inflow ? Fin[q] : 0.0);
                s_out[q] += parts ? b[(BR_FOUTP + q) * nf + f] : (inflow ? 0.0 : -Fin[q]);
            }
            const double H = b[BR_HIN * nf + f];
            h_in += parts ? b[BR_HINP * nf + f] : (inflow ? H : 0.0);
            h_out += parts ? b[BR_HOUTP * nf + f] : (inflow ? 0.0 : -H);
            const double Pf = b[BR_PFACE * nf + f];
            if (E.is_vacuum) {
                double Fo[DV_NG];
                for (int q = 0; q < DV_NG; ++q) Fo[q] = inflow ? 0.0 : -Fin[q];
                double Ft = p.pump_water ? (Fo[0] + Fo[1] + Fo[2]) : (Fo[0] + Fo[2]);
                double ratio = npmax(p.P_amb / npmax(Pf, 1.0), 1.0);
                double eta = p.eta_vac;
                if (p.vac_krishnamurthy) {
                    double pb = Pf / 1e5;
                    eta = npmax(0.8 * 19.55 * pb / (1.0 + 19.55 * pb), 1e-3);
                }
                wp += pre * b[BR_TLAY * nf + f] * Ft * (pow(ratio, ex) - 1.0) / eta;
            }
            if (E.is_feed) {
                double Ft;
                if (parts) Ft = b[(BR_FINP + 0) * nf + f] + b[(BR_FINP + 1) * nf + f] + b[(BR_FINP + 2) * nf + f];
                else Ft = (inflow ? Fin[0] : 0.0) + (inflow ? Fin[1] : 0.0) + (inflow ? Fin[2] : 0.0);
                double ratio = npmax(Pf / p.P_amb, 1.0);
                wf += pre * E.T_ext * Ft * (pow(ratio, ex) - 1.0) / p.eta_bl;
            }
        }
        for (int q = 0; q < DV_NG; ++q) {
            a[base + q] = block_sum(s_in[q], sh);
            a[base + DV_NG + q] = block_sum(s_out[q], sh);
        }
        a[base + 6] = block_sum(h_in, sh);
        a[base + 7] = block_sum(h_out, sh);
        if (E.is_vacuum) a[base + 8] = block_sum(wp, sh);
        if (E.is_feed) a[base + 9] = block_sum(wf, sh);
    }
    double jp = 0, jn = 0, qa = 0, qw = 0;
    for (int w = t; w < nw; w += blockDim.x) {
        jp += npmax(Qj[w], 0.0);
        jn += npmin(Qj[w], 0.0);
        qa += Qa[w];
        qw += Qw[w];
    }
    a[30] = block_sum(jp, sh);
    a[31] = block_sum(jn, sh);
    a[32] = block_sum(qa, sh);
    a[33] = block_sum(qw, sh);
    if (p.hx_on) {
        double hp = 0, hn = 0;
        for (int64_t c = t; c < nc; c += blockDim.x) {
            hp += npmax(Qhx[c], 0.0);
            hn += npmin(Qhx[c], 0.0);
        }
        a[34] = block_sum(hp, sh);
        a[35] = block_sum(hn, sh);
    }
    if (t == 0)
        for (int q = 0; q < DV_NACC; ++q) acc[q] = a[q];
}

// All colour perturbations of the forward-difference Jacobian in one launch.
// blockIdx.y = slot * 7 + col_var: the perturbed column is unknown `col_var` of neighbour `slot`
// of the row cell.  With a distance-2 colouring every row sees exactly one perturbed column of
// each colour, so evaluating the row cell with that single column perturbed reproduces the
// coloured evaluation of core/jacobian.py:78-84 (colour = colour[column]).
template <class TJ>
__global__ void __launch_bounds__(128) k_fd_jacobian(dv_step_params p, Aux aux, double t, const double* __restrict__ y,
                                                     const double* __restrict__ f0, TJ* __restrict__ J) {
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int slot = blockIdx.y / DV_NB, cv = blockIdx.y % DV_NB;
    int i, j, k;
    cell_ijk(p, c, i, j, k);
    int ni = i, nj = j, nk = k;
    bool ok = true;
    switch (slot) {
        case 0: break;
        case 1: nk = k - 1; ok = nk >= 0; break;
        case 2: nk = k + 1; ok = nk < p.Nz; break;
        case 3: nk = k - 2; ok = nk >= 0; break;
        case 4: nk = k + 2; ok = nk < p.Nz; break;
        case 5: ni = i - 1; ok = ni >= 0; break;
        case 6: ni = i + 1; ok = ni < p.Nr; break;
        case 7: ok = p.Nth > 1; nj = (j == 0) ? p.Nth - 1 : j - 1; break;
        default: ok = p.Nth > 1; nj = (j == p.Nth - 1) ? 0 : j + 1; break;
    }
    if (cv == DV_NV) ok = ok && p.wall_on && (ni == p.Nr - 1);
    TJ* Jb = J + ((int64_t)slot * DV_NB * DV_NB + cv) * nc + c;         // row stride DV_NB*nc
    if (!ok) {
#pragma unroll
        for (int rv = 0; rv < DV_NB; ++rv) Jb[(int64_t)rv * DV_NB * nc] = (TJ)0.0;
        return;
    }
    const int64_t ncell_n = ((int64_t)ni * p.Nth + nj) * p.Nz + nk;
    const int64_t col = (cv < DV_NV) ? (int64_t)cv * nc + ncell_n : (int64_t)DV_NV * nc + (int64_t)nj * p.Nz + nk;
    const double yv = y[col];
    double h = 1.5e-8 * npmax(fabs(yv), p.typ[cv]);
    h = (yv + h) - yv;                                   // core/jacobian.py:75-76
    LoadPert ld{y, col, h};
    double f[DV_NV], fw = 0.0;
    const bool outer_wall = (i == p.Nr - 1) && p.wall_on;
    cell_eval(p, aux, ld, t, i, j, k, f, outer_wall ? &fw : nullptr, (const Rec*)nullptr);
#pragma unroll
    for (int rv = 0; rv < DV_NV; ++rv) Jb[(int64_t)rv * DV_NB * nc] = (TJ)((f[rv] - f0[rv * nc + c]) / h);
    Jb[(int64_t)DV_NV * DV_NB * nc] =
        (TJ)(outer_wall ? (fw - f0[(int64_t)DV_NV * nc + (int64_t)j * p.Nz + k]) / h : 0.0);
}

// ---------------------------------------------------------------- split residual
// The residual as three launches with short per-thread chains: per-cell properties and uptake
// (k_cprops), the flux through every face once (k_faces), per-cell divergence and sources
// (k_assemble, through cell_tail).  Each step evaluates the same expressions on the same inputs
// as cell_eval, so the results are the same bits; the thread-per-cell kernel computes the
// properties of every cell seven times and every face twice.
enum { SP_C0 = 0, SP_T = 3, SP_P, SP_CPOS, SP_Y0, SP_MU = SP_Y0 + 3, SP_KG, SP_RHO, SP_CPM, SP_DM, SP_LAM0,
       SP_RATE0, SP_QS0 = SP_RATE0 + 2, SP_NCELL = SP_QS0 + 2 };

struct Split {
    double* cell;          // [SP_NCELL][nc]
    double* zf;            // [4][ncol (Nz+1)]: +z flux through face kf of a column (kf 0 = top end, Nz = bottom end)
    double* rf;            // [4][(Nr-1) Nth Nz]: +r flux between rings i and i+1 at (j, k)
    double* tf;            // [4][Nr Nth Nz]: +theta flux between sectors j and j+1 (periodic) at (i, k)
    int64_t nc, nzf, nrf, ntf;
};

int64_t split_doubles(const dv_step_params& p) {
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz, ncol = (int64_t)p.Nr * p.Nth;
    return SP_NCELL * nc + 4 * (ncol * (p.Nz + 1) + (int64_t)(p.Nr - 1) * p.Nth * p.Nz + nc);
}

static Split split_of(const dv_step_params& p, double* base) {
    Split S;
    S.nc = (int64_t)p.Nr * p.Nth * p.Nz;
    S.nzf = (int64_t)p.Nr * p.Nth * (p.Nz + 1);
    S.nrf = (int64_t)(p.Nr - 1) * p.Nth * p.Nz;
    S.ntf = S.nc;
    S.cell = base;
    S.zf = S.cell + SP_NCELL * S.nc;
    S.rf = S.zf + 4 * S.nzf;
    S.tf = S.rf + 4 * S.nrf;
    return S;
}

static __device__ __forceinline__ void sp_get(const Split& S, int64_t c, Cell& s, Props& o) {
    const double* a = S.cell;
    const int64_t nc = S.nc;
#pragma unroll
    for (int q = 0; q < DV_NG; ++q) {
        s.c[q] = a[(SP_C0 + q) * nc + c];
        o.y[q] = a[(SP_Y0 + q) * nc + c];
    }
    s.q[0] = s.q[1] = s.e = 0.0;            // not read by the face and wall terms
    o.T = a[SP_T * nc + c];
    o.P = a[SP_P * nc + c];
    o.Tp = 0.0;                             // only the uptake reads it (done in k_cprops)
    o.Cpos = a[SP_CPOS * nc + c];
    o.mu = a[SP_MU * nc + c];
    o.kg = a[SP_KG * nc + c];
    o.rho = a[SP_RHO * nc + c];
    o.cpm = a[SP_CPM * nc + c];
    o.Dm = a[SP_DM * nc + c];
    o.lam0 = a[SP_LAM0 * nc + c];
}

static __device__ __forceinline__ void flux_put(double* base, int64_t stride, int64_t ix, const Flux& F) {
#pragma unroll
    for (int q = 0; q < DV_NG; ++q) base[q * stride + ix] = F.F[q];
    base[DV_NG * stride + ix] = F.H;
}

static __device__ __forceinline__ void flux_get(const double* base, int64_t stride, int64_t ix, Flux& F) {
#pragma unroll
    for (int q = 0; q < DV_NG; ++q) F.F[q] = base[q * stride + ix];
    F.H = base[DV_NG * stride + ix];
}

// Direction scale of the finite-difference matvec: sig = sqrt(eps) ||z|| / ||v|| (core/solver.py:196-203).
static __device__ __forceinline__ double matvec_sig(const double* scal) {
    return 1.4901161193847656e-08 * scal[1] / scal[0];
}

// Two warps per 32 cells: warp 0 evaluates the transport properties of its cells, warp 1 the
// temperature, isotherms and LDF rates of the same cells (the two halves of the per-cell chain run
// side by side; uptake reads only the clipped temperature of the properties).
// The work of one 64-thread block `vb` (cells vb*32 .. vb*32 + 31).  Used by the cooperative FD
// matvec (k_matvec_coop, whose phases share 64-thread blocks); k_cprops runs the eight-warp form
// below, which gives the same bits.
template <int MODE>
__device__ __forceinline__ void cprops_block(const dv_step_params& p, const Split& S, const double* __restrict__ y,
                                             const double* __restrict__ u, const double* __restrict__ sc,
                                             const double* __restrict__ scal, int64_t vb) {
    const int64_t nc = S.nc;
    const int64_t c = vb * 32 + (threadIdx.x & 31);
    const bool half = (threadIdx.x >> 5) != 0;             // warp-uniform
    if (c >= nc) return;
    Cell s;
    if (MODE == M_MATVEC) {
        if (scal[0] == 0.0) return;         // zero direction: k_assemble writes zeros
        LoadDir ld{y, u, sc, matvec_sig(scal)};
        load_cell(ld, nc, c, s);
    } else {
        LoadPlain ld{y};
        load_cell(ld, nc, c, s);
    }
    double* a = S.cell;
    if (!half) {
        Props o;
        cell_props(p, s, o);
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) {
            a[(SP_C0 + q) * nc + c] = s.c[q];
            a[(SP_Y0 + q) * nc + c] = o.y[q];
        }
        a[SP_T * nc + c] = o.T;
        a[SP_P * nc + c] = o.P;
        a[SP_CPOS * nc + c] = o.Cpos;
        a[SP_MU * nc + c] = o.mu;
        a[SP_KG * nc + c] = o.kg;
        a[SP_RHO * nc + c] = o.rho;
        a[SP_CPM * nc + c] = o.cpm;
        a[SP_DM * nc + c] = o.Dm;
        a[SP_LAM0 * nc + c] = o.lam0;
    } else {
        Props o;                            // uptake reads o.Tp only (same expression as cell_props)
        o.Tp = npclip(cell_T(p, s), 150.0, 1500.0);
        double rate[DV_NA], qstar[DV_NA];
        uptake(p, s, o, rate, qstar);
#pragma unroll
        for (int q = 0; q < DV_NA; ++q) {
            a[(SP_RATE0 + q) * nc + c] = rate[q];
            a[(SP_QS0 + q) * nc + c] = qstar[q];
        }
    }
}

// Eight warps per 32 cells.  The transcendental terms of a cell's properties and uptake that do not
// depend on one another (each power is a called routine, so one thread evaluates them strictly one
// after another) are spread over the warps of its block, then combined after one barrier:
//   warp 0: viscosities and the CO2-air Fuller diffusivity     warps 1-3: conductivity of gas 0-2
//   warp 4: the CO2-water Fuller diffusivity                    warp 5: water saturation and GAB loading
//   warp 6: the dry CO2 Toth term                               warp 7: the wet CO2 Toth term (wadst)
// then warp 0 mixes the transport properties and warp 1 finishes the loadings and LDF rates.  Every
// value is the same expression on the same operands as in cell_props / uptake, so the results are
// bit-identical to the one-thread-per-cell evaluation.
#define CP_WARPS 8
static_assert(DV_NG == 3 && CP_WARPS == 8, "the warp roles assume three gases");
template <int MODE>
__device__ __forceinline__ void cprops_split(const dv_step_params& p, const Split& S, const double* __restrict__ y,
                                             const double* __restrict__ u, const double* __restrict__ sc,
                                             const double* __restrict__ scal, int64_t vb) {
    __shared__ double xk[DV_NG][32], xdcw[32], xqw[32], xqd[32], xqwet[32];
    const int64_t nc = S.nc;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t c = vb * 32 + lane;
    const bool in = c < nc;
    if (MODE == M_MATVEC && scal[0] == 0.0) return;    // zero direction (grid-uniform): k_assemble writes zeros
    Cell s;
    if (in) {
        if (MODE == M_MATVEC) {
            LoadDir ld{y, u, sc, matvec_sig(scal)};
            load_cell(ld, nc, c, s);
        } else {
            LoadPlain ld{y};
            load_cell(ld, nc, c, s);
        }
    } else {
        s = Cell{};
    }
    Props o;
    double ycl[DV_NG];
    props_state(p, s, o, ycl);
    const double T = o.Tp, T3 = T / 300.0;
    const double pp = npmax(s.c[0] * DV_R * o.Tp, 0.0);
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    double mu[DV_NG], sq[DV_NG], D_ca = 0.0;
    if (w == 0) {
#pragma unroll
        for (int s2 = 0; s2 < DV_NG; ++s2) {
            mu[s2] = gas_mu(p, s2, T);
            sq[s2] = sqrt(mu[s2]);
        }
        D_ca = fuller(p, 0, T, npmax(o.P, 1.0));
    } else if (w <= DV_NG) {
        xk[w - 1][lane] = gas_k(p, w - 1, T3);
    } else if (w == 4) {
        xdcw[lane] = fuller(p, 1, T, npmax(o.P, 1.0));
    } else if (w == 5) {
        xqw[lane] = q_h2o(p, s.c[1] * DV_R * o.Tp, o.Tp, psat_h2o(o.Tp));
    } else if (w == 6) {
        xqd[lane] = co2_needs_qw(p) ? nan : co2_toth_dry(p, pp, o.Tp);
    } else {
        xqwet[lane] = (p.coads == DV_COADS_WADST) ? co2_toth_wet(p, pp, o.Tp) : nan;
    }
    __syncthreads();
    if (!in || w > 1) return;
    double* a = S.cell;
    if (w == 0) {
        double kk[DV_NG];
#pragma unroll
        for (int s2 = 0; s2 < DV_NG; ++s2) kk[s2] = xk[s2][lane];
        double mu_m, k_m;
        wilke_mix(p, ycl, mu, kk, sq, mu_m, k_m);
        o.mu = mu_m;
        o.kg = k_m;
        o.rho = o.Cpos * wsum3(p.M, ycl);
        o.cpm = wsum3(p.cpg, ycl);
        o.Dm = blanc_Dm(ycl, D_ca, xdcw[lane]);
        o.lam0 = stagnant(p, o.kg);
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) {
            a[(SP_C0 + q) * nc + c] = s.c[q];
            a[(SP_Y0 + q) * nc + c] = o.y[q];
        }
        a[SP_T * nc + c] = o.T;
        a[SP_P * nc + c] = o.P;
        a[SP_CPOS * nc + c] = o.Cpos;
        a[SP_MU * nc + c] = o.mu;
        a[SP_KG * nc + c] = o.kg;
        a[SP_RHO * nc + c] = o.rho;
        a[SP_CPM * nc + c] = o.cpm;
        a[SP_DM * nc + c] = o.Dm;
        a[SP_LAM0 * nc + c] = o.lam0;
    } else {
        double rate[DV_NA], qstar[DV_NA];
        const double qw_eq = xqw[lane];
        const double basis = p.basis_state ? s.q[1] : qw_eq;
        qstar[0] = q_co2_raw(p, pp, o.Tp, basis, xqd[lane], xqwet[lane]) * (pp / (pp + p.p_reg));
        qstar[1] = qw_eq;
        ldf_rates(p, s, o.Tp, qstar, rate);
#pragma unroll
        for (int q = 0; q < DV_NA; ++q) {
            a[(SP_RATE0 + q) * nc + c] = rate[q];
            a[(SP_QS0 + q) * nc + c] = qstar[q];
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(CP_WARPS * 32) k_cprops(dv_step_params p, Split S, const double* __restrict__ y,
                                                          const double* __restrict__ u, const double* __restrict__ sc,
                                                          const double* __restrict__ scal) {
    pdl_wait();                             // (launched programmatically inside the GMRES graph)
    pdl_trigger();
    cprops_split<MODE>(p, S, y, u, sc, scal, blockIdx.x);
}

// MUSCL slope of cell kk of a column starting at cell index base (zero next to the ends).
static __device__ __forceinline__ void sp_slope(const dv_step_params& p, const Split& S, int64_t base, int kk,
                                                bool muscl, double s[4]) {
    s[0] = s[1] = s[2] = s[3] = 0.0;
    if (!muscl || kk < 1 || kk > p.Nz - 2) return;
    const double* a = S.cell;
    const int64_t nc = S.nc, c = base + kk;
#pragma unroll
    for (int q = 0; q < DV_NG; ++q) {
        const double* cq = a + (SP_C0 + q) * nc;
        s[q] = limited_slope(p.limiter, cq[c] - cq[c - 1], cq[c + 1] - cq[c]);
    }
    const double* T = a + SP_T * nc;
    s[3] = limited_slope(p.limiter, T[c] - T[c - 1], T[c + 1] - T[c]);
}

// One thread per face: interior z faces, r faces, theta faces, then the two end faces of every
// column (kept last so the warps of each range run one kind of face).
// The face of index g (all kinds in the order above).
template <bool REC>
__device__ __forceinline__ void faces_at(const dv_step_params& p, const Aux& aux, const Split& S, const Rec& rec,
                                         double t, const double* __restrict__ scal,
                                         const double* __restrict__ dargs, int64_t g) {
    if (scal && scal[0] == 0.0) return;
    if (dargs) t = dargs[0];
    const int Nr = p.Nr, Nth = p.Nth, Nz = p.Nz;
    const int64_t ncol = (int64_t)Nr * Nth;
    const int64_t nzi = ncol * (Nz - 1);
    const int64_t nr = (Nr > 1) ? S.nrf : 0;
    const int64_t nt = (Nth > 1) ? S.ntf : 0;
    if (g < nzi) {
        const int64_t col = g / (Nz - 1);
        const int k = (int)(g % (Nz - 1));
        const int i = (int)(col / Nth);
        const int64_t base = col * Nz;
        const bool muscl = (Nz >= 3 && p.limiter != DV_LIM_UPWIND);
        double sL[4], sR[4];
        sp_slope(p, S, base, k, muscl, sL);
        sp_slope(p, S, base, k + 1, muscl, sR);
        Cell a, b;
        Props L, R;
        sp_get(S, base + k, a, L);
        sp_get(S, base + k + 1, b, R);
        Flux F;
        double uz;
        zface(p, i, L, R, a, b, sL, sR, muscl, aux.n_nom[col], F, &uz);
        flux_put(S.zf, S.nzf, col * (Nz + 1) + k + 1, F);
        if (REC) rec.uz[col * (Nz - 1) + k] = uz;
        return;
    }
    g -= nzi;
    if (g < nr) {                       // between (i, j, k) and (i+1, j, k); g = that first cell's index
        const int i = (int)(g / ((int64_t)Nth * Nz));
        Cell a, b;
        Props A, B;
        sp_get(S, g, a, A);
        sp_get(S, g + (int64_t)Nth * Nz, b, B);
        Flux F;
        double ur;
        tface(p, A, B, a, b, p.drc[i], p.Ar[i], F, &ur);
        flux_put(S.rf, S.nrf, g, F);
        if (REC) rec.ur[g] = ur;
        return;
    }
    g -= nr;
    if (g < nt) {                       // between (i, j, k) and (i, j+1 mod Nth, k); g = the first cell
        const int k = (int)(g % Nz);
        const int64_t r = g / Nz;
        const int j = (int)(r % Nth);
        const int i = (int)(r / Nth);
        const int jp = (j == Nth - 1) ? 0 : j + 1;
        Cell a, b;
        Props A, B;
        sp_get(S, g, a, A);
        sp_get(S, ((int64_t)i * Nth + jp) * Nz + k, b, B);
        Flux F;
        double ut;
        tface(p, A, B, a, b, p.arc[i], p.Ath[i], F, &ut);
        flux_put(S.tf, S.ntf, g, F);
        if (REC) rec.uth[g] = ut;
        return;
    }
    g -= nt;
    if (g < 2 * ncol) {
        const int e = (int)(g / ncol);
        const int64_t col = g % ncol;
        const int i = (int)(col / Nth);
        const int64_t c = col * Nz + (e == 0 ? 0 : Nz - 1);
        Cell s;
        Props o;
        sp_get(S, c, s, o);
        double F_in[DV_NG], H_in;
        end_face(p, p.ends[e], t, i, s, o, aux.feed_flux[col], F_in, H_in,
                 REC ? rec.bnd + (int64_t)e * BR_N * ncol + col : nullptr, ncol);
        Flux F;                           // stored as the +z flux through the face
#pragma unroll
        for (int q = 0; q < DV_NG; ++q) F.F[q] = (e == 0) ? F_in[q] : -F_in[q];
        F.H = (e == 0) ? H_in : -H_in;
        flux_put(S.zf, S.nzf, col * (Nz + 1) + (e == 0 ? 0 : Nz), F);
    }
}

template <bool REC>
__global__ void __launch_bounds__(64) k_faces(dv_step_params p, Aux aux, Split S, Rec rec, double t,
                                              const double* __restrict__ scal, const double* __restrict__ dargs) {
    pdl_wait();
    pdl_trigger();
    faces_at<REC>(p, aux, S, rec, t, scal, dargs, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// The assembly of cell c.
template <int MODE, bool REC>
__device__ __forceinline__ void assemble_at(const dv_step_params& p, const Aux& aux, const Split& S, const Rec& rec,
                                            double t, const double* __restrict__ y, const double* __restrict__ u,
                                            const double* __restrict__ sc, const double* __restrict__ f0,
                                            const double* __restrict__ scal, double gh, double* __restrict__ out,
                                            const double* __restrict__ dargs, int64_t c) {
    const int64_t nc = S.nc;
    if (c >= nc) return;
    if (dargs) {                  // launched from a CUDA graph: time and step factor live on the device
        t = dargs[0];
        gh = dargs[1];
    }
    int i, j, k;
    cell_ijk(p, c, i, j, k);
    const int Nr = p.Nr, Nth = p.Nth, Nz = p.Nz;
    const bool outer_wall = (i == Nr - 1) && p.wall_on;
    const int64_t iw = (int64_t)DV_NV * nc + (int64_t)j * Nz + k;
    if (MODE == M_MATVEC && scal[0] == 0.0) {      // matvec of a zero direction is zero
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) out[v * nc + c] = 0.0;
        if (outer_wall) out[iw] = 0.0;
        return;
    }
    Cell s0;
    Props P0;
    sp_get(S, c, s0, P0);
    double rate[DV_NA], qstar[DV_NA];
#pragma unroll
    for (int q = 0; q < DV_NA; ++q) {
        rate[q] = S.cell[(SP_RATE0 + q) * nc + c];
        qstar[q] = S.cell[(SP_QS0 + q) * nc + c];
    }
    const int64_t col = (int64_t)i * Nth + j;
    Flux Fzm, Fzp, Frm, Frp, Ftm, Ftp;
    flux_get(S.zf, S.nzf, col * (Nz + 1) + k, Fzm);
    flux_get(S.zf, S.nzf, col * (Nz + 1) + k + 1, Fzp);
    if (Nr > 1) {
        if (i > 0) flux_get(S.rf, S.nrf, c - (int64_t)Nth * Nz, Frm);
        if (i < Nr - 1) flux_get(S.rf, S.nrf, c, Frp);
    }
    if (Nth > 1) {
        const int jm = (j == 0) ? Nth - 1 : j - 1;
        flux_get(S.tf, S.ntf, ((int64_t)i * Nth + jm) * Nz + k, Ftm);
        flux_get(S.tf, S.ntf, c, Ftp);
    }
    double f[DV_NV], fw = 0.0;
    if (MODE == M_MATVEC) {
        const double sig = matvec_sig(scal);
        LoadDir ld{y, u, sc, sig};
        cell_tail(p, aux, ld, t, i, j, k, P0, rate, qstar, Fzm, Fzp, Frm, Frp, Ftm, Ftp, f,
                  outer_wall ? &fw : nullptr, REC ? &rec : nullptr);
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) {
            const int64_t ix = v * nc + c;
            const double vv = u[ix] * sc[ix];
            out[ix] = (vv - gh * (f[v] - f0[ix]) / sig) / sc[ix];
        }
        if (outer_wall) {
            const double vv = u[iw] * sc[iw];
            out[iw] = (vv - gh * (fw - f0[iw]) / sig) / sc[iw];
        }
        return;
    }
    LoadPlain ld{y};
    cell_tail(p, aux, ld, t, i, j, k, P0, rate, qstar, Fzm, Fzp, Frm, Frp, Ftm, Ftp, f,
              outer_wall ? &fw : nullptr, REC ? &rec : nullptr);
    if (MODE == M_RHS) {
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) out[v * nc + c] = f[v];
        if (outer_wall) out[iw] = fw;
    } else {
#pragma unroll
        for (int v = 0; v < DV_NV; ++v) {
            const int64_t ix = v * nc + c;
            out[ix] = y[ix] - gh * f[v] - u[ix];
        }
        if (outer_wall) out[iw] = y[iw] - gh * fw - u[iw];
    }
}

template <int MODE, bool REC>
__global__ void __launch_bounds__(64) k_assemble(dv_step_params p, Aux aux, Split S, Rec rec, double t,
                                                 const double* __restrict__ y, const double* __restrict__ u,
                                                 const double* __restrict__ sc, const double* __restrict__ f0,
                                                 const double* __restrict__ scal, double gh,
                                                 double* __restrict__ out, const double* __restrict__ dargs) {
    pdl_wait();
    assemble_at<MODE, REC>(p, aux, S, rec, t, y, u, sc, f0, scal, gh, out, dargs,
                           (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// The FD matvec of the GMRES graph in one cooperative launch: the blocks of k_cprops, k_faces and
// k_assemble (the same per-block / per-index code, in the same 64-thread blocks) taken in grid-
// stride order, the three phases separated by two bounded grid barriers (bar[0..1]; bit 4 of *err
// on a timeout).  Saves two kernel boundaries per Arnoldi step; results are bit-identical.
__global__ void __launch_bounds__(64) k_matvec_coop(dv_step_params p, Aux aux, Split S, Rec rec,
                                                    const double* __restrict__ z, const double* __restrict__ u,
                                                    const double* __restrict__ sc, const double* __restrict__ f0,
                                                    const double* __restrict__ scal, double* __restrict__ out,
                                                    const double* __restrict__ dargs, unsigned* bar, int* err,
                                                    int64_t nb_props, int64_t nb_faces, int64_t nb_cells) {
    for (int64_t vb = blockIdx.x; vb < nb_props; vb += gridDim.x)
        cprops_block<M_MATVEC>(p, S, z, u, sc, scal, vb);
    grid_sync_bounded(bar, bar + 1, err);
    for (int64_t vb = blockIdx.x; vb < nb_faces; vb += gridDim.x)
        faces_at<false>(p, aux, S, rec, 0.0, scal, dargs, vb * 64 + threadIdx.x);
    grid_sync_bounded(bar, bar + 1, err);
    for (int64_t vb = blockIdx.x; vb < nb_cells; vb += gridDim.x)
        assemble_at<M_MATVEC, false>(p, aux, S, rec, 0.0, z, u, sc, f0, scal, 0.0, out, dargs, vb * 64 + threadIdx.x);
}

static Aux aux_of(const dv_model* m) { return Aux{m->aux.feed_flux, m->aux.n_nom, m->aux.cov}; }

static unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// The split residual: properties, faces, assembly (three launches counted under `kind`).
template <int MODE, bool REC>
static int split_residual(dv_model* m, const Rec& rec, double t, const double* y, const double* u, const double* sc,
                          const double* f0, const double* scal, double gh, double* out, cudaStream_t s, int kind) {
    const dv_step_params& p = m->p;
    const Split S = split_of(p, m->d_split);
    const int64_t ncol = (int64_t)p.Nr * p.Nth;
    const int64_t nfaces = ncol * (p.Nz - 1) + (p.Nr > 1 ? S.nrf : 0) + (p.Nth > 1 ? S.ntf : 0) + 2 * ncol;
    DV_LAUNCH(kind, s, k_cprops<MODE><<<nblk(m->nc, 32), CP_WARPS * 32, 0, s>>>(p, S, y, u, sc, scal));
    DV_LAUNCH(kind, s, k_faces<REC><<<nblk(nfaces, 64), 64, 0, s>>>(p, aux_of(m), S, rec, t,
                                                                  MODE == M_MATVEC ? scal : nullptr, nullptr));
    DV_LAUNCH(kind, s, k_assemble<MODE, REC><<<nblk(m->nc, 64), 64, 0, s>>>(p, aux_of(m), S, rec, t, y, u, sc, f0,
                                                                           scal, gh, out, nullptr));
    m->nfev += 1;
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

int launch_rhs(dv_model* m, double t, const double* y, double* f, double* acc, cudaStream_t s) {
    Rec rec = make_rec(m->rl, m->d_rec);
    if (acc) {
        int rc = split_residual<M_RHS, true>(m, rec, t, y, nullptr, nullptr, nullptr, nullptr, 0.0, f, s,
                                             dv::K_RESIDUAL);
        if (rc != DV_OK) return rc;
        DV_LAUNCH(dv::K_RESIDUAL, s, k_accumulators<<<1, 256, 0, s>>>(m->p, rec.bnd, rec.Qj, rec.Qa, rec.Qw, rec.Qhx, acc));
        DV_CUDA(cudaGetLastError());
        return DV_OK;
    }
    return split_residual<M_RHS, false>(m, rec, t, y, nullptr, nullptr, nullptr, nullptr, 0.0, f, s, dv::K_RESIDUAL);
}

int launch_stage_residual(dv_model* m, double t, const double* y, double gamma_h, const double* rhs_known,
                          double* R, cudaStream_t s) {
    Rec rec = make_rec(m->rl, m->d_rec);
    return split_residual<M_STAGE, false>(m, rec, t, y, rhs_known, nullptr, nullptr, nullptr, gamma_h, R, s,
                                          dv::K_RESIDUAL);
}

int launch_diag(dv_model* m, double t, const double* y, double* diag, cudaStream_t s) {
    Rec rec = make_rec(m->rl, diag);      // f is discarded into the model's record scratch
    return split_residual<M_RHS, true>(m, rec, t, y, nullptr, nullptr, nullptr, nullptr, 0.0, m->d_rec, s,
                                       dv::K_RESIDUAL);
}

int launch_matvec(dv_model* m, double t, const double* z, const double* u, const double* sc, const double* f0,
                  double dh, const double* scal, double* out, cudaStream_t s) {
    Rec rec = make_rec(m->rl, m->d_rec);
    return split_residual<M_MATVEC, false>(m, rec, t, z, u, sc, f0, scal, dh, out, s, dv::K_MATVEC);
}

// Launch with programmatic stream serialisation (the kernel must begin with pdl_wait()).
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// co-resident 64-thread blocks of k_matvec_coop (-1: not asked yet; 0: refused)
static int g_matvec_coop_cap = -1;

// DVTSA_MATVEC_COOP=1 runs the FD matvec inside the GMRES graph as one cooperative launch (read
// once; off by default: bit-identical, but measured 5 % slower on the 8x8x32 heating window, the
// two grid barriers costing more than the two kernel boundaries they replace).
static bool matvec_coop_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_MATVEC_COOP");
        v = (e && e[0] == '1') ? 1 : 0;
    }
    return v == 1;
}

int matvec_capture_kernels() { return (g_matvec_coop_cap > 0 && matvec_coop_enabled()) ? 1 : 3; }

int matvec_capture(dv_model* m, const double* dargs, const double* z, const double* u, const double* sc,
                   const double* f0, const double* scal, double* out, cudaStream_t s, unsigned* bar) {
    const dv_step_params& p = m->p;
    const Split S = split_of(p, m->d_split);
    const Rec rec = make_rec(m->rl, m->d_rec);
    const int64_t ncol = (int64_t)p.Nr * p.Nth;
    const int64_t nfaces = ncol * (p.Nz - 1) + (p.Nr > 1 ? S.nrf : 0) + (p.Nth > 1 ? S.ntf : 0) + 2 * ncol;
    int& coop_cap = g_matvec_coop_cap;
    if (coop_cap < 0) {
        int dev = 0, nsm = 0, bps = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_matvec_coop, 64, 0) != cudaSuccess) bps = 0;
        coop_cap = bps * nsm;
        cudaGetLastError();
    }
    if (bar && coop_cap > 0 && matvec_coop_enabled()) {
        const int64_t nbp = nblk(m->nc, 32), nbf = nblk(nfaces, 64), nbc = nblk(m->nc, 64);
        const int64_t want = std::max(nbp, std::max(nbf, nbc));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)std::min<int64_t>(want, coop_cap));
        cfg.blockDim = dim3(64);
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaLaunchKernelEx(&cfg, k_matvec_coop, p, aux_of(m), S, rec, z, u, sc, f0, scal, out, dargs, bar,
                               m->d_err, nbp, nbf, nbc) == cudaSuccess)
            return DV_OK;
        cudaGetLastError();                   // a driver that refuses the cooperative node: three kernels
        coop_cap = 0;
    }
    if (pdl_enabled()) {       // each kernel may start while its predecessor drains (pdl_wait in the kernel)
        DV_CUDA(launch_pdl(k_cprops<M_MATVEC>, nblk(m->nc, 32), CP_WARPS * 32, s, p, S, z, u, sc, scal));
        DV_CUDA(launch_pdl(k_faces<false>, nblk(nfaces, 64), 64, s, p, aux_of(m), S, rec, 0.0, scal, dargs));
        DV_CUDA(launch_pdl(k_assemble<M_MATVEC, false>, nblk(m->nc, 64), 64, s, p, aux_of(m), S, rec, 0.0, z, u, sc, f0,
                           scal, 0.0, out, dargs));
        return DV_OK;
    }
    k_cprops<M_MATVEC><<<nblk(m->nc, 32), CP_WARPS * 32, 0, s>>>(p, S, z, u, sc, scal);
    k_faces<false><<<nblk(nfaces, 64), 64, 0, s>>>(p, aux_of(m), S, rec, 0.0, scal, dargs);
    k_assemble<M_MATVEC, false><<<nblk(m->nc, 64), 64, 0, s>>>(p, aux_of(m), S, rec, 0.0, z, u, sc, f0, scal, 0.0,
                                                             out, dargs);
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

static int fdjac_block(const dv_model* m) { return m->tune.fdjac_block == 64 ? 64 : 128; }

int launch_fd_jacobian(dv_model* m, double t, const double* y, const double* f0, double* J, cudaStream_t s) {
    const int bl = fdjac_block(m);
    dim3 grid(nblk(m->nc, bl), DV_NSLOT * DV_NB);
    DV_LAUNCH(dv::K_FDJAC, s, k_fd_jacobian<double><<<grid, bl, 0, s>>>(m->p, aux_of(m), t, y, f0, J));
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

int launch_fd_jacobian32(dv_model* m, double t, const double* y, const double* f0, float* J, cudaStream_t s) {
    const int bl = fdjac_block(m);
    dim3 grid(nblk(m->nc, bl), DV_NSLOT * DV_NB);
    DV_LAUNCH(dv::K_FDJAC, s, k_fd_jacobian<float><<<grid, bl, 0, s>>>(m->p, aux_of(m), t, y, f0, J));
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

// ---------------------------------------------------------------- outlet record
// The summary of one accepted step that the step runner records (the columns of the outlet time
// series, steps/_runner.py:50-84,104-121), reduced on the device from the diagnostics record so that
// only DV_OUTLET_N doubles leave the GPU per step.  Per end: the net outflow (minus the summed inflow
// records), the area-weighted face pressure, and the composition and temperature of the gas leaving
// (weighted by each face's outflow, over the faces with outflow; valve ends use their outflow part)
// or, with no outflow, the area-weighted layer averages.  Fixed-order block reductions.
constexpr int OUTLET_THREADS = 256;

__device__ double outlet_sum(double v, double* red) {
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int st = OUTLET_THREADS / 2; st > 0; st >>= 1) {
        if (tid < st) red[tid] += red[tid + st];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(OUTLET_THREADS) k_outlet(dv_step_params p, Rec rec, const double* __restrict__ y,
                                                           double c_feed, double* __restrict__ out) {
    __shared__ double red[OUTLET_THREADS];
    const int tid = threadIdx.x;
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz;
    const int nf = p.Nr * p.Nth;
    double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};          // V T, V P, V q_CO2, V q_H2O, V
    for (int64_t c = tid; c < nc; c += OUTLET_THREADS) {
        const double V = p.V[c / ((int64_t)p.Nth * p.Nz)];
        a[0] += rec.T[c] * V;
        a[1] += rec.P[c] * V;
        a[2] += y[3 * nc + c] * V;
        a[3] += y[4 * nc + c] * V;
        a[4] += V;
    }
    double bed[5];
    for (int q = 0; q < 5; ++q) bed[q] = outlet_sum(a[q], red);
    if (tid == 0) {
        out[24] = bed[0] / bed[4];
        out[25] = bed[1] / bed[4];
        out[26] = bed[2] / bed[4];
        out[27] = bed[3] / bed[4];
    }
    for (int e = 0; e < 2; ++e) {
        const int klay = e == 0 ? 0 : p.Nz - 1;
        const double* b = rec.bnd + (int64_t)e * BR_N * nf;
        const bool part = p.ends[e].kind == DV_END_VALVE;
        // A, P A, net outflow, leaving flow, leaving species (3), T leaving flow, y A (3), T A,
        // net outflow and its CO2 over the faces with net outflow, loading q_CO2 of the layer
        double sm[15];
        for (int q = 0; q < 15; ++q) sm[q] = 0.0;
        for (int f = tid; f < nf; f += OUTLET_THREADS) {
            const double A = p.Az[f / p.Nth];
            const int64_t cell = (int64_t)f * p.Nz + klay;
            double Fo[DV_NG], tot = 0.0, tot2 = 0.0;
            for (int k = 0; k < DV_NG; ++k) tot += -b[(BR_FIN + k) * nf + f];
            for (int k = 0; k < DV_NG; ++k) {
                Fo[k] = part ? b[(BR_FOUTP + k) * nf + f] : -b[(BR_FIN + k) * nf + f];
                tot2 += Fo[k];
            }
            const bool leaving = tot2 > 0.0;
            const double Tl = rec.T[cell];
            sm[0] += A;
            sm[1] += b[BR_PFACE * nf + f] * A;
            sm[2] += tot;
            if (leaving) {
                sm[3] += tot2;
                for (int k = 0; k < DV_NG; ++k) sm[4 + k] += Fo[k];
                sm[7] += Tl * tot2;
            }
            for (int k = 0; k < DV_NG; ++k) sm[8 + k] += rec.y[(int64_t)k * nc + cell] * A;
            sm[11] += Tl * A;
            if (tot > 0.0) {
                sm[12] += tot;
                sm[13] += -b[BR_FIN * nf + f];
            }
            sm[14] += y[(int64_t)DV_NG * nc + cell];
        }
        double r[15];
        for (int q = 0; q < 15; ++q) r[q] = outlet_sum(sm[q], red);
        if (tid == 0) {
            double* o = out + 12 * e;
            const double Pf = r[1] / r[0];
            double ys[DV_NG], Tg;
            if (r[3] > 1e-14) {
                for (int k = 0; k < DV_NG; ++k) ys[k] = r[4 + k] / r[3];
                Tg = r[7] / r[3];
            } else {
                for (int k = 0; k < DV_NG; ++k) ys[k] = r[8 + k] / r[0];
                Tg = r[11] / r[0];
            }
            o[0] = r[2];
            o[1] = Pf;
            o[2] = Tg;
            for (int k = 0; k < DV_NG; ++k) o[3 + k] = ys[k];
            const double cco2 = ys[0] * Pf / (DV_R * Tg);
            o[6] = cco2;
            o[7] = c_feed > 0.0 ? cco2 / c_feed : __longlong_as_double(0x7ff8000000000000LL);
            o[8] = r[3];
            o[9] = r[12] > 0.0 ? r[13] / r[12] : 0.0;
            o[10] = r[14] / nf;
            o[11] = 0.0;
        }
    }
    if (tid == 0)
        for (int q = 28; q < DV_OUTLET_N; ++q) out[q] = 0.0;
}

int launch_outlet(dv_model* m, double t, const double* y, double c_feed, double* row, cudaStream_t s) {
    DV_TRY(launch_diag(m, t, y, m->d_diag, s));
    Rec rec = make_rec(m->rl, m->d_diag);
    DV_LAUNCH(dv::K_RESIDUAL, s, k_outlet<<<1, OUTLET_THREADS, 0, s>>>(m->p, rec, y, c_feed, row));
    return launch_ok("k_outlet");
}

}  // namespace dv

// ---------------------------------------------------------------- allocation-free residual + accumulators
// dv_rhs_acc_noalloc evaluates f = dy/dt and the accumulator rates without a dv_model, so without
// any device allocation.  It exists for callers that may not allocate device memory once they are
// running: a plant controller or state estimator that reserves its device memory at start-up and
// forbids allocation inside its loop, or a host framework whose allocator owns the device and
// does not let plugins call cudaMalloc.  dv_model_create allocates the model's workspaces, so
// those callers cannot use dv_rhs.  The face and wall records that dv_rhs keeps in the model live
// here in one file-scope device array instead, shared by every call on the device.

namespace {

constexpr size_t kNoAllocScratchBytes = 2u << 20;    // 2 MiB per device, held until process exit
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

// Device address of g_noalloc_scratch per device, looked up once with that device current (in
// host code the symbol names a host-side shadow, never a device address).
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
static std::mutex g_noalloc_mu;

}  // namespace

extern "C" int dv_rhs_acc_noalloc(const dv_step_params* p, const double* feed_flux, const double* n_nom,
                                  const double* coverage, double t, const double* y, double* f, double* acc,
                                  void* stream) {
    using namespace dv;
    if (!p || !feed_flux || !n_nom || !coverage || !y || !f || !acc) {
        set_error("dv_rhs_acc_noalloc: null argument");
        return DV_ERR_ARG;
    }
    if (p->Nr < 1 || p->Nth < 1 || p->Nz < 1 || p->Nr > DV_MAX_NR) {
        set_error("dv_rhs_acc_noalloc: bad grid size");
        return DV_ERR_ARG;
    }
    const RecLayout rl = rec_layout(*p);
    const size_t need = sizeof(double) * (size_t)rl.total;
    if (need > kNoAllocScratchBytes) {
        set_error("dv_rhs_acc_noalloc: the grid needs " + std::to_string(need) + " bytes of record scratch; the "
                  "static scratch holds " + std::to_string(kNoAllocScratchBytes) + " (use dv_model_create + dv_rhs)");
        return DV_ERR_ARG;
    }
    int dev = 0;
    DV_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("dv_rhs_acc_noalloc: device index out of range");
        return DV_ERR_ARG;
    }
    double* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {                   // first call on this device: look up the address
            void* ptr = nullptr;
            DV_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
            g_noalloc_ptr[dev] = (double*)ptr;
        }
        base = g_noalloc_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    // The array keeps the previous call's records; records that this grid and step never write
    // (ends without a valve, the wall of a wall-less column) must read as zero.
    DV_CUDA(cudaMemsetAsync(base, 0, need, s));
    Rec rec = make_rec(rl, base);
    const int64_t nc = (int64_t)p->Nr * p->Nth * p->Nz;
    count_launch(K_RESIDUAL);
    k_cells<M_RHS, true><<<nblk(nc, 128), 128, 0, s>>>(*p, Aux{feed_flux, n_nom, coverage}, rec, t, y, nullptr,
                                                      nullptr, nullptr, nullptr, 0.0, f);
    count_launch(K_RESIDUAL);
    k_accumulators<<<1, 256, 0, s>>>(*p, rec.bnd, rec.Qj, rec.Qa, rec.Qw, rec.Qhx, acc);
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}
