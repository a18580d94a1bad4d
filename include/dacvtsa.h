/*
 * dacvtsa.h -- C ABI of the B200 implicit stepping path of the dac_vtsa TVSA simulator.
 *
 * The reference (Navneet07rkt/dac_vtsa) is pure Python; its "plugin interface" for this path
 * is the object protocol the step runner drives (steps/_runner.py:87-153):
 *   TVSAModel (core/residual.py:40-482)  -> dv_model_* , dv_rhs, dv_stage_residual, dv_rhs_diag
 *   FDJacobian (core/jacobian.py:21-91), color_columns (numerics/sparsity.py:88-107)
 *                                        -> dv_colour_columns, dv_fd_jacobian
 *   TRBDF2._factor / splu (core/solver.py:334-337)
 *                                        -> dv_precond_factor, dv_precond_solve, dv_precond_partitions
 *   newton_krylov (core/solver.py:154-294) -> dv_newton_stage
 *   TRBDF2.integrate (core/solver.py:370-511) -> dv_integrator_*
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Plain C types only.  Vectors are DEVICE pointers (FP64) unless stated; `stream` is a
 *    cudaStream_t passed as void* (NULL = legacy default stream).  Calls are asynchronous on
 *    `stream` unless they return host values (documented per call).
 *  - State layout (variable-major, core/residual.py:110-118):
 *      y = [c_CO2 | c_H2O | c_N2 | q_CO2 | q_H2O | e | Tw]
 *    each cell block ncell long in C order (i_r*Ntheta + j_theta)*Nz + k_z, then Tw over
 *    (Ntheta, Nz).  n_core = 6*ncell + Ntheta*Nz (wall enabled) or 6*ncell.
 *  - Return value: 0 = success; < 0 = error (dv_last_error() gives the message):
 *      DV_ERR_ARG (-1) bad argument / size, DV_ERR_CUDA (-2) CUDA runtime error,
 *      DV_ERR_UNSUPPORTED (-3) configuration without a GPU implementation,
 *      DV_ERR_STEPS (-10) too many steps (reference: SolverError "too many steps"),
 *      DV_ERR_UNDERFLOW (-11) step size underflow (reference: SolverError "step size underflow").
 *  - Handles are not thread-safe (the reference model/integrator are not either); one handle
 *    per thread.  No entry point allocates device memory except *_create.
 */
#ifndef DACVTSA_H
#define DACVTSA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DV_ABI_VERSION 1
#define DV_MAX_NR 64          /* radial rings supported by the per-ring parameter arrays      */
#define DV_NG 3               /* gas species CO2, H2O, N2 (components.water = true)            */
#define DV_NA 2               /* adsorbed species CO2, H2O                                     */
#define DV_NV 6               /* unknowns per cell: 3 c, 2 q, e                                */
#define DV_NACC 36            /* accumulator rates (core/residual.py:126-133)                  */
#define DV_NSLOT 9            /* Jacobian neighbour slots: self, z-1, z+1, z-2, z+2, r-1, r+1, th-1, th+1 */
#define DV_NB 7               /* Jacobian block size: 6 cell unknowns + the wall unknown of the cell  */

#define DV_OK 0
#define DV_ERR_ARG (-1)
#define DV_ERR_CUDA (-2)
#define DV_ERR_UNSUPPORTED (-3)
#define DV_ERR_STEPS (-10)
#define DV_ERR_UNDERFLOW (-11)

enum dv_end_kind { DV_END_CLOSED = 0, DV_END_FEED = 1, DV_END_PUMP = 2, DV_END_VALVE = 3, DV_END_PRESSURE = 4 };
enum dv_limiter { DV_LIM_VAN_ALBADA = 0, DV_LIM_VAN_ALBADA_TVD = 1, DV_LIM_VAN_LEER = 2, DV_LIM_MINMOD = 3,
                  DV_LIM_UPWIND = 4 };
enum dv_coads { DV_COADS_NONE = 0, DV_COADS_WADST = 1, DV_COADS_MECHANISTIC = 2, DV_COADS_STAMPI = 3 };
enum dv_disp { DV_DISP_EDWARDS_RICHARDSON = 0, DV_DISP_YOUNG2021 = 1, DV_DISP_WAKAO_KAGEI = 2 };
enum dv_bedcond { DV_BED_ZEHNER_SCHLUNDER = 0, DV_BED_PARALLEL = 1, DV_BED_CONSTANT = 2 };
enum dv_wallhtc { DV_HTC_MARTIN_NILLES = 0, DV_HTC_CONSTANT = 1 };

/* One column end for one cycle step (valves/valve_logic.py:48-109, boundaries/conditions.py:75-160). */
typedef struct dv_end {
    int32_t kind;            /* dv_end_kind */
    int32_t valve;           /* 0,1,2 = V1,V2,V3 open at this end; -1 = none */
    int32_t check_valve, is_vacuum, is_feed, pad_;
    double P_target, T_ext, speed, P_start;   /* P_start: mean layer pressure at step start */
    double y_ext[DV_NG];
} dv_end;

/* Per-step constants of the residual (everything TVSAModel.__init__ derives, core/residual.py:41-123). */
typedef struct dv_step_params {
    int32_t Nr, Nth, Nz, wall_on;
    /* geometry (core/grid.py:61-96); per-ring arrays have Nr entries, per-r-face arrays Nr-1 */
    double dz, dth, half_dr_outer, A_wall_in, A_wall_out, wall_C, wall_kz, wall_kt;
    double Az[DV_MAX_NR], V[DV_MAX_NR], Ath[DV_MAX_NR], arc[DV_MAX_NR], Ar[DV_MAX_NR], drc[DV_MAX_NR];
    /* sorbent + thermodynamics (physics/energy.py:31-52) */
    double eps_b, eps_t, rho_b, cp_s, dp, T_ref;
    double cpg[DV_NG], cpa[DV_NA], dH[DV_NA];
    /* gas data (properties/ideal_gas_backend.py): mu_s = sum_t mu_w*(mu_D*T + mu_E);
       k_s = sum_t k_w*k_0*(T/300)^k_n ; nt = number of terms (air = N2/O2 blend) */
    double M[DV_NG];
    double mu_w[DV_NG][2], mu_D[DV_NG][2], mu_E[DV_NG][2];
    double k_w[DV_NG][2], k_0[DV_NG][2], k_n[DV_NG][2];
    int32_t mu_nt[DV_NG], k_nt[DV_NG];
    double mass_q[DV_NG][DV_NG], wilke_den[DV_NG][DV_NG];
    double fuller_sqrtM[2], fuller_s[2];       /* pairs CO2-AIR, CO2-H2O (utils/diffusion.py:19-26) */
    /* isotherms (physics/isotherms.py) */
    double co2_q_inf0, co2_chi, co2_b0, co2_dH0, co2_tau0, co2_alpha, co2_T0, p_reg;
    double h2o_q_m, h2o_C, h2o_D, h2o_F, h2o_G, h2o_E10_slope, h2o_E10_intercept, rh_cap;
    double wadst_b0, wadst_q_inf0, wadst_tau0, wadst_chi, wadst_alpha, wadst_dH, wadst_A;
    double mech_f_blocked_max, mech_k, mech_phi_dry, mech_A, mech_dH_wet, mech_n;
    double sb_gamma, sb_beta;
    int32_t coads, basis_state;
    /* LDF kinetics (physics/kinetics.py) */
    double k_ldf[DV_NA], Ea[DV_NA], T_ref_kin;
    int32_t ea_zero;
    /* transport (physics/pressure.py, dispersion.py, heat_transfer.py) */
    int32_t disp_model, bed_model, htc_model, lumped;
    double ka, kb, g1, g2, er_beta, Pe_T, lam_const, zs_B, zs_s, lam_s, Pe_r, Pe_z, alpha_const, N_ratio, U_lumped;
    double u_nom;
    int32_t limiter, pad0_;
    /* ends 0 = top (z = 0), 1 = bottom (z = L) */
    dv_end ends[2];
    double tau_valve;
    /* jacket, wall, exchanger (core/residual.py:87-100,328-359) */
    int32_t jacket_on, hx_on;
    double T_jac_set, T_jac_prev, jac_tau, h_jac, h_amb, T_amb, P_amb, hA_v;
    /* energy accounting (core/residual.py:102-108,395-409) */
    double gam, eta_vac, eta_bl;
    int32_t vac_krishnamurthy, pump_water;
    /* solver constants per variable block (core/residual.py:135-144, core/jacobian.py:39-48);
       index 0..5 = cell unknowns, 6 = wall */
    double atol[DV_NB], typ[DV_NB];
} dv_step_params;

typedef struct dv_model dv_model;
typedef struct dv_integrator dv_integrator;

/* ------------------------------------------------------------------ library */
int dv_abi_version(void);
size_t dv_step_params_size(void);
/* sizeof of the ABI's other structs, by name ("dv_newton_opts", "dv_newton_result", "dv_solver_opts",
 * "dv_step_report", "dv_tuning"); 0 for an unknown name.  Lets a binding check its mirrors. */
size_t dv_struct_size(const char* name);
/* No reference counterpart.  The device and pinned host memory of destroyed models and integrators
 * is kept by the library and handed to the next handle of the same sizes (the reference creates one
 * model and one integrator per cycle step).  dv_pool_cached_bytes: bytes kept now; dv_pool_release:
 * frees them all (handles alive are not affected). */
int64_t dv_pool_cached_bytes(void);
int dv_pool_release(void);
const char* dv_last_error(void);
int dv_device_count(int* n);

/* Launch accounting (no reference counterpart; instrumentation of this library).  Every kernel launch
 * is counted per kind: 0 residual (rhs / stage residual / diagnostics / accumulators), 1 finite-
 * difference matvec residual, 2 FD Jacobian, 3 preconditioner assembly + factorisation,
 * 4 preconditioner sweep, 5 vector / reduction kernels, 6 learned-predictor network kernels,
 * 7 assembled-Jacobian (mixed-precision) operator kernels.  With profiling enabled each launch is also
 * bracketed by CUDA events on its own stream; dv_profile_read synchronises the device and returns the
 * launches, the timed launches and their summed device time [ms].  dv_profile_enable resets. */
int dv_profile_enable(int32_t on);
int dv_profile_read(int32_t kind, int64_t* launches, int64_t* timed, double* total_ms);
int64_t dv_launch_count(void);

/* ------------------------------------------------------------------ model
 * Replaces TVSAModel.__init__ (core/residual.py:41-123).  Host inputs: feed_flux and n_nom over
 * (Nr, Ntheta) [mol/s per inlet face; mol/m2/s nominal column flux, zeros without feed],
 * coverage over (Ntheta, Nz).  Allocates all device workspaces of the model. */
int dv_model_create(const dv_step_params* p, const double* feed_flux, const double* n_nom,
                    const double* coverage, dv_model** out);
int dv_model_destroy(dv_model* m);
/* host values: n_core, ncell, wall unknowns, Jacobian block doubles, diagnostics doubles */
int dv_model_sizes(const dv_model* m, int64_t* n_core, int64_t* ncell, int64_t* n_wall,
                   int64_t* jac_doubles, int64_t* diag_doubles);
/* host value: right-hand-side evaluations issued so far (TVSAModel.nfev, core/residual.py:123,213) */
int64_t dv_model_nfev(const dv_model* m);

/* f = dy/dt (TVSAModel.rhs, core/residual.py:211-365); acc (36 accumulator rates,
 * core/residual.py:371-417) is written when non-NULL. */
int dv_rhs(dv_model* m, double t, const double* y, double* f, double* acc, void* stream);
/* R = y - gamma_h f(t, y) - rhs_known (TVSAModel.stage_residual, core/residual.py:420-423) */
int dv_stage_residual(dv_model* m, double t, const double* y, double gamma_h, const double* rhs_known,
                      double* R, void* stream);
/* Diagnostics of TVSAModel.rhs(diag=True) (core/residual.py:366-368) into `diag` (diag_doubles):
 * T, P [ncell]; y [3 ncell]; qstar [2 ncell]; uz [Nr Nth (Nz-1)]; ur [(Nr-1) Nth Nz]; uth [ncell];
 * boundary records [2 ends][16][Nr Nth] = F_in(3) H_in u_out P_face F_inpart(3) F_outpart(3)
 * H_inpart H_outpart T_layer 0; Q_jac, Q_amb, Q_wb, R_bed [Nth Nz]; Q_hx [ncell]. */
int dv_rhs_diag(dv_model* m, double t, const double* y, double* diag, void* stream);

/* Outlet summary of one state (the quantities the reference's runner records after every accepted
 * step, steps/_runner.py:50-84,104-121), reduced on the device from the diagnostics of t, y into
 * `row` (DEVICE, DV_OUTLET_N doubles): per end e (top 0, bottom 1) at row[12 e + ...]: 0 net outflow
 * [mol/s], 1 area-weighted face pressure [Pa], 2 temperature of the leaving gas [K], 3..5 its mole
 * fractions, 6 its CO2 concentration [mol/m3], 7 that over c_feed_co2 (NaN if c_feed_co2 <= 0),
 * 8 the leaving flow, 9 the CO2 fraction of the net outflow over the faces with net outflow (0 when
 * none), 10 the mean q_CO2 of the end layer; row[24..27] volume means of T, P, q_CO2, q_H2O.  These
 * also give the stop criteria of core/residual.py:445-469.  Asynchronous on `stream`. */
#define DV_OUTLET_N 32
int dv_outlet_row(dv_model* m, double t, const double* y, double c_feed_co2, double* row, void* stream);

/* ------------------------------------------------------------------ Jacobian
 * Greedy distance-2 column colouring of the stencil pattern, bit-identical to
 * color_columns(build_pattern(...)) (numerics/sparsity.py:29-107).  Host call; colour has
 * n_core entries. */
int dv_colour_columns(int32_t Nr, int32_t Nth, int32_t Nz, int32_t wall, int64_t* colour, int32_t* ncolours);
/* Forward-difference Jacobian df/dy at (t, y) with f0 = f(t, y) (FDJacobian.__call__,
 * core/jacobian.py:71-86): every colour perturbation in one launch.  J is the block layout
 * J[slot][row 0..6][col 0..6][cell] (jac_doubles): d f_row(cell) / d y_col(neighbour `slot`),
 * row/col 6 = the wall unknown of an outer-ring cell.  Same step rule h = 1.5e-8 max(|y|, typ). */
int dv_fd_jacobian(dv_model* m, double t, const double* y, const double* f0, double* J, void* stream);

/* ------------------------------------------------------------------ preconditioner
 * Factorise M = I - dh J restricted to partitions of the cross-section as a block-pentadiagonal
 * LU along z (replaces splu of TRBDF2._factor, core/solver.py:334-337).  mode 0 = theta sectors
 * (all rings of a sector + its wall), 1 = whole cross-sections, 2 = the innermost ring of all
 * sectors as one partition and rings 1.. of each sector (+ wall) as the others (keeps the inner
 * ring's theta coupling, as the reference's theta_block keeps its innermost rings'; falls back to
 * mode 0 below 2 rings or 2 sectors).  Stored in the model. */
int dv_precond_factor(dv_model* m, const double* J, double dh, int32_t mode, void* stream);
/* Mixed-precision Krylov (no reference counterpart), a mask:
 *  DV_KRYLOV_FP32_FACTORS   the factorisation also stores an FP32 copy of its blocks, which
 *                           dv_precond_solve, GMRES and the Newton step stream (sums stay FP64);
 *                           takes effect at the next dv_precond_factor;
 *  DV_KRYLOV_FP32_OPERATOR  GMRES's operator is the assembled Jacobian in FP32 (products and sums in
 *                           FP32) instead of the FP64 finite-difference matvec (core/solver.py:196-
 *                           203); the integrator refreshes that Jacobian at the start of every step
 *                           (and with every in-stage refresh), dv_newton_stage at its z0.
 * The residual, the Jacobian's differencing, the Newton update, the line search and the balances stay
 * FP64: each Newton iteration is an FP64 refinement of the FP32 Krylov solution, and the unchanged
 * FP64 convergence test decides. */
#define DV_KRYLOV_FP32_FACTORS 1
#define DV_KRYLOV_FP32_OPERATOR 2
int dv_model_set_krylov_fp32(dv_model* m, int32_t mask);
/* Layout of the stored factors (no reference counterpart; for accounting): partition mode (3 = the
 * split form mode 2 takes when a sector or the core ring exceeds the shared-memory kernels: rings
 * 1.. of each sector in groups of at most 48 unknowns, the wall node with the outer group, and the
 * core ring in theta groups), the first twisted separator plane (0: one direction), and each
 * partition's block size (up to cap entries).  Host call. */
int dv_precond_partitions(const dv_model* m, int32_t* mode, int32_t* zs, int32_t* nb, int32_t cap, int32_t* nparts);
/* Host self-check of the partition maps the factorisation and sweep use for grid p in `mode` (no
 * reference counterpart; no device work): *violations counts unknowns not covered exactly once,
 * indices outside the state and disagreements between the forward and inverse maps. */
int dv_precond_check_maps(const dv_step_params* p, int32_t mode, int32_t* nparts, int32_t* nb, int64_t* violations);
/* x = M^-1 b with the stored factors (lu.solve). b and x may alias. */
int dv_precond_solve(dv_model* m, const double* b, double* x, void* stream);

/* ------------------------------------------------------------------ stage solve */
typedef struct dv_newton_opts {
    int32_t max_iter, krylov_dim, allow_refresh, precond_mode;
    double kappa, eta, rtol, cons_tol;
    int32_t max_polish;        /* conservation-polish iterations after convergence (reference: 2; 0 = 2) */
    int32_t polish_cycles;     /* GMRES restart cycles of one polish iteration's linear solve, stopping at its
                                  tolerance (reference: 1, scipy gmres maxiter=1; 0 = 1; at most 8) */
    int32_t balance_projection;   /* 1: a converged stage whose balances are not closed is first corrected
                                     by the balance projection (no reference counterpart; 0 = the
                                     reference's polish only) */
    int32_t pad_;
} dv_newton_opts;

typedef struct dv_newton_result {
    int32_t ok, iters, refreshed, pad_;
    double rate;
    int64_t gmres_iters, gmres_polish, balance_unclosed, jac_refresh_in_newton;
    int64_t balance_projected;    /* stage solutions closed by the balance projection */
} dv_newton_result;

/* Inexact Newton for R(z) = z - dh f(t, z) - rhs_known = 0 from z0 (newton_krylov,
 * core/solver.py:154-294): GMRES(krylov_dim, one cycle) on the finite-difference operator,
 * right-preconditioned by the stored factors; Armijo backtracking on ||M^-1 R/s||; positivity
 * truncation; conservation polish.  With allow_refresh, a stalled GMRES re-linearises at the
 * current iterate (Jacobian + factors are replaced in the model).  Synchronises `stream`. */
int dv_newton_stage(dv_model* m, double t, const double* z0, const double* rhs_known, double dh,
                    const dv_newton_opts* o, double* z_out, dv_newton_result* r, void* stream);

/* ------------------------------------------------------------------ integrator */
typedef struct dv_solver_opts {
    int32_t scheme;            /* 0 = sdirk2, 1 = trbdf2 (solver.scheme) */
    int32_t max_newton_iter, jacobian_max_age, gmres_refresh, precond_mode;
    int32_t krylov_fp32;       /* DV_KRYLOV_FP32_* mask (see dv_model_set_krylov_fp32) */
    int64_t max_steps;
    double rtol, newton_kappa, refactor_ratio, conservation_tol, h_max, h_init;
    int32_t newton_mode;       /* 0 krylov (default), 1 hybrid, 2 modified (solver.newton_mode); modified with
                                  partitioned factors runs as hybrid, as the reference does (core/solver.py:328) */
    int32_t max_polish;        /* conservation-polish iterations of a stage (reference: 2; 0 = 2) */
    int32_t polish_cycles;     /* GMRES restart cycles of a polish iteration (reference: 1; 0 = 1; at most 8) */
    int32_t balance_projection;   /* see dv_newton_opts */
} dv_solver_opts;

typedef struct dv_step_report {
    double t, h_used, err_norm;
    int64_t n_steps, n_reject, n_newton_fail, n_krylov, n_jac, n_lu, nfev;
    int64_t gmres_iters, gmres_polish, balance_unclosed, jac_refresh_in_newton, krylov_ok, krylov_fail;
    double acc[DV_NACC];       /* accumulator integrals since start (host copy) */
    int64_t newton_iters;      /* Newton iterations of all stage solves */
    int64_t pred_net, pred_extrap;   /* stage starts taken from the network / from the extrapolation */
    int64_t pred_retry;        /* stage solves repeated from the extrapolation after the network's start failed */
    int64_t modified_fail;     /* hybrid mode: modified-Newton attempts that fell back to Newton-Krylov */
    int64_t balance_projected;    /* stage solutions closed by the balance projection */
} dv_step_report;

/* TRBDF2(model, cfg, h_max, h_init) (core/solver.py:298-329) */
int dv_integrator_create(dv_model* m, const dv_solver_opts* o, dv_integrator** out);
int dv_integrator_destroy(dv_integrator* g);
/* integrate() prologue (core/solver.py:374-393): t = 0, y = y0 (device, copied), f_n, g_n. */
int dv_integrator_start(dv_integrator* g, const double* y0, double t_end, void* stream);
/* Advance until ONE step is accepted without passing t_target (core/solver.py:394-506):
 * step-size limiting, Jacobian/LU reuse policy, two implicit stages, M^-1-filtered error test,
 * accumulator quadrature, step-size update.  Host report; synchronises.  Returns DV_ERR_STEPS /
 * DV_ERR_UNDERFLOW like the reference's SolverError. */
int dv_integrator_advance(dv_integrator* g, double t_target, dv_step_report* rep, void* stream);
/* Device pointer to the current state y (n_core, owned by the integrator). */
const double* dv_integrator_y(const dv_integrator* g);
/* Copy the current state into dst (device or host memory); synchronises `stream`. */
int dv_integrator_copy_y(const dv_integrator* g, double* dst, void* stream);

/* ------------------------------------------------------------------ launch tuning
 * No reference counterpart.  Launch parameters of the hot kernels, per model: the Arnoldi steps the
 * GMRES graph runs ahead of its WHILE node (gmres_prefix, -1 = library default), the depth of the
 * preconditioner sweep's shared-memory ring of factor blocks (sweep_nbuf 2 or 3, 0 = deepest that
 * fits), the block sizes of the FP32 Jacobian product and of the FD Jacobian (0 = 128), and the Arnoldi
 * steps per pass through the WHILE node (gmres_body 1 or 2, 0 = library default: every pass costs a
 * device-side relaunch; a step after the stop returns at once).  None of them changes a result bit;
 * they only change the time. */
typedef struct dv_tuning {
    int32_t gmres_prefix, sweep_nbuf, spmv_block, fdjac_block;
    int32_t gmres_body, pad_;
} dv_tuning;
int dv_model_set_tuning(dv_model* m, const dv_tuning* t);
int dv_model_get_tuning(const dv_model* m, dv_tuning* t);
/* Autotuner: at state y (time t) and stage coefficient dh, factorise I - dh J, then time every
 * candidate of each parameter (`reps` launches each; the GMRES prefix by whole Newton stage solves)
 * with CUDA events on `stream`, keep the fastest in the model and return it in *best.  times_us
 * (optional, ntimes entries) receives the measured per-launch times in the order: fdjac 64, 128;
 * sweep nbuf 2, 3; spmv 64, 128, 256; stage solve with prefix 0, 2, 4, 6, 8; stage solve with the
 * chosen prefix and body 1, 2 (0 where a candidate does not apply).  Synchronises. */
#define DV_TUNE_NTIMES 14
int dv_autotune(dv_model* m, double t, const double* y, double dh, int32_t reps, dv_tuning* best, double* times_us,
                int32_t ntimes, void* stream);

/* ------------------------------------------------------------------ learned Newton predictor
 * No counterpart in the reference, which starts each implicit stage from a linear extrapolation
 * (core/solver.py:420 stage 1, :432/:435 stage 2).  A per-cell network (DV_MLP_NIN inputs -> three tanh
 * layers of DV_MLP_NH -> DV_MLP_NOUT outputs, BF16 weights and activations, FP32 accumulation on the
 * tcgen05 tensor cores) predicts a correction to that extrapolation for the six cell unknowns, from the
 * cell's and its six face neighbours' states at the two latest levels, f at the latest level, the step-
 * size ratio, the stage and the cycle step.  The correction of unknown v is out_v * norm[13 + v] *
 * (|z_ext - A| + 0.01 s): in units of the cell's extrapolated increment plus 1 % of its error scale
 * s = atol + rtol |A|.  Parameters (fp32, DV_MLP_NPARAM): W1 [NH x NIN], b1 [NH],
 * W2 [NH x NH], b2, W3 [NH x NH], b3, W4 [NOUT x NH], b4 [NOUT]; normalisation constants (double,
 * DV_MLP_NNORM): [0,6) level scales, [6,12) neighbour-difference scales, [12] scale of the solver-unit
 * features, [13,19) output scale per unknown, [19] target clip, [20] gate: corrections smaller than
 * this (in increment units) are not applied. */
#define DV_MLP_NIN 112
#define DV_MLP_NH 128
#define DV_MLP_NOUT 16
#define DV_MLP_NPARAM 49552
#define DV_MLP_NNORM 32
#define DV_MLP_BATCH 4096
typedef struct dv_mlp dv_mlp;
/* Network with random hidden weights (seeded) and a zero output layer (predicts no correction), and
 * room for `sample_capacity` recorded training samples. */
int dv_mlp_create(int64_t sample_capacity, uint64_t seed, dv_mlp** out);
int dv_mlp_destroy(dv_mlp* net);
/* Inference buffers for models of up to ncell cells (dv_integrator_set_predictor calls it). */
int dv_mlp_reserve(dv_mlp* net, int64_t ncell);
/* Host parameters in / out (resets the optimiser state); norm may be NULL (unchanged). */
int dv_mlp_set_params(dv_mlp* net, const float* params, int64_t nparams, const double* norm, int32_t nnorm);
int dv_mlp_get_params(const dv_mlp* net, float* params, double* norm);
int64_t dv_mlp_sample_count(const dv_mlp* net);
int dv_mlp_clear_samples(dv_mlp* net);
/* Recorded samples [first, first + count) to host: features X [count][DV_MLP_NIN] (fp32 values of the
 * stored BF16) and targets T [count][8] (the six corrections in increment units, then 1, 0); either
 * pointer may be NULL.  Synchronous. */
int dv_mlp_get_samples(const dv_mlp* net, int64_t first, int64_t count, float* X, float* T);
/* Forward pass of host feature rows X [rows][DV_MLP_NIN] (rounded to BF16) -> out [rows][DV_MLP_NOUT]. */
int dv_mlp_forward_host(dv_mlp* net, const float* X, int64_t rows, float* out);
/* One BF16 tensor-core product D[M][N] = A[M][K] B[N][K]^T (host fp32 in, rounded to BF16; FP32 out)
 * by the network's product kernel: M a multiple of 128, N in 16..128 a multiple of 16, K a multiple
 * of 16.  A check of the kernel; allocates its own device buffers. */
int dv_mlp_gemm_host(int32_t M, int32_t N, int32_t K, const float* A, const float* B, float* D);
/* Gradient of the mean squared error of the first 6 outputs against T [rows][8] (rows <= DV_MLP_BATCH)
 * by the backward kernels, into grad [DV_MLP_NPARAM]; *loss = the mean squared error. */
int dv_mlp_gradient_host(dv_mlp* net, const float* X, const float* T, int64_t rows, float* grad, double* loss);
/* `steps` Adam steps (learning rate lr) on batches of DV_MLP_BATCH recorded samples drawn by a hash of
 * seed; output scales set from the recorded targets first unless keep_scales; per-step mean loss into
 * loss_hist (host, optional).  Synchronises `stream`. */
int dv_mlp_train(dv_mlp* net, int32_t steps, float lr, uint64_t seed, int32_t keep_scales, float* loss_hist,
                 void* stream);
/* Attach a network to an integrator (net NULL detaches).  predict != 0: each stage starts from the
 * network's guess or the extrapolation, whichever has the smaller scaled stage residual, and a Newton
 * failure from the network's guess is retried from the extrapolation.  record_stride > 0: every
 * record_stride-th cell of every converged stage is appended to the network's training samples.
 * step_code: 0 adsorption, 1 blowdown, 2 heating, 3 cooling (a network input). */
int dv_integrator_set_predictor(dv_integrator* g, dv_mlp* net, int32_t predict, int32_t record_stride,
                                int32_t step_code);

/* ------------------------------------------------------------------ allocation-free residual
 * No counterpart in the reference: an addition of this library.  Same results as dv_rhs with
 * accumulators (f = dy/dt and the DV_NACC rates) for callers that must not allocate device
 * memory while they run -- a controller or estimator that reserves its memory at start-up, or a
 * host framework whose allocator owns the device -- and therefore cannot call dv_model_create.
 * The caller passes the step constants (p, host) and DEVICE arrays: feed_flux and n_nom over
 * (Nr, Ntheta), coverage over (Ntheta, Nz) (the arrays dv_model_create takes on the host), y and
 * f (n_core), acc (DV_NACC).  The face and wall records live in a static 2 MiB device array per
 * device (enough for 16x16x64); larger grids are rejected with DV_ERR_ARG.  The first call on a
 * device looks up that array's address with the device current; make that first call before any
 * stream capture.  The address is kept for the life of the process: a device reset (cudaDeviceReset)
 * after the first call on that device is not supported.  Each call clears the part it uses on
 * `stream` before its kernels run.  Every
 * call on a device shares the array: calls that overlap on the GPU (other streams, other threads)
 * race and must be serialised by the caller.  Asynchronous on `stream`. */
int dv_rhs_acc_noalloc(const dv_step_params* p, const double* feed_flux, const double* n_nom,
                       const double* coverage, double t, const double* y, double* f, double* acc, void* stream);

/* Failure-detection self-test (no reference counterpart): runs the library's two bounded device
 * waits against events that never happen -- the sweep's mbarrier wait on a barrier nothing arrives
 * at, and the cooperative Gram-Schmidt kernel's grid barrier with one block that never arrives --
 * each giving up after `polls` polls.  *bits receives the device error word they set (1: the
 * bulk-copy wait, 4: the grid barrier; 5 when both timed out as they must).  The waits return,
 * so the CUDA context stays usable.  Synchronous; allocates 16 bytes of device memory. */
int dv_selftest_wait_timeout(int32_t polls, int32_t* bits);
/* Failure-injection hook on the host (no reference counterpart): sets the model's device error word
 * to `bits` as a bounded wait that gave up would.  The model's next synchronising call reports
 * DV_ERR_CUDA with the wait named, then clears the word and the reduction tickets the abandoned wait
 * left, so the call after that runs normally. */
int dv_model_flag_wait_timeout(dv_model* m, int32_t bits);

#ifdef __cplusplus
}
#endif
#endif /* DACVTSA_H */
