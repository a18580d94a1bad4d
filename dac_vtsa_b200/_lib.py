"""ctypes binding of the C ABI in include/dacvtsa.h (loaded from the in-tree libdacvtsa.so)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdacvtsa.so")

DV_MAX_NR, DV_NG, DV_NA, DV_NV, DV_NACC, DV_NSLOT, DV_NB = 64, 3, 2, 6, 36, 9, 7
DV_OK, DV_ERR_ARG, DV_ERR_CUDA, DV_ERR_UNSUPPORTED, DV_ERR_STEPS, DV_ERR_UNDERFLOW = 0, -1, -2, -3, -10, -11
END_KIND = {"closed": 0, "feed": 1, "pump": 2, "valve": 3, "pressure": 4}
LIMITER = {"van_albada": 0, "van_albada_tvd": 1, "van_leer": 2, "minmod": 3, "upwind": 4}
COADS = {"none": 0, "wadst": 1, "mechanistic": 2, "stampi_bombelli": 3}
DISP = {"edwards_richardson": 0, "young2021": 1, "wakao_kagei": 2}
BEDCOND = {"zehner_schlunder": 0, "parallel": 1, "constant": 2}
WALLHTC = {"martin_nilles": 0, "constant": 1}

D = C.c_double
I32 = C.c_int32
I64 = C.c_int64


class DvEnd(C.Structure):
    _fields_ = [("kind", I32), ("valve", I32), ("check_valve", I32), ("is_vacuum", I32), ("is_feed", I32),
                ("pad_", I32), ("P_target", D), ("T_ext", D), ("speed", D), ("P_start", D), ("y_ext", D * DV_NG)]


def _arr(n):
    return D * n


class DvStepParams(C.Structure):
    _fields_ = [
        ("Nr", I32), ("Nth", I32), ("Nz", I32), ("wall_on", I32),
        ("dz", D), ("dth", D), ("half_dr_outer", D), ("A_wall_in", D), ("A_wall_out", D), ("wall_C", D),
        ("wall_kz", D), ("wall_kt", D),
        ("Az", _arr(DV_MAX_NR)), ("V", _arr(DV_MAX_NR)), ("Ath", _arr(DV_MAX_NR)), ("arc", _arr(DV_MAX_NR)),
        ("Ar", _arr(DV_MAX_NR)), ("drc", _arr(DV_MAX_NR)),
        ("eps_b", D), ("eps_t", D), ("rho_b", D), ("cp_s", D), ("dp", D), ("T_ref", D),
        ("cpg", _arr(DV_NG)), ("cpa", _arr(DV_NA)), ("dH", _arr(DV_NA)),
        ("M", _arr(DV_NG)),
        ("mu_w", _arr(2) * DV_NG), ("mu_D", _arr(2) * DV_NG), ("mu_E", _arr(2) * DV_NG),
        ("k_w", _arr(2) * DV_NG), ("k_0", _arr(2) * DV_NG), ("k_n", _arr(2) * DV_NG),
        ("mu_nt", I32 * DV_NG), ("k_nt", I32 * DV_NG),
        ("mass_q", _arr(DV_NG) * DV_NG), ("wilke_den", _arr(DV_NG) * DV_NG),
        ("fuller_sqrtM", _arr(2)), ("fuller_s", _arr(2)),
        ("co2_q_inf0", D), ("co2_chi", D), ("co2_b0", D), ("co2_dH0", D), ("co2_tau0", D), ("co2_alpha", D),
        ("co2_T0", D), ("p_reg", D),
        ("h2o_q_m", D), ("h2o_C", D), ("h2o_D", D), ("h2o_F", D), ("h2o_G", D), ("h2o_E10_slope", D),
        ("h2o_E10_intercept", D), ("rh_cap", D),
        ("wadst_b0", D), ("wadst_q_inf0", D), ("wadst_tau0", D), ("wadst_chi", D), ("wadst_alpha", D),
        ("wadst_dH", D), ("wadst_A", D),
        ("mech_f_blocked_max", D), ("mech_k", D), ("mech_phi_dry", D), ("mech_A", D), ("mech_dH_wet", D),
        ("mech_n", D),
        ("sb_gamma", D), ("sb_beta", D),
        ("coads", I32), ("basis_state", I32),
        ("k_ldf", _arr(DV_NA)), ("Ea", _arr(DV_NA)), ("T_ref_kin", D),
        ("ea_zero", I32),
        ("disp_model", I32), ("bed_model", I32), ("htc_model", I32), ("lumped", I32),
        ("ka", D), ("kb", D), ("g1", D), ("g2", D), ("er_beta", D), ("Pe_T", D), ("lam_const", D), ("zs_B", D),
        ("zs_s", D), ("lam_s", D), ("Pe_r", D), ("Pe_z", D), ("alpha_const", D), ("N_ratio", D), ("U_lumped", D),
        ("u_nom", D),
        ("limiter", I32), ("pad0_", I32),
        ("ends", DvEnd * 2),
        ("tau_valve", D),
        ("jacket_on", I32), ("hx_on", I32),
        ("T_jac_set", D), ("T_jac_prev", D), ("jac_tau", D), ("h_jac", D), ("h_amb", D), ("T_amb", D),
        ("P_amb", D), ("hA_v", D),
        ("gam", D), ("eta_vac", D), ("eta_bl", D),
        ("vac_krishnamurthy", I32), ("pump_water", I32),
        ("atol", _arr(DV_NB)), ("typ", _arr(DV_NB)),
    ]


class DvNewtonOpts(C.Structure):
    _fields_ = [("max_iter", I32), ("krylov_dim", I32), ("allow_refresh", I32), ("precond_mode", I32),
                ("kappa", D), ("eta", D), ("rtol", D), ("cons_tol", D), ("max_polish", I32),
                ("polish_cycles", I32), ("balance_projection", I32), ("pad_", I32)]


class DvNewtonResult(C.Structure):
    _fields_ = [("ok", I32), ("iters", I32), ("refreshed", I32), ("pad_", I32), ("rate", D),
                ("gmres_iters", I64), ("gmres_polish", I64), ("balance_unclosed", I64),
                ("jac_refresh_in_newton", I64), ("balance_projected", I64)]


class DvSolverOpts(C.Structure):
    _fields_ = [("scheme", I32), ("max_newton_iter", I32), ("jacobian_max_age", I32), ("gmres_refresh", I32),
                ("precond_mode", I32), ("krylov_fp32", I32), ("max_steps", I64),
                ("rtol", D), ("newton_kappa", D), ("refactor_ratio", D), ("conservation_tol", D),
                ("h_max", D), ("h_init", D), ("newton_mode", I32), ("max_polish", I32), ("polish_cycles", I32),
                ("balance_projection", I32)]


class DvTuning(C.Structure):
    _fields_ = [("gmres_prefix", I32), ("sweep_nbuf", I32), ("spmv_block", I32), ("fdjac_block", I32),
                ("gmres_body", I32), ("pad_", I32)]


class DvStepReport(C.Structure):
    _fields_ = [("t", D), ("h_used", D), ("err_norm", D),
                ("n_steps", I64), ("n_reject", I64), ("n_newton_fail", I64), ("n_krylov", I64), ("n_jac", I64),
                ("n_lu", I64), ("nfev", I64), ("gmres_iters", I64), ("gmres_polish", I64),
                ("balance_unclosed", I64), ("jac_refresh_in_newton", I64), ("krylov_ok", I64),
                ("krylov_fail", I64), ("acc", D * DV_NACC), ("newton_iters", I64), ("pred_net", I64),
                ("pred_extrap", I64), ("pred_retry", I64), ("modified_fail", I64),
                ("balance_projected", I64)]


STRUCT_MIRRORS = {"dv_newton_opts": DvNewtonOpts, "dv_newton_result": DvNewtonResult, "dv_solver_opts": DvSolverOpts,
                  "dv_step_report": DvStepReport, "dv_tuning": DvTuning}

P = C.c_void_p
# (name, restype, argtypes) of every entry point declared in include/dacvtsa.h
SIGNATURES = [
    ("dv_abi_version", C.c_int, []),
    ("dv_step_params_size", C.c_size_t, []),
    ("dv_struct_size", C.c_size_t, [C.c_char_p]),
    ("dv_pool_cached_bytes", C.c_int64, []),
    ("dv_pool_release", C.c_int, []),
    ("dv_last_error", C.c_char_p, []),
    ("dv_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("dv_profile_enable", C.c_int, [I32]),
    ("dv_profile_read", C.c_int, [I32, C.POINTER(I64), C.POINTER(I64), C.POINTER(D)]),
    ("dv_launch_count", I64, []),
    ("dv_model_create", C.c_int, [C.POINTER(DvStepParams), P, P, P, C.POINTER(P)]),
    ("dv_model_destroy", C.c_int, [P]),
    ("dv_model_sizes", C.c_int, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    ("dv_model_nfev", I64, [P]),
    ("dv_rhs", C.c_int, [P, D, P, P, P, P]),
    ("dv_stage_residual", C.c_int, [P, D, P, D, P, P, P]),
    ("dv_rhs_diag", C.c_int, [P, D, P, P, P]),
    ("dv_outlet_row", C.c_int, [P, D, P, D, P, P]),
    ("dv_precond_partitions", C.c_int, [P, C.POINTER(I32), C.POINTER(I32), P, I32, C.POINTER(I32)]),
    ("dv_precond_check_maps", C.c_int, [C.POINTER(DvStepParams), I32, C.POINTER(I32), C.POINTER(I32), C.POINTER(I64)]),
    ("dv_colour_columns", C.c_int, [I32, I32, I32, I32, P, C.POINTER(I32)]),
    ("dv_fd_jacobian", C.c_int, [P, D, P, P, P, P]),
    ("dv_precond_factor", C.c_int, [P, P, D, I32, P]),
    ("dv_precond_solve", C.c_int, [P, P, P, P]),
    ("dv_model_set_krylov_fp32", C.c_int, [P, I32]),
    ("dv_newton_stage", C.c_int, [P, D, P, P, D, C.POINTER(DvNewtonOpts), P, C.POINTER(DvNewtonResult), P]),
    ("dv_integrator_create", C.c_int, [P, C.POINTER(DvSolverOpts), C.POINTER(P)]),
    ("dv_integrator_destroy", C.c_int, [P]),
    ("dv_integrator_start", C.c_int, [P, P, D, P]),
    ("dv_integrator_advance", C.c_int, [P, D, C.POINTER(DvStepReport), P]),
    ("dv_integrator_y", P, [P]),
    ("dv_integrator_copy_y", C.c_int, [P, P, P]),
    ("dv_rhs_acc_noalloc", C.c_int, [C.POINTER(DvStepParams), P, P, P, D, P, P, P, P]),
    ("dv_selftest_wait_timeout", C.c_int, [I32, C.POINTER(I32)]),
    ("dv_model_flag_wait_timeout", C.c_int, [P, I32]),
    ("dv_model_set_tuning", C.c_int, [P, C.POINTER(DvTuning)]),
    ("dv_model_get_tuning", C.c_int, [P, C.POINTER(DvTuning)]),
    ("dv_autotune", C.c_int, [P, D, P, D, I32, C.POINTER(DvTuning), P, I32, P]),
    ("dv_mlp_create", C.c_int, [I64, C.c_uint64, C.POINTER(P)]),
    ("dv_mlp_destroy", C.c_int, [P]),
    ("dv_mlp_reserve", C.c_int, [P, I64]),
    ("dv_mlp_set_params", C.c_int, [P, P, I64, P, I32]),
    ("dv_mlp_get_params", C.c_int, [P, P, P]),
    ("dv_mlp_sample_count", I64, [P]),
    ("dv_mlp_clear_samples", C.c_int, [P]),
    ("dv_mlp_get_samples", C.c_int, [P, I64, I64, P, P]),
    ("dv_mlp_forward_host", C.c_int, [P, P, I64, P]),
    ("dv_mlp_gradient_host", C.c_int, [P, P, P, I64, P, C.POINTER(D)]),
    ("dv_mlp_gemm_host", C.c_int, [I32, I32, I32, P, P, P]),
    ("dv_mlp_train", C.c_int, [P, I32, C.c_float, C.c_uint64, I32, P, P]),
    ("dv_integrator_set_predictor", C.c_int, [P, P, I32, I32, I32]),
]

_lib = None


class LibraryError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it was not built (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LibraryError(f"{path} is missing: build it with `python -m dac_vtsa_b200.build` "
                           "(or __graft_entry__.build()); the stepping path has no CPU fallback")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.dv_step_params_size() != C.sizeof(DvStepParams):
        raise LibraryError("dv_step_params layout mismatch between include/dacvtsa.h and the ctypes mirror")
    for cname, mirror in STRUCT_MIRRORS.items():
        if lib.dv_struct_size(cname.encode()) != C.sizeof(mirror):
            raise LibraryError(f"{cname} layout mismatch between include/dacvtsa.h and the ctypes mirror")
    _lib = lib
    return lib


def check(rc: int, what: str = ""):
    if rc == DV_OK:
        return
    msg = (_lib.dv_last_error() or b"").decode()
    if rc in (DV_ERR_STEPS, DV_ERR_UNDERFLOW):
        from .solver import SolverError
        raise SolverError(msg)
    if rc == DV_ERR_UNSUPPORTED:
        raise NotImplementedError(f"{what}: {msg}")
    raise LibraryError(f"{what} failed ({rc}): {msg}")


KERNEL_KINDS = ("residual", "matvec", "fd_jacobian", "precond_factor", "precond_apply", "vector", "mlp",
                "spmv")


def profile_enable(on: bool = True):
    check(load().dv_profile_enable(int(bool(on))), "dv_profile_enable")


def profile_read():
    """{kind: (launches, timed launches, device ms)} for the library's kernels since profile_enable."""
    lib = load()
    out = {}
    for k, name in enumerate(KERNEL_KINDS):
        a, b, ms = I64(0), I64(0), D(0.0)
        check(lib.dv_profile_read(k, C.byref(a), C.byref(b), C.byref(ms)), "dv_profile_read")
        out[name] = (a.value, b.value, ms.value)
    return out


def pool_cached_bytes() -> int:
    """Device and pinned memory of destroyed handles that the library keeps for the next ones."""
    return int(load().dv_pool_cached_bytes())


def pool_release():
    """Free the memory the library keeps for future handles."""
    check(load().dv_pool_release(), "dv_pool_release")


def launch_count() -> int:
    return int(load().dv_launch_count())


def colour_columns(Nr: int, Nth: int, Nz: int, wall: bool = True):
    """Greedy distance-2 colouring of the stencil pattern (host code of the library)."""
    lib = load()
    n = 6 * Nr * Nth * Nz + (Nth * Nz if wall else 0)
    out = np.empty(n, dtype=np.int64)
    nc = I32(0)
    check(lib.dv_colour_columns(Nr, Nth, Nz, int(bool(wall)), out.ctypes.data, C.byref(nc)), "dv_colour_columns")
    return out, int(nc.value)
