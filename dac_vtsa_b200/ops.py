"""PyTorch operators over the C ABI: ``torch.ops.dacvtsa.*``.

Thin ``torch.library`` registrations of the stepping path's entry points, for callers that compose
them with other PyTorch code (the same kernels the Python classes call; no other implementation
exists, there is no CPU kernel).  A model / integrator is passed as its C handle (``model.handle.value``
/ ``integ.handle.value``, an int); tensors are contiguous float64 CUDA tensors on the model's device.

  dacvtsa::rhs(model, t, y) -> (f, acc)                       TVSAModel.rhs          core/residual.py:211-417
  dacvtsa::stage_residual(model, t, y, gamma_h, rhs_known)    TVSAModel.stage_residual core/residual.py:420-423
  dacvtsa::fd_jacobian(model, t, y, f0) -> J (block layout)   FDJacobian.__call__    core/jacobian.py:71-86
  dacvtsa::precond_factor(model, J, dh, mode) -> ()           TRBDF2._factor         core/solver.py:334-337
  dacvtsa::newton_stage(model, t, z0, rhs_known, dh, max_iter, kappa) -> (z, info)
                                                              newton_krylov          core/solver.py:154-294
  dacvtsa::step(integrator, t_target) -> info                 one accepted step of   core/solver.py:394-506
      info = [t, h, err_norm, steps, rejected, newton_fail, ...] (float64, DvStepReport order)

Each has a fake (meta) implementation, so the operators trace under torch.compile / FakeTensor
(shapes only; the stepping path itself is not compiled).
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import torch
from torch import Tensor

from ._lib import DV_NACC, DvNewtonOpts, DvNewtonResult, DvStepReport, check, load

_P = C.c_void_p


def _s():
    return _P(torch.cuda.current_stream().cuda_stream)


def _p(t: Tensor):
    return _P(t.data_ptr())


def _check_in(*ts: Tensor):
    for t in ts:
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError("dacvtsa operators take contiguous float64 CUDA tensors")


def _jac_doubles(model: int) -> int:
    sz = [C.c_int64() for _ in range(5)]
    check(load().dv_model_sizes(_P(model), *[C.byref(x) for x in sz]), "dv_model_sizes")
    return sz[3].value


@torch.library.custom_op("dacvtsa::rhs", mutates_args=(), device_types="cuda")
def rhs(model: int, t: float, y: Tensor) -> Tuple[Tensor, Tensor]:
    _check_in(y)
    f = torch.empty_like(y)
    acc = torch.empty(DV_NACC, dtype=torch.float64, device=y.device)
    check(load().dv_rhs(_P(model), float(t), _p(y), _p(f), _p(acc), _s()), "dv_rhs")
    return f, acc


@rhs.register_fake
def _(model, t, y):
    return torch.empty_like(y), y.new_empty(DV_NACC)


@torch.library.custom_op("dacvtsa::stage_residual", mutates_args=(), device_types="cuda")
def stage_residual(model: int, t: float, y: Tensor, gamma_h: float, rhs_known: Tensor) -> Tensor:
    _check_in(y, rhs_known)
    R = torch.empty_like(y)
    check(load().dv_stage_residual(_P(model), float(t), _p(y), float(gamma_h), _p(rhs_known), _p(R), _s()),
          "dv_stage_residual")
    return R


@stage_residual.register_fake
def _(model, t, y, gamma_h, rhs_known):
    return torch.empty_like(y)


@torch.library.custom_op("dacvtsa::fd_jacobian", mutates_args=(), device_types="cuda")
def fd_jacobian(model: int, t: float, y: Tensor, f0: Tensor) -> Tensor:
    _check_in(y, f0)
    J = torch.empty(_jac_doubles(model), dtype=torch.float64, device=y.device)
    check(load().dv_fd_jacobian(_P(model), float(t), _p(y), _p(f0), _p(J), _s()), "dv_fd_jacobian")
    return J


@fd_jacobian.register_fake
def _(model, t, y, f0):
    ctx = torch.library.get_ctx()
    return y.new_empty(ctx.new_dynamic_size())


@torch.library.custom_op("dacvtsa::precond_factor", mutates_args=(), device_types="cuda")
def precond_factor(model: int, J: Tensor, dh: float, mode: int) -> None:
    _check_in(J)
    check(load().dv_precond_factor(_P(model), _p(J), float(dh), int(mode), _s()), "dv_precond_factor")


@precond_factor.register_fake
def _(model, J, dh, mode):
    return None


@torch.library.custom_op("dacvtsa::newton_stage", mutates_args=(), device_types="cuda")
def newton_stage(model: int, t: float, z0: Tensor, rhs_known: Tensor, dh: float, max_iter: int,
                 kappa: float, rtol: float, cons_tol: float, precond_mode: int) -> Tuple[Tensor, Tensor]:
    _check_in(z0, rhs_known)
    o = DvNewtonOpts()
    o.max_iter, o.krylov_dim, o.allow_refresh, o.precond_mode = int(max_iter), 30, 0, int(precond_mode)
    o.kappa, o.eta, o.rtol, o.cons_tol = float(kappa), 1e-2, float(rtol), float(cons_tol)
    r = DvNewtonResult()
    z = torch.empty_like(z0)
    check(load().dv_newton_stage(_P(model), float(t), _p(z0), _p(rhs_known), float(dh), C.byref(o), _p(z),
                                 C.byref(r), _s()), "dv_newton_stage")
    info = torch.tensor([r.ok, r.iters, r.rate, r.gmres_iters, r.gmres_polish, r.balance_unclosed],
                        dtype=torch.float64)
    return z, info


@newton_stage.register_fake
def _(model, t, z0, rhs_known, dh, max_iter, kappa, rtol, cons_tol, precond_mode):
    return torch.empty_like(z0), torch.empty(6, dtype=torch.float64)


REPORT_FIELDS = ("t", "h_used", "err_norm", "n_steps", "n_reject", "n_newton_fail", "n_krylov", "n_jac", "n_lu",
                 "nfev", "gmres_iters", "gmres_polish", "balance_unclosed", "jac_refresh_in_newton", "krylov_ok",
                 "krylov_fail", "newton_iters", "pred_net", "pred_extrap", "pred_retry", "modified_fail")


@torch.library.custom_op("dacvtsa::step", mutates_args=())
def step(integrator: int, t_target: float) -> Tensor:
    """Advance a started integrator by one accepted step (not past t_target); host report."""
    rep = DvStepReport()
    check(load().dv_integrator_advance(_P(integrator), float(t_target), C.byref(rep), _s()), "dv_integrator_advance")
    return torch.tensor([float(getattr(rep, k)) for k in REPORT_FIELDS], dtype=torch.float64)


@step.register_fake
def _(integrator, t_target):
    return torch.empty(len(REPORT_FIELDS), dtype=torch.float64)
