"""TRBDF2 on the GPU: drop-in for the reference integrator (core/solver.py:297-511).

``TRBDF2(model, cfg, h_max, h_init=None, logger=None).integrate(y0, t_end, t_out, on_step, stop_fn,
stop_value, stop_direction)`` returns an ``IntegrationResult`` with the reference's fields, and
exposes ``.jac.ngroups`` and ``.stats`` the step runner reads (steps/_runner.py:149-152).

The whole step loop -- step-size limiting, Jacobian / factorisation reuse, the two implicit stages
solved by Newton-Krylov, the M^-1-filtered error test, accumulator quadrature and step-size update --
runs inside the library (dv_integrator_advance); Python only receives each accepted step to apply
the caller's stop criterion, ``on_step`` callback and snapshot times, exactly where the reference
does.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np
import torch

from . import counters
from ._lib import DvSolverOpts, DvStepReport, check, load
from .config import gpu_option
from .jacobian import FDJacobian
from .model import PRECOND_MODES

KRYLOV_FP32_FACTORS, KRYLOV_FP32_OPERATOR = 1, 2
GAMMA = 2.0 - np.sqrt(2.0)
D = GAMMA / 2.0
G_SD = 1.0 - 1.0 / np.sqrt(2.0)


class SolverError(RuntimeError):
    """Unrecoverable integration failure (same role as core/solver.py:62-63)."""


@dataclass
class IntegrationResult:
    y: np.ndarray
    acc: np.ndarray
    t: float
    n_steps: int = 0
    n_reject: int = 0
    n_newton_fail: int = 0
    n_krylov: int = 0
    n_jac: int = 0
    n_lu: int = 0
    nfev: int = 0
    wall_time: float = 0.0
    snapshots: List = field(default_factory=list)
    stopped_early: bool = False
    stop_value: Optional[float] = None


class TRBDF2:
    def __init__(self, model, cfg, h_max: float, h_init: Optional[float] = None, logger=None):
        self.m = model
        self.lib = load()
        s = cfg.solver
        self.rtol = s.rtol
        self.atol = model.atol
        self.h_max = h_max
        self.h_init = h_init if h_init is not None else s.h_initial
        self.max_iter = s.max_newton_iter
        self.kappa = s.newton_kappa
        self.jac_max_age = s.jacobian_max_age
        self.max_steps = s.max_steps_per_step
        self.scheme = s.scheme
        self.precond = s.preconditioner if model.grid.Nth > 1 else "full"
        self.jac = FDJacobian(model)
        self.log = logger or (lambda *a, **k: None)
        self.stats = {"modified_fail": 0, "krylov_ok": 0, "krylov_fail": 0}
        o = DvSolverOpts()
        o.scheme = 0 if s.scheme == "sdirk2" else 1
        o.max_newton_iter = s.max_newton_iter
        o.jacobian_max_age = s.jacobian_max_age
        o.gmres_refresh = s.gmres_refresh
        # theta_block: the reference keeps the theta couplings of its innermost precond_theta_rings
        # rings; the GPU partitions keep those of the innermost ring (mode 2), or none when 0 rings
        if self.precond == "theta_block":
            o.precond_mode = PRECOND_MODES["theta_block" if s.precond_theta_rings >= 1 else "sector"]
        else:
            o.precond_mode = PRECOND_MODES["full"]
        o.max_steps = s.max_steps_per_step
        o.rtol = s.rtol
        o.newton_kappa = s.newton_kappa
        o.refactor_ratio = s.refactor_ratio
        o.conservation_tol = float(s.conservation_tol or 0.0)
        o.h_max = h_max
        o.h_init = self.h_init
        # newton_mode: krylov (default), hybrid (modified Newton first, Krylov fallback) or modified
        o.newton_mode = {"krylov": 0, "hybrid": 1, "modified": 2}[s.newton_mode]
        # gpu.max_polish: conservation-polish iterations per stage (the reference's 2 by default)
        o.max_polish = int(gpu_option(cfg, "max_polish", 2))
        # gpu.polish_cycles: GMRES restart cycles of one polish iteration (the reference runs one)
        o.polish_cycles = int(gpu_option(cfg, "polish_cycles", 1))
        # gpu.balance_projection: close the balances of a converged stage by the balance projection
        # before the reference's polish iterations (no reference counterpart)
        o.balance_projection = int(bool(gpu_option(cfg, "balance_projection", False)))
        self.mode = "hybrid" if (s.newton_mode == "modified" and self.precond == "theta_block") else s.newton_mode
        # gpu.krylov_precision: fp64 (default, the parity path); fp32 (GMRES on the FP32 assembled
        # Jacobian with FP32 preconditioner factors, FP64 residual / Newton update as refinement);
        # fp32_factors (only the factors in FP32)
        self.krylov_precision = gpu_option(cfg, "krylov_precision", "fp64")
        o.krylov_fp32 = {"fp64": 0, "fp32_factors": KRYLOV_FP32_FACTORS,
                         "fp32": KRYLOV_FP32_FACTORS | KRYLOV_FP32_OPERATOR}[self.krylov_precision]
        self.opts = o

        h = C.c_void_p()
        check(self.lib.dv_integrator_create(model.handle, C.byref(o), C.byref(h)), "dv_integrator_create")
        self.handle = h
        self._y_host = None
        # gpu.predictor: extrapolation (default, the reference's predictor) or learned (the trained
        # network of gpu.predictor_weights, or the packaged one, corrects each stage's start)
        self.predictor = None
        if gpu_option(cfg, "predictor", "extrapolation") == "learned":
            from .predictor import default_network
            default_network(gpu_option(cfg, "predictor_weights", "")).attach(
                self, model.step.get("type", "adsorption"), predict=True)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.dv_integrator_destroy(h)
            except Exception:
                pass
            self.handle = None

    def scale(self, y):
        return self.atol + self.rtol * np.abs(y)

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def state(self, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Current state as a device tensor (copied)."""
        m = self.m
        if out is None:
            out = torch.empty(m.n_core, dtype=torch.float64, device=m.device)
        check(self.lib.dv_integrator_copy_y(self.handle, C.c_void_p(out.data_ptr()), self._stream()),
              "dv_integrator_copy_y")
        return out

    def y_ptr(self) -> int:
        """Device address of the integrator's current state (it moves from step to step)."""
        return int(self.lib.dv_integrator_y(self.handle) or 0)

    def _host_y(self) -> np.ndarray:
        if self._y_host is None:
            self._y_host = torch.empty(self.m.n_core, dtype=torch.float64).pin_memory()
        check(self.lib.dv_integrator_copy_y(self.handle, C.c_void_p(self._y_host.data_ptr()), self._stream()),
              "dv_integrator_copy_y")
        counters.d2h(8 * self.m.n_core)
        return self._y_host.numpy().copy()

    def integrate(self, y0, t_end: float, t_out, on_step: Optional[Callable] = None,
                  stop_fn: Optional[Callable] = None, stop_value: Optional[float] = None,
                  stop_direction: int = 1, keep_on_device: bool = False,
                  on_step_device: Optional[Callable] = None) -> IntegrationResult:
        """Adaptive integration over [0, t_end] (core/solver.py:370-511).

        y0: numpy array (host, copied) or float64 CUDA tensor.  With keep_on_device=True the result's
        ``y`` is a device tensor and snapshots are skipped unless callbacks need host copies.
        on_step_device(t, y_ptr, acc): called where on_step is, with the device address of the
        accepted state (valid until the next step) instead of a host copy."""
        m = self.m
        wall0 = time.time()
        with torch.cuda.device(m.device):
            if isinstance(y0, torch.Tensor):
                y0d = y0
                y0h = None
            else:
                y0h = np.ascontiguousarray(y0, dtype=np.float64)
                y0d = torch.from_numpy(y0h).to(m.device)
                counters.h2d(y0h.nbytes)
            check(self.lib.dv_integrator_start(self.handle, C.c_void_p(y0d.data_ptr()), float(t_end),
                                               self._stream()), "dv_integrator_start")
            acc = np.zeros(m.n_acc)
            res = IntegrationResult(y=None, acc=acc, t=0.0)
            t_out = np.asarray(sorted(set(np.clip(np.atleast_1d(t_out), 0.0, t_end)) | {t_end}))
            k_out = 0
            if t_out[0] <= 0.0:
                if not keep_on_device:
                    res.snapshots.append((0.0, (y0h if y0h is not None else y0d.cpu().numpy()).copy(), acc.copy()))
                k_out = 1
            rep = DvStepReport()
            t = 0.0
            need_host = on_step is not None or (stop_fn is not None and stop_value is not None)
            while t < t_end * (1.0 - 1e-12):
                t_target = t_out[k_out] if k_out < len(t_out) else t_end
                check(self.lib.dv_integrator_advance(self.handle, float(t_target), C.byref(rep), self._stream()),
                      "dv_integrator_advance")
                if rep.t <= t:          # nothing left to integrate
                    break
                t = rep.t
                acc = np.array(rep.acc[:m.n_acc])
                yh = self._host_y() if (need_host or (not keep_on_device and k_out < len(t_out)
                                                      and t >= t_out[k_out] * (1.0 - 1e-12))) else None
                if stop_fn is not None and stop_value is not None:
                    sv = stop_fn(t, yh)
                    if sv is not None and (sv - stop_value) * stop_direction >= 0.0:
                        res.stopped_early = True
                        res.stop_value = sv
                        if on_step:
                            on_step(t, yh, acc)
                        if on_step_device:
                            on_step_device(t, self.y_ptr(), acc)
                        res.snapshots.append((t, yh.copy(), acc.copy()))
                        break
                if on_step:
                    on_step(t, yh, acc)
                if on_step_device:
                    on_step_device(t, self.y_ptr(), acc)
                if k_out < len(t_out) and t >= t_out[k_out] * (1.0 - 1e-12):
                    if not keep_on_device:
                        res.snapshots.append((t, yh.copy(), acc.copy()))
                    k_out += 1
            res.t = t
            res.acc = acc
            res.y = self.state() if keep_on_device else self._host_y()
            res.n_steps, res.n_reject, res.n_newton_fail = rep.n_steps, rep.n_reject, rep.n_newton_fail
            res.n_krylov, res.n_jac, res.n_lu, res.nfev = rep.n_krylov, rep.n_jac, rep.n_lu, m.nfev
            self.stats.update({"krylov_ok": rep.krylov_ok, "krylov_fail": rep.krylov_fail,
                               "gmres_iters": rep.gmres_iters, "gmres_polish": rep.gmres_polish,
                               "balance_unclosed": rep.balance_unclosed,
                               "jac_refresh_in_newton": rep.jac_refresh_in_newton,
                               "newton_iters": rep.newton_iters, "pred_net": rep.pred_net,
                               "pred_extrap": rep.pred_extrap, "pred_retry": rep.pred_retry,
                               "modified_fail": rep.modified_fail, "balance_projected": rep.balance_projected})
            res.wall_time = time.time() - wall0
            return res
