"""Oracle: 2-stage L-stable implicit RK integrator with Newton-Krylov stage solves.

Restates core/solver.py:47-511 of the reference (TR-BDF2 and SDIRK2 share M = I - d h J with
d = (2 - sqrt 2)/2; GMRES(30, one cycle) right-preconditioned by a SuperLU factorisation of the
theta-block Jacobian; Armijo line search on the affine-invariant norm ||M^-1 R / s||;
positivity truncation; conservation polish; Hairer-Wanner early exit; M^-1-filtered error
control).  scipy's splu/gmres are the reference's own dependencies (requirements.txt: scipy).

``fixed_step_run`` is the replay harness: it advances the same stage equations over a given
step-size sequence and solves every stage to a tight residual, so two correct solvers of the
same discretisation agree far below the adaptive tolerances.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .jacobian import OracleFDJacobian

GAMMA = 2.0 - np.sqrt(2.0)                     # core/solver.py:47-59
D = GAMMA / 2.0
C1 = 1.0 / (GAMMA * (2.0 - GAMMA))
C2 = (1.0 - GAMMA) ** 2 / (GAMMA * (2.0 - GAMMA))
W1 = (3.0 * GAMMA - 1.0) / (6.0 * GAMMA)
W2 = 1.0 / (6.0 * GAMMA * (1.0 - GAMMA))
W3 = (2.0 - 3.0 * GAMMA) / (6.0 * (1.0 - GAMMA))
SQRT_EPS = np.sqrt(np.finfo(float).eps)
G_SD = 1.0 - 1.0 / np.sqrt(2.0)
SW1 = (3.0 * G_SD - 1.0) / (6.0 * G_SD)
SW2 = 1.0 / (6.0 * G_SD * (1.0 - G_SD))
SW3 = (2.0 - 3.0 * G_SD) / (6.0 * (1.0 - G_SD))


class SolverError(RuntimeError):
    pass


@dataclass
class Result:
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
    steps: List = field(default_factory=list)        # accepted (t_start, h) -- for replay


def _rms(x):
    return float(np.sqrt(np.mean(x * x)))


def _cons_ok(W, R, s, tol):                     # core/solver.py:88-96
    if W is None or tol <= 0.0:
        return True
    return bool(np.all(np.abs(W @ R) <= tol * (W @ s)))


def _truncate(z_new, z_old, pos, floor=0.1):    # core/solver.py:99-108
    lo = floor * np.maximum(z_old[pos], 0.0)
    z_new[pos] = np.maximum(z_new[pos], lo)
    return z_new


def newton_krylov(model, t, z0, rhs_known, dh, lu, scale, max_iter, kappa, krylov_dim=30, eta=1e-2,
                  counter=None, pos=None, cons=None, cons_tol=0.0, stats=None, refresh=None):
    """Inexact Newton, GMRES direction, backtracking on ||M^-1 R/s|| (core/solver.py:154-294)."""
    z = z0.copy()
    f, _ = model.rhs(t, z, want_acc=False)
    s = scale(z)
    R = z - dh * f - rhs_known
    rn = _rms(R / s)
    if not np.isfinite(rn):
        return z0, False, 0, np.inf, None
    pnorm = lambda RR, ss: _rms(lu.solve(RR) / ss)        # noqa: E731
    pn = pnorm(R, s)
    n = len(z)
    step_prev, polish, best, new_lu, it = None, 0, None, None, -1
    while it + 1 < max_iter + polish:
        it += 1
        s = scale(z)
        b = -R / s
        zs = max(1.0, _rms(z / s))

        def matvec(u, z=z, f=f, s=s, zs=zs):
            un = _rms(u)
            if un == 0.0:
                return np.zeros_like(u)
            sig = SQRT_EPS * zs / un
            v = u * s
            fp, _ = model.rhs(t, z + sig * v, want_acc=False)
            return (v - dh * (fp - f) / sig) / s

        def prec(r, s=s, lu=lu):
            return lu.solve(r * s) / s

        AP = spla.LinearOperator((n, n), matvec=lambda w, prec=prec: matvec(prec(w)), dtype=float)
        if polish and stats is not None:
            def cb(_x):
                stats["gmres_polish"] = stats.get("gmres_polish", 0) + 1
        elif counter is not None:
            def cb(_x):
                counter[0] += 1
        else:
            cb = None
        floor = (1e-4 if polish else 0.1 * kappa) * np.sqrt(n)
        w, info = spla.gmres(AP, b, rtol=(1e-3 if polish else eta), atol=floor, restart=krylov_dim,
                             maxiter=1, callback=cb, callback_type="pr_norm")
        if info != 0 and refresh is not None and new_lu is None and not polish:
            lu = new_lu = refresh(z)
            pnorm = lambda RR, ss, lu=lu: _rms(lu.solve(RR) / ss)   # noqa: E731
            pn = pnorm(R, s)
            if stats is not None:
                stats["jac_refresh_in_newton"] = stats.get("jac_refresh_in_newton", 0) + 1

            def prec(r, s=s, lu=lu):
                return lu.solve(r * s) / s

            AP = spla.LinearOperator((n, n), matvec=lambda w, prec=prec: matvec(prec(w)), dtype=float)
            w, info = spla.gmres(AP, b, rtol=eta, atol=floor, restart=krylov_dim, maxiter=1, callback=cb,
                                 callback_type="pr_norm")
        dz = prec(w) * s
        if not np.all(np.isfinite(dz)):
            return z0, False, it + 1, np.inf, new_lu
        lam = 1.0
        for ls in range(4):
            z_try = _truncate(z + lam * dz, z, pos)
            f_try, _ = model.rhs(t, z_try, want_acc=False)
            R_try = z_try - dh * f_try - rhs_known
            rn_try = _rms(R_try / s)
            pn_try = pnorm(R_try, s) if np.isfinite(rn_try) else np.inf
            if np.isfinite(pn_try) and (pn_try <= (1.0 - 1e-4 * lam) * pn or ls == 3):
                break
            lam *= 0.5
        if not np.isfinite(pn_try):
            return z0, False, it + 1, np.inf, new_lu
        step = _rms((z_try - z) / s)
        z, f, R, rn, pn = z_try, f_try, R_try, rn_try, pn_try
        rate = 0.0 if step_prev is None else step / max(step_prev, 1e-300)
        converged = ((lam == 1.0 and step <= kappa and (info == 0 or step_prev is not None))
                     or (step_prev is not None and lam == 1.0 and info == 0 and rate < 1.0
                         and rate / (1.0 - rate) * step <= kappa)
                     or pn <= kappa)
        if converged:
            if best is None or rn < best[0]:
                best = (rn, z.copy())
            if _cons_ok(cons, R, scale(z), cons_tol):
                return z, True, it + 1, rate, new_lu
            if polish < 2:
                polish += 1
                step_prev = None
                continue
            if stats is not None:
                stats["balance_unclosed"] = stats.get("balance_unclosed", 0) + 1
            return best[1], True, it + 1, rate, new_lu
        if best is not None:
            if stats is not None:
                stats["balance_unclosed"] = stats.get("balance_unclosed", 0) + 1
            return best[1], True, it + 1, rate, new_lu
        if step_prev is not None and lam == 1.0 and info == 0:
            left = max_iter - it - 1
            if it >= 2 and (rate >= 1.0 or rate ** left / (1.0 - rate) * step > kappa * 1e3):
                return z, False, it + 1, rate, new_lu
        step_prev = step
    return z, False, it + 1, 1.0, new_lu


class OracleTRBDF2:
    """Adaptive integrator (core/solver.py:297-511), Krylov Newton mode."""

    def __init__(self, model, cfg, h_max, h_init=None, logger=None):
        s = cfg.solver
        self.m = model
        self.rtol, self.atol = s.rtol, model.atol
        self.h_max = h_max
        self.h_init = h_init if h_init is not None else s.h_initial
        self.max_iter, self.kappa = s.max_newton_iter, s.newton_kappa
        self.jac_max_age, self.max_steps = s.jacobian_max_age, s.max_steps_per_step
        self.jac = OracleFDJacobian(model)
        self.I = sp.identity(model.n_core, format="csc")
        self.stats = {"modified_fail": 0, "krylov_ok": 0, "krylov_fail": 0}
        self._gm = [0]
        self.pos = np.arange(model.off_e)
        self.scheme = s.scheme
        if s.newton_mode != "krylov":
            raise NotImplementedError("oracle restates the default newton_mode=krylov path")
        self.gmres_refresh = s.gmres_refresh
        self.log_refactor = np.log(s.refactor_ratio)
        self.precond = s.preconditioner if model.grid.Nth > 1 else "full"
        self.cons = model.conservation_matrix()
        self.cons_tol = float(s.conservation_tol or 0.0)
        self._new_lu = self._new_J = None
        self._fresh = False
        self.cap_after_fail, self.cap_relax = 0.5, 1.15

    def scale(self, y):
        return self.atol + self.rtol * np.abs(y)

    def _factor(self, J, h):                    # core/solver.py:334-337
        Jp = self.jac.theta_block(J) if self.precond == "theta_block" else J
        return spla.splu((self.I - (D * h) * Jp).tocsc(), permc_spec="COLAMD")

    def _solve_stage(self, t, z0, rhs_known, dh, lu, res):   # core/solver.py:339-368
        h = dh / D

        def refresh(zc):
            fc, _ = self.m.rhs(t, zc, want_acc=False)
            Jn = self.jac(t, zc, fc)
            res.n_jac += 1
            res.n_lu += 1
            self._new_J = (Jn, h)
            return self._factor(Jn, h)

        self._new_J = None
        z, ok, it, rate, new_lu = newton_krylov(self.m, t, z0, rhs_known, dh, lu, self.scale, self.max_iter,
                                                self.kappa, counter=self._gm, pos=self.pos, cons=self.cons,
                                                cons_tol=self.cons_tol, stats=self.stats,
                                                refresh=None if self._fresh else refresh)
        if new_lu is not None:
            self._new_lu = new_lu
        res.n_krylov += 1
        self.stats["krylov_ok" if ok else "krylov_fail"] += 1
        return z, ok, (0.0 if ok else rate)

    def integrate(self, y0, t_end, t_out, on_step=None, stop_fn=None, stop_value=None, stop_direction=1):
        m = self.m
        wall0 = time.time()
        t = 0.0
        y = y0.copy()
        acc = np.zeros(m.n_acc)
        f_n, g_n = m.rhs(t, y)
        res = Result(y=y, acc=acc, t=t)
        t_out = np.asarray(sorted(set(np.clip(t_out, 0.0, t_end)) | {t_end}))
        k_out = 0
        if t_out[0] <= 0.0:
            res.snapshots.append((0.0, y.copy(), acc.copy()))
            k_out = 1
        h = min(self.h_init, self.h_max, t_end)
        J = lu = h_lu = None
        jac_age, fresh, slope_prev, h_cap = 0, False, None, np.inf
        self._gm = [0]
        while t < t_end * (1.0 - 1e-12):
            gm0 = self._gm[0]
            if res.n_steps + res.n_reject + res.n_newton_fail > self.max_steps:
                raise SolverError(f"too many steps in '{m.step['name']}' at t={t:.4g}s")
            t_target = t_out[k_out] if k_out < len(t_out) else t_end
            h_desired = h
            h = min(h, self.h_max, t_target - t)
            truncated = h < h_desired * (1.0 - 1e-9)
            if h < 1e-10 * max(1.0, t_end):
                raise SolverError(f"step size underflow (h={h:.3e}) in '{m.step['name']}' at t={t:.6g}s")
            if J is None or jac_age >= self.jac_max_age:
                J = self.jac(t, y, f_n)
                res.n_jac += 1
                jac_age, fresh, lu = 0, True, None
            if lu is None or abs(np.log(h / h_lu)) > self.log_refactor:
                lu = self._factor(J, h)
                h_lu = h
                res.n_lu += 1
            dh = D * h
            sd = self.scheme == "sdirk2"
            c_mid = G_SD if sd else GAMMA
            rhs1 = y if sd else y + dh * f_n
            z_pred = y if slope_prev is None else _truncate(y + c_mid * h * slope_prev, y, self.pos)
            self._new_lu = None
            self._fresh = fresh
            z1, ok, r1 = self._solve_stage(t + c_mid * h, z_pred, rhs1, dh, lu, res)
            if self._new_lu is not None:
                lu, (J, h_lu) = self._new_lu, self._new_J
                jac_age, fresh, self._new_lu = 0, True, None
            if ok:
                if sd:
                    rhs2 = y + (1.0 - G_SD) * h * ((z1 - y) / dh)
                    z2_pred = _truncate(y + (z1 - y) / G_SD, y, self.pos)
                else:
                    rhs2 = C1 * z1 - C2 * y
                    z2_pred = _truncate(y + (z1 - y) / GAMMA, y, self.pos)
                z2, ok, r2 = self._solve_stage(t + h, z2_pred, rhs2, dh, lu, res)
                if self._new_lu is not None:
                    lu, (J, h_lu) = self._new_lu, self._new_J
                    jac_age, fresh, self._new_lu = 0, True, None
            if not ok:
                res.n_newton_fail += 1
                if not fresh:
                    J = None
                else:
                    h_cap = min(h_cap, self.cap_after_fail * h)
                    h *= 0.3
                    lu = None
                continue
            f1, g1 = m.rhs(t + c_mid * h, z1)
            f2, g2 = m.rhs(t + h, z2)
            if sd:
                y3 = y + h * (SW1 * f_n + SW2 * f1 + SW3 * f2)
            else:
                y3 = y + h * (W1 * f_n + W2 * f1 + W3 * f2)
            err = lu.solve(z2 - y3)
            sc = self.atol + self.rtol * np.maximum(np.abs(y), np.abs(z2))
            en = _rms(err / sc)
            if not np.isfinite(en):
                en = 1e6
            if en > 1.0:
                res.n_reject += 1
                h *= max(0.2, 0.9 * en ** (-1.0 / 3.0))
                continue
            if sd:
                acc = acc + h * ((1.0 - G_SD) * g1 + G_SD * g2)
            else:
                acc_g = acc + D * h * (g_n + g1)
                acc = C1 * acc_g - C2 * acc + D * h * g2
            res.steps.append((t, h))
            slope_prev = (z2 - y) / h
            t_new = t + h
            if stop_fn is not None and stop_value is not None:
                sv = stop_fn(t_new, z2)
                if sv is not None and (sv - stop_value) * stop_direction >= 0.0:
                    t, y, f_n, g_n = t_new, z2, f2, g2
                    res.stopped_early, res.stop_value = True, sv
                    res.n_steps += 1
                    if on_step:
                        on_step(t, y, acc)
                    res.snapshots.append((t, y.copy(), acc.copy()))
                    break
            t, y, f_n, g_n = t_new, z2, f2, g2
            res.n_steps += 1
            jac_age += 1
            fresh = False
            if on_step:
                on_step(t, y, acc)
            if k_out < len(t_out) and t >= t_out[k_out] * (1.0 - 1e-12):
                res.snapshots.append((t, y.copy(), acc.copy()))
                k_out += 1
            if self._gm[0] - gm0 > self.gmres_refresh:
                jac_age = self.jac_max_age
            fac = 4.0 if en < 1e-8 else min(4.0, max(0.2, 0.9 * en ** (-1.0 / 3.0)))
            if 1.0 <= fac < 1.25:
                fac = 1.0
            h = max(h * fac, h_desired) if truncated else h * fac
            h_cap *= self.cap_relax
            h = min(h, h_cap)
        res.y, res.acc, res.t = y, acc, t
        self.stats["gmres_iters"] = self._gm[0]
        res.nfev = m.nfev
        res.wall_time = time.time() - wall0
        return res


def solve_stage_exact(model, jac, t, z0, rhs_known, dh, scale, tol=1e-12, max_iter=30):
    """Full Newton with a fresh exact sparse LU each iteration until RMS(dz/s) <= tol."""
    z = z0.copy()
    I = sp.identity(model.n_core, format="csc")
    for _ in range(max_iter):
        f, _ = model.rhs(t, z, want_acc=False)
        R = z - dh * f - rhs_known
        J = jac(t, z, f)
        dz = spla.splu((I - dh * J).tocsc(), permc_spec="COLAMD").solve(-R)
        z = z + dz
        if _rms(dz / scale(z)) <= tol:
            return z
    raise SolverError("replay stage did not converge")


def fixed_step_run(model, y0, hs, scheme="trbdf2", rtol=1e-4, tol=1e-12):
    """Replay harness: advance over step sizes ``hs`` solving each stage exactly; returns the
    list of step-end states and the accumulator integral (same stage quadrature as integrate)."""
    jac = OracleFDJacobian(model)
    scale = lambda y: model.atol + rtol * np.abs(y)     # noqa: E731
    t, y = 0.0, y0.copy()
    acc = np.zeros(model.n_acc)
    f_n, g_n = model.rhs(t, y)
    out = []
    sd = scheme == "sdirk2"
    c_mid = G_SD if sd else GAMMA
    for h in hs:
        dh = D * h
        rhs1 = y if sd else y + dh * f_n
        z1 = solve_stage_exact(model, jac, t + c_mid * h, y, rhs1, dh, scale, tol)
        rhs2 = (y + (1.0 - G_SD) * h * ((z1 - y) / dh)) if sd else C1 * z1 - C2 * y
        z2 = solve_stage_exact(model, jac, t + h, y + (z1 - y) / c_mid, rhs2, dh, scale, tol)
        f1, g1 = model.rhs(t + c_mid * h, z1)
        f2, g2 = model.rhs(t + h, z2)
        if sd:
            acc = acc + h * ((1.0 - G_SD) * g1 + G_SD * g2)
        else:
            acc = C1 * (acc + D * h * (g_n + g1)) - C2 * acc + D * h * g2
        t, y, f_n, g_n = t + h, z2, f2, g2
        out.append(y.copy())
    return out, acc


def explicit_dt(model, y, safety=0.5):
    """Explicit stability limit (restates numerics/cfl.py:26-56)."""
    g, cfg = model.grid, model.cfg
    d = model.rhs(0.0, y, diag=True)
    P = d["P"]
    eps = model.eps_b
    dp = cfg.sorbent.particle_diameter
    dx_min = min(g.dz, float(np.min(g.dr)), float(np.min(g.r_c * g.dth)) if g.Nth > 1 else np.inf)
    v = float(np.max(np.abs(d["uz"]))) / eps if d["uz"].size else 0.0
    v = max(v, cfg.feed.velocity / eps)
    K = eps ** 3 * dp ** 2 / (150.0 * (1.0 - eps) ** 2)
    D_P = K * float(np.max(P)) / (model.eps_t * 1.8e-5)
    lim = [0.9 * dx_min / max(v, 1e-12), 0.5 * dx_min ** 2 / 1e-4,
           0.5 * dx_min ** 2 * model.rho_b * cfg.sorbent.cp_solid / 0.3, 0.5 * dx_min ** 2 / D_P,
           1.0 / max(cfg.kinetics.k_ldf_co2, cfg.kinetics.k_ldf_h2o)]
    return safety * min(lim)


def integrate_rk4(model, y0, t_end, dt):
    """Classical RK4 with accumulators (restates core/ode_solver.py:19-43)."""
    n = int(np.ceil(t_end / dt))
    dt = t_end / n
    y = y0.copy()
    acc = np.zeros(model.n_acc)
    t = 0.0
    for _ in range(n):
        k1, a1 = model.rhs(t, y)
        k2, a2 = model.rhs(t + 0.5 * dt, y + 0.5 * dt * k1)
        k3, a3 = model.rhs(t + 0.5 * dt, y + 0.5 * dt * k2)
        k4, a4 = model.rhs(t + dt, y + dt * k3)
        y = y + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
        acc += dt / 6.0 * (a1 + 2 * a2 + 2 * a3 + a4)
        t += dt
    return y, acc, t, n
