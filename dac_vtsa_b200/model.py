"""TVSAModel on the GPU: drop-in for the reference's core/residual.py:40-482.

Same constructor (cfg, grid, props, step, state0, T_jacket_prev), same attributes
(n_core, n_c, n_q, off_q, off_e, off_w, n_w, ng, na, species, adsorbed, i_co2, i_h2o, water,
n_acc, acc_names, acc_index, atol, nfev, step, conds, jacket_on, grid, cfg, rho_b, eps_t, wall.C)
and methods (rhs, stage_residual, pack, unpack, to_state, inventories, conservation_matrix,
T_jacket, stop_metric, q_feed_eq).  ``rhs`` and ``stage_residual`` run on the GPU through the C
ABI (dv_rhs, dv_stage_residual, dv_rhs_diag).  They accept numpy arrays (copied to and from the
device, like the reference's ownership model) or float64 CUDA tensors (kept on the device).
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace
from typing import Dict, List, Optional

import numpy as np
import torch

from . import counters, host
from ._lib import DV_NACC, DvNewtonOpts, DvNewtonResult, DvStepParams, check, load
from .params import build_params

R_GAS = host.R_GAS


# preconditioner partitions (dv_precond_factor modes)
PRECOND_MODES = {"sector": 0, "full": 1, "theta_block": 2}


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


class _Thermo:
    """T <-> e algebra of physics/energy.py:31-60 on the host (used once per step by pack/to_state)."""

    def __init__(self, m):
        self.eps_t, self.rho_b, self.cp_s, self.T_ref = m.eps_t, m.rho_b, m.cp_s, m.T_ref
        self.cpg, self.cpa, self.dH = m.cpg, m.cpa, m.dH

    def _terms(self, c, q):
        Cg = c[0] + c[1] + c[2]
        gas_cp = self.cpg[0] * c[0] + self.cpg[1] * c[1] + self.cpg[2] * c[2]
        A = self.eps_t * gas_cp + self.rho_b * (self.cp_s + (self.cpa[0] * q[0] + self.cpa[1] * q[1]))
        return A, self.eps_t * R_GAS * Cg, self.rho_b * (self.dH[0] * q[0] + self.dH[1] * q[1])

    def temperature(self, e, c, q):
        A, B, Hq = self._terms(c, q)
        return (e - Hq + A * self.T_ref) / (A - B)

    def energy(self, T, c, q):
        A, B, Hq = self._terms(c, q)
        return A * (T - self.T_ref) - B * T + Hq

    def heat_capacity(self, c, q):
        A, B, _ = self._terms(c, q)
        return A - B


class TVSAModel:
    """Semi-discrete model dy/dt = f(t, y) of one cycle step, evaluated by sm_100a kernels."""

    def __init__(self, cfg, grid, props, step: Dict, state0, T_jacket_prev: Optional[float] = None,
                 device: Optional[torch.device] = None):
        self.lib = load()
        if not torch.cuda.is_available():
            raise RuntimeError("TVSAModel (GPU) needs a CUDA device; the stepping path has no CPU fallback")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.cfg, self.grid, self.props, self.step = cfg, grid, props, step
        g = grid
        gas = props if hasattr(props, "mu_terms") else host.GasData(props.species, cfg.properties.cp_reference_T)
        self.species = list(gas.species)
        self.ng = len(self.species)
        self.water = bool(cfg.components.water)
        self.adsorbed = ["CO2", "H2O"] if self.water else ["CO2"]
        self.na = len(self.adsorbed)
        self.i_co2 = self.species.index("CO2")
        self.i_h2o = self.species.index("H2O") if self.water else None
        self.i_inert = self.species.index("N2")
        self.ads_to_gas = [self.species.index(s) for s in self.adsorbed]
        so, th = cfg.sorbent, cfg.thermo
        self.eps_b, self.eps_t, self.rho_b = so.bed_voidage, so.total_voidage, cfg.derived.bulk_density
        self.cp_s, self.T_ref = so.cp_solid, th.T_ref
        self.cpg = np.asarray(gas.cp, dtype=float)
        self.cpa = np.array([th.cp_ads_co2, th.cp_ads_h2o])
        self.dH = np.array([th.dH_ads_co2, th.dH_ads_h2o])
        self.thermo = _Thermo(self)
        P0 = state0.P
        self.P_start = {"top": float(np.mean(P0[:, :, 0])), "bottom": float(np.mean(P0[:, :, -1]))}
        self.params, feed, nnom, cov, ex = build_params(cfg, g, gas, step, self.P_start, T_jacket_prev)
        self.conds = ex["conds"]
        self.jacket_on = bool(self.params.jacket_on)
        self.T_jac_set = self.params.T_jac_set
        self.T_jac_prev = self.params.T_jac_prev
        self.jac_tau = self.params.jac_tau
        self.tau_valve = cfg.operation.valve_time_constant
        self.u_nom = self.params.u_nom
        self.feed_flux = feed
        self.cov = cov
        w = cfg.wall
        self.wall = SimpleNamespace(enabled=bool(w.enabled), C=w.density * w.cp * g.V_wall, T_ref=th.T_ref)
        n = g.ncell
        self.n_c, self.n_q = self.ng * n, self.na * n
        self.off_q, self.off_e = self.n_c, self.n_c + self.n_q
        self.off_w = self.off_e + n
        self.n_w = g.Nth * g.Nz if self.wall.enabled else 0
        self.n_core = self.off_w + self.n_w
        self.acc_names = self._acc_names()
        self.n_acc = len(self.acc_names)
        self.acc_index = {nm: i for i, nm in enumerate(self.acc_names)}
        parts = [np.full(n, a) for a in self.params.atol[:6]]
        if self.n_w:
            parts.append(np.full(self.n_w, self.params.atol[6]))
        self.atol = np.concatenate(parts)
        self._nfev_host = 0
        with torch.cuda.device(self.device):
            h = C.c_void_p()
            check(self.lib.dv_model_create(C.byref(self.params), feed.ctypes.data, nnom.ctypes.data,
                                           cov.ctypes.data, C.byref(h)), "dv_model_create")
            self.handle = h
            sz = [C.c_int64() for _ in range(5)]
            check(self.lib.dv_model_sizes(h, *[C.byref(x) for x in sz]), "dv_model_sizes")
            self.jac_doubles, self.diag_doubles = sz[3].value, sz[4].value
            assert sz[0].value == self.n_core
            self._y = torch.empty(self.n_core, dtype=torch.float64, device=self.device)
            self._f = torch.empty(self.n_core, dtype=torch.float64, device=self.device)
            self._b = torch.empty(self.n_core, dtype=torch.float64, device=self.device)
            self._acc = torch.empty(DV_NACC, dtype=torch.float64, device=self.device)
            self._diag = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.dv_model_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------------ layout helpers
    def _acc_names(self) -> List[str]:
        names = []
        for v in ("V1", "V2", "V3"):
            names += [f"n_in_{v}_{s}" for s in self.species] + [f"n_out_{v}_{s}" for s in self.species]
            names += [f"H_in_{v}", f"H_out_{v}", f"W_pump_{v}", f"W_fan_{v}"]
        names += ["Q_jac_pos", "Q_jac_neg", "Q_amb", "Q_wb", "Q_hx_pos", "Q_hx_neg"]
        return names

    @property
    def nfev(self) -> int:
        return int(self.lib.dv_model_nfev(self.handle))

    # ------------------------------------------------------------------ state layout
    def _blocks(self):
        """(name, slice, shape) of every variable block of y in order: the gas species, the adsorbed
        species, e and (with a wall) Tw -- the variable-major layout of core/residual.py:110-118."""
        g, n = self.grid, self.grid.ncell
        out = [(f"c_{sp}", slice(k * n, (k + 1) * n), g.shape) for k, sp in enumerate(self.species)]
        out += [(f"q_{sp}", slice(self.off_q + j * n, self.off_q + (j + 1) * n), g.shape)
                for j, sp in enumerate(self.adsorbed)]
        out.append(("e", slice(self.off_e, self.off_w), g.shape))
        if self.n_w:
            out.append(("Tw", slice(self.off_w, self.n_core), g.wall_shape))
        return out

    def _weights(self):
        """Per-unknown weights of the four balances: moles of each gas species (gas + adsorbed,
        rows 0..ng-1) and energy of bed and wall (row ng); W @ y are the inventories."""
        if getattr(self, "_W", None) is None:
            Vc = np.broadcast_to(self.grid.V, self.grid.shape).ravel()
            W = np.zeros((self.ng + 1, self.n_core))
            for name, sl, _ in self._blocks():
                kind, sp = name.split("_", 1) if "_" in name else (name, None)
                if kind == "c":
                    W[self.species.index(sp), sl] = self.eps_t * Vc
                elif kind == "q":
                    W[self.species.index(sp), sl] = self.rho_b * Vc
                elif name == "e":
                    W[self.ng, sl] = Vc
                else:
                    W[self.ng, sl] = self.wall.C
            self._W = W
        return self._W

    def conservation_matrix(self):
        """Sparse W (ng+1, n_core) with W @ y = inventories (core/residual.py:146-168)."""
        import scipy.sparse as sp
        return sp.csr_matrix(self._weights())

    def pack(self, st) -> np.ndarray:
        """CycleState -> y (core/residual.py:170-183); e from T by the host thermo algebra."""
        y = np.empty(self.n_core)
        src = {f"c_{sp}": st.c[k] for k, sp in enumerate(self.species)}
        src.update({f"q_{sp}": st.q[j] for j, sp in enumerate(self.adsorbed)})
        src["e"] = self.thermo.energy(st.T, st.c, st.q)
        if self.n_w:
            src["Tw"] = st.Tw
        for name, sl, _ in self._blocks():
            y[sl] = np.asarray(src[name]).ravel()
        return y

    def unpack(self, y):
        """y -> (c, q, e, Tw) views (core/residual.py:185-190); Tw is None without a wall."""
        if isinstance(y, torch.Tensor):
            y = y.detach().cpu().numpy()
        parts = {name: y[sl].reshape(shape) for name, sl, shape in self._blocks()}
        c = np.stack([parts[f"c_{sp}"] for sp in self.species])
        q = np.stack([parts[f"q_{sp}"] for sp in self.adsorbed])
        return c, q, parts["e"], parts.get("Tw")

    def to_state(self, y, template, t_abs: float, step_name: str):
        """y -> CycleState at absolute time t_abs (core/residual.py:192-202)."""
        c, q, e, Tw = self.unpack(y)
        st = template.copy()
        st.c, st.q = c.copy(), q.copy()
        st.T = self.thermo.temperature(e, c, q)
        st.Tw = st.T[-1].copy() if Tw is None else Tw.copy()
        st.t, st.step = t_abs, step_name
        return st

    def T_jacket(self, t):
        """Jacket temperature: first-order approach from the previous step's to the set point."""
        lag = np.exp(-t / self.jac_tau) if self.jac_tau > 0 else 0.0
        return self.T_jac_set + (self.T_jac_prev - self.T_jac_set) * lag

    # ------------------------------------------------------------------ device plumbing
    def _to_dev(self, y, buf):
        if isinstance(y, torch.Tensor):
            if y.device != self.device or y.dtype != torch.float64 or not y.is_contiguous():
                raise ValueError("device inputs must be contiguous float64 tensors on the model's device")
            return y, True
        a = np.ascontiguousarray(y, dtype=np.float64)
        if a.shape != (self.n_core,):
            raise ValueError(f"state vector must have shape ({self.n_core},), got {a.shape}")
        buf.copy_(torch.from_numpy(a), non_blocking=False)
        counters.h2d(a.nbytes)
        return buf, False

    # ------------------------------------------------------------------ RHS
    def rhs(self, t: float, y, want_acc: bool = True, diag: bool = False):
        """(dy/dt, accumulator rates) -- or the diagnostics dict if diag=True (core/residual.py:211-417)."""
        with torch.cuda.device(self.device):
            yd, on_dev = self._to_dev(y, self._y)
            if diag:
                return self._diag_dict(t, yd)
            f = torch.empty_like(yd) if on_dev else self._f
            acc = self._acc if want_acc else None
            check(self.lib.dv_rhs(self.handle, float(t), _ptr(yd), _ptr(f), _ptr(acc) if acc is not None else None,
                                  _stream()), "dv_rhs")
            if on_dev:
                return f, (acc.clone() if acc is not None else None)
            fh = f.cpu().numpy()
            counters.d2h(fh.nbytes + (8 * DV_NACC if acc is not None else 0))
            return fh, (acc.cpu().numpy() if acc is not None else None)

    def stage_residual(self, t, y, gamma_h, rhs_known):
        """R(y) = y - gamma_h f(t, y) - rhs_known (core/residual.py:420-423)."""
        with torch.cuda.device(self.device):
            yd, on_dev = self._to_dev(y, self._y)
            kd, _ = self._to_dev(rhs_known, self._b)
            R = torch.empty_like(yd) if on_dev else self._f
            check(self.lib.dv_stage_residual(self.handle, float(t), _ptr(yd), float(gamma_h), _ptr(kd), _ptr(R),
                                             _stream()), "dv_stage_residual")
            if on_dev:
                return R
            counters.d2h(8 * self.n_core)
            return R.cpu().numpy()

    def _diag_dict(self, t, yd):
        g = self.grid
        if self._diag is None:
            self._diag = torch.empty(self.diag_doubles, dtype=torch.float64, device=self.device)
        check(self.lib.dv_rhs_diag(self.handle, float(t), _ptr(yd), _ptr(self._diag), _stream()), "dv_rhs_diag")
        d = self._diag.cpu().numpy()
        counters.d2h(d.nbytes)
        Nr, Nth, Nz = g.shape
        nc, nf, nw = g.ncell, Nr * Nth, Nth * Nz
        o = 0

        def take(cnt, shape):
            nonlocal o
            a = d[o:o + cnt].reshape(shape)
            o += cnt
            return a
        T = take(nc, g.shape)
        P = take(nc, g.shape)
        yk = take(3 * nc, (3,) + g.shape)
        qstar = take(2 * nc, (2,) + g.shape)
        uz = take(nf * (Nz - 1), (Nr, Nth, Nz - 1))
        ur = take((Nr - 1) * Nth * Nz, (Nr - 1, Nth, Nz))
        uth = take(nc, g.shape)
        bnd_raw = take(2 * 16 * nf, (2, 16, Nr, Nth))
        Qj, Qa, Qw, Rb = (take(nw, (Nth, Nz)) for _ in range(4))
        Qhx = take(nc, g.shape)
        bnd = {}
        for e, end in enumerate(("top", "bottom")):
            b = bnd_raw[e]
            rec = {"F_in": b[0:3].copy(), "H_in": b[3].copy(), "u_out": b[4].copy(), "P_face": b[5].copy()}
            if self.conds[end].kind == "valve":
                rec.update({"F_inpart": b[6:9].copy(), "F_outpart": b[9:12].copy(), "H_inpart": b[12].copy(),
                            "H_outpart": b[13].copy()})
            bnd[end] = rec
        if self.wall.enabled:
            Q_jac, Q_amb, Q_wb = Qj.copy(), Qa.copy(), Qw.copy()
        else:
            Q_jac, Q_amb, Q_wb = Qj.copy(), Qa.copy(), Qw.copy()
        return {"T": T.copy(), "P": P.copy(), "y": yk.copy(), "qstar": qstar.copy(), "uz": uz.copy(),
                "ur": ur.copy() if Nr > 1 else None, "uth": uth.copy() if Nth > 1 else None, "bnd": bnd,
                "Q_jac": Q_jac, "Q_wb": Q_wb, "Q_amb": Q_amb,
                "Q_hx": Qhx.copy() if self.params.hx_on else None,
                "R_bed": (1.0 / self.cfg.transport.lumped_U) if self.params.lumped else Rb.copy()}

    # ------------------------------------------------------------------ linear algebra entry points
    def set_krylov_precision(self, precision: str):
        """"fp64" (default), "fp32_factors" (the preconditioner factors the sweep streams are FP32;
        takes effect at the next factorisation) or "fp32" (those factors and GMRES on the FP32
        assembled Jacobian, refreshed by newton_stage at its start)."""
        masks = {"fp64": 0, "fp32_factors": 1, "fp32": 3}
        if precision not in masks:
            raise ValueError(f"krylov precision must be one of {sorted(masks)}, not {precision!r}")
        check(self.lib.dv_model_set_krylov_fp32(self.handle, masks[precision]), "dv_model_set_krylov_fp32")

    def precond_factor(self, J_block: torch.Tensor, dh: float, mode: str = "theta_block"):
        """Factorise I - dh J (block layout J) along z per partition: "theta_block" (the innermost ring
        of all sectors as one partition, rings 1.. of each sector as the others), "sector" (whole
        sectors) or "full" (whole cross-sections)."""
        with torch.cuda.device(self.device):
            check(self.lib.dv_precond_factor(self.handle, _ptr(J_block), float(dh), PRECOND_MODES[mode],
                                             _stream()), "dv_precond_factor")

    def precond_partitions(self):
        """(mode, first twisted separator plane, block size of every partition) of the stored factors."""
        mode, zs, npart = C.c_int32(), C.c_int32(), C.c_int32()
        nb = np.zeros(4096, dtype=np.int32)
        check(self.lib.dv_precond_partitions(self.handle, C.byref(mode), C.byref(zs), nb.ctypes.data, nb.size,
                                             C.byref(npart)), "dv_precond_partitions")
        return mode.value, zs.value, nb[:npart.value].tolist()

    def precond_solve(self, b):
        """x = M^-1 b with the stored factors (the reference's lu.solve)."""
        with torch.cuda.device(self.device):
            bd, on_dev = self._to_dev(b, self._b)
            x = torch.empty_like(bd)
            check(self.lib.dv_precond_solve(self.handle, _ptr(bd), _ptr(x), _stream()), "dv_precond_solve")
            return x if on_dev else x.cpu().numpy()

    def newton_stage(self, t, z0, rhs_known, dh, max_iter=7, kappa=0.01, eta=1e-2, rtol=None, cons_tol=None,
                     krylov_dim=30, allow_refresh=False, precond_mode="theta_block"):
        """Solve z - dh f(t, z) = rhs_known by Newton-Krylov (core/solver.py:154-294) from z0 using the
        stored factors.  Returns (z device tensor, ok, iterations, rate, stats dict)."""
        s = self.cfg.solver
        o = DvNewtonOpts()
        o.max_iter, o.krylov_dim, o.allow_refresh = int(max_iter), int(krylov_dim), int(bool(allow_refresh))
        o.precond_mode = PRECOND_MODES[precond_mode]
        o.kappa, o.eta = float(kappa), float(eta)
        o.rtol = float(s.rtol if rtol is None else rtol)
        o.cons_tol = float((s.conservation_tol or 0.0) if cons_tol is None else cons_tol)
        r = DvNewtonResult()
        with torch.cuda.device(self.device):
            z0d = z0 if isinstance(z0, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(z0)).to(self.device)
            kd = rhs_known if isinstance(rhs_known, torch.Tensor) else \
                torch.from_numpy(np.ascontiguousarray(rhs_known)).to(self.device)
            z = torch.empty_like(z0d)
            check(self.lib.dv_newton_stage(self.handle, float(t), _ptr(z0d), _ptr(kd), float(dh), C.byref(o),
                                           _ptr(z), C.byref(r), _stream()), "dv_newton_stage")
        stats = {"gmres_iters": r.gmres_iters, "gmres_polish": r.gmres_polish,
                 "balance_unclosed": r.balance_unclosed, "jac_refresh_in_newton": r.jac_refresh_in_newton}
        return z, bool(r.ok), int(r.iters), float(r.rate), stats

    # ------------------------------------------------------------------ inventories / diagnostics
    def inventories(self, y) -> Dict[str, float]:
        """Moles of each species (gas + adsorbed) and bed + wall energy (core/residual.py:426-443)."""
        if isinstance(y, torch.Tensor):
            y = y.detach().cpu().numpy()
        W = self._weights()
        out = {}
        for k, sp in enumerate(self.species):
            gas = sum(float(W[k, sl] @ y[sl]) for name, sl, _ in self._blocks() if name == f"c_{sp}")
            ads = sum(float(W[k, sl] @ y[sl]) for name, sl, _ in self._blocks() if name == f"q_{sp}")
            out[f"gas_{sp}"], out[f"ads_{sp}"], out[f"tot_{sp}"] = gas, ads, gas + ads
        blocks = {name: sl for name, sl, _ in self._blocks()}
        out["E_bed"] = float(W[self.ng, blocks["e"]] @ y[blocks["e"]])
        out["E_wall"] = (float(self.wall.C * np.sum(y[blocks["Tw"]] - self.wall.T_ref)) if "Tw" in blocks else 0.0)
        out["E_total"] = out["E_bed"] + out["E_wall"]
        return out

    def q_feed_eq(self) -> float:
        """Equilibrium CO2 loading with the feed gas (core/residual.py:471-482), via a one-cell evaluation
        of the device isotherms would be overkill: closed-form host evaluation of the same formulas."""
        cfg = self.cfg
        T = cfg.feed.T
        psat = float(host.arden_buck(T))
        yv = host.humid_air_composition(self.species, cfg.feed.P, T, cfg.feed.RH, cfg.feed.y_co2_dry, psat)
        p = yv * cfg.feed.P
        return float(_q_co2_host(cfg, p[self.i_co2], T, _q_h2o_host(cfg, p[self.i_h2o], T, psat)))

    def _summary(self, t, y) -> np.ndarray:
        """The device outlet summary (dv_outlet_row, DV_OUTLET_N doubles) of state y."""
        with torch.cuda.device(self.device):
            yd, _ = self._to_dev(y, self._y)
            if getattr(self, "_row", None) is None:
                self._row = torch.empty(32, dtype=torch.float64, device=self.device)
            check(self.lib.dv_outlet_row(self.handle, float(t), _ptr(yd), 0.0, _ptr(self._row), _stream()),
                  "dv_outlet_row")
            v = self._row.cpu().numpy()
            counters.d2h(v.nbytes)
            return v

    def stop_metric(self, t, y) -> Optional[float]:
        """Value of the step's stop criterion at (t, y) (core/residual.py:445-469), from the device
        summary: bed mean temperature, CO2 loading of the last layer over the feed equilibrium, or the
        CO2 fraction leaving the product end over the feed's."""
        stop = self.step.get("stop_on")
        if not stop:
            return None
        crit = stop["criterion"]
        if crit not in ("min_temperature", "max_temperature", "end_saturation", "outlet_ratio"):
            return None
        v = self._summary(t, y)
        if crit in ("min_temperature", "max_temperature"):
            return float(v[24])
        if crit == "end_saturation":
            return float(v[12 + 10] / self.q_feed_eq())
        end = 1 if self.conds["top"].kind == "feed" else 0
        y_ext = self.conds["top"].y_ext
        yf = y_ext[self.i_co2] if y_ext is not None else 4e-4
        return float(v[12 * end + 9] / yf)

def _toth_host(p, T, q_inf0, chi, b0, dH0, tau0, alpha, T0):
    p = max(p, 0.0)
    qinf = q_inf0 * np.exp(chi * (1.0 - T / T0))
    b = b0 * np.exp(-dH0 / (R_GAS * T))
    tau = tau0 + alpha * (1.0 - T0 / T)
    bp = b * p
    return qinf * bp / (1.0 + bp ** tau) ** (1.0 / tau)


def _q_h2o_host(cfg, pw, T, psat):
    h = cfg.isotherm.h2o
    x = max(pw / psat, -0.2)
    lo = h.rh_cap - 0.02
    over = max(x - lo, 0.0)
    x = x if x <= lo else (h.rh_cap if over >= 0.04 else lo + over - over ** 2 / 0.08)
    E1 = h.C - np.exp(h.D * T)
    E29 = h.F + h.G * T
    E10 = h.E10_slope * T + h.E10_intercept
    c = np.exp((E1 - E10) / (R_GAS * T))
    k = np.exp((E29 - E10) / (R_GAS * T))
    kx = k * x
    return h.q_m * c * kx / ((1.0 - kx) * (1.0 + (c - 1.0) * kx))


def _q_co2_host(cfg, p, T, qw):
    iso = cfg.isotherm
    c = iso.co2
    co = iso.coadsorption
    pp = max(p, 0.0)
    dry = (c.q_inf0, c.chi, c.b0, c.dH0, c.tau0, c.alpha, c.T0)
    qw = max(qw, 1e-12)
    if co.model == "none":
        raw = _toth_host(pp, T, *dry)
    elif co.model == "wadst":
        wd = co.wadst
        w = np.exp(-wd.A / qw)
        raw = (1.0 - w) * _toth_host(pp, T, *dry) + w * _toth_host(pp, T, wd.q_inf0_wet, wd.chi_wet, wd.b0_wet,
                                                                   wd.dH_wet, wd.tau0_wet, wd.alpha_wet, c.T0)
    elif co.model == "mechanistic":
        m = co.mechanistic
        w = np.exp(-m.A / qw)
        f_bl = m.f_blocked_max * (1.0 - np.exp(-(m.k * qw) ** m.n))
        phi = m.phi_dry + ((1.0 - f_bl) - m.phi_dry) * w
        raw = (phi / m.phi_dry) * _toth_host(pp, T, c.q_inf0, c.chi, c.b0, (1.0 - w) * c.dH0 + w * m.dH_wet,
                                             c.tau0, c.alpha, c.T0)
    else:
        sb = co.stampi_bombelli
        raw = _toth_host(pp, T, c.q_inf0 / (1.0 - sb.gamma * qw), c.chi, c.b0 * (1.0 + sb.beta * qw), c.dH0,
                         c.tau0, c.alpha, c.T0)
    return raw * (pp / (pp + c.p_regularization))
