"""Step runner and cycle driver on the GPU classes.

``run_step`` has the signature and result of the reference's steps/_runner.py:87-188 (build the
model and integrator of one cycle step, record the outlet at every accepted step through
``model.rhs(diag=True)``, return the end state and a ``StepResult``); ``run_cycle`` chains the
steps of ``cfg.cycle`` like vtsa_cycle.py:72-90 without the CSV hand-off (states stay in memory).

``run_cycle_device`` is the device-resident variant used for throughput measurements: the state
stays on the GPU between steps, no outlet recording, only the per-step constants (end pressures
at step start) are read back.
"""
from __future__ import annotations

import gzip
import json
import os
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

import ctypes as C

from . import counters, host
from ._lib import check
from .model import TVSAModel
from .solver import TRBDF2

R_GAS = host.R_GAS


@dataclass
class StepResult:
    name: str
    type: str
    cycle: int
    t_start_cycle: float
    duration_planned: float
    duration: float
    stopped_early: bool
    acc: Dict[str, float]
    inv_start: Dict[str, float]
    inv_end: Dict[str, float]
    outlet: List[Dict] = field(default_factory=list)
    snapshots: List[Dict] = field(default_factory=list)
    solver: Dict = field(default_factory=dict)
    wall_time: float = 0.0
    T_jacket: float = 298.15
    jacket_on: bool = True
    product_port: str = "V3"
    valves: Dict = field(default_factory=dict)
    ads_start: Dict[str, float] = field(default_factory=dict)
    ads_end: Dict[str, float] = field(default_factory=dict)


OUTLET_N = 32          # DV_OUTLET_N: doubles of one device outlet summary (include/dacvtsa.h)
_END_FIELDS = ("flow_out_mol_s", "P_Pa", "T_K")


def feed_co2_concentration(cfg, model) -> float:
    """CO2 concentration of the humid feed [mol/m3] (the reference of the C/C_feed column)."""
    yf = host.humid_air_composition(model.species, cfg.feed.P, cfg.feed.T, cfg.feed.RH if model.water else 0.0,
                                    cfg.feed.y_co2_dry, float(host.arden_buck(cfg.feed.T)))
    return float(yf[model.i_co2] * cfg.feed.P / (R_GAS * cfg.feed.T))


class OutletRecorder:
    """The outlet time series of one cycle step (the reference runner's per-step records).

    Every record is reduced on the GPU from the model's diagnostics (dv_outlet_row) into one row of
    a device ring; the ring is copied to the host once, when the step's rows are assembled.  Host
    side per record: the time and the accumulator integrals (already on the host)."""

    def __init__(self, model, c_feed_co2: float, capacity: int = 1024):
        self.m = model
        self.c_feed = float(c_feed_co2)
        self.ring = torch.empty((capacity, OUTLET_N), dtype=torch.float64, device=model.device)
        self.times: List[float] = []
        self.accs: List[np.ndarray] = []

    def record(self, t: float, y_ptr: int, acc):
        k = len(self.times)
        if k == self.ring.shape[0]:
            self.ring = torch.cat([self.ring, torch.empty_like(self.ring)])
        check(self.m.lib.dv_outlet_row(self.m.handle, float(t), C.c_void_p(y_ptr), self.c_feed,
                                       C.c_void_p(self.ring[k].data_ptr()),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)), "dv_outlet_row")
        self.times.append(float(t))
        self.accs.append(np.array(acc, dtype=float, copy=True))

    @property
    def last_t(self) -> float:
        return self.times[-1] if self.times else -np.inf

    def rows(self, head: Dict) -> List[Dict]:
        """Row dicts with the reference runner's keys; head supplies cycle, step and time offsets."""
        vals = self.ring[:len(self.times)].cpu().numpy()
        counters.d2h(vals.nbytes)
        m = self.m
        ai = m.acc_index
        valve = {e: (m.conds[e].valve or "closed", m.conds[e].state.value) for e in ("top", "bottom")}
        out = []
        for t, v, acc in zip(self.times, vals, self.accs):
            row = {"cycle": head["cycle"], "step": head["step"], "t_step_s": t, "t_cycle_s": head["t_cycle0"] + t,
                   "t_total_s": head["t_total0"] + t}
            for e, end in enumerate(("top", "bottom")):
                b = v[12 * e:12 * e + 12]
                row[f"{end}_valve"], row[f"{end}_valve_state"] = valve[end]
                for q, name in enumerate(_END_FIELDS):
                    row[f"{end}_{name}"] = float(b[q])
                for k, sp in enumerate(m.species):
                    row[f"{end}_y_{sp}"] = float(b[3 + k])
                row[f"{end}_c_CO2_mol_m3"] = float(b[6])
                row[f"{end}_C_over_Cfeed"] = float(b[7])
            row["bed_T_mean_K"], row["bed_P_mean_Pa"] = float(v[24]), float(v[25])
            for n, sp in enumerate(m.adsorbed):
                row[f"bed_q_{sp}_mean"] = float(v[26 + n])
            for vv in ("V1", "V2", "V3"):
                row[f"cum_CO2_out_{vv}_mol"] = float(acc[ai[f"n_out_{vv}_CO2"]])
            row["cum_Q_jacket_J"] = float(acc[ai["Q_jac_pos"]] + acc[ai["Q_jac_neg"]])
            out.append(row)
        return out


def _stop_rule(model, step):
    """(stop_fn, value, direction) of a step's stop_on entry, or Nones (steps/_runner.py semantics)."""
    stop = step.get("stop_on")
    if not stop:
        return None, None, 1
    return model.stop_metric, stop["value"], (-1 if stop["criterion"] == "min_temperature" else 1)


def run_step(state_in, cfg, grid, props, step: Dict, cycle_idx: int = 1, t_cycle0: float = 0.0,
             T_jacket_prev: Optional[float] = None, logger=None, snapshots: Optional[int] = None,
             record_outlet: bool = True):
    """One cycle step on the GPU: same arguments and result as the reference's run_step
    (steps/_runner.py:87-188): the end state and a StepResult with accumulators, inventories,
    solver counters, snapshots and the outlet time series (recorded after every
    outlet_record_every-th accepted step, on the device)."""
    log = logger or (lambda *a, **k: None)
    model = TVSAModel(cfg, grid, props, step, state_in, T_jacket_prev)
    dur = float(step["duration"])
    y0 = model.pack(state_in)
    y0_dev = torch.from_numpy(y0).to(model.device)
    counters.h2d(y0.nbytes)
    rec = OutletRecorder(model, feed_co2_concentration(cfg, model)) if record_outlet else None
    every = max(1, int(cfg.solver.outlet_record_every))
    accepted = [0]

    def after_step(t, y_ptr, acc):
        accepted[0] += 1
        if accepted[0] % every == 0:
            rec.record(t, y_ptr, acc)

    if rec is not None:
        rec.record(0.0, y0_dev.data_ptr(), np.zeros(model.n_acc))
    stop_fn, stop_val, direction = _stop_rule(model, step)
    n_snap = snapshots if snapshots is not None else cfg.run.snapshots_per_step
    wall0 = time.time()
    integ = TRBDF2(model, cfg, h_max=cfg.solver.h_max_fraction * dur)
    res = integ.integrate(y0_dev, dur, np.linspace(0.0, dur, max(2, n_snap)),
                          on_step_device=after_step if rec is not None else None, stop_fn=stop_fn,
                          stop_value=stop_val, stop_direction=direction)
    if rec is not None and rec.last_t < res.t:
        rec.record(res.t, integ.y_ptr(), res.acc)
    wall = time.time() - wall0
    st_out = model.to_state(res.y, state_in, state_in.t + res.t, step["name"])
    st_out.cycle = cycle_idx
    snaps = []
    for ts, ys, _ in res.snapshots:
        s = model.to_state(ys, state_in, state_in.t + ts, step["name"])
        s.cycle = cycle_idx
        snaps.append({"cycle": cycle_idx, "step": step["name"], "t_step": ts, "t_cycle": t_cycle0 + ts,
                      "t_total": state_in.t + ts, "state": s})
    inv_start, inv_end = model.inventories(y0), model.inventories(res.y)
    solver_stats = dict({"method": "trbdf2", "steps": res.n_steps, "rejected": res.n_reject,
                         "newton_fail": res.n_newton_fail, "krylov": res.n_krylov, "jacobians": res.n_jac,
                         "lu": res.n_lu, "nfev": res.nfev, "groups": integ.jac.ngroups}, **integ.stats)
    outlet = rec.rows({"cycle": cycle_idx, "step": step["name"], "t_cycle0": t_cycle0, "t_total0": state_in.t}) \
        if rec is not None else []
    sr = StepResult(name=step["name"], type=step["type"], cycle=cycle_idx, t_start_cycle=t_cycle0,
                    duration_planned=dur, duration=res.t, stopped_early=res.stopped_early,
                    acc=dict(zip(model.acc_names, (float(a) for a in res.acc))), inv_start=inv_start,
                    inv_end=inv_end, outlet=outlet, snapshots=snaps, solver=solver_stats, wall_time=wall,
                    T_jacket=float(model.T_jacket(res.t) if model.jacket_on else cfg.ambient.T),
                    jacket_on=model.jacket_on, product_port=step.get("product_port", "V3"),
                    valves=dict(step["valves"]),
                    ads_start={sp: inv_start[f"ads_{sp}"] for sp in model.adsorbed},
                    ads_end={sp: inv_end[f"ads_{sp}"] for sp in model.adsorbed})
    log(f"    {step['name']:<14s} {res.t:9.1f} s  steps={res.n_steps:>5}  wall={wall:6.2f}s")
    return st_out, sr


def run_cycle(state, cfg, grid, props, cycle_idx: int = 1, T_jac_prev=None, logger=None, record_outlet=True):
    """All steps of cfg.cycle in order (vtsa_cycle.py:72-90, states handed over in memory)."""
    steps_out = []
    t_cycle = 0.0
    for step in cfg.cycle:
        state, sr = run_step(state, cfg, grid, props, step, cycle_idx=cycle_idx, t_cycle0=t_cycle,
                             T_jacket_prev=T_jac_prev, logger=logger, record_outlet=record_outlet)
        t_cycle += sr.duration
        T_jac_prev = sr.T_jacket if sr.jacket_on else T_jac_prev
        steps_out.append(sr)
    return state, steps_out, T_jac_prev


class _PState:
    """State stand-in carrying only the start pressures a model reads."""

    def __init__(self, P):
        self.P = P


def run_cycle_device(y0: torch.Tensor, cfg, grid, props, T_jac_prev=None, predictor=None, predict=True,
                     record_stride=0, writer=None, handoff=None, inventories=False):
    """Device-resident cycle: y stays on the GPU from step to step; returns (y_end, per-step stats).

    Per step only the start pressure field (for the valve ramps) is evaluated, through the model's
    diagnostics kernel on the device state; the hand-off keeps e (internal energy) as the unknown,
    which is what the reference's T round trip (pack(to_state(y))) reproduces to round-off.
    predictor: a NewtonPredictor attached to every step's integrator (predict and/or record samples).
    writer + handoff (template state, cycle index, directory): each step's end state is also written
    as the reference's hand-off CSV by the AsyncStateWriter while the next step runs.
    inventories: each step's stats also carry the bed inventories at its start and end ("inv_start",
    "inv_end"; two host copies of the state per step), the inputs of the balance rows."""
    y = y0
    stats = []
    last_model = None
    for step in cfg.cycle:
        P = last_model.rhs(0.0, y, diag=True)["P"] if last_model is not None else _pressure_host(cfg, grid, props, y)
        model = TVSAModel(cfg, grid, props, step, _PState(P), T_jac_prev)
        dur = float(step["duration"])
        integ = TRBDF2(model, cfg, h_max=cfg.solver.h_max_fraction * dur)
        if predictor is not None:
            predictor.attach(integ, step["type"], predict=predict, record_stride=record_stride)
        inv0 = model.inventories(y) if inventories else None
        res = integ.integrate(y, dur, np.array([dur]), keep_on_device=True)
        y = res.y
        stats.append({"step": step["name"], "steps": res.n_steps, "rejected": res.n_reject, "nfev": res.nfev,
                      "jac": res.n_jac, "lu": res.n_lu, **integ.stats, "t": res.t,
                      "acc": dict(zip(model.acc_names, (float(a) for a in res.acc)))})
        if inventories:
            stats[-1].update(inv_start=inv0, inv_end=model.inventories(y))
        if writer is not None:
            template, cyc, folder = handoff
            writer.submit(y, model, template, template.t + res.t, step["name"], cyc, grid,
                          os.path.join(folder, f"state_after_{step['name']}.csv"))
        T_jac_prev = model.T_jacket(res.t) if model.jacket_on else T_jac_prev
        last_model = model
    return y, stats, T_jac_prev


def cycle_balance_errors(cfg, stats) -> Dict[str, float]:
    """Worst mass / energy balance errors (validation/conservation_checks.py:29-67) of a device cycle
    run with ``inventories=True``."""
    from types import SimpleNamespace
    from . import balances
    steps = [SimpleNamespace(cycle=1, name=st["step"], acc=st["acc"], inv_start=st["inv_start"], inv_end=st["inv_end"],
                             product_port=step.get("product_port", "V3"), valves=dict(step["valves"]))
             for step, st in zip(cfg.cycle, stats)]
    return balances.worst_balance_errors(steps, ("CO2", "H2O", "N2"))


def _pressure_host(cfg, grid, props, y):
    yh = y.detach().cpu().numpy() if isinstance(y, torch.Tensor) else y
    n = grid.ncell
    c = yh[:3 * n].reshape((3,) + grid.shape)
    q = yh[3 * n:5 * n].reshape((2,) + grid.shape)
    e = yh[5 * n:6 * n].reshape(grid.shape)
    so, th = cfg.sorbent, cfg.thermo
    eps_t, rho_b = so.total_voidage, cfg.derived.bulk_density
    cpg = np.asarray(props.cp)
    A = eps_t * (cpg[0] * c[0] + cpg[1] * c[1] + cpg[2] * c[2]) + rho_b * (so.cp_solid + th.cp_ads_co2 * q[0]
                                                                           + th.cp_ads_h2o * q[1])
    B = eps_t * R_GAS * (c[0] + c[1] + c[2])
    Hq = rho_b * (th.dH_ads_co2 * q[0] + th.dH_ads_h2o * q[1])
    T = (e - Hq + A * th.T_ref) / (A - B)
    return (c[0] + c[1] + c[2]) * R_GAS * T


# ---------------------------------------------------------------------------- command line
# Operating point of the cycle benchmark (jackets 288 K, heating 373 K, vacuum 10 kPa, feed 288 K
# at 50 % RH) on top of the reference defaults.
BENCH_POINT = {"solver.scheme": "trbdf2", "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0,
               "operation.T_heat": 373.0, "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5,
               "ambient.T": 288.0}


def main(argv=None):
    """Run one cycle step (or a window of it) of a bed from the seeded constant-pressure state on
    the GPU and print its solver statistics as JSON, like the reference's per-step command lines
    (steps/_runner.py:244): ``python -m dac_vtsa_b200.runner --grid 8 8 32 --step adsorption
    --duration 600``."""
    import argparse
    from .config import load_config
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--grid", type=int, nargs=3, default=(8, 8, 32), metavar=("NR", "NTHETA", "NZ"))
    ap.add_argument("--step", default="adsorption", help="name of a step of the configured cycle")
    ap.add_argument("--duration", type=float, default=None, help="bed-seconds to integrate (default: whole step)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--trace", default=None, metavar="FILE",
                    help="integrate once untraced, then again under a CUDA activity trace (torch.profiler) "
                         "written to FILE (gzipped Chrome JSON); adds the GPU timeline summary to the output")
    a = ap.parse_args(argv)
    over = dict(BENCH_POINT, **{"grid.Nr": a.grid[0], "grid.Ntheta": a.grid[1], "grid.Nz": a.grid[2]})
    cfg = load_config(override_dict=over)
    grid = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, grid, props, seed=a.seed)
    steps = {s["name"]: s for s in cfg.cycle}
    if a.step not in steps:
        raise SystemExit(f"unknown step {a.step!r}; the cycle has {sorted(steps)}")
    step = dict(steps[a.step])
    full = float(step["duration"])
    dur = full if a.duration is None else min(a.duration, full)
    def once():
        model = TVSAModel(cfg, grid, props, step, st)
        integ = TRBDF2(model, cfg, h_max=cfg.solver.h_max_fraction * full)
        y0 = torch.from_numpy(model.pack(st)).to(model.device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = integ.integrate(y0, dur, np.array([dur]), keep_on_device=True)
        torch.cuda.synchronize()
        return res, integ, time.perf_counter() - t0

    res, integ, wall = once()
    out = {"grid": list(a.grid), "step": a.step, "bed_s": res.t, "wall_s": wall, "bed_s_per_wall_s": res.t / wall,
           "steps": res.n_steps, "rejected": res.n_reject, "jac": res.n_jac, "lu": res.n_lu, "nfev": res.nfev,
           **integ.stats}
    if a.trace:
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
            _, _, wall_t = once()
        tmp = a.trace + ".tmp.json"
        prof.export_chrome_trace(tmp)
        with open(tmp, "rb") as f:
            events = json.load(f)["traceEvents"]
        with open(tmp, "rb") as f, gzip.open(a.trace, "wb") as g:
            g.write(f.read())
        os.remove(tmp)
        out["trace"] = dict(timeline_summary(events), wall_s_traced=wall_t, file=a.trace)
    print(json.dumps(out))


def timeline_summary(events, top=8):
    """GPU busy fraction and idle gaps of a CUDA activity trace (Chrome trace events), counted from
    the first preconditioner sweep (model setup excluded): total kernel time, the idle time between
    consecutive device activities by the pair of kernels around it, and the kernels by total time."""
    acts = sorted((e for e in events if e.get("cat") in ("kernel", "gpu_memcpy", "gpu_memset")),
                  key=lambda e: e["ts"])

    def name(e):
        if e.get("cat") != "kernel":
            return e["cat"] + ":" + e["name"].split(" (")[0]
        return e["name"].split("(")[0].replace("void ", "").replace("dv::", "")

    start = next((e["ts"] for e in acts if "k_pc_apply" in e["name"]), acts[0]["ts"] if acts else 0.0)
    acts = [e for e in acts if e["ts"] >= start]
    if not acts:
        return {}
    span = acts[-1]["ts"] + acts[-1]["dur"] - start
    busy = sum(e["dur"] for e in acts if e.get("cat") == "kernel")
    gaps, per_kernel = {}, {}
    for e0, e1 in zip(acts, acts[1:]):
        gap = e1["ts"] - (e0["ts"] + e0["dur"])
        if gap > 5.0:
            key = name(e0) + " -> " + name(e1)
            n, t = gaps.get(key, (0, 0.0))
            gaps[key] = (n + 1, t + gap)
    for e in acts:
        if e.get("cat") == "kernel":
            n, t = per_kernel.get(name(e), (0, 0.0))
            per_kernel[name(e)] = (n + 1, t + e["dur"])
    by_t = lambda d: sorted(d.items(), key=lambda kv: -kv[1][1])[:top]
    return {"span_us": span, "kernel_us": busy, "busy_fraction": busy / span,
            "idle_gaps_over_5us": [{"between": k, "count": n, "total_us": round(t)} for k, (n, t) in by_t(gaps)],
            "kernels": [{"kernel": k, "count": n, "total_us": round(t), "avg_us": round(t / n, 2)}
                        for k, (n, t) in by_t(per_kernel)]}


if __name__ == "__main__":
    main()

