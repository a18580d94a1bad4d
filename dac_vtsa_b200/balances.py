"""Cycle accounting on the host from the step results: balance closure, CO2 flows and the cyclic-
steady-state test.

These are the reference's acceptance metrics, computed from the integrated accumulators and the
inventories of each StepResult:

* balance closure per step and species / energy, relative to the larger of the step's own flows and
  a floor of 1e-3 of the cycle's throughput (validation/conservation_checks.py:29-67 with
  postprocessing/reporting.py:113-140); ``worst_balance_errors`` gives the two numbers the cycle log
  prints;
* fed / product / vented CO2 of a cycle (postprocessing/reporting.py:30-49) and its closure
  (validation/cyclic_steady_state.py:37-39);
* the state change between consecutive cycle ends, volume-weighted RMS with the reference's scales
  (validation/cyclic_steady_state.py:22-34), and the CSS decision (:42-44).
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

VALVES = ("V1", "V2", "V3")
FLOOR = 1e-3


def _valve_sum(acc: Dict[str, float], prefix: str, sp: str) -> float:
    return float(sum(acc.get(f"{prefix}_{v}_{sp}", 0.0) for v in VALVES))


def _energy_terms(acc: Dict[str, float]) -> Dict[str, float]:
    return {"H_in_J": float(sum(acc.get(f"H_in_{v}", 0.0) for v in VALVES)),
            "H_out_J": float(sum(acc.get(f"H_out_{v}", 0.0) for v in VALVES)),
            "Q_jacket_J": float(acc["Q_jac_pos"] + acc["Q_jac_neg"]),
            "Q_internal_hx_J": float(acc["Q_hx_pos"] + acc["Q_hx_neg"]),
            "Q_ambient_J": float(acc["Q_amb"])}


def balance_rows(steps: Sequence, species: Sequence[str]):
    """(mass rows, energy rows) of a cycle: one row per step and species / per step, then the whole
    cycle's row; each row carries its residual and relative error."""
    thr = {sp: sum(_valve_sum(sr.acc, "n_in", sp) + _valve_sum(sr.acc, "n_out", sp) for sr in steps)
           for sp in species}
    e_thr = 0.0
    for sr in steps:
        a = sr.acc
        e_thr += sum(abs(a.get(f"H_in_{v}", 0.0)) + abs(a.get(f"H_out_{v}", 0.0)) for v in VALVES)
        e_thr += sum(abs(a[k]) for k in ("Q_jac_pos", "Q_jac_neg", "Q_hx_pos", "Q_hx_neg", "Q_amb"))
    mass, energy = [], []
    for sr in steps:
        for sp in species:
            a, b = sr.inv_start[f"tot_{sp}"], sr.inv_end[f"tot_{sp}"]
            fin, fout = _valve_sum(sr.acc, "n_in", sp), _valve_sum(sr.acc, "n_out", sp)
            res = (b - a) - (fin - fout)
            den = max(abs(fin), abs(fout), abs(a), abs(b), FLOOR * max(thr[sp], 1e-30))
            mass.append({"cycle": sr.cycle, "step": sr.name, "species": sp, "inventory_start_mol": a,
                         "inventory_end_mol": b, "in_mol": fin, "out_mol": fout, "residual_mol": res,
                         "relative_error": res / den})
        E0, E1 = sr.inv_start["E_total"], sr.inv_end["E_total"]
        t = _energy_terms(sr.acc)
        res = (E1 - E0) - (t["H_in_J"] - t["H_out_J"] + t["Q_jacket_J"] + t["Q_internal_hx_J"] + t["Q_ambient_J"])
        den = max(abs(E1 - E0), *(abs(v) for v in t.values()), FLOOR * e_thr, 1e-30)
        energy.append({"cycle": sr.cycle, "step": sr.name, "E_start_J": E0, "E_end_J": E1, "dE_J": E1 - E0, **t,
                       "residual_J": res, "relative_error": res / den})
    for sp in species:
        a, b = steps[0].inv_start[f"tot_{sp}"], steps[-1].inv_end[f"tot_{sp}"]
        rows = [r for r in mass if r["species"] == sp]
        fin, fout = sum(r["in_mol"] for r in rows), sum(r["out_mol"] for r in rows)
        res = (b - a) - (fin - fout)
        mass.append({"cycle": steps[0].cycle, "step": "CYCLE", "species": sp, "inventory_start_mol": a,
                     "inventory_end_mol": b, "in_mol": fin, "out_mol": fout, "residual_mol": res,
                     "relative_error": res / max(abs(fin), abs(fout), abs(a), 1e-30)})
    E0, E1 = steps[0].inv_start["E_total"], steps[-1].inv_end["E_total"]
    tot = {k: sum(r[k] for r in energy) for k in ("H_in_J", "H_out_J", "Q_jacket_J", "Q_internal_hx_J", "Q_ambient_J")}
    res = (E1 - E0) - (tot["H_in_J"] - tot["H_out_J"] + tot["Q_jacket_J"] + tot["Q_internal_hx_J"] + tot["Q_ambient_J"])
    energy.append({"cycle": steps[0].cycle, "step": "CYCLE", "E_start_J": E0, "E_end_J": E1, "dE_J": E1 - E0, **tot,
                   "residual_J": res, "relative_error": res / max(abs(E1 - E0), *(abs(v) for v in tot.values()), 1e-30)})
    return mass, energy


def worst_balance_errors(steps: Sequence, species: Sequence[str]) -> Dict[str, float]:
    mass, energy = balance_rows(steps, species)
    return {"mass": max(abs(r["relative_error"]) for r in mass),
            "energy": max(abs(r["relative_error"]) for r in energy)}


def co2_flows(steps: Sequence) -> Dict[str, float]:
    """Fed, product (out of the step's product port when that valve is open) and vented CO2 [mol]."""
    fed = prod = out = 0.0
    for sr in steps:
        fed += _valve_sum(sr.acc, "n_in", "CO2")
        allout = _valve_sum(sr.acc, "n_out", "CO2")
        pp = sr.product_port
        if pp in VALVES and sr.valves.get(pp, "CLOSED") != "CLOSED":
            prod += float(sr.acc.get(f"n_out_{pp}_CO2", 0.0))
        out += allout
    return {"CO2_fed_mol": fed, "CO2_product_mol": prod, "CO2_vented_mol": out - prod}


def cycle_co2_balance(flows: Dict[str, float]) -> float:
    fed = flows["CO2_fed_mol"]
    return abs(fed - flows["CO2_product_mol"] - flows["CO2_vented_mol"]) / fed if fed > 0 else float("inf")


def state_change(prev, now, grid, cfg) -> Dict[str, float]:
    """Volume-weighted RMS change of each field between two cycle-end states, scaled: loadings by
    their RMS, T by the heating swing, concentrations by the RMS total concentration."""
    w = np.asarray(grid.volume_full())
    rms = lambda a: float(np.sqrt(np.sum(w * a * a) / np.sum(w)))
    out = {}
    for n, sp in enumerate(now.adsorbed):
        out[f"q_{sp}"] = rms(now.q[n] - prev.q[n]) / max(rms(now.q[n]), 1e-6)
    out["T"] = rms(now.T - prev.T) / max(cfg.operation.T_heat - cfg.feed.T, 1.0)
    Csc = max(rms(now.c.sum(axis=0)), 1e-9)
    for k, sp in enumerate(now.species):
        out[f"c_{sp}"] = rms(now.c[k] - prev.c[k]) / Csc
    out["max"] = max(out.values())
    return out


def is_css(change: Dict[str, float], flows: Dict[str, float], cfg, cycle: int) -> bool:
    return (cycle >= cfg.run.min_cycles and change["max"] < cfg.run.css_tolerance
            and cycle_co2_balance(flows) < cfg.run.css_mb_tolerance)
