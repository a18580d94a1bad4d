"""Cycles to cyclic steady state with the state kept on the GPU (the reference's vtsa_cycle.run_to_css,
vtsa_cycle.py:93-138, and validation/cyclic_steady_state.py:22-44).

Each cycle runs its steps device-resident (runner.run_cycle_device); per cycle one host copy of the
end state feeds the state-change measure, and the step accumulators give the cycle's CO2 flows.  With
``run_dir`` every step's end state is also written as the reference's hand-off CSV
(cycle_NNN/state_after_<step>.csv) by a background writer while the GPU continues.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field
from types import SimpleNamespace
from typing import Dict, List, Optional

import numpy as np
import torch

from . import balances, host
from .handoff import AsyncStateWriter, save_state_csv
from .model import TVSAModel
from .runner import run_cycle_device


@dataclass
class CycleRecord:
    cycle: int
    change: Dict[str, float]
    co2: Dict[str, float]
    co2_balance: float
    wall_time: float
    solver: List[Dict] = field(default_factory=list)


@dataclass
class CssResult:
    cycles: List[CycleRecord]
    final_state: object
    converged: bool
    y_end: Optional[torch.Tensor] = None


def _step_records(cfg, stats):
    return [SimpleNamespace(acc=st["acc"], product_port=step.get("product_port", "V3"), valves=dict(step["valves"]))
            for step, st in zip(cfg.cycle, stats)]


def run_to_css(cfg, grid=None, props=None, state=None, run_dir: Optional[str] = None,
               max_cycles: Optional[int] = None, log=None, predictor=None) -> CssResult:
    log = log or (lambda *a, **k: None)
    grid = grid or host.Grid.from_config(cfg)
    props = props or host.get_backend(cfg)
    state = state or host.initial_state(cfg, grid, props)
    m0 = TVSAModel(cfg, grid, props, cfg.cycle[0], state)
    y = torch.from_numpy(m0.pack(state)).to(m0.device)
    writer = AsyncStateWriter() if run_dir else None
    records, prev_end, T_jac, converged = [], state.copy(), None, False
    n_max = max_cycles or cfg.run.max_cycles
    now = state
    try:
        for n in range(1, n_max + 1):
            t0 = time.perf_counter()
            handoff = None
            if run_dir:
                cdir = os.path.join(run_dir, f"cycle_{n:03d}")
                os.makedirs(cdir, exist_ok=True)
                save_state_csv(now, grid, os.path.join(cdir, "state_cycle_start.csv"))
                handoff = (now, n, cdir)
            y, stats, T_jac = run_cycle_device(y, cfg, grid, props, T_jac, predictor=predictor, writer=writer,
                                               handoff=handoff)
            now = m0.to_state(y.cpu().numpy(), state, prev_end.t + sum(st["t"] for st in stats), cfg.cycle[-1]["name"])
            now.cycle = n
            ch = balances.state_change(prev_end, now, grid, cfg)
            flows = balances.co2_flows(_step_records(cfg, stats))
            rec = CycleRecord(n, ch, flows, balances.cycle_co2_balance(flows), time.perf_counter() - t0, stats)
            records.append(rec)
            log(f"cycle {n}: CSS change {ch['max']:.2e}  CO2 cycle balance {rec.co2_balance:.2e}  "
                f"| {rec.wall_time:.1f} s")
            if balances.is_css(ch, flows, cfg, n):
                converged = True
                break
            prev_end = now
    finally:
        if writer is not None:
            writer.close()
    return CssResult(records, now, converged, y)
