"""Ensemble of independent columns with uneven grids and operating points, solved concurrently on one GPU.

The reference runs independent cases as separate processes (analysis/sensitivity.py:121).  Here every
column gets its own model, integrator and CUDA stream, and a host thread that drives its full cycle
(runner.run_cycle_device); the library's calls release the interpreter lock, so the columns' small
kernels overlap on the GPU instead of running one column at a time.  Each column may carry its own
copy of the learned predictor (the network's inference buffers are per copy) and the mixed-precision
Krylov setting.

``draw_columns(n, seed)`` draws the ensemble of the batched-ensemble study: nr, ntheta in {4, 8, 16},
nz in {16, 32, 64}, T_heat ~ U(363, 393) K, P_vacuum ~ U(5, 30) kPa, feed RH ~ U(0.2, 0.8), feed CO2 ~
U(350, 450) ppm.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import host
from .config import load_config
from .model import TVSAModel
from .runner import BENCH_POINT, run_cycle_device

CYCLE_KEYS = ("steps", "rejected", "newton_iters", "gmres_iters", "gmres_polish", "pred_net", "pred_extrap")


def draw_columns(n: int, seed: int = 0) -> List[Dict]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        over = dict(BENCH_POINT)
        over.update({"grid.Nr": int(rng.choice([4, 8, 16])), "grid.Ntheta": int(rng.choice([4, 8, 16])),
                     "grid.Nz": int(rng.choice([16, 32, 64])), "operation.T_heat": float(rng.uniform(363.0, 393.0)),
                     "operation.P_vacuum": float(rng.uniform(5e3, 3e4)), "feed.RH": float(rng.uniform(0.2, 0.8)),
                     "feed.y_co2_dry": float(rng.uniform(350e-6, 450e-6))})
        out.append(over)
    return out


@dataclass
class ColumnResult:
    over: Dict
    bed_s: float
    wall_s: float
    y: np.ndarray
    stats: Dict = field(default_factory=dict)


def _column(over: Dict, precision: str, weights: Optional[tuple], device: int) -> ColumnResult:
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        cfg = load_config(override_dict=dict(over, **{"gpu.krylov_precision": precision}))
        g = host.Grid.from_config(cfg)
        props = host.get_backend(cfg)
        st = host.seeded_state(cfg, g, props, seed=0)
        y0 = torch.from_numpy(TVSAModel(cfg, g, props, cfg.cycle[0], st).pack(st)).cuda()
        net = None
        if weights is not None:
            from .predictor import NewtonPredictor
            net = NewtonPredictor(sample_capacity=0)
            net.set_params(*weights)
        stream.synchronize()
        t0 = time.perf_counter()
        y, stats, _ = run_cycle_device(y0, cfg, g, props, predictor=net, predict=net is not None)
        stream.synchronize()
        wall = time.perf_counter() - t0
        tot = {k: int(sum(s.get(k, 0) for s in stats)) for k in CYCLE_KEYS}
        return ColumnResult(over, float(sum(s["t"] for s in stats)), wall, y.cpu().numpy(), tot)


def run_ensemble(columns: List[Dict], precision: str = "fp64", predictor=None, threads: Optional[int] = None,
                 device: int = 0):
    """Run every column's full cycle concurrently; returns (results, aggregate bed-s per wall-s, wall s)."""
    weights = predictor.params() if predictor is not None else None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads or len(columns)) as ex:
        res = list(ex.map(lambda o: _column(o, precision, weights, device), columns))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return res, sum(r.bed_s for r in res) / wall, wall


def column_errors(a: List[ColumnResult], b: List[ColumnResult]):
    """Per column: largest relative difference of the end states (|a - b| / (|b| + tiny))."""
    out = []
    for x, y in zip(a, b):
        scale = np.abs(y.y) + 1e-12 * np.abs(y.y).max()
        out.append(float(np.max(np.abs(x.y - y.y) / scale)))
    return out
