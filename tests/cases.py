"""Shared helpers of the test suite: golden fixtures and model construction."""
from __future__ import annotations

import json
import os
from types import SimpleNamespace

import numpy as np

from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def rhs_cases():
    d = golden("rhs_cases.npz")
    meta = json.loads(str(d["meta"]))
    for m in meta:
        n = m["name"]
        yield m, {k: d[f"{n}__{k}"] for k in ("y", "f", "acc", "T", "P", "P0")}


def state_like(P0):
    """Minimal stand-in for a CycleState: models read only ``.P`` (start pressures of the ends)."""
    return SimpleNamespace(P=np.asarray(P0))


def build(model_cls, over, step_index, P0, T_jacket_prev=None, duration=None):
    cfg = load_config(override_dict=over)
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    step = dict(cfg.cycle[step_index])
    if duration is not None:
        step["duration"] = duration
    return model_cls(cfg, g, props, step, state_like(P0), T_jacket_prev), cfg


def config0_overrides():
    return {"grid.Nr": 4, "grid.Ntheta": 4, "grid.Nz": 16, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}
