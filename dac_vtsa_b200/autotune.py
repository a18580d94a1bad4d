"""Launch-parameter autotuner: picks the hot kernels' launch parameters per grid shape and caches them.

``tune(model, y, dh)`` runs the library's timer (dv_autotune) on the model at state y: every candidate
of the FD-Jacobian block size, the preconditioner sweep's ring depth, the FP32 Jacobian product's
block size and the GMRES graph's prefix of unrolled Arnoldi steps, timed with CUDA events on the
model's own matrices; the fastest of each is kept in the model.  ``cached(model)`` applies an earlier
result for the same grid, preconditioner, precision and GPU from the cache file (``$DVTSA_TUNE_CACHE``,
default ``~/.cache/dac_vtsa_b200/tune.json``) and tunes on a miss.  The parameters never change a result
bit, only the time.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Dict, Optional

import numpy as np
import torch

from ._lib import DvTuning, check, load

FIELDS = ("gmres_prefix", "sweep_nbuf", "spmv_block", "fdjac_block", "gmres_body")
TIMES = ("fdjac_64", "fdjac_128", "sweep_nbuf2", "sweep_nbuf3", "spmv_64", "spmv_128", "spmv_256",
         "stage_prefix0", "stage_prefix2", "stage_prefix4", "stage_prefix6", "stage_prefix8",
         "stage_body1", "stage_body2")


def cache_path() -> str:
    return os.environ.get("DVTSA_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "dac_vtsa_b200",
                                                                "tune.json")


def key(model, precision: str = "fp64") -> str:
    g = model.grid
    name = torch.cuda.get_device_name(model.device).replace(" ", "_")
    return f"{name}/{g.Nr}x{g.Nth}x{g.Nz}/wall{int(model.n_w > 0)}/{model.cfg.solver.preconditioner}/{precision}"


def get(model) -> Dict[str, int]:
    t = DvTuning()
    check(model.lib.dv_model_get_tuning(model.handle, C.byref(t)), "dv_model_get_tuning")
    return {f: int(getattr(t, f)) for f in FIELDS}


def apply(model, params: Dict[str, int]):
    t = DvTuning(**{f: int(params.get(f, 0 if f != "gmres_prefix" else -1)) for f in FIELDS})
    check(model.lib.dv_model_set_tuning(model.handle, C.byref(t)), "dv_model_set_tuning")


def tune(model, y, dh: float, t: float = 0.0, reps: int = 50):
    """Returns (chosen parameters, per-candidate microseconds)."""
    best = DvTuning()
    times = np.zeros(len(TIMES))
    with torch.cuda.device(model.device):
        yd, _ = model._to_dev(y, model._y)
        check(load().dv_autotune(model.handle, float(t), C.c_void_p(yd.data_ptr()), float(dh), int(reps),
                                 C.byref(best), times.ctypes.data, len(TIMES),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)), "dv_autotune")
    return {f: int(getattr(best, f)) for f in FIELDS}, dict(zip(TIMES, times.tolist()))


def cached(model, y, dh: float, precision: str = "fp64", path: Optional[str] = None) -> Dict[str, int]:
    path = path or cache_path()
    k = key(model, precision)
    table = {}
    if os.path.exists(path):
        try:
            table = json.load(open(path))
        except ValueError:
            table = {}
    if k in table:
        apply(model, table[k]["params"])
        return table[k]["params"]
    params, times = tune(model, y, dh)
    table[k] = {"params": params, "times_us": times}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return params
