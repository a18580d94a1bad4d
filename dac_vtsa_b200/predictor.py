"""Learned Newton predictor: a per-cell network that corrects the extrapolated start of each implicit stage.

The reference starts each TR-BDF2 / SDIRK2 stage from a straight-line extrapolation through the two
latest states (core/solver.py:420 for stage 1, :432/:435 for stage 2).  ``NewtonPredictor`` wraps the
library's network (dv_mlp_*, BF16 weights, FP32 accumulation on the tcgen05 tensor cores) and its
training loop; attached to a ``TRBDF2`` it

* records training samples (features of every ``record_stride``-th cell and the converged stage
  solution, scaled by the solver's error scale) from the plain solver's own stage solves, and/or
* predicts a correction to the extrapolation; each stage then starts from whichever of the two guesses
  has the smaller scaled stage residual, and a Newton failure from the network's guess is retried from
  the extrapolation.  The Newton tolerance is unchanged, so the converged state is the plain method's
  up to that tolerance.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from ._lib import check, load

NIN, NH, NOUT, NPARAM, NNORM, BATCH = 112, 128, 16, 49552, 32, 4096
STEP_CODES = {"adsorption": 0, "blowdown": 1, "heating": 2, "cooling": 3}


class NewtonPredictor:
    def __init__(self, sample_capacity: int = 1 << 20, seed: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.dv_mlp_create(int(sample_capacity), int(seed), C.byref(h)), "dv_mlp_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.dv_mlp_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------------ parameters
    def params(self):
        P = np.empty(NPARAM, dtype=np.float32)
        nrm = np.empty(NNORM, dtype=np.float64)
        check(self.lib.dv_mlp_get_params(self.handle, P.ctypes.data, nrm.ctypes.data), "dv_mlp_get_params")
        return P, nrm

    def set_params(self, P, norm=None):
        P = np.ascontiguousarray(P, dtype=np.float32)
        nrm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float64)
        check(self.lib.dv_mlp_set_params(self.handle, P.ctypes.data, P.size,
                                         nrm.ctypes.data if nrm is not None else None,
                                         NNORM if nrm is not None else 0), "dv_mlp_set_params")

    def save(self, path: str):
        P, nrm = self.params()
        np.savez_compressed(path, params=P, norm=nrm)

    @classmethod
    def load(cls, path: str, sample_capacity: int = 0):
        d = np.load(path)
        net = cls(sample_capacity=sample_capacity)
        net.set_params(d["params"], d["norm"])
        return net

    # ------------------------------------------------------------------ samples and training
    @property
    def samples(self) -> int:
        return int(self.lib.dv_mlp_sample_count(self.handle))

    def get_samples(self, first: int = 0, count=None):
        """Recorded (features [count][112], targets [count][8]) as numpy arrays."""
        count = self.samples - first if count is None else count
        X = np.empty((count, NIN), dtype=np.float32)
        T = np.empty((count, 8), dtype=np.float32)
        check(self.lib.dv_mlp_get_samples(self.handle, int(first), int(count), X.ctypes.data, T.ctypes.data),
              "dv_mlp_get_samples")
        return X, T

    def clear_samples(self):
        check(self.lib.dv_mlp_clear_samples(self.handle), "dv_mlp_clear_samples")

    def train(self, steps: int, lr: float = 1e-3, seed: int = 0, keep_scales: bool = False) -> np.ndarray:
        """Adam on the recorded samples; returns the per-step batch loss."""
        hist = np.zeros(max(1, steps), dtype=np.float32)
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        check(self.lib.dv_mlp_train(self.handle, int(steps), float(lr), int(seed), int(bool(keep_scales)),
                                    hist.ctypes.data, s), "dv_mlp_train")
        return hist[:steps]

    # ------------------------------------------------------------------ direct evaluation (tests)
    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty((X.shape[0], NOUT), dtype=np.float32)
        check(self.lib.dv_mlp_forward_host(self.handle, X.ctypes.data, X.shape[0], out.ctypes.data),
              "dv_mlp_forward_host")
        return out

    def gradient(self, X: np.ndarray, T: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.empty(NPARAM, dtype=np.float32)
        L = C.c_double(0.0)
        check(self.lib.dv_mlp_gradient_host(self.handle, X.ctypes.data, T.ctypes.data, X.shape[0], g.ctypes.data,
                                            C.byref(L)), "dv_mlp_gradient_host")
        return g, L.value

    # ------------------------------------------------------------------ integration
    def attach(self, integ, step_type: str, predict: bool = True, record_stride: int = 0):
        """Attach to a dac_vtsa_b200.solver.TRBDF2 for its next integrate()."""
        check(self.lib.dv_integrator_set_predictor(integ.handle, self.handle, int(bool(predict)), int(record_stride),
                                                   STEP_CODES.get(step_type, 0)), "dv_integrator_set_predictor")
        integ.predictor = self


def detach(integ):
    check(load().dv_integrator_set_predictor(integ.handle, None, 0, 0, 0), "dv_integrator_set_predictor")
    integ.predictor = None


PACKAGED = {"default": "predictor_weights.npz"}
_CACHE = {}


def default_network(path: str = ""):
    """The network of `path` (or the packaged trained weights), loaded once per process."""
    import os
    if not path:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), PACKAGED["default"])
    if path not in _CACHE:
        if not os.path.exists(path):
            raise FileNotFoundError(f"gpu.predictor = learned needs trained weights: {path} is missing "
                                    f"(train them with python -m dac_vtsa_b200.train_predictor)")
        _CACHE[path] = NewtonPredictor.load(path)
    return _CACHE[path]
