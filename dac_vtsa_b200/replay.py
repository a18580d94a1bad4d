"""Replay harness: advance a model over a GIVEN step-size sequence, every stage solved tightly.

Adaptive solvers with the same tolerances take different accepted steps as soon as their
arithmetic differs in the last bit (both accept/reject decisions and Newton iteration counts
depend on it), so two correct implementations agree only to about the tolerance.  Replaying the
reference's accepted step sizes and solving each implicit stage to a residual far below the
adaptive tolerance removes that freedom: the step-end states of two correct implementations of
the same discretisation (the stage equations of core/solver.py:415-436 with the residual of
core/residual.py) then agree to ~1e-10.
"""
from __future__ import annotations

import numpy as np
import torch

from .jacobian import FDJacobian

GAMMA = 2.0 - np.sqrt(2.0)
D = GAMMA / 2.0
C1 = 1.0 / (GAMMA * (2.0 - GAMMA))
C2 = (1.0 - GAMMA) ** 2 / (GAMMA * (2.0 - GAMMA))
G_SD = 1.0 - 1.0 / np.sqrt(2.0)


def fixed_step_run(model, y0, hs, scheme="trbdf2", kappa=1e-11, max_iter=30):
    """Returns (list of step-end states as numpy arrays, accumulator integrals)."""
    jac = FDJacobian(model)
    dev = model.device
    y = torch.from_numpy(np.ascontiguousarray(y0, dtype=np.float64)).to(dev)
    t = 0.0
    f_n, g_n = model.rhs(t, y)
    acc = np.zeros(model.n_acc)
    g_n = g_n.cpu().numpy()
    sd = scheme == "sdirk2"
    c_mid = G_SD if sd else GAMMA
    out = []
    for h in hs:
        dh = D * h
        J = jac.block(t, y, f_n)
        model.precond_factor(J, dh)
        rhs1 = y.clone() if sd else y + dh * f_n
        z1, ok1, _, _, _ = model.newton_stage(t + c_mid * h, y, rhs1, dh, max_iter=max_iter, kappa=kappa, cons_tol=0.0)
        rhs2 = (y + (1.0 - G_SD) * h * ((z1 - y) / dh)) if sd else C1 * z1 - C2 * y
        z2, ok2, _, _, _ = model.newton_stage(t + h, y + (z1 - y) / c_mid, rhs2, dh, max_iter=max_iter, kappa=kappa,
                                              cons_tol=0.0)
        if not (ok1 and ok2):
            raise RuntimeError(f"replay stage did not converge at t={t}")
        _, g1 = model.rhs(t + c_mid * h, z1)
        f2, g2 = model.rhs(t + h, z2)
        g1, g2 = g1.cpu().numpy(), g2.cpu().numpy()
        if sd:
            acc = acc + h * ((1.0 - G_SD) * g1 + G_SD * g2)
        else:
            acc = C1 * (acc + D * h * (g_n + g1)) - C2 * acc + D * h * g2
        t, y, f_n, g_n = t + h, z2, f2, g2
        out.append(y.cpu().numpy())
    return out, acc
