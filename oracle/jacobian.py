"""Oracle: coloured forward-difference Jacobian (restates core/jacobian.py:21-91).

One RHS evaluation per colour; perturbation h = 1.5e-8 max(|y|, typ) rounded to an exactly
representable step (:75-76); theta-block reduction keeps couplings inside a theta sector plus
all couplings among the innermost ``precond_theta_rings`` rings (:50-69, 88-91).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .sparsity import greedy_colour, pattern


def typical_magnitudes(model):
    """Per-unknown typical magnitude of the perturbation size (core/jacobian.py:39-48)."""
    n = model.grid.ncell
    typ = [np.full(n, {"CO2": 1e-3, "H2O": 1e-2, "N2": 1.0}[s]) for s in model.species]
    typ += [np.full(n, 1e-3)] * model.na
    typ.append(np.full(n, model.rho_b * model.cfg.sorbent.cp_solid))
    if model.n_w:
        typ.append(np.ones(model.n_w))
    return np.concatenate(typ)


class OracleFDJacobian:
    def __init__(self, model):
        g = model.grid
        self.model = model
        self.P = pattern(g.Nr, g.Nth, g.Nz, model.ng, model.na, model.n_w > 0).tocsc()
        self.color = greedy_colour(self.P)
        self.indptr, self.indices = self.P.indptr, self.P.indices
        self.n = self.P.shape[0]
        self.ngroups = int(self.color.max()) + 1
        self.entry_col = np.repeat(np.arange(self.n), np.diff(self.indptr))
        self.entry_row = self.indices
        self.groups = [np.where(self.color == k)[0] for k in range(self.ngroups)]
        eg = self.color[self.entry_col]
        order = np.argsort(eg, kind="stable")
        bounds = np.searchsorted(eg[order], np.arange(self.ngroups + 1))
        self.group_entries = [order[bounds[k]:bounds[k + 1]] for k in range(self.ngroups)]
        self.typ = typical_magnitudes(model)
        n = g.ncell
        nv = model.ng + model.na + 1
        idx = np.arange(self.n)
        cellpart = idx < nv * n
        sector = np.where(cellpart, ((idx % n) // g.Nz) % g.Nth, (idx - nv * n) // max(g.Nz, 1))
        ring = np.where(cellpart, (idx % n) // (g.Nth * g.Nz), g.Nr - 1)
        cut = model.cfg.solver.precond_theta_rings - 1
        er, ec = self.entry_row, self.entry_col
        keep = (sector[er] == sector[ec]) | ((ring[er] <= cut) & (ring[ec] <= cut))
        self.keep_theta = np.where(keep)[0]
        self.red_indices = er[self.keep_theta]
        self.red_indptr = np.concatenate([[0], np.cumsum(np.bincount(ec[self.keep_theta], minlength=self.n))])

    def steps(self, y):
        h = 1.5e-8 * np.maximum(np.abs(y), self.typ)
        return (y + h) - y

    def __call__(self, t, y, f0=None):
        m = self.model
        if f0 is None:
            f0, _ = m.rhs(t, y, want_acc=False)
        h = self.steps(y)
        data = np.empty(len(self.entry_row))
        for k in range(self.ngroups):
            cols = self.groups[k]
            yp = y.copy()
            yp[cols] += h[cols]
            fp, _ = m.rhs(t, yp, want_acc=False)
            ent = self.group_entries[k]
            data[ent] = (fp[self.entry_row[ent]] - f0[self.entry_row[ent]]) / h[self.entry_col[ent]]
        return sp.csc_matrix((data, self.indices, self.indptr), shape=(self.n, self.n))

    def theta_block(self, J):
        return sp.csc_matrix((J.data[self.keep_theta], self.red_indices, self.red_indptr), shape=(self.n, self.n))
