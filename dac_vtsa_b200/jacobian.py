"""FDJacobian on the GPU: drop-in for core/jacobian.py:21-91 of the reference.

The colouring comes from the library's host code (bit-identical to numerics/sparsity.py:88-107);
the values come from dv_fd_jacobian, which evaluates every colour perturbation in one launch into
the block layout J[slot][row 0..6][col 0..6][cell].  ``__call__`` returns the same scipy CSC matrix
the reference does (pattern and entry order of build_pattern), ``block`` keeps J on the device.
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache

import numpy as np
import scipy.sparse as sp
import torch

from ._lib import DV_NB, DV_NSLOT, DV_NV, check, colour_columns

# neighbour slots: (dk, di, dj) of the column cell relative to the row cell
SLOTS = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (-2, 0, 0), (2, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]


@lru_cache(maxsize=16)
def block_pattern(Nr, Nth, Nz, wall):
    """Structural entries of the stencil pattern as (block index, row, col) in CSC order.

    Block index = ((slot*7 + rv)*7 + cv)*ncell + cell of dv_fd_jacobian's layout; rows/cols are
    global unknown indices.  Pattern rules of numerics/sparsity.py:29-85."""
    nc = Nr * Nth * Nz
    cell = np.arange(nc)
    k = cell % Nz
    j = (cell // Nz) % Nth
    i = cell // (Nz * Nth)
    offw = DV_NV * nc
    B, R, Cc = [], [], []
    for s, (dk, di, dj) in enumerate(SLOTS):
        if s in (7, 8) and Nth == 1:
            continue
        nk, ni = k + dk, i + di
        nj = (j + dj) % Nth
        ok = (nk >= 0) & (nk < Nz) & (ni >= 0) & (ni < Nr)
        ncell = (ni * Nth + nj) * Nz + nk
        outer = i == Nr - 1
        for rv in range(DV_NB):
            for cv in range(DV_NB):
                if rv in (0, 1, 2, DV_NV - 1):                 # gas / energy rows
                    if cv < DV_NV:
                        valid = ok
                    elif s == 0 and wall:                      # outer cell <- its wall node
                        valid = ok & outer
                    else:
                        continue
                elif rv in (3, 4):                               # loading rows: own cell only
                    if s != 0 or cv == DV_NV:
                        continue
                    valid = ok
                else:                                            # wall row of an outer cell
                    if not wall or (cv < DV_NV and s != 0) or (cv == DV_NV and s not in (0, 1, 2, 7, 8)):
                        continue
                    valid = ok & outer
                if not np.any(valid):
                    continue
                cs = cell[valid]
                row = (rv * nc + cs) if rv < DV_NV else offw + j[valid] * Nz + k[valid]
                col = (cv * nc + ncell[valid]) if cv < DV_NV else offw + nj[valid] * Nz + nk[valid]
                B.append(((s * DV_NB + rv) * DV_NB + cv) * nc + cs)
                R.append(row)
                Cc.append(col)
    B, R, Cc = np.concatenate(B), np.concatenate(R), np.concatenate(Cc)
    order = np.lexsort((R, Cc))
    B, R, Cc = B[order], R[order], Cc[order]
    n = DV_NV * nc + (Nth * Nz if wall else 0)
    indptr = np.concatenate([[0], np.cumsum(np.bincount(Cc, minlength=n))])
    return B, R.astype(np.int32), indptr.astype(np.int32), n


@lru_cache(maxsize=16)
def _colouring(Nr, Nth, Nz, wall):
    c, nc = colour_columns(Nr, Nth, Nz, wall)
    c.setflags(write=False)
    return c, nc


@lru_cache(maxsize=16)
def _pattern_views(Nr, Nth, Nz, wall, cut):
    """Boolean pattern matrix, entry columns and the theta-block reduction (core/jacobian.py:50-69:
    same sector, or both in the innermost `cut + 1` rings) of a grid shape, built once per shape
    (the reference's runner builds one Jacobian per cycle step)."""
    _, indices, indptr, n = block_pattern(Nr, Nth, Nz, wall)
    P = sp.csc_matrix((np.ones(len(indices), dtype=bool), indices, indptr), shape=(n, n))
    entry_col = np.repeat(np.arange(n), np.diff(indptr))
    nc = Nr * Nth * Nz
    idx = np.arange(n)
    cellpart = idx < DV_NV * nc
    sector = np.where(cellpart, ((idx % nc) // Nz) % Nth, (idx - DV_NV * nc) // max(Nz, 1))
    ring = np.where(cellpart, (idx % nc) // (Nth * Nz), Nr - 1)
    er, ec = indices, entry_col
    keep = (sector[er] == sector[ec]) | ((ring[er] <= cut) & (ring[ec] <= cut))
    keep_theta = np.where(keep)[0]
    red_indptr = np.concatenate([[0], np.cumsum(np.bincount(ec[keep_theta], minlength=n))])
    for a in (entry_col, keep_theta, red_indptr):
        a.setflags(write=False)
    return P, entry_col, keep_theta, er[keep_theta], red_indptr


class FDJacobian:
    """Coloured forward-difference Jacobian of a GPU TVSAModel."""

    def __init__(self, model):
        g = model.grid
        wall = model.n_w > 0
        self.model = model
        self.color, self.ngroups = _colouring(g.Nr, g.Nth, g.Nz, wall)
        self._blk, self.indices, self.indptr, self.n = block_pattern(g.Nr, g.Nth, g.Nz, wall)
        self.entry_row = self.indices
        self.nevals = 0
        self._J = None
        (self.P, self.entry_col, self.keep_theta, self.red_indices,
         self.red_indptr) = _pattern_views(g.Nr, g.Nth, g.Nz, wall, model.cfg.solver.precond_theta_rings - 1)

    def block(self, t, y, f0=None):
        """J on the device in the block layout (float64 tensor of jac_doubles)."""
        m = self.model
        yd, _ = m._to_dev(y, m._y)
        if f0 is None:
            f0d = torch.empty_like(yd)
            check(m.lib.dv_rhs(m.handle, float(t), C.c_void_p(yd.data_ptr()), C.c_void_p(f0d.data_ptr()), None,
                               C.c_void_p(torch.cuda.current_stream().cuda_stream)), "dv_rhs")
        else:
            f0d, _ = m._to_dev(f0, m._b)
        if self._J is None:
            self._J = torch.empty(m.jac_doubles, dtype=torch.float64, device=m.device)
        check(m.lib.dv_fd_jacobian(m.handle, float(t), C.c_void_p(yd.data_ptr()), C.c_void_p(f0d.data_ptr()),
                                   C.c_void_p(self._J.data_ptr()),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)), "dv_fd_jacobian")
        self.nevals += 1
        return self._J

    def __call__(self, t, y, f0=None) -> sp.csc_matrix:
        Jb = self.block(t, y, f0).cpu().numpy()
        return sp.csc_matrix((Jb[self._blk], self.indices, self.indptr), shape=(self.n, self.n))

    def theta_block(self, J: sp.csc_matrix) -> sp.csc_matrix:
        return sp.csc_matrix((J.data[self.keep_theta], self.red_indices, self.red_indptr), shape=(self.n, self.n))
