"""Oracle: Jacobian sparsity pattern and greedy distance-2 column colouring.

Restates numerics/sparsity.py:29-123 of the reference:

* pattern (build_pattern :29-85) -- gas-species and energy rows of cell (i,j,k) couple to all
  cell unknowns of (i,j,k), (i,j,k+-1), (i,j,k+-2), (i+-1,j,k), (i,j+-1 mod Nth,k); loading rows
  only to their own cell; wall rows to wall neighbours (j+-1, k+-1) and the outer bed cell;
  outer-cell flux rows to their wall cell;
* colouring (color_columns :88-107) -- conflict graph G = P^T P, columns visited in order of
  decreasing degree of G (stable on ties), each given the smallest colour not used by a
  G-neighbour.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def pattern(Nr, Nth, Nz, ng, na, wall):
    n = Nr * Nth * Nz
    nv = ng + na + 1
    cell = np.arange(n).reshape(Nr, Nth, Nz)
    rc, cc = [cell.ravel()], [cell.ravel()]
    for dk in (1, 2):
        if Nz > dk:
            rc += [cell[:, :, dk:].ravel(), cell[:, :, :-dk].ravel()]
            cc += [cell[:, :, :-dk].ravel(), cell[:, :, dk:].ravel()]
    if Nr > 1:
        rc += [cell[1:].ravel(), cell[:-1].ravel()]
        cc += [cell[:-1].ravel(), cell[1:].ravel()]
    if Nth > 1:
        nb = np.roll(cell, -1, axis=1)
        rc += [cell.ravel(), nb.ravel()]
        cc += [nb.ravel(), cell.ravel()]
    rc, cc = np.concatenate(rc), np.concatenate(cc)
    flux_rows = list(range(ng)) + [ng + na]
    R, C = [], []
    for vr in flux_rows:
        for vc in range(nv):
            R.append(vr * n + rc)
            C.append(vc * n + cc)
    own = cell.ravel()
    for vr in range(ng, ng + na):
        for vc in range(nv):
            R.append(vr * n + own)
            C.append(vc * n + own)
    if wall:
        base = nv * n
        w = np.arange(Nth * Nz).reshape(Nth, Nz)
        outer = cell[-1]
        wr, wc = [w.ravel()], [w.ravel()]
        if Nz > 1:
            wr += [w[:, 1:].ravel(), w[:, :-1].ravel()]
            wc += [w[:, :-1].ravel(), w[:, 1:].ravel()]
        if Nth > 1:
            nbw = np.roll(w, -1, axis=0)
            wr += [w.ravel(), nbw.ravel()]
            wc += [nbw.ravel(), w.ravel()]
        R.append(base + np.concatenate(wr))
        C.append(base + np.concatenate(wc))
        for vc in range(nv):
            R.append(base + w.ravel())
            C.append(vc * n + outer.ravel())
        for vr in flux_rows:
            R.append(vr * n + outer.ravel())
            C.append(base + w.ravel())
    R, C = np.concatenate(R), np.concatenate(C)
    N = nv * n + (Nth * Nz if wall else 0)
    P = sp.csc_matrix((np.ones(len(R), dtype=np.int8), (R, C)), shape=(N, N))
    P.sum_duplicates()
    P.data[:] = 1
    return P.astype(bool)


def greedy_colour(P):
    P = P.astype(np.int8).tocsc()
    G = (P.T @ P).tocsr()
    n = P.shape[1]
    colour = np.full(n, -1, dtype=np.int64)
    deg = np.diff(G.indptr)
    for j in np.argsort(-deg, kind="stable"):
        used = colour[G.indices[G.indptr[j]:G.indptr[j + 1]]]
        used = used[used >= 0]
        if used.size == 0:
            colour[j] = 0
        else:
            taken = np.zeros(used.max() + 2, dtype=bool)
            taken[used] = True
            colour[j] = int(np.argmin(taken))
    return colour


def colouring_is_valid(P, colour):
    Pr = P.tocsr()
    for r in range(Pr.shape[0]):
        cc = colour[Pr.indices[Pr.indptr[r]:Pr.indptr[r + 1]]]
        if len(np.unique(cc)) != len(cc):
            return False
    return True
