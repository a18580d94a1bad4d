"""Step-to-step state hand-off files in the reference's CSV format, written off the critical path.

Format (simio/checkpoint.py:1-12 of the reference, kept alike because the reference's cycle driver
and post-processing read these files): ``<name>.csv`` holds one row per bed cell with the columns
i_r, i_theta, i_z, r_m, theta_deg, z_m, T_K, P_Pa, c_<gas>_mol_m3..., y_<gas>..., q_<ads>_mol_kg...
after a one-line ``# t_s=... cycle=... step=... grid=NrxNthxNz`` comment; ``<name>_wall.csv`` holds
i_theta, i_z, theta_deg, z_m, T_wall_K.  Floats carry 17 significant digits, so a write / read round
trip is bit-exact.

``AsyncStateWriter`` takes a device state at a step end, starts its copy to pinned host memory on the
current stream, and formats and writes the files on a worker thread, so the GPU goes on with the
next step.
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import List, Sequence

import numpy as np
import torch

from . import host

FLOAT = "%.17g"


def _cell_table(state, grid):
    """(column names, formats, columns) of the cell file."""
    r, th, z = np.meshgrid(grid.r_c, grid.th_c, grid.z_c, indexing="ij")
    idx = np.meshgrid(np.arange(grid.Nr), np.arange(grid.Nth), np.arange(grid.Nz), indexing="ij")
    y = state.y
    spec = [("i_r", "%d", idx[0]), ("i_theta", "%d", idx[1]), ("i_z", "%d", idx[2]), ("r_m", FLOAT, r),
            ("theta_deg", FLOAT, np.degrees(th)), ("z_m", FLOAT, z), ("T_K", FLOAT, state.T), ("P_Pa", FLOAT, state.P)]
    spec += [(f"c_{sp}_mol_m3", FLOAT, state.c[k]) for k, sp in enumerate(state.species)]
    spec += [(f"y_{sp}", FLOAT, y[k]) for k, sp in enumerate(state.species)]
    spec += [(f"q_{sp}_mol_kg", FLOAT, state.q[n]) for n, sp in enumerate(state.adsorbed)]
    return [s[0] for s in spec], [s[1] for s in spec], np.column_stack([np.ravel(s[2]) for s in spec])


def save_state_csv(state, grid, path: str) -> str:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    names, fmts, table = _cell_table(state, grid)
    first = (f"# t_s={float(state.t)!r} cycle={int(state.cycle)} step={state.step} "
             f"grid={grid.Nr}x{grid.Nth}x{grid.Nz}")
    np.savetxt(path, table, delimiter=",", header=first + "\n" + ",".join(names), comments="", fmt=fmts)
    jw, kw = np.meshgrid(np.arange(grid.Nth), np.arange(grid.Nz), indexing="ij")
    wall = np.column_stack([jw.ravel(), kw.ravel(), np.degrees(grid.th_c)[jw.ravel()], grid.z_c[kw.ravel()],
                            np.ravel(state.Tw)])
    np.savetxt(path[:-4] + "_wall.csv", wall, delimiter=",", header="i_theta,i_z,theta_deg,z_m,T_wall_K",
               comments="", fmt=["%d", "%d", FLOAT, FLOAT, FLOAT])
    return path


def load_state_csv(path: str, grid, species: Sequence[str], adsorbed: Sequence[str]):
    with open(path) as fh:
        meta = dict(tok.split("=", 1) for tok in fh.readline().lstrip("# ").split() if "=" in tok)
        cols = {h: i for i, h in enumerate(fh.readline().strip().split(","))}
    tab = np.loadtxt(path, delimiter=",", skiprows=2, ndmin=2)
    if tab.shape[0] != grid.ncell:
        raise ValueError(f"{path}: has {tab.shape[0]} cells but the grid has {grid.ncell} "
                         f"({grid.Nr}x{grid.Nth}x{grid.Nz}); use the same grid as the run that wrote it")
    where = tuple(tab[:, cols[k]].astype(int) for k in ("i_r", "i_theta", "i_z"))

    def field(name):
        if name not in cols:
            raise ValueError(f"{path}: missing column {name} (was the run dry/humid?)")
        out = np.empty(grid.shape)
        out[where] = tab[:, cols[name]]
        return out

    T = field("T_K")
    c = np.stack([field(f"c_{sp}_mol_m3") for sp in species])
    q = np.stack([field(f"q_{sp}_mol_kg") for sp in adsorbed])
    Tw = np.empty(grid.wall_shape)
    wpath = path[:-4] + "_wall.csv"
    if os.path.exists(wpath):
        w = np.loadtxt(wpath, delimiter=",", skiprows=1, ndmin=2)
        Tw[w[:, 0].astype(int), w[:, 1].astype(int)] = w[:, 4]
    else:
        Tw[:] = T[-1]
    return host.CycleState(c=c, q=q, T=T, Tw=Tw, t=float(meta.get("t_s", 0.0)), cycle=int(meta.get("cycle", 1)),
                           step=meta.get("step", "loaded"), species=tuple(species), adsorbed=tuple(adsorbed))


class AsyncStateWriter:
    """Writes step-end states while the GPU continues: submit() queues a device-to-pinned copy on the
    current stream and hands the formatting and file writes to a worker thread; wait() joins."""

    def __init__(self):
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.jobs: List = []
        self.lock = threading.Lock()

    def submit(self, y_dev: torch.Tensor, model, template, t_abs: float, step_name: str, cycle: int, grid,
               path: str):
        pinned = torch.empty(y_dev.numel(), dtype=torch.float64, pin_memory=True)
        pinned.copy_(y_dev, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()

        def job():
            ev.synchronize()
            st = model.to_state(pinned.numpy(), template, t_abs, step_name)
            st.cycle = cycle
            return save_state_csv(st, grid, path)

        with self.lock:
            self.jobs.append(self.pool.submit(job))

    def wait(self) -> List[str]:
        with self.lock:
            jobs, self.jobs = self.jobs, []
        return [j.result() for j in jobs]

    def close(self):
        self.wait()
        self.pool.shutdown()
