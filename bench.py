#!/usr/bin/env python
"""Throughput of the implicit stepping path: simulated bed-seconds per wall-second.

Workload of the line (default ``heat_window_8x8x32``, the same for ``--impl ours`` and ``--impl
reference``): the heating step of the 8x8x32 cycle (2048 cells, 12 544 unknowns, FP64, TR-BDF2 at the
reference defaults, T_heat 373 K, 10 kPa product vacuum) restarted from the reference's own state after
adsorption, blowdown and 4000 s of heating (tests/golden/bench_state_8x8x32_heat4000.npz) at the
reference's last step size, integrated for 2000 bed-seconds.  A "step" of this benchmark is one such
window.  ``cycle_8x8x32`` / ``cycle_16x16x64`` / ``cycle_4x4x16`` make one full adsorption (8000 s) ->
blowdown (60 s) -> heating (22400 s) -> cooling (400 s) cycle the step instead (GPU arm only).

ours (default):
  value  device-resident (state stays on the GPU; the model is built once), CUDA events per step, L2
         flushed between steps (a 256 MB write), max over ranks; N GPUs run N independent replicas
  e2e    the same window through the public API the reference's runner uses (TRBDF2(...).integrate
         with a host numpy state in and out), host copies inside the timed region
  roofline: the dominant kernel of one profiled window, timed back to back on its stream
  cpu_baseline: the CPU oracle (numpy restatement of the reference) on the same window, 1 core
  cycles: full cycles of the 8x8x32 and 16x16x64 beds -- plain FP64 (the reference's algorithm),
         with the balance projection, and with it mixed precision (FP32 preconditioner factors) and
         the learned predictor -- with their balance errors and state difference to the FP64 cycle,
         and the 8x8x32 cycle's step-end states against the reference's
--impl reference: the oracle on the host cores (one process per core, up to 16), each process one
  window per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CYCLE_BED_S = 8000.0 + 60.0 + 22400.0 + 400.0
WORKLOADS = {
    "heat_window_8x8x32": {"grid": (8, 8, 32), "window": True},
    "cycle_8x8x32": {"grid": (8, 8, 32)},
    "cycle_16x16x64": {"grid": (16, 16, 64)},
    "cycle_4x4x16": {"grid": (4, 4, 16)},
}
SAMPLE_STATE = os.path.join(ROOT, "tests", "golden", "bench_state_8x8x32_heat4000.npz")
REF_CYCLE = os.path.join(ROOT, "tests", "golden", "cycle_8x8x32.npz")
WINDOW_BED_S = 2000.0
CPU_FULL_CYCLE = "1838 s for the 30 860 bed-s 8x8x32 cycle (16.8 bed-s/wall-s) on one core of the build host"


def overrides(grid):
    Nr, Nth, Nz = grid
    return {"grid.Nr": Nr, "grid.Ntheta": Nth, "grid.Nz": Nz, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}


def setup(grid, extra=None):
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    cfg = load_config(override_dict=dict(overrides(grid), **(extra or {})))
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, g, props, seed=0)
    return cfg, g, props, st


def window_description():
    return (f"heating step of the 8x8x32 cycle restarted from the reference's own state after adsorption, "
            f"blowdown and 4000 s of heating (tests/golden/{os.path.basename(SAMPLE_STATE)}), at the reference's "
            f"last step size, integrated for {WINDOW_BED_S:g} bed-s at the reference defaults (TR-BDF2)")


class Window:
    """The benchmark window: configuration, the restart state and the model's constants."""

    def __init__(self, model_cls):
        import numpy as np
        from dac_vtsa_b200 import host
        from dac_vtsa_b200.config import load_config
        d = np.load(SAMPLE_STATE)
        self.cfg = load_config(override_dict=json.loads(str(d["over"])))
        self.grid = host.Grid.from_config(self.cfg)
        self.props = host.get_backend(self.cfg)
        self.y = np.ascontiguousarray(d["y"])
        self.step = dict(self.cfg.cycle[2])
        self.T_jacket = float(d["T_jacket"])
        self.h_init = float(d["h_last"][-2])
        st = host.seeded_state(self.cfg, self.grid, self.props, seed=0)
        tmp = model_cls(self.cfg, self.grid, self.props, self.step, st)
        c, q, e, Tw = tmp.unpack(self.y)
        st.c, st.q, st.Tw = c.copy(), q.copy(), Tw.copy()
        thermo = getattr(tmp, "thermo", tmp)          # the GPU model keeps e -> T in its thermo helper
        st.T = thermo.temperature(e, c, q)
        self.state = st
        self.h_max = self.cfg.solver.h_max_fraction * float(self.step["duration"])

    def model(self, model_cls):
        return model_cls(self.cfg, self.grid, self.props, self.step, self.state, self.T_jacket)


# ---------------------------------------------------------------------------- CPU oracle sample
def _cpu_sample(workload, duration=WINDOW_BED_S):
    """The CPU oracle on the window; returns (bed-seconds, wall seconds)."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle.residual import OracleModel
    from oracle.solver import OracleTRBDF2
    w = Window(OracleModel)
    m = w.model(OracleModel)
    t0 = time.perf_counter()
    integ = OracleTRBDF2(m, w.cfg, h_max=w.h_max, h_init=w.h_init)
    res = integ.integrate(w.y, duration, [duration])
    return res.t, time.perf_counter() - t0


def _cpu_worker(args):
    return _cpu_sample(*args)


def cpu_parallel(workload, procs):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        out = pool.map(_cpu_worker, [(workload,)] * procs)
    wall = time.perf_counter() - t0
    return sum(o[0] for o in out), wall


def cpu_model_name():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(a, rank):
    """The reference's CPU path (the oracle port: the reference is Python and cannot travel) on the
    host cores: each step is one window per core, run in parallel processes."""
    if rank != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, 16))
    for _ in range(a.warmup):
        cpu_parallel(a.workload, procs)
    bed = wall = 0.0
    for _ in range(a.steps):
        b, w = cpu_parallel(a.workload, procs)
        bed += b
        wall += w
    value = bed / wall
    line = {"impl": "reference", "metric": "bed-s simulated per wall-s", "value": value, "unit": "bed-s/wall-s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": a.workload, "window": window_description(), "parallelism": f"{procs} processes"},
            "cpu_baseline": {"value": value, "unit": "bed-s/wall-s", "cores": procs, "kind": "port",
                             "sample": f"{procs} processes x one window each per step ({window_description()}), "
                                       f"{cpu_model_name()}"},
            "e2e": {"value": value, "unit": "bed-s/wall-s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------- ranks
def max_over_ranks(x, dist=None, device=None):
    """Max of a per-rank number over all ranks (a job's time is its slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, steps, bed_s_per_step, seconds):
    """Whole-job bed-seconds per wall-second: every rank integrates `steps` independent steps."""
    return world * steps * bed_s_per_step / seconds


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------- roofline
ALG_BYTES_DOC = {
    "matvec": "FD matvec residual: reads z, u, s, f (4 n_core) + writes n_core doubles",
    "residual": "residual: reads y (+ rhs_known) and writes f: 2 n_core doubles",
    "precond_apply": "sweep: reads the 5 nb x nb factor blocks of every plane of every partition + 3 n_core doubles",
    "fd_jacobian": "reads y, f0 (2 n_core) + writes the 9*49*ncell block layout",
    "precond_factor": "assembly + factorisation: writes and re-reads 5 blocks per plane",
    "vector": "Krylov vector kernels: ~3 n_core doubles per launch (average)",
    "spmv": "FP32 Jacobian product: reads 9*49*ncell floats + 2 n_core doubles, writes n_core doubles",
    "mlp": "network kernels: features and activations",
}


def alg_bytes_per_launch(kind, m, nbs=None, fp32=False):
    n = m.n_core
    if kind == "matvec":
        return 5 * n * 8
    if kind == "residual":
        return 2 * n * 8
    if kind == "fd_jacobian":
        return (2 * n + m.jac_doubles) * 8
    if kind == "spmv":
        return m.jac_doubles * 4 + 3 * n * 8
    blocks = m.grid.Nz * 5 * sum(nb * nb for nb in nbs) * (4 if fp32 else 8)
    if kind == "precond_apply":
        return blocks + 3 * n * 8
    if kind == "precond_factor":
        return 2 * blocks
    return 3 * n * 8


def sweep_seconds(m, y, dh, launches=200):
    """Average duration of the preconditioner sweep: the factors of I - dh J at state y (the solver's
    partitions), then `launches` back-to-back dv_precond_solve calls bracketed by CUDA events on the
    launching stream (the queue never drains, so no host latency is counted).  Returns (seconds,
    block sizes of the partitions)."""
    import ctypes as C
    import torch
    from dac_vtsa_b200.jacobian import FDJacobian
    yd = y.contiguous() if isinstance(y, torch.Tensor) else torch.from_numpy(y).to(m.device)
    m.precond_factor(FDJacobian(m).block(0.0, yd), dh)
    _, _, nbs = m.precond_partitions()
    b = torch.randn(m.n_core, dtype=torch.float64, device=m.device)
    x = torch.empty_like(b)
    s = torch.cuda.current_stream()
    args = (m.handle, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(s.cuda_stream))
    for _ in range(20):
        m.lib.dv_precond_solve(*args)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(launches):
        m.lib.dv_precond_solve(*args)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / launches, nbs


def load_peaks():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------- cycles (extra keys)
# Cycle variants: the plain FP64 path (the reference's algorithm, the defaults), the same with the
# balance projection, and with it mixed precision (FP32 preconditioner factors and sweep; FP64
# operator, residual and Newton update) and the learned predictor.
PROJ = {"gpu.balance_projection": True}
VARIANTS = {"fp64": {}, "fp64_projection": PROJ,
            "mixed_projection": dict(PROJ, **{"gpu.krylov_precision": "fp32_factors"}),
            "learned_mixed_projection": dict(PROJ, **{"gpu.krylov_precision": "fp32_factors"})}


def cycle_runs(grid, variants, weights_path, dev, y_ref_fp64=None):
    """Device-resident full cycles of `grid` in each variant of VARIANTS: throughput, solver totals
    and the end state's difference to the FP64 cycle."""
    import numpy as np
    import torch
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.predictor import NewtonPredictor
    from dac_vtsa_b200.runner import cycle_balance_errors, run_cycle_device
    out, y64 = {}, None
    for var in variants:
        cfg, g, props, st = setup(grid, VARIANTS[var])
        m0 = TVSAModel(cfg, g, props, cfg.cycle[0], st)
        y0 = torch.from_numpy(m0.pack(st)).to(dev)
        net = None
        if var.startswith("learned"):
            if not os.path.exists(weights_path):
                out[var] = {"skipped": f"no trained weights at {os.path.relpath(weights_path, ROOT)}"}
                continue
            net = NewtonPredictor.load(weights_path)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        y, stats, _ = run_cycle_device(y0, cfg, g, props, predictor=net, predict=net is not None, inventories=True)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0                # (includes two host copies of the state per step)
        yh = y.cpu().numpy()
        keys = ("steps", "rejected", "newton_iters", "gmres_iters", "gmres_polish", "balance_unclosed",
                "pred_net", "pred_extrap", "pred_retry")
        keys += ("balance_projected",)
        rec = {"value": CYCLE_BED_S / wall, "wall_s": wall, "config": VARIANTS[var],
               "balance_errors": cycle_balance_errors(cfg, stats),
               "solver": {k: int(sum(s.get(k, 0) for s in stats)) for k in keys}}
        if var == "fp64":
            y64 = yh
        elif y64 is not None:
            sc = m0.atol + cfg.solver.rtol * np.abs(y64)
            rec["state_diff_vs_fp64_rel_max"] = float(np.max(np.abs(yh - y64) / (np.abs(y64) + m0.atol)))
            rec["state_diff_vs_fp64_scaled_rms"] = float(np.sqrt(np.mean(((yh - y64) / sc) ** 2)))
            rec["speedup_vs_fp64"] = rec["value"] / out["fp64"]["value"]
        out[var] = rec
    return out


def reference_cycle_parity(dev):
    """The 8x8x32 cycle through the public step runner against the reference's own cycle: step-end
    states (scaled by the solver's error scale) and the worst mass / energy balance errors."""
    import numpy as np
    from dac_vtsa_b200 import balances, host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.runner import run_step
    d = np.load(REF_CYCLE)
    cfg = load_config(override_dict=json.loads(str(d["over"])))
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    tmpl = host.initial_state(cfg, g, props)
    m0 = TVSAModel(cfg, g, props, cfg.cycle[0], tmpl)
    st = m0.to_state(d["y0"], tmpl, 0.0, "initial")
    steps, T_prev, t_cycle, per_step = [], None, 0.0, []
    t0 = time.perf_counter()
    for k, step in enumerate(cfg.cycle):
        st, sr = run_step(st, cfg, g, props, step, cycle_idx=1, t_cycle0=t_cycle, T_jacket_prev=T_prev,
                          record_outlet=False)
        y = m0.pack(st)
        yr = d[f"s{k}_y"]
        sc = m0.atol + cfg.solver.rtol * np.abs(yr)
        per_step.append({"step": step["name"], "scaled_rms": float(np.sqrt(np.mean(((y - yr) / sc) ** 2))),
                         "rel_max": float(np.max(np.abs(y - yr) / (np.abs(yr) + m0.atol)))})
        t_cycle += sr.duration
        T_prev = sr.T_jacket if sr.jacket_on else T_prev
        steps.append(sr)
    return {"wall_s": time.perf_counter() - t0, "step_end_vs_reference": per_step,
            "balance_errors": balances.worst_balance_errors(steps, ("CO2", "H2O", "N2")),
            "reference_balance_errors": {"mass": float(np.abs(d["mass_rel_err"]).max()),
                                         "energy": float(np.abs(d["energy_rel_err"]).max())}}


# ---------------------------------------------------------------------------- GPU arm
def gpu_arm(a, rank, world, local_rank):
    import numpy as np
    import torch
    from dac_vtsa_b200 import _lib, counters
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.runner import run_cycle, run_cycle_device
    from dac_vtsa_b200.solver import TRBDF2

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    wl = WORKLOADS[a.workload]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if wl.get("window"):
        w = Window(TVSAModel)
        model = w.model(TVSAModel)
        integ = TRBDF2(model, w.cfg, h_max=w.h_max, h_init=w.h_init)
        y0_dev = torch.from_numpy(w.y).to(dev)
        bed_per_step = WINDOW_BED_S

        def one_step():
            r = integ.integrate(y0_dev, WINDOW_BED_S, [WINDOW_BED_S], keep_on_device=True)
            return r.y, dict(integ.stats, steps=r.n_steps, rejected=r.n_reject)
    else:
        cfg, grid, props, st = setup(wl["grid"])
        m0 = TVSAModel(cfg, grid, props, cfg.cycle[0], st)
        y0_dev = torch.from_numpy(m0.pack(st)).to(dev)
        bed_per_step = CYCLE_BED_S

        def one_step():
            y, stats, _ = run_cycle_device(y0_dev.clone(), cfg, grid, props)
            return y, stats

    for _ in range(a.warmup):
        one_step()
    # ---- timed region: K device-resident steps
    sampler = ClockSampler(local_rank if "CUDA_VISIBLE_DEVICES" not in os.environ else
                           os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local_rank])
    sampler.start()
    barrier()
    total_ms = 0.0
    launches0 = _lib.launch_count()
    stream = torch.cuda.current_stream()
    stats_last = None
    for _ in range(a.steps):
        flush.fill_(1.0)                         # evict L2 between timed steps (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        y_end, stats_last = one_step()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    barrier()
    launches = _lib.launch_count() - launches0
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, dist, dev)
    value = replica_throughput(world, a.steps, bed_per_step, total_ms / 1e3)
    # ---- e2e: the public API with host states in and out (one untimed warm-up step of the same path)
    def e2e_step():
        if wl.get("window"):
            m = w.model(TVSAModel)
            r = TRBDF2(m, w.cfg, h_max=w.h_max, h_init=w.h_init).integrate(w.y, WINDOW_BED_S, [WINDOW_BED_S])
            assert np.all(np.isfinite(r.y))
        else:
            run_cycle(st.copy(), cfg, grid, props, record_outlet=True)

    e2e_step()
    counters.reset()
    barrier()
    nE = max(1, a.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(nE):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e = {"value": replica_throughput(world, nE, bed_per_step, e2e_s), "unit": "bed-s/wall-s",
           "h2d_bytes_per_step": counters.TRAFFIC["h2d"] // nE, "d2h_bytes_per_step": counters.TRAFFIC["d2h"] // nE,
           "path": ("TRBDF2(TVSAModel(...)).integrate(host numpy y0) per window, the reference runner's usage"
                    if wl.get("window") else "runner.run_cycle, outlet recorded at every accepted step")}
    # ---- one profiled step: per-kernel device time from CUDA events around every launch
    _lib.profile_enable(True)
    one_step()
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    kinds = {k: v for k, v in prof.items() if v[1] > 0}
    dom = max((k for k in kinds if k != "vector"), key=lambda k: kinds[k][2])
    n_l, n_t, ms = kinds[dom]
    avg_step_s = ms / 1e3 / n_t
    mref = model if wl.get("window") else m0
    nbs = None
    if dom in ("precond_apply", "precond_factor"):
        sweep_s, nbs = sweep_seconds(mref, y_end, 0.29 * 100.0)
    avg_s = sweep_s if dom == "precond_apply" else avg_step_s
    peak, peak_src = load_peaks()
    alg = alg_bytes_per_launch(dom, mref, nbs)
    achieved = alg / avg_s / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_path):
        try:
            traffic = json.load(open(tr_path)).get(a.workload, {}).get(dom)
        except ValueError:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 3), "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "alg_bytes_per_launch": alg, "avg_launch_us": avg_s * 1e6,
                "avg_launch_us_in_step": avg_step_s * 1e6, "partition_nb": nbs,
                "alg_bytes_rule": ALG_BYTES_DOC.get(dom, ""),
                "kernel_share": {k: round(v[2] / sum(x[2] for x in kinds.values()), 4) for k, v in kinds.items()},
                "launches_per_step": int(sum(x[0] for x in kinds.values())),
                "kernel_avg_us": {k: round(1e3 * v[2] / v[1], 3) for k, v in kinds.items()}}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu and wl.get("window"):
        bed, wall = _cpu_sample(a.workload)
        cpu = {"value": bed / wall, "unit": "bed-s/wall-s", "cores": 1, "kind": "port",
               "sample": f"{window_description()}; the whole window, 1 process, {cpu_model_name()}"}
    # ---- extra keys: full cycles (not part of the timed line)
    cycles = None
    if rank == 0 and not a.no_cycles:
        weights = os.path.join(ROOT, "dac_vtsa_b200", "predictor_weights.npz")
        cycles = {"8x8x32": cycle_runs((8, 8, 32), tuple(VARIANTS), weights, dev)}
        if os.path.exists(REF_CYCLE):
            cycles["8x8x32"]["reference_parity"] = reference_cycle_parity(dev)
        cycles["8x8x32"]["reference_cpu_cycle"] = CPU_FULL_CYCLE
        if not a.no_big:
            cycles["16x16x64"] = cycle_runs((16, 16, 64), tuple(VARIANTS), weights, dev)
    if rank == 0:
        line = {"metric": "bed-s simulated per wall-s", "value": value, "unit": "bed-s/wall-s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": a.workload, "grid": list(wl["grid"]),
                           "step": window_description() if wl.get("window") else "full cycle",
                           "bed_s_per_step": bed_per_step, "scheme": "trbdf2", "precision": "fp64",
                           "l2": "flushed between timed steps (256 MB write)",
                           "parallelism": f"{world} independent replicas (one per GPU)"},
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks, "solver": stats_last, "cycles": cycles}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="heat_window_8x8x32")
    ap.add_argument("--e2e-steps", type=int, default=5, help="steps of the e2e measurement (their mean)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-cycles", action="store_true", help="skip the full-cycle extra keys")
    ap.add_argument("--no-big", action="store_true", help="skip the 16x16x64 cycles among them")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        if WORKLOADS[a.workload].get("window"):
            reference_arm(a, rank)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the CPU reference runs bounded windows only "
                              "(heat_window_8x8x32); a full cycle takes 1838 s per core"}), flush=True)
        return
    gpu_arm(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
