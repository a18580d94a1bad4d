#!/usr/bin/env python
"""Throughput of the implicit stepping path: simulated bed-seconds per wall-second.

Workload (default ``cycle_8x8x32``): one full adsorption (8000 s) -> blowdown (60 s) -> heating
(22400 s) -> cooling (400 s) cycle of an 8x8x32 bed (2048 cells, 12 544 unknowns, FP64), TR-BDF2
scheme, reference solver defaults, from the seeded constant-pressure initial state (clean bed,
T = 288 (1 +- 1 %), numpy default_rng(0)); feed 400 ppm CO2 at 50 % RH and 288 K, T_heat 373 K,
P_vacuum 10 kPa.  A "step" of this benchmark is one such cycle.

ours (default):
  value  device-resident cycle (state stays on the GPU), CUDA events per cycle, L2 flushed between
         cycles (a 256 MB buffer is written), max over ranks; N GPUs run N independent replicas
  e2e    the same cycle through the public step-runner API with host numpy states and outlet
         recording at every accepted step (the reference's steps/_runner.py usage)
  roofline: per-kernel shares of one profiled cycle (CUDA events around each launch); the
         dominant kernel (the sweep) timed back to back on its stream for its duration
  cpu_baseline: the CPU oracle (numpy restatement of the reference) on a bounded sample, 1 core
--impl reference: the oracle timed on the host cores (one process per core) on a bounded sample.
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
    "cycle_8x8x32": {"grid": (8, 8, 32)},
    "cycle_4x4x16": {"grid": (4, 4, 16)},
}
SAMPLE_STATE = os.path.join(ROOT, "tests", "golden", "bench_state_8x8x32_heat4000.npz")
SAMPLE_BED_S = 2000.0        # CPU sample window: bed-seconds of heating restarted from SAMPLE_STATE
CPU_FULL_CYCLE = "1779 s for the 30 860 bed-s cycle (17.3 bed-s/wall-s) on one core of the build host"


def overrides(grid):
    Nr, Nth, Nz = grid
    return {"grid.Nr": Nr, "grid.Ntheta": Nth, "grid.Nz": Nz, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}


def setup(workload):
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    cfg = load_config(override_dict=overrides(WORKLOADS[workload]["grid"]))
    grid = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, grid, props, seed=0)
    return cfg, grid, props, st


# ---------------------------------------------------------------------------- CPU oracle sample
def sample_description():
    return (f"heating step of the 8x8x32 cycle restarted from the reference's own state after adsorption, "
            f"blowdown and 4000 s of heating (tests/golden/{os.path.basename(SAMPLE_STATE)}), at the reference's "
            f"last step size, integrated for {SAMPLE_BED_S:g} bed-s at the reference defaults.  Mid-heating is the "
            f"CPU path's fastest regime (about 5x its cycle average), so this sample overstates the CPU "
            f"throughput of a full cycle; the full reference cycle measured {CPU_FULL_CYCLE}")


def _cpu_sample(workload, duration=SAMPLE_BED_S):
    """The CPU oracle on the bounded sample; returns (bed-seconds, wall seconds)."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import numpy as np
    from oracle.residual import OracleModel
    from oracle.solver import OracleTRBDF2
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    d = np.load(SAMPLE_STATE)
    cfg = load_config(override_dict=json.loads(str(d["over"])))
    grid = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    y = d["y"]
    step = dict(cfg.cycle[2])
    st = host.seeded_state(cfg, grid, props, seed=0)
    tmp = OracleModel(cfg, grid, props, step, st)
    c, q, e, Tw = tmp.unpack(y)
    st.c, st.q, st.T, st.Tw = c.copy(), q.copy(), tmp.temperature(e, c, q), Tw.copy()
    m = OracleModel(cfg, grid, props, step, st, float(d["T_jacket"]))
    t0 = time.perf_counter()
    integ = OracleTRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * step["duration"], h_init=float(d["h_last"][-2]))
    res = integ.integrate(y, duration, [duration])
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
    host cores: each step is a batch of one bounded sample per core, run in parallel processes."""
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
            "config": {"workload": a.workload, "sample": sample_description(), "parallelism": f"{procs} processes"},
            "cpu_baseline": {"value": value, "unit": "bed-s/wall-s", "cores": procs, "kind": "port",
                             "sample": f"{procs} processes x ({sample_description()}), {cpu_model_name()}"},
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


def replica_throughput(world, cycles, seconds):
    """Whole-job bed-seconds per wall-second: every rank runs `cycles` independent cycles."""
    return world * cycles * CYCLE_BED_S / seconds


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


# ---------------------------------------------------------------------------- GPU arm
ALG_BYTES_DOC = {
    "matvec": "FD matvec residual: reads z, u, s, f (4 n_core) + writes n_core doubles",
    "residual": "residual: reads y (+ rhs_known) and writes f: 2 n_core doubles",
    "precond_apply": "sweep: reads the 5 nb x nb factor blocks of every plane of every partition + 3 n_core doubles",
    "fd_jacobian": "reads y, f0 (2 n_core) + writes the 9*49*ncell block layout",
    "precond_factor": "assembly + factorisation: writes and re-reads 5 blocks per plane",
    "vector": "Krylov vector kernels: ~3 n_core doubles per launch (average)",
}


def partition_sizes(m):
    """Unknowns per z-partition of the preconditioner the solver builds for model m (block nb of
    each partition): theta_block with >= 1 coupled ring = the innermost ring of all sectors plus
    rings 1.. of each sector with its wall node; theta_block with 0 rings = whole sectors; full =
    one partition (also for a single sector)."""
    g, s, w = m.grid, m.cfg.solver, (1 if m.n_w else 0)
    mode = s.preconditioner if g.Nth > 1 else "full"
    if mode == "theta_block" and s.precond_theta_rings >= 1 and g.Nr >= 2:
        return [6 * (g.Nr - 1) + w] * g.Nth + [6 * g.Nth]
    if mode == "theta_block":
        return [6 * g.Nr + w] * g.Nth
    return [6 * g.Nr * g.Nth + w * g.Nth]


def alg_bytes_per_launch(kind, m):
    n = m.n_core
    if kind == "matvec":
        return 5 * n * 8
    if kind == "residual":
        return 2 * n * 8
    if kind == "fd_jacobian":
        return (2 * n + m.jac_doubles) * 8
    blocks = m.grid.Nz * 5 * sum(nb * nb for nb in partition_sizes(m)) * 8
    if kind == "precond_apply":
        return blocks + 3 * n * 8
    if kind == "precond_factor":
        return 2 * blocks
    return 3 * n * 8


def sweep_seconds(m, y, launches=200):
    """Average duration of the preconditioner sweep: the factors of I - dh J at state y (the
    solver's partitions), then `launches` back-to-back dv_precond_solve calls bracketed by CUDA
    events on the launching stream (the queue never drains, so no host latency is counted)."""
    import ctypes as C
    import torch
    from dac_vtsa_b200.jacobian import FDJacobian
    yd = y.contiguous() if isinstance(y, torch.Tensor) else torch.from_numpy(y).to(m.device)
    m.precond_factor(FDJacobian(m).block(0.0, yd), 2.1)
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
    return e0.elapsed_time(e1) / 1e3 / launches


def gpu_arm(a, rank, world, local_rank):
    import numpy as np
    import torch
    from dac_vtsa_b200 import _lib, counters
    from dac_vtsa_b200.runner import run_cycle, run_cycle_device

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    cfg, grid, props, st = setup(a.workload)
    from dac_vtsa_b200.model import TVSAModel
    m0 = TVSAModel(cfg, grid, props, cfg.cycle[0], st)
    y0_host = torch.from_numpy(m0.pack(st)).pin_memory()
    y0_dev = y0_host.to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def one_cycle():
        y, stats, _ = run_cycle_device(y0_dev.clone(), cfg, grid, props)
        return y, stats

    for _ in range(a.warmup):
        one_cycle()
    # ---- timed region: K device-resident cycles
    sampler = ClockSampler(local_rank if "CUDA_VISIBLE_DEVICES" not in os.environ else
                           os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local_rank])
    sampler.start()
    barrier()
    total_ms = 0.0
    launches0 = _lib.launch_count()
    stream = torch.cuda.current_stream()
    stats_last = None
    for _ in range(a.steps):
        flush.fill_(1.0)                         # evict L2 between timed cycles (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        y_end, stats_last = one_cycle()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    barrier()
    launches = _lib.launch_count() - launches0
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, dist, dev)
    value = replica_throughput(world, a.steps, total_ms / 1e3)
    # ---- e2e: public step-runner API, host states, outlet recording per accepted step
    counters.reset()
    barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, a.e2e_steps)):
        st_in = st.copy()
        run_cycle(st_in, cfg, grid, props, record_outlet=True)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    nE = max(1, a.e2e_steps)
    e2e_s = max_over_ranks(e2e_s, dist, dev)
    e2e = {"value": replica_throughput(world, nE, e2e_s), "unit": "bed-s/wall-s",
           "h2d_bytes_per_step": counters.TRAFFIC["h2d"] // nE, "d2h_bytes_per_step": counters.TRAFFIC["d2h"] // nE,
           "path": "runner.run_cycle (steps/_runner.py-compatible run_step per cycle step, outlet recorded at "
                   "every accepted step)"}
    # ---- mixed precision (gpu.krylov_precision = fp32: FP32 factor storage in the preconditioner
    # sweep), the same cycle, one warm-up and one timed cycle; state difference to the FP64 cycle
    mixed = None
    if not a.no_mixed:
        from dac_vtsa_b200.config import load_config
        cfg32 = load_config(override_dict=dict(overrides(WORKLOADS[a.workload]["grid"]),
                                               **{"gpu.krylov_precision": "fp32"}))
        run_cycle_device(y0_dev.clone(), cfg32, grid, props)
        flush.fill_(1.0)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        y32, st32, _ = run_cycle_device(y0_dev.clone(), cfg32, grid, props)
        e1.record(stream)
        e1.synchronize()
        ms32 = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        y64h, y32h = y_end.double().cpu().numpy(), y32.double().cpu().numpy()
        sc = m0.atol + cfg.solver.rtol * np.abs(y64h)
        dev_scaled = (y32h - y64h) / sc
        mixed = {"value": replica_throughput(world, 1, ms32 / 1e3), "unit": "bed-s/wall-s", "ms_per_step": ms32,
                 "precision": "FP32 preconditioner factors, FP64 residual/Jacobian/Newton/GMRES vectors",
                 "state_diff_vs_fp64_scaled_rms": float(np.sqrt(np.mean(dev_scaled ** 2))),
                 "state_diff_vs_fp64_scaled_max": float(np.abs(dev_scaled).max()),
                 "state_diff_vs_fp64_rel_max": float(np.max(np.abs(y32h - y64h) / (np.abs(y64h) + m0.atol))),
                 "solver": st32}
    # ---- one profiled cycle: per-kernel device time from CUDA events around every launch
    _lib.profile_enable(True)
    _, _ = one_cycle()
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    kinds = {k: v for k, v in prof.items() if v[1] > 0}
    # the roofline names one kernel; "vector" is the class of small Krylov kernels, not one kernel
    dom = max((k for k in kinds if k != "vector"), key=lambda k: kinds[k][2])
    n_l, n_t, ms = kinds[dom]
    avg_cycle_s = ms / 1e3 / n_t
    # the per-launch events of the profiled cycle also hold each launch's host latency (the GPU
    # waits for the host there), so the kernel's own duration is timed back to back on its stream
    avg_s = sweep_seconds(m0, y_end) if dom == "precond_apply" else avg_cycle_s
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    alg = alg_bytes_per_launch(dom, m0)
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
                "avg_launch_us_in_cycle": avg_cycle_s * 1e6,
                "alg_bytes_rule": ALG_BYTES_DOC.get(dom, ""),
                "kernel_share": {k: round(v[2] / sum(x[2] for x in kinds.values()), 4) for k, v in kinds.items()},
                "launches_per_cycle": int(sum(x[0] for x in kinds.values())),
                "kernel_avg_us": {k: round(1e3 * v[2] / v[1], 3) for k, v in kinds.items()}}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        bed, wall = _cpu_sample(a.workload)
        cpu = {"value": bed / wall, "unit": "bed-s/wall-s", "cores": 1, "kind": "port",
               "sample": f"{sample_description()}; 1 process, {cpu_model_name()}"}
    if rank == 0:
        line = {"metric": "bed-s simulated per wall-s", "value": value, "unit": "bed-s/wall-s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": a.workload, "grid": list(WORKLOADS[a.workload]["grid"]),
                           "cycle_bed_s": CYCLE_BED_S, "scheme": "trbdf2", "precision": "fp64",
                           "l2": "flushed between timed cycles (256 MB write)",
                           "parallelism": f"{world} independent replicas (one per GPU)"},
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "mixed_precision": mixed,
                "clocks": clocks, "solver": stats_last}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cycle_8x8x32")
    ap.add_argument("--e2e-steps", type=int, default=2, help="cycles of the e2e measurement (their mean)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision cycle")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank)
        return
    gpu_arm(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
