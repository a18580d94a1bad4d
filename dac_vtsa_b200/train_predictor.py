"""Train the learned Newton predictor on the GPU from the plain solver's own stage solutions.

    python -m dac_vtsa_b200.train_predictor --grid 8 8 32 --points 32 --out weights.npz

1. Operating points are drawn from a seed: T_heat ~ U(363, 393) K, P_vacuum ~ U(5, 30) kPa, feed
   RH ~ U(0.2, 0.8) (the ranges of the learned-predictor and ensemble studies).
2. For each point one full adsorption -> blowdown -> heating -> cooling cycle runs with the plain
   extrapolation predictor while the network records every ``stride``-th cell of every converged
   stage (features of the two latest levels, target = the stage solution's offset from the
   extrapolation in units of the cell's extrapolated increment plus 1 % of its error scale).
3. Adam on those samples with the library's BF16 tensor-core forward / backward kernels.
4. The gain: a held-out operating point's cycle with and without the network (Newton iterations,
   GMRES iterations, wall time).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import host
from .config import load_config
from .predictor import NewtonPredictor
from .runner import BENCH_POINT, run_cycle_device


def operating_points(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return [{"operation.T_heat": float(rng.uniform(363.0, 393.0)), "operation.P_vacuum": float(rng.uniform(5e3, 3e4)),
             "feed.RH": float(rng.uniform(0.2, 0.8))} for _ in range(n)]


def setup(grid, point, extra=None):
    over = dict(BENCH_POINT, **{"grid.Nr": grid[0], "grid.Ntheta": grid[1], "grid.Nz": grid[2]}, **point,
                **(extra or {}))
    cfg = load_config(override_dict=over)
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, g, props, seed=0)
    from .model import TVSAModel
    y0 = torch.from_numpy(TVSAModel(cfg, g, props, cfg.cycle[0], st).pack(st)).cuda()
    return cfg, g, props, y0


def cycle_stats(stats):
    keys = ("steps", "rejected", "newton_iters", "gmres_iters", "gmres_polish", "krylov_ok", "krylov_fail",
            "pred_net", "pred_extrap", "pred_retry")
    return {k: int(sum(s.get(k, 0) for s in stats)) for k in keys}


def timed_cycle(cfg, g, props, y0, predictor=None):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    y, stats, _ = run_cycle_device(y0.clone(), cfg, g, props, predictor=predictor, predict=predictor is not None)
    torch.cuda.synchronize()
    return y, stats, time.perf_counter() - t0


def record(net, grid, points, stride, log=print):
    for i, pt in enumerate(points):
        cfg, g, props, y0 = setup(grid, pt)
        t0 = time.perf_counter()
        run_cycle_device(y0, cfg, g, props, predictor=net, predict=False, record_stride=stride)
        torch.cuda.synchronize()
        log(f"  point {i}: {json.dumps(pt)} -> {net.samples} samples ({time.perf_counter() - t0:.1f} s)")


def evaluate(net, grid, point, extra=None):
    cfg, g, props, y0 = setup(grid, point, extra)
    timed_cycle(cfg, g, props, y0)                         # warm-up (graphs, colouring)
    y_p, s_p, w_p = timed_cycle(cfg, g, props, y0)
    y_n, s_n, w_n = timed_cycle(cfg, g, props, y0, predictor=net)
    a, b = y_p.cpu().numpy(), y_n.cpu().numpy()
    return {"plain": dict(cycle_stats(s_p), wall_s=w_p), "learned": dict(cycle_stats(s_n), wall_s=w_n),
            "state_rel_max": float(np.max(np.abs(b - a) / (np.abs(a) + 1e-30 + np.abs(a).max() * 1e-12)))}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, nargs=3, default=(8, 8, 32))
    ap.add_argument("--points", type=int, default=32)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--stride", type=int, default=0, help="record every stride-th cell (0: about 1e6 samples)")
    ap.add_argument("--steps", type=int, default=3000, help="Adam steps of 4096 samples")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default="predictor_weights.npz")
    ap.add_argument("--eval", action="store_true", help="compare a held-out point's cycle with and without")
    ap.add_argument("--load", default="", help="evaluate these weights (no recording or training)")
    ap.add_argument("--eval-grid", type=int, nargs=3, default=None, help="grid of the evaluation (default --grid)")
    a = ap.parse_args(argv)
    torch.cuda.init()
    eval_grid = tuple(a.eval_grid or a.grid)
    if a.load:
        held_out = operating_points(a.points + 1, a.seed)[-1]
        net = NewtonPredictor.load(a.load)
        print(json.dumps({"weights": a.load, "grid": list(eval_grid), "held_out_point": held_out,
                          "gain": evaluate(net, eval_grid, held_out)}), flush=True)
        return
    ncell = a.grid[0] * a.grid[1] * a.grid[2]
    # about 1200 converged stage solves per cycle: pick the stride for ~1e6 samples in total
    stride = a.stride or max(1, int(round(ncell * 1200 * a.points / 1.0e6)))
    pts = operating_points(a.points + 1, a.seed)
    train_pts, held_out = pts[:-1], pts[-1]
    net = NewtonPredictor(sample_capacity=int(1.3e6), seed=a.seed)
    t0 = time.perf_counter()
    print(f"recording: {a.points} operating points, grid {a.grid}, every {stride}th cell", flush=True)
    record(net, tuple(a.grid), train_pts, stride)
    t_rec = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = net.train(a.steps, lr=a.lr, seed=a.seed)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    net.save(a.out)
    out = {"grid": list(a.grid), "samples": net.samples, "stride": stride, "record_s": t_rec, "train_s": t_train,
           "steps": a.steps, "loss_first": float(np.mean(hist[:20])), "loss_last": float(np.mean(hist[-50:])),
           "weights": a.out}
    if a.eval:
        out["held_out_point"] = held_out
        out["gain"] = evaluate(net, eval_grid, held_out)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
