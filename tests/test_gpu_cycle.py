"""Full 8x8x32 cycle (adsorption 8000 s, blowdown 60 s, heating 22 400 s, cooling 400 s, TR-BDF2 at
the reference defaults, seeded constant-pressure start) through the public step runner, against the
reference's own cycle from the same state (tests/golden/cycle_8x8x32.npz):

* every step-end state agrees entry by entry within the solver's own error scale atol + rtol |y|
  (the tolerance both solvers are held to; two correct adaptive solvers agree to about that);
* the accepted step counts agree within 5 %;
* the balance closures of the cycle (validation/conservation_checks.py:29-67, computed by
  dac_vtsa_b200.balances, which reproduces the reference's rows) stay within the reference's stored
  default-run balance errors (validation/baseline/default_kpis.json:33-34: mass 6.77e-6, energy
  4.37e-6) and far inside its alarm threshold 1e-4.
"""
import json

import numpy as np
import pytest

from cases import golden

pytestmark = pytest.mark.gpu

REF_BASELINE = {"mass": 6.77e-6, "energy": 4.37e-6}


def _run_cycle(over_extra=None):
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.runner import run_step
    d = golden("cycle_8x8x32.npz")
    over = json.loads(str(d["over"]))
    over.update(over_extra or {})
    cfg = load_config(override_dict=over)
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    tmpl = host.initial_state(cfg, g, props)
    m0 = TVSAModel(cfg, g, props, cfg.cycle[0], tmpl)
    st = m0.to_state(d["y0"], tmpl, 0.0, "initial")
    steps, ys, T_prev, t_cycle = [], [], None, 0.0
    for step in cfg.cycle:
        st, sr = run_step(st, cfg, g, props, step, cycle_idx=1, t_cycle0=t_cycle, T_jacket_prev=T_prev,
                          record_outlet=False)
        ys.append(m0.pack(st))
        t_cycle += sr.duration
        T_prev = sr.T_jacket if sr.jacket_on else T_prev
        steps.append(sr)
    return d, cfg, m0, steps, ys


def test_cycle_matches_the_reference_cycle():
    from dac_vtsa_b200 import balances
    d, cfg, m0, steps, ys = _run_cycle()
    for k, (sr, y) in enumerate(zip(steps, ys)):
        yr = d[f"s{k}_y"]
        scaled = np.abs(y - yr) / (m0.atol + cfg.solver.rtol * np.abs(yr))
        assert scaled.max() <= 1.0, (sr.name, float(scaled.max()))
        ref_steps = json.loads(str(d[f"s{k}_solver"]))["steps"]
        assert abs(sr.solver["steps"] - ref_steps) <= max(3, 0.05 * ref_steps), (sr.name, sr.solver["steps"], ref_steps)
    worst = balances.worst_balance_errors(steps, ("CO2", "H2O", "N2"))
    assert worst["mass"] <= REF_BASELINE["mass"], worst
    assert worst["energy"] <= REF_BASELINE["energy"], worst
    # the same input in the reference: energy closes as tightly, species within a small factor
    assert worst["energy"] <= 2.0 * float(np.abs(d["energy_rel_err"]).max()), worst
    assert worst["mass"] <= 10.0 * float(np.abs(d["mass_rel_err"]).max()), worst


def test_cycle_with_restarted_polish_closes_balances_better_than_the_reference():
    """gpu.polish_cycles 4: the polish iterations' linear solves reach their tolerance as the
    reference's exact sparse-LU solves do, and both balances close at least as tightly as in the
    reference's own cycle from the same input; the states stay within the error scale."""
    from dac_vtsa_b200 import balances
    d, cfg, m0, steps, ys = _run_cycle({"gpu.polish_cycles": 4})
    for k, (sr, y) in enumerate(zip(steps, ys)):
        yr = d[f"s{k}_y"]
        assert (np.abs(y - yr) / (m0.atol + cfg.solver.rtol * np.abs(yr))).max() <= 1.0, sr.name
    worst = balances.worst_balance_errors(steps, ("CO2", "H2O", "N2"))
    assert worst["mass"] <= float(np.abs(d["mass_rel_err"]).max()), worst
    assert worst["energy"] <= float(np.abs(d["energy_rel_err"]).max()), worst


def test_cycle_with_balance_projection():
    """gpu.balance_projection: balances better than the reference's on the same input; the step-end
    states within the error scale; the accepted steps within 35 % (the projection moves each stage
    solution by about |W R| / |W z|, which the step-size control sees)."""
    from dac_vtsa_b200 import balances
    d, cfg, m0, steps, ys = _run_cycle({"gpu.balance_projection": True})
    for k, (sr, y) in enumerate(zip(steps, ys)):
        yr = d[f"s{k}_y"]
        assert (np.abs(y - yr) / (m0.atol + cfg.solver.rtol * np.abs(yr))).max() <= 1.0, sr.name
        ref_steps = json.loads(str(d[f"s{k}_solver"]))["steps"]
        assert sr.solver["steps"] <= 1.35 * ref_steps + 3, (sr.name, sr.solver["steps"], ref_steps)
    worst = balances.worst_balance_errors(steps, ("CO2", "H2O", "N2"))
    assert worst["mass"] <= float(np.abs(d["mass_rel_err"]).max()), worst
    assert worst["energy"] <= float(np.abs(d["energy_rel_err"]).max()), worst


def test_16x16x64_cycle_with_balance_projection():
    """The 16x16x64 bed (99 328 unknowns; the reference cannot run it): one full cycle from the
    seeded constant-pressure state with the balance projection closes mass and energy to 1e-6 (the
    reference's stored default-run errors are 6.77e-6 / 4.37e-6)."""
    import torch
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.runner import BENCH_POINT, cycle_balance_errors, run_cycle_device
    cfg = load_config(override_dict=dict(BENCH_POINT, **{"grid.Nr": 16, "grid.Ntheta": 16, "grid.Nz": 64,
                                                         "gpu.balance_projection": True}))
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, g, props, seed=0)
    y0 = torch.from_numpy(TVSAModel(cfg, g, props, cfg.cycle[0], st).pack(st)).cuda()
    y, stats, _ = run_cycle_device(y0, cfg, g, props, inventories=True)
    assert np.all(np.isfinite(y.cpu().numpy()))
    worst = cycle_balance_errors(cfg, stats)
    assert worst["mass"] <= 1e-6 and worst["energy"] <= 1e-6, worst
