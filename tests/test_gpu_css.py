"""Cycles to cyclic steady state on the GPU (dac_vtsa_b200.css.run_to_css, the reference's
vtsa_cycle.run_to_css, vtsa_cycle.py:93-138): a 3x4x6 bed with a shortened cycle (adsorption 200 s,
blowdown 10 s, heating 200 s, cooling 50 s), two cycles."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DURATIONS = (200.0, 10.0, 200.0, 50.0)


def _setup():
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    cyc = [dict(s) for s in load_config().cycle]
    for s, d in zip(cyc, DURATIONS):
        s["duration"] = d
    cfg = load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6, "solver.scheme": "trbdf2",
                                     "cycle": cyc})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    return cfg, g, props, host.initial_state(cfg, g, props)


def test_two_cycles_with_handoff_files(tmp_path):
    """Every cycle writes the reference's hand-off files (cycle start, every step end); cycle 1's
    final file holds exactly the state a plain device-resident cycle reaches from the same start; the
    cycle records carry the state change and CO2 balance computed from those states and flows."""
    from dac_vtsa_b200 import balances
    from dac_vtsa_b200.css import run_to_css
    from dac_vtsa_b200.handoff import load_state_csv
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.runner import run_cycle_device
    cfg, g, props, st0 = _setup()
    res = run_to_css(cfg, g, props, st0, run_dir=str(tmp_path), max_cycles=2)
    torch.cuda.synchronize()
    assert len(res.cycles) == 2 and not res.converged
    for n in (1, 2):
        d = tmp_path / f"cycle_{n:03d}"
        names = ["state_cycle_start"] + [f"state_after_{s['name']}" for s in cfg.cycle]
        for nm in names:
            assert (d / f"{nm}.csv").exists() and (d / f"{nm}_wall.csv").exists(), (n, nm)
    m0 = TVSAModel(cfg, g, props, cfg.cycle[0], st0)
    y1, stats, _ = run_cycle_device(torch.from_numpy(m0.pack(st0)).to(m0.device), cfg, g, props)
    end1 = m0.to_state(y1.cpu().numpy(), st0, 0.0, cfg.cycle[-1]["name"])
    back = load_state_csv(str(tmp_path / "cycle_001" / "state_after_cooling.csv"), g, st0.species, st0.adsorbed)
    for k in ("c", "q", "T", "Tw"):
        assert np.array_equal(getattr(back, k), getattr(end1, k)), k
    # the records: cycle 1 against the initial state, cycle 2 against cycle 1's end
    assert res.cycles[0].change == pytest.approx(balances.state_change(st0, end1, g, cfg), rel=1e-12)
    end2 = load_state_csv(str(tmp_path / "cycle_002" / "state_after_cooling.csv"), g, st0.species, st0.adsorbed)
    assert res.cycles[1].change == pytest.approx(balances.state_change(end1, end2, g, cfg), rel=1e-9)
    assert res.cycles[0].co2["CO2_fed_mol"] > 0.0
    assert res.cycles[1].change["max"] < res.cycles[0].change["max"]
