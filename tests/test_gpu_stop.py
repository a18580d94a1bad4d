"""Step stop criteria (core/residual.py:445-482, core/solver.py:476-494) on the GPU against the reference.

Fixture: the reference's young2021 1-D case (1x1x30 bed, lumped heat transfer, no wall), its
adsorption step with ``stop_on: end_saturation 0.9895`` from the case's initial state, run by the
reference's own step runner (tests/golden/make_golden.py --stop)."""
import json

import numpy as np
import pytest
import yaml

from cases import golden

pytestmark = pytest.mark.gpu


def _setup(tmp_path):
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    d = golden("stop_young2021.npz")
    case = tmp_path / "young2021.yaml"
    case.write_text(yaml.safe_dump(json.loads(str(d["case_yaml"]))))
    cfg = load_config(user_yaml=str(case))
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    return d, cfg, g, props


def test_stop_metric_and_feed_equilibrium_match_reference(tmp_path):
    from cases import state_like
    from dac_vtsa_b200.model import TVSAModel
    d, cfg, g, props = _setup(tmp_path)
    step = cfg.cycle[int(d["step_index"])]
    m = TVSAModel(cfg, g, props, step, state_like(d["P0"]))
    assert m.q_feed_eq() == pytest.approx(float(d["q_feed_eq"]), rel=1e-12)
    assert m.stop_metric(0.0, d["y0"]) == pytest.approx(float(d["metric0"]), rel=1e-10, abs=1e-14)
    # the criterion on the reference's own end state gives the reference's stop value
    assert m.stop_metric(float(d["t_stop"]), d["y_end"]) == pytest.approx(float(d["stop_value"]), rel=1e-10)


def test_adsorption_stops_on_end_saturation_like_the_reference(tmp_path):
    """The runner integrates until the end-layer CO2 loading reaches 98.95 % of the feed equilibrium:
    it stops early, past the threshold, within one maximum step of the reference's stop time, and
    the outlet series ends at the stop."""
    from dac_vtsa_b200.runner import run_step
    d, cfg, g, props = _setup(tmp_path)
    st = host_state(cfg, g, props)
    step = cfg.cycle[int(d["step_index"])]
    st1, sr = run_step(st, cfg, g, props, step, snapshots=2)
    thr = float(step["stop_on"]["value"])
    h_max = cfg.solver.h_max_fraction * float(step["duration"])
    assert sr.stopped_early
    assert sr.duration < float(step["duration"])
    assert abs(sr.duration - float(d["t_stop"])) <= h_max, (sr.duration, float(d["t_stop"]))
    assert sr.outlet[-1]["t_step_s"] == pytest.approx(sr.duration)
    from dac_vtsa_b200.model import TVSAModel
    m = TVSAModel(cfg, g, props, step, st)
    v = m.stop_metric(sr.duration, m.pack(st1))
    assert thr <= v < thr + 0.05, v


def host_state(cfg, g, props):
    from dac_vtsa_b200 import host
    return host.initial_state(cfg, g, props)
