"""Cyclic-steady-state measures (dac_vtsa_b200.balances: state_change, co2_flows, cycle_co2_balance,
is_css) against the reference's own values (validation/cyclic_steady_state.py:22-44,
postprocessing/reporting.py:30-41), stored by tests/golden/make_golden.py --css."""
import json
import os

import numpy as np
import pytest

from cases import GOLDEN
from dac_vtsa_b200 import balances, host
from dac_vtsa_b200.config import load_config

CSS = os.path.join(GOLDEN, "css_3x4x6.npz")


def _states(d):
    cfg = load_config(override_dict=json.loads(str(d["over"])))
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    out = []
    for i in range(2):
        st = host.initial_state(cfg, g, props)
        st.c, st.q, st.T, st.Tw = d[f"s{i}_c"], d[f"s{i}_q"], d[f"s{i}_T"], d[f"s{i}_Tw"]
        out.append(st)
    return cfg, g, out


def test_state_change_equals_the_reference():
    d = np.load(CSS)
    cfg, g, (a, b) = _states(d)
    ch = balances.state_change(a, b, g, cfg)
    ref = json.loads(str(d["change"]))
    assert set(ch) == set(ref)
    for k in ref:
        assert ch[k] == pytest.approx(ref[k], rel=1e-12), k


def test_cycle_flows_and_css_decision_equal_the_reference():
    from test_balances import golden_steps
    d = np.load(CSS)
    cyc = np.load(os.path.join(GOLDEN, "cycle_8x8x32.npz"))
    _, steps = golden_steps(cyc)
    flows = balances.co2_flows(steps)
    ref = json.loads(str(d["flows"]))
    for k in ref:
        assert flows[k] == pytest.approx(ref[k], rel=1e-12), k
    assert balances.cycle_co2_balance(flows) == pytest.approx(float(d["co2_balance"]), rel=1e-12)
    cfg, g, (a, b) = _states(d)
    ch = balances.state_change(a, b, g, cfg)
    assert [balances.is_css(ch, flows, cfg, n) for n in range(1, 5)] == list(d["is_css"])
    relaxed = load_config(override_dict=dict(json.loads(str(d["over"])),
                                             **{"run.css_tolerance": 1.0, "run.css_mb_tolerance": 0.5}))
    assert [balances.is_css(ch, flows, relaxed, n) for n in range(1, 5)] == list(d["is_css_relaxed"])
