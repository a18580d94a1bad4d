"""Cycle accounting (dac_vtsa_b200/balances.py) against the reference's own numbers: the balance rows
its cycle driver computed for its 8x8x32 cycle (validation/conservation_checks.py:29-67, stored by
tests/golden/make_golden.py --cycle with the step accumulators and inventories they come from)."""
import json
import os
from types import SimpleNamespace

import numpy as np
import pytest

from cases import GOLDEN
from dac_vtsa_b200 import balances
from dac_vtsa_b200.config import load_config

CYCLE = os.path.join(GOLDEN, "cycle_8x8x32.npz")
ACC_NAMES = [f"{p}_{v}_{s}" for v in ("V1", "V2", "V3") for p in ("n_in", "n_out") for s in ("CO2", "H2O", "N2")]


def _acc_names():
    names = []
    for v in ("V1", "V2", "V3"):
        names += [f"n_in_{v}_{s}" for s in ("CO2", "H2O", "N2")] + [f"n_out_{v}_{s}" for s in ("CO2", "H2O", "N2")]
        names += [f"H_in_{v}", f"H_out_{v}", f"W_pump_{v}", f"W_fan_{v}"]
    return names + ["Q_jac_pos", "Q_jac_neg", "Q_amb", "Q_wb", "Q_hx_pos", "Q_hx_neg"]


def golden_steps(d):
    cfg = load_config(override_dict=json.loads(str(d["over"])))
    steps = []
    for k, step in enumerate(cfg.cycle):
        inv = json.loads(str(d[f"s{k}_inv"]))
        meta = json.loads(str(d[f"s{k}_meta"]))
        steps.append(SimpleNamespace(cycle=1, name=meta["name"], acc=dict(zip(_acc_names(), d[f"s{k}_acc"])),
                                     inv_start=inv["start"], inv_end=inv["end"],
                                     product_port=step.get("product_port", "V3"), valves=dict(step["valves"])))
    return cfg, steps


@pytest.mark.skipif(not os.path.exists(CYCLE), reason="cycle golden not generated")
def test_balance_rows_equal_the_reference_cycle_check():
    d = np.load(CYCLE)
    cfg, steps = golden_steps(d)
    mass, energy = balances.balance_rows(steps, ("CO2", "H2O", "N2"))
    ref = json.loads(str(d["balance_rows"]))
    assert len(mass) == len(ref["mass"]) and len(energy) == len(ref["energy"])
    for a, b in zip(mass + energy, ref["mass"] + ref["energy"]):
        assert a["step"] == b["step"]
        assert a["relative_error"] == pytest.approx(b["relative_error"], rel=1e-9, abs=1e-18)
    worst = balances.worst_balance_errors(steps, ("CO2", "H2O", "N2"))
    assert worst["mass"] == pytest.approx(np.abs(d["mass_rel_err"]).max(), rel=1e-9)
    assert worst["energy"] == pytest.approx(np.abs(d["energy_rel_err"]).max(), rel=1e-9)


@pytest.mark.skipif(not os.path.exists(CYCLE), reason="cycle golden not generated")
def test_cycle_co2_flows_close():
    d = np.load(CYCLE)
    cfg, steps = golden_steps(d)
    f = balances.co2_flows(steps)
    assert f["CO2_fed_mol"] > 0 and f["CO2_product_mol"] > 0
    # cycle 1 starts from a clean bed: what is fed and not produced or vented stays in the bed
    accumulated = steps[-1].inv_end["tot_CO2"] - steps[0].inv_start["tot_CO2"]
    net = f["CO2_fed_mol"] - f["CO2_product_mol"] - f["CO2_vented_mol"]
    assert abs(net - accumulated) <= 1e-5 * f["CO2_fed_mol"]
    assert balances.cycle_co2_balance(f) == pytest.approx(abs(net) / f["CO2_fed_mol"])
