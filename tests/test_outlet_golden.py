"""Outlet records (steps/_runner.py:50-84,104-121): the runner's outlet_row built from the
reference's own diagnostics (golden fixture) gives the reference's row; the model object only
supplies end conditions, species and layout (the CPU oracle model here)."""
import json

import numpy as np

from cases import build, golden


def _cases():
    d = golden("outlet_cases.npz")
    for m in json.loads(str(d["meta"])):
        yield d, m


def _ref_diag(d, m):
    n = m["name"]
    bnd = {end: {k: d[f"{n}__{end}__{k}"] for k in m["bnd_keys"][end]} for end in ("top", "bottom")}
    return {"T": d[f"{n}__T"], "P": d[f"{n}__P"], "y": d[f"{n}__yk"], "bnd": bnd}


def _same_row(row, ref, rtol, atol=0.0):
    assert set(row) == set(ref), set(row) ^ set(ref)
    for k, v in ref.items():
        a = row[k]
        a = a.value if hasattr(a, "value") else a
        if isinstance(v, str):
            assert a == v, (k, a, v)
        elif v is None or (isinstance(v, float) and np.isnan(v)):
            assert a is None or np.isnan(a), (k, a, v)
        else:
            assert abs(a - v) <= rtol * abs(v) + atol, (k, a, v)


def test_outlet_row_matches_reference_on_reference_diagnostics():
    from dac_vtsa_b200.runner import outlet_row
    from oracle.residual import OracleModel
    for d, m in _cases():
        om, _ = build(OracleModel, m["over"], m["step"], d[f"{m['name']}__P0"])
        row = outlet_row(om, _ref_diag(d, m), d[f"{m['name']}__y"], d[f"{m['name']}__acc"], m["c_feed_co2"],
                         om.grid.volume_full())
        _same_row(row, m["row"], rtol=1e-14, atol=1e-300)
