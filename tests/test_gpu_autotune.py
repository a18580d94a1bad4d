"""Launch-parameter autotuner: valid choices from measured candidates, cached per shape, and no
result bit changed by any choice."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _c0():
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_gpu_solver import _c0_model
    from dac_vtsa_b200.model import TVSAModel
    return _c0_model(TVSAModel)


def test_autotune_choices_are_measured_candidates():
    from dac_vtsa_b200 import autotune
    d, m, cfg, meta = _c0()
    params, times = autotune.tune(m, d["s0_y0"], dh=0.5, reps=10)
    assert params["fdjac_block"] in (64, 128)
    assert params["spmv_block"] in (64, 128, 256)
    assert params["gmres_prefix"] in (0, 2, 4, 6, 8)
    assert params["sweep_nbuf"] in (0, 2, 3)
    assert params["gmres_body"] in (1, 2)
    assert all(times[k] > 0 for k in ("fdjac_64", "fdjac_128", "spmv_64", "spmv_128", "spmv_256", "stage_prefix0"))
    assert autotune.get(m) == params


def test_tuned_parameters_do_not_change_results(tmp_path, monkeypatch):
    """The same 200 s adsorption with the library defaults and with every parameter at a non-default
    candidate ends in the bit-identical state with the same step and GMRES counts; the cache file
    holds the tuned choice for the next model of the shape."""
    from dac_vtsa_b200 import autotune
    from dac_vtsa_b200.solver import TRBDF2
    monkeypatch.setenv("DVTSA_TUNE_CACHE", str(tmp_path / "tune.json"))
    runs = []
    for params in (None, {"gmres_prefix": 0, "sweep_nbuf": 2, "spmv_block": 256, "fdjac_block": 64,
                          "gmres_body": 1}):
        d, m, cfg, meta = _c0()
        if params:
            autotune.apply(m, params)
        dur = meta["duration"]
        integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
        r = integ.integrate(d["s0_y0"], dur, [dur])
        runs.append((r.y, r.n_steps, integ.stats["gmres_iters"]))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1:] == runs[1][1:]
    d, m, cfg, meta = _c0()
    chosen = autotune.cached(m, d["s0_y0"], dh=0.5)
    table = json.load(open(tmp_path / "tune.json"))
    assert list(table.values())[0]["params"] == chosen
    d, m2, _, _ = _c0()
    assert autotune.cached(m2, d["s0_y0"], dh=0.5) == chosen and autotune.get(m2) == chosen
