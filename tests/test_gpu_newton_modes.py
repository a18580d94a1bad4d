"""The reference's other Newton modes on the GPU (core/solver.py:111-151,339-347): hybrid (modified
Newton with the stored factors first, Newton-Krylov when it stalls) and modified (the full
factorisation, no Krylov).  A free-running 200 s adsorption of the 4x4x16 bed ends within the
solver's own error scale of the reference's end state, with a step count close to the reference's."""
import json

import numpy as np
import pytest

from cases import build, golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["hybrid", "modified"])
def test_newton_mode_matches_reference(mode):
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d = golden("newton_modes_4x4x16.npz")
    over = json.loads(str(d[f"{mode}_over"]))
    ref = json.loads(str(d[f"{mode}_stats"]))
    m, cfg = build(TVSAModel, over, 0, d[f"{mode}_P0"], duration=200.0)
    integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * 200.0)
    res = integ.integrate(d[f"{mode}_y0"], 200.0, [200.0])
    y_ref = d[f"{mode}_y"]
    sc = m.atol + cfg.solver.rtol * np.abs(y_ref)
    err = np.sqrt(np.mean(((res.y - y_ref) / sc) ** 2))
    assert res.t == pytest.approx(200.0)
    assert err < 5.0, err
    assert abs(res.n_steps - ref["steps"]) <= max(5, 0.25 * ref["steps"]), (res.n_steps, ref["steps"])
    if mode == "modified":
        assert integ.mode == "modified" and res.n_krylov == 0     # full factors: no Krylov at all
    else:
        assert integ.stats["modified_fail"] > 0 and res.n_krylov > 0
