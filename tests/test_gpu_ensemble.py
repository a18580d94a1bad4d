"""Ensemble of uneven columns solved concurrently on one GPU (dac_vtsa_b200.ensemble): three beds of
different grids and operating points with a shortened cycle (adsorption 200 s, blowdown 10 s,
heating 200 s, cooling 50 s)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = ((3, 4, 6), (4, 4, 8), (2, 4, 12))


def _columns():
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.ensemble import draw_columns
    cyc = [dict(s) for s in load_config().cycle]
    for s, d in zip(cyc, (200.0, 10.0, 200.0, 50.0)):
        s["duration"] = d
    cols = draw_columns(len(GRIDS), seed=4)
    for c, (nr, nt, nz) in zip(cols, GRIDS):
        c.update({"grid.Nr": nr, "grid.Ntheta": nt, "grid.Nz": nz, "cycle": cyc})
    return cols


def test_concurrent_columns_equal_one_at_a_time():
    """Columns on their own streams and host threads give bit-identical end states and solver
    statistics to the same columns run one after another: the columns share no device state."""
    from dac_vtsa_b200.ensemble import column_errors, run_ensemble
    cols = _columns()
    seq, rate1, _ = run_ensemble(cols, threads=1)
    par, rate3, _ = run_ensemble(cols, threads=3)
    for a, b in zip(par, seq):
        assert np.array_equal(a.y, b.y)
        assert a.stats == b.stats
        assert a.bed_s == pytest.approx(460.0)
    assert max(column_errors(par, seq)) == 0.0
    assert rate1 > 0.0 and rate3 > 0.0
