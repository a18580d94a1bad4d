"""The library's buffer pool: the device and pinned memory of destroyed models and integrators is
handed to the next handles of the same sizes (the reference's runner builds one model and one
integrator per cycle step), and results do not depend on whether a buffer is new or reused."""
import gc
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def _run(check_reuse=None):
    from test_gpu_solver import _c0_model
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d, m, cfg, meta = _c0_model(TVSAModel)
    dur = meta["duration"]
    integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
    if check_reuse is not None:
        assert _lib.pool_cached_bytes() < check_reuse       # the new handles took kept buffers
    r = integ.integrate(d["s0_y0"], dur, [dur])
    out = (np.array(r.y, copy=True), r.n_steps, integ.stats["gmres_iters"])
    del integ, m
    gc.collect()
    return out


def test_destroyed_handles_memory_is_reused_with_identical_results():
    """200 s adsorption of the 4x4x16 bed three times: after the first, the handles' buffers stay
    in the pool; the second run's handles take them (the kept bytes drop) and give back the same
    amount; after dv_pool_release nothing is kept and a third run with fresh buffers ends in the
    bit-identical state with the same step and GMRES counts."""
    from dac_vtsa_b200 import _lib
    _lib.pool_release()
    assert _lib.pool_cached_bytes() == 0
    a = _run()
    kept = _lib.pool_cached_bytes()
    assert kept > 0
    b = _run(check_reuse=kept)
    assert _lib.pool_cached_bytes() == kept
    _lib.pool_release()
    assert _lib.pool_cached_bytes() == 0
    c = _run()
    for x in (b, c):
        assert np.array_equal(x[0], a[0]) and x[1:] == a[1:]
