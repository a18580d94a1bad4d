"""The drop-in claim on the host side: the reference's own configuration, grid, property backend and
cycle-state objects, handed to this package in place of its own, give the same per-step constants
(the bytes of dv_step_params and the three per-step arrays) for every step of the cycle.  Runs where
a checkout of the reference is importable ($DVTSA_REFERENCE_ROOT, or the default location of this
build's container); skipped elsewhere."""
import os
import sys

import numpy as np
import pytest

from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config
from dac_vtsa_b200.params import build_params, params_bytes

REF = os.environ.get("DVTSA_REFERENCE_ROOT", "/root/reference")
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "core")), reason="reference checkout absent")

OVER = {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6, "jacket.theta_coverage_deg": [0.0, 180.0],
        "feed.profile": "cosine_theta", "feed.profile_amplitude": 0.3, "operation.P_vacuum": 2e4}


def _reference_objects():
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import config.parameters as rp
    from core.grid import Grid
    from core.state import initial_state
    from properties import get_backend
    cfg = rp.load_config(override_dict=OVER)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    return cfg, g, props, initial_state(cfg, g, props)


def test_reference_objects_give_the_same_step_constants():
    """build_params on the reference's cfg / Grid / property backend (as TVSAModel receives them from
    the reference's runner) equals build_params on this package's own objects, step by step."""
    cfg_r, g_r, props_r, st_r = _reference_objects()
    cfg = load_config(override_dict=OVER)
    g = host.Grid.from_config(cfg)
    gas = host.get_backend(cfg)
    # TVSAModel takes a backend without the package's gas tables the way it does here
    gas_r = host.GasData(props_r.species, cfg_r.properties.cp_reference_T)
    P_start = {"top": float(np.mean(st_r.P[:, :, 0])), "bottom": float(np.mean(st_r.P[:, :, -1]))}
    for k, step in enumerate(cfg.cycle):
        T_prev = 300.0 if k else None
        a = build_params(cfg_r, g_r, gas_r, cfg_r.cycle[k], P_start, T_prev)
        b = build_params(cfg, g, gas, step, P_start, T_prev)
        assert params_bytes(a[0]) == params_bytes(b[0]), step["name"]
        for x, y in zip(a[1:4], b[1:4]):
            assert np.array_equal(x, y), step["name"]
