"""Config loader and host-side set-up (no GPU)."""
import math

import numpy as np
import pytest

from dac_vtsa_b200 import host
from dac_vtsa_b200.config import ConfigError, load_config, with_overrides


def test_defaults_and_derived():
    cfg = load_config()
    assert math.isclose(cfg.derived.bulk_density, 880 * 0.6)
    assert math.isclose(cfg.derived.particle_porosity, (0.54 - 0.40) / 0.60)
    assert cfg.cycle[2]["jacket"]["T"] == cfg.operation.T_heat
    assert [s["name"] for s in cfg.cycle] == ["adsorption", "blowdown", "heating", "cooling"]


@pytest.mark.parametrize("key,val", [("geometry.bed_radius", -1.0), ("sorbent.bed_voidage", 1.2),
                                     ("grid.Nr", 0), ("isotherm.coadsorption.model", "magic"),
                                     ("grid.Ntheta", 2), ("solver.scheme", "rk45")])
def test_invalid_values_rejected(key, val):
    with pytest.raises(ConfigError):
        load_config(override_dict={key: val})


def test_unknown_key_rejected():
    with pytest.raises(ConfigError):
        load_config(override_dict={"sorbent.bed_vodage": 0.4})


def test_string_overrides_and_references():
    cfg = load_config(overrides=["operation.T_heat=363.0", "grid.Nz=20"])
    assert cfg.grid.Nz == 20 and cfg.cycle[2]["jacket"]["T"] == 363.0
    cfg2 = with_overrides(cfg, {"operation.T_heat": 380.0})
    assert cfg2.cycle[2]["jacket"]["T"] == 380.0


def test_grid_telescoping_geometry():
    g = host.Grid(R=0.025, L=0.01, Nr=5, Nth=6, Nz=7)
    assert math.isclose(float(np.sum(g.volume_full())), g.bed_volume, rel_tol=1e-13)
    assert math.isclose(float(np.sum(g.Az * np.ones((5, 6)))), g.cross_section, rel_tol=1e-13)
    assert g.coverage_fraction([0.0, 180.0], [0.0, 1.0]).sum() == pytest.approx(3 * 7)


def test_end_conditions_per_step():
    cfg = load_config()
    props = host.get_backend(cfg)
    kinds = [tuple(host.end_conditions(cfg, s, props.species, props)[e].kind for e in ("top", "bottom"))
             for s in cfg.cycle]
    assert kinds == [("feed", "valve"), ("closed", "pump"), ("closed", "pump"), ("closed", "closed")]


def test_seeded_state_constant_pressure():
    cfg = load_config(override_dict={"grid.Nr": 4, "grid.Ntheta": 4, "grid.Nz": 16})
    g = host.Grid.from_config(cfg)
    st = host.seeded_state(cfg, g, host.get_backend(cfg), seed=0)
    assert np.allclose(st.P, 101325.0, rtol=1e-13)
    assert np.all(np.abs(st.T / 288.0 - 1.0) <= 0.01)
