"""Run configuration for the implicit stepping path.

The GPU model and integrator read parameters through attribute paths
(``cfg.sorbent.bed_voidage``, ``cfg.solver.rtol`` ...).  Those paths, their
default values and the cycle-step description follow the reference's
parameter file (config/defaults.yaml, validated by config/schema.py:529-571),
so a reference ``Config`` object and the one built here are interchangeable
inputs of :class:`dac_vtsa_b200.model.TVSAModel`.

Only the keys the stepping path reads are kept, plus the run/cycle keys a
driver needs.  ``load_config`` mirrors the reference loader signature
(config/parameters.py:25-28): defaults, then an optional YAML file, then
``override_dict`` and ``key=value`` overrides, then validation and the
derived quantities of config/schema.py:562-571.
"""
from __future__ import annotations

import copy
import math
from typing import Any, Dict, Optional, Sequence


class ConfigError(ValueError):
    """Invalid or unknown configuration entry (same role as the reference's ConfigError)."""


# Parameter values of the reference's config/defaults.yaml:18-241 (numbers only).
_DEFAULTS: Dict[str, Any] = {
    "run": {"name": "default_3d", "results_dir": "results", "max_cycles": 12, "min_cycles": 2,
            "css_tolerance": 1.0e-3, "css_mb_tolerance": 5.0e-3, "handoff_via_csv": True,
            "snapshots_per_step": 12, "write_fields_every_cycle": False, "initial_state": "clean",
            "initial_state_csv": None, "make_plots": True},
    "components": {"water": True},
    "geometry": {"bed_length": 0.01, "bed_radius": 0.025, "wall_thickness": 0.002},
    "grid": {"Nr": 8, "Ntheta": 8, "Nz": 12, "radial_spacing": "uniform"},
    "sorbent": {"name": "Lewatit VP OC 1065", "particle_diameter": 5.2e-4, "particle_density": 880.0,
                "bed_voidage": 0.40, "total_voidage": 0.54, "cp_solid": 1580.0,
                "particle_conductivity": 0.16, "max_temperature": 393.15},
    "isotherm": {
        "co2": {"q_inf0": 4.86, "chi": 0.0, "b0": 2.85e-21, "dH0": -117798.0, "tau0": 0.209,
                "alpha": 0.523, "T0": 298.15, "p_regularization": 0.01},
        "h2o": {"q_m": 3.63, "C": 47110.0, "D": 0.023744, "F": 57706.0, "G": -47.814,
                "E10_slope": -44.38, "E10_intercept": 57220.0, "rh_cap": 0.97},
        "coadsorption": {
            "model": "wadst", "water_loading_basis": "state",
            "wadst": {"b0_wet": 1.230e-18, "q_inf0_wet": 9.035, "tau0_wet": 0.053, "chi_wet": 0.0,
                      "alpha_wet": 0.053, "dH_wet": -203687.0, "A": 1.532},
            "mechanistic": {"f_blocked_max": 0.433, "k": 0.795, "phi_dry": 1.0, "A": 1.535,
                            "dH_wet": -130155.0, "n": 1.425},
            "stampi_bombelli": {"gamma": -0.137, "beta": 5.612},
        },
    },
    "kinetics": {"k_ldf_co2": 0.003, "k_ldf_h2o": 0.0086, "Ea_co2": 0.0, "Ea_h2o": 0.0, "T_ref": 298.15},
    "thermo": {"dH_ads_co2": -70000.0, "dH_ads_h2o": -46000.0, "cp_ads_co2": 37.1, "cp_ads_h2o": 75.3,
               "T_ref": 298.15},
    "properties": {"backend": "ideal_gas", "cp_reference_T": 330.0},
    "transport": {"dispersion_model": "edwards_richardson", "er_gamma1": 0.73, "er_gamma2": 0.5,
                  "er_beta": 13.0, "Pe_mass_radial_inf": 10.0, "Pe_heat_radial_inf": 10.0,
                  "Pe_heat_axial_inf": 2.0, "bed_conductivity_model": "zehner_schlunder",
                  "bed_conductivity_constant": 0.12, "zs_shape_factor": 1.25,
                  "wall_htc_model": "martin_nilles", "wall_htc_constant": 300.0, "ergun_A": 150.0,
                  "ergun_B": 1.75, "heat_transfer_mode": "resolved", "lumped_U": 14.0},
    "wall": {"enabled": True, "density": 7800.0, "cp": 513.0, "conductivity": 16.0},
    "jacket": {"h_jacket": 26.0, "theta_coverage_deg": [0.0, 360.0], "z_coverage": [0.0, 1.0],
               "h_ambient": 5.0, "ramp_time": 0.0},
    "internal_hx": {"enabled": False, "hA_per_volume": 2000.0, "follows_jacket": True},
    "feed": {"T": 288.15, "P": 101325.0, "RH": 0.55, "y_co2_dry": 4.0e-4, "velocity": 0.0706,
             "profile": "uniform", "profile_amplitude": 0.0, "profile_theta0_deg": 0.0,
             "profile_radius_fraction": 0.5, "profile_sector_deg": 90.0},
    "ambient": {"T": 288.15, "P": 101325.0, "RH": 0.55, "y_co2_dry": 4.0e-4},
    "operation": {"P_vacuum": 2.0e4, "T_heat": 373.15, "T_cool": 288.15, "T_adsorption_jacket": 288.15,
                  "vent_model": "valve", "vent_conductance": 500.0, "valve_time_constant": 5.0,
                  "vacuum_model": "pump", "pump_speed_per_area": 5.0e-3, "vacuum_check_valve": True},
    "ports": {"V1": "top", "V2": "bottom", "V3": "bottom"},
    "cycle": [
        {"name": "adsorption", "type": "adsorption", "duration": 8000.0,
         "valves": {"V1": "OPEN", "V2": "OPEN_ATMOSPHERIC", "V3": "CLOSED"},
         "jacket": {"mode": "temperature", "T": "operation.T_adsorption_jacket"}},
        {"name": "blowdown", "type": "blowdown", "duration": 60.0,
         "valves": {"V1": "CLOSED", "V2": "OPEN_VACUUM", "V3": "CLOSED"},
         "jacket": {"mode": "temperature", "T": "operation.T_adsorption_jacket"}},
        {"name": "heating", "type": "heating", "duration": 22400.0,
         "valves": {"V1": "CLOSED", "V2": "CLOSED", "V3": "OPEN_VACUUM"},
         "jacket": {"mode": "temperature", "T": "operation.T_heat"}},
        {"name": "cooling", "type": "cooling", "duration": 400.0,
         "valves": {"V1": "CLOSED", "V2": "CLOSED", "V3": "CLOSED"},
         "jacket": {"mode": "temperature", "T": "operation.T_cool"}},
    ],
    "energy": {"eta_vacuum": 0.7, "vacuum_efficiency_model": "constant", "eta_blower": 0.5,
               "gamma_gas": 1.4, "pump_handles_water": False, "eta_turbine": 0.75, "T_low_equiv": 288.15},
    "solver": {"method": "trbdf2", "scheme": "sdirk2", "rtol": 1.0e-4, "atol_c_co2": 1.0e-6,
               "atol_c_h2o": 1.0e-5, "atol_c_inert": 1.0e-4, "atol_q": 1.0e-6, "atol_T": 1.0e-3,
               "h_initial": 1.0e-4, "h_max_fraction": 0.02, "max_newton_iter": 7, "newton_mode": "krylov",
               "preconditioner": "theta_block", "precond_theta_rings": 3, "refactor_ratio": 3.0,
               "gmres_refresh": 20, "newton_kappa": 0.01, "conservation_tol": 1.0e-3,
               "jacobian_max_age": 40, "limiter": "van_albada", "max_steps_per_step": 200000,
               "outlet_record_every": 1},
    # GPU-only knobs live in their own namespace so reference configs stay valid.
    "gpu": {"krylov_precision": "fp64", "predictor": "extrapolation", "predictor_weights": "", "max_polish": 2,
            "polish_cycles": 1, "balance_projection": False},
}

# Choices checked by validate(); everything else is type-checked against the default.
_CHOICES = {
    "grid.radial_spacing": ("uniform", "equal_area"),
    "isotherm.coadsorption.model": ("none", "wadst", "mechanistic", "stampi_bombelli"),
    "isotherm.coadsorption.water_loading_basis": ("state", "equilibrium"),
    "transport.dispersion_model": ("edwards_richardson", "young2021", "wakao_kagei"),
    "transport.bed_conductivity_model": ("zehner_schlunder", "parallel", "constant"),
    "transport.wall_htc_model": ("martin_nilles", "constant"),
    "transport.heat_transfer_mode": ("resolved", "lumped"),
    "feed.profile": ("uniform", "cosine_theta", "linear_r", "central_disc", "sector"),
    "operation.vent_model": ("valve", "ramp"),
    "operation.vacuum_model": ("pump", "ramp"),
    "energy.vacuum_efficiency_model": ("constant", "krishnamurthy"),
    "solver.scheme": ("sdirk2", "trbdf2"),
    "solver.newton_mode": ("krylov", "hybrid", "modified"),
    "solver.preconditioner": ("theta_block", "full"),
    "solver.limiter": ("van_albada", "van_albada_tvd", "van_leer", "minmod", "upwind"),
    "gpu.krylov_precision": ("fp64", "fp32", "fp32_factors"),
    "gpu.predictor": ("extrapolation", "learned"),
}
_POSITIVE = ("geometry.bed_length", "geometry.bed_radius", "grid.Nr", "grid.Ntheta", "grid.Nz",
             "sorbent.particle_diameter", "sorbent.particle_density")
_VALVES = ("V1", "V2", "V3")
_VALVE_STATES = ("CLOSED", "OPEN", "OPEN_ATMOSPHERIC", "OPEN_VACUUM")
_STEP_TYPES = ("adsorption", "blowdown", "heating", "cooling", "pressurization")


class Config:
    """Read-only attribute view of a nested parameter dictionary."""

    def __init__(self, data: Dict[str, Any]):
        object.__setattr__(self, "_data", data)

    def __getattr__(self, name):
        try:
            v = self._data[name]
        except KeyError:
            raise AttributeError(name) from None
        return Config(v) if isinstance(v, dict) else v

    def __setattr__(self, key, value):
        raise AttributeError("Config is read-only; use with_overrides()")

    def __getitem__(self, name):
        return self.__getattr__(name)

    def get(self, dotted: str, default=None):
        node: Any = self._data
        for part in dotted.split("."):
            if not isinstance(node, dict) or part not in node:
                return default
            node = node[part]
        return node

    def to_dict(self) -> Dict[str, Any]:
        return copy.deepcopy(self._data)

    def __repr__(self):
        return f"Config({list(self._data)})"


def _set_dotted(d: Dict, dotted: str, value: Any) -> None:
    parts = dotted.split(".")
    node = d
    for p in parts[:-1]:
        if p not in node or not isinstance(node[p], dict):
            raise ConfigError(f"unknown configuration key: {dotted}")
        node = node[p]
    if parts[-1] not in node:
        raise ConfigError(f"unknown configuration key: {dotted}")
    node[parts[-1]] = value


def _get_dotted(d: Dict, dotted: str):
    node = d
    for p in dotted.split("."):
        node = node[p]
    return node


def _flatten(d: Dict, prefix: str = "") -> Dict[str, Any]:
    out = {}
    for k, v in d.items():
        key = f"{prefix}{k}"
        if isinstance(v, dict) and not key.endswith(("theta_coverage_deg", "z_coverage")):
            out.update(_flatten(v, key + "."))
        else:
            out[key] = v
    return out


def _parse_value(text: str) -> Any:
    import yaml
    return yaml.safe_load(text)


def _check(key: str, value: Any, default: Any) -> Any:
    if key in _CHOICES:
        if value not in _CHOICES[key]:
            raise ConfigError(f"{key} = {value!r} not in {_CHOICES[key]}")
        return value
    if isinstance(default, bool):
        if not isinstance(value, bool):
            raise ConfigError(f"{key} must be a bool")
        return value
    if isinstance(default, (int, float)) and isinstance(value, str):
        # YAML 1.1 (PyYAML) reads e.g. 2.0e4 as a string: numeric strings count as numbers, as in the
        # reference's schema (config/schema.py:386-391)
        try:
            value = float(value)
        except ValueError:
            raise ConfigError(f"{key}: expected a number, got {value!r}") from None
    if isinstance(default, int) and not isinstance(default, bool):
        if isinstance(value, bool) or not isinstance(value, (int, float)) or int(value) != value:
            raise ConfigError(f"{key} must be an integer")
        value = int(value)
    elif isinstance(default, float):
        if isinstance(value, bool) or not isinstance(value, (int, float)) or not math.isfinite(value):
            raise ConfigError(f"{key} must be a finite number")
        value = float(value)
    if key in _POSITIVE and value <= 0:
        raise ConfigError(f"{key} must be > 0")
    return value


def _resolve(raw: Dict, value: Any) -> Any:
    if isinstance(value, str):
        try:                                   # a numeric string (YAML 1.1 reads 2.0e4 as one) is a number
            return float(value)
        except ValueError:
            pass
    if isinstance(value, str) and "." in value:
        try:
            return float(_get_dotted(raw, value))
        except (KeyError, TypeError, ValueError):
            raise ConfigError(f"cannot resolve reference {value!r}") from None
    return value


def _validate_cycle(raw: Dict):
    steps = raw.get("cycle")
    if not isinstance(steps, list) or not steps:
        raise ConfigError("cycle: must be a non-empty list of steps")
    out, names = [], set()
    for i, st in enumerate(steps):
        st = copy.deepcopy(st)
        name = st.get("name") or st.get("type")
        if name in names:
            raise ConfigError(f"cycle: duplicate step name {name!r}")
        names.add(name)
        st["name"] = name
        if st.get("type") not in _STEP_TYPES:
            raise ConfigError(f"cycle[{i}].type must be one of {_STEP_TYPES}")
        dur = _resolve(raw, st.get("duration"))
        if not isinstance(dur, (int, float)) or dur <= 0:
            raise ConfigError(f"cycle[{i}].duration must be > 0 s")
        st["duration"] = float(dur)
        valves = st.get("valves") or {}
        vv = {}
        for v in _VALVES:
            s = valves.get(v, "CLOSED")
            if s not in _VALVE_STATES:
                raise ConfigError(f"cycle[{i}].valves.{v} = {s!r} not in {_VALVE_STATES}")
            vv[v] = s
        st["valves"] = vv
        jk = st.get("jacket") or {"mode": "adiabatic"}
        mode = jk.get("mode", "temperature")
        if mode not in ("temperature", "adiabatic"):
            raise ConfigError(f"cycle[{i}].jacket.mode must be temperature|adiabatic")
        jout = {"mode": mode}
        if mode == "temperature":
            src = jk.get("T_source", jk.get("T"))
            T = _resolve(raw, src)
            if not isinstance(T, (int, float)) or not (150 < T < 900):
                raise ConfigError(f"cycle[{i}].jacket.T invalid ({T!r})")
            jout["T"] = float(T)
            if isinstance(src, str):
                jout["T_source"] = src
        st["jacket"] = jout
        stop = st.get("stop_on")
        if stop is not None:
            crit = stop.get("criterion")
            if crit not in ("outlet_ratio", "end_saturation", "min_temperature", "max_temperature"):
                raise ConfigError(f"cycle[{i}].stop_on.criterion invalid: {crit!r}")
            stop = {"criterion": crit, "value": float(_resolve(raw, stop.get("value_source", stop.get("value"))))}
        st["stop_on"] = stop
        pp = st.get("product_port") or "V3"
        if pp not in _VALVES + ("none",):
            raise ConfigError(f"cycle[{i}].product_port must be V1/V2/V3/none")
        st["product_port"] = pp
        open_by_end = {"top": [], "bottom": []}
        for v, s in vv.items():
            if s != "CLOSED":
                open_by_end[raw["ports"][v]].append(v)
            if s == "OPEN" and v != "V1":
                raise ConfigError(f"step {name!r}: OPEN (feed blower) is only valid for V1")
        for end, lst in open_by_end.items():
            if len(lst) > 1:
                raise ConfigError(f"step {name!r}: valves {lst} are open at the same end ({end})")
        out.append(st)
    return out


def validate(raw: Dict[str, Any]) -> Config:
    raw = copy.deepcopy(raw)
    raw.pop("derived", None)
    flat = _flatten({k: v for k, v in raw.items() if k != "cycle"})
    ref = _flatten({k: v for k, v in _DEFAULTS.items() if k != "cycle"})
    unknown = [k for k in flat if k not in ref]
    if unknown:
        raise ConfigError(f"unknown configuration keys (typo?): {unknown}")
    for key, dv in ref.items():
        try:
            v = _get_dotted(raw, key)
        except (KeyError, TypeError):
            raise ConfigError(f"missing configuration key: {key}") from None
        if dv is None or isinstance(dv, (list, str)) and key not in _CHOICES:
            continue
        _set_dotted(raw, key, _check(key, v, dv))
    s = raw["sorbent"]
    if not (0.0 < s["bed_voidage"] < 1.0) or not (s["bed_voidage"] <= s["total_voidage"] < 1.0):
        raise ConfigError("sorbent voidages must satisfy 0 < bed_voidage <= total_voidage < 1")
    if raw["grid"]["Ntheta"] == 2:
        raise ConfigError("grid.Ntheta = 2 is degenerate; use 1 (axisymmetric) or >= 3")
    if raw["operation"]["P_vacuum"] >= raw["ambient"]["P"]:
        raise ConfigError("operation.P_vacuum must be below ambient.P")
    th, zc = raw["jacket"]["theta_coverage_deg"], raw["jacket"]["z_coverage"]
    if len(th) != 2 or not (0 <= th[0] < th[1] <= 360):
        raise ConfigError("jacket.theta_coverage_deg must be [start, end] within [0, 360]")
    if len(zc) != 2 or not (0 <= zc[0] < zc[1] <= 1):
        raise ConfigError("jacket.z_coverage must be [start, end] within [0, 1]")
    raw["cycle"] = _validate_cycle(raw)
    eb, et = s["bed_voidage"], s["total_voidage"]
    R, L = raw["geometry"]["bed_radius"], raw["geometry"]["bed_length"]
    raw["derived"] = {"particle_porosity": (et - eb) / (1.0 - eb),
                      "bulk_density": s["particle_density"] * (1.0 - eb),
                      "bed_volume": math.pi * R ** 2 * L, "cross_section": math.pi * R ** 2}
    raw["derived"]["sorbent_mass"] = raw["derived"]["bulk_density"] * raw["derived"]["bed_volume"]
    return Config(raw)


def load_config(user_yaml: Optional[str] = None, overrides: Optional[Sequence[str]] = None,
                override_dict: Optional[Dict[str, Any]] = None) -> Config:
    """Defaults + optional YAML + overrides, validated (reference: config/parameters.py:25-28)."""
    raw = copy.deepcopy(_DEFAULTS)
    if user_yaml:
        import yaml
        with open(user_yaml) as fh:
            user = yaml.safe_load(fh) or {}
        user.pop("derived", None)
        if "cycle" in user:
            raw["cycle"] = user.pop("cycle")
        _deep_merge(raw, user)
    for k, v in (override_dict or {}).items():
        _set_dotted(raw, k, v)
    for ov in overrides or []:
        if "=" not in ov:
            raise ConfigError(f"override must be key=value: {ov!r}")
        k, v = ov.split("=", 1)
        _set_dotted(raw, k.strip(), _parse_value(v.strip()))
    return validate(raw)


def with_overrides(cfg, override_dict: Dict[str, Any]) -> Config:
    raw = cfg.to_dict()
    raw.pop("derived", None)
    for k, v in override_dict.items():
        _set_dotted(raw, k, v)
    return validate(raw)


def _deep_merge(base: Dict, upd: Dict) -> None:
    for k, v in upd.items():
        if isinstance(v, dict) and isinstance(base.get(k), dict):
            _deep_merge(base[k], v)
        else:
            base[k] = copy.deepcopy(v)


def gpu_option(cfg, key: str, default):
    """GPU-only knob (``gpu.<key>``); reference configs have no such namespace -> default."""
    try:
        return getattr(cfg.gpu, key)
    except AttributeError:
        return default
