"""Host-side set-up of one cycle step: geometry, gas data, valve boundary conditions, states.

Everything here runs once per cycle step on the host and produces the constants that the
device kernels read (see :mod:`dac_vtsa_b200.params`).  The formulas follow the reference
so that the per-step constants agree with it to the last bit where the arithmetic is the
same:

* cylindrical finite-volume geometry            -- core/grid.py:61-96
* pure-gas data and mixing-rule constants        -- properties/ideal_gas_backend.py:24-45,59-71,140-166
* Fuller binary diffusion constants              -- utils/diffusion.py:15-26
* humid air, end conditions, feed flux / profile -- valves/valve_logic.py:63-148
* cycle state container and initial states       -- core/state.py:23-93
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field
from enum import Enum
from typing import Dict, Optional, Tuple

import numpy as np

R_GAS = 8.314462618                      # properties/ideal_gas_backend.py:24

# Pure-component tables (Young 2021 ESI S6/S7; Incropera A.4), properties/ideal_gas_backend.py:26-45
CP_POLY = {"N2": (1.06569e-5, -6.4057779e-3, 30.1318), "CO2": (-3.23753e-5, 6.17517420e-2, 21.9165),
           "H2O": (1.72619108e-3, -1.22971184026, 250.9868), "O2": (9.08259e-6, 1.00528795e-3, 28.3000)}
MU_LIN = {"N2": (3.96929e-8, 6.15036e-6), "CO2": (4.41697e-8, 1.90440e-6),
          "H2O": (3.55595e-8, -9.930767e-7), "O2": (4.75391e-8, 6.53871e-6)}
K_POW = {"N2": (0.02598, 0.81), "O2": (0.02676, 0.84), "CO2": (0.01655, 1.335), "H2O": (0.0186, 1.18)}
MOLAR_MASS = {"CO2": 0.04401, "H2O": 0.018015, "N2": 0.028960}
AIR_FRAC = (("N2", 0.79), ("O2", 0.21))
# Fuller diffusion volumes and molar masses [g/mol], utils/diffusion.py:15-16
DIFF_VOLUME = {"CO2": 26.7, "H2O": 13.1, "N2": 18.5, "O2": 16.3, "AIR": 19.7, "Ar": 16.2}
MOLAR_MASS_G = {"CO2": 44.01, "H2O": 18.015, "N2": 28.013, "O2": 31.999, "AIR": 28.96, "Ar": 39.948}


def species_for(cfg):
    return ["CO2", "H2O", "N2"] if cfg.components.water else ["CO2", "N2"]


def arden_buck(T):
    """Saturation pressure of water over liquid [Pa] (properties/ideal_gas_backend.py:48-51)."""
    Tc = np.asarray(T, dtype=float) - 273.15
    return 611.21 * np.exp((18.678 - Tc / 234.5) * (Tc / (257.14 + Tc)))


def fuller_const(a: str, b: str) -> float:
    """sqrt(M_ab) (V_a^1/3 + V_b^1/3)^2 of the Fuller correlation (utils/diffusion.py:19-26)."""
    Ma, Mb = MOLAR_MASS_G[a], MOLAR_MASS_G[b]
    Mab = 2.0 / (1.0 / Ma + 1.0 / Mb)
    s = DIFF_VOLUME[a] ** (1 / 3) + DIFF_VOLUME[b] ** (1 / 3)
    return float(np.sqrt(Mab) * s * s)


class GasData:
    """Constant-cp ideal-gas mixture data for the species list (the ``props`` object).

    Exposes the attributes the model reads from the reference backend: ``species``, ``cp``
    (J/mol/K at ``cp_reference_T``), ``M``, and ``p_sat``; plus the per-species linear
    viscosity and power-law conductivity coefficients the kernels evaluate.
    """

    name = "ideal_gas"

    def __init__(self, species, cp_reference_T=330.0):
        self.species = list(species)
        self.ng = len(self.species)
        self.M = np.array([MOLAR_MASS[s] for s in self.species])
        self.cp = np.array([self._cp_pure(s, cp_reference_T) for s in self.species])
        self.i_co2 = self.species.index("CO2")
        self.i_h2o = self.species.index("H2O") if "H2O" in self.species else None
        self.i_inert = self.species.index("N2")
        Mi, Mj = self.M[:, None], self.M[None, :]
        self.wilke_den = np.sqrt(8.0 * (1.0 + Mi / Mj))
        self.mass_q = (Mj / Mi) ** 0.25

    @staticmethod
    def _cp_pure(s, T):
        if s == "N2":
            return sum(f * np.polyval(CP_POLY[c], T) for c, f in AIR_FRAC)
        return float(np.polyval(CP_POLY[s], T))

    def mu_terms(self):
        """Per species a list of (weight, D, E): mu = sum weight*(D T + E) (air = N2/O2 blend)."""
        out = []
        for s in self.species:
            if s == "N2":
                out.append([(f, MU_LIN[c][0], MU_LIN[c][1]) for c, f in AIR_FRAC])
            else:
                out.append([(1.0, MU_LIN[s][0], MU_LIN[s][1])])
        return out

    def k_terms(self):
        """Per species a list of (weight, k300, n): k = sum weight*k300*(T/300)^n."""
        out = []
        for s in self.species:
            if s == "N2":
                out.append([(f, K_POW[c][0], K_POW[c][1]) for c, f in AIR_FRAC])
            else:
                out.append([(1.0, K_POW[s][0], K_POW[s][1])])
        return out

    def p_sat(self, T):
        return arden_buck(T)


def get_backend(cfg, species=None) -> GasData:
    if cfg.properties.backend != "ideal_gas":
        raise NotImplementedError("only the ideal_gas property backend has a GPU implementation")
    return GasData(species or species_for(cfg), cfg.properties.cp_reference_T)


@dataclass
class Grid:
    """Cylindrical (r, theta, z) finite-volume grid; z = 0 is the feed (top) end.

    Same construction as core/grid.py:61-96: per-ring face areas and volumes, so that
    the sum over cells of every flux divergence telescopes to the boundary flows.
    """
    R: float
    L: float
    Nr: int
    Nth: int
    Nz: int
    wall_thickness: float = 0.002
    radial_spacing: str = "uniform"
    r_f: np.ndarray = field(init=False)

    def __post_init__(self):
        Nr, Nth, Nz = self.Nr, self.Nth, self.Nz
        if self.radial_spacing == "equal_area":
            self.r_f = self.R * np.sqrt(np.linspace(0.0, 1.0, Nr + 1))
        else:
            self.r_f = np.linspace(0.0, self.R, Nr + 1)
        self.r_c = 0.5 * (self.r_f[1:] + self.r_f[:-1])
        self.dr = np.diff(self.r_f)
        self.dth = 2.0 * np.pi / Nth
        self.th_f = np.linspace(0.0, 2.0 * np.pi, Nth + 1)
        self.th_c = 0.5 * (self.th_f[1:] + self.th_f[:-1])
        self.dz = self.L / Nz
        self.z_f = np.linspace(0.0, self.L, Nz + 1)
        self.z_c = 0.5 * (self.z_f[1:] + self.z_f[:-1])
        ring = 0.5 * (self.r_f[1:] ** 2 - self.r_f[:-1] ** 2)
        self.Az = (ring * self.dth)[:, None]
        self.V = (ring * self.dth * self.dz)[:, None, None]
        self.Ar = (self.r_f[1:-1] * self.dth * self.dz)[:, None, None]
        self.Ath = (self.dr * self.dz)[:, None, None]
        self.drc = np.diff(self.r_c)[:, None, None]
        self.arc = (self.r_c * self.dth)[:, None, None]
        self.dzc = self.dz
        self.A_wall_in = self.R * self.dth * self.dz
        Ro = self.R + self.wall_thickness
        self.A_wall_out = Ro * self.dth * self.dz
        self.V_wall = 0.5 * (Ro ** 2 - self.R ** 2) * self.dth * self.dz
        self.A_wall_axial = 0.5 * (Ro ** 2 - self.R ** 2) * self.dth
        self.R_wall_mid = self.R + 0.5 * self.wall_thickness
        self.half_dr_outer = self.R - self.r_c[-1]
        self.cross_section = np.pi * self.R ** 2
        self.bed_volume = self.cross_section * self.L
        self.ncell = Nr * Nth * Nz
        self.shape = (Nr, Nth, Nz)
        self.wall_shape = (Nth, Nz)

    @classmethod
    def from_config(cls, cfg) -> "Grid":
        return cls(R=cfg.geometry.bed_radius, L=cfg.geometry.bed_length, Nr=cfg.grid.Nr,
                   Nth=cfg.grid.Ntheta, Nz=cfg.grid.Nz, wall_thickness=cfg.geometry.wall_thickness,
                   radial_spacing=cfg.grid.radial_spacing)

    def volume_full(self) -> np.ndarray:
        return np.broadcast_to(self.V, self.shape)

    def coverage_fraction(self, theta_deg, z_frac) -> np.ndarray:
        """Jacket-covered fraction of each wall cell (Nth, Nz) (core/grid.py:98-104)."""
        t0, t1 = np.radians(theta_deg[0]), np.radians(theta_deg[1])
        z0, z1 = z_frac[0] * self.L, z_frac[1] * self.L
        ov_t = np.clip(np.minimum(self.th_f[1:], t1) - np.maximum(self.th_f[:-1], t0), 0, None) / self.dth
        ov_z = np.clip(np.minimum(self.z_f[1:], z1) - np.maximum(self.z_f[:-1], z0), 0, None) / self.dz
        return ov_t[:, None] * ov_z[None, :]

    def describe(self) -> str:
        return (f"Grid: Nr={self.Nr} Ntheta={self.Nth} Nz={self.Nz} ({self.ncell} cells), "
                f"R={self.R} m, L={self.L} m")


# ------------------------------------------------------------------ valves -> end conditions

class ValveState(str, Enum):
    """Valve states of a cycle step (valves/valve_logic.py:41-45)."""
    CLOSED = "CLOSED"
    OPEN = "OPEN"
    OPEN_ATMOSPHERIC = "OPEN_ATMOSPHERIC"
    OPEN_VACUUM = "OPEN_VACUUM"


@dataclass
class EndCondition:
    """Boundary condition of one column end for one step (valves/valve_logic.py:48-60)."""
    end: str
    valve: Optional[str]
    state: ValveState
    kind: str                      # closed | feed | pump | valve | pressure
    P_target: float = 101325.0
    y_ext: Optional[np.ndarray] = None
    T_ext: float = 298.15
    check_valve: bool = False
    is_product: bool = False
    is_vacuum: bool = False
    is_feed: bool = False
    speed: float = 0.0


def humid_air_composition(species, P, T, RH, y_co2_dry, p_sat):
    """Mole fractions of humid air in species order (valves/valve_logic.py:63-68)."""
    y_w = RH * p_sat / P if "H2O" in species else 0.0
    y = {"H2O": y_w, "CO2": y_co2_dry * (1.0 - y_w)}
    y["N2"] = 1.0 - y["CO2"] - y_w
    return np.array([y[s] for s in species])


def end_conditions(cfg, step: Dict, species, props) -> Dict[str, EndCondition]:
    """Valve states of a step -> condition at the top (z=0) and bottom (z=L) ends
    (valves/valve_logic.py:71-109)."""
    feed, amb = cfg.feed, cfg.ambient
    water = "H2O" in species
    y_feed = humid_air_composition(species, feed.P, feed.T, feed.RH if water else 0.0,
                                   feed.y_co2_dry, float(props.p_sat(feed.T)))
    y_amb = humid_air_composition(species, amb.P, amb.T, amb.RH if water else 0.0,
                                  amb.y_co2_dry, float(props.p_sat(amb.T)))
    ports = cfg.ports
    out = {}
    for end in ("top", "bottom"):
        valve = None
        for v in ("V1", "V2", "V3"):
            if ports[v] == end and step["valves"][v] != "CLOSED":
                valve = v
        if valve is None:
            out[end] = EndCondition(end, None, ValveState.CLOSED, "closed")
            continue
        st = ValveState(step["valves"][valve])
        is_prod = step.get("product_port", "V3") == valve
        if st == ValveState.OPEN:
            out[end] = EndCondition(end, valve, st, "feed", feed.P, y_feed, feed.T, is_feed=True)
        elif st == ValveState.OPEN_ATMOSPHERIC:
            kind = "valve" if cfg.operation.vent_model == "valve" else "pressure"
            kv = cfg.operation.vent_conductance
            if valve == "V1":
                out[end] = EndCondition(end, valve, st, kind, feed.P, y_feed, feed.T,
                                        is_product=is_prod, is_feed=True, speed=kv)
            else:
                out[end] = EndCondition(end, valve, st, kind, amb.P, y_amb, amb.T, is_product=is_prod, speed=kv)
        else:
            kind = "pump" if cfg.operation.vacuum_model == "pump" else "pressure"
            out[end] = EndCondition(end, valve, st, kind, cfg.operation.P_vacuum, y_amb, amb.T,
                                    check_valve=bool(cfg.operation.vacuum_check_valve),
                                    is_product=is_prod, is_vacuum=True, speed=cfg.operation.pump_speed_per_area)
    return out


def feed_molar_flux(cfg) -> float:
    """Feed molar flux per unit cross-section [mol/m2/s] (valves/valve_logic.py:112-114)."""
    return cfg.feed.velocity * cfg.feed.P / (R_GAS * cfg.feed.T)


def feed_profile(cfg, grid: Grid) -> np.ndarray:
    """Inlet distribution (Nr, Nth) with area-weighted mean 1 (valves/valve_logic.py:117-148)."""
    prof = cfg.feed.profile
    A = cfg.feed.profile_amplitude
    rr, th = np.meshgrid(grid.r_c, grid.th_c, indexing="ij")
    if prof == "uniform":
        f = np.ones_like(rr)
    elif prof == "cosine_theta":
        f = 1.0 + A * np.cos(th - np.radians(cfg.feed.profile_theta0_deg))
    elif prof == "linear_r":
        f = 1.0 + A * (2.0 * rr / grid.R - 1.0)
    elif prof == "central_disc":
        r_in = cfg.feed.profile_radius_fraction * grid.R
        lo, hi = grid.r_f[:-1], grid.r_f[1:]
        frac = np.clip((np.minimum(hi, r_in) ** 2 - lo ** 2) / (hi ** 2 - lo ** 2), 0.0, 1.0)
        f = np.repeat(frac[:, None], grid.Nth, axis=1)
    elif prof == "sector":
        half = 0.5 * np.radians(cfg.feed.profile_sector_deg)
        t0 = np.radians(cfg.feed.profile_theta0_deg)
        lo, hi = grid.th_f[:-1] - t0, grid.th_f[1:] - t0
        ov = np.zeros(grid.Nth)
        for sh in (-2 * np.pi, 0.0, 2 * np.pi):
            ov += np.clip(np.minimum(hi + sh, half) - np.maximum(lo + sh, -half), 0.0, None)
        f = np.repeat((ov / grid.dth)[None, :], grid.Nr, axis=0)
    else:
        raise ValueError(prof)
    w = grid.Az * np.ones_like(f)
    return f * w.sum() / (f * w).sum()


# ------------------------------------------------------------------ state

@dataclass
class CycleState:
    """Bed state handed from step to step (core/state.py:23-58): c (ng,Nr,Nth,Nz) mol/m3,
    q (na,...) mol/kg, T (Nr,Nth,Nz) K, Tw (Nth,Nz) K."""
    c: np.ndarray
    q: np.ndarray
    T: np.ndarray
    Tw: np.ndarray
    t: float = 0.0
    cycle: int = 1
    step: str = "initial"
    species: Tuple[str, ...] = ("CO2", "H2O", "N2")
    adsorbed: Tuple[str, ...] = ("CO2", "H2O")
    meta: Dict = field(default_factory=dict)

    @property
    def P(self) -> np.ndarray:
        return self.c.sum(axis=0) * R_GAS * self.T

    @property
    def y(self) -> np.ndarray:
        return self.c / np.maximum(self.c.sum(axis=0), 1e-30)

    def copy(self) -> "CycleState":
        return copy.deepcopy(self)


def initial_state(cfg, grid: Grid, props) -> CycleState:
    """Clean bed (q = 0) in feed air at feed T, P (core/state.py:62-93, modes clean / csv)."""
    species = tuple(props.species)
    adsorbed = ("CO2", "H2O") if cfg.components.water else ("CO2",)
    if cfg.run.initial_state == "csv":
        raise NotImplementedError("state CSV hand-off is host I/O outside the stepping path")
    T0, P0 = cfg.feed.T, cfg.feed.P
    y = humid_air_composition(species, P0, T0, cfg.feed.RH if cfg.components.water else 0.0,
                              cfg.feed.y_co2_dry, float(props.p_sat(T0)))
    C = P0 / (R_GAS * T0)
    c = np.empty((len(species),) + grid.shape)
    for k in range(len(species)):
        c[k] = C * y[k]
    T = np.full(grid.shape, T0)
    q = np.zeros((len(adsorbed),) + grid.shape)
    if cfg.run.initial_state == "feed_equilibrium":
        raise NotImplementedError("feed_equilibrium initial state is not on the stepping path")
    Tw = np.full(grid.wall_shape, T0)
    return CycleState(c=c, q=q, T=T, Tw=Tw, species=species, adsorbed=adsorbed)


def seeded_state(cfg, grid: Grid, props, seed: int = 0, amplitude: float = 0.01,
                 T_base: float = 288.0, P: float = 101325.0) -> CycleState:
    """Benchmark initial state: clean bed, T = T_base (1 + a (2U - 1)) with
    ``numpy.random.default_rng(seed)`` over (Nr, Nth, Nz) in C order, gas at constant
    pressure P (c = y_feed P / (R T) per cell), wall at T_base."""
    st = initial_state(cfg, grid, props)
    rng = np.random.default_rng(seed)
    T = T_base * (1.0 + amplitude * (2.0 * rng.random(grid.shape) - 1.0))
    y = st.c / st.c.sum(axis=0)
    st.c = y * (P / (R_GAS * T))[None]
    st.T = T
    st.Tw = np.full(grid.wall_shape, T_base)
    return st
