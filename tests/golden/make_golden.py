"""Generate the golden fixtures of the stepping path by running the reference itself.

Run once in a container where the reference is importable:

    python tests/golden/make_golden.py <path of the reference checkout> [--outlet | --cycle ...]

Writes (all small, committed):
  rhs_cases.npz          f(t, y) and the 36 accumulator rates of TVSAModel.rhs for seeded,
                         non-trivial states: every step type, every end-condition kind,
                         alternative closures (core/residual.py:211-417)
  colouring.npz          greedy colouring (numerics/sparsity.py:88-107): full arrays for small
                         grids, sha256 + colour count for the benchmark and ensemble grids
  jacobian_3x4x6.npz     coloured FD Jacobian values (core/jacobian.py:71-86)
  outlet_cases.npz       (--outlet) the reference's diagnostics at seeded states of every cycle
                         step and the outlet record its runner builds from them
                         (steps/_runner.py:50-84,104-121)
  trajectory_c0.npz      TR-BDF2 integration of a 4x4x16 bed: 200 s adsorption from the seeded
                         constant-pressure state, then 10 s blowdown and 100 s heating; accepted
                         step sequence, end states, accumulators and solver counters
                         (core/solver.py:370-511)
  state_csv/seeded_3x4x6*  (--csv) a seeded state written by the reference's save_state_csv
                         (the 17-digit hand-off format, simio/checkpoint.py:27-53)
  newton_modes_4x4x16.npz (--modes) 200 s adsorption with newton_mode hybrid and modified
  stop_young2021.npz     (--stop) the young2021 1-D case's adsorption step, stopped by its
                         end_saturation criterion (core/residual.py:445-482, core/solver.py:
                         476-494): stop time, stop value, end state
  css_3x4x6.npz          (--css) the reference's cyclic-steady-state measures
                         (validation/cyclic_steady_state.py:22-44) between two seeded 3x4x6 states,
                         and its step flows / cycle CO2 balance (postprocessing/reporting.py:30-41)
                         of the 8x8x32 cycle golden's steps
  cycle_8x8x32[_rtolX].npz  (--cycle [--rtol X]) one full adsorption -> blowdown -> heating ->
                         cooling cycle of the 8x8x32 bed through the reference's own step runner
                         (steps/_runner.py:87-188, states handed over in memory as vtsa_cycle.py:
                         72-90 does with the bit-exact CSV hand-off): per step the end state, the
                         accepted step times, accumulators, inventories and solver counters, and
                         the balance rows of validation/conservation_checks.py:29-67
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.jacobian import FDJacobian
    from core.residual import TVSAModel
    from core.solver import TRBDF2
    from core.state import initial_state
    from numerics.sparsity import build_pattern, color_columns
    from properties import R_GAS, get_backend

    def seeded(cfg, grid, props, seed=0):
        st = initial_state(cfg, grid, props)
        rng = np.random.default_rng(seed)
        T = 288.0 * (1.0 + 0.01 * (2.0 * rng.random(grid.shape) - 1.0))
        y = st.c / st.c.sum(axis=0)
        st.c = y * (101325.0 / (R_GAS * T))[None]
        st.T = T
        st.Tw = np.full(grid.wall_shape, 288.0)
        return st

    # ------------------------------------------------------------ rhs cases
    base = {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6, "jacket.theta_coverage_deg": [0.0, 180.0],
            "feed.profile": "cosine_theta", "feed.profile_amplitude": 0.3}
    cases = []
    for s in range(4):
        cases.append((f"step{s}", base, s))
    cases += [
        ("ramp_ports_ads", {**base, "operation.vent_model": "ramp", "operation.vacuum_model": "ramp"}, 0),
        ("ramp_ports_blow", {**base, "operation.vent_model": "ramp", "operation.vacuum_model": "ramp",
                             "operation.vacuum_check_valve": False}, 1),
        ("pump_no_check", {**base, "operation.vacuum_check_valve": False}, 2),
        ("mech_hx_jacket_ramp", {**base, "isotherm.coadsorption.model": "mechanistic",
                                 "internal_hx.enabled": True, "jacket.ramp_time": 50.0}, 2),
        ("no_wall", {**base, "wall.enabled": False}, 0),
        ("no_wall_lumped", {**base, "wall.enabled": False, "transport.heat_transfer_mode": "lumped"}, 2),
        ("sb_wk_krish", {**base, "isotherm.coadsorption.model": "stampi_bombelli",
                         "transport.dispersion_model": "wakao_kagei",
                         "energy.vacuum_efficiency_model": "krishnamurthy"}, 2),
        ("minmod_parallel_const", {**base, "solver.limiter": "minmod",
                                   "transport.bed_conductivity_model": "parallel",
                                   "transport.wall_htc_model": "constant"}, 0),
        ("vanleer_young_none", {**base, "solver.limiter": "van_leer", "transport.dispersion_model": "young2021",
                                "isotherm.coadsorption.model": "none", "feed.profile": "linear_r"}, 0),
        ("tvd_equilibrium_basis", {**base, "solver.limiter": "van_albada_tvd",
                                   "isotherm.coadsorption.water_loading_basis": "equilibrium",
                                   "feed.profile": "sector"}, 0),
        ("upwind_disc_pump_water", {**base, "solver.limiter": "upwind", "feed.profile": "central_disc",
                                    "energy.pump_handles_water": True, "wall.enabled": False}, 1),
        ("axisym_2x1x4", {"grid.Nr": 2, "grid.Ntheta": 1, "grid.Nz": 4}, 1),
        ("line_1x1x30", {"grid.Nr": 1, "grid.Ntheta": 1, "grid.Nz": 30}, 0),
        ("equal_area_4x3x5", {"grid.Nr": 4, "grid.Ntheta": 3, "grid.Nz": 5, "grid.radial_spacing": "equal_area",
                              "jacket.z_coverage": [0.2, 0.7]}, 3),
        ("nz2_3x4x2", {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 2}, 0),
    ]
    rhs = {}
    meta = []
    for i, (name, over, step_i) in enumerate(cases):
        cfg = rp.load_config(override_dict=over)
        g = Grid.from_config(cfg)
        props = get_backend(cfg)
        st = initial_state(cfg, g, props)
        rng = np.random.default_rng(100 + i)
        st.T = st.T + 5.0 * rng.random(st.T.shape)
        st.q = st.q + 0.5 * rng.random(st.q.shape)
        st.c = st.c * (1.0 + 0.05 * rng.random(st.c.shape))
        st.Tw = st.Tw + 3.0 * rng.random(st.Tw.shape)
        m = TVSAModel(cfg, g, props, cfg.cycle[step_i], st, T_jacket_prev=300.0 if "ramp" in name else None)
        y = m.pack(st)
        t = 3.0
        f, acc = m.rhs(t, y)
        d = m.rhs(t, y, diag=True)
        rhs[f"{name}__y"] = y
        rhs[f"{name}__f"] = f
        rhs[f"{name}__acc"] = acc
        rhs[f"{name}__T"] = d["T"]
        rhs[f"{name}__P"] = d["P"]
        rhs[f"{name}__P0"] = st.P
        meta.append({"name": name, "over": over, "step": step_i, "t": t,
                     "T_jacket_prev": 300.0 if "ramp" in name else None})
    rhs["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "rhs_cases.npz"), **rhs)

    # ------------------------------------------------------------ colouring
    col = {}
    small = [(3, 4, 6), (4, 4, 16), (2, 1, 4), (1, 1, 30), (8, 8, 12), (3, 1, 8), (4, 3, 5)]
    for d in small:
        c = color_columns(build_pattern(*d, 3, 2, True))
        col["full_%dx%dx%d" % d] = c.astype(np.uint8)
    big = [(8, 8, 32), (16, 16, 64)] + [(a, b, c) for a in (4, 8, 16) for b in (4, 8, 16) for c in (16, 32, 64)]
    hashes = {}
    for d in sorted(set(big)):
        c = color_columns(build_pattern(*d, 3, 2, True)).astype(np.int64)
        hashes["%dx%dx%d" % d] = [hashlib.sha256(c.tobytes()).hexdigest(), int(c.max()) + 1]
    col["hashes"] = np.array(json.dumps(hashes))
    np.savez_compressed(os.path.join(HERE, "colouring.npz"), **col)

    # ------------------------------------------------------------ jacobian
    cfg = rp.load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = initial_state(cfg, g, props)
    st.T = st.T + np.random.default_rng(0).random(st.T.shape)
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    y = m.pack(st)
    J = FDJacobian(m)(5.0, y)
    np.savez_compressed(os.path.join(HERE, "jacobian_3x4x6.npz"), y=y, t=5.0, data=J.data, indices=J.indices,
                        indptr=J.indptr, P0=st.P)

    # ------------------------------------------------------------ trajectory (4x4x16)
    over = {"grid.Nr": 4, "grid.Ntheta": 4, "grid.Nz": 16, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}
    cfg = rp.load_config(override_dict=over)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = seeded(cfg, g, props)
    out = {"over": np.array(json.dumps(over))}
    T_jac_prev = None
    for k, (si, dur) in enumerate(((0, 200.0), (1, 10.0), (2, 100.0))):
        step = dict(cfg.cycle[si])
        step["duration"] = dur
        m = TVSAModel(cfg, g, props, step, st, T_jac_prev)
        y0 = m.pack(st)
        integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
        hs = []
        res = integ.integrate(y0, dur, np.linspace(0.0, dur, 12), on_step=lambda t, y, a: hs.append(t))
        out[f"s{k}_y0"] = y0
        out[f"s{k}_P0"] = st.P
        out[f"s{k}_y"] = res.y
        out[f"s{k}_acc"] = res.acc
        out[f"s{k}_t_accepted"] = np.array(hs)
        out[f"s{k}_stats"] = np.array([res.n_steps, res.n_reject, res.n_newton_fail, res.n_jac, res.n_lu,
                                       res.nfev, integ.stats["gmres_iters"]])
        out[f"s{k}_snap_t"] = np.array([s[0] for s in res.snapshots])
        out[f"s{k}_snap_y"] = np.array([s[1] for s in res.snapshots])
        out[f"s{k}_meta"] = np.array(json.dumps({"step": si, "duration": dur, "T_jacket_prev": T_jac_prev}))
        st = m.to_state(res.y, st, st.t + res.t, step["name"])
        T_jac_prev = m.T_jacket(res.t) if m.jacket_on else T_jac_prev
    np.savez_compressed(os.path.join(HERE, "trajectory_c0.npz"), **out)
    print("golden fixtures written to", HERE)




def make_bench_state(ref_root, t_mid=4000.0):
    """Reference state of the 8x8x32 benchmark bed after t_mid seconds of adsorption from the seeded
    constant-pressure initial state (input of the CPU throughput sample in bench.py)."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.residual import TVSAModel
    from core.solver import TRBDF2
    from core.state import initial_state
    from properties import R_GAS, get_backend
    over = {"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}
    cfg = rp.load_config(override_dict=over)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = initial_state(cfg, g, props)
    rng = np.random.default_rng(0)
    T = 288.0 * (1.0 + 0.01 * (2.0 * rng.random(g.shape) - 1.0))
    y = st.c / st.c.sum(axis=0)
    st.c = y * (101325.0 / (R_GAS * T))[None]
    st.T = T
    st.Tw = np.full(g.wall_shape, 288.0)
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    ts = [0.0]
    res = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * 8000.0).integrate(
        m.pack(st), t_mid, [t_mid], on_step=lambda t, y, a: ts.append(t))
    np.savez_compressed(os.path.join(HERE, "bench_state_8x8x32_ads4000.npz"), y=res.y, t=res.t,
                        over=np.array(json.dumps(over)), n_steps=res.n_steps, wall=res.wall_time,
                        h_last=np.diff(ts)[-3:])
    print("bench state written:", res.n_steps, "steps,", res.wall_time, "s")


def make_bench_state_heating(ref_root, t_heat=4000.0):
    """Reference state of the 8x8x32 benchmark bed after the full adsorption (8000 s) and blowdown
    (60 s) steps of the cycle and t_heat seconds of heating, from the seeded constant-pressure initial
    state (input of the heating half of the CPU throughput sample in bench.py)."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.residual import TVSAModel
    from core.solver import TRBDF2
    from core.state import initial_state
    from properties import R_GAS, get_backend
    from steps._runner import run_step
    over = {"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32, "solver.scheme": "trbdf2",
            "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0, "operation.T_heat": 373.0,
            "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5, "ambient.T": 288.0}
    cfg = rp.load_config(override_dict=over)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = initial_state(cfg, g, props)
    rng = np.random.default_rng(0)
    T = 288.0 * (1.0 + 0.01 * (2.0 * rng.random(g.shape) - 1.0))
    y = st.c / st.c.sum(axis=0)
    st.c = y * (101325.0 / (R_GAS * T))[None]
    st.T = T
    st.Tw = np.full(g.wall_shape, 288.0)
    T_prev = None
    for si in (0, 1):
        st, sr = run_step(st, cfg, g, props, cfg.cycle[si], T_jacket_prev=T_prev, snapshots=2)
        T_prev = sr.T_jacket
        print(sr.name, sr.duration, "s", sr.solver, sr.wall_time, "s", flush=True)
    step = cfg.cycle[2]
    m = TVSAModel(cfg, g, props, step, st, T_prev)
    ts = [0.0]
    res = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * float(step["duration"])).integrate(
        m.pack(st), t_heat, [t_heat], on_step=lambda t, y, a: ts.append(t))
    print(step["name"], res.n_steps, "steps", res.wall_time, "s", flush=True)
    np.savez_compressed(os.path.join(HERE, "bench_state_8x8x32_heat4000.npz"), y=res.y, t=res.t,
                        T_jacket=float(m.T_jacket(t_heat)), over=np.array(json.dumps(over)),
                        n_steps=res.n_steps, wall=res.wall_time, h_last=np.diff(ts)[-3:])
    print("heating bench state written")


def make_outlet_cases(ref_root):
    """Outlet records of the reference's runner at seeded states of each cycle step (3x4x6 bed,
    one seeded state per step), with the diagnostics they are built from."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.residual import TVSAModel
    from core.state import initial_state
    from properties import R_GAS, get_backend
    from steps._runner import _end_summary
    from valves.valve_logic import humid_air_composition

    base = {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6, "jacket.theta_coverage_deg": [0.0, 180.0],
            "feed.profile": "cosine_theta", "feed.profile_amplitude": 0.3}
    out, meta = {}, []
    for step_i in range(4):
        name = f"step{step_i}"
        cfg = rp.load_config(override_dict=base)
        g = Grid.from_config(cfg)
        props = get_backend(cfg)
        st = initial_state(cfg, g, props)
        rng = np.random.default_rng(500 + step_i)
        st.T = st.T + 5.0 * rng.random(st.T.shape)
        st.q = st.q + 0.5 * rng.random(st.q.shape)
        st.c = st.c * (1.0 + 0.05 * rng.random(st.c.shape))
        st.Tw = st.Tw + 3.0 * rng.random(st.Tw.shape)
        step = cfg.cycle[step_i]
        m = TVSAModel(cfg, g, props, step, st)
        y = m.pack(st)
        t = 3.0
        _, acc = m.rhs(t, y)
        d = m.rhs(t, y, diag=True)
        yf = humid_air_composition(m.species, cfg.feed.P, cfg.feed.T, cfg.feed.RH if m.water else 0.0,
                                   cfg.feed.y_co2_dry, float(props.p_sat(cfg.feed.T)))
        c_feed = yf[m.i_co2] * cfg.feed.P / (R_GAS * cfg.feed.T)
        row = {}
        for end in ("top", "bottom"):
            row.update(_end_summary(m, d, end, c_feed))
        V = g.volume_full()
        Vt = float(V.sum())
        row["bed_T_mean_K"] = float(np.sum(d["T"] * V) / Vt)
        row["bed_P_mean_Pa"] = float(np.sum(d["P"] * V) / Vt)
        c, q, e, Tw = m.unpack(y)
        for n, sp in enumerate(m.adsorbed):
            row[f"bed_q_{sp}_mean"] = float(np.sum(q[n] * V) / Vt)
        ai = m.acc_index
        for v in ("V1", "V2", "V3"):
            row[f"cum_CO2_out_{v}_mol"] = float(acc[ai[f"n_out_{v}_CO2"]])
        row["cum_Q_jacket_J"] = float(acc[ai["Q_jac_pos"]] + acc[ai["Q_jac_neg"]])
        out[f"{name}__y"] = y
        out[f"{name}__P0"] = st.P
        out[f"{name}__acc"] = acc
        out[f"{name}__T"] = d["T"]
        out[f"{name}__P"] = d["P"]
        out[f"{name}__yk"] = d["y"]
        for end in ("top", "bottom"):
            for key, val in d["bnd"][end].items():
                out[f"{name}__{end}__{key}"] = np.asarray(val, dtype=float)
        meta.append({"name": name, "over": base, "step": step_i, "t": t, "c_feed_co2": c_feed,
                     "bnd_keys": {end: sorted(d["bnd"][end].keys()) for end in ("top", "bottom")},
                     "row": {k: (v.value if hasattr(v, "value") else v) for k, v in row.items()}})
        print(name, step["name"], {k: row[k] for k in ("top_flow_out_mol_s", "bottom_flow_out_mol_s")}, flush=True)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "outlet_cases.npz"), **out)


CYCLE_POINT = {"solver.scheme": "trbdf2", "operation.T_adsorption_jacket": 288.0, "operation.T_cool": 288.0,
               "operation.T_heat": 373.0, "operation.P_vacuum": 1e4, "feed.T": 288.0, "feed.RH": 0.5,
               "ambient.T": 288.0}


def make_cycle_golden(ref_root, grid=(8, 8, 32), rtol=None):
    """The reference's full first cycle of a bed from the seeded constant-pressure state, step by
    step through its runner, with the balance check of its cycle driver (vtsa_cycle.py:107-110)."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.state import initial_state
    from properties import R_GAS, get_backend
    from steps import RUNNERS
    from validation.conservation_checks import check_cycle
    import time
    over = dict(CYCLE_POINT, **{"grid.Nr": grid[0], "grid.Ntheta": grid[1], "grid.Nz": grid[2]})
    if rtol is not None:
        over["solver.rtol"] = rtol
    cfg = rp.load_config(override_dict=over)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = initial_state(cfg, g, props)
    rng = np.random.default_rng(0)
    T = 288.0 * (1.0 + 0.01 * (2.0 * rng.random(g.shape) - 1.0))
    yfrac = st.c / st.c.sum(axis=0)
    st.c = yfrac * (101325.0 / (R_GAS * T))[None]
    st.T = T
    st.Tw = np.full(g.wall_shape, 288.0)
    out = {"over": np.array(json.dumps(over))}
    steps, T_prev, t_cycle = [], None, 0.0
    from core.residual import TVSAModel
    out["y0"] = TVSAModel(cfg, g, props, cfg.cycle[0], st).pack(st)
    wall0 = time.time()
    for k, step in enumerate(cfg.cycle):
        m = TVSAModel(cfg, g, props, step, st, T_prev)
        out[f"s{k}_P0"] = st.P
        out[f"s{k}_T_jacket_prev"] = np.array(np.nan if T_prev is None else T_prev)
        st, sr = RUNNERS[step["type"]](st, cfg, g, props, step=step, cycle_idx=1, t_cycle0=t_cycle,
                                       T_jacket_prev=T_prev)
        out[f"s{k}_y"] = m.pack(st)
        out[f"s{k}_t_accepted"] = np.array([r["t_step_s"] for r in sr.outlet])
        out[f"s{k}_acc"] = np.array([sr.acc[nm] for nm in m.acc_names])
        out[f"s{k}_inv"] = np.array(json.dumps({"start": sr.inv_start, "end": sr.inv_end}))
        out[f"s{k}_solver"] = np.array(json.dumps({kk: (vv if not isinstance(vv, np.generic) else vv.item())
                                                    for kk, vv in sr.solver.items()}))
        out[f"s{k}_meta"] = np.array(json.dumps({"name": sr.name, "duration": sr.duration, "T_jacket": sr.T_jacket,
                                                 "jacket_on": sr.jacket_on, "wall_time": sr.wall_time}))
        print(sr.name, sr.duration, sr.solver, f"{sr.wall_time:.1f} s", flush=True)
        t_cycle += sr.duration
        T_prev = sr.T_jacket if sr.jacket_on else T_prev
        steps.append(sr)
    mb, eb, ok = check_cycle(steps, list(props.species))
    out["mass_rel_err"] = np.array([r["relative_error"] for r in mb])
    out["energy_rel_err"] = np.array([r["relative_error"] for r in eb])
    out["balance_rows"] = np.array(json.dumps({"mass": mb, "energy": eb}, default=float))
    out["wall_s"] = np.array(time.time() - wall0)
    tag = "" if rtol is None else f"_rtol{rtol:g}"
    name = f"cycle_{grid[0]}x{grid[1]}x{grid[2]}{tag}.npz"
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, "max |mass err|", np.abs(out["mass_rel_err"]).max(), "max |energy err|",
          np.abs(out["energy_rel_err"]).max(), "wall", float(out["wall_s"]), flush=True)


def make_csv_golden(ref_root):
    """A seeded non-trivial 3x4x6 state written by the reference's save_state_csv (simio/checkpoint.py:
    27-53), with the arrays it came from."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.state import initial_state
    from properties import get_backend
    from simio.checkpoint import save_state_csv
    cfg = rp.load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = Grid.from_config(cfg)
    st = initial_state(cfg, g, get_backend(cfg))
    rng = np.random.default_rng(11)
    st.T = st.T + 7.0 * rng.random(st.T.shape)
    st.q = st.q + rng.random(st.q.shape)
    st.c = st.c * (1.0 + 0.1 * rng.random(st.c.shape))
    st.Tw = st.Tw + 3.0 * rng.random(st.Tw.shape)
    st.t, st.cycle, st.step = 1234.5678901234567, 3, "heating"
    d = os.path.join(HERE, "state_csv")
    save_state_csv(st, g, os.path.join(d, "seeded_3x4x6.csv"))
    np.savez_compressed(os.path.join(d, "seeded_3x4x6.npz"), c=st.c, q=st.q, T=st.T, Tw=st.Tw,
                        meta=np.array(json.dumps({"t": st.t, "cycle": st.cycle, "step": st.step})))


def make_stop_golden(ref_root):
    """The adsorption step of the reference's young2021 1-D case (config/cases/
    young2021_1d_equivalent.yaml: 1x1x30 bed, stop_on end_saturation 0.9895) from its initial state,
    run by the reference's step runner until the stop criterion fires: stop time and value, the
    stop metric at the start, the end state and the solver counters."""
    sys.path.insert(0, ref_root)
    import yaml
    import config.parameters as rp
    from core.grid import Grid
    from core.residual import TVSAModel
    from core.state import initial_state
    from properties import get_backend
    from steps import RUNNERS
    case = os.path.join(ref_root, "config", "cases", "young2021_1d_equivalent.yaml")
    with open(case) as fh:
        raw = yaml.safe_load(fh)
    cfg = rp.load_config(user_yaml=case)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    st = initial_state(cfg, g, props)
    k = [i for i, s_ in enumerate(cfg.cycle) if s_.get("stop_on")][0]
    step = cfg.cycle[k]
    m = TVSAModel(cfg, g, props, step, st)
    y0 = m.pack(st)
    metric0 = m.stop_metric(0.0, y0)
    st1, sr = RUNNERS[step["type"]](st, cfg, g, props, step=step, cycle_idx=1, snapshots=2)
    y1 = TVSAModel(cfg, g, props, step, st).pack(st1)
    out = {"case_yaml": np.array(json.dumps(raw)), "step_index": np.array(k), "y0": y0, "P0": st.P,
           "metric0": np.array(metric0), "q_feed_eq": np.array(m.q_feed_eq()), "y_end": y1,
           "t_stop": np.array(sr.duration), "stopped_early": np.array(sr.stopped_early),
           "stop_value": np.array(m.stop_metric(sr.duration, y1)),
           "solver": np.array(json.dumps({kk: (vv.item() if isinstance(vv, np.generic) else vv)
                                          for kk, vv in sr.solver.items()}))}
    np.savez_compressed(os.path.join(HERE, "stop_young2021.npz"), **out)
    print("stop golden:", sr.duration, sr.stopped_early, out["stop_value"], sr.solver, flush=True)


if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1].startswith("--"):
        raise SystemExit("usage: make_golden.py <reference checkout> [--outlet | --bench-state | "
                         "--bench-state-heating | --cycle [--rtol X] | --stop | --csv | --modes | --css]")
    root = sys.argv[1]
    if "--modes" in sys.argv or "--css" in sys.argv:
        pass                        # handled below
    elif "--stop" in sys.argv:
        make_stop_golden(root)
    elif "--csv" in sys.argv:
        make_csv_golden(root)
    elif "--cycle" in sys.argv:
        rt = float(sys.argv[sys.argv.index("--rtol") + 1]) if "--rtol" in sys.argv else None
        make_cycle_golden(root, rtol=rt)
    elif "--outlet" in sys.argv:
        make_outlet_cases(root)
    elif "--bench-state" in sys.argv:
        make_bench_state(root)
    elif "--bench-state-heating" in sys.argv:
        make_bench_state_heating(root)
    else:
        main(root)


def make_modes_golden(ref_root):
    """200 s adsorption of the 4x4x16 bed from the seeded constant-pressure state with the
    reference's other Newton modes (core/solver.py:111-151,339-347): hybrid with its theta-block
    factors, and modified with the full factorisation: end states, accepted steps and counters."""
    sys.path.insert(0, ref_root)
    import config.parameters as rp
    from core.grid import Grid
    from core.residual import TVSAModel
    from core.solver import TRBDF2
    from core.state import initial_state
    from properties import R_GAS, get_backend
    out = {}
    for name, extra in (("hybrid", {"solver.newton_mode": "hybrid"}),
                        ("modified", {"solver.newton_mode": "modified", "solver.preconditioner": "full"})):
        over = dict(CYCLE_POINT, **{"grid.Nr": 4, "grid.Ntheta": 4, "grid.Nz": 16}, **extra)
        cfg = rp.load_config(override_dict=over)
        g = Grid.from_config(cfg)
        props = get_backend(cfg)
        st = initial_state(cfg, g, props)
        rng = np.random.default_rng(0)
        T = 288.0 * (1.0 + 0.01 * (2.0 * rng.random(g.shape) - 1.0))
        st.c = (st.c / st.c.sum(axis=0)) * (101325.0 / (R_GAS * T))[None]
        st.T = T
        st.Tw = np.full(g.wall_shape, 288.0)
        step = dict(cfg.cycle[0])
        step["duration"] = 200.0
        m = TVSAModel(cfg, g, props, step, st)
        integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * 200.0)
        y0 = m.pack(st)
        res = integ.integrate(y0, 200.0, [200.0])
        out[f"{name}_over"] = np.array(json.dumps(over))
        out[f"{name}_y0"] = y0
        out[f"{name}_P0"] = st.P
        out[f"{name}_y"] = res.y
        out[f"{name}_stats"] = np.array(json.dumps({"steps": res.n_steps, "rejected": res.n_reject,
                                                    "newton_fail": res.n_newton_fail, "krylov": res.n_krylov,
                                                    **{k: int(v) for k, v in integ.stats.items()}}))
        print(name, res.n_steps, integ.stats, flush=True)
    np.savez_compressed(os.path.join(HERE, "newton_modes_4x4x16.npz"), **out)


if __name__ == "__main__" and "--modes" in sys.argv:
    make_modes_golden(sys.argv[1])


def make_css_golden(ref_root):
    """The reference's CSS test quantities: state_change between two seeded 3x4x6 states, is_css at
    cycles 1..4, and the CO2 flows and cycle balance of the 8x8x32 cycle golden's steps."""
    sys.path.insert(0, ref_root)
    from types import SimpleNamespace
    import config.parameters as rp
    from core.grid import Grid
    from core.state import initial_state
    from postprocessing.reporting import step_flows
    from properties import get_backend
    from validation.cyclic_steady_state import cycle_co2_balance, is_css, state_change
    over = {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}
    cfg = rp.load_config(override_dict=over)
    g = Grid.from_config(cfg)
    props = get_backend(cfg)
    states = []
    for seed in (21, 22):
        st = initial_state(cfg, g, props)
        rng = np.random.default_rng(seed)
        st.T = st.T + 9.0 * rng.random(st.T.shape)
        st.q = st.q + 0.5 * rng.random(st.q.shape)
        st.c = st.c * (1.0 + 0.2 * rng.random(st.c.shape))
        states.append(st)
    ch = state_change(states[0], states[1], g, cfg)
    cyc = np.load(os.path.join(HERE, "cycle_8x8x32.npz"))
    ccfg = rp.load_config(override_dict=json.loads(str(cyc["over"])))
    names = [f"{p}_{v}_{s}" for v in ("V1", "V2", "V3") for p in ("n_in", "n_out") for s in ("CO2", "H2O", "N2")]
    acc_names = []
    for v in ("V1", "V2", "V3"):
        acc_names += [f"n_in_{v}_{s}" for s in ("CO2", "H2O", "N2")] + [f"n_out_{v}_{s}" for s in ("CO2", "H2O", "N2")]
        acc_names += [f"H_in_{v}", f"H_out_{v}", f"W_pump_{v}", f"W_fan_{v}"]
    acc_names += ["Q_jac_pos", "Q_jac_neg", "Q_amb", "Q_wb", "Q_hx_pos", "Q_hx_neg"]
    tot = {"fed": 0.0, "product": 0.0, "vented": 0.0}
    for k, step in enumerate(ccfg.cycle):
        sr = SimpleNamespace(acc=dict(zip(acc_names, cyc[f"s{k}_acc"])), product_port=step.get("product_port", "V3"),
                             valves=dict(step["valves"]))
        fl = step_flows(sr, ["CO2", "H2O", "N2"])["CO2"]
        for key in tot:
            tot[key] += fl[key]
    kp = {"CO2_fed_mol": tot["fed"], "CO2_product_mol": tot["product"], "CO2_vented_mol": tot["vented"]}
    flags = [bool(is_css(ch, kp, cfg, n)) for n in range(1, 5)]
    run0 = {"min_cycles": cfg.run.min_cycles, "css_tolerance": cfg.run.css_tolerance,
            "css_mb_tolerance": cfg.run.css_mb_tolerance}
    relaxed = rp.load_config(override_dict=dict(over, **{"run.css_tolerance": 1.0, "run.css_mb_tolerance": 0.5}))
    flags_relaxed = [bool(is_css(ch, kp, relaxed, n)) for n in range(1, 5)]     # both criteria met
    np.savez_compressed(os.path.join(HERE, "css_3x4x6.npz"), over=np.array(json.dumps(over)),
                        **{f"s{i}_{f}": getattr(st, f) for i, st in enumerate(states) for f in ("c", "q", "T", "Tw")},
                        change=np.array(json.dumps(ch)), flows=np.array(json.dumps(kp)),
                        co2_balance=np.array(cycle_co2_balance(kp)), is_css=np.array(flags),
                        is_css_relaxed=np.array(flags_relaxed), run=np.array(json.dumps(run0)))
    print(ch, kp, flags, flags_relaxed)


if __name__ == "__main__" and "--css" in sys.argv:
    make_css_golden(sys.argv[1])
