"""Pin the CPU oracle against the reference's own outputs (golden fixtures made by importing the
reference, tests/golden/make_golden.py) and its known-answer tests
(tests/test_physics_and_numerics.py of the reference)."""
import hashlib
import json

import numpy as np
import pytest

from cases import build, config0_overrides, golden, rhs_cases, state_like
from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config, with_overrides
from oracle.jacobian import OracleFDJacobian
from oracle.residual import OracleModel
from oracle.sparsity import colouring_is_valid, greedy_colour, pattern
from oracle.solver import OracleTRBDF2

CASES = list(rhs_cases())


@pytest.mark.parametrize("meta,data", CASES, ids=[m["name"] for m, _ in CASES])
def test_oracle_rhs_matches_reference_exactly(meta, data):
    m, _ = build(OracleModel, meta["over"], meta["step"], data["P0"], meta["T_jacket_prev"])
    f, acc = m.rhs(meta["t"], data["y"])
    assert np.array_equal(f, data["f"])
    assert np.array_equal(acc, data["acc"])
    d = m.rhs(meta["t"], data["y"], diag=True)
    assert np.array_equal(d["T"], data["T"]) and np.array_equal(d["P"], data["P"])


def test_colouring_matches_reference_small_grids():
    d = golden("colouring.npz")
    for key in d.files:
        if not key.startswith("full_"):
            continue
        dims = tuple(int(x) for x in key[5:].split("x"))
        P = pattern(*dims, 3, 2, True)
        c = greedy_colour(P)
        assert np.array_equal(c, d[key].astype(np.int64)), dims
        assert colouring_is_valid(P, c)


@pytest.mark.parametrize("dims", ["8x8x32", "4x16x64"])
def test_colouring_matches_reference_hashes(dims):
    hashes = json.loads(str(golden("colouring.npz")["hashes"]))
    c = greedy_colour(pattern(*(int(x) for x in dims.split("x")), 3, 2, True)).astype(np.int64)
    assert [hashlib.sha256(c.tobytes()).hexdigest(), int(c.max()) + 1] == hashes[dims]


def test_fd_jacobian_matches_reference_exactly():
    d = golden("jacobian_3x4x6.npz")
    m, _ = build(OracleModel, {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}, 0, d["P0"])
    J = OracleFDJacobian(m)(float(d["t"]), d["y"])
    assert np.array_equal(J.indptr, d["indptr"]) and np.array_equal(J.indices, d["indices"])
    assert np.array_equal(J.data, d["data"])


def test_integrator_matches_reference_trajectory():
    """200 s adsorption of the 4x4x16 bed: same accepted steps, same end state, bit for bit."""
    d = golden("trajectory_c0.npz")
    over = json.loads(str(d["over"]))
    meta = json.loads(str(d["s0_meta"]))
    m, cfg = build(OracleModel, over, meta["step"], d["s0_P0"], duration=meta["duration"])
    ts = []
    res = OracleTRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * meta["duration"]).integrate(
        d["s0_y0"], meta["duration"], np.linspace(0.0, meta["duration"], 12), on_step=lambda t, y, a: ts.append(t))
    assert np.array_equal(np.array(ts), d["s0_t_accepted"])
    assert np.array_equal(res.y, d["s0_y"]) and np.array_equal(res.acc, d["s0_acc"])
    assert [res.n_steps, res.n_reject, res.n_newton_fail, res.n_jac, res.n_lu, res.nfev] == list(d["s0_stats"][:6])


def test_isotherm_known_values():
    """Reference known-answer test (tests/test_physics_and_numerics.py:53-65): GAB 4.091, dry Toth
    1.0226, WADST 1.511, mechanistic 1.462 at 288.15 K, 55 % RH, 400 ppm."""
    cfg = load_config()
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    P0 = np.full(g.shape, 101325.0)
    m = OracleModel(cfg, g, props, cfg.cycle[0], state_like(P0))
    T = 288.15
    ps = float(host.arden_buck(T))
    pw = 0.55 * ps
    pc = 4e-4 * (101325 - pw)
    qw = float(m.q_h2o(pw, T, ps))
    assert abs(qw - 4.091) < 5e-3
    assert abs(float(m.q_co2_dry(pc, T)) - 1.0226) < 2e-3
    assert abs(float(m.q_co2(pc, T, qw)) - 1.511) < 3e-3
    mech = OracleModel(with_overrides(cfg, {"isotherm.coadsorption.model": "mechanistic"}), g, props,
                       cfg.cycle[0], state_like(P0))
    assert abs(float(mech.q_co2(pc, T, qw)) - 1.462) < 3e-3
    assert abs(float(host.arden_buck(373.15)) - 101325) / 101325 < 3e-3
    q = m.q_co2(np.array([-1.0, 0.0, 1e-9]), 300.0, np.array([0.0, 1.0, 2.0]))
    assert np.all(np.isfinite(q)) and q[0] == 0.0 and q[1] == 0.0


def test_temperature_energy_roundtrip():
    cfg = load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.initial_state(cfg, g, props)
    st.T = st.T + np.random.default_rng(3).random(st.T.shape)
    m = OracleModel(cfg, g, props, cfg.cycle[0], st)
    c, q, e, _ = m.unpack(m.pack(st))
    assert np.max(np.abs(m.temperature(e, c, q) - st.T)) < 1e-9
