"""GPU residual kernels vs the reference's outputs (golden fixtures) and the oracle.

Tolerance: the kernels do the same IEEE additions / multiplications as numpy (no FMA contraction);
only exp/log/pow/tanh/log1p differ from glibc by ~1 ulp.  Entries are compared per variable block
relative to the largest magnitude of that block: |f_gpu - f_ref| <= 1e-11 * max|f_ref(block)|."""
import numpy as np
import pytest
import torch

from cases import build, rhs_cases

pytestmark = pytest.mark.gpu
CASES = list(rhs_cases())
TOL = 1e-11


def _blocks(m, v):
    n = m.grid.ncell
    out = [v[k * n:(k + 1) * n] for k in range(6)]
    if m.n_w:
        out.append(v[m.off_w:])
    return out


@pytest.mark.parametrize("meta,data", CASES, ids=[m["name"] for m, _ in CASES])
def test_rhs_matches_reference(meta, data):
    from dac_vtsa_b200.model import TVSAModel
    m, _ = build(TVSAModel, meta["over"], meta["step"], data["P0"], meta["T_jacket_prev"])
    f, acc = m.rhs(meta["t"], data["y"])
    for a, b in zip(_blocks(m, f), _blocks(m, data["f"])):
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= TOL * scale
    accs = np.abs(data["acc"]).max()
    assert np.abs(acc - data["acc"]).max() <= TOL * max(accs, 1e-300)
    d = m.rhs(meta["t"], data["y"], diag=True)
    assert np.abs(d["T"] - data["T"]).max() <= 1e-12 * np.abs(data["T"]).max()
    assert np.abs(d["P"] - data["P"]).max() <= 1e-12 * np.abs(data["P"]).max()


@pytest.mark.parametrize("meta,data", CASES[:4], ids=[m["name"] for m, _ in CASES[:4]])
def test_rhs_conserves_species_and_energy(meta, data):
    """Reference semi-discrete conservation test (tests/test_physics_and_numerics.py:79-104) on the GPU
    outputs: sum V d(inventory)/dt equals the boundary accumulator rates."""
    from dac_vtsa_b200.model import TVSAModel
    m, _ = build(TVSAModel, meta["over"], meta["step"], data["P0"], meta["T_jacket_prev"])
    g = m.grid
    f, acc = m.rhs(meta["t"], data["y"])
    ai = m.acc_index
    dc = f[:m.n_c].reshape((m.ng,) + g.shape)
    dq = f[m.off_q:m.off_e].reshape((m.na,) + g.shape)
    for k, s in enumerate(m.species):
        dinv = np.sum(m.eps_t * dc[k] * g.V)
        if s in m.adsorbed:
            dinv += np.sum(m.rho_b * dq[m.adsorbed.index(s)] * g.V)
        net = sum(acc[ai[f"n_in_{v}_{s}"]] - acc[ai[f"n_out_{v}_{s}"]] for v in ("V1", "V2", "V3"))
        assert abs(dinv - net) <= 1e-12 * max(1.0, abs(net)) + 1e-18
    de = f[m.off_e:m.off_w].reshape(g.shape)
    dTw = f[m.off_w:m.n_core].reshape(g.wall_shape)
    dE = np.sum(de * g.V) + np.sum(m.wall.C * dTw)
    netH = (sum(acc[ai[f"H_in_{v}"]] - acc[ai[f"H_out_{v}"]] for v in ("V1", "V2", "V3"))
            + acc[ai["Q_jac_pos"]] + acc[ai["Q_jac_neg"]] + acc[ai["Q_amb"]] + acc[ai["Q_hx_pos"]] + acc[ai["Q_hx_neg"]])
    assert abs(dE - netH) <= 1e-9 * max(1.0, abs(netH))


def test_stage_residual_and_device_inputs():
    from dac_vtsa_b200.model import TVSAModel
    meta, data = CASES[0]
    m, _ = build(TVSAModel, meta["over"], meta["step"], data["P0"])
    y = data["y"]
    rk = y * 0.999
    R = m.stage_residual(2.0, y, 0.3, rk)
    f, _ = m.rhs(2.0, y, want_acc=False)
    assert np.array_equal(R, y - 0.3 * f - rk)
    yd = torch.from_numpy(y).cuda()
    fd, accd = m.rhs(2.0, yd)
    assert fd.is_cuda and np.array_equal(fd.cpu().numpy(), f)


def test_axisymmetric_state_stays_axisymmetric():
    """Reference symmetry test (tests/test_physics_and_numerics.py:166-179) on the GPU residual."""
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    cfg = load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.initial_state(cfg, g, props)
    st.T = st.T + 5.0 * np.random.default_rng(5).random((g.Nr, 1, g.Nz))
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    f, _ = m.rhs(10.0, m.pack(st), want_acc=False)
    c, q, e, Tw = m.unpack(f)
    for arr in (c, q, e[None]):
        spread = np.abs(arr - arr.mean(axis=-2, keepdims=True)).max()
        assert spread <= 1e-9 * max(np.abs(arr).max(), 1e-30)


def test_outlet_records_match_reference():
    """GPU diagnostics of every cycle step at a seeded state: the boundary records the outlet is
    built from match the reference's, and so does the outlet row reduced on the device (the
    reference's runner record, steps/_runner.py:50-121)."""
    import json
    from cases import golden
    from outlet_rows import same_row as _same_row
    from dac_vtsa_b200.model import TVSAModel
    import torch
    from dac_vtsa_b200.runner import OutletRecorder
    d = golden("outlet_cases.npz")
    for meta in json.loads(str(d["meta"])):
        n = meta["name"]
        m, _ = build(TVSAModel, meta["over"], meta["step"], d[f"{n}__P0"])
        y = d[f"{n}__y"]
        dg = m.rhs(meta["t"], y, diag=True)
        for end in ("top", "bottom"):
            assert sorted(dg["bnd"][end]) == meta["bnd_keys"][end], (n, end)
            for k in meta["bnd_keys"][end]:
                ref = d[f"{n}__{end}__{k}"]
                scale = max(np.abs(ref).max(), 1e-300)
                assert np.abs(dg["bnd"][end][k] - ref).max() <= TOL * scale, (n, end, k)
        rec = OutletRecorder(m, meta["c_feed_co2"], capacity=2)
        yd = torch.from_numpy(np.ascontiguousarray(y)).to(m.device)
        rec.record(meta["t"], yd.data_ptr(), d[f"{n}__acc"])
        row = rec.rows({"cycle": 1, "step": "x", "t_cycle0": 0.0, "t_total0": 0.0})[0]
        for k in ("cycle", "step", "t_step_s", "t_cycle_s", "t_total_s"):
            row.pop(k)
        _same_row(row, meta["row"], rtol=1e-10, atol=1e-18)


def test_split_residual_is_bit_identical_to_the_thread_per_cell_evaluation():
    """The split residual (per-cell properties with their independent transcendental terms spread
    over the warps of a block, every face once, per-cell assembly) and the thread-per-cell kernel
    behind dv_rhs_acc_noalloc evaluate the same expressions on the same operands: f and the 36
    accumulator rates agree bit for bit on every golden case (every closure and co-adsorption
    model)."""
    import ctypes as C
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.params import build_params
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for meta, data in CASES:
        m, _ = build(TVSAModel, meta["over"], meta["step"], data["P0"], meta["T_jacket_prev"])
        f, acc = m.rhs(meta["t"], data["y"])
        params, feed_h, nnom_h, cov_h, _ = build_params(m.cfg, m.grid, m.props, m.step, m.P_start,
                                                        meta["T_jacket_prev"])
        put = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(m.device)  # noqa: E731
        feed, nnom, cov, y = put(feed_h), put(nnom_h), put(cov_h), put(data["y"])
        f2 = torch.full_like(y, np.nan)
        acc2 = torch.full((36,), np.nan, dtype=torch.float64, device=m.device)
        rc = lib.dv_rhs_acc_noalloc(C.byref(params), feed.data_ptr(), nnom.data_ptr(), cov.data_ptr(), meta["t"],
                                    y.data_ptr(), f2.data_ptr(), acc2.data_ptr(), stream)
        assert rc == 0, lib.dv_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(f, f2.cpu().numpy()), meta["name"]
        assert np.array_equal(acc, acc2.cpu().numpy()), meta["name"]
