"""GPU preconditioner, Newton-Krylov stage solve and integrator vs the oracle / reference."""
import json

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cases import build, config0_overrides, golden

pytestmark = pytest.mark.gpu


def _partition_of(m, mode):
    """Partition id of every unknown: theta sector ("sector"), sector with the innermost ring of all
    sectors split off as one more partition ("theta_block"), or one partition ("full")."""
    g = m.grid
    n = g.ncell
    idx = np.arange(m.n_core)
    cellpart = idx < 6 * n
    sector = np.where(cellpart, ((idx % n) // g.Nz) % g.Nth, (idx - 6 * n) // g.Nz)
    ring = np.where(cellpart, (idx % n) // (g.Nth * g.Nz), g.Nr - 1)
    if mode == "sector":
        return sector
    if mode == "theta_block":
        split = _split_groups(g.Nr, g.Nth, m.n_w > 0)
        if split is None:
            return np.where(ring == 0, g.Nth, sector)
        rg, tg = split
        ring_group = np.array([_group_of(g.Nr - 1, rg, i - 1) if i > 0 else 0 for i in range(g.Nr)])
        theta_group = np.array([_group_of(g.Nth, tg, j) for j in range(g.Nth)])
        return np.where(ring == 0, g.Nth * rg + theta_group[sector], sector * rg + ring_group[ring])
    return np.zeros_like(idx)


def _group_of(n, G, t):
    base, extra = n // G, n % G
    return t // (base + 1) if t < extra * (base + 1) else extra + (t - extra * (base + 1)) // base


def _split_groups(Nr, Nth, wall, limit=56, target=48):
    """(ring groups, theta groups) of the split theta_block partitions, or None when the sectors
    and the core ring fit the shared-memory kernels whole: rings 1..Nr-1 of a sector in the fewest
    contiguous groups (larger groups inside, the wall node with the outermost) of at most `target`
    unknowns, the core ring's sectors likewise."""
    if Nr < 2 or Nth < 2 or max(6 * (Nr - 1) + (1 if wall else 0), 6 * Nth) <= limit:
        return None

    def ring_nb(G):
        n, out = Nr - 1, 0
        base, extra = n // G, n % G
        for gi in range(G):
            size = base + (1 if gi < extra else 0)
            out = max(out, 6 * size + (1 if (wall and gi == G - 1) else 0))
        return out
    rg = 1
    while rg < Nr - 1 and ring_nb(rg) > target:
        rg += 1
    tg = 1
    while tg < Nth and 6 * -(-Nth // tg) > target:
        tg += 1
    return rg, tg


def _pc_model(Nz, Nr=3, Nth=4):
    """Nr x Nth x Nz bed and a state: the golden Jacobian state for 3 x 4 x 6, else a seeded state."""
    from dac_vtsa_b200.model import TVSAModel
    if Nz == 6 and Nr == 3 and Nth == 4:
        d = golden("jacobian_3x4x6.npz")
        m, _ = build(TVSAModel, {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}, 0, d["P0"])
        return m, d["y"]
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    cfg = load_config(override_dict={"grid.Nr": Nr, "grid.Ntheta": Nth, "grid.Nz": Nz})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, g, props, seed=3, amplitude=0.05)
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    return m, m.pack(st)


def _restricted(m, Jc, mode, dh):
    """I - dh J with the couplings across partitions dropped."""
    Jc = Jc.tocoo()
    part = _partition_of(m, mode)
    keep = part[Jc.row] == part[Jc.col]
    Jk = sp.csc_matrix((Jc.data[keep], (Jc.row[keep], Jc.col[keep])), shape=Jc.shape)
    return (sp.identity(m.n_core, format="csc") - dh * Jk).tocsc()


def _dominant_jacobian(m, seed):
    """Random values on the stencil pattern (block layout on the device + the same matrix in CSC),
    small enough that I - J is strongly diagonally dominant: every block elimination order is
    stable on it, so a solve is exact to rounding."""
    import torch
    from dac_vtsa_b200.jacobian import FDJacobian
    jac = FDJacobian(m)
    Jb = np.zeros(m.jac_doubles)
    Jb[jac._blk] = np.random.default_rng(seed).uniform(-1.0, 1.0, len(jac._blk)) * (0.5 / 63)
    Jc = sp.csc_matrix((Jb[jac._blk], jac.indices, jac.indptr), shape=(jac.n, jac.n))
    return torch.from_numpy(Jb).to(m.device), Jc


# Nz = 6, 7: one elimination direction; Nz >= 8: twisted (Nz = 17: top-down over 7 planes,
# bottom-up over 8, separator planes 7 and 8)
@pytest.mark.parametrize("Nz", [6, 8, 17, 32])
@pytest.mark.parametrize("mode", ["theta_block", "sector", "full"])
def test_preconditioner_exact_on_dominant_system(mode, Nz):
    """dv_precond_solve == sparse LU solve of I - J restricted to the partition couplings, to
    rounding, on a diagonally dominant J that fills the whole stencil pattern."""
    _check_dominant(mode, Nz, 3)


# 8 rings: sector partitions of nb 49 (ld 64, two-deep ring, shared stride 52), theta_block
# partitions of nb 43 / 24
@pytest.mark.parametrize("mode", ["sector", "theta_block"])
def test_preconditioner_exact_on_dominant_system_8_rings(mode):
    """The same check on an 8-ring bed, whose sector blocks take the widest shared-memory layout."""
    _check_dominant(mode, 12, 8)


# beds whose theta_block partitions exceed the shared-memory kernels: 11 rings (sector rings split
# 5 + 5, the wall with the outer group), 10 sectors (core ring split 5 + 5), and the 16 x 16 cross-
# section (rings 8 + 7 + wall, core 8 + 8 sectors)
@pytest.mark.parametrize("Nr,Nth,Nz", [(11, 4, 9), (3, 10, 12), (16, 16, 8)])
def test_split_partitions_exact_on_dominant_system(Nr, Nth, Nz):
    """Large cross-sections factorise split partitions (ring groups per sector, theta groups of the
    core ring): the solve equals a sparse LU of I - J restricted to exactly those partitions."""
    assert _split_groups(Nr, Nth, True) is not None
    _check_dominant("theta_block", Nz, Nr, Nth)


def _check_dominant(mode, Nz, Nr, Nth=4):
    m, _ = _pc_model(Nz, Nr, Nth)
    Jd, Jc = _dominant_jacobian(m, 40 + Nz)
    m.precond_factor(Jd, 1.0, mode)
    M = _restricted(m, Jc, mode, 1.0)
    b = np.random.default_rng(7).standard_normal(m.n_core)
    x_ref = spla.spsolve(M, b)
    x = m.precond_solve(b)
    assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max()


@pytest.mark.parametrize("mode", ["theta_block", "sector", "full"])
def test_preconditioner_solves_partition_system(mode):
    """dv_precond_solve == exact sparse solve of I - dh J restricted to the partition couplings."""
    from dac_vtsa_b200.jacobian import FDJacobian
    m, y = _pc_model(6)
    jac = FDJacobian(m)
    Jc = jac(5.0, y)
    dh = 0.3 * 7.0
    m.precond_factor(jac.block(5.0, y), dh, mode)
    M = _restricted(m, Jc, mode, dh)
    b = np.random.default_rng(7).standard_normal(m.n_core) * m.atol
    x_ref = spla.spsolve(M, b)
    x = m.precond_solve(b)
    # componentwise backward error |M x - b| / (|M| |x| + |b|): block LU with partial pivoting is
    # backward stable; the forward error may grow with cond(M) (stiff pressure couplings)
    Ma = abs(M)
    berr = np.abs(M @ x - b) / (Ma @ np.abs(x) + np.abs(b))
    berr_ref = np.abs(M @ x_ref - b) / (Ma @ np.abs(x_ref) + np.abs(b))
    assert berr.max() <= max(1e-12, 10 * berr_ref.max()), (berr.max(), berr_ref.max())
    assert np.abs(x - x_ref).max() <= 1e-6 * np.abs(x_ref).max()


@pytest.mark.parametrize("mode", ["theta_block", "sector"])
@pytest.mark.parametrize("Nz", [8, 17, 32])
def test_twisted_factorisation_matches_one_directional(Nz, mode, monkeypatch):
    """The twisted factorisation (eliminations from both ends meeting at two separator planes)
    factorises the same partition matrix as the top-down one: on a dominant system the solves
    agree to rounding, and differ (the two orders round differently), which shows the twisted path
    ran; DVTSA_PC_TWIST=0 selects the top-down form."""
    m, _ = _pc_model(Nz)
    Jd, _ = _dominant_jacobian(m, 3)
    b = np.random.default_rng(5).standard_normal(m.n_core)
    m.precond_factor(Jd, 1.0, mode)
    x_tw = m.precond_solve(b)
    monkeypatch.setenv("DVTSA_PC_TWIST", "0")
    m.precond_factor(Jd, 1.0, mode)
    x_one = m.precond_solve(b)
    rel = np.abs(x_tw - x_one).max() / np.abs(x_one).max()
    assert 0.0 < rel < 1e-13, rel


@pytest.mark.parametrize("dh", [2.1, 300.0])
@pytest.mark.parametrize("Nz", [17, 32])
def test_twisted_separator_inverse_on_stiff_stage_matrix(Nz, dh, monkeypatch):
    """The separator stored as its explicit inverse, on poorly conditioned systems: I - dh J with the
    finite-difference Jacobian of a seeded 3 x 4 x Nz bed, whose separator Schur complements have
    condition numbers of about 6e7 (Nz 17, dh 2.1) to 1.6e10 (Nz 32, dh 300) in the solver's scaled
    variables (numpy, same matrices).  Twisted and top-down factorisations both keep a componentwise
    backward error within 10x of the sparse LU's."""
    from dac_vtsa_b200.jacobian import FDJacobian
    m, y = _pc_model(Nz)
    jac = FDJacobian(m)
    Jc = jac(5.0, y)
    Jb = jac.block(5.0, y)
    M = _restricted(m, Jc, "theta_block", dh)
    b = np.random.default_rng(11).standard_normal(m.n_core) * m.atol
    x_ref = spla.spsolve(M, b)
    Ma = abs(M)

    def berr(x):
        return float((np.abs(M @ x - b) / (Ma @ np.abs(x) + np.abs(b))).max())

    m.precond_factor(Jb, dh, "theta_block")
    x_tw = m.precond_solve(b)
    monkeypatch.setenv("DVTSA_PC_TWIST", "0")
    m.precond_factor(Jb, dh, "theta_block")
    x_one = m.precond_solve(b)
    ref = berr(x_ref)
    assert berr(x_tw) <= max(1e-12, 10 * ref), (berr(x_tw), ref)
    assert berr(x_one) <= max(1e-12, 10 * ref), (berr(x_one), ref)


def test_implicit_solver_matches_rk4_on_short_transient():
    """Reference integration test (tests/test_physics_and_numerics.py:182-200): SDIRK2 Newton-Krylov
    on the GPU vs classical RK4 (oracle) on a 2x1x4 blowdown, 2 ms, scaled RMS error < 1."""
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    from oracle.residual import OracleModel
    from oracle.solver import explicit_dt, integrate_rk4
    cfg = load_config(override_dict={"grid.Nr": 2, "grid.Ntheta": 1, "grid.Nz": 4, "solver.rtol": 1e-6,
                                     "solver.newton_kappa": 1e-3})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.initial_state(cfg, g, props)
    mo = OracleModel(cfg, g, props, cfg.cycle[1], st)
    y0 = mo.pack(st)
    t_end = 2e-3
    y_rk = integrate_rk4(mo, y0, t_end, explicit_dt(mo, y0, safety=0.25))[0]
    m = TVSAModel(cfg, g, props, cfg.cycle[1], st)
    res = TRBDF2(m, cfg, h_max=t_end, h_init=1e-6).integrate(y0, t_end, np.array([t_end]))
    sc = m.atol + 1e-4 * np.abs(y_rk)
    err = np.sqrt(np.mean(((res.y - y_rk) / sc) ** 2))
    assert err < 1.0, err


def _c0_model(cls, k=0):
    d = golden("trajectory_c0.npz")
    over = json.loads(str(d["over"]))
    meta = json.loads(str(d[f"s{k}_meta"]))
    m, cfg = build(cls, over, meta["step"], d[f"s{k}_P0"], meta["T_jacket_prev"], duration=meta["duration"])
    return d, m, cfg, meta


def test_replay_step_end_states_within_1e8():
    """Replay the reference's first accepted steps of the 4x4x16 adsorption: GPU and oracle solve the
    same stage equations tightly; step-end states agree to 1e-8 relative."""
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.replay import fixed_step_run as gpu_run
    from oracle.residual import OracleModel
    from oracle.solver import fixed_step_run as cpu_run
    d, m, cfg, meta = _c0_model(TVSAModel)
    _, mo, _, _ = _c0_model(OracleModel)
    ts = np.concatenate([[0.0], d["s0_t_accepted"]])
    hs = np.diff(ts)[:12]
    y0 = d["s0_y0"]
    ys_gpu, acc_gpu = gpu_run(m, y0, hs, scheme="trbdf2")
    ys_cpu, acc_cpu = cpu_run(mo, y0, hs, scheme="trbdf2", tol=1e-12)
    worst = 0.0
    for a, b in zip(ys_gpu, ys_cpu):
        rel = np.abs(a - b) / (np.abs(b) + m.atol)
        worst = max(worst, float(rel.max()))
    assert worst <= 1e-8, worst
    assert np.allclose(acc_gpu, acc_cpu, rtol=1e-8, atol=1e-20)


@pytest.mark.parametrize("precision", ["fp32_factors", "fp32"])
def test_mixed_precision_replay_matches_fp64_within_1e6(precision):
    """Mixed precision (FP32 factors; and GMRES on the FP32 assembled Jacobian with FP32 factors) with
    the FP64 residual and Newton update, replaying the reference's first accepted steps of the
    4x4x16 adsorption with every stage solved tightly: the step-end states agree with the FP64
    path's to <= 1e-6 relative per entry (the stated mixed-mode tolerance).  The FP32 operator's
    Newton iteration contracts linearly, so its stages are solved to 1e-9 of the error scale in up
    to 60 iterations (the FP64 path: 1e-11)."""
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.replay import fixed_step_run as gpu_run
    d, m64, cfg, meta = _c0_model(TVSAModel)
    _, m32, _, _ = _c0_model(TVSAModel)
    m32.set_krylov_precision(precision)
    ts = np.concatenate([[0.0], d["s0_t_accepted"]])
    hs = np.diff(ts)[:12]
    y0 = d["s0_y0"]
    ys64, acc64 = gpu_run(m64, y0, hs, scheme="trbdf2")
    kw = {"kappa": 1e-9, "max_iter": 60} if precision == "fp32" else {}
    ys32, acc32 = gpu_run(m32, y0, hs, scheme="trbdf2", **kw)
    worst = max(float((np.abs(a - b) / (np.abs(b) + m64.atol)).max()) for a, b in zip(ys32, ys64))
    assert worst <= 1e-6, worst
    assert np.allclose(acc32, acc64, rtol=1e-6, atol=1e-20)


def test_free_running_adsorption_matches_reference_to_tolerance():
    """Adaptive 200 s adsorption of the 4x4x16 bed (TR-BDF2, reference defaults): the end state agrees
    with the reference's within its own tolerance scale, and mass/energy balances close as tightly."""
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d, m, cfg, meta = _c0_model(TVSAModel)
    dur = meta["duration"]
    res = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur).integrate(d["s0_y0"], dur, np.linspace(0, dur, 12))
    y_ref = d["s0_y"]
    sc = m.atol + cfg.solver.rtol * np.abs(y_ref)
    err = np.sqrt(np.mean(((res.y - y_ref) / sc) ** 2))
    assert res.t == pytest.approx(dur)
    assert err < 5.0, err
    # balances: inventory change == accumulated boundary flows
    inv0, inv1 = m.inventories(d["s0_y0"]), m.inventories(res.y)
    ai = m.acc_index
    for s in m.species:
        fin = sum(res.acc[ai[f"n_in_{v}_{s}"]] for v in ("V1", "V2", "V3"))
        fout = sum(res.acc[ai[f"n_out_{v}_{s}"]] for v in ("V1", "V2", "V3"))
        resid = (inv1[f"tot_{s}"] - inv0[f"tot_{s}"]) - (fin - fout)
        scale = max(abs(fin), abs(fout), abs(inv0[f"tot_{s}"]), abs(inv1[f"tot_{s}"]))
        assert abs(resid) / scale < 1e-4


def test_results_do_not_depend_on_unwritten_memory(monkeypatch):
    """The same 200 s adsorption with every new workspace pre-filled by different bytes (zeros, a
    huge finite value, NaN) gives bit-identical states and solver statistics: no kernel or host step
    reads memory that nothing wrote (such a read once let the energy balance test pick up bytes past
    the end of the residual vector)."""
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    runs = []
    for fill in ("0x00", "0x7f", "0xff"):
        monkeypatch.setenv("DVTSA_FILL", fill)
        d, m, cfg, meta = _c0_model(TVSAModel)
        dur = meta["duration"]
        integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
        res = integ.integrate(d["s0_y0"], dur, [dur])
        runs.append((res.y, res.n_steps, res.n_krylov, dict(integ.stats)))
    for y, n_steps, n_krylov, stats in runs[1:]:
        assert np.array_equal(y, runs[0][0])
        assert (n_steps, n_krylov, stats) == runs[0][1:]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_step_statistics_track_the_reference(k):
    """Free-running adsorption (200 s), blowdown (10 s) and heating (100 s) of the 4x4x16 bed take
    about as many accepted and rejected steps as the reference did on the same input: the GPU
    preconditioner is not SuperLU's, so GMRES counts differ, but a solver fault (a wrong matvec, a
    stale norm) shows up as many more steps, rejections or Newton failures."""
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d, m, cfg, meta = _c0_model(TVSAModel, k)
    dur = meta["duration"]
    integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
    res = integ.integrate(d[f"s{k}_y0"], dur, [dur])
    ref_steps, ref_rej, ref_fail = (int(v) for v in d[f"s{k}_stats"][:3])
    ref_gmres = int(d[f"s{k}_stats"][6])
    assert abs(res.n_steps - ref_steps) <= max(5, 0.15 * ref_steps), (res.n_steps, ref_steps)
    assert res.n_reject <= ref_rej + 5, (res.n_reject, ref_rej)
    assert res.n_newton_fail <= ref_fail + 3, (res.n_newton_fail, ref_fail)
    assert integ.stats["gmres_iters"] <= 2 * ref_gmres + 50, (integ.stats["gmres_iters"], ref_gmres)


@pytest.mark.parametrize("Nz", [6, 17])
def test_fp32_factors_solve_to_single_precision(Nz):
    """The sweep over FP32-stored factors (mixed-precision Krylov) solves the same partition system
    as the FP64 one to single-precision accuracy (one-directional and twisted factors)."""
    m, _ = _pc_model(Nz)
    J, _ = _dominant_jacobian(m, 11)
    b = np.random.default_rng(11).standard_normal(m.n_core)
    m.precond_factor(J, 1.0)
    x64 = m.precond_solve(b)
    m.set_krylov_precision("fp32_factors")
    m.precond_factor(J, 1.0)
    x32 = m.precond_solve(b)
    rel = np.abs(x32 - x64).max() / np.abs(x64).max()
    assert 0.0 < rel < 1e-5, rel


@pytest.mark.parametrize("precision,step_slack", [("fp32_factors", 0.15), ("fp32", 0.5)])
def test_mixed_precision_adsorption_stays_within_solver_tolerance(precision, step_slack):
    """Free-running 200 s adsorption of the 4x4x16 bed with gpu.krylov_precision = fp32_factors /
    fp32: the end state matches the FP64 run within the solver's own error scale (atol + rtol |y|);
    the Newton tolerance judges every stage.  The step count stays within 15 % with FP32 factors;
    the FP32 operator (an inexact Newton with the step start's Jacobian, in FP32) needs up to 50 %
    more steps (measured 128 against 97)."""
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d, m, cfg, meta = _c0_model(TVSAModel)
    dur = meta["duration"]
    r64 = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur).integrate(d["s0_y0"], dur, [dur])
    over = json.loads(str(d["over"]))
    over["gpu.krylov_precision"] = precision
    d2, m2, cfg2, _ = _c0_model(TVSAModel)
    cfg32 = load_config(override_dict=over)
    integ = TRBDF2(m2, cfg32, h_max=cfg32.solver.h_max_fraction * dur)
    r32 = integ.integrate(d["s0_y0"], dur, [dur])
    sc = m.atol + cfg.solver.rtol * np.abs(r64.y)
    err = np.sqrt(np.mean(((r32.y - r64.y) / sc) ** 2))
    assert err < 1.0, err
    assert abs(r32.n_steps - r64.n_steps) <= max(5, step_slack * r64.n_steps), (r32.n_steps, r64.n_steps)


_GRAPH_FORM_RUN = r"""
import hashlib, json, sys
import numpy as np
sys.path.insert(0, {tests!r})
from cases import golden
from test_gpu_solver import _c0_model
from dac_vtsa_b200.model import TVSAModel
from dac_vtsa_b200.solver import TRBDF2
d, m, cfg, meta = _c0_model(TVSAModel)
dur = meta["duration"]
integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * dur)
r = integ.integrate(d["s0_y0"], dur, [dur])
print(json.dumps({{"y": hashlib.sha256(np.ascontiguousarray(r.y).tobytes()).hexdigest(), "steps": r.n_steps,
                  "gmres": integ.stats["gmres_iters"], "polish": integ.stats["gmres_polish"]}}))
"""


def test_gmres_graph_forms_give_identical_results():
    """The GMRES graph's Arnoldi steps ahead of its WHILE node (DVTSA_GMRES_PREFIX), its steps per
    WHILE pass (DVTSA_GMRES_BODY), its programmatic dependent launches (DVTSA_PDL), its FD matvec
    (DVTSA_MATVEC_COOP) and its CGS2 as one cooperative launch each (DVTSA_GMRES_COOP) change
    where the same kernels' arithmetic runs, not the arithmetic: a 200 s adsorption of the 4x4x16 bed
    ends in the bit-identical state with the same step and GMRES counts in every form."""
    import os
    import subprocess
    import sys
    tests = os.path.dirname(os.path.abspath(__file__))
    code = _GRAPH_FORM_RUN.format(tests=tests)
    out = {}
    for name, env in {"default": {}, "three_kernel_cgs": {"DVTSA_GMRES_COOP": "0"},
                      "no_prefix": {"DVTSA_GMRES_PREFIX": "0"}, "one_step_body": {"DVTSA_GMRES_BODY": "1"},
                      "pdl": {"DVTSA_PDL": "1"}, "coop_matvec": {"DVTSA_MATVEC_COOP": "1"}}.items():
        e = dict(os.environ, **env)
        r = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, timeout=600,
                           cwd=os.path.dirname(tests))
        assert r.returncode == 0, r.stderr[-2000:]
        out[name] = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["default"] == out["three_kernel_cgs"] == out["no_prefix"] == out["one_step_body"] == out["pdl"] == out["coop_matvec"], out
