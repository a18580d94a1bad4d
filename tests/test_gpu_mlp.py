"""The learned predictor's tensor-core kernels against the network oracle, and its training loop.

Forward and backward run as BF16 products on the tcgen05 tensor cores with FP32 accumulation; the
oracle (oracle/mlp.py) rounds to BF16 at the same points and sums in float64, so the two agree to
FP32 summation order plus the occasional BF16 rounding flip that it causes (tolerances below)."""
import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _net(seed=3):
    from dac_vtsa_b200.predictor import NewtonPredictor
    net = NewtonPredictor(sample_capacity=0, seed=seed)
    P = om.init_params(seed=seed + 2, scale_out=1.0)
    nrm = np.zeros(32)
    nrm[:20] = [0.02, 0.5, 40, 1, 5, 1e7, 2e-3, 5e-2, 4, 0.1, 0.5, 1e6, 10, 1, 1, 1, 1, 1, 1, 8]
    net.set_params(P, nrm)
    return net, P


def _inputs(rows, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((rows, om.NIN)).astype(np.float32)
    X[:, 97:] = 0.0
    T = rng.standard_normal((rows, 8)).astype(np.float32)
    return X, T


@pytest.mark.parametrize("rows", [128, 300, 1000])
def test_forward_matches_oracle(rows):
    net, P = _net()
    X, _ = _inputs(rows, rows)
    out = net.forward(X)
    ref, _ = om.forward(P, X)
    assert out.shape == (rows, om.NOUT)
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err < 2e-2, err


def test_parameters_round_trip():
    net, P = _net()
    P2, nrm = net.params()
    assert np.array_equal(P2, P)
    assert nrm[12] == 10.0


@pytest.mark.parametrize("rows", [700, 4096])
def test_gradient_matches_oracle(rows):
    """Every parameter block of the backward kernels' gradient against the oracle's (BF16-rounded
    back-propagation), and the loss."""
    net, P = _net()
    X, T = _inputs(rows, 7 + rows)
    g, L = net.gradient(X, T)
    go, Lo = om.gradient(P, X, T)
    assert L == pytest.approx(Lo, rel=2e-3)
    o = 0
    for name, shape in om.SIZES:
        n = int(np.prod(shape))
        a, b = g[o:o + n].astype(np.float64), go[o:o + n]
        o += n
        if name == "b4":
            b = b.copy()
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 2e-2, (name, rel)


def test_training_reduces_the_loss_on_recorded_stage_solutions():
    """Samples recorded from the plain solver's own stage solutions (4x4x16 adsorption, every cell of
    every converged stage), then Adam on the GPU: the batch loss falls well below its starting value
    (the untrained network predicts no correction)."""
    import json
    import torch
    from cases import golden, build
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.predictor import NewtonPredictor
    from dac_vtsa_b200.solver import TRBDF2
    d = golden("trajectory_c0.npz")
    over = json.loads(str(d["over"]))
    meta = json.loads(str(d["s0_meta"]))
    m, cfg = build(TVSAModel, over, meta["step"], d["s0_P0"], meta["T_jacket_prev"], duration=meta["duration"])
    net = NewtonPredictor(sample_capacity=1 << 16, seed=1)
    integ = TRBDF2(m, cfg, h_max=cfg.solver.h_max_fraction * meta["duration"])
    net.attach(integ, "adsorption", predict=False, record_stride=1)
    res = integ.integrate(d["s0_y0"], meta["duration"], [meta["duration"]])
    assert res.t == pytest.approx(meta["duration"])
    assert net.samples >= 4096, net.samples
    hist = net.train(300, lr=2e-3, seed=5)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(hist))
    first, last = float(np.mean(hist[:10])), float(np.mean(hist[-20:]))
    assert last < 0.5 * first, (first, last)
