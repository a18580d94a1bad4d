"""What the trained network gains, on an operating point it was not trained on (the held-out 33rd
point of the seeded draw; 8x8x32 bed, full cycle).  The packaged weights
(dac_vtsa_b200/predictor_weights.npz) were trained on the GPU by
``python -m dac_vtsa_b200.train_predictor --grid 8 8 32 --points 32 --steps 10000`` from 1.1 million
cell-stage samples of plain cycles at the other 32 points."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _held_out():
    from dac_vtsa_b200.train_predictor import operating_points, setup
    return setup((8, 8, 32), operating_points(33, 2024)[-1])


def test_network_starts_closer_to_the_stage_solutions():
    """Every sampled cell of every converged stage of the held-out cycle: the network's corrected start
    is closer to the stage solution than the extrapolated start, in RMS over the samples of each of
    the six cell unknowns (units of the cell's extrapolated increment, the units the network is
    trained in)."""
    from dac_vtsa_b200.predictor import NewtonPredictor, default_network
    from dac_vtsa_b200.runner import run_cycle_device
    import torch
    cfg, g, props, y0 = _held_out()
    rec = NewtonPredictor(sample_capacity=400000)
    run_cycle_device(y0, cfg, g, props, predictor=rec, predict=False, record_stride=13)
    torch.cuda.synchronize()
    X, T = rec.get_samples()
    assert len(X) > 100000
    net = default_network()
    P, nrm = net.params()
    O = np.concatenate([net.forward(X[i:i + 65536]) for i in range(0, len(X), 65536)])
    err = T[:, :6] - O[:, :6] * nrm[13:19]
    rms = lambda a: float(np.sqrt(np.mean(np.asarray(a, dtype=np.float64) ** 2)))
    ratios = [rms(err[:, v]) / rms(T[:, v]) for v in range(6)]
    assert max(ratios) < 1.0, ratios                        # closer for every unknown
    assert float(np.exp(np.mean(np.log(ratios)))) < 0.9, ratios   # by 10 % or more on (geometric) average


def test_cycle_with_the_network_reaches_the_plain_states():
    """The held-out cycle with the network: the unchanged Newton tolerance judges every start, so the
    step-end state equals the plain method's within the solver's error scale; the Newton work stays
    within 10 % of the plain method's (the measured gain of this network on this solver is about
    zero: a stage takes two to three Newton iterations from either start, because convergence is
    declared on a step of at most 1 % of the error scale)."""
    from dac_vtsa_b200.predictor import default_network
    from dac_vtsa_b200.train_predictor import cycle_stats, timed_cycle
    cfg, g, props, y0 = _held_out()
    yp, sp, _ = timed_cycle(cfg, g, props, y0)
    yn, sn, _ = timed_cycle(cfg, g, props, y0, predictor=default_network())
    a, b = yp.cpu().numpy(), yn.cpu().numpy()
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200 import host
    st = host.seeded_state(cfg, g, props, seed=0)
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    scaled = np.abs(b - a) / (m.atol + cfg.solver.rtol * np.abs(a))
    assert np.sqrt(np.mean(scaled ** 2)) < 1.0
    p, n = cycle_stats(sp), cycle_stats(sn)
    assert n["pred_net"] > 0
    assert n["newton_iters"] <= 1.1 * p["newton_iters"], (p, n)
