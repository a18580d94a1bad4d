"""The network oracle (oracle/mlp.py) against its own finite differences, and its BF16 rounding.

The learned predictor has no counterpart in the reference, so the oracle that checks its tensor-core
kernels is pinned here: without BF16 rounding its analytic gradient equals a central difference of its
loss in float64."""
import numpy as np

from oracle import mlp as om


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.0e38], dtype=np.float32)
    r = om.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # exactly half an ulp above 1: ties to the even neighbour 1.0
    assert r[2] == np.float32(1.0 + 2 ** -7)  # above the tie: rounds up
    assert r[3] == -2.5 and r[4] == 0.0
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = om.init_params(seed=1, scale_out=1.0).astype(np.float64)
    X = rng.standard_normal((40, om.NIN))
    X[:, 97:] = 0.0
    T = rng.standard_normal((40, 8))
    g, L = om.gradient(P, X, T, rounding=False)
    assert abs(L - om.loss(P, X, T, rounding=False)) < 1e-12
    idx = np.concatenate([rng.choice(om.NPARAM, 60, replace=False), [om.NPARAM - 1, om.NPARAM - 16, 0]])
    eps = 1e-6
    for q in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[q] += eps
        Pm[q] -= eps
        fd = (om.loss(Pp, X, T, rounding=False) - om.loss(Pm, X, T, rounding=False)) / (2 * eps)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (q, fd, g[q])


def test_rounded_gradient_stays_close_to_exact():
    """The BF16-rounded gradient (what the device computes) is within BF16 accuracy of the exact one."""
    rng = np.random.default_rng(2)
    P = om.init_params(seed=3, scale_out=1.0)
    X = rng.standard_normal((256, om.NIN)).astype(np.float32)
    X[:, 97:] = 0.0
    T = rng.standard_normal((256, 8)).astype(np.float32)
    g1, _ = om.gradient(P, X, T, rounding=True)
    g0, _ = om.gradient(P, X, T, rounding=False)
    assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 3e-2
