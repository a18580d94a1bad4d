"""GPU coloured FD Jacobian (all colours in one launch) vs the reference's FDJacobian values."""
import numpy as np
import pytest

from cases import build, golden

pytestmark = pytest.mark.gpu


def test_fd_jacobian_matches_reference():
    from dac_vtsa_b200.jacobian import FDJacobian
    from dac_vtsa_b200.model import TVSAModel
    d = golden("jacobian_3x4x6.npz")
    m, _ = build(TVSAModel, {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}, 0, d["P0"])
    jac = FDJacobian(m)
    J = jac(float(d["t"]), d["y"])
    assert np.array_equal(J.indptr, d["indptr"]) and np.array_equal(J.indices, d["indices"])
    ref = d["data"]
    # compare column by column relative to the column's largest entry: the forward difference
    # amplifies ulp-level residual differences by 1/h (h = 1.5e-8 max(|y|, typ)).
    col = np.repeat(np.arange(J.shape[1]), np.diff(J.indptr))
    colmax = np.zeros(J.shape[1])
    np.maximum.at(colmax, col, np.abs(ref))
    err = np.abs(J.data - ref) / np.maximum(colmax[col], 1e-300)
    assert err.max() <= 1e-6, err.max()


def test_jacobian_matches_dense_fd_and_colouring_is_valid():
    """Reference test (tests/test_physics_and_numerics.py:118-138) on the GPU: 12 random columns of the
    coloured Jacobian vs one-column-at-a-time differences of the GPU residual, 1e-3 relative."""
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.jacobian import FDJacobian
    from dac_vtsa_b200.model import TVSAModel
    cfg = load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.initial_state(cfg, g, props)
    st.T = st.T + np.random.default_rng(0).random(st.T.shape)
    m = TVSAModel(cfg, g, props, cfg.cycle[0], st)
    y = m.pack(st)
    jac = FDJacobian(m)
    J = jac(5.0, y).toarray()
    f0, _ = m.rhs(5.0, y, want_acc=False)
    for j in np.random.default_rng(2).choice(len(y), 12, replace=False):
        h = 1e-7 * max(abs(y[j]), 1e-3)
        yp = y.copy()
        yp[j] += h
        col_fd = (m.rhs(5.0, yp, want_acc=False)[0] - f0) / h
        scale = max(np.abs(col_fd).max(), 1e-12)
        assert np.abs(col_fd - J[:, j]).max() / scale < 1e-3
    Pr = jac.P.tocsr()
    for r in range(Pr.shape[0]):
        cc = jac.color[Pr.indices[Pr.indptr[r]:Pr.indptr[r + 1]]]
        assert len(np.unique(cc)) == len(cc)
