"""torch.ops.dacvtsa.* registrations (CPU: schemas and fake-tensor shapes; GPU: the same numbers as
the C-ABI calls the Python classes make)."""
import numpy as np
import pytest
import torch

from dac_vtsa_b200 import ops  # noqa: F401  (registers the operators)


def test_operators_are_registered():
    names = {n for n in dir(torch.ops.dacvtsa) if not n.startswith("_")}
    assert {"rhs", "stage_residual", "fd_jacobian", "precond_factor", "newton_stage", "step"} <= names


def test_fake_tensors_give_shapes_without_a_gpu():
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode(allow_non_fake_inputs=True):
        y = torch.empty(1600, dtype=torch.float64, device="cuda")
        R = torch.ops.dacvtsa.stage_residual(0, 1.0, y, 0.5, y)
        f, acc = torch.ops.dacvtsa.rhs(0, 1.0, y)
        z, info = torch.ops.dacvtsa.newton_stage(0, 1.0, y, y, 0.1, 7, 0.01, 1e-4, 1e-3, 2)
    assert R.shape == y.shape and f.shape == y.shape and acc.shape == (36,)
    assert z.shape == y.shape and info.shape == (6,)


@pytest.mark.gpu
def test_operators_match_the_model_methods():
    from cases import build, rhs_cases
    from dac_vtsa_b200.model import TVSAModel
    m_meta, arrs = next(iter(rhs_cases()))
    m, cfg = build(TVSAModel, m_meta["over"], m_meta["step"], arrs["P0"])
    y = torch.from_numpy(arrs["y"]).cuda()
    t = m_meta["t"]
    f_op, acc_op = torch.ops.dacvtsa.rhs(m.handle.value, t, y)
    f_m, acc_m = m.rhs(t, y)
    assert torch.equal(f_op, f_m) and torch.equal(acc_op, acc_m)
    R_op = torch.ops.dacvtsa.stage_residual(m.handle.value, t, y, 0.3, y)
    assert torch.equal(R_op, m.stage_residual(t, y, 0.3, y))
    J_op = torch.ops.dacvtsa.fd_jacobian(m.handle.value, t, y, f_m)
    from dac_vtsa_b200.jacobian import FDJacobian
    assert torch.equal(J_op, FDJacobian(m).block(t, y, f_m))
