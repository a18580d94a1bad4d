"""Failure detection on the GPU without a fault: the library's bounded device waits run against
events that never happen, give up, record the error word and return; the context stays usable."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_waits_time_out_and_report():
    from dac_vtsa_b200 import _lib
    lib = _lib.load()
    bits = C.c_int32(-1)
    rc = lib.dv_selftest_wait_timeout(1000, C.byref(bits))
    assert rc == 0, lib.dv_last_error()
    assert bits.value == 5, bits.value          # 1: the sweep's copy wait, 4: the grid barrier


def test_context_usable_after_timeouts():
    from cases import build, golden
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200.model import TVSAModel
    lib = _lib.load()
    bits = C.c_int32(0)
    assert lib.dv_selftest_wait_timeout(200, C.byref(bits)) == 0
    d = golden("jacobian_3x4x6.npz")
    m, _ = build(TVSAModel, {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}, 0, d["P0"])
    f, _ = m.rhs(5.0, d["y"], want_acc=False)
    assert np.all(np.isfinite(f))


def test_model_recovers_after_a_reported_timeout():
    """A wait that gave up (injected on the host into the model's error word) is reported once as a
    CUDA-class error naming the wait; the next integration on the same model runs normally."""
    import ctypes as C
    from cases import build, golden
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200._lib import LibraryError
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.solver import TRBDF2
    d = golden("jacobian_3x4x6.npz")
    m, cfg = build(TVSAModel, {"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6}, 0, d["P0"], duration=2.0)
    lib = _lib.load()
    assert lib.dv_model_flag_wait_timeout(m.handle, 4) == 0
    with pytest.raises(LibraryError, match="grid barrier"):
        TRBDF2(m, cfg, h_max=0.5).integrate(d["y"], 2.0, [2.0])
    res = TRBDF2(m, cfg, h_max=0.5).integrate(d["y"], 2.0, [2.0])
    assert res.t == pytest.approx(2.0) and np.all(np.isfinite(res.y))
