"""dv_rhs_acc_noalloc: the residual + accumulators without a model handle and without allocation.

That entry point serves callers that may not allocate device memory once they run (a controller
or estimator with memory reserved at start-up, a host framework whose allocator owns the device),
so they cannot create a dv_model.  Its face/wall records live in one static device array per
device, shared by every call.  The test calls it through the C ABI twice in a row, on two
different steps and states (three calls), and checks every call against dv_rhs of a model built for the same
step: the second call must not see the first call's records.

The file is named to be collected last, so a failure here does not hide the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from tests.cases import build, rhs_cases

pytestmark = pytest.mark.gpu

TOL = 1e-11          # the residual tests' per-block relative tolerance


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _cases():
    # heating (vacuum end, jacket, wall), then a wall-less column (its wall records are never
    # written, so stale ones from the first call would show), then adsorption (feed + vent ends)
    want = ("step2", "no_wall", "step0")
    out = {m["name"]: (m, d) for m, d in rhs_cases() if m["name"] in want}
    return [out[w] for w in want]


def test_noalloc_matches_dv_rhs_on_consecutive_calls():
    import torch
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200.model import TVSAModel
    from dac_vtsa_b200.params import build_params
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for meta, d in _cases():
        m, _ = build(TVSAModel, meta["over"], meta["step"], d["P0"], meta.get("T_jacket_prev"))
        t = meta["t"]
        f_ref, acc_ref = m.rhs(t, d["y"])
        params, feed_h, nnom_h, cov_h, _ = build_params(m.cfg, m.grid, m.props, m.step, m.P_start,
                                                        meta.get("T_jacket_prev"))
        dev = m.device

        def put(a):
            return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        feed, nnom, cov, y = put(feed_h), put(nnom_h), put(cov_h), put(d["y"])
        f = torch.full_like(y, np.nan)
        acc = torch.full((_lib.DV_NACC,), np.nan, dtype=torch.float64, device=dev)
        rc = lib.dv_rhs_acc_noalloc(C.byref(params), feed.data_ptr(), nnom.data_ptr(), cov.data_ptr(), t,
                                    y.data_ptr(), f.data_ptr(), acc.data_ptr(), stream)
        assert rc == 0, lib.dv_last_error()
        torch.cuda.synchronize()
        fh, ah = f.cpu().numpy(), acc.cpu().numpy()
        assert _rel(fh, f_ref) <= TOL, (meta["name"], _rel(fh, f_ref))
        assert _rel(ah, acc_ref) <= TOL, (meta["name"], _rel(ah, acc_ref))


def test_noalloc_rejects_grids_beyond_its_scratch():
    from dac_vtsa_b200 import _lib
    lib = _lib.load()
    p = _lib.DvStepParams()
    p.Nr, p.Nth, p.Nz, p.wall_on = 64, 64, 64, 1
    rc = lib.dv_rhs_acc_noalloc(C.byref(p), 8, 8, 8, 0.0, 8, 8, 8, None)
    assert rc == _lib.DV_ERR_ARG
    assert b"scratch" in lib.dv_last_error()
