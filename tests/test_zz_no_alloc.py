"""dv_rhs_acc_noalloc: the residual + accumulators without a model handle and without allocation.

That entry point serves callers that may not allocate device memory once they run (a controller
or estimator with memory reserved at start-up, a host framework whose allocator owns the device),
so they cannot create a dv_model.  Its face/wall records live in one static device array per
device, shared by every call.  The tests call it through the C ABI on consecutive steps and states
and check every call against the reference's own residual (golden fixtures) and against dv_rhs of
a model built for the same step: a call must not see the previous call's records.  Device memory
is the same before and after a series of calls, and the documented limit holds: a 16x16x64 bed
with a wall fits the static array, a larger grid is rejected.

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


def _rel_blocks(a, b, ncell):
    """Worst relative error over the variable blocks (each scaled by its own largest entry)."""
    edges = list(range(0, 6 * ncell + 1, ncell)) + ([len(b)] if len(b) > 6 * ncell else [])
    return max(_rel(a[i:j], b[i:j]) for i, j in zip(edges, edges[1:]))


def _cases():
    # heating (vacuum end, jacket, wall), then a wall-less column (its wall records are never
    # written, so stale ones from the first call would show), then adsorption (feed + vent ends)
    want = ("step2", "no_wall", "step0")
    out = {m["name"]: (m, d) for m, d in rhs_cases() if m["name"] in want}
    return [out[w] for w in want]


class _Call:
    """Inputs of one dv_rhs_acc_noalloc call, prepared (and allocated) before the calls run."""

    def __init__(self, model, t, y, T_jacket_prev=None):
        import torch
        from dac_vtsa_b200.params import build_params
        self.params, feed_h, nnom_h, cov_h, _ = build_params(model.cfg, model.grid, model.props, model.step,
                                                             model.P_start, T_jacket_prev)
        put = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(model.device)
        self.feed, self.nnom, self.cov, self.y = put(feed_h), put(nnom_h), put(cov_h), put(y)
        self.t = t
        self.f = torch.full_like(self.y, np.nan)
        self.acc = torch.full((36,), np.nan, dtype=torch.float64, device=model.device)

    def run(self, lib, stream):
        return lib.dv_rhs_acc_noalloc(C.byref(self.params), self.feed.data_ptr(), self.nnom.data_ptr(),
                                      self.cov.data_ptr(), self.t, self.y.data_ptr(), self.f.data_ptr(),
                                      self.acc.data_ptr(), stream)


def test_noalloc_matches_reference_and_dv_rhs_on_consecutive_calls():
    import torch
    from dac_vtsa_b200 import _lib
    from dac_vtsa_b200.model import TVSAModel
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    calls = []
    for meta, d in _cases():
        m, _ = build(TVSAModel, meta["over"], meta["step"], d["P0"], meta.get("T_jacket_prev"))
        f_model, acc_model = m.rhs(meta["t"], d["y"])
        calls.append((meta, d, m.grid.ncell, f_model, acc_model, _Call(m, meta["t"], d["y"], meta.get("T_jacket_prev"))))
    torch.cuda.synchronize()
    # the first call on the device looks up the static array's address (set-up); after it, a series
    # of calls leaves the device's free memory and the framework allocator's use exactly as they were
    assert calls[0][-1].run(lib, stream) == 0, lib.dv_last_error()
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    for rep in range(2):                                   # every case twice, in a row
        for meta, d, ncell, f_model, acc_model, call in calls:
            call.f.fill_(np.nan)
            call.acc.fill_(np.nan)
            assert call.run(lib, stream) == 0, lib.dv_last_error()
            torch.cuda.synchronize()
            fh, ah = call.f.cpu().numpy(), call.acc.cpu().numpy()
            assert _rel_blocks(fh, d["f"], ncell) <= TOL, (meta["name"], rep, _rel_blocks(fh, d["f"], ncell))
            assert _rel(ah, d["acc"]) <= TOL, (meta["name"], rep, _rel(ah, d["acc"]))
            assert _rel_blocks(fh, f_model, ncell) <= TOL, (meta["name"], rep)
            assert _rel(ah, acc_model) <= TOL, (meta["name"], rep)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_takes_a_16x16x64_bed_with_a_wall():
    """The documented limit: the face and wall records of a 16x16x64 bed with a wall fit the static
    array; the call succeeds and matches dv_rhs of a model of that bed."""
    import torch
    from dac_vtsa_b200 import _lib, host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.model import TVSAModel
    lib = _lib.load()
    cfg = load_config(override_dict={"grid.Nr": 16, "grid.Ntheta": 16, "grid.Nz": 64})
    g = host.Grid.from_config(cfg)
    props = host.get_backend(cfg)
    st = host.seeded_state(cfg, g, props, seed=4, amplitude=0.05)
    m = TVSAModel(cfg, g, props, cfg.cycle[2], st)
    y = m.pack(st)
    f_model, acc_model = m.rhs(7.0, y)
    call = _Call(m, 7.0, y)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert call.run(lib, stream) == 0, lib.dv_last_error()
    torch.cuda.synchronize()
    assert _rel_blocks(call.f.cpu().numpy(), f_model, g.ncell) <= TOL
    assert _rel(call.acc.cpu().numpy(), acc_model) <= TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    from dac_vtsa_b200 import _lib
    lib = _lib.load()
    p = _lib.DvStepParams()
    p.Nr, p.Nth, p.Nz, p.wall_on = 64, 64, 64, 1
    rc = lib.dv_rhs_acc_noalloc(C.byref(p), 8, 8, 8, 0.0, 8, 8, 8, None)
    assert rc == _lib.DV_ERR_ARG
    assert b"scratch" in lib.dv_last_error()
