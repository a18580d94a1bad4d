"""C ABI: the library loads and exports every entry point of include/dacvtsa.h; struct layouts
agree; the host-side colouring is bit-identical to the reference's (no GPU needed)."""
import hashlib
import json
import os
import re

import numpy as np

from cases import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "dacvtsa.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    from dac_vtsa_b200 import _lib
    lib = _lib.load()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert {n for n, _, _ in _lib.SIGNATURES} == set(names)
    assert lib.dv_abi_version() == 1
    assert lib.dv_step_params_size() == ctypes.sizeof(_lib.DvStepParams)
    for cname, mirror in _lib.STRUCT_MIRRORS.items():
        assert lib.dv_struct_size(cname.encode()) == ctypes.sizeof(mirror), cname
    assert lib.dv_struct_size(b"no_such_struct") == 0


def test_colouring_bit_identical_to_reference():
    from dac_vtsa_b200 import _lib
    d = golden("colouring.npz")
    for key in d.files:
        if key.startswith("full_"):
            dims = tuple(int(x) for x in key[5:].split("x"))
            c, nc = _lib.colour_columns(*dims)
            assert np.array_equal(c, d[key].astype(np.int64)), dims
            assert nc == int(d[key].max()) + 1
    hashes = json.loads(str(d["hashes"]))
    for dims in ("8x8x32", "16x16x64", "4x8x16", "16x4x64"):
        c, nc = _lib.colour_columns(*(int(x) for x in dims.split("x")))
        assert [hashlib.sha256(c.tobytes()).hexdigest(), nc] == hashes[dims]


def test_block_pattern_equals_reference_pattern():
    from dac_vtsa_b200.jacobian import block_pattern
    from oracle.sparsity import pattern
    for dims in [(3, 4, 6), (2, 1, 4), (1, 1, 30), (4, 3, 5), (3, 4, 2), (3, 4, 1)]:
        for wall in (True, False):
            _, rows, indptr, _ = block_pattern(*dims, wall)
            P = pattern(*dims, 3, 2, wall).tocsc()
            assert np.array_equal(P.indptr, indptr) and np.array_equal(P.indices, rows)


def test_params_struct_builds_for_every_case():
    from cases import rhs_cases
    from dac_vtsa_b200 import host
    from dac_vtsa_b200.config import load_config
    from dac_vtsa_b200.params import build_params
    for meta, data in rhs_cases():
        cfg = load_config(override_dict=meta["over"])
        g = host.Grid.from_config(cfg)
        P0 = data["P0"]
        ps = {"top": float(np.mean(P0[:, :, 0])), "bottom": float(np.mean(P0[:, :, -1]))}
        p, feed, nnom, cov, _ = build_params(cfg, g, host.get_backend(cfg), cfg.cycle[meta["step"]], ps)
        assert p.Nr == g.Nr and feed.shape == (g.Nr, g.Nth) and cov.shape == (g.Nth, g.Nz)
