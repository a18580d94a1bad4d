"""Partition maps of the preconditioner (host code of the library, no GPU): for every partition mode
and grid, each unknown of the state belongs to exactly one (partition, plane, local index), every
index lies inside the state, and the inverse map of cells and wall nodes agrees.  Covers the split
form large cross-sections take (ring groups per sector, theta groups of the core ring)."""
import ctypes as C

import pytest

from dac_vtsa_b200 import _lib, host
from dac_vtsa_b200.config import load_config
from dac_vtsa_b200.params import build_params

# grid -> (partitions, largest block) of theta_block (mode 2, split when too large)
EXPECT = {(8, 8, 32): (9, 48), (16, 16, 64): (34, 48), (11, 4, 9): (9, 31), (3, 10, 12): (12, 30),
          (4, 4, 16): (5, 24), (8, 16, 64): (18, 48), (16, 4, 32): (9, 48), (4, 16, 16): (18, 48)}


@pytest.mark.parametrize("grid", sorted(EXPECT))
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_partition_maps_are_a_bijection(grid, mode):
    lib = _lib.load()
    cfg = load_config(override_dict={"grid.Nr": grid[0], "grid.Ntheta": grid[1], "grid.Nz": grid[2]})
    g = host.Grid.from_config(cfg)
    p = build_params(cfg, g, host.get_backend(cfg), cfg.cycle[0], {"top": 1e5, "bottom": 1e5})[0]
    nparts, nb, bad = C.c_int32(), C.c_int32(), C.c_int64()
    assert lib.dv_precond_check_maps(C.byref(p), mode, C.byref(nparts), C.byref(nb), C.byref(bad)) == 0
    assert bad.value == 0
    if mode == 2:
        assert (nparts.value, nb.value) == EXPECT[grid]


def test_wall_free_bed():
    lib = _lib.load()
    cfg = load_config(override_dict={"grid.Nr": 12, "grid.Ntheta": 12, "grid.Nz": 10, "wall.enabled": False})
    g = host.Grid.from_config(cfg)
    p = build_params(cfg, g, host.get_backend(cfg), cfg.cycle[0], {"top": 1e5, "bottom": 1e5})[0]
    for mode in (0, 1, 2):
        nparts, nb, bad = C.c_int32(), C.c_int32(), C.c_int64()
        assert lib.dv_precond_check_maps(C.byref(p), mode, C.byref(nparts), C.byref(nb), C.byref(bad)) == 0
        assert bad.value == 0
