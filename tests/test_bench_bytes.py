"""The bench's algorithmic-bytes rule of the sweep: partitions as the solver builds them."""
from types import SimpleNamespace

import bench
from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config


def _model(over):
    cfg = load_config(override_dict=over)
    g = host.Grid.from_config(cfg)
    nw = g.Nth * g.Nz if cfg.wall.enabled else 0
    return SimpleNamespace(grid=g, cfg=cfg, n_w=nw, n_core=6 * g.ncell + nw, jac_doubles=0)


def test_partition_sizes_follow_the_solver():
    m = _model({"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32})
    assert bench.partition_sizes(m) == [43] * 8 + [48]                 # theta_block: ring 0 of all sectors apart
    m = _model({"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32, "solver.precond_theta_rings": 0})
    assert bench.partition_sizes(m) == [49] * 8                        # whole sectors
    m = _model({"grid.Nr": 4, "grid.Ntheta": 1, "grid.Nz": 8})
    assert bench.partition_sizes(m) == [6 * 4 + 1]                     # one sector: the full cross-section


def test_sweep_bytes_of_the_benchmark_bed():
    m = _model({"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32})
    blocks = 32 * 5 * (8 * 43 * 43 + 48 * 48) * 8
    assert bench.alg_bytes_per_launch("precond_apply", m) == blocks + 3 * m.n_core * 8 == 22183936
