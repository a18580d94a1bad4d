"""The bench's algorithmic-bytes rules: the sweep streams the 5 blocks of every plane of every
partition the solver factorised (their sizes come from the library), plus 3 state vectors."""
from types import SimpleNamespace

import bench
from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config


def _model(over):
    cfg = load_config(override_dict=over)
    g = host.Grid.from_config(cfg)
    nw = g.Nth * g.Nz if cfg.wall.enabled else 0
    return SimpleNamespace(grid=g, cfg=cfg, n_w=nw, n_core=6 * g.ncell + nw, jac_doubles=9 * 49 * g.ncell)


def test_sweep_bytes_of_the_benchmark_bed():
    m = _model({"grid.Nr": 8, "grid.Ntheta": 8, "grid.Nz": 32})
    nbs = [43] * 8 + [48]                  # theta_block: rings 1.. of each sector (+ wall), ring 0 of all
    blocks = 32 * 5 * (8 * 43 * 43 + 48 * 48) * 8
    assert bench.alg_bytes_per_launch("precond_apply", m, nbs) == blocks + 3 * m.n_core * 8 == 22183936
    assert bench.alg_bytes_per_launch("precond_apply", m, nbs, fp32=True) == blocks // 2 + 3 * m.n_core * 8


def test_operator_bytes():
    m = _model({"grid.Nr": 16, "grid.Ntheta": 16, "grid.Nz": 64})
    assert bench.alg_bytes_per_launch("spmv", m) == 9 * 49 * 16384 * 4 + 3 * m.n_core * 8
    assert bench.alg_bytes_per_launch("matvec", m) == 5 * m.n_core * 8
