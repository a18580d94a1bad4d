"""State hand-off files: the reference's CSV format written byte for byte, read back bit-exactly
(simio/checkpoint.py:27-96 of the reference), including by the background writer."""
import filecmp
import json
import os

import numpy as np
import pytest

from cases import GOLDEN
from dac_vtsa_b200 import host
from dac_vtsa_b200.config import load_config
from dac_vtsa_b200.handoff import load_state_csv, save_state_csv


def _fixture():
    d = np.load(os.path.join(GOLDEN, "state_csv", "seeded_3x4x6.npz"))
    cfg = load_config(override_dict={"grid.Nr": 3, "grid.Ntheta": 4, "grid.Nz": 6})
    g = host.Grid.from_config(cfg)
    meta = json.loads(str(d["meta"]))
    st = host.CycleState(c=d["c"], q=d["q"], T=d["T"], Tw=d["Tw"], t=meta["t"], cycle=meta["cycle"],
                         step=meta["step"])
    return g, st


def test_writer_reproduces_the_reference_files_byte_for_byte(tmp_path):
    g, st = _fixture()
    out = save_state_csv(st, g, str(tmp_path / "s.csv"))
    ref = os.path.join(GOLDEN, "state_csv", "seeded_3x4x6.csv")
    assert filecmp.cmp(out, ref, shallow=False)
    assert filecmp.cmp(out[:-4] + "_wall.csv", ref[:-4] + "_wall.csv", shallow=False)


def test_reading_the_reference_file_is_bit_exact():
    g, st = _fixture()
    back = load_state_csv(os.path.join(GOLDEN, "state_csv", "seeded_3x4x6.csv"), g, st.species, st.adsorbed)
    for k in ("c", "q", "T", "Tw"):
        assert np.array_equal(getattr(back, k), getattr(st, k)), k
    assert back.t == st.t and back.cycle == st.cycle and back.step == st.step


def test_grid_mismatch_is_rejected(tmp_path):
    g, st = _fixture()
    cfg = load_config(override_dict={"grid.Nr": 2, "grid.Ntheta": 4, "grid.Nz": 6})
    with pytest.raises(ValueError, match="cells but the grid has"):
        load_state_csv(os.path.join(GOLDEN, "state_csv", "seeded_3x4x6.csv"), host.Grid.from_config(cfg),
                       st.species, st.adsorbed)
