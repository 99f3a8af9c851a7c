"""The 2048-water oracle fixture (tests/golden/c5_2048) belongs to the box the generator makes
now: its input fingerprint matches (CPU only)."""
import sys
from pathlib import Path

import numpy as np

from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, water_box

GOLDEN = Path(__file__).parent / "golden" / "c5_2048"


def test_fixture_inputs_match_the_generator(product):
    sys.path.insert(0, str(GOLDEN))
    from make_fixture import STRIDE, fingerprint
    g = np.load(GOLDEN / "oracle_hot_path.npz")
    cfg = CONFIGS["c5_2048"]
    b = water_box(Model(data_dir(cfg["variant"])), cfg["nm"], cfg["box"], cfg["seed"])
    assert np.allclose(fingerprint(b), g["fingerprint"], rtol=1e-12, atol=0.0)
    assert list(g["sel"]) == list(range(0, cfg["nm"], STRIDE))
    assert g["site_forces"].shape == (3, len(g["sel"]), b.xs.shape[1])
    assert int(g["ind_iters"]) > 0
