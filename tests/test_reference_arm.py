"""The CPU reference arm of bench.py builds its box with the oracle alone: the same arrays,
bit for bit, as the product's route (library model + generator), and nothing of the package
imported or loaded while it does so."""
import json
import subprocess
import sys

import numpy as np

from conftest import ROOT


def test_reference_box_is_bit_identical(product):
    sys.path.insert(0, str(ROOT))
    import bench
    _, _, ref_box, _ = bench.reference_inputs()
    _, box, _ = bench.build_inputs(0)
    for k in ("x", "y", "z", "q", "xs", "ys", "zs", "v", "jb"):
        a, b = getattr(ref_box, k), getattr(box, k)
        assert a.shape == b.shape and np.array_equal(a, b), k
    assert ref_box.box == box.box and ref_box.nm == box.nm


def test_reference_inputs_load_nothing_of_the_package():
    code = (
        "import json, sys\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "import bench\n"
        "O, M, box, cfg = bench.reference_inputs()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'pkg': [m for m in sys.modules if m.startswith('ccpol23_plus')],\n"
        "                  'lib': 'libccpol23_b200' in maps, 'oracle': 'libccpol_oracle' in maps,\n"
        "                  'nm': box.nm}))\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         check=True, timeout=600)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["pkg"] == [] and not r["lib"], r
    assert r["oracle"] and r["nm"] == 512
