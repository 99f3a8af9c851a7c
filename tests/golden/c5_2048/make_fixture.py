"""Generates oracle_hot_path.npz: the oracle's FP64 hot path (oracle/oracle.py hot_path) on
the 2048-water FS2+FS3 box of the large-box benchmark (L = 39.40 A, seed 5005), so that the
GPU test can check the library at that size without running the oracle (several minutes on
a CPU) on the GPU box.

  python tests/golden/c5_2048/make_fixture.py        # writes oracle_hot_path.npz beside it

Stored: a fingerprint of the generated inputs (so the test detects a changed generator), the
six energies, the virial and the dipole iteration count, the norms of the full site-force,
COM-force and dipole arrays, and the site forces, COM forces and dipoles of every 32nd
molecule.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

STRIDE = 32


def fingerprint(b):
    return np.array([b.x.sum(), b.y.sum(), b.z.sum(), np.abs(b.xs).sum(), np.abs(b.ys).sum(),
                     np.abs(b.zs).sum(), b.x[0], b.y[1], b.z[2]])


def main():
    import oracle as O
    from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
    from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, water_box
    O.build()
    O.set_threads(0)
    cfg = CONFIGS["c5_2048"]
    m = Model(data_dir(cfg["variant"]))
    b = water_box(m, cfg["nm"], cfg["box"], cfg["seed"])
    M = O.make_model(O.read_inputs(data_dir(cfg["variant"])), b.nm, b.box)
    eo, st = O.hot_path(M, b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    assert eo["ind_status"] == 0
    sel = np.arange(0, b.nm, STRIDE)
    F = np.stack([st.fxs, st.fys, st.fzs])
    C2 = np.stack([st.fxfs2, st.fyfs2, st.fzfs2])
    C3 = np.stack([st.fxfs3, st.fyfs3, st.fzfs3])
    D = np.stack([st.idmx, st.idmy, st.idmz])
    keys = ("scpe", "rcpe", "kcpe", "indpe", "fs2pe", "fs3pe", "vir")
    np.savez_compressed(
        HERE / "oracle_hot_path.npz", fingerprint=fingerprint(b),
        energies=np.array([eo[k] for k in keys]), energy_keys=np.array(keys),
        ind_iters=np.array(eo["ind_iters"]), sel=sel,
        norms=np.array([np.linalg.norm(F), np.linalg.norm(C2), np.linalg.norm(C3),
                        np.linalg.norm(D)]),
        site_forces=F[:, sel], com_fs2=C2[:, sel], com_fs3=C3[:, sel], dipoles=D[:, sel])


if __name__ == "__main__":
    main()
