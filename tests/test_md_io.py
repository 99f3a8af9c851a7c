"""The MD driver's file formats (REVCON, OUTPUT rows, HISTORY frames) on the host."""
import numpy as np

from ccpol23_plus_2025_mbmd_b200.md import history_frame, output_row, read_revcon, write_revcon


def test_revcon_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    nm = 5
    q = rng.normal(size=(nm, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    st = {"x": rng.normal(size=nm), "y": rng.normal(size=nm), "z": rng.normal(size=nm),
          "v": rng.normal(size=(nm, 3)), "j": rng.normal(size=(nm, 3)), "q": q}
    write_revcon(tmp_path / "REVCON", 12, 0.006, 15.64, st)
    r = read_revcon(tmp_path / "REVCON", nm)
    assert r["step"] == 12 and r["t"] == 0.006 and r["box"] == 15.64
    for k in ("x", "y", "z", "v", "j", "q"):
        assert np.array_equal(r[k], st[k]), k  # %.17g round-trips every double


def test_revcon_reads_fortran_list_directed(tmp_path):
    """A REVCON in the reference's list-directed style (D exponents, free spacing)."""
    body = " Created by Ommair\n           7   3.5000000000000003E-003   15.640000000000001  0.0 0.0\n"
    body += "  1.0D0 2.0 3.0  0.1 0.2 0.3  1.0 2.0 3.0  1.0 0.0 0.0 0.0\n"
    (tmp_path / "REVCON").write_text(body)
    r = read_revcon(tmp_path / "REVCON", 1)
    assert r["step"] == 7 and abs(r["t"] - 0.0035) < 1e-15 and r["x"][0] == 1.0
    assert np.array_equal(r["q"][0], [1.0, 0.0, 0.0, 0.0])


def test_output_row_fortran_layout():
    s = {k: -1234.5678 for k in ("sys_temp", "tke", "rke", "vdwpe", "cpe", "indpe", "pe3b", "pe",
                                 "te", "vir", "pres")}
    row = output_row(3, 0.0015, s, 512, 24.84, 18.01528)
    assert len(row) == 1 + 8 + 15 * 16  # '(1x,i8,1p,15e16.8)'
    assert row[1:9] == "       3" and row[9:25] == "  1.50000000E-03"


def test_history_frame_layout():
    nm = 2
    st = {"x": np.zeros(nm), "y": np.zeros(nm), "z": np.zeros(nm)}
    z = np.zeros((nm, 28))
    dip = [np.ones((nm, 28)) * 0.5 for _ in range(3)]
    fr = history_frame(50, 0.0005, 24.84, ["O", "H", "H", "D1", "D1"], [15.9994, 1.00797, 1.00797, 0, 0],
                       [0.29, 0.56, 0.56, -0.7, -0.7], st, z, z, z, dip).splitlines()
    assert fr[0].startswith("timestep") and len(fr) == 4 + nm * 5 * 3
    assert fr[4][:8] == "O       " and int(fr[4][8:18]) == 1
