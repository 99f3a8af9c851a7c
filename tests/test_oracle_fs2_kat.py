"""Pins the oracle's FS2 restatement with the reference's own FS2 test, run the way the
reference runs it: FS2_term called directly on bohr coordinates of the fixture with the
test's globals (nm=3, ns=5, alpha3=6.51292, rcutsd3=6.1^2, delta33=10)."""
import numpy as np
import pytest

from fs2_kat import run, site_offsets


def test_oracle_fs2_known_answer(oracle):
    O = oracle
    M = O.OrcModel()
    M.nm, M.ns, M.npol = 3, 5, 0
    M.alpha3, M.rcutsd3, M.delta33 = 6.51292, 6.1 ** 2, 10.0
    M.s2_term, M.s3_term = 1, 0
    s = site_offsets()

    def calc(r, box):
        st = O.State(3, 5)
        e = O.fs2_term_bohr(M, r[0], r[1], r[2], s[0], s[1], s[2], box, st)
        return (e, st.vir.value, st.fxs, st.fys, st.fzs, st.fxfs2, st.fyfs2, st.fzfs2)

    log = run(calc)
    assert all(ok for *_, ok in log)
    # the fixture is not trivial: FS2 is non-zero for every geometry
    assert abs(calc(np.array([[0.0, 5.5, 2.0], [0.0, 0.3, 5.0], [0.0, 0.2, 0.7]]), 40.0)[0]) > 1e-4
