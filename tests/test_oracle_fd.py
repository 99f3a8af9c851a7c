"""Self-validation of the oracle for the terms the reference ships no numbers for (the 2-body
CCpol23+ term, FS3, Ewald, induction): central finite differences of each term's energy against its analytic
COM forces, torques and rigid-scaling virial, the same identities the reference's
validators use (initialization.f90:1093-1491, source/tests/check_fs2_periodic.py:72-84)."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

TERMS = ["vdw", "self", "rspace", "kspace", "induction", "fs2", "fs3"]


def run_term(O, M, term, x, y, z, xs, ys, zs, box):
    st = O.State(len(x), xs.shape[1])
    if term == "vdw":
        e = O.ccpol23plus(M, x, y, z, xs, ys, zs, box, st)
    elif term == "self":
        e = O.ewald_self_correction(M, M.alpha, box, x, y, z, xs, ys, zs, st)
    elif term == "rspace":
        e = O.rspace_ewald(M, x, y, z, xs, ys, zs, box, M.alpha, st)
    elif term == "kspace":
        e = O.kspace_ewald(M, x, y, z, xs, ys, zs, M.kmax1, M.kmax2, M.kmax3, M.alpha, box, st)
    elif term == "induction":
        e, status, _ = O.nb_induction(M, x, y, z, xs, ys, zs, box, st)
        assert status == 0
    else:
        M.s2_term, M.s3_term = int(term == "fs2"), int(term == "fs3")
        e2, e3 = O.threebody_term(M, x, y, z, xs, ys, zs, box, st)
        e = e2 if term == "fs2" else e3
    fcom = np.stack([st.fxs.sum(1), st.fys.sum(1), st.fzs.sum(1)], 1)
    fcom += np.stack([st.fxfs2, st.fyfs2, st.fzfs2], 1) if term == "fs2" else 0.0
    fcom += np.stack([st.fxfs3, st.fyfs3, st.fzfs3], 1) if term == "fs3" else 0.0
    tq = np.stack([(ys * st.fzs - zs * st.fys).sum(1), (zs * st.fxs - xs * st.fzs).sum(1),
                   (xs * st.fys - ys * st.fxs).sum(1)], 1)
    vsite = np.sum(st.fxs * xs + st.fys * ys + st.fzs * zs)
    return e, fcom / 418.4, tq / 418.4, (st.vir.value + vsite) / 418.4


def rotate(xs, ys, zs, i, axis, ang):
    c, s = np.cos(ang), np.sin(ang)
    xs, ys, zs = xs.copy(), ys.copy(), zs.copy()
    p = [xs, ys, zs]
    a, b = [(1, 2), (2, 0), (0, 1)][axis]
    pa, pb = p[a][i].copy(), p[b][i].copy()
    p[a][i] = c * pa - s * pb
    p[b][i] = s * pa + c * pb
    return xs, ys, zs


@pytest.fixture(scope="module")
def small(oracle):
    m = Model(data_dir("fs2fs3"))
    inp = oracle.read_inputs(data_dir("fs2fs3"))
    nm, box = 14, 7.6
    b = water_box(m, nm, box, 11)
    M = oracle.make_model(inp, nm, box)
    return M, b


@pytest.mark.parametrize("term", TERMS)
def test_oracle_term_derivatives(oracle, small, term):
    O = oracle
    M, b = small
    x, y, z, xs, ys, zs, box = b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box
    e0, f, tq, vir = run_term(O, M, term, x, y, z, xs, ys, zs, box)
    assert np.isfinite(e0) and e0 != 0.0
    h = 1e-5
    scale = max(1.0, np.abs(f).max())
    for i in (0, 7):
        for a in range(3):
            X = [x.copy(), y.copy(), z.copy()]
            X[a][i] += h
            ep = run_term(O, M, term, *X, xs, ys, zs, box)[0]
            X[a][i] -= 2 * h
            em = run_term(O, M, term, *X, xs, ys, zs, box)[0]
            assert abs(-(ep - em) / (2 * h) - f[i, a]) < 1e-6 * scale, (term, i, a)
            ep = run_term(O, M, term, x, y, z, *rotate(xs, ys, zs, i, a, h), box)[0]
            em = run_term(O, M, term, x, y, z, *rotate(xs, ys, zs, i, a, -h), box)[0]
            assert abs(-(ep - em) / (2 * h) - tq[i, a]) < 1e-6 * max(1.0, np.abs(tq).max()), (term, i, a)
    # rigid scaling of COMs and box: dE/de = vir/418.4 + sum f_s . s / 418.4
    if term != "kspace" or True:
        ep = run_term(O, M, term, x * (1 + h), y * (1 + h), z * (1 + h), xs, ys, zs, box * (1 + h))[0]
        em = run_term(O, M, term, x * (1 - h), y * (1 - h), z * (1 - h), xs, ys, zs, box * (1 - h))[0]
        assert abs((ep - em) / (2 * h) - vir) < 1e-6 * max(1.0, abs(vir)), (term, vir)


def test_oracle_fs3_covers_all_branches(oracle):
    """The FS3 switch: SR below 4.5 A, blend in (4.5, 5.5), LR above 5.5; the blended energy
    is continuous in R_avg (C1 of the switch) - checked through the FD test on a box whose
    triples populate all three branches."""
    m = Model(data_dir("fs3"))
    b = water_box(m, 24, 9.0, 3)
    L = b.box
    com = np.stack([b.x, b.y, b.z], 1)
    nb = {"sr": 0, "blend": 0, "lr": 0}
    for i in range(24):
        for j in range(i + 1, 24):
            for k in range(j + 1, 24):
                d = []
                xij = com[i] - com[j]; xij -= L * np.round(xij / L)
                xik = com[i] - com[k]; xik -= L * np.round(xik / L)
                xjk = xik - xij
                r = [np.linalg.norm(v) for v in (xij, xik, xjk)]
                if max(r) < 6.3:
                    ra = sum(r) / 3
                    nb["sr" if ra <= 4.5 else ("lr" if ra >= 5.5 else "blend")] += 1
    assert all(v > 0 for v in nb.values()), nb
