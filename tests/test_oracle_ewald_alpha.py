"""A check of the oracle's Ewald machinery that needs no reference numbers: the total of an
Ewald-summed quantity does not depend on the splitting parameter alpha once the real-space
and reciprocal sums have converged.  Each part (intramolecular/self correction, real space,
reciprocal space) changes by orders of magnitude more than the bar between the two alphas,
so a wrong prefactor, sign, k-vector weight or missing image in any part of
ewald.f90:45-1173 or of the induction fields (nb_induction_model.f90:128-2829, which split
the charge and dipole fields the same way) would show.  The box is 37 waters FS2+FS3 at
L = 10.37 A; alpha is large enough that erfc(alpha L/2) is negligible under the minimum
image, and k-max follows from exp(-k^2/4 alpha^2)."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

SPLITS = [(1.35, 26), (1.65, 31)]  # (alpha / A^-1, k-max per axis)


@pytest.fixture(scope="module")
def box37(oracle):
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    inp = oracle.read_inputs(data_dir("fs2fs3"))
    return b, inp


def _model(O, inp, b, alpha, kmax):
    M = O.make_model(inp, b.nm, b.box)
    M.alpha = alpha
    M.kmax1 = M.kmax2 = M.kmax3 = kmax
    return M


def test_coulomb_total_is_independent_of_alpha(oracle, box37):
    O = oracle
    b, inp = box37
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    tot, parts = [], []
    for alpha, kmax in SPLITS:
        M = _model(O, inp, b, alpha, kmax)
        st = O.State(b.nm, b.xs.shape[1])
        es = O.ewald_self_correction(M, alpha, b.box, *args, st)
        er = O.rspace_ewald(M, *args, b.box, alpha, st)
        ek = O.kspace_ewald(M, *args, kmax, kmax, kmax, alpha, b.box, st)
        tot.append(es + er + ek)
        parts.append((es, er, ek))
    # the parts move by far more than the bar
    assert max(abs(a - c) for a, c in zip(*parts)) > 1e6 * 1e-9 * abs(tot[0])
    # measured: 7e-10 kcal/mol apart on a total of -11.4 (parts of several thousand)
    assert abs(tot[0] - tot[1]) <= 1e-9 * abs(tot[0]), (tot, parts)


def test_induction_energy_is_independent_of_alpha(oracle, box37):
    O = oracle
    b, inp = box37
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    out = []
    for alpha, kmax in SPLITS:
        M = _model(O, inp, b, alpha, kmax)
        st = O.State(b.nm, b.xs.shape[1])
        e, status, _ = O.nb_induction(M, *args, b.box, st)
        assert status == 0
        out.append((e, np.stack([st.idmx, st.idmy, st.idmz])))
    (e1, mu1), (e2, mu2) = out
    # measured: 1e-15 relative apart, the same Jacobi iteration count
    assert abs(e1 - e2) <= 1e-12 * abs(e1), (e1, e2)
    assert np.linalg.norm(mu1 - mu2) <= 1e-10 * np.linalg.norm(mu1)
