"""The regroupings the reciprocal kernels rely on, checked in numpy on a k-vector list built the
way the library builds it (half space, spherical cut-off, n innermost: ewald.f90:933-1082).

- The row form of the dipole step (k_iter_a_rows / k_iter_b_rows): the structure factors
  S(k) = sum_s (k.mu_s) XY(s, l, m) Z(s, n), regrouped as sum_s Z(s, n) (B + k_n C) per row of
  the list, and the gather sum_k k Re[XY Z conj F(k)], regrouped as sums over the n of a row
  followed by one contraction with XY, equal the per-(site, k) sums to rounding.
- The gathers' per-k-vector weights (k_kgather): the mode factor times the sums, staged once
  per k-vector, give the weight of every (site, k) pair that the reference's expressions give
  (nb_induction_model.f90:4171-4839 for the induction forces)."""
import numpy as np
import pytest


def kvec_list(lmax, mmax, nmax, box):
    """(l, m, n, k_l, k_m, k_n, a) in the library's order, with a random weight a."""
    rng = np.random.default_rng(3)
    klm = min(lmax, mmax, nmax)
    out, mmin, nmin = [], 0, 1
    for ll in range(lmax + 1):
        if ll > 0:
            mmin = -mmax
        for mm in range(mmin, mmax + 1):
            for nn in range(nmin, nmax + 1):
                if ll * ll + mm * mm + nn * nn <= klm * klm:
                    tw = 2.0 * np.pi
                    out.append((ll, mm, nn, tw * ll / box, tw * mm / box, tw * nn / box,
                                rng.uniform(0.1, 1.0)))
            nmin = -nmax
    return out


def rows_of(kv):
    """[(k_l, k_m, kbeg, len, nlo, l, m)] by decreasing length, ties in list order."""
    rows = []
    for k, K in enumerate(kv):
        if k > 0 and K[0] == kv[k - 1][0] and K[1] == kv[k - 1][1]:
            rows[-1][3] += 1
            continue
        rows.append([K[3], K[4], k, 1, K[2], K[0], K[1]])
    return sorted(rows, key=lambda r: -r[3])


@pytest.fixture(scope="module")
def system():
    rng = np.random.default_rng(11)
    lmax = mmax = nmax = 6
    kv = kvec_list(lmax, mmax, nmax, 13.0)
    nw = 23
    XY = {(l, m): np.exp(1j * rng.uniform(0, 2 * np.pi, nw)) for l in range(lmax + 1)
          for m in range(-mmax, mmax + 1)}
    Z = {n: np.exp(1j * rng.uniform(0, 2 * np.pi, nw)) for n in range(-nmax, nmax + 1)}
    mu = rng.normal(size=(nw, 3))
    return kv, rows_of(kv), XY, Z, mu


def test_rows_cover_the_list_once(system):
    kv, rows, _, _, _ = system
    seen = np.zeros(len(kv), int)
    for rl, rm, kbeg, ln, nlo, l, m in rows:
        for j in range(ln):
            K = kv[kbeg + j]
            assert (K[0], K[1], K[2]) == (l, m, nlo + j)
            seen[kbeg + j] += 1
    assert (seen == 1).all()
    lens = [r[3] for r in rows]
    assert lens == sorted(lens, reverse=True)


def test_structure_factors_by_rows(system):
    kv, rows, XY, Z, mu = system
    direct = np.array([np.sum((K[3] * mu[:, 0] + K[4] * mu[:, 1] + K[5] * mu[:, 2])
                              * XY[K[0], K[1]] * Z[K[2]]) for K in kv])
    by_rows = np.zeros(len(kv), complex)
    for rl, rm, kbeg, ln, nlo, l, m in rows:
        B = XY[l, m] * (rl * mu[:, 0] + rm * mu[:, 1])
        C = XY[l, m] * mu[:, 2]
        for j in range(ln):
            by_rows[kbeg + j] = np.sum(Z[nlo + j] * (B + kv[kbeg + j][5] * C))
    assert np.abs(by_rows - direct).max() <= 1e-13 * np.abs(direct).max()


def test_gather_by_rows(system):
    kv, rows, XY, Z, mu = system
    rng = np.random.default_rng(5)
    F = rng.normal(size=len(kv)) + 1j * rng.normal(size=len(kv))
    direct = np.zeros((len(mu), 3))
    for k, K in enumerate(kv):
        t = (XY[K[0], K[1]] * Z[K[2]] * np.conj(F[k])).real
        direct += np.outer(t, K[3:6])
    by_rows = np.zeros_like(direct)
    for rl, rm, kbeg, ln, nlo, l, m in rows:
        Q = sum(Z[nlo + j] * np.conj(F[kbeg + j]) for j in range(ln))
        Qz = sum(kv[kbeg + j][5] * Z[nlo + j] * np.conj(F[kbeg + j]) for j in range(ln))
        a = (XY[l, m] * Q).real
        by_rows[:, 0] += rl * a
        by_rows[:, 1] += rm * a
        by_rows[:, 2] += (XY[l, m] * Qz).real
    assert np.abs(by_rows - direct).max() <= 1e-12 * np.abs(direct).max()


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_folded_gather_weights(mode):
    """g of a (site, k) pair from the staged weights W against the reference's expression."""
    rng = np.random.default_rng(mode)
    r4pie0 = 332.0637  # any constant: it only scales mode 0
    for _ in range(200):
        ak, c, s, q = rng.uniform(-2, 2, 4)
        S = rng.uniform(-2, 2, 4)
        mk = rng.uniform(-2, 2)
        if mode == 0:
            ref = 4.0 * r4pie0 * ak * ((q * s) * S[0] - (q * c) * S[1])
            f = 4.0 * r4pie0 * ak
            W = (f * S[0], -f * S[1])
            got = q * (s * W[0] + c * W[1])
        elif mode == 1:
            ref = 4.0 * ak * (s * S[0] - c * S[1])
            f = 4.0 * ak
            W = (f * S[0], -f * S[1])
            got = s * W[0] + c * W[1]
        elif mode == 2:
            ref = -4.0 * ak * (c * S[0] + s * S[1])
            f = -4.0 * ak
            W = (f * S[0], f * S[1])
            got = c * W[0] + s * W[1]
        else:
            mufac = -4.0 * ak * (c * S[2] + s * S[3])
            qfac = -4.0 * ak * (-c * S[0] - s * S[1])
            mufaci = -4.0 * ak * (c * S[3] - s * S[2])
            ref = q * mufac + mk * (qfac + mufaci)
            f = -4.0 * ak
            W = (f * S[2], f * S[3], f * (S[3] - S[0]), -f * (S[1] + S[2]))
            got = q * (c * W[0] + s * W[1]) + mk * (c * W[2] + s * W[3])
        assert got == pytest.approx(ref, rel=1e-12, abs=1e-12)
