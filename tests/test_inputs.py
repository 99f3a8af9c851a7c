"""Host-side logic on CPU: the product's C++ readers against the oracle's independent
Python readers, the FS3 coefficient index, Ewald set-up and site placement."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import CcpError, Model, data_dir, ewald_setup
from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, config_box, water_box


@pytest.mark.parametrize("variant", ["fs3", "fs2fs3"])
def test_readers_agree(product, oracle, variant):
    m = Model(data_dir(variant))
    inp = oracle.read_inputs(data_dir(variant))
    assert m.ns == inp.ns == 28 and m.npol == inp.npol == 3
    assert np.array_equal(m.charge, inp.charge)
    assert np.array_equal(m.polarizability, inp.polarizability)
    pc, pmi, totm = oracle.principal_frame(inp)
    assert np.array_equal(m.pcoord, pc)
    assert np.array_equal(m.pmi, pmi)
    assert m.get_double("totm") == totm
    c = inp.control
    assert m.get_int("S2_term") == c["S2_term"] and m.get_int("S3_term") == c["S3_term"]
    assert m.get_double("rcut") == c["rcut"] and m.get_double("alpha3") == c["alpha3"]
    assert m.get_double("rcut3") == c["rcut3"] and m.get_double("delta33") == c["delta33"]
    # P1..P3 sit exactly on O, H, H (the reference's dist2 == 0 skips rely on it)
    assert np.array_equal(m.pcoord[25:28], m.pcoord[0:3])


def test_fs3_index_has_364_classes(product, oracle):
    ind, n = oracle.fill_index()
    m = Model(data_dir("fs3"))
    assert n == 364 == m.get_int("nclass") == m.get_int("nlin")
    assert np.array_equal(m.array("ind_lin", ind.size), ind.astype(float))
    # symmetric under the six permutations of (site, power) pairs
    T = ind.reshape(17, 17, 17, 2, 2, 2)  # [i, j, k, ip, jp, kp]
    assert np.array_equal(T, T.transpose(1, 0, 2, 4, 3, 5))
    assert np.array_equal(T, T.transpose(2, 1, 0, 5, 4, 3))


def test_type_coefficients_match_index(product, oracle):
    m = Model(data_dir("fs2fs3"))
    inp = oracle.read_inputs(data_dir("fs2fs3"))
    ind, _ = oracle.fill_index()
    coef = m.array("coef_sr", 6 * 6 * 6 * 8).reshape(6, 6, 6, 8)
    types = [0, 1, 1, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5]
    T = ind.reshape(17, 17, 17, 2, 2, 2)
    rng = np.random.default_rng(0)
    for _ in range(500):
        i, j, k = rng.integers(0, 17, 3)
        ip, jp, kp = rng.integers(0, 2, 3)
        assert coef[types[i], types[j], types[k], ip * 4 + jp * 2 + kp] == \
            inp.fs3_sr["cs"][T[i, j, k, ip, jp, kp] - 1]


@pytest.mark.parametrize("box,kmax", [(15.64, 6), (19.71, 7), (24.84, 9), (39.40, 14)])
def test_ewald_setup(product, oracle, box, kmax):
    a, k1, k2, k3 = ewald_setup(1e-6, 9.0, box)
    assert (k1, k2, k3) == (kmax, kmax, kmax)
    assert abs(a - 0.358185) < 1e-6
    assert (a, k1, k2, k3) == oracle.ewald_setup(9.0, box)


def test_sites_match_oracle(product, oracle):
    m = Model(data_dir("fs3"))
    b = water_box(m, 20, 8.5, 5, ld=50)
    pc = oracle.principal_frame(oracle.read_inputs(data_dir("fs3")))[0]
    xs, ys, zs = oracle.sites(pc, b.q, 50)
    assert np.array_equal(xs, b.xs) and np.array_equal(ys, b.ys) and np.array_equal(zs, b.zs)


def test_generator_is_seeded_and_sane(product):
    m = Model(data_dir("fs3"))
    b1 = config_box("c1_128", m)
    b2 = config_box("c1_128", m)
    assert np.array_equal(b1.x, b2.x) and np.array_equal(b1.q, b2.q)
    assert b1.nm == 128 and np.allclose(np.linalg.norm(b1.q, axis=1), 1.0)
    L = b1.box
    o = np.stack([b1.x + b1.xs[:, 0], b1.y + b1.ys[:, 0], b1.z + b1.zs[:, 0]], 1)
    d = o[:, None, :] - o[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1)) + np.eye(128) * 10
    assert r.min() >= 2.5
    assert np.all(np.abs(b1.x) <= L / 2 + 1e-12)


def test_bad_inputs_raise(product, tmp_path):
    with pytest.raises(CcpError) as e:
        Model(tmp_path)
    assert e.value.code == 5  # CCP_ERR_IO
    (tmp_path / "CONTROL").write_text((data_dir("fs3") / "CONTROL").read_text())
    (tmp_path / "FIELD").write_text("broken\n1\n")
    with pytest.raises(CcpError):
        Model(tmp_path)
