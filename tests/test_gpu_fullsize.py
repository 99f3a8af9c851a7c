"""Full-size boxes (512 and 2048 waters, the benchmark configurations) checked through
properties that hold at any size, where the CPU oracle would take minutes: the total force
vanishes (the energy is translation invariant), and a rigid translation of every molecule or
a relabelling of the molecules leaves energies, forces, induced dipoles and the Jacobi
iteration count unchanged."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, water_box

from conftest import rel

pytestmark = pytest.mark.gpu

ENERGIES = ("scpe", "rcpe", "kcpe", "indpe", "fs2pe", "fs3pe", "vir")


@pytest.fixture(scope="module", params=["c2_512", "c5_2048"])
def box(request, product):
    cfg = CONFIGS[request.param]
    m = Model(data_dir(cfg["variant"]))
    return m, water_box(m, cfg["nm"], cfg["box"], cfg["seed"])


def _eval(m, b, x, y, z, xs, ys, zs):
    with Context(m, b.nm, b.box) as c:
        return c.hot_path(x, y, z, xs, ys, zs, b.box)


def _forces(r):
    return np.stack([r.fxs, r.fys, r.fzs]), np.stack([r.fxfs2 + r.fxfs3, r.fyfs2 + r.fyfs3,
                                                       r.fzfs2 + r.fzfs3])


def test_total_force_vanishes(box):
    m, b = box
    r = _eval(m, b, b.x, b.y, b.z, b.xs, b.ys, b.zs)
    F, Fc = _forces(r)
    total = F.sum(axis=(1, 2)) + Fc.sum(axis=1)
    assert np.linalg.norm(total) <= 1e-9 * np.linalg.norm(F), total


def test_translation_invariance(box):
    m, b = box
    r0 = _eval(m, b, b.x, b.y, b.z, b.xs, b.ys, b.zs)
    r1 = _eval(m, b, b.x + 1.37, b.y - 0.71, b.z + 2.13, b.xs, b.ys, b.zs)
    for k in ENERGIES:
        assert r1.energies[k] == pytest.approx(r0.energies[k], rel=1e-10), k
    assert r1.energies["ind_iters"] == r0.energies["ind_iters"]
    for a, c in zip(_forces(r1), _forces(r0)):
        assert rel(a, c) <= 1e-9
    assert rel(np.stack([r1.idmx, r1.idmy, r1.idmz]), np.stack([r0.idmx, r0.idmy, r0.idmz])) <= 1e-9


def test_relabelling_invariance(box):
    m, b = box
    perm = np.random.default_rng(7).permutation(b.nm)
    r0 = _eval(m, b, b.x, b.y, b.z, b.xs, b.ys, b.zs)
    r1 = _eval(m, b, *(np.ascontiguousarray(a[perm]) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)))
    for k in ENERGIES:
        assert r1.energies[k] == pytest.approx(r0.energies[k], rel=1e-10), k
    assert r1.energies["ind_iters"] == r0.energies["ind_iters"]
    F0, C0 = _forces(r0)
    F1, C1 = _forces(r1)
    assert rel(F1, F0[:, perm]) <= 1e-9
    assert rel(C1, C0[:, perm]) <= 1e-9


def test_cell_list_matches_all_pairs(product):
    """At 2048 waters the neighbour lists come from the cell-list search; with it switched off
    the all-pairs scan must give the same lists, hence the same triples, pairs, iteration
    count and results (atomic summation order aside)."""
    cfg = CONFIGS["c5_2048"]
    m = Model(data_dir(cfg["variant"]))
    b = water_box(m, cfg["nm"], cfg["box"], cfg["seed"])
    out = {}
    for cells in (1, 0):
        with Context(m, b.nm, b.box) as c:
            c.set_option("cell_list", cells)
            out[cells] = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
            assert c.get_option("cell_list_active") == cells
    e1, e0 = out[1].energies, out[0].energies
    for k in ("ind_iters", "n_fs3_triples", "n_fs3_blend", "n_fs2_triples"):
        assert e1[k] == e0[k], k
    for k in ENERGIES:
        assert e1[k] == pytest.approx(e0[k], rel=1e-12), k
    for a, c in zip(_forces(out[1]), _forces(out[0])):
        assert rel(a, c) <= 1e-12
