"""The evaluation's stream layouts give the same results: with the terms overlapping, FS3,
FS2 and the reciprocal-space branch run on their own streams and add their forces into a
separate block; with `overlap` off everything runs in order on one stream.  Also a term mask
that forks the reciprocal branch without the induction (k-space Ewald + FS3) equals the sum
of its terms run one at a time, and FS3 blocks of one triple each (no reuse of a molecule
pair's tables between triples) give the results of the default runs of several triples."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Context, Model, _lib, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

ENERGIES = ("scpe", "rcpe", "kcpe", "indpe", "fs2pe", "fs3pe", "vir")


@pytest.fixture(scope="module")
def box(product):
    m = Model(data_dir("fs2fs3"))
    return m, water_box(m, 128, 15.64, 77, ld=28)


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device=torch.device("cuda:0"))


def _zeros(shape):
    import torch
    return torch.zeros(shape, dtype=torch.float64, device=torch.device("cuda:0"))


def _run(m, b, terms, overlap, **opts):
    nm, ld = b.xs.shape
    args = [_dev(a) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
    f = [_zeros((nm, ld)) for _ in range(3)]
    c2 = [_zeros(nm) for _ in range(3)]
    c3 = [_zeros(nm) for _ in range(3)]
    mu = [_zeros((nm, ld)) for _ in range(3)]
    with Context(m, nm, b.box) as c:
        c.set_option("overlap", overlap)
        for k, v in opts.items():
            c.set_option(k, v)
        e = c.terms_device(terms, *args, b.box, *f, *c2, *c3, *mu)
    fn = lambda ts: np.stack([t.cpu().numpy() for t in ts])
    return e, fn(f), fn(c2), fn(c3), fn(mu)


def test_overlap_matches_in_order(box):
    m, b = box
    e1, f1, c21, c31, mu1 = _run(m, b, _lib.TERM_HOT, 1)
    e0, f0, c20, c30, mu0 = _run(m, b, _lib.TERM_HOT, 0)
    for k in ENERGIES:
        assert e1[k] == pytest.approx(e0[k], rel=1e-12), k
    assert e1["ind_iters"] == e0["ind_iters"]
    assert rel(f1, f0) <= 1e-12
    assert rel(c21, c20) <= 1e-12
    assert rel(c31, c30) <= 1e-12
    assert rel(mu1, mu0) <= 1e-12


def test_kspace_with_fs3_equals_separate_terms(box):
    m, b = box
    eb, fb, _, c3b, _ = _run(m, b, _lib.TERM_KSPACE | _lib.TERM_FS3, 1)
    ek, fk, _, _, _ = _run(m, b, _lib.TERM_KSPACE, 1)
    e3, f3, _, c33, _ = _run(m, b, _lib.TERM_FS3, 1)
    assert eb["kcpe"] == pytest.approx(ek["kcpe"], rel=1e-12)
    assert eb["fs3pe"] == pytest.approx(e3["fs3pe"], rel=1e-12)
    assert rel(fb, fk + f3) <= 1e-12
    assert rel(c3b, c33) <= 1e-12


@pytest.mark.parametrize("precision,fp32_passes", [("fp64", 0), ("mixed", 0), ("mixed", 1)])
def test_fs3_table_reuse_matches_single_triple_blocks(box, precision, fp32_passes):
    m, b = box
    nm, ld = b.xs.shape
    out = []
    for tpb in (8, 1):
        args = [_dev(a) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
        f = [_zeros((nm, ld)) for _ in range(3)]
        c3 = [_zeros(nm) for _ in range(3)]
        with Context(m, nm, b.box, precision=precision) as c:
            c.set_option("fs3_triples_per_block", tpb)
            c.set_option("fs3_fp32_passes", fp32_passes)
            e = c.terms_device(_lib.TERM_FS3, *args, b.box, *f, None, None, None, *c3)
        out.append((e, np.stack([t.cpu().numpy() for t in f]), np.stack([t.cpu().numpy() for t in c3])))
    (e8, f8, c8), (e1, f1, c1) = out
    assert e8["fs3pe"] == pytest.approx(e1["fs3pe"], rel=1e-12)
    assert e8["vir"] == pytest.approx(e1["vir"], rel=1e-12)
    assert rel(f8, f1) <= 1e-12
    assert rel(c8, c1) <= 1e-12


@pytest.mark.parametrize("sum_sites", [32, 7])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_row_form_matches_factor_tables(box, precision, sum_sites):
    """Without the full phase matrix the dipole step runs in its row form (the reciprocal sums
    regrouped by k-vector rows) or on the factor tables: the same step to rounding, with the
    same iteration count.  A chunk of 7 sites leaves ragged chunks and tiles."""
    m, b = box
    nm, ld = b.xs.shape
    out = []
    for rows in (1, 0):
        args = [_dev(a) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
        f = [_zeros((nm, ld)) for _ in range(3)]
        mu = [_zeros((nm, ld)) for _ in range(3)]
        with Context(m, nm, b.box, precision=precision) as c:
            c.set_option("phase_matrix_full", 0)
            c.set_option("dipole_row_form", rows)
            c.set_option("dipole_sum_sites", sum_sites)
            e = c.terms_device(_lib.TERM_HOT, *args, b.box, *f, None, None, None, None, None,
                               None, *mu)
            assert c.get_option("phase_matrix_full_active") == 0
            assert c.get_option("dipole_row_form_active") == rows
        out.append((e, np.stack([t.cpu().numpy() for t in f]),
                    np.stack([t.cpu().numpy() for t in mu])))
    (e1, f1, m1), (e0, f0, m0) = out
    assert e1["ind_iters"] == e0["ind_iters"]
    for k in ENERGIES:
        assert e1[k] == pytest.approx(e0[k], rel=1e-12), k
    assert rel(f1, f0) <= 1e-12
    assert rel(m1, m0) <= 1e-12


@pytest.mark.parametrize("opt,values", [("pdl", (1, 0)), ("fs3_high_priority", (1, 0)),
                                        ("graph_loop", (1, 0)), ("phase_matrix_full", (1, 0)),
                                        ("dipole_row_form", (1, 0)),
                                        ("dipole_gather_sites", (4, 3)),
                                        ("dipole_gather_sites", (4, 8)),
                                        ("dipole_sum_sites", (32, 100))])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_launch_options_give_the_same_results(box, opt, values, precision):
    """Programmatic dependent launch of the dipole steps, FS3's stream priority, the graph
    against the host-driven loop, the full phase matrix against the row form of the dipole
    step, and the dipole step's block shapes change how the work is done, not what it
    computes.  (This box's phase matrix fits in L2, so `dipole_row_form` alone changes
    nothing here; the row form's own test turns the matrix off.)"""
    m, b = box
    nm, ld = b.xs.shape
    out = []
    for v in values:
        args = [_dev(a) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
        f = [_zeros((nm, ld)) for _ in range(3)]
        mu = [_zeros((nm, ld)) for _ in range(3)]
        with Context(m, nm, b.box, precision=precision) as c:
            c.set_option(opt, v)
            assert c.get_option(opt) == v
            e = c.terms_device(_lib.TERM_HOT, *args, b.box, *f, None, None, None, None, None,
                               None, *mu)
            if opt == "phase_matrix_full":  # this box's matrix fits in L2: the option decides
                assert c.get_option("phase_matrix_full_active") == v
        out.append((e, np.stack([t.cpu().numpy() for t in f]),
                    np.stack([t.cpu().numpy() for t in mu])))
    (e1, f1, m1), (e0, f0, m0) = out
    assert e1["ind_iters"] == e0["ind_iters"]
    for k in ENERGIES:
        assert e1[k] == pytest.approx(e0[k], rel=1e-12), k
    assert rel(f1, f0) <= 1e-12
    assert rel(m1, m0) <= 1e-12
