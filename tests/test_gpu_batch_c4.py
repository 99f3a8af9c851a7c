"""The differentiation batch at its own size: 32 frames of 256 waters (FS3 variant,
L = 19.71 A, seeds 4004 + f), the three-body plus induction terms.  FS3 runs fused over the
batch (one neighbour search, one triple list and one FS3 launch for every frame); energies,
forces, COM forces, dipoles and the parameter gradients must equal the single-frame calls
and the unfused batch to round-off."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Batch, Context, Model, data_dir, _lib
from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, water_box

from conftest import rel

pytestmark = pytest.mark.gpu

NF = 32
TERMS = _lib.TERM_INDUCTION | _lib.TERM_FS3 | _lib.TERM_FS2


@pytest.fixture(scope="module")
def c4(product):
    import torch
    cfg = CONFIGS["c4_256"]
    m = Model(data_dir(cfg["variant"]))
    boxes = [water_box(m, cfg["nm"], cfg["box"], cfg["seed"] + f) for f in range(NF)]
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    args = [T(np.stack([getattr(b, k) for b in boxes])) for k in ("x", "y", "z", "xs", "ys", "zs")]
    return m, cfg, boxes, args


def _outputs(args):
    import torch
    x, xs = args[0], args[3]
    return ([torch.zeros_like(xs) for _ in range(3)] + [torch.zeros_like(x) for _ in range(6)] +
            [torch.zeros_like(xs) for _ in range(3)])


def _batch(m, cfg, args, fuse, slots=8, pgrad=None):
    out = _outputs(args)
    with Batch(m, cfg["nm"], cfg["box"], slots=slots) as bt:
        bt.set_option("fuse_fs3", fuse)
        if pgrad is not None:
            bt.set_option("fs3_param_grad", 1)
        es = bt.terms_device(TERMS, [cfg["box"]] * NF, *args, *out, pgrad=pgrad)
    return es, [t.cpu().numpy() for t in out]


def test_fused_batch_equals_single_frames(c4):
    m, cfg, boxes, args = c4
    es, got = _batch(m, cfg, args, 1)
    with Context(m, cfg["nm"], cfg["box"]) as c:
        for f in range(NF):
            a1 = [a[f] for a in args]
            o1 = [t[f].clone().zero_() for t in _outputs(args)]
            e1 = c.terms_device(TERMS, *a1, cfg["box"], *o1)
            for k in ("indpe", "fs2pe", "fs3pe", "vir"):
                assert es[f][k] == pytest.approx(e1[k], rel=1e-12, abs=1e-12), (f, k)
            for k in ("ind_iters", "n_fs3_triples", "n_fs3_blend"):
                assert es[f][k] == e1[k], (f, k)
            for g, a in zip(got, o1):
                assert rel(g[f], a.cpu().numpy()) <= 1e-12, f


def test_fused_and_unfused_batches_agree(c4):
    m, cfg, boxes, args = c4
    ncoef = m.get_int("nclass")
    pg = [np.zeros((NF, 2 * ncoef + 2 * 3 * 289)) for _ in range(2)]
    e1, o1 = _batch(m, cfg, args, 1, pgrad=pg[0])
    e0, o0 = _batch(m, cfg, args, 0, pgrad=pg[1])
    for f in range(NF):
        for k in ("indpe", "fs3pe", "vir"):
            assert e1[f][k] == pytest.approx(e0[f][k], rel=1e-12, abs=1e-12), (f, k)
    for a, b in zip(o1, o0):
        assert rel(a, b) <= 1e-12
    assert rel(pg[0], pg[1]) <= 1e-11
    assert np.abs(pg[0]).max() > 0
