"""Batches of independent frames (ccp_batch_*): frame-by-frame equality with the single-frame
entry point, the batched torch.autograd binding, and error reporting of a failing frame."""
import ctypes as C

import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Batch, CcpError, Context, Model, data_dir, _lib
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

NM, NF, BOX = 37, 5, 10.37


@pytest.fixture(scope="module")
def frames(product):
    import torch
    m = Model(data_dir("fs2fs3"))
    boxes = [water_box(m, NM, BOX, 100 + f, ld=30) for f in range(NF)]
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    x, y, z = (T(np.stack([getattr(b, k) for b in boxes])) for k in ("x", "y", "z"))
    xs, ys, zs = (T(np.stack([getattr(b, k) for b in boxes])) for k in ("xs", "ys", "zs"))
    return m, boxes, (x, y, z, xs, ys, zs)


def _single(m, b, terms, args1):
    import torch
    x, y, z, xs, ys, zs = args1
    out = [torch.zeros_like(xs) for _ in range(3)] + [torch.zeros_like(x) for _ in range(6)]
    with Context(m, NM, BOX) as c:
        e = c.terms_device(terms, x, y, z, xs, ys, zs, b.box, *out)
    return e, [t.cpu().numpy() for t in out]


@pytest.mark.parametrize("slots", [1, 3])
def test_batch_equals_single_frames(frames, slots):
    import torch
    m, boxes, (x, y, z, xs, ys, zs) = frames
    terms = _lib.TERM_ALL
    out = [torch.zeros_like(xs) for _ in range(3)] + [torch.zeros_like(x) for _ in range(6)]
    with Batch(m, NM, BOX, slots=slots) as bt:
        es = bt.terms_device(terms, [b.box for b in boxes], x, y, z, xs, ys, zs, *out)
    got = [t.cpu().numpy() for t in out]
    for f, b in enumerate(boxes):
        e1, o1 = _single(m, b, terms, (x[f], y[f], z[f], xs[f], ys[f], zs[f]))
        for k in ("scpe", "rcpe", "kcpe", "indpe", "fs2pe", "fs3pe", "vdwpe", "vir"):
            assert es[f][k] == pytest.approx(e1[k], rel=1e-12, abs=1e-12), (f, k)
        assert es[f]["ind_iters"] == e1["ind_iters"]
        for a, g in zip(o1, got):
            assert rel(g[f], a) <= 1e-12


def test_batched_autograd(frames):
    """Batched energies and gradients against the single-frame binding, with a different
    weight on every frame's energy."""
    import torch
    from ccpol23_plus_2025_mbmd_b200.autograd import fs3_param_tensors, three_body_induction_energy
    m, boxes, (x, y, z, xs, ys, zs) = frames
    com = torch.stack([x, y, z], dim=-1)
    sites = torch.stack([xs, ys, zs], dim=-1)
    w = torch.tensor([1.0, -0.5, 2.0, 0.25, 1.5][:NF], dtype=torch.float64, device=x.device)
    with Batch(m, NM, BOX, slots=2) as bt:
        p = fs3_param_tensors(bt, x.device)
        c, s = com.clone().requires_grad_(True), sites.clone().requires_grad_(True)
        E = three_body_induction_energy(bt, BOX, c, s, *p)
        assert E.shape == (NF,)
        (w * E).sum().backward()
    with Context(m, NM, BOX) as ctx:
        p1 = fs3_param_tensors(ctx, x.device)
        gp = [torch.zeros_like(q) for q in p1]
        for f in range(NF):
            c1, s1 = com[f].clone().requires_grad_(True), sites[f].clone().requires_grad_(True)
            q = [t.detach().clone().requires_grad_(True) for t in p1]
            E1 = three_body_induction_energy(ctx, BOX, c1, s1, *q)
            assert E[f].item() == pytest.approx(E1.item(), rel=1e-12)
            (w[f] * E1).backward()
            assert rel(c.grad[f].cpu().numpy(), c1.grad.cpu().numpy()) <= 1e-12
            assert rel(s.grad[f].cpu().numpy(), s1.grad.cpu().numpy()) <= 1e-12
            for a, t in zip(gp, q):
                a += t.grad
    for a, t in zip(gp, p):
        assert rel(t.grad.cpu().numpy(), a.cpu().numpy()) <= 1e-10


def test_batch_reports_failing_frame(frames):
    import torch
    m, boxes, (x, y, z, xs, ys, zs) = frames
    with Batch(m, NM, BOX, slots=2) as bt:
        h = C.c_void_p()
        assert _lib.lib().ccp_batch_context(bt._h, 1, C.byref(h)) == 0
        assert _lib.lib().ccp_context_set_maxit(h, 2) == 0   # slot 1 runs frames 1 and 3
        with pytest.raises(CcpError) as e:
            bt.terms_device(_lib.TERM_HOT, [b.box for b in boxes], x, y, z, xs, ys, zs)
        assert e.value.code == 2 and "frame 1" in str(e.value)
        assert _lib.lib().ccp_context_set_maxit(h, 500) == 0
        es = bt.terms_device(_lib.TERM_HOT, [b.box for b in boxes], x, y, z, xs, ys, zs)
        assert all(e["ind_iters"] > 2 for e in es)
