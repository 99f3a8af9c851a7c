"""torch.autograd binding of the three-body plus induction energy.

``three_body_induction_energy(context, box, com, sites, cs_sr, cs_lr, bgr_sr, bgr_lr)``
returns E = FS2 + FS3 + induction energy (kcal/mol) of one box, differentiable with respect
to the molecular centres ``com`` (nm, 3), the site offsets ``sites`` (nm, ns, 3) (both in
Angstrom, float64 CUDA tensors, as the reference's x and xs) and the FS3 fit: linear
coefficients ``cs_sr``/``cs_lr`` (nclass each) and site-pair (b, g, r0) ``bgr_sr``/``bgr_lr``
(3, 289), index is*17 + js.

The adjoint is hand-written in the library, not traced:
- positions: the kernels' analytic forces.  The converged induced dipoles make the
  induction energy stationary, so no derivative flows through the Jacobi iterations
  (the reference's own force expressions use the same property);
- FS3 parameters: the FS3 kernel's gradient form accumulates, per triple, the derivative of
  the energy sum with respect to every coefficient-table entry and every site-pair
  (b, g, r0), from the same tabulated pair terms as the energy, with no per-triple storage.

One forward call is one evaluation (energy, forces and, when any FS3 parameter requires a
gradient, the parameter gradient); backward only scales them by the incoming gradient.

Batches: with a ``Batch`` in place of the context, ``com`` (B, nm, 3) and ``sites``
(B, nm, ns, 3) hold B independent frames and the result is the (B,) vector of their
energies.  The frames are evaluated concurrently (``ccp_batch_terms_device``); the
parameter gradient of frame f is kept per frame, so backward weights it by the incoming
gradient of that frame's energy.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

KCAL = 418.4  # internal force unit (10 J/mol/A) per kcal/mol/A
CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream, named explicitly


class _ThreeBodyInduction(torch.autograd.Function):
    @staticmethod
    def forward(fctx, context, box, com, sites, cs_sr, cs_lr, bgr_sr, bgr_lr):
        dev = com.device
        params = [cs_sr, cs_lr, bgr_sr, bgr_lr]
        cur = context.fs3_params()
        new = [p.detach().cpu().numpy().astype(np.float64).reshape(c.shape) for p, c in zip(params, cur)]
        if any(not np.array_equal(a, b) for a, b in zip(new, cur)):
            context.set_fs3_params(*new)
        want_p = any(p.requires_grad for p in params)
        context.set_option("fs3_param_grad", 1 if want_p else 0)
        nm, ns = sites.shape[0], sites.shape[1]
        x, y, z = (com[:, a].contiguous() for a in range(3))
        xs, ys, zs = (sites[:, :, a].contiguous() for a in range(3))
        f = [torch.zeros((nm, ns), dtype=torch.float64, device=dev) for _ in range(3)]
        c2 = [torch.zeros(nm, dtype=torch.float64, device=dev) for _ in range(3)]
        c3 = [torch.zeros(nm, dtype=torch.float64, device=dev) for _ in range(3)]
        terms = _lib.TERM_INDUCTION | _lib.TERM_FS2 | _lib.TERM_FS3
        # The input copies and the zero-filled outputs above are queued on torch's current
        # stream; the evaluation runs on the context's stream.  Queue it on torch's stream for
        # this call so that it starts after them (the call returns once it has finished).
        # torch's default stream has the handle 0, which the library reads as "the context's
        # own stream"; cudaStreamLegacy (1) names that default stream explicitly.
        prev = context.stream
        context.set_stream(torch.cuda.current_stream(dev).cuda_stream or CUDA_STREAM_LEGACY)
        try:
            e = context.terms_device(terms, x, y, z, xs, ys, zs, box, *f, *c2, *c3)
        finally:
            context.set_stream(prev)
        energy = e["fs2pe"] + e["fs3pe"] + e["indpe"]
        F = torch.stack(f, dim=-1)                                     # (nm, ns, 3)
        Fc = torch.stack([c2[a] + c3[a] for a in range(3)], dim=-1)    # (nm, 3)
        g_sites = -F / KCAL
        g_com = -(F.sum(dim=1) + Fc) / KCAL
        if want_p:
            gp = [torch.as_tensor(g, device=p.device, dtype=p.dtype).reshape(p.shape)
                  for g, p in zip(context.fs3_param_grad(), params)]
        else:
            gp = [None] * 4
        fctx.save_for_backward(g_com, g_sites)
        fctx.gp = gp
        return torch.tensor(energy, dtype=torch.float64, device=dev)

    @staticmethod
    def backward(fctx, grad):
        g_com, g_sites = fctx.saved_tensors
        gp = [None if g is None else grad * g for g in fctx.gp]
        return (None, None, grad * g_com, grad * g_sites, *gp)


class _ThreeBodyInductionBatch(torch.autograd.Function):
    @staticmethod
    def forward(fctx, batch, box, com, sites, cs_sr, cs_lr, bgr_sr, bgr_lr):
        dev = com.device
        params = [cs_sr, cs_lr, bgr_sr, bgr_lr]
        cur = batch.fs3_params()
        new = [p.detach().cpu().numpy().astype(np.float64).reshape(c.shape) for p, c in zip(params, cur)]
        if any(not np.array_equal(a, b) for a, b in zip(new, cur)):
            batch.set_fs3_params(*new)
        want_p = any(p.requires_grad for p in params)
        batch.set_option("fs3_param_grad", 1 if want_p else 0)
        nf, nm, ns = sites.shape[0], sites.shape[1], sites.shape[2]
        x, y, z = (com[:, :, a].contiguous() for a in range(3))
        xs, ys, zs = (sites[:, :, :, a].contiguous() for a in range(3))
        f = [torch.zeros((nf, nm, ns), dtype=torch.float64, device=dev) for _ in range(3)]
        c2 = [torch.zeros((nf, nm), dtype=torch.float64, device=dev) for _ in range(3)]
        c3 = [torch.zeros((nf, nm), dtype=torch.float64, device=dev) for _ in range(3)]
        ncoef = cur[0].size
        pg = np.zeros((nf, 2 * ncoef + 2 * 3 * 289)) if want_p else None
        terms = _lib.TERM_INDUCTION | _lib.TERM_FS2 | _lib.TERM_FS3
        # Every slot of the batch runs on its own streams, which do not wait for torch's
        # stream: finish the input copies and the zero fills queued above first (the call
        # returns once every frame has finished).
        torch.cuda.current_stream(dev).synchronize()
        es = batch.terms_device(terms, box, x, y, z, xs, ys, zs, *f, *c2, *c3, pgrad=pg)
        energy = [e["fs2pe"] + e["fs3pe"] + e["indpe"] for e in es]
        F = torch.stack(f, dim=-1)                                     # (nf, nm, ns, 3)
        Fc = torch.stack([c2[a] + c3[a] for a in range(3)], dim=-1)    # (nf, nm, 3)
        fctx.save_for_backward(-(F.sum(dim=2) + Fc) / KCAL, -F / KCAL)
        if want_p:
            parts = np.split(pg, [ncoef, 2 * ncoef, 2 * ncoef + 867], axis=1)
            fctx.gp = [torch.as_tensor(g, device=p.device, dtype=p.dtype).reshape((nf,) + tuple(p.shape))
                       for g, p in zip(parts, params)]
        else:
            fctx.gp = [None] * 4
        return torch.tensor(energy, dtype=torch.float64, device=dev)

    @staticmethod
    def backward(fctx, grad):
        g_com, g_sites = fctx.saved_tensors
        gp = [None if g is None else torch.tensordot(grad.to(g.device), g, dims=1) for g in fctx.gp]
        return (None, None, grad[:, None, None] * g_com, grad[:, None, None, None] * g_sites, *gp)


def three_body_induction_energy(context, box, com, sites, cs_sr, cs_lr, bgr_sr, bgr_lr):
    """FS2 + FS3 + induction energy (kcal/mol) with analytic gradients (see module doc).
    With a ``Batch`` as ``context``: batched frames, (B,) energies; ``box`` is one length or
    one per frame."""
    from .api import Batch
    if isinstance(context, Batch):
        return _ThreeBodyInductionBatch.apply(context, box, com, sites, cs_sr, cs_lr, bgr_sr,
                                              bgr_lr)
    return _ThreeBodyInduction.apply(context, box, com, sites, cs_sr, cs_lr, bgr_sr, bgr_lr)


def fs3_param_tensors(context, device, requires_grad=True):
    """The current FS3 fit of a context (or batch) as float64 tensors, ready to be
    optimised."""
    return [torch.tensor(a, dtype=torch.float64, device=device, requires_grad=requires_grad)
            for a in context.fs3_params()]
