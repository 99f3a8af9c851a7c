"""The torch.autograd binding of the three-body plus induction energy: gradients with respect
to positions and to the FS3 fit against central finite differences of the same energy, and
the position gradient against the oracle's analytic forces (the reference's expressions)."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

KCAL = 418.4


@pytest.fixture(scope="module")
def setup(product):
    import torch
    from ccpol23_plus_2025_mbmd_b200.autograd import fs3_param_tensors
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    dev = torch.device("cuda:0")
    com = torch.tensor(np.stack([b.x, b.y, b.z], axis=1), dtype=torch.float64, device=dev)
    sites = torch.tensor(np.stack([b.xs, b.ys, b.zs], axis=2), dtype=torch.float64, device=dev)
    ctx = Context(m, b.nm, b.box)
    params = fs3_param_tensors(ctx, dev)
    yield m, b, ctx, com, sites, params
    ctx.close()


def _energy(ctx, b, com, sites, params):
    from ccpol23_plus_2025_mbmd_b200.autograd import three_body_induction_energy
    return three_body_induction_energy(ctx, b.box, com, sites, *params)


def test_position_gradient_matches_oracle_forces(setup, oracle):
    import torch
    m, b, ctx, com, sites, params = setup
    c = com.clone().requires_grad_(True)
    s = sites.clone().requires_grad_(True)
    E = _energy(ctx, b, c, s, [p.detach() for p in params])
    E.backward()
    O = oracle
    M = O.make_model(O.read_inputs(data_dir("fs2fs3")), b.nm, b.box)
    st = O.State(b.nm, b.xs.shape[1])
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    e2, e3 = O.threebody_term(M, *args, b.box, st)
    ei, status, _ = O.nb_induction(M, *args, b.box, st)
    assert status == 0
    assert abs(E.item() - (e2 + e3 + ei)) <= 1e-10 * abs(e2 + e3 + ei)
    F = np.stack([st.fxs, st.fys, st.fzs], axis=2)              # (nm, ns, 3)
    Fc = np.stack([st.fxfs2 + st.fxfs3, st.fyfs2 + st.fyfs3, st.fzfs2 + st.fzfs3], axis=1)
    assert rel(s.grad.cpu().numpy(), -F / KCAL) <= 1e-10
    assert rel(c.grad.cpu().numpy(), -(F.sum(axis=1) + Fc) / KCAL) <= 1e-10


def test_position_gradient_finite_differences(setup):
    import torch
    m, b, ctx, com, sites, params = setup
    fixed = [p.detach() for p in params]
    c = com.clone().requires_grad_(True)
    s = sites.clone().requires_grad_(True)
    _energy(ctx, b, c, s, fixed).backward()
    gc, gs = c.grad.cpu().numpy(), s.grad.cpu().numpy()
    h = 1e-5
    rng = np.random.default_rng(5)
    off = np.stack([b.xs[0], b.ys[0], b.zs[0]], axis=1)
    same = np.all(np.abs(off[:, None, :] - off[None, :, :]) == 0.0, axis=2)
    scale = max(np.abs(gc).max(), np.abs(gs).max())
    for _ in range(6):
        i, a = rng.integers(b.nm), rng.integers(3)
        cp, cm = com.clone(), com.clone()
        cp[i, a] += h
        cm[i, a] -= h
        fd = (_energy(ctx, b, cp, sites, fixed).item() - _energy(ctx, b, cm, sites, fixed).item()) / (2 * h)
        assert abs(fd - gc[i, a]) <= 1e-6 * scale, ("com", i, a, fd, gc[i, a])
        # sites that coincide (the polarisable sites sit on O, H, H) move together: apart by
        # 1e-5 A they would form a charge-dipole pair the model never contains
        k = rng.integers(sites.shape[1])
        group = [q for q in range(sites.shape[1]) if same[k, q]]
        sp_, sm_ = sites.clone(), sites.clone()
        for q in group:
            sp_[i, q, a] += h
            sm_[i, q, a] -= h
        fd = (_energy(ctx, b, com, sp_, fixed).item() - _energy(ctx, b, com, sm_, fixed).item()) / (2 * h)
        an = sum(gs[i, q, a] for q in group)
        assert abs(fd - an) <= 1e-6 * scale, ("site", i, group, a, fd, an)


def test_fs3_parameter_gradient_finite_differences(setup):
    import torch
    m, b, ctx, com, sites, params = setup
    p = [q.detach().clone().requires_grad_(True) for q in params]
    _energy(ctx, b, com, sites, p).backward()
    grads = [q.grad.cpu().numpy().reshape(-1) for q in p]
    base = [q.detach().cpu().numpy().reshape(-1) for q in p]
    names = ("cs_sr", "cs_lr", "bgr_sr", "bgr_lr")
    checked = 0
    for w in range(4):
        order = np.argsort(-np.abs(grads[w]))[:4]
        for k in order:
            if grads[w][k] == 0.0:
                continue
            step = 1e-6 * max(abs(base[w][k]), 1e-3)
            vals = []
            for sgn in (1.0, -1.0):
                q = [t.detach().clone() for t in p]
                flat = q[w].view(-1)
                flat[k] += sgn * step
                vals.append(_energy(ctx, b, com, sites, q).item())
            fd = (vals[0] - vals[1]) / (2 * step)
            assert abs(fd - grads[w][k]) <= 1e-5 * abs(grads[w][k]), (names[w], k, fd, grads[w][k])
            checked += 1
    assert checked >= 12
    # restore the fit for the other tests of this module
    with torch.no_grad():
        _energy(ctx, b, com, sites, [q.detach() for q in params])


def test_linear_coefficient_gradient_reproduces_energy(setup):
    """The FS3 energy is linear in the coefficients: sum_c c dE/dc over both fits equals
    the FS3 energy itself (a size-independent check of every coefficient gradient)."""
    import torch
    m, b, ctx, com, sites, params = setup
    x, y, z = (com[:, a].contiguous() for a in range(3))
    xs, ys, zs = (sites[:, :, a].contiguous() for a in range(3))
    ctx.set_option("fs3_param_grad", 1)
    from ccpol23_plus_2025_mbmd_b200 import _lib
    e = ctx.terms_device(_lib.TERM_FS3, x, y, z, xs, ys, zs, b.box)
    g_sr, g_lr, _, _ = ctx.fs3_param_grad()
    cs_sr, cs_lr, _, _ = ctx.fs3_params()
    lin = float(np.dot(cs_sr, g_sr) + np.dot(cs_lr, g_lr))
    # both sides are sums with heavy cancellation (sum |c g| / |sum c g| ~ 1e5), accumulated
    # in different orders with FP64 atomics: agreement is bounded by ~1e-16 x 1e5 x terms
    assert abs(lin - e["fs3pe"]) <= 1e-9 * abs(e["fs3pe"]), (lin, e["fs3pe"])
    ctx.set_option("fs3_param_grad", 0)


def test_mixed_form_position_gradient(setup):
    import torch
    m, b, ctx, com, sites, params = setup
    fixed = [q.detach() for q in params]
    out = {}
    for prec in ("fp64", "mixed"):
        with Context(m, b.nm, b.box, precision=prec) as c2:
            s = sites.clone().requires_grad_(True)
            cc = com.clone().requires_grad_(True)
            _energy(c2, b, cc, s, fixed).backward()
            out[prec] = (cc.grad.cpu().numpy(), s.grad.cpu().numpy())
    # measured on this box: site gradients 2.5e-6, molecular-centre gradients 6.6e-5 apart.
    # The centre gradient of a molecule is the sum of its site forces plus the three-body
    # COM forces, a sum that cancels to a small fraction of its parts, so the FP32 terms of
    # the mixed form (FS3's ik/jk gradient passes, FS2's spectator terms) weigh more in it
    assert rel(out["mixed"][1], out["fp64"][1]) <= 1e-5
    assert rel(out["mixed"][0], out["fp64"][0]) <= 2e-4
