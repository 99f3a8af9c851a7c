"""ccp_kspace_ewald_fixed -- the reciprocal-space Ewald sum with the library's fixed device
scratch -- against the context entry point ccp_kspace_ewald on the same box, on two calls in
a row (the second call reuses the scratch the first one left behind).  Collected last, so in
a full run it follows every other test's use of the device; it also passes on its own."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import CcpError, Context, Model, data_dir, ewald_setup
from ccpol23_plus_2025_mbmd_b200.api import kspace_ewald_fixed
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-10          # same bar as the FP64 parity tests
EWALD_PRECISION = 1e-6


@pytest.mark.parametrize("variant,nm,L,seed,ld", [("fs3", 128, 15.64, 1001, 28),
                                                  ("fs2fs3", 37, 10.37, 9, 31)])
def test_fixed_scratch_matches_context(product, variant, nm, L, seed, ld):
    import torch
    m = Model(data_dir(variant))
    b = water_box(m, nm, L, seed, ld=ld)
    alpha, k1, k2, k3 = ewald_setup(EWALD_PRECISION, m.get_double("rcut"), b.box)
    fx, fy, fz = (np.zeros_like(b.xs) for _ in range(3))
    vir = np.zeros(1)
    with Context(m, b.nm, b.box) as c:
        e_ref = c.kspace_ewald(b.x, b.y, b.z, b.xs, b.ys, b.zs, k1, k2, k3, alpha, b.box,
                               fx, fy, fz, vir)
    F_ref = np.stack([fx, fy, fz])
    dev = torch.device("cuda:0")
    args = [torch.as_tensor(a, device=dev) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
    for call in range(2):
        f = [torch.zeros(b.xs.shape, dtype=torch.float64, device=dev) for _ in range(3)]
        q = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
        v = torch.zeros(1, dtype=torch.float64, device=dev)
        kspace_ewald_fixed(m, *args, k1, k2, k3, alpha, b.box, q, *f, v)
        torch.cuda.synchronize()
        F = np.stack([t.cpu().numpy() for t in f])
        assert abs(q.item() - e_ref) <= TOL * abs(e_ref), (call, q.item(), e_ref)
        assert rel(F, F_ref) <= TOL, (call, rel(F, F_ref))
        assert abs(v.item() - vir[0]) <= TOL * abs(vir[0]), (call, v.item(), vir[0])


def test_fixed_scratch_rejects_oversize(product):
    """A box whose tables exceed the fixed scratch is refused by the C entry point before
    anything is launched: the buffers passed are real but far smaller than the molecule
    count claims, which is safe only because nothing reads them."""
    import torch
    from ccpol23_plus_2025_mbmd_b200 import _lib
    m = Model(data_dir("fs3"))
    buf = torch.zeros(28, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    rc = _lib.lib().ccp_kspace_ewald_fixed(m.handle, 100000, p, p, p, p, p, p, 28, 14, 14, 14,
                                           0.358, 150.0, p, p, p, p, p, None)
    assert rc == 6
    assert "bytes of scratch" in _lib.lib().ccp_last_error().decode()
    torch.cuda.synchronize()
    assert float(buf.abs().sum()) == 0.0  # untouched
