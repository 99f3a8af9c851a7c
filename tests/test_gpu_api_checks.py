"""Argument checks and stream ordering of the torch-facing API on the GPU: tensors of the
wrong dtype, layout, size or device are refused before the library runs; non-finite
coordinates are refused by the evaluation itself, which stays usable; the autograd forward
runs after work that torch has queued ahead of it on its current stream."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import CcpError, Context, Model, _lib, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(product):
    import torch
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return m, b, [T(a) for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]


def test_terms_device_refuses_wrong_tensors(setup):
    import torch
    m, b, args = setup
    with Context(m, b.nm, b.box) as c:
        with pytest.raises(ValueError, match="float64"):
            c.terms_device(_lib.TERM_FS3, *args[:3], *(a.float() for a in args[3:]), b.box)
        with pytest.raises(ValueError, match="contiguous"):
            xs_t = args[3].t().contiguous().t()  # same shape, column-major strides
            c.terms_device(_lib.TERM_FS3, *args[:3], xs_t, *args[4:], b.box)
        with pytest.raises(ValueError, match="molecules"):
            c.terms_device(_lib.TERM_FS3, *(a[:-1] for a in args), b.box)
        with pytest.raises(ValueError, match="CUDA"):
            c.terms_device(_lib.TERM_FS3, *args, b.box, torch.zeros(b.xs.shape, dtype=torch.float64))
        with pytest.raises(ValueError, match="shape"):
            c.hot_path_device(*args, b.box, torch.zeros(b.nm, 3, device="cuda:0",
                                                          dtype=torch.float64))
        e = c.terms_device(_lib.TERM_FS3, *args, b.box)  # the context stays usable
        assert e["fs3pe"] != 0.0


@pytest.mark.parametrize("where,value", [("x", np.nan), ("zs", np.inf), ("ys", -np.inf)])
def test_non_finite_coordinates_are_refused(setup, where, value):
    """A NaN or infinite COM coordinate or site offset, through the host-buffer and the
    device entry points: CCP_ERR_BAD_INPUT naming the cause; the next valid call works."""
    m, b, args = setup
    bad = {k: getattr(b, k).copy() for k in ("x", "y", "z", "xs", "ys", "zs")}
    bad[where].flat[5] = value
    with Context(m, b.nm, b.box) as c:
        good = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box).energies
        with pytest.raises(CcpError, match="non-finite"):
            c.hot_path(*(bad[k] for k in ("x", "y", "z", "xs", "ys", "zs")), b.box)
        again = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box).energies
        assert again["fs3pe"] == pytest.approx(good["fs3pe"], rel=1e-12)
        import torch
        dev_bad = [torch.as_tensor(np.ascontiguousarray(bad[k]), device="cuda:0")
                   for k in ("x", "y", "z", "xs", "ys", "zs")]
        with pytest.raises(CcpError, match="non-finite"):
            c.terms_device(_lib.TERM_HOT, *dev_bad, b.box)
        e = c.terms_device(_lib.TERM_HOT, *args, b.box)
        assert e["indpe"] == pytest.approx(good["indpe"], rel=1e-12)


def test_autograd_forward_waits_for_queued_torch_work(setup):
    """The inputs are produced by a torch kernel queued behind a ~0.1 s device spin on torch's
    stream; the evaluation must see them, not the memory before they were written."""
    import torch
    from ccpol23_plus_2025_mbmd_b200.autograd import fs3_param_tensors, three_body_induction_energy
    m, b, args = setup
    dev = torch.device("cuda:0")
    com0 = torch.stack(args[:3], dim=1)
    sites0 = torch.stack(args[3:], dim=2)
    with Context(m, b.nm, b.box) as c:
        params = [p.detach() for p in fs3_param_tensors(c, dev, requires_grad=False)]
        ref = three_body_induction_energy(c, b.box, com0, sites0, *params).item()
        for _ in range(3):
            torch.cuda.synchronize()
            torch.cuda._sleep(200_000_000)  # bounded spin (~0.1 s) on torch's current stream
            com = com0 * 1.0                # written only after the spin
            sites = sites0 * 1.0
            e = three_body_induction_energy(c, b.box, com, sites, *params).item()
            assert e == pytest.approx(ref, rel=1e-12)
