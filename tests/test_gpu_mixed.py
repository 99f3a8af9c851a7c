"""The mixed-precision form's own parts against the FP64 form and the oracle.

- The dipole solve by preconditioned conjugate gradients (PCG; the mixed form's default, to
  1e-8 D RMS): at the reference's own criterion it reproduces the oracle's Jacobi solution;
  its graph and host-driven loops agree; it reports non-convergence at maxit like Jacobi.
- FS2 with FP32 spectator terms: energy, site forces and COM forces against the FP64 form.
- FS3 with its ik/jk gradient passes in FP32 (an option, off by default): against the FP64
  kernel.
"""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import CcpError, Context, Model, _lib, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import CONFIGS, water_box

from conftest import rel

pytestmark = pytest.mark.gpu

PCG_TOL = 1e-9  # PCG at the reference's criterion vs the oracle's Jacobi solution


@pytest.fixture(scope="module")
def boxes(product, oracle):
    out = {}
    for key, variant, nm, L, seed, ld in [("c1", "fs3", 128, 15.64, 1001, 28),
                                          ("ragged_37", "fs2fs3", 37, 10.37, 9, 31)]:
        m = Model(data_dir(variant))
        b = water_box(m, nm, L, seed, ld=ld)
        M = oracle.make_model(oracle.read_inputs(data_dir(variant)), nm, L)
        out[key] = (m, b, M)
    return out


def _induction(c, b):
    fx, fy, fz, mx, my, mz = (np.zeros_like(b.xs) for _ in range(6))
    vir = np.zeros(1)
    e, it = c.nb_induction(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box, mx, my, mz, fx, fy, fz, vir)
    return e, it, np.stack([mx, my, mz]), np.stack([fx, fy, fz]), vir[0]


@pytest.mark.parametrize("key", ["c1", "ragged_37"])
def test_pcg_at_reference_criterion_matches_oracle(oracle, boxes, key):
    O = oracle
    m, b, M = boxes[key]
    st = O.State(b.nm, b.xs.shape[1])
    eo, status, it_o = O.nb_induction(M, b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box, st)
    assert status == 0
    with Context(m, b.nm, b.box, precision="fp64") as c:
        c.set_option("dipole_solver", 1)
        e, it, mu, F, vir = _induction(c, b)
        assert c.get_option("dipole_solver_pcg_active") == 1
    assert it < it_o, (it, it_o)
    assert abs(e - eo) <= PCG_TOL * abs(eo), (e, eo)
    assert rel(mu, np.stack([st.idmx, st.idmy, st.idmz])) <= PCG_TOL
    assert rel(F, np.stack([st.fxs, st.fys, st.fzs])) <= PCG_TOL
    assert abs(vir - st.vir.value) <= PCG_TOL * abs(st.vir.value)


def test_solver_defaults(boxes):
    m, b, M = boxes["ragged_37"]
    with Context(m, b.nm, b.box, precision="fp64") as c:
        assert c.get_option("dipole_solver") == 0
        _induction(c, b)
        assert c.get_option("dipole_solver_pcg_active") == 0
    with Context(m, b.nm, b.box, precision="mixed") as c:
        assert c.get_option("dipole_solver") == 2
        _induction(c, b)
        assert c.get_option("dipole_solver_pcg_active") == 1
        with pytest.raises(CcpError):
            c.set_option("dipole_solver", 3)


def test_pcg_graph_and_host_loops_agree(boxes):
    m, b, M = boxes["c1"]
    out = []
    for graph in (1, 0):
        with Context(m, b.nm, b.box, precision="mixed") as c:
            c.set_option("graph_loop", graph)
            out.append(_induction(c, b))
    assert out[0][1] == out[1][1]
    assert rel(out[0][2], out[1][2]) <= 1e-13
    assert abs(out[0][0] - out[1][0]) <= 1e-13 * abs(out[1][0])


def test_pcg_maxit_reports_not_converged(boxes):
    m, b, M = boxes["ragged_37"]
    with Context(m, b.nm, b.box, precision="mixed") as c:
        c.set_maxit(2)
        with pytest.raises(CcpError) as e:
            _induction(c, b)
        assert e.value.code == 2
        c.set_maxit(500)
        e, it, *_ = _induction(c, b)  # the context stays usable
        assert 2 < it < 500


def test_mixed_solver_error_against_fp64(product):
    """At the benchmark box the mixed form's dipoles (PCG to 1e-8 D RMS) stay within 1e-7 of
    the FP64 form's (Jacobi at the reference's criterion), in fewer steps."""
    cfg = CONFIGS["c2_512"]
    m = Model(data_dir(cfg["variant"]))
    b = water_box(m, cfg["nm"], cfg["box"], cfg["seed"])
    r = {}
    for prec in ("fp64", "mixed"):
        with Context(m, b.nm, b.box, precision=prec) as c:
            r[prec] = _induction(c, b)
    assert r["mixed"][1] < r["fp64"][1]
    assert rel(r["mixed"][2], r["fp64"][2]) <= 1e-7
    assert rel(r["mixed"][3], r["fp64"][3]) <= 1e-7
    assert abs(r["mixed"][0] - r["fp64"][0]) <= 1e-8 * abs(r["fp64"][0])


@pytest.mark.parametrize("name", ["c2_512", "ragged_37"])
def test_mixed_fs2_against_fp64(product, name):
    """FS2 alone (FS3 switched off in the model) with FP32 spectator terms against the FP64
    kernel: energy within 1e-4 (the FS2 sum over a spectator's five charges, which add up to
    zero, and over spectators of both signs cancels to ~1e-2-1e-3 of its terms; 2.7e-5
    measured at 512 waters), site forces, COM forces and virial within 1e-5."""
    cfg = CONFIGS[name] if name in CONFIGS else dict(nm=37, box=10.37, variant="fs2fs3", seed=9)
    m = Model(data_dir(cfg["variant"]))
    m.set("S3_term", 0)
    b = water_box(m, cfg["nm"], cfg["box"], cfg["seed"], ld=31 if name == "ragged_37" else None)
    out = {}
    for prec in ("fp64", "mixed"):
        with Context(m, b.nm, b.box, precision=prec) as c:
            fx, fy, fz = (np.zeros_like(b.xs) for _ in range(3))
            c2 = [np.zeros(b.nm) for _ in range(3)]
            c3 = [np.zeros(b.nm) for _ in range(3)]
            vir = np.zeros(1)
            e2, e3 = c.threebody_term(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box, fx, fy, fz, *c2,
                                      *c3, vir)
            assert e3 == 0.0
            out[prec] = (e2, np.stack([fx, fy, fz]), np.stack(c2), vir[0])
    e64, F64, C64, v64 = out["fp64"]
    emx, Fmx, Cmx, vmx = out["mixed"]
    assert abs(emx - e64) <= 1e-4 * abs(e64), (emx, e64)
    assert rel(Cmx, C64) <= 1e-5, rel(Cmx, C64)
    assert rel(Fmx, F64) <= 1e-5, rel(Fmx, F64)
    assert abs(vmx - v64) <= 1e-5 * abs(v64), (vmx, v64)


def test_fs3_fp32_passes_against_fp64(product):
    """FS3 alone with its ik/jk gradient passes in FP32 (option fs3_fp32_passes) against the
    FP64 kernel at 512 waters: the energy comes from the FP64 family-0 pass and the COM forces
    from the energy (both within 1e-12), the site forces within 1e-5 (about 2e-6 measured)."""
    import torch
    cfg = CONFIGS["c2_512"]
    m = Model(data_dir(cfg["variant"]))
    b = water_box(m, cfg["nm"], cfg["box"], cfg["seed"])
    dev = torch.device("cuda:0")
    out = {}
    for opt in (0, 1):
        args = [torch.as_tensor(np.ascontiguousarray(a), device=dev)
                for a in (b.x, b.y, b.z, b.xs, b.ys, b.zs)]
        f = [torch.zeros(b.xs.shape, dtype=torch.float64, device=dev) for _ in range(3)]
        c3 = [torch.zeros(b.nm, dtype=torch.float64, device=dev) for _ in range(3)]
        with Context(m, b.nm, b.box, precision="mixed") as c:
            assert c.get_option("fs3_fp32_passes") == 0
            c.set_option("fs3_fp32_passes", opt)
            e = c.terms_device(_lib.TERM_FS3, *args, b.box, *f, None, None, None, *c3)
        out[opt] = (e, np.stack([t.cpu().numpy() for t in f]),
                    np.stack([t.cpu().numpy() for t in c3]))
    (e0, f0, c0), (e1, f1, c1) = out[0], out[1]
    assert e1["fs3pe"] == pytest.approx(e0["fs3pe"], rel=1e-12)
    assert rel(c1, c0) <= 1e-12
    assert 0.0 < rel(f1, f0) <= 1e-5
