"""GPU parity: every C-ABI entry point of the FP64 form against the CPU oracle on the same
seeded boxes, to 1e-10 relative (energies as scalars, forces/dipoles normwise, virial as a
scalar); the reference's own FS2 known-answer test through the GPU; mixed precision within
its stated tolerance."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import CcpError, Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import config_box, water_box

from conftest import rel
from fs2_kat import BOHR2A, run as run_fs2_kat, site_offsets

pytestmark = pytest.mark.gpu

TOL = 1e-10          # FP64 form vs oracle
MIXED_FTOL = 1e-5    # mixed form: relative error of site forces and torques vs the FP64 form


def _state(O, nm, ld):
    return O.State(nm, ld)


@pytest.fixture(scope="module")
def boxes(product, oracle):
    out = {}
    for key, variant, nm, L, seed, ld in [("c1", "fs3", 128, 15.64, 1001, 28),
                                          ("fs2fs3_128", "fs2fs3", 128, 15.64, 77, 50),
                                          ("ragged_37", "fs2fs3", 37, 10.37, 9, 31)]:
        m = Model(data_dir(variant))
        b = water_box(m, nm, L, seed, ld=ld)
        inp = oracle.read_inputs(data_dir(variant))
        M = oracle.make_model(inp, nm, L)
        out[key] = (m, b, M)
    return out


def _ctx(m, b, precision="fp64"):
    return Context(m, b.nm, b.box, device=0, precision=precision)


@pytest.mark.parametrize("key", ["c1", "ragged_37"])
def test_ewald_terms(oracle, boxes, key):
    O = oracle
    m, b, M = boxes[key]
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    with _ctx(m, b) as c:
        for name in ("self", "rspace", "kspace"):
            st = _state(O, b.nm, b.xs.shape[1])
            fx, fy, fz = (np.zeros_like(b.xs) for _ in range(3))
            vir = np.zeros(1)
            if name == "self":
                eo = O.ewald_self_correction(M, M.alpha, b.box, *args, st)
                eg = c.ewald_self_correction(M.alpha, b.box, *args, fx, fy, fz, vir)
            elif name == "rspace":
                eo = O.rspace_ewald(M, *args, b.box, M.alpha, st)
                eg = c.rspace_ewald(*args, b.box, M.alpha, fx, fy, fz, vir)
            else:
                eo = O.kspace_ewald(M, *args, M.kmax1, M.kmax2, M.kmax3, M.alpha, b.box, st)
                eg = c.kspace_ewald(*args, M.kmax1, M.kmax2, M.kmax3, M.alpha, b.box, fx, fy, fz, vir)
            assert abs(eg - eo) <= TOL * abs(eo), (name, eg, eo)
            F = np.stack([fx, fy, fz])
            Fo = np.stack([st.fxs, st.fys, st.fzs])
            assert rel(F, Fo) <= TOL, (name, rel(F, Fo))
            assert abs(vir[0] - st.vir.value) <= TOL * abs(st.vir.value), (name, vir[0], st.vir.value)


@pytest.mark.parametrize("key", ["c1", "fs2fs3_128", "ragged_37"])
def test_ccpol23plus(oracle, boxes, key):
    """The 2-body term (vdw_ccpol23plus.f90:174-477): energy, site forces (overwritten) and
    virial (set) against the oracle."""
    O = oracle
    m, b, M = boxes[key]
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    st = _state(O, b.nm, b.xs.shape[1])
    for a in (st.fxs, st.fys, st.fzs):  # both zero the site forces of the ns sites first
        a[:] = 1.0
    eo = O.ccpol23plus(M, *args, b.box, st)
    with _ctx(m, b) as c:
        fx, fy, fz = (np.full_like(b.xs, 1.0) for _ in range(3))
        vir = np.full(1, 7.0)
        eg = c.ccpol23plus(*args, b.box, fx, fy, fz, vir)
    assert abs(eg - eo) <= TOL * abs(eo), (eg, eo)
    assert rel(np.stack([fx, fy, fz]), np.stack([st.fxs, st.fys, st.fzs])) <= TOL
    assert abs(vir[0] - st.vir.value) <= TOL * abs(st.vir.value), (vir[0], st.vir.value)


@pytest.mark.parametrize("key", ["c1", "ragged_37"])
def test_nb_induction(oracle, boxes, key):
    O = oracle
    m, b, M = boxes[key]
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    st = _state(O, b.nm, b.xs.shape[1])
    eo, status, it_o = O.nb_induction(M, *args, b.box, st)
    assert status == 0
    with _ctx(m, b) as c:
        fx, fy, fz, mx, my, mz = (np.zeros_like(b.xs) for _ in range(6))
        vir = np.zeros(1)
        eg, it_g = c.nb_induction(*args, b.box, mx, my, mz, fx, fy, fz, vir)
    assert it_g == it_o
    assert abs(eg - eo) <= TOL * abs(eo), (eg, eo)
    assert rel(np.stack([mx, my, mz]), np.stack([st.idmx, st.idmy, st.idmz])) <= TOL
    assert rel(np.stack([fx, fy, fz]), np.stack([st.fxs, st.fys, st.fzs])) <= TOL
    assert abs(vir[0] - st.vir.value) <= TOL * abs(st.vir.value)


@pytest.mark.parametrize("key,graph_loop,phase_matrix,full,rows",
                         [("c1", 1, 0, 1, 1), ("c1", 0, 1, 1, 1), ("c1", 0, 0, 1, 1),
                          ("c1", 1, 1, 0, 1), ("ragged_37", 1, 1, 0, 1), ("c1", 1, 1, 0, 0)])
def test_nb_induction_loop_forms(oracle, boxes, key, graph_loop, phase_matrix, full, rows):
    """The dipole solve's other execution forms (host-driven loop; tiled on-the-fly
    reciprocal kernels instead of the phase tables; without the full phase matrix, the row
    form or the factor-table kernels) give the same results."""
    O = oracle
    m, b, M = boxes[key]
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    st = _state(O, b.nm, b.xs.shape[1])
    eo, status, it_o = O.nb_induction(M, *args, b.box, st)
    with _ctx(m, b) as c:
        c.set_option("graph_loop", graph_loop)
        c.set_option("phase_matrix", phase_matrix)
        c.set_option("phase_matrix_full", full)
        c.set_option("dipole_row_form", rows)
        fx, fy, fz, mx, my, mz = (np.zeros_like(b.xs) for _ in range(6))
        vir = np.zeros(1)
        eg, it_g = c.nb_induction(*args, b.box, mx, my, mz, fx, fy, fz, vir)
        assert c.get_option("phase_matrix_active") == phase_matrix
        assert c.get_option("dipole_row_form_active") == (phase_matrix and not full and rows)
    assert it_g == it_o
    assert abs(eg - eo) <= TOL * abs(eo), (eg, eo)
    assert rel(np.stack([mx, my, mz]), np.stack([st.idmx, st.idmy, st.idmz])) <= TOL
    assert rel(np.stack([fx, fy, fz]), np.stack([st.fxs, st.fys, st.fzs])) <= TOL


@pytest.mark.parametrize("key", ["c1", "fs2fs3_128", "ragged_37"])
def test_threebody_term(oracle, boxes, key):
    O = oracle
    m, b, M = boxes[key]
    args = (b.x, b.y, b.z, b.xs, b.ys, b.zs)
    st = _state(O, b.nm, b.xs.shape[1])
    e2o, e3o = O.threebody_term(M, *args, b.box, st)
    with _ctx(m, b) as c:
        fx, fy, fz = (np.zeros_like(b.xs) for _ in range(3))
        c2 = [np.zeros(b.nm) for _ in range(3)]
        c3 = [np.zeros(b.nm) for _ in range(3)]
        vir = np.zeros(1)
        e2g, e3g = c.threebody_term(*args, b.box, fx, fy, fz, *c2, *c3, vir)
    assert abs(e3g - e3o) <= TOL * abs(e3o), (e3g, e3o)
    if M.s2_term:
        assert abs(e2g - e2o) <= TOL * abs(e2o), (e2g, e2o)
        assert rel(np.stack(c2), np.stack([st.fxfs2, st.fyfs2, st.fzfs2])) <= TOL
    assert rel(np.stack([fx, fy, fz]), np.stack([st.fxs, st.fys, st.fzs])) <= TOL
    assert rel(np.stack(c3), np.stack([st.fxfs3, st.fyfs3, st.fzfs3])) <= TOL
    assert abs(vir[0] - st.vir.value) <= TOL * abs(st.vir.value)


@pytest.mark.parametrize("key", ["c1", "fs2fs3_128"])
def test_hot_path(oracle, boxes, key):
    O = oracle
    m, b, M = boxes[key]
    eo, st = O.hot_path(M, b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    with _ctx(m, b) as c:
        r = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
        assert c.last_launches() > 0
    e = r.energies
    for k in ("scpe", "rcpe", "kcpe", "indpe", "fs3pe") + (("fs2pe",) if M.s2_term else ()):
        assert abs(e[k] - eo[k]) <= TOL * abs(eo[k]), (k, e[k], eo[k])
    assert abs(e["vir"] - eo["vir"]) <= TOL * abs(eo["vir"])
    assert e["ind_iters"] == eo["ind_iters"]
    assert rel(np.stack([r.fxs, r.fys, r.fzs]), np.stack([st.fxs, st.fys, st.fzs])) <= TOL
    assert rel(np.stack([r.idmx, r.idmy, r.idmz]), np.stack([st.idmx, st.idmy, st.idmz])) <= TOL
    assert rel(np.stack([r.fxfs3, r.fyfs3, r.fzfs3]), np.stack([st.fxfs3, st.fyfs3, st.fzfs3])) <= TOL


@pytest.mark.parametrize("nm", [1, 2, 3])
def test_tiny_systems_match_oracle(product, oracle, nm):
    """One, two and three molecules in a 20 A box: empty neighbour and triple lists, one pair
    and one close triple (centres 3 A apart), through the whole hot path against the oracle;
    terms that vanish must vanish on both sides."""
    O = oracle
    m = Model(data_dir("fs2fs3"))
    L = 20.0
    b = water_box(m, nm, L, 11)
    b.x[:] = [0.0, 3.0, 1.5][:nm]
    b.y[:] = [0.0, 0.0, 2.6][:nm]
    b.z[:] = [0.0, 0.2, -0.3][:nm]
    M = O.make_model(O.read_inputs(data_dir("fs2fs3")), nm, L)
    eo, st = O.hot_path(M, b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    with _ctx(m, b) as c:
        r = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    e = r.energies
    for k in ("scpe", "rcpe", "kcpe", "indpe", "fs2pe", "fs3pe", "vir"):
        if eo[k] == 0.0:
            assert e[k] == 0.0, (k, e[k])
        else:
            assert abs(e[k] - eo[k]) <= TOL * abs(eo[k]), (k, e[k], eo[k])
    if nm < 3:
        assert eo["fs3pe"] == 0.0 and e["n_fs3_triples"] == 0
    else:
        assert e["n_fs3_triples"] == 1 and eo["fs3pe"] != 0.0
    assert e["ind_iters"] == eo["ind_iters"]
    for a, ao in ((np.stack([r.fxs, r.fys, r.fzs]), np.stack([st.fxs, st.fys, st.fzs])),
                  (np.stack([r.idmx, r.idmy, r.idmz]), np.stack([st.idmx, st.idmy, st.idmz])),
                  (np.stack([r.fxfs2, r.fyfs2, r.fzfs2]), np.stack([st.fxfs2, st.fyfs2, st.fzfs2])),
                  (np.stack([r.fxfs3, r.fyfs3, r.fzfs3]), np.stack([st.fxfs3, st.fyfs3, st.fzfs3]))):
        assert rel(a, ao) <= TOL
    # the mixed form (PCG dipoles on as few as three polarisable sites) within its force bar
    with _ctx(m, b, "mixed") as c:
        rm = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    assert rel(np.stack([rm.fxs, rm.fys, rm.fzs]), np.stack([st.fxs, st.fys, st.fzs])) <= MIXED_FTOL


def test_hot_path_device_matches_host(product, boxes):
    import torch
    m, b, M = boxes["fs2fs3_128"]
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(a, device=dev)
    with _ctx(m, b) as c:
        r = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
        f = [torch.zeros(b.xs.shape, dtype=torch.float64, device=dev) for _ in range(3)]
        e = c.hot_path_device(T(b.x), T(b.y), T(b.z), T(b.xs), T(b.ys), T(b.zs), b.box, *f)
    assert e["fs3pe"] == pytest.approx(r.energies["fs3pe"], rel=1e-12)
    assert rel(np.stack([t.cpu().numpy() for t in f]), np.stack([r.fxs, r.fys, r.fzs])) <= 1e-12


def test_fs2_known_answer_on_gpu(product):
    """The reference's FS2 test (periodicity, finite differences, rigid virial) through the
    C ABI: coordinates go in as Angstrom (bohr * bohr2a)."""
    from pathlib import Path
    m = Model(Path(__file__).parent / "golden" / "fs2_kat")
    s = site_offsets()
    with Context(m, 3, 40.0 * BOHR2A) as c:
        def calc(r, box):
            xs, ys, zs = (np.ascontiguousarray(s[a] * BOHR2A) for a in range(3))
            fx, fy, fz = (np.zeros((3, 5)) for _ in range(3))
            c2 = [np.zeros(3) for _ in range(3)]
            c3 = [np.zeros(3) for _ in range(3)]
            vir = np.zeros(1)
            e2, _ = c.threebody_term(*(np.ascontiguousarray(r[a] * BOHR2A) for a in range(3)), xs, ys,
                                     zs, box * BOHR2A, fx, fy, fz, *c2, *c3, vir)
            return e2, vir[0], fx, fy, fz, c2[0], c2[1], c2[2]
        log = run_fs2_kat(calc)
    assert all(ok for *_, ok in log)


def test_mixed_precision_hot_path(product, boxes):
    """Mixed form (FP32 ik/jk gradient passes of FS3 and FP32 FS2 spectator terms; FP64 FS3
    tables and energy pass, Ewald, and the dipole solve by PCG to 1e-8 D RMS) against the FP64
    form on the same box: site forces and torques within 1e-5, per-molecule forces within
    2e-5.  The FS3 sum is ill-conditioned (sum |terms| / |sum| is
    1e4-6e5 per molecular triple, coefficients up to 9e5 of both signs), which is why its
    energy pass, and with it the R_avg-damping COM force, stays FP64: the FS3 energy then
    agrees with the FP64 form to round-off."""
    m, b, M = boxes["fs2fs3_128"]
    out = {}
    for prec in ("fp64", "mixed"):
        with _ctx(m, b, prec) as c:
            out[prec] = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)

    def mol(r):
        F = np.stack([r.fxs, r.fys, r.fzs])
        tot = F.sum(2) + np.stack([r.fxfs2, r.fyfs2, r.fzfs2]) + np.stack([r.fxfs3, r.fyfs3, r.fzfs3])
        tq = np.stack([(b.ys * F[2] - b.zs * F[1]).sum(1), (b.zs * F[0] - b.xs * F[2]).sum(1),
                       (b.xs * F[1] - b.ys * F[0]).sum(1)])
        return tot, tq

    t64, q64 = mol(out["fp64"])
    tmx, qmx = mol(out["mixed"])
    F64 = np.stack([out["fp64"].fxs, out["fp64"].fys, out["fp64"].fzs])
    Fmx = np.stack([out["mixed"].fxs, out["mixed"].fys, out["mixed"].fzs])
    assert rel(Fmx, F64) <= MIXED_FTOL, rel(Fmx, F64)
    assert rel(qmx, q64) <= MIXED_FTOL, rel(qmx, q64)
    # the per-molecule sums cancel more than the site forces they add up; at 512 waters
    # this error is 7e-6, in this 128-water box 1.2e-5
    assert rel(tmx, t64) <= 2 * MIXED_FTOL, rel(tmx, t64)
    C64 = np.stack([out["fp64"].fxfs3, out["fp64"].fyfs3, out["fp64"].fzfs3])
    Cmx = np.stack([out["mixed"].fxfs3, out["mixed"].fyfs3, out["mixed"].fzfs3])
    assert rel(Cmx, C64) <= 1e-10, rel(Cmx, C64)
    e64, emx = out["fp64"].energies, out["mixed"].energies
    for k in ("scpe", "rcpe", "kcpe"):  # FP64 in both forms
        assert emx[k] == pytest.approx(e64[k], rel=1e-12)
    # the dipoles by PCG to 1e-8 D RMS instead of Jacobi to the reference's criterion
    assert emx["indpe"] == pytest.approx(e64["indpe"], rel=1e-8)
    assert emx["ind_iters"] < e64["ind_iters"]
    assert emx["fs2pe"] == pytest.approx(e64["fs2pe"], rel=1e-4)  # FP32 spectator terms
    assert emx["fs3pe"] == pytest.approx(e64["fs3pe"], rel=1e-10)


def test_maxit_reports_not_converged(product, boxes):
    m, b, M = boxes["ragged_37"]
    with _ctx(m, b) as c:
        c.set_maxit(2)
        with pytest.raises(CcpError) as e:
            c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
        assert e.value.code == 2
        c.set_maxit(500)
        r = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)  # context stays usable
        assert r.energies["ind_iters"] > 2
