"""Randomised small boxes through the whole hot path against the oracle (hypothesis): 3 to 24
waters of either parameter set, at densities from liquid water to a third of it (boxes of
at least 6.5 A), with a random seed and row stride.  The FP64 form must match the oracle at 1e-10 in every energy,
the virial, the iteration count, the site forces, both COM force sets and the dipoles; terms
that vanish must vanish on both sides.  Examples are drawn deterministically, so a failure
reproduces."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from ccpol23_plus_2025_mbmd_b200 import Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-10
RHO = 0.0334  # waters per cubic Angstrom in liquid water


@settings(max_examples=30, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(nm=st.integers(3, 24), variant=st.sampled_from(["fs3", "fs2fs3"]),
       dilution=st.floats(1.0, 3.0), seed=st.integers(0, 2**31 - 1), pad=st.integers(0, 4))
def test_random_boxes_match_oracle(product, oracle, nm, variant, dilution, seed, pad):
    O = oracle
    m = Model(data_dir(variant))
    L = max(float((nm * dilution / RHO) ** (1.0 / 3.0)), 6.5)  # the generator packs no tighter
    b = water_box(m, nm, L, seed, ld=m.ns + pad)
    M = O.make_model(O.read_inputs(data_dir(variant)), nm, L)
    eo, so = O.hot_path(M, b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    assert eo["ind_status"] == 0
    with Context(m, nm, b.box) as c:
        r = c.hot_path(b.x, b.y, b.z, b.xs, b.ys, b.zs, b.box)
    e = r.energies
    keys = ("scpe", "rcpe", "kcpe", "indpe", "fs3pe", "vir") + (("fs2pe",) if M.s2_term else ())
    for k in keys:
        if eo[k] == 0.0:
            assert e[k] == 0.0, (k, e[k])
        else:
            assert abs(e[k] - eo[k]) <= TOL * abs(eo[k]), (k, e[k], eo[k])
    assert e["ind_iters"] == eo["ind_iters"]
    pairs = ((np.stack([r.fxs, r.fys, r.fzs]), np.stack([so.fxs, so.fys, so.fzs])),
             (np.stack([r.idmx, r.idmy, r.idmz]), np.stack([so.idmx, so.idmy, so.idmz])),
             (np.stack([r.fxfs3, r.fyfs3, r.fzfs3]), np.stack([so.fxfs3, so.fyfs3, so.fzfs3])))
    if M.s2_term:
        pairs += ((np.stack([r.fxfs2, r.fyfs2, r.fzfs2]), np.stack([so.fxfs2, so.fyfs2, so.fzfs2])),)
    for a, ao in pairs:
        assert rel(a, ao) <= TOL
