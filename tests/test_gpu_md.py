"""The device NVE integrator (nve_1 + nosquish, evolve.f90:621-1061, 8107-8203) against the
oracle's step-by-step restatement of the same integrator with the oracle's forces: state and
per-step energies after a few steps of a 37-water FS2+FS3 box."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200.generator import water_box

from conftest import rel

pytestmark = pytest.mark.gpu

DT = 0.0005   # ps, as the benchmark configurations
NSTEPS = 3


@pytest.fixture(scope="module")
def md_case(product, oracle):
    O = oracle
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    inp = O.read_inputs(data_dir("fs2fs3"))
    pcoord, pmi, totm = O.principal_frame(inp)
    M = O.make_model(inp, b.nm, b.box)
    s = O.MDState(b.x, b.y, b.z, b.v, b.q, b.jb)
    ref = O.nve_run(M, (True, True), pcoord, pmi, totm, s, b.box, DT, NSTEPS, b.xs.shape[1])
    return m, b, s, ref


def test_nve_matches_oracle_integrator(md_case):
    m, b, s_ref, ref = md_case
    with Context(m, b.nm, b.box) as c:
        c.md_set_state(b.box, b.x, b.y, b.z, b.v, b.q, b.jb)
        stats = c.md_nve(NSTEPS, DT)
        st = c.md_get_state()
    for k, (g, o) in enumerate(zip(stats, ref)):
        for key in ("vdwpe", "cpe", "indpe", "pe3b", "pe", "tke", "rke", "te", "vir"):
            assert abs(g[key] - o[key]) <= 1e-9 * max(abs(o[key]), 1.0), (k, key, g[key], o[key])
        assert g["sys_temp"] == pytest.approx(o["sys_temp"], rel=1e-9)
        assert g["pres"] == pytest.approx(o["pres"], rel=1e-8, abs=1e-9)
    assert rel(np.stack([st["x"], st["y"], st["z"]]), np.stack([s_ref.x, s_ref.y, s_ref.z])) <= 1e-12
    assert rel(st["v"], s_ref.v) <= 1e-9
    assert rel(st["q"], s_ref.q) <= 1e-12
    assert rel(st["j"], s_ref.j) <= 1e-9


def test_nve_continues_across_calls(md_case):
    """Two calls of one step each equal one call of two steps (the forces of the last
    evaluation stay on the device between calls)."""
    m, b, _, _ = md_case
    out = []
    for split in ((2,), (1, 1)):
        with Context(m, b.nm, b.box) as c:
            c.md_set_state(b.box, b.x, b.y, b.z, b.v, b.q, b.jb)
            stats = []
            for n in split:
                stats += c.md_nve(n, DT)
            out.append((stats[-1]["te"], c.md_get_state()))
    assert out[0][0] == pytest.approx(out[1][0], rel=1e-12)
    assert rel(out[0][1]["v"], out[1][1]["v"]) <= 1e-12


def test_nve_equilibration_matches_oracle(product, oracle):
    """Equilibration steps (md.f90:187-193): after each of the first nequil steps the COM
    velocities and angular momenta are rescaled to temp0; the rows report the state before
    the rescale."""
    O = oracle
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9, temperature=450.0)
    inp = O.read_inputs(data_dir("fs2fs3"))
    pcoord, pmi, totm = O.principal_frame(inp)
    M = O.make_model(inp, b.nm, b.box)
    s = O.MDState(b.x, b.y, b.z, b.v, b.q, b.jb)
    ref = O.nve_run(M, (True, True), pcoord, pmi, totm, s, b.box, DT, 3, b.xs.shape[1],
                    temp0=298.15, nequil=2)
    with Context(m, b.nm, b.box) as c:
        c.md_set_state(b.box, b.x, b.y, b.z, b.v, b.q, b.jb)
        c.md_set_equilibration(298.15, 2)
        stats = c.md_nve(3, DT)
        st = c.md_get_state()
    for k, (g, o) in enumerate(zip(stats, ref)):
        for key in ("tke", "rke", "te", "pe"):
            assert abs(g[key] - o[key]) <= 1e-9 * max(abs(o[key]), 1.0), (k, key, g[key], o[key])
    assert rel(st["v"], s.v) <= 1e-9
    assert rel(st["j"], s.j) <= 1e-9
    # the rescale took the 450 K start towards 298 K
    assert stats[1]["sys_temp"] < stats[0]["sys_temp"]


def test_md_stats_of_initial_state(product, oracle):
    O = oracle
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    inp = O.read_inputs(data_dir("fs2fs3"))
    pcoord, pmi, totm = O.principal_frame(inp)
    M = O.make_model(inp, b.nm, b.box)
    s = O.MDState(b.x, b.y, b.z, b.v, b.q, b.jb)
    ref = O.state_stats(M, (True, True), pcoord, pmi, totm, s, b.box, b.xs.shape[1])
    with Context(m, b.nm, b.box) as c:
        c.md_set_state(b.box, b.x, b.y, b.z, b.v, b.q, b.jb)
        g = c.md_stats()
    for key in ("vdwpe", "cpe", "indpe", "pe3b", "pe", "tke", "rke", "te", "vir", "sys_temp"):
        assert abs(g[key] - ref[key]) <= 1e-9 * max(abs(ref[key]), 1.0), (key, g[key], ref[key])
    assert g["pres"] == pytest.approx(ref["pres"], rel=1e-8, abs=1e-9)


def _run_dir(path, nm, nsteps, hist, restart, nequil=0, ensemble="nve  1.0  2.0"):
    import shutil
    path.mkdir()
    src = data_dir("fs2fs3")
    for f in ("FIELD", "CONTROL", "data3b_full", "data3b_full_LR_4p5"):
        shutil.copy(src / f, path / f)
    ctl = (path / "CONTROL").read_text().splitlines()
    ctl[1] = f"   {ensemble}     # ensemble"
    ctl[5] = f"   {nsteps}    # nsteps"
    ctl[7] = f"   {nequil}    # nequil"
    ctl[9] = f"   {hist}     # history frequency"
    ctl[15] = f"   {'T' if restart else 'F'}     # restart"
    (path / "CONTROL").write_text("\n".join(ctl) + "\n")
    fld = (path / "FIELD").read_text().splitlines()
    fld[1] = f"  {nm}    nom    -number of molecules"
    (path / "FIELD").write_text("\n".join(fld) + "\n")
    return path


def test_md_driver_files_and_restart(product, tmp_path):
    """The md.f90-style driver: OUTPUT rows, HISTORY frames, REVCON; and 2 + 2 steps through
    a REVCON restart equal 4 steps in one run, with the equilibration rescale (nequil = 3)
    running across the restart."""
    import shutil
    from ccpol23_plus_2025_mbmd_b200.md import read_revcon, run
    a = _run_dir(tmp_path / "a", 37, 4, 2, False, nequil=3)
    stats = run(a)
    out = (a / "OUTPUT").read_text().splitlines()
    assert len(out) == 3 + 1 + 4  # header, the initial state's row (t = 0), 4 steps
    assert int(out[3].split()[0]) == 0 and int(out[-1].split()[0]) == 4
    assert abs(float(out[-1].split()[9]) - stats[-1]["te"]) <= 1e-7 * abs(stats[-1]["te"])
    hist = (a / "HISTORY").read_text().splitlines()
    # frames every 2 steps, only after the equilibration (md.f90:220): step 4
    assert [int(ln.split()[1]) for ln in hist if ln.startswith("timestep")] == [4]
    ra = read_revcon(a / "REVCON", 37)
    assert ra["step"] == 4
    b = _run_dir(tmp_path / "b", 37, 2, 2, False, nequil=3)
    run(b)
    c = _run_dir(tmp_path / "c", 37, 2, 2, True, nequil=3)
    shutil.copy(b / "REVCON", c / "REVCON")
    run(c)
    rc = read_revcon(c / "REVCON", 37)
    assert rc["step"] == 4 and abs(rc["t"] - ra["t"]) < 1e-15
    for k in ("x", "y", "z", "v", "q", "j"):
        assert rel(rc[k], ra[k]) <= 1e-10, k


@pytest.mark.parametrize("ensemble", ["nvt_b", "npt_b", "nvt_h", "npt_h", "npt_mtk"])
def test_thermostat_ensembles_match_oracle(product, oracle, ensemble):
    """nvt_b, npt_b_1, nvt_hov_3 and npt_hov_2 (evolve.f90:1063-1644, 7485-8104, 3316-3834,
    5567-6155) on the device against the oracle's restatement: per-step statistics, box,
    thermostat and barostat variables and final state after 3 steps (the Nose-Hoover
    ensembles from non-zero chit and chip, as after a restart)."""
    O = oracle
    m = Model(data_dir("fs2fs3"))
    b = water_box(m, 37, 10.37, 9)
    inp = O.read_inputs(data_dir("fs2fs3"))
    pcoord, pmi, totm = O.principal_frame(inp)
    M = O.make_model(inp, b.nm, b.box)
    s = O.MDState(b.x, b.y, b.z, b.v, b.q, b.jb)
    temp0, taut, pres0, taup = 298.15, 0.05, 0.001, 0.1
    ref = O.md_run(M, (True, True), pcoord, pmi, totm, s, b.box, DT, 3, b.xs.shape[1], ensemble,
                   temp0=temp0, taut=taut, pres0=pres0 / O.PRSUNT, taup=taup,
                   rcut=m.get_double("rcut"), chit0=0.3, chip0=0.02)
    with Context(m, b.nm, b.box) as c:
        c.md_set_state(b.box, b.x, b.y, b.z, b.v, b.q, b.jb)
        c.md_set_ensemble(ensemble, temp0, taut, pres0, taup)
        c.md_set_thermostat(0.3, 0.02)
        stats = c.md_run(3, DT)
        st = c.md_get_state()
    for k, (g, o) in enumerate(zip(stats, ref)):
        for key in ("pe", "tke", "rke", "te", "sys_temp", "vir", "box", "volm"):
            assert abs(g[key] - o[key]) <= 1e-9 * max(abs(o[key]), 1.0), (k, key, g[key], o[key])
        assert g["pres"] == pytest.approx(o["pres"], rel=1e-8, abs=1e-9)
        if ensemble in ("nvt_h", "npt_h", "npt_mtk"):
            assert g["chit"] == pytest.approx(o["chit"], rel=1e-9, abs=1e-12)
            assert g["consv"] == pytest.approx(o["consv"], rel=1e-9, abs=1e-9)
        if ensemble in ("npt_h", "npt_mtk"):
            assert g["chip"] == pytest.approx(o["chip"], rel=1e-9, abs=1e-12)
    if ensemble in ("npt_b", "npt_h", "npt_mtk"):
        assert stats[-1]["box"] != b.box
    assert rel(np.stack([st["x"], st["y"], st["z"]]), np.stack([s.x, s.y, s.z])) <= 1e-12
    assert rel(st["v"], s.v) <= 1e-9
    assert rel(st["j"], s.j) <= 1e-9


def test_md_driver_npt_b(product, tmp_path):
    """The driver with the shipped CONTROL's ensemble (npt_b, taut 1 ps, taup 2 ps): the box
    changes every step, OUTPUT's volume column follows it and REVCON holds the final box."""
    from ccpol23_plus_2025_mbmd_b200.md import read_revcon, run
    a = _run_dir(tmp_path / "a", 37, 3, 3, False, ensemble="npt_b  1.0  2.0")
    stats = run(a)
    boxes = [s["box"] for s in stats]
    assert len(set(boxes)) == 3
    out = (a / "OUTPUT").read_text().splitlines()
    for row, s in zip(out[4:], stats):
        assert abs(float(row.split()[12]) - s["volm"]) <= 1e-7 * s["volm"]
    assert read_revcon(a / "REVCON", 37)["box"] == pytest.approx(boxes[-1], rel=1e-15)


def test_md_driver_nvt_h_restart(product, tmp_path):
    """nvt_h through the driver: 2 + 2 steps through a REVCON restart (which carries the
    thermostat variable chit) equal 4 steps in one run."""
    import shutil
    from ccpol23_plus_2025_mbmd_b200.md import read_revcon, run
    ens = "nvt_h  0.05  2.0"
    a = _run_dir(tmp_path / "a", 37, 4, 4, False, ensemble=ens)
    run(a)
    ra = read_revcon(a / "REVCON", 37)
    assert ra["chit"] != 0.0
    b = _run_dir(tmp_path / "b", 37, 2, 2, False, ensemble=ens)
    run(b)
    c = _run_dir(tmp_path / "c", 37, 2, 2, True, ensemble=ens)
    shutil.copy(b / "REVCON", c / "REVCON")
    run(c)
    rc = read_revcon(c / "REVCON", 37)
    assert rc["chit"] == pytest.approx(ra["chit"], rel=1e-12)
    for k in ("x", "y", "z", "v", "q", "j"):
        assert rel(rc[k], ra[k]) <= 1e-10, k
