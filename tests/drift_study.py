"""Where the NVE energy drift of the model comes from: the same start run through the oracle's
integrator (the reference's nve_1 restated in Python over the oracle's FP64 C forces) and
through the device integrator, with the FS3 term on and off.

FS3 has a hard cut-off at 6.3 A on every COM distance of a triple
(threebody_potential.f90:860-892) and the term does not vanish there, so each triple that
enters or leaves the list changes the potential energy by its FS3 value while the forces
carry no such impulse.  If that is the drift's source, both implementations show the same
drift with FS3 on, and little with it off.

Two halves, so that the slow oracle half can run on any CPU:
  python tests/drift_study.py oracle OUT.json   # equilibrate and run the oracle (CPU only)
  python tests/drift_study.py gpu OUT.json      # device runs from the same state, comparison
The box is 80 waters of the FS3 variant (flags T T F) at L = 13.39 A (1 g/cm^3, seed 9),
dt = 0.5 fs, with the real-space and 2-body cut-off lowered from 9 to 6.5 A so that every
cut-off (FS3's 6.3 A included) stays below half the box: with a cut-off beyond L/2 the
minimum image itself switches pairs between images discontinuously, in the reference as
here, and that would swamp the effect studied.  The start is the state after a
velocity-rescaled equilibration of the oracle with FS3 off.
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

DT = 0.0005          # ps
NM, L, SEED = 80, 13.39, 9
VARIANT, RCUT = "fs3", 6.5
N_EQUIL = 400        # rescaled FS3-off steps before the comparison runs
N_RUN = 300          # steps of each comparison run
N_LONG = 20000       # steps of the device-only runs that fix the slopes


def slope_per_ns(te):
    t = np.arange(1, len(te) + 1) * DT * 1e-3
    return float(np.polyfit(t, np.asarray(te), 1)[0])


def run_oracle(out):
    import oracle as O
    from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
    from ccpol23_plus_2025_mbmd_b200.generator import water_box
    O.build()
    O.set_threads(0)
    m = Model(data_dir(VARIANT))
    b = water_box(m, NM, L, SEED)
    inp = O.read_inputs(data_dir(VARIANT))
    inp.control["rcut"] = RCUT
    pcoord, pmi, totm = O.principal_frame(inp)
    ld = b.xs.shape[1]
    s = O.MDState(b.x, b.y, b.z, b.v, b.q, b.jb)
    M0 = O.make_model(inp, NM, L, s3=0)
    O.nve_run(M0, (True, True), pcoord, pmi, totm, s, L, DT, N_EQUIL, ld, temp0=298.0,
              nequil=N_EQUIL)
    start = {"x": s.x.tolist(), "y": s.y.tolist(), "z": s.z.tolist(), "v": s.v.tolist(),
             "q": s.q.tolist(), "j": s.j.tolist()}
    res = {"start": start, "oracle": {}}
    for s3 in (1, 0):
        st = O.MDState(*(np.array(start[k]) for k in ("x", "y", "z", "v", "q", "j")))
        t0 = time.time()
        rows = O.nve_run(O.make_model(inp, NM, L, s3=s3), (True, True), pcoord, pmi, totm, st,
                         L, DT, N_RUN, ld)
        res["oracle"][f"fs3_{s3}"] = {"te": [r["te"] for r in rows],
                                      "s_per_step": (time.time() - t0) / N_RUN}
    Path(out).write_text(json.dumps(res))


def run_gpu(out):
    from ccpol23_plus_2025_mbmd_b200 import Context, Model, data_dir
    res = json.loads(Path(out).read_text())
    s0 = {k: np.array(v) for k, v in res["start"].items()}
    res["gpu"] = {}
    for s3 in (1, 0):
        m = Model(data_dir(VARIANT))
        m.set("S3_term", s3)
        m.set("rcut", RCUT)
        with Context(m, NM, L) as c:
            c.md_set_state(L, s0["x"], s0["y"], s0["z"], s0["v"], s0["q"], s0["j"])
            te = [r["te"] for r in c.md_nve(N_RUN, DT)]
            c.md_set_state(L, s0["x"], s0["y"], s0["z"], s0["v"], s0["q"], s0["j"])
            te_long = [r["te"] for r in c.md_nve(N_LONG, DT)]
        o = np.array(res["oracle"][f"fs3_{s3}"]["te"])
        res["gpu"][f"fs3_{s3}"] = {
            "max_abs_te_diff_vs_oracle": float(np.max(np.abs(np.array(te) - o))),
            "slope_run_kcal_mol_ns": slope_per_ns(te),
            "oracle_slope_run_kcal_mol_ns": slope_per_ns(o),
            "slope_long_kcal_mol_ns": slope_per_ns(te_long),
            "te_rms_fluct_long": float(np.std(te_long)),
            "long_steps": N_LONG}
    summary = {k: v for k, v in res["gpu"].items()}
    summary["config"] = {"nm": NM, "box_A": L, "seed": SEED, "dt_ps": DT, "equil": N_EQUIL,
                         "run": N_RUN, "variant": VARIANT, "rcut_A": RCUT}
    print(json.dumps(summary), flush=True)
    Path(out).write_text(json.dumps(res))


if __name__ == "__main__":
    {"oracle": run_oracle, "gpu": run_gpu}[sys.argv[1]](sys.argv[2])
