"""Molecular dynamics driver with the reference's files (md.f90 for the nve, nvt_b and npt_b
ensembles; nve_1, nvt_b and npt_b_1 of evolve.f90 as motion() selects them).

    python -m ccpol23_plus_2025_mbmd_b200.md RUN_DIR [--steps N] [--precision fp64|mixed]

RUN_DIR holds the reference's inputs: CONTROL, FIELD, data3b_full, data3b_full_LR_4p5 and,
when CONTROL's restart flag is T, REVCON.  The run writes, in the reference's formats:
- OUTPUT: the initial state's row when the run starts at t = 0, then one row per step
  (md.f90:148-152, 213-215);
- HISTORY: sites 1-5 of every molecule with their induced dipoles, every hist_freq steps
  (md.f90:227-238);
- REVCON: the final state (md.f90:266-276).

The state stays on the device between steps; only the per-step scalars and the HISTORY frames
come back.  With nve, steps up to CONTROL's nequil rescale the velocities and angular
momenta to its temperature after the step, as the reference does.  With npt_b the box
changes every step; OUTPUT rows carry each step's volume and density, HISTORY frames the
box of their step and REVCON the final box.  REVCON carries the thermostat and barostat
variables (chit, chip) of the last step, and a restart takes them back (nvt_h continues its
thermostat from chit).  Without a REVCON the start is
the seeded lattice of generator.water_box at the FIELD's molecule count and 0.997 g/cm^3,
with Maxwell-Boltzmann velocities at CONTROL's temperature.  The reference also writes induced-dipole sums (fort.501) and averages; this
driver does not.
"""
from __future__ import annotations

import argparse
import math
from pathlib import Path

import numpy as np

from .api import Context, Model

PI = math.pi
BOLTZ = 8.31451115e-1   # (10 J/mol)/K
DIPMAP = (25, 26, 27, 3, 4)  # md.f90:28, 0-based: dipole site written for sites 1-5

OUTPUT_COLUMNS = ("STEP", "TIME(ps)", "SYS_TEMP(K)", "KE(kcal/mol)", "VDW(kcal/mol)",
                  "COUL(kcal/mol)", "IND(kcal/mol)", "3B(kcal/mol)", "TOTPE(kcal/mol)",
                  "TOTE(kcal/mol)", "VIR(kcal/mol)", "Pres(katm)", "Volm(A^3)",
                  "dens(g/cm^3)", "enthl(kcal/mol)", " HV(kcal/mol)")


def _ffloat(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "E"))


def read_revcon(path, nm):
    """REVCON (initialization.f90:57-70): a title line; step, t, box, chit, chip; then per
    molecule x y z vx vy vz jx jy jz q0 q1 q2 q3 (list-directed)."""
    toks = Path(path).read_text().split("\n", 1)[1].split()
    head = toks[:5]
    vals = np.array([_ffloat(t) for t in toks[5:5 + 13 * nm]]).reshape(nm, 13)
    return {"step": int(float(head[0])), "t": _ffloat(head[1]), "box": _ffloat(head[2]),
            "chit": _ffloat(head[3]), "chip": _ffloat(head[4]),
            "x": vals[:, 0].copy(), "y": vals[:, 1].copy(), "z": vals[:, 2].copy(),
            "v": vals[:, 3:6].copy(), "j": vals[:, 6:9].copy(), "q": vals[:, 9:13].copy()}


def write_revcon(path, step, t, box, state, chit=0.0, chip=0.0):
    """REVCON as md.f90:266-276 writes it (list-directed, one molecule per line)."""
    lines = [" Created by Ommair", f" {step:d} {t!r} {box!r} {chit!r} {chip!r}"]
    for i in range(len(state["x"])):
        row = [state["x"][i], state["y"][i], state["z"][i], *state["v"][i], *state["j"][i],
               *state["q"][i]]
        lines.append(" " + " ".join(f"{v:.17g}" for v in row))
    Path(path).write_text("\n".join(lines) + "\n")


def _e16(v):  # Fortran 1p,e16.8
    return f"{v:16.8E}"


def output_row(step, t, s, nm, box, totm, initial=False):
    # the step's volume when the statistics carry it (npt_b changes the box), else box^3
    """One OUTPUT row (md.f90:169-176, 213-215): '(1x,i8,1p,15e16.8)'.  The row of the
    initial state (md.f90:119-152) forms HV as -pe/nm + 0.0019872036 T, the rows of the
    steps as (-pe + 0.0019872036 T)/nm; both as the reference writes them."""
    volm = s.get("volm") or box ** 3
    rho = (totm * nm) / (volm * 1e-24 * 6.022e23)
    enth = (s["pe"] + (s["pres"] * volm) * 2.42e-26) / nm
    if initial:
        hv = -s["pe"] / nm + 0.0019872036 * s["sys_temp"]
    else:
        hv = (-s["pe"] + 0.0019872036 * s["sys_temp"]) / nm
    vals = (t, s["sys_temp"], s["tke"] + s["rke"], s["vdwpe"], s["cpe"], s["indpe"], s["pe3b"],
            s["pe"], s["te"], s["vir"], s["pres"], volm, rho, enth, hv)
    return " " + f"{step:8d}" + "".join(_e16(v) for v in vals)


def history_frame(step, dt, box, names, masses, charges, state, xs, ys, zs, dip):
    """One HISTORY frame (md.f90:227-238): sites 1-5 of every molecule with the induced
    dipole of the mapped polarisable site."""
    nm = len(state["x"])
    out = [f"{'timestep':8s}{step:10d}{nm * 5:10d}{0:10d}{1:10d}{dt:12.6f}"]
    for row in ((box, 0.0, 0.0), (0.0, box, 0.0), (0.0, 0.0, box)):
        out.append("".join(f"{v:12.4G}" for v in row))
    k = 0
    for j in range(nm):
        for s in range(5):
            k += 1
            out.append(f"{names[s]:8s}{k:10d}{masses[s]:12.6f}{charges[s]:12.6f}")
            out.append("".join(f"{v:12.4E}" for v in (state["x"][j] + xs[j, s],
                                                      state["y"][j] + ys[j, s],
                                                      state["z"][j] + zs[j, s])))
            d = DIPMAP[s]
            out.append("".join(f"{v:16.8E}" for v in (dip[0][j, d], dip[1][j, d], dip[2][j, d])))
    return "\n".join(out) + "\n"


def _field_names(directory):
    lines = (Path(directory) / "FIELD").read_text().splitlines()
    ns = int(lines[2].split()[0])
    names, masses, charges = [], [], []
    for ln in lines[5:5 + ns]:
        t = ln.split()
        names.append(t[0])
        masses.append(float(t[4]))
        charges.append(float(t[5]))
    return names, masses, charges


def run(directory, nsteps=None, precision="fp64", device=0, out_dir=None):
    """A run of CONTROL's ensemble (nve, nvt_b or npt_b) from RUN_DIR's inputs; returns the
    per-step statistics."""
    directory = Path(directory)
    out_dir = Path(out_dir or directory)
    m = Model(directory)
    kind = m.get_int("ensemble_kind")
    if kind < 0:
        raise ValueError("CONTROL's ensemble is not one of nve, nvt_b, npt_b, nvt_h, npt_h, "
                         "npt_mtk")
    ensemble = ("nve", "nvt_b", "npt_b", "nvt_h", "npt_h", "npt_mtk")[kind]
    nm, ns = m.get_int("nm"), m.ns
    nsteps = m.get_int("nsteps") if nsteps is None else nsteps
    dt = m.get_double("dt")
    hist = max(m.get_int("hist_freq"), 1)
    nequil = m.get_int("nequil")
    totm = m.get_double("totm")
    step0, t0, chit, chip = 0, 0.0, 0.0, 0.0
    if m.get_int("restart"):
        rc = read_revcon(directory / "REVCON", nm)
        box, step0, t0, chit, chip = rc["box"], rc["step"], rc["t"], rc["chit"], rc["chip"]
        state = rc
        for a in ("x", "y", "z"):  # initialization.f90:72-77: images into the box
            state[a] = state[a] - box * np.round(state[a] / box)
    else:
        from .generator import water_box
        box = (nm * totm / (0.997 * 0.6022)) ** (1.0 / 3.0)
        b = water_box(m, nm, box, 1, temperature=m.get_double("temp0"))
        state = {"x": b.x, "y": b.y, "z": b.z, "v": b.v, "q": b.q, "j": b.jb}
    names, masses, charges = _field_names(directory)
    stats = []
    with Context(m, nm, box, device=device, precision=precision) as c:
        c.md_set_state(box, state["x"], state["y"], state["z"], state["v"], state["q"], state["j"])
        c.md_set_ensemble(ensemble, m.get_double("temp0"), m.get_double("taut"),
                          m.get_double("pres0"), m.get_double("taup"))
        c.md_set_thermostat(chit, chip)
        if ensemble == "nve":  # md.f90:187-193: steps up to nequil are followed by a rescale
            c.md_set_equilibration(m.get_double("temp0"), min(max(nequil - step0, 0), nsteps))
        with open(out_dir / "OUTPUT", "w") as fo, open(out_dir / "HISTORY", "w") as fh:
            fo.write("-" * 250 + "\n")
            fo.write("".join(f"{c_:>16s}" for c_ in OUTPUT_COLUMNS) + "\n")
            fo.write("-" * 250 + "\n")
            if t0 == 0.0:  # md.f90:148-152: the initial state's row
                fo.write(output_row(step0, t0, c.md_stats(), nm, box, totm, initial=True) + "\n")
            fh.write(" Created by Ommair\n" + f"{0:10d}{1:10d}{nm * 3:10d}\n")
            done = 0
            while done < nsteps:
                n = min(hist - (step0 + done) % hist or hist, nsteps - done)
                chunk = c.md_run(n, dt)
                for k, s in enumerate(chunk):
                    step = step0 + done + k + 1
                    fo.write(output_row(step, t0 + (done + k + 1) * dt, s, nm, box, totm) + "\n")
                stats += chunk
                done += n
                box = chunk[-1]["box"]
                if (step0 + done) % hist == 0 and step0 + done > nequil:
                    st = c.md_get_state()
                    q = st["q"]
                    pc = m.pcoord
                    R = _rot(q)
                    xs, ys, zs = (np.einsum("ik,sk->is", R[:, a, :], pc) for a in range(3))
                    fh.write(history_frame(step0 + done, dt, box, names, masses, charges, st,
                                           xs, ys, zs, c.md_dipoles()))
        st = c.md_get_state()
    if stats:
        chit, chip = stats[-1]["chit"], stats[-1]["chip"]
    write_revcon(out_dir / "REVCON", step0 + nsteps, t0 + nsteps * dt, box, st, chit, chip)
    return stats


def _rot(q):
    """quat_to_rot (molecular_sites.f90:95-111) for every molecule: (nm, 3, 3)."""
    q0, q1, q2, q3 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack([
        np.stack([q0 ** 2 + q1 ** 2 - q2 ** 2 - q3 ** 2, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)], -1),
        np.stack([2 * (q1 * q2 + q0 * q3), q0 ** 2 - q1 ** 2 + q2 ** 2 - q3 ** 2, 2 * (q2 * q3 - q0 * q1)], -1),
        np.stack([2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), q0 ** 2 - q1 ** 2 - q2 ** 2 + q3 ** 2], -1),
    ], 1)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("run_dir")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    run(args.run_dir, args.steps, args.precision, args.device)


if __name__ == "__main__":
    main()
