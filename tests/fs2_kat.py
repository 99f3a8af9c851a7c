"""The reference's FS2 known-answer test (source/tests/check_fs2_periodic.py:29-85),
restated as a driver over any FS2 evaluator.

`calc(r, box)` takes COM coordinates r[a, i] (bohr, axis a, molecule i) and the box (bohr),
with the fixture's site offsets, and returns (energy kcal/mol, vir, fxs, fys, fzs, fxfs2,
fyfs2, fzfs2) in the reference's units (forces 10 J/mol/A).  Checks and tolerances are the
reference test's: periodic energy 1e-10, virial and forces 1e-7, central finite differences
of forces and of the rigid-scaling virial 1e-7 with h = 1e-5, each relative to
max(1, |expected|).
"""
import numpy as np

BOHR2A = 0.529177249
SITE_X = [0.0, 1.43, -1.43, 0.3, -0.3]
SITE_Y = [-0.1, 1.0, 1.0, -0.5, -0.5]
SITE_Z = [0.0, 0.0, 0.0, 0.5, -0.5]


def site_offsets():
    s = np.zeros((3, 3, 5))  # (axis, molecule, site)
    for i in range(3):
        s[0, i], s[1, i], s[2, i] = SITE_X, SITE_Y, SITE_Z
    return s


class Failure(AssertionError):
    pass


def near(actual, expected, tol, label, log):
    ok = abs(actual - expected) <= tol * max(1.0, abs(expected))
    log.append((label, actual, expected, ok))
    if not ok:
        raise Failure(f"FAIL: {label} {actual} {expected}")


def run(calc):
    h = 1e-5
    conv = BOHR2A / 418.4
    s = site_offsets()
    log = []
    for geometry in (1, 2, 3):
        g = geometry ** 0.5
        r = np.array([[0.0, 5.5, 2.0], [0.0, 0.3, 5.0], [0.0, 0.2, 0.7]]) * g
        rbase = r.copy()
        e, vir, fxs, fys, fzs, cx, cy, cz = calc(r, 40.0)
        eb, vb = e, vir
        fb = np.stack([cx + fxs.sum(1), cy + fys.sum(1), cz + fzs.sum(1)])
        sb = np.stack([fxs, fys, fzs])
        for i in range(3):
            for a in range(3):
                for sgn in (-1, 1):
                    r = rbase.copy()
                    r[a, i] += sgn * 40.0
                    e, vir, fxs, fys, fzs, cx, cy, cz = calc(r, 40.0)
                    near(e, eb, 1e-10, "periodic energy", log)
                    near(vir, vb, 1e-7, "periodic virial", log)
                    f = np.stack([cx + fxs.sum(1), cy + fys.sum(1), cz + fzs.sum(1)])
                    near(np.max(np.abs(f - fb)), 0.0, 1e-7, "periodic molecular forces", log)
                    near(np.max(np.abs(fxs - sb[0])), 0.0, 1e-7, "periodic site x forces", log)
                    near(np.max(np.abs(fys - sb[1])), 0.0, 1e-7, "periodic site y forces", log)
                    near(np.max(np.abs(fzs - sb[2])), 0.0, 1e-7, "periodic site z forces", log)
        r = rbase.copy()
        r[0, 0] += 40.0
        r[1, 1] -= 40.0
        e, vir, fxs, fys, fzs, cx, cy, cz = calc(r, 40.0)
        vcom = np.sum(fxs * s[0] + fys * s[1] + fzs * s[2]) * conv
        v = vir / 418.4 + vcom
        f = fb * conv
        for i in range(3):
            for a in range(3):
                r[a, i] += h
                ep = calc(r, 40.0)[0]
                r[a, i] -= 2 * h
                em = calc(r, 40.0)[0]
                r[a, i] += h
                near(f[a, i], -(ep - em) / (2 * h), 1e-7, "finite difference force", log)
        ep = calc(r * (1 + h), 40.0 * (1 + h))[0]
        em = calc(r * (1 - h), 40.0 * (1 - h))[0]
        near(v, (ep - em) / (2 * h), 1e-7, "finite difference rigid virial", log)
    return log
