"""Python side of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module.  It loads ``oracle/_build/libccpol_oracle.so`` (built by ``oracle/Makefile``) and
restates, independently of the product library:

* the input readers of the reference: CONTROL (initialization.f90:463-489), FIELD and the
  FS3 parameter files (initialization.f90:491-720);
* the molecular frame set-up: shift_to_com (initialization.f90:728-748),
  principle_moment_inertia with the DL_POLY Jacobi diagonaliser
  (initialization.f90:750-845, utility.f90:458-596);
* site placement from quaternions: sites/transform/quat_to_rot
  (molecular_sites.f90:14-111).

Arrays follow the reference layout: COM arrays ``x[nm]``; site arrays ``xs[nm, ld]`` in C
order, i.e. site index fastest (the Fortran ``xs(nsite, nom)`` column-major layout).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libccpol_oracle.so"

BOHR2A = 0.529177249
R4PIE0 = 138935.4835
H2KCAL = 627.510
EWP = 1.0e-6


class OrcModel(C.Structure):
    _fields_ = [
        ("nm", C.c_int), ("ns", C.c_int), ("npol", C.c_int),
        ("charge", C.c_double * 50), ("polarizability", C.c_double * 50),
        ("alpha", C.c_double), ("kmax1", C.c_int), ("kmax2", C.c_int), ("kmax3", C.c_int),
        ("rcut", C.c_double), ("rcutsd", C.c_double),
        ("rcut3", C.c_double), ("rcutsd3", C.c_double),
        ("alpha3", C.c_double), ("delta33", C.c_double),
        ("s2_term", C.c_int), ("s3_term", C.c_int), ("damped", C.c_int),
        ("bS3_s", C.c_double * 289), ("gS3_s", C.c_double * 289), ("r0S3_s", C.c_double * 289),
        ("bS3_l", C.c_double * 289), ("gS3_l", C.c_double * 289), ("r0S3_l", C.c_double * 289),
        ("cs3_s", C.c_double * 5000), ("cs3_l", C.c_double * 5000),
        ("nlin", C.c_int),
        ("ind_lin", C.c_int * (17 * 17 * 17 * 8)),
        ("nclass", C.c_int),
        ("nvdw", C.c_int),
        ("vdw", (C.c_double * 12) * 64),
        ("vdw_row", C.c_int * (50 * 50)),
    ]


_lib = None

# The compiler flags of the Makefile's build, reported beside every CPU timing of the oracle.
BUILD_FLAGS = "gcc -O3 -fopenmp -ffp-contract=off"


def build():
    """Compile the oracle with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = C.POINTER(C.c_int)
        mp = C.POINTER(OrcModel)
        d = C.c_double
        pd = C.POINTER(C.c_double)
        L.orc_tt.restype = d
        L.orc_tt.argtypes = [C.c_int, d, d]
        L.orc_dtt.restype = d
        L.orc_dtt.argtypes = [C.c_int, d, d]
        L.orc_fill_index.restype = C.c_int
        L.orc_fill_index.argtypes = [np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")]
        L.orc_ewald_setup.argtypes = [d, d, d, pd, ip, ip, ip]
        L.orc_threebody_term.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, d, pd, pd,
                                         dp, dp, dp, dp, dp, dp, dp, dp, dp, pd]
        L.orc_fs2_term_bohr.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, d, pd,
                                        dp, dp, dp, dp, dp, dp, pd]
        L.orc_ewald_self_correction.argtypes = [mp, d, d, dp, dp, dp, dp, dp, dp, C.c_int, pd,
                                                dp, dp, dp, pd]
        L.orc_ccpol23plus.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, d, pd, dp, dp, dp, pd]
        L.orc_rspace_ewald.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, d, d, pd,
                                       dp, dp, dp, pd]
        L.orc_kspace_ewald.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int,
                                       C.c_int, d, d, pd, dp, dp, dp, pd]
        L.orc_nb_induction.restype = C.c_int
        L.orc_nb_induction.argtypes = [mp, dp, dp, dp, dp, dp, dp, C.c_int, d, C.c_int, pd,
                                       dp, dp, dp, dp, dp, dp, pd, ip]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# --------------------------------------------------------------------------- readers
def _fortran_logical(tok: str) -> bool:
    t = tok.strip().strip(".").upper()
    return t.startswith("T")


@dataclass
class Inputs:
    """Values the reference reads from CONTROL, FIELD and the FS3 parameter files."""
    control: dict
    system_name: str
    nm: int
    ns: int
    npol: int
    names: list
    coords: np.ndarray          # (ns, 3) as read
    mass: np.ndarray
    charge: np.ndarray
    polarizability: np.ndarray
    vdw: list = field(default_factory=list)  # (an1, an2, [14 floats]) rows
    fs3_sr: dict | None = None
    fs3_lr: dict | None = None


def read_control(path) -> dict:
    """CONTROL, 17 list-directed records (initialization.f90:463-489)."""
    lines = Path(path).read_text().splitlines()
    tok = [ln.split() for ln in lines]
    c = {}
    c["pot_name"] = tok[0][0]
    c["ensemble"], c["taut"], c["taup"] = tok[1][0], float(tok[1][1]), float(tok[1][2])
    c["initial_config"] = tok[2][0]
    c["temp0"] = float(tok[3][0])
    c["pres0"] = float(tok[4][0])
    c["nsteps"] = int(tok[5][0])
    c["dt"] = float(tok[6][0])
    c["nequil"] = int(tok[7][0])
    c["rcut"] = float(tok[8][0])
    c["hist_freq"] = int(tok[9][0])
    c["rand_vcom"] = _fortran_logical(tok[10][0])
    c["rand_quat"] = _fortran_logical(tok[11][0])
    c["induction"] = _fortran_logical(tok[12][0])
    c["ind_model"], c["induction_type"], c["method"] = tok[12][1], tok[12][2], tok[12][3]
    c["nonadditive_3B"] = _fortran_logical(tok[13][0])
    c["S3_term"] = _fortran_logical(tok[13][1])
    c["S2_term"] = _fortran_logical(tok[13][2])
    c["rcut3"], c["alpha3"], c["r0_tilda"], c["delta33"] = (float(v) for v in tok[14][:4])
    c["restart"] = _fortran_logical(tok[15][0])
    c["check_forces"] = _fortran_logical(tok[16][0])
    c["hsize"] = float(tok[16][1])
    return c


def read_fs3_table(path) -> dict:
    """data3b_full / data3b_full_LR_4p5 (initialization.f90:642-701): header, 289 rows
    `b g r0 is js` read in (is, js) order, a header, nlin, then nlin rows `idx c`; the
    coefficients fill the array in row order."""
    lines = Path(path).read_text().splitlines()
    b = np.zeros(289)
    g = np.zeros(289)
    r0 = np.zeros(289)
    for n in range(289):
        t = lines[1 + n].split()
        b[n], g[n], r0[n] = float(t[0]), float(t[1]), float(t[2])
    nlin = int(lines[1 + 289 + 1].split()[0])
    cs = np.zeros(5000)
    for n in range(nlin):
        t = lines[1 + 289 + 2 + n].split()
        cs[n] = float(t[1])
    return {"b": b, "g": g, "r0": r0, "cs": cs, "nlin": nlin}


def read_inputs(directory) -> Inputs:
    d = Path(directory)
    control = read_control(d / "CONTROL")
    lines = (d / "FIELD").read_text().splitlines()
    system_name = lines[0].split()[0]
    nm = int(lines[1].split()[0])
    ns = int(lines[2].split()[0])
    npol = int(lines[3].split()[0])
    names, coords, mass, charge, pol = [], [], [], [], []
    for s in range(ns):
        t = lines[5 + s].split()
        names.append(t[0])
        coords.append([float(t[1]), float(t[2]), float(t[3])])
        mass.append(float(t[4]))
        charge.append(float(t[5]))
        pol.append(float(t[6]))
    npi = int(lines[5 + ns + 1].split()[0])
    vdw = []
    for k in range(npi):
        t = lines[5 + ns + 3 + k].split()
        vdw.append((t[0], t[1], [float(v) for v in t[2:16]]))
    inp = Inputs(control, system_name, nm, ns, npol, names, np.array(coords), np.array(mass),
                 np.array(charge), np.array(pol), vdw)
    if control["nonadditive_3B"]:
        inp.fs3_sr = read_fs3_table(d / "data3b_full")
        inp.fs3_lr = read_fs3_table(d / "data3b_full_LR_4p5")
    return inp


# ------------------------------------------------------------------ molecular frame
def jacobi(a: np.ndarray):
    """DL_POLY cyclic Jacobi diagonaliser restated from utility.f90:458-596 (processes
    the lower triangle; returns the rotated matrix and the eigenvector matrix)."""
    n = a.shape[0]
    a = a.copy()
    v = np.eye(n)
    rho = 1.0e-16
    tes = 0.0
    scl = 0.0
    for i in range(n):
        if abs(a[i, i]) > scl:
            scl = abs(a[i, i])
    for i in range(n):
        for j in range(i + 1):
            a[i, j] = a[i, j] / scl
    for i in range(1, n):
        for j in range(i):
            tes = tes + 2.0 * a[i, j] * a[i, j]
    tes = math.sqrt(tes)
    while tes > rho:
        tes = tes / float(n)
        if tes < rho:
            tes = rho
        passing = True
        while passing:
            passing = False
            for i in range(1, n):
                for j in range(i):
                    if abs(a[i, j]) >= tes:
                        passing = True
                        v1, v2, v3 = a[j, j], a[i, j], a[i, i]
                        u = 0.5 * (v1 - v3)
                        if abs(u) < rho:
                            omg = -1.0
                        else:
                            omg = -v2 / math.sqrt(v2 * v2 + u * u)
                            if u < 0.0:
                                omg = -omg
                        s = omg / math.sqrt(2.0 * (1.0 + math.sqrt(1.0 - omg * omg)))
                        c = math.sqrt(1.0 - s * s)
                        for k in range(n):
                            if k >= i:
                                tem = a[k, j] * c - a[k, i] * s
                                a[k, i] = a[k, j] * s + a[k, i] * c
                                a[k, j] = tem
                            elif k < j:
                                tem = a[j, k] * c - a[i, k] * s
                                a[i, k] = a[j, k] * s + a[i, k] * c
                                a[j, k] = tem
                            else:
                                tem = a[k, j] * c - a[i, k] * s
                                a[i, k] = a[k, j] * s + a[i, k] * c
                                a[k, j] = tem
                            tem = v[k, j] * c - v[k, i] * s
                            v[k, i] = v[k, j] * s + v[k, i] * c
                            v[k, j] = tem
                        a[j, j] = v1 * c * c + v3 * s * s - 2.0 * v2 * s * c
                        a[i, i] = v1 * s * s + v3 * c * c + 2.0 * v2 * s * c
                        a[i, j] = (v1 - v3) * s * c + v2 * (c * c - s * s)
    for i in range(n):
        for j in range(i + 1):
            a[i, j] = scl * a[i, j]
    return a, v


def principal_frame(inp: Inputs):
    """shift_to_com + principle_moment_inertia (initialization.f90:728-845).  Returns
    (pcoord (ns,3), pmi (3,), totm)."""
    ns = inp.ns
    totm = 0.0
    for s in range(ns):
        if inp.mass[s] != 0.0:
            totm = totm + inp.mass[s]
    coords = inp.coords.copy()
    r = [0.0, 0.0, 0.0]
    for s in range(ns):
        for a in range(3):
            r[a] = r[a] + inp.mass[s] * coords[s, a] / totm
    for s in range(ns):
        for a in range(3):
            coords[s, a] = coords[s, a] - r[a]
    rmi = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            for s in range(ns):
                rmi[i, j] = rmi[i, j] - inp.mass[s] * coords[s, i] * coords[s, j]
                if i == j:
                    rmi[i, j] = rmi[i, j] + inp.mass[s] * (
                        coords[s, 0] ** 2 + coords[s, 1] ** 2 + coords[s, 2] ** 2)
    rmi, rot = jacobi(rmi)
    pmi = np.array([rmi[0, 0], rmi[1, 1], rmi[2, 2]])
    pc = np.empty_like(coords)
    for s in range(ns):
        rx, ry, rz = coords[s]
        pc[s, 0] = rx * rot[0, 0] + ry * rot[1, 0] + rz * rot[2, 0]
        pc[s, 1] = rx * rot[0, 1] + ry * rot[1, 1] + rz * rot[2, 1]
        pc[s, 2] = rx * rot[0, 2] + ry * rot[1, 2] + rz * rot[2, 2]
    return pc, pmi, totm


class SiteFrame:
    """The molecular frame of the inputs (principal axes, moments, mass) with the site
    placement of molecular_sites.f90:14-47: what the box generator needs from a model, here
    computed by the oracle alone."""

    def __init__(self, inp: Inputs):
        self.pcoord, self.pmi, self.totm = principal_frame(inp)
        self.ns = inp.ns

    def get_double(self, name):
        if name != "totm":
            raise KeyError(name)
        return self.totm

    def sites(self, q, ld=None):
        return sites(self.pcoord, q, ld)


def quat_to_rot(q0, q1, q2, q3):
    """molecular_sites.f90:93-111 (row-major 3x3 flattened as rott(1..9)).  Fortran's
    integer power q0**2 is the product q0*q0 (numpy's float power can differ by an ulp)."""
    a0, a1, a2, a3 = q0 * q0, q1 * q1, q2 * q2, q3 * q3
    return np.array([
        a0 + a1 - a2 - a3, 2.0 * (q1 * q2 - q0 * q3), 2.0 * (q1 * q3 + q0 * q2),
        2.0 * (q1 * q2 + q0 * q3), a0 - a1 + a2 - a3, 2.0 * (q2 * q3 - q0 * q1),
        2.0 * (q1 * q3 - q0 * q2), 2.0 * (q2 * q3 + q0 * q1), a0 - a1 - a2 + a3])


def sites(pcoord: np.ndarray, q: np.ndarray, ld: int | None = None):
    """sites (molecular_sites.f90:14-47): site offsets from the COM for every molecule.
    q is (nm, 4).  Returns xs, ys, zs of shape (nm, ld)."""
    nm = q.shape[0]
    ns = pcoord.shape[0]
    ld = ld or ns
    xs = np.zeros((nm, ld))
    ys = np.zeros((nm, ld))
    zs = np.zeros((nm, ld))
    for j in range(nm):
        rott = quat_to_rot(*q[j])
        for s in range(ns):
            r1, r2, r3 = pcoord[s]
            xs[j, s] = r1 * rott[0] + r2 * rott[1] + r3 * rott[2]
            ys[j, s] = r1 * rott[3] + r2 * rott[4] + r3 * rott[5]
            zs[j, s] = r1 * rott[6] + r2 * rott[7] + r3 * rott[8]
    return xs, ys, zs


def ewald_setup(rcut: float, box: float, ewps: float = EWP):
    a = C.c_double()
    k1, k2, k3 = C.c_int(), C.c_int(), C.c_int()
    lib().orc_ewald_setup(ewps, rcut, box, C.byref(a), C.byref(k1), C.byref(k2), C.byref(k3))
    return a.value, k1.value, k2.value, k3.value


def make_model(inp: Inputs, nm: int, box: float, *, s2=None, s3=None,
               rcut3=None, alpha3=None, delta33=None) -> OrcModel:
    c = inp.control
    M = OrcModel()
    M.nm = nm
    M.ns = inp.ns
    M.npol = inp.npol
    for s in range(inp.ns):
        M.charge[s] = inp.charge[s]
        M.polarizability[s] = inp.polarizability[s]
    alp, k1, k2, k3 = ewald_setup(c["rcut"], box)
    M.alpha, M.kmax1, M.kmax2, M.kmax3 = alp, k1, k2, k3
    M.rcut = c["rcut"]
    M.rcutsd = c["rcut"] ** 2
    M.rcut3 = c["rcut3"] if rcut3 is None else rcut3
    M.rcutsd3 = M.rcut3 ** 2
    M.alpha3 = c["alpha3"] if alpha3 is None else alpha3
    M.delta33 = c["delta33"] if delta33 is None else delta33
    M.s2_term = int(c["S2_term"] if s2 is None else s2)
    M.s3_term = int(c["S3_term"] if s3 is None else s3)
    M.damped = int(c["induction_type"] == "damped")
    if inp.fs3_sr is not None:
        for n in range(289):
            M.bS3_s[n], M.gS3_s[n], M.r0S3_s[n] = inp.fs3_sr["b"][n], inp.fs3_sr["g"][n], inp.fs3_sr["r0"][n]
            M.bS3_l[n], M.gS3_l[n], M.r0S3_l[n] = inp.fs3_lr["b"][n], inp.fs3_lr["g"][n], inp.fs3_lr["r0"][n]
        for n in range(inp.fs3_sr["nlin"]):
            M.cs3_s[n] = inp.fs3_sr["cs"][n]
        for n in range(inp.fs3_lr["nlin"]):
            M.cs3_l[n] = inp.fs3_lr["cs"][n]
        M.nlin = inp.fs3_sr["nlin"]
    ind = np.zeros(17 * 17 * 17 * 8, dtype=np.int32)
    M.nclass = lib().orc_fill_index(ind)
    C.memmove(M.ind_lin, ind.ctypes.data, ind.nbytes)
    # ccpol23plus rows (initialization.f90:612-628: c0..c10 to internal units, x 418.4)
    M.nvdw = len(inp.vdw)
    for k, (a, b, p) in enumerate(inp.vdw):
        beta, c0, c1, c2, c3, c6, c8, c10, d1, d6, d8, d10 = p[:12]
        for n, v in enumerate((beta, c0 * 418.4, c1 * 418.4, c2 * 418.4, c3 * 418.4, c6 * 418.4,
                               c8 * 418.4, c10 * 418.4, d1, d6, d8, d10)):
            M.vdw[k][n] = v
    for i in range(50 * 50):
        M.vdw_row[i] = -1
    for si in range(inp.ns):
        for sj in range(inp.ns):
            for k, (a, b, p) in enumerate(inp.vdw):
                if (inp.names[si] == a and inp.names[sj] == b) or (inp.names[sj] == a and inp.names[si] == b):
                    M.vdw_row[si * 50 + sj] = k
                    break
    return M


def fill_index():
    ind = np.zeros(17 * 17 * 17 * 8, dtype=np.int32)
    n = lib().orc_fill_index(ind)
    return ind, n


# ------------------------------------------------------------------------ wrappers
def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class State:
    """Per-call outputs of the reference entry points (site forces accumulate)."""

    def __init__(self, nm, ld):
        self.fxs = np.zeros((nm, ld))
        self.fys = np.zeros((nm, ld))
        self.fzs = np.zeros((nm, ld))
        self.fxfs2 = np.zeros(nm)
        self.fyfs2 = np.zeros(nm)
        self.fzfs2 = np.zeros(nm)
        self.fxfs3 = np.zeros(nm)
        self.fyfs3 = np.zeros(nm)
        self.fzfs3 = np.zeros(nm)
        self.idmx = np.zeros((nm, ld))
        self.idmy = np.zeros((nm, ld))
        self.idmz = np.zeros((nm, ld))
        self.vir = C.c_double(0.0)


def threebody_term(M, x, y, z, xs, ys, zs, box, st: State):
    q2, q3 = C.c_double(0.0), C.c_double(0.0)
    ld = xs.shape[1]
    lib().orc_threebody_term(C.byref(M), _c(x), _c(y), _c(z), _c(xs), _c(ys), _c(zs), ld, box,
                             C.byref(q2), C.byref(q3), st.fxs, st.fys, st.fzs,
                             st.fxfs2, st.fyfs2, st.fzfs2, st.fxfs3, st.fyfs3, st.fzfs3,
                             C.byref(st.vir))
    return q2.value, q3.value


def fs2_term_bohr(M, xx, yy, zz, xxs, yys, zzs, boxi, st: State):
    q = C.c_double(0.0)
    lib().orc_fs2_term_bohr(C.byref(M), _c(xx), _c(yy), _c(zz), _c(xxs), _c(yys), _c(zzs),
                            xxs.shape[1], boxi, C.byref(q), st.fxs, st.fys, st.fzs,
                            st.fxfs2, st.fyfs2, st.fzfs2, C.byref(st.vir))
    return q.value


def ewald_self_correction(M, alp, box, x, y, z, xs, ys, zs, st: State):
    q = C.c_double(0.0)
    lib().orc_ewald_self_correction(C.byref(M), alp, box, _c(x), _c(y), _c(z), _c(xs), _c(ys),
                                    _c(zs), xs.shape[1], C.byref(q), st.fxs, st.fys, st.fzs,
                                    C.byref(st.vir))
    return q.value


def ccpol23plus(M, x, y, z, xs, ys, zs, box, st: State):
    """2-body CCpol23+ (vdw_ccpol23plus.f90:174-477): zeroes st's site forces of the ns
    sites and sets st.vir, as the reference does; returns the energy (kcal/mol)."""
    q = C.c_double(0.0)
    lib().orc_ccpol23plus(C.byref(M), _c(x), _c(y), _c(z), _c(xs), _c(ys), _c(zs),
                          xs.shape[1], box, C.byref(q), st.fxs, st.fys, st.fzs, C.byref(st.vir))
    return q.value


def rspace_ewald(M, x, y, z, xs, ys, zs, box, alp, st: State):
    q = C.c_double(0.0)
    lib().orc_rspace_ewald(C.byref(M), _c(x), _c(y), _c(z), _c(xs), _c(ys), _c(zs),
                           xs.shape[1], box, alp, C.byref(q), st.fxs, st.fys, st.fzs,
                           C.byref(st.vir))
    return q.value


def kspace_ewald(M, x, y, z, xs, ys, zs, lmax, mmax, nmax, alp, box, st: State):
    q = C.c_double(0.0)
    lib().orc_kspace_ewald(C.byref(M), _c(x), _c(y), _c(z), _c(xs), _c(ys), _c(zs),
                           xs.shape[1], lmax, mmax, nmax, alp, box, C.byref(q),
                           st.fxs, st.fys, st.fzs, C.byref(st.vir))
    return q.value


def nb_induction(M, x, y, z, xs, ys, zs, box, st: State, maxit: int = 500):
    q = C.c_double(0.0)
    it = C.c_int(0)
    status = lib().orc_nb_induction(C.byref(M), _c(x), _c(y), _c(z), _c(xs), _c(ys), _c(zs),
                                    xs.shape[1], box, maxit, C.byref(q), st.idmx, st.idmy,
                                    st.idmz, st.fxs, st.fys, st.fzs, C.byref(st.vir),
                                    C.byref(it))
    return q.value, status, it.value


def hot_path(M, x, y, z, xs, ys, zs, box, induction=True):
    """The reference force-evaluation sequence after the 2-body term (evolve.f90:842-877):
    Ewald self, real, reciprocal; induction; three-body.  Returns (energies, State)."""
    nm, ld = xs.shape
    st = State(nm, ld)
    e = {}
    e["scpe"] = ewald_self_correction(M, M.alpha, box, x, y, z, xs, ys, zs, st)
    e["rcpe"] = rspace_ewald(M, x, y, z, xs, ys, zs, box, M.alpha, st)
    e["kcpe"] = kspace_ewald(M, x, y, z, xs, ys, zs, M.kmax1, M.kmax2, M.kmax3, M.alpha, box, st)
    if induction:
        e["indpe"], status, it = nb_induction(M, x, y, z, xs, ys, zs, box, st)
        e["ind_status"], e["ind_iters"] = status, it
    e["fs2pe"], e["fs3pe"] = threebody_term(M, x, y, z, xs, ys, zs, box, st)
    e["vir"] = st.vir.value
    return e, st


# ------------------------------------------------------------------- NVE integration
BOLTZ = 8.31451115e-1     # (10 J/mol)/K (utility.f90)
PRSUNT = 0.163882576      # internal pressure unit to katm


def force_field(M, inp_flags, pcoord, x, y, z, q, box, ld):
    """sites + every force routine of one MD step, in nve_1's order (evolve.f90:800-877):
    ccpol23plus (zeroes the forces and sets vir), Ewald self/real/reciprocal, nb_induction,
    threebody_term.  Returns (xs, ys, zs, State, energies)."""
    induction, three_body = inp_flags
    nm = len(x)
    xs, ys, zs = sites(pcoord, q, ld)
    st = State(nm, ld)
    e = {}
    e["vdwpe"] = ccpol23plus(M, x, y, z, xs, ys, zs, box, st)
    e["scpe"] = ewald_self_correction(M, M.alpha, box, x, y, z, xs, ys, zs, st)
    e["rcpe"] = rspace_ewald(M, x, y, z, xs, ys, zs, box, M.alpha, st)
    e["kcpe"] = kspace_ewald(M, x, y, z, xs, ys, zs, M.kmax1, M.kmax2, M.kmax3, M.alpha, box, st)
    e["indpe"] = 0.0
    if induction:
        e["indpe"], status, _ = nb_induction(M, x, y, z, xs, ys, zs, box, st)
        assert status == 0
    e["fs2pe"] = e["fs3pe"] = 0.0
    if three_body:
        e["fs2pe"], e["fs3pe"] = threebody_term(M, x, y, z, xs, ys, zs, box, st)
    return xs, ys, zs, st, e


def _com_force_torque(st, xs, ys, zs, ns, three_body):
    """evolve.f90:664-704: per-molecule force and torque from the site forces (plus the
    three-body COM forces), and the site-site to molecule-molecule virial correction."""
    fxs, fys, fzs = st.fxs[:, :ns], st.fys[:, :ns], st.fzs[:, :ns]
    sx, sy, sz = xs[:, :ns], ys[:, :ns], zs[:, :ns]
    nm = fxs.shape[0]
    F = np.zeros((nm, 3))
    T = np.zeros((nm, 3))
    lvir = 0.0
    for i in range(nm):
        qf = [0.0, 0.0, 0.0]
        qt = [0.0, 0.0, 0.0]
        for s in range(ns):
            qf[0] += fxs[i, s]
            qf[1] += fys[i, s]
            qf[2] += fzs[i, s]
            qt[0] += sy[i, s] * fzs[i, s] - sz[i, s] * fys[i, s]
            qt[1] += sz[i, s] * fxs[i, s] - sx[i, s] * fzs[i, s]
            qt[2] += sx[i, s] * fys[i, s] - sy[i, s] * fxs[i, s]
            lvir += fxs[i, s] * sx[i, s] + fys[i, s] * sy[i, s] + fzs[i, s] * sz[i, s]
        F[i] = qf
        T[i] = qt
        if three_body:
            F[i, 0] += st.fxfs2[i] + st.fxfs3[i]
            F[i, 1] += st.fyfs2[i] + st.fyfs3[i]
            F[i, 2] += st.fzfs2[i] + st.fzfs3[i]
    return F, T, lvir


def _quat_torque_and_momenta(q, T, J):
    """Principal-frame torque, quaternion torque and quaternion momenta (evolve.f90:712-741)."""
    q0, q1, q2, q3 = q
    r = quat_to_rot(q0, q1, q2, q3)
    tqx = T[0] * r[0] + T[1] * r[3] + T[2] * r[6]
    tqy = T[0] * r[1] + T[1] * r[4] + T[2] * r[7]
    tqz = T[0] * r[2] + T[1] * r[5] + T[2] * r[8]
    qt = [2.0 * (-q1 * tqx - q2 * tqy - q3 * tqz), 2.0 * (q0 * tqx - q3 * tqy + q2 * tqz),
          2.0 * (q3 * tqx + q0 * tqy - q1 * tqz), 2.0 * (-q2 * tqx + q1 * tqy + q0 * tqz)]
    ox, oy, oz = J
    p = [2.0 * (-q1 * ox - q2 * oy - q3 * oz), 2.0 * (q0 * ox - q3 * oy + q2 * oz),
         2.0 * (q3 * ox + q0 * oy - q1 * oz), 2.0 * (-q2 * ox + q1 * oy + q0 * oz)]
    return qt, p


def _momenta_to_j(q, p):
    q0, q1, q2, q3 = q
    return [0.5 * (-q1 * p[0] + q0 * p[1] + q3 * p[2] - q2 * p[3]),
            0.5 * (-q2 * p[0] - q3 * p[1] + q0 * p[2] + q1 * p[3]),
            0.5 * (-q3 * p[0] + q2 * p[1] - q1 * p[2] + q0 * p[3])]


def nosquish(tstep, q, p, pmi):
    """evolve.f90:8107-8203: free rotation of a rigid body by symplectic splitting, 10
    sub-steps of z/2, y/2, x, y/2, z/2 rotations."""
    qq0, qq1, qq2, qq3 = q
    pp0, pp1, pp2, pp3 = p
    mrot = 10
    ov4, ov8 = 0.25, 0.125
    trstep = tstep / float(mrot)
    for _ in range(mrot):
        zetaz = ov8 / pmi[2] * trstep * (-pp0 * qq3 + pp1 * qq2 - pp2 * qq1 + pp3 * qq0)
        cs, sn = np.cos(zetaz), np.sin(zetaz)
        qn1 = [cs * qq0 - sn * qq3, cs * qq1 + sn * qq2, cs * qq2 - sn * qq1, cs * qq3 + sn * qq0]
        pq2 = [cs * pp0 - sn * pp3, cs * pp1 + sn * pp2, cs * pp2 - sn * pp1, cs * pp3 + sn * pp0]
        zetay = ov8 / pmi[1] * trstep * (-pq2[0] * qn1[2] - pq2[1] * qn1[3] + pq2[2] * qn1[0] + pq2[3] * qn1[1])
        cs, sn = np.cos(zetay), np.sin(zetay)
        qn2 = [cs * qn1[0] - sn * qn1[2], cs * qn1[1] - sn * qn1[3], cs * qn1[2] + sn * qn1[0], cs * qn1[3] + sn * qn1[1]]
        pq3 = [cs * pq2[0] - sn * pq2[2], cs * pq2[1] - sn * pq2[3], cs * pq2[2] + sn * pq2[0], cs * pq2[3] + sn * pq2[1]]
        zetax = ov4 / pmi[0] * trstep * (-pq3[0] * qn2[1] + pq3[1] * qn2[0] + pq3[2] * qn2[3] - pq3[3] * qn2[2])
        cs, sn = np.cos(zetax), np.sin(zetax)
        qn3 = [cs * qn2[0] - sn * qn2[1], cs * qn2[1] + sn * qn2[0], cs * qn2[2] + sn * qn2[3], cs * qn2[3] - sn * qn2[2]]
        pq4 = [cs * pq3[0] - sn * pq3[1], cs * pq3[1] + sn * pq3[0], cs * pq3[2] + sn * pq3[3], cs * pq3[3] - sn * pq3[2]]
        zetay = ov8 / pmi[1] * trstep * (-pq4[0] * qn3[2] - pq4[1] * qn3[3] + pq4[2] * qn3[0] + pq4[3] * qn3[1])
        cs, sn = np.cos(zetay), np.sin(zetay)
        qn2 = [cs * qn3[0] - sn * qn3[2], cs * qn3[1] - sn * qn3[3], cs * qn3[2] + sn * qn3[0], cs * qn3[3] + sn * qn3[1]]
        pq3 = [cs * pq4[0] - sn * pq4[2], cs * pq4[1] - sn * pq4[3], cs * pq4[2] + sn * pq4[0], cs * pq4[3] + sn * pq4[1]]
        zetaz = ov8 / pmi[2] * trstep * (-pq3[0] * qn2[3] + pq3[1] * qn2[2] - pq3[2] * qn2[1] + pq3[3] * qn2[0])
        cs, sn = np.cos(zetaz), np.sin(zetaz)
        qq0, qq1, qq2, qq3 = (cs * qn2[0] - sn * qn2[3], cs * qn2[1] + sn * qn2[2],
                              cs * qn2[2] - sn * qn2[1], cs * qn2[3] + sn * qn2[0])
        pp0, pp1, pp2, pp3 = (cs * pq3[0] - sn * pq3[3], cs * pq3[1] + sn * pq3[2],
                              cs * pq3[2] - sn * pq3[1], cs * pq3[3] + sn * pq3[0])
    return [qq0, qq1, qq2, qq3], [pp0, pp1, pp2, pp3]


class MDState:
    """Rigid-water MD state of the reference's NVE integrator: COM positions x, y, z (A),
    COM velocities v (nm, 3) (A/ps), unit quaternions q (nm, 4), principal-frame angular
    momenta j (nm, 3) (amu A^2/ps)."""

    def __init__(self, x, y, z, v, q, j):
        self.x, self.y, self.z = (np.array(a, dtype=np.float64) for a in (x, y, z))
        self.v = np.array(v, dtype=np.float64)
        self.q = np.array(q, dtype=np.float64)
        self.j = np.array(j, dtype=np.float64)


def state_stats(M, flags, pcoord, pmi, totm, s: MDState, box, ld):
    """Statistics of the state itself, no step (initialization.f90:76-89, 357-399): the
    energies of a force evaluation there, kinetic energies of v and j, temperature, virial
    (vir + sum f . xs) and pressure, in the units of nve_run's rows."""
    nm = len(s.x)
    ns = pcoord.shape[0]
    xs, ys, zs, st, e = force_field(M, flags, pcoord, s.x, s.y, s.z, s.q, box, ld)
    _, _, lvir = _com_force_torque(st, xs, ys, zs, ns, flags[1])
    tke = 0.5 * totm * float(np.sum(s.v[:, 0] ** 2 + s.v[:, 1] ** 2 + s.v[:, 2] ** 2))
    rke = 0.5 * float(np.sum(s.j[:, 0] ** 2 / pmi[0] + s.j[:, 1] ** 2 / pmi[1] + s.j[:, 2] ** 2 / pmi[2]))
    cpe = e["scpe"] + e["rcpe"] + e["kcpe"]
    pe3 = e["fs2pe"] + e["fs3pe"]
    pe = e["vdwpe"] + cpe + e["indpe"] + pe3
    qvir = st.vir.value + lvir
    return {"vdwpe": e["vdwpe"], "cpe": cpe, "indpe": e["indpe"], "pe3b": pe3, "pe": pe,
            "tke": tke / 418.4, "rke": rke / 418.4, "te": (tke + rke) / 418.4 + pe,
            "sys_temp": 2.0 * (tke + rke) / (3.0 * BOLTZ * (2.0 * nm - 1.0)),
            "vir": qvir / 418.4, "pres": PRSUNT * (2.0 * tke - qvir) / (3.0 * box ** 3)}


BETTA = 0.007372  # isothermal compressibility of the Berendsen barostat (evolve.f90:7514)


def nve_run(M, flags, pcoord, pmi, totm, s: MDState, box, dt, nsteps, ld, temp0=None,
            nequil=0):
    """nve_1 (evolve.f90:621-1061) for nsteps steps with the oracle's forces, starting from
    a force evaluation at the initial state (initialization.f90:357-381).  Returns the per-step
    energies (kcal/mol: vdw, coul, ind, 3b, pe, ke, te; temperature; virial, pressure).
    During the first nequil steps the velocities and angular momenta are rescaled after the
    step to temp0 (md.f90:187-193, equilibrationGRU utility.f90:353-368 with
    rescale_velocities :257-275 and the temperatures of trans_temp / rot_temp :196-227);
    the step's statistics are those before the rescale."""
    return md_run(M, flags, pcoord, pmi, totm, s, box, dt, nsteps, ld, "nve", temp0=temp0,
                  nequil=nequil)


def md_run(M, flags, pcoord, pmi, totm, s: MDState, box, dt, nsteps, ld, ensemble, temp0=None,
           nequil=0, taut=None, pres0=None, taup=None, rcut=None, chit0=0.0, chip0=0.0):
    """The reference's rigid-molecule integrators with the oracle's forces:
    - "nve": nve_1 (evolve.f90:621-1061), with the equilibration rescale of nve_run;
    - "nvt_b": nvt_b (evolve.f90:1063-1644): nve_1's steps without the periodic wrap, then
      velocities and angular momenta times chit = sqrt(1 + dt/taut (temp0/T - 1)) of the
      system temperature T; the statistics are those after the scaling;
    - "npt_b": npt_b_1 (evolve.f90:7485-8104): before the step the Berendsen barostat
      chip = 1 + betta dt (P - pres0)/taup from the current kinetic energy and virial scales
      the volume by chip, the box by chip^(1/3) and the centres inside the drift
      (x = s x + dt v), with k-max reset for the new box (ewald_setup, rcut); after it the
      system's COM velocity (utility.f90:293-351) is removed, the nvt_b thermostat applied,
      and the centres are wrapped into the new box.
    - "nvt_h": nvt_hov_3 (evolve.f90:3316-3834): nve_1's step, then the Nose-Hoover
      thermostat of nptqscl_t_dl4 (evolve.f90:8305-8369) with its step dt/4, from the
      thermostat variable chit (chit0 at the start, 0 for a fresh run, initialization.f90:169);
      the statistics follow the scaling;
    - "npt_h": npt_hov_2 (evolve.f90:5567-6155): before and after the step the thermostat /
      barostat / thermostat sequence of nptqscl_t_dl4 (dt/4) and nptqscl_p_dl4 (dt/2,
      :8435-8495); the volume grows by exp(3 dt chip) and the centres are scaled by
      exp(dt chip) about the system's centre (taken as the mean of the centres: the site
      offsets sum to zero about each centre) in the drift; the forces of the step still use
      the old box and its k-max; the new box takes effect after the step, before the COM
      velocity is removed and the centres wrapped;
    - "npt_mtk": npt_mtk (evolve.f90:6158-6745): npt_h with the MTK barostat
      nptqscl_p_dl4_mtk (:8497-8558, kinetic term and velocity scaling times 1 + 3/(dof-dofr))
      and the centres scaled about the origin.
    pres0 is in internal units (katm / PRSUNT, initialization.f90:160).  Rows carry the box
    and volume of the step and, for nvt_h, chit and the conserved quantity.  Mutates s;
    returns the per-step rows."""
    nm = len(s.x)
    ns = pcoord.shape[0]
    three_body = flags[1]
    volm = box ** 3.0
    xs, ys, zs, st, e = force_field(M, flags, pcoord, s.x, s.y, s.z, s.q, box, ld)
    out = []
    chit, chip, cint = chit0, chip0, 0.0
    dof, dofr = 6.0 * nm - 3.0, 3.0 * nm
    sigma0 = dof * BOLTZ * (temp0 or 0.0) / 2.0  # sigma_Text, utility.f90:240-255
    qmass, ceng = 2.0 * sigma0 * (taut or 0.0) ** 2, 2.0 * sigma0
    pmass = 0.0
    nh_baro = ensemble in ("npt_h", "npt_mtk")
    fmtk = 3.0 / (dof - dofr) if ensemble == "npt_mtk" else 0.0  # evolve.f90:8510
    if nh_baro:  # evolve.f90:5644-5650
        tmpt = (2.0 * sigma0) / (BOLTZ * dof)
        ceng = 2.0 * sigma0 + BOLTZ * tmpt
        pmass = ((dof - dofr) + 3.0) * BOLTZ * tmpt * taup ** 2

    def kinetic():
        tke = 0.5 * totm * float(np.sum(s.v[:, 0] ** 2 + s.v[:, 1] ** 2 + s.v[:, 2] ** 2))
        rke = 0.5 * float(np.sum(s.j[:, 0] ** 2 / pmi[0] + s.j[:, 1] ** 2 / pmi[1] +
                                 s.j[:, 2] ** 2 / pmi[2]))
        return tke, rke

    def systemp(tke, rke):
        return 2.0 * (tke + rke) / (3.0 * BOLTZ * (2.0 * nm - 1.0))

    def thermo(ttt):  # nptqscl_t_dl4 (evolve.f90:8305-8369)
        nonlocal chit, cint
        h, q = 0.5 * ttt, 0.25 * ttt
        f1 = pmass * chip ** 2.0
        cint = cint + q * chit
        tke, rke = kinetic()
        chit = chit + h * (2.0 * (tke + rke) + f1 - ceng) / qmass
        cint = cint + h * chit
        sc = np.exp(-ttt * chit)
        s.v = sc * s.v
        s.j = sc * s.j
        tke, rke = tke * sc ** 2.0, rke * sc ** 2.0
        chit = chit + h * (2.0 * (tke + rke) + f1 - ceng) / qmass
        cint = cint + q * chit

    def baro(ttt, boxi, qvir):  # nptqscl_p_dl4 (evolve.f90:8435-8495)
        nonlocal chip
        h, q = 0.5 * ttt, 0.25 * ttt
        vi = boxi ** 3.0
        chip = chip * np.exp(-q * chit)
        tke, _ = kinetic()
        chip = chip + h * ((2.0 * (1.0 + fmtk) * tke - qvir) - 3.0 * pres0 * vi) / pmass
        chip = chip * np.exp(-q * chit)
        sc = np.exp(-ttt * (1.0 + fmtk) * chip)
        s.v = sc * s.v
        tke = tke * sc ** 2.0
        chip = chip * np.exp(-q * chit)
        chip = chip + h * ((2.0 * (1.0 + fmtk) * tke - qvir) - 3.0 * pres0 * vi) / pmass
        chip = chip * np.exp(-q * chit)

    for _ in range(nsteps):
        F, T, lvir0 = _com_force_torque(st, xs, ys, zs, ns, three_body)
        scale = 1.0
        centre = np.zeros(3)
        if nh_baro:
            qvir0 = st.vir.value + lvir0
            thermo(0.25 * dt)
            baro(0.5 * dt, box, qvir0)
            thermo(0.25 * dt)
            volmi = box ** 3.0 * np.exp(3.0 * dt * chip)
            boxi = volmi ** (1.0 / 3.0)
            scale = np.exp(dt * chip)
            centre = np.array([s.x.mean(), s.y.mean(), s.z.mean()])
        if ensemble == "npt_b":
            tke0, _ = kinetic()
            qpres = (2.0 * tke0 - (st.vir.value + lvir0)) / (3.0 * volm)
            chip = 1.0 + BETTA * dt * (qpres - pres0) / taup
            scale = chip ** (1.0 / 3.0)
            volm = volm * chip
            box = scale * box
            _, M.kmax1, M.kmax2, M.kmax3 = ewald_setup(rcut, box)
        P = np.zeros((nm, 4))
        for i in range(nm):
            qt, p = _quat_torque_and_momenta(s.q[i], T[i], s.j[i])
            P[i] = [p[k] + qt[k] * 0.5 * dt for k in range(4)]
            s.v[i] = s.v[i] + 0.5 * F[i] * dt / totm
        if ensemble == "npt_h":  # evolve.f90:5708-5712
            s.x = scale * (s.x - centre[0]) + dt * s.v[:, 0] + centre[0]
            s.y = scale * (s.y - centre[1]) + dt * s.v[:, 1] + centre[1]
            s.z = scale * (s.z - centre[2]) + dt * s.v[:, 2] + centre[2]
        else:
            s.x = scale * s.x + dt * s.v[:, 0]
            s.y = scale * s.y + dt * s.v[:, 1]
            s.z = scale * s.z + dt * s.v[:, 2]
        for i in range(nm):
            qn, pn = nosquish(dt, list(s.q[i]), list(P[i]), pmi)
            s.q[i] = qn
            s.j[i] = _momenta_to_j(qn, pn)
        xs, ys, zs, st, e = force_field(M, flags, pcoord, s.x, s.y, s.z, s.q, box, ld)
        F, T, lvir = _com_force_torque(st, xs, ys, zs, ns, three_body)
        for i in range(nm):
            qt, p = _quat_torque_and_momenta(s.q[i], T[i], s.j[i])
            p = [p[k] + qt[k] * 0.5 * dt for k in range(4)]
            s.v[i] = s.v[i] + 0.5 * F[i] * dt / totm
            s.j[i] = _momenta_to_j(s.q[i], p)
        if nh_baro:  # evolve.f90:6061-6080
            thermo(0.25 * dt)
            baro(0.5 * dt, boxi, st.vir.value + lvir)
            thermo(0.25 * dt)
            box, volm = boxi, volmi
        tke, rke = kinetic()
        if ensemble in ("npt_b", "npt_h", "npt_mtk"):  # utility.f90:293-351: remove the COM velocity
            vcom = np.zeros(3)
            for i in range(nm):
                vcom = vcom + totm * s.v[i] / (nm * totm)
            s.v = s.v - vcom
            tke, rke = kinetic()
        if ensemble in ("nvt_b", "npt_b"):
            chit = np.sqrt(1.0 + dt / taut * (temp0 / systemp(tke, rke) - 1.0))
            s.v = chit * s.v
            s.j = chit * s.j
            tke, rke = kinetic()
        if ensemble == "nvt_h":  # nptqscl_t_dl4 with ttt = dt/4, pmass = chip = 0
            tq = 0.25 * dt
            hq, qq = 0.5 * tq, 0.25 * tq
            cint = cint + qq * chit
            chit = chit + hq * (2.0 * (tke + rke) - ceng) / qmass
            cint = cint + hq * chit
            sc = np.exp(-tq * chit)
            s.v = sc * s.v
            s.j = sc * s.j
            tke, rke = tke * sc ** 2.0, rke * sc ** 2.0
            chit = chit + hq * (2.0 * (tke + rke) - ceng) / qmass
            cint = cint + qq * chit
            tke, rke = kinetic()
        if ensemble in ("nve", "npt_b", "nvt_h", "npt_h", "npt_mtk"):
            s.x = s.x - box * np.round(s.x / box)
            s.y = s.y - box * np.round(s.y / box)
            s.z = s.z - box * np.round(s.z / box)
        cpe = e["scpe"] + e["rcpe"] + e["kcpe"]
        pe3 = e["fs2pe"] + e["fs3pe"]
        pe = e["vdwpe"] + cpe + e["indpe"] + pe3
        qvir = st.vir.value + lvir
        out.append({"vdwpe": e["vdwpe"], "cpe": cpe, "indpe": e["indpe"], "pe3b": pe3, "pe": pe,
                    "tke": tke / 418.4, "rke": rke / 418.4, "te": (tke + rke) / 418.4 + pe,
                    "sys_temp": systemp(tke, rke), "vir": qvir / 418.4,
                    "pres": PRSUNT * (2.0 * tke - qvir) / (3.0 * volm), "box": box,
                    "volm": volm, "chit": chit, "chip": chip,
                    "consv": 0.5 * qmass * chit ** 2.0 + ceng * cint + (
                        0.5 * pmass * chip ** 2.0 + pres0 * volm if nh_baro else 0.0)})
        if ensemble == "nve" and len(out) <= nequil:
            ttemp = 2.0 * tke / ((3.0 * nm - 3.0) * BOLTZ)
            rtemp = 2.0 * rke / ((3.0 * nm) * BOLTZ)
            s.v = s.v * np.sqrt(temp0 / ttemp)
            s.j = s.j * np.sqrt(temp0 / rtemp)
    return out
