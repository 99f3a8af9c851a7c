"""Python mirror of the reference's hot-path entry points, over the C ABI.

Names, argument meaning, units and side effects follow the Fortran module procedures of
ommair/CCpol23_plus_2025_MBMD (ewald.f90, nb_induction_model.f90,
threebody_potential.f90): positions in Angstrom; energies returned in kcal/mol; site forces
accumulate into ``fxs/fys/fzs`` (internal units, 10 J/mol/A); 3-body COM forces are
overwritten; the virial accumulates into ``vir`` (a 1-element float64 array, standing in
for the module global).  Site arrays are ``(nm, ld)`` float64, site index fastest.
Errors raise :class:`CcpError` where the reference would ``stop``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import CcpEnergies, check, ptr

DATA = Path(__file__).resolve().parent / "data"


def data_dir(variant: str) -> Path:
    """Parameter directory shipped with the package: "fs3" or "fs2fs3"."""
    return DATA / variant


NPHASE = 10  # CCP_NPHASE


def _device_array(t, shape, name, device=None):
    """Checks that ``t`` is a contiguous float64 CUDA tensor of ``shape`` on ``device`` (an
    ordinal; None = the current device) and returns its device address.  The library reads and writes these buffers
    through raw pointers, so a wrong dtype, stride, size or device would make its kernels
    read or write outside them; every such case is refused here instead."""
    import torch
    if not isinstance(t, torch.Tensor):
        raise ValueError(f"{name}: expected a torch tensor, got {type(t).__name__}")
    if not t.is_cuda:
        raise ValueError(f"{name}: expected a CUDA tensor, got one on {t.device}")
    if t.dtype != torch.float64:
        raise ValueError(f"{name}: expected float64, got {t.dtype}")
    if device is None:
        device = torch.cuda.current_device()
    if t.device.index != device:
        raise ValueError(f"{name}: on cuda:{t.device.index}, expected cuda:{device}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name}: shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: must be contiguous")
    return t.data_ptr()


def _optional_device_array(t, shape, name, device):
    return None if t is None else _device_array(t, shape, name, device)


def _site_layout(xs, ns, name="xs"):
    """(nm, ld) of a site array, with ld >= the model's sites per molecule."""
    if len(xs.shape) != 2:
        raise ValueError(f"{name}: expected (nm, ld), got shape {tuple(xs.shape)}")
    nm, ld = int(xs.shape[0]), int(xs.shape[1])
    if ld < ns:
        raise ValueError(f"{name}: ld = {ld} is below the model's {ns} sites per molecule")
    return nm, ld


class Model:
    """Parameters read from CONTROL, FIELD, data3b_full, data3b_full_LR_4p5."""

    def __init__(self, directory):
        L = _lib.lib()
        h = C.c_void_p()
        check(L.ccp_model_load(str(directory).encode(), C.byref(h)))
        self._h = h
        self._free = L.ccp_model_free  # kept: module globals may be gone at interpreter exit

    def __del__(self):
        if getattr(self, "_h", None):
            self._free(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def get_int(self, name):
        v = C.c_int()
        check(_lib.lib().ccp_model_get_int(self._h, name.encode(), C.byref(v)))
        return v.value

    def get_double(self, name):
        v = C.c_double()
        check(_lib.lib().ccp_model_get_double(self._h, name.encode(), C.byref(v)))
        return v.value

    def set(self, name, value):
        L = _lib.lib()
        if isinstance(value, (bool, int, np.integer)) and name not in ("rcut", "rcut3", "alpha3", "delta33"):
            check(L.ccp_model_set_int(self._h, name.encode(), int(value)))
        else:
            check(L.ccp_model_set_double(self._h, name.encode(), float(value)))

    def array(self, name, n):
        out = np.zeros(n)
        check(_lib.lib().ccp_model_get_array(self._h, name.encode(), out.ctypes.data, n))
        return out

    @property
    def ns(self):
        return self.get_int("ns")

    @property
    def npol(self):
        return self.get_int("npol")

    @property
    def charge(self):
        return self.array("charge", self.ns)

    @property
    def polarizability(self):
        return self.array("polarizability", self.ns)

    @property
    def mass(self):
        return self.array("mass", self.ns)

    @property
    def pcoord(self):
        return self.array("pcoord", self.ns * 3).reshape(self.ns, 3)

    @property
    def pmi(self):
        return self.array("pmi", 3)

    def sites(self, q: np.ndarray, ld: int | None = None):
        """Site offsets from the COM for quaternions q (nm, 4) (molecular_sites.f90:14-47)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        nm = q.shape[0]
        ld = ld or self.ns
        xs, ys, zs = (np.zeros((nm, ld)) for _ in range(3))
        check(_lib.lib().ccp_sites(self._h, nm, q.ctypes.data, ld, xs.ctypes.data, ys.ctypes.data,
                                   zs.ctypes.data))
        return xs, ys, zs


def fma_peak_tflops(device: int = 0, precision: str = "fp64") -> float:
    """Measured FMA-pipe peak of the device (TFLOP/s)."""
    v = C.c_double()
    prec = {"fp64": _lib.CCP_FP64, "mixed": _lib.CCP_MIXED}[precision]
    check(_lib.lib().ccp_device_fma_peak(device, prec, C.byref(v)))
    return v.value


def mufu_peak_tops(device: int = 0) -> float:
    """Measured special-function (MUFU exp) peak of the device (Tops/s)."""
    v = C.c_double()
    check(_lib.lib().ccp_device_mufu_peak(device, C.byref(v)))
    return v.value


def ewald_setup(ewps: float, rcut: float, box: float):
    """ewald.f90:17-43 -> (alpha, kmax1, kmax2, kmax3)."""
    a = C.c_double()
    k1, k2, k3 = C.c_int(), C.c_int(), C.c_int()
    check(_lib.lib().ccp_ewald_setup(ewps, rcut, box, C.byref(a), C.byref(k1), C.byref(k2),
                                     C.byref(k3)))
    return a.value, k1.value, k2.value, k3.value


def kspace_ewald_fixed(model: Model, x, y, z, xs, ys, zs, lmax, mmax, nmax, alp, box, qkcpe,
                       fxs, fys, fzs, vir, stream: int | None = None) -> None:
    """kspace_ewald (ewald.f90:754-1173) on device arrays with the library's fixed scratch:
    no device memory is allocated.  All arrays are contiguous torch CUDA float64 tensors on
    the current device: x, y, z (nm,), xs, ys, zs and the forces (nm, ld); qkcpe and vir
    have one element each.  Forces and vir are added to, qkcpe is overwritten.  The work is
    enqueued on `stream` (a cudaStream_t address, None = the legacy default stream) and is
    not waited for.  Arguments that do not match raise ValueError before the library is
    called."""
    dev = None  # the current device
    nm, ld = _site_layout(xs, model.ns)
    a = [_device_array(t, (nm,), n, dev) for t, n in ((x, "x"), (y, "y"), (z, "z"))]
    a += [_device_array(t, (nm, ld), n, dev) for t, n in ((xs, "xs"), (ys, "ys"), (zs, "zs"))]
    q = _device_array(qkcpe, (1,), "qkcpe", dev)
    f = [_device_array(t, (nm, ld), n, dev) for t, n in ((fxs, "fxs"), (fys, "fys"), (fzs, "fzs"))]
    v = _device_array(vir, (1,), "vir", dev)
    check(_lib.lib().ccp_kspace_ewald_fixed(
        model.handle, nm, *a, ld, lmax, mmax, nmax, alp, box, q, *f, v, stream))


@dataclass
class HotPathResult:
    energies: dict
    fxs: np.ndarray
    fys: np.ndarray
    fzs: np.ndarray
    fxfs2: np.ndarray
    fyfs2: np.ndarray
    fzfs2: np.ndarray
    fxfs3: np.ndarray
    fyfs3: np.ndarray
    fzfs3: np.ndarray
    idmx: np.ndarray
    idmy: np.ndarray
    idmz: np.ndarray


def _energies(e: CcpEnergies) -> dict:
    return {k: getattr(e, k) for k, _ in CcpEnergies._fields_}


class Context:
    """Device-resident state for boxes of ``nm`` molecules on one GPU."""

    def __init__(self, model: Model, nm: int, box0: float, device: int = 0,
                 precision: str = "fp64"):
        prec = {"fp64": _lib.CCP_FP64, "mixed": _lib.CCP_MIXED}[precision]
        h = C.c_void_p()
        check(_lib.lib().ccp_context_create(model.handle, nm, box0, device, prec, C.byref(h)))
        self._h = h
        self.model = model
        self.nm = nm
        self.device = device
        self.precision = precision
        self.stream = None  # cudaStream_t address set by set_stream (None: the context's own)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ccp_context_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_ewald(self, alpha, k1, k2, k3):
        check(_lib.lib().ccp_context_set_ewald(self._h, alpha, k1, k2, k3))

    def set_maxit(self, maxit):
        check(_lib.lib().ccp_context_set_maxit(self._h, maxit))

    def set_stream(self, stream_ptr: int | None):
        """Enqueue the context's work on a caller's CUDA stream (a cudaStream_t address, e.g.
        ``torch.cuda.current_stream().cuda_stream``); None returns to the context's own."""
        check(_lib.lib().ccp_context_set_stream(self._h, stream_ptr))
        self.stream = stream_ptr

    def _device_args(self, x, y, z, xs, ys, zs, outs):
        """Validated device addresses of the inputs and of the optional outputs (site arrays
        (nm, ld), COM-force arrays (nm,), dipoles (nm, ld), in that order of ``outs``)."""
        nm, ld = _site_layout(xs, self.model.ns)
        if nm != self.nm:
            raise ValueError(f"xs: {nm} molecules, the context holds {self.nm}")
        d = self.device
        a = [_device_array(t, (nm,), n, d) for t, n in ((x, "x"), (y, "y"), (z, "z"))]
        a += [_device_array(t, (nm, ld), n, d) for t, n in ((xs, "xs"), (ys, "ys"), (zs, "zs"))]
        shapes = [(nm, ld)] * 3 + [(nm,)] * 6 + [(nm, ld)] * 3
        names = ["fxs", "fys", "fzs", "fxfs2", "fyfs2", "fzfs2", "fxfs3", "fyfs3", "fzfs3",
                 "idmx", "idmy", "idmz"]
        o = [_optional_device_array(t, sh, n, d) for t, sh, n in zip(outs, shapes, names)]
        return a, ld, o

    def set_option(self, name: str, value: int):
        """Execution options of the dipole solve: "graph_loop", "phase_matrix" (0/1)."""
        check(_lib.lib().ccp_context_set_option(self._h, name.encode(), int(value)))

    def get_option(self, name: str) -> int:
        v = C.c_int()
        check(_lib.lib().ccp_context_get_option(self._h, name.encode(), C.byref(v)))
        return v.value

    def set_timing(self, on: bool = True):
        check(_lib.lib().ccp_context_set_timing(self._h, int(on)))

    def phase_ms(self) -> np.ndarray:
        """Durations (ms) of the last evaluation's phases, in the order of CCP_NPHASE's
        comment: packing+neighbours, real space, reciprocal, induction set-up, dipole
        iteration, induction forces, FS2, FS3 triple list, FS3 kernel, 2-body term."""
        out = np.zeros(NPHASE)
        check(_lib.lib().ccp_context_phase_ms(self._h, out.ctypes.data, NPHASE))
        return out

    def last_launches(self) -> int:
        v = C.c_int()
        check(_lib.lib().ccp_context_last_launches(self._h, C.byref(v)))
        return v.value

    # -- reference entry points -------------------------------------------------------
    def ewald_self_correction(self, alp, box, x, y, z, xs, ys, zs, fxs, fys, fzs, vir):
        q = C.c_double()
        v = C.c_double(float(vir[0]))
        check(_lib.lib().ccp_ewald_self_correction(self._h, alp, box, ptr(x), ptr(y), ptr(z),
                                                   ptr(xs), ptr(ys), ptr(zs), xs.shape[1],
                                                   C.byref(q), ptr(fxs), ptr(fys), ptr(fzs),
                                                   C.byref(v)))
        vir[0] = v.value
        return q.value

    def rspace_ewald(self, x, y, z, xs, ys, zs, box, alp, fxs, fys, fzs, vir):
        q = C.c_double()
        v = C.c_double(float(vir[0]))
        check(_lib.lib().ccp_rspace_ewald(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys),
                                          ptr(zs), xs.shape[1], box, alp, C.byref(q), ptr(fxs),
                                          ptr(fys), ptr(fzs), C.byref(v)))
        vir[0] = v.value
        return q.value

    def ccpol23plus(self, x, y, z, xs, ys, zs, box, fxs, fys, fzs, vir):
        """vdw_ccpol23plus.f90:174-477; overwrites fxs.. and vir[0] as the reference does."""
        q = C.c_double()
        ld = xs.shape[1]
        check(_lib.lib().ccp_ccpol23plus(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys),
                                          ptr(zs), ld, box, C.byref(q), ptr(fxs), ptr(fys),
                                          ptr(fzs), vir.ctypes.data_as(C.POINTER(C.c_double))))
        return q.value

    def kspace_ewald(self, x, y, z, xs, ys, zs, lmax, mmax, nmax, alp, box, fxs, fys, fzs, vir):
        q = C.c_double()
        v = C.c_double(float(vir[0]))
        check(_lib.lib().ccp_kspace_ewald(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys),
                                          ptr(zs), xs.shape[1], lmax, mmax, nmax, alp, box,
                                          C.byref(q), ptr(fxs), ptr(fys), ptr(fzs), C.byref(v)))
        vir[0] = v.value
        return q.value

    def nb_induction(self, x, y, z, xs, ys, zs, box, idmx, idmy, idmz, fxs, fys, fzs, vir):
        q = C.c_double()
        v = C.c_double(float(vir[0]))
        it = C.c_int()
        check(_lib.lib().ccp_nb_induction(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys),
                                          ptr(zs), xs.shape[1], box, C.byref(q), ptr(idmx),
                                          ptr(idmy), ptr(idmz), ptr(fxs), ptr(fys), ptr(fzs),
                                          C.byref(v), C.byref(it)))
        vir[0] = v.value
        return q.value, it.value

    def threebody_term(self, x, y, z, xs, ys, zs, box, fxs, fys, fzs, fxfs2, fyfs2, fzfs2,
                       fxfs3, fyfs3, fzfs3, vir):
        q2, q3 = C.c_double(), C.c_double()
        v = C.c_double(float(vir[0]))
        check(_lib.lib().ccp_threebody_term(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys),
                                            ptr(zs), xs.shape[1], box, C.byref(q2), C.byref(q3),
                                            ptr(fxs), ptr(fys), ptr(fzs), ptr(fxfs2), ptr(fyfs2),
                                            ptr(fzfs2), ptr(fxfs3), ptr(fyfs3), ptr(fzfs3),
                                            C.byref(v)))
        vir[0] = v.value
        return q2.value, q3.value

    def hot_path(self, x, y, z, xs, ys, zs, box) -> HotPathResult:
        nm, ld = xs.shape
        out = [np.zeros((nm, ld)) for _ in range(3)] + [np.zeros(nm) for _ in range(6)] + \
              [np.zeros((nm, ld)) for _ in range(3)]
        e = CcpEnergies()
        check(_lib.lib().ccp_hot_path(self._h, ptr(x), ptr(y), ptr(z), ptr(xs), ptr(ys), ptr(zs),
                                      ld, box, C.byref(e), *[ptr(a) for a in out]))
        return HotPathResult(_energies(e), *out)

    def terms_device(self, terms, x, y, z, xs, ys, zs, box, fxs=None, fys=None, fzs=None,
                     fxfs2=None, fyfs2=None, fzfs2=None, fxfs3=None, fyfs3=None, fzfs3=None,
                     idmx=None, idmy=None, idmz=None) -> dict:
        """The terms selected by the bit mask `terms` (_lib.TERM_*) on contiguous torch CUDA
        float64 tensors on the context's device, in the layouts of hot_path_device; energies
        of terms not run are 0.  Mismatched arrays raise ValueError."""
        a, ld, o = self._device_args(x, y, z, xs, ys, zs, (fxs, fys, fzs, fxfs2, fyfs2, fzfs2,
                                                           fxfs3, fyfs3, fzfs3, idmx, idmy, idmz))
        e = CcpEnergies()
        check(_lib.lib().ccp_terms_device(self._h, int(terms), *a, ld, box, C.byref(e), *o))
        return _energies(e)

    # -- NVE molecular dynamics (device-resident state) -------------------------------
    def md_set_state(self, box, x, y, z, v, q, j):
        """Upload a rigid-water state (COM x, y, z; velocities v (nm, 3); quaternions
        q (nm, 4); principal-frame angular momenta j (nm, 3)) and evaluate its forces."""
        a = [np.ascontiguousarray(t, dtype=np.float64) for t in (x, y, z, v, q, j)]
        check(_lib.lib().ccp_md_set_state(self._h, float(box), *[ptr(t) for t in a]))

    def md_get_state(self) -> dict:
        nm = self.nm
        out = {"x": np.zeros(nm), "y": np.zeros(nm), "z": np.zeros(nm), "v": np.zeros((nm, 3)),
               "q": np.zeros((nm, 4)), "j": np.zeros((nm, 3))}
        check(_lib.lib().ccp_md_get_state(self._h, *[ptr(out[k]) for k in ("x", "y", "z", "v", "q", "j")]))
        return out

    def md_dipoles(self):
        """Induced dipoles (nm, ns) x 3 of the current MD state."""
        ns = self.model.ns
        out = [np.zeros((self.nm, ns)) for _ in range(3)]
        check(_lib.lib().ccp_md_get_dipoles(self._h, ns, *[ptr(a) for a in out]))
        return out

    def md_set_equilibration(self, temp0: float, nsteps: int):
        """The next nsteps md_nve steps rescale velocities and angular momenta to temp0."""
        check(_lib.lib().ccp_md_set_equilibration(self._h, float(temp0), int(nsteps)))

    def md_stats(self) -> dict:
        """Statistics of the current MD state (no step)."""
        s = _lib.CcpMdStats()
        check(_lib.lib().ccp_md_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.CcpMdStats._fields_}

    def md_set_ensemble(self, ensemble: str, temp0: float = 0.0, taut: float = 0.0,
                        pres0_katm: float = 0.0, taup: float = 0.0):
        """Ensemble of md_run: "nve" (nve_1), "nvt_b" (nvt_b), "npt_b" (npt_b_1), "nvt_h"
        (nvt_hov_3), "npt_h" (npt_hov_2) or "npt_mtk" (npt_mtk), with CONTROL's temp0 (K), taut (ps), pres0 (katm) and taup (ps)."""
        check(_lib.lib().ccp_md_set_ensemble(self._h, _lib.MD_ENSEMBLES[ensemble], float(temp0),
                                             float(taut), float(pres0_katm), float(taup)))

    def md_set_thermostat(self, chit: float, chip: float = 0.0):
        """Thermostat and barostat variables (REVCON's chit, chip)."""
        check(_lib.lib().ccp_md_set_thermostat(self._h, float(chit), float(chip)))

    def md_run(self, nsteps: int, dt: float) -> list:
        """nsteps steps of the ensemble set by md_set_ensemble; per-step statistics."""
        stats = (_lib.CcpMdStats * max(nsteps, 1))()
        check(_lib.lib().ccp_md_run(self._h, int(nsteps), float(dt), stats))
        return [{k: getattr(s, k) for k, _ in _lib.CcpMdStats._fields_} for s in stats[:nsteps]]

    def md_nve(self, nsteps: int, dt: float) -> list:
        """nve_1 steps on the device; per-step energies, temperature, virial, pressure."""
        stats = (_lib.CcpMdStats * max(nsteps, 1))()
        check(_lib.lib().ccp_md_nve(self._h, int(nsteps), float(dt), stats))
        return [{k: getattr(s, k) for k, _ in _lib.CcpMdStats._fields_} for s in stats[:nsteps]]

    # -- FS3 parameters --------------------------------------------------------------
    def fs3_params(self):
        """(cs_sr, cs_lr, bgr_sr, bgr_lr): class coefficients (nclass each) and site-pair
        (b, g, r0) as (3, 289) arrays, index is*17 + js."""
        n = self.model.get_int("nclass")
        cs_sr, cs_lr = np.zeros(n), np.zeros(n)
        b_sr, b_lr = np.zeros((3, 289)), np.zeros((3, 289))
        check(_lib.lib().ccp_context_get_fs3_params(self._h, ptr(cs_sr), ptr(cs_lr), n,
                                                     ptr(b_sr), ptr(b_lr)))
        return cs_sr, cs_lr, b_sr, b_lr

    def set_fs3_params(self, cs_sr, cs_lr, bgr_sr, bgr_lr):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (cs_sr, cs_lr, bgr_sr, bgr_lr)]
        check(_lib.lib().ccp_context_set_fs3_params(self._h, ptr(a[0]), ptr(a[1]), a[0].size,
                                                     ptr(a[2]), ptr(a[3])))

    def fs3_param_grad(self):
        """Gradient of the last evaluation's FS3 energy (kcal/mol) with respect to
        (cs_sr, cs_lr, bgr_sr, bgr_lr); needs set_option("fs3_param_grad", 1)."""
        n = self.model.get_int("nclass")
        g = [np.zeros(n), np.zeros(n), np.zeros((3, 289)), np.zeros((3, 289))]
        check(_lib.lib().ccp_context_fs3_param_grad(self._h, *[ptr(v) for v in g[:2]], n,
                                                     *[ptr(v) for v in g[2:]]))
        return tuple(g)

    def hot_path_device(self, x, y, z, xs, ys, zs, box, fxs=None, fys=None, fzs=None,
                        fxfs2=None, fyfs2=None, fzfs2=None, fxfs3=None, fyfs3=None,
                        fzfs3=None, idmx=None, idmy=None, idmz=None) -> dict:
        """All arrays are contiguous torch CUDA float64 tensors on the context's device (or
        None); nothing crosses PCIe.  Mismatched arrays raise ValueError."""
        a, ld, o = self._device_args(x, y, z, xs, ys, zs, (fxs, fys, fzs, fxfs2, fyfs2, fzfs2,
                                                           fxfs3, fyfs3, fzfs3, idmx, idmy, idmz))
        e = CcpEnergies()
        check(_lib.lib().ccp_hot_path_device(self._h, *a, ld, box, C.byref(e), *o))
        return _energies(e)


class Batch:
    """Independent frames of ``nm`` molecules evaluated concurrently: ``slots`` contexts
    (own device buffers and CUDA streams each), frame f on slot f % slots, one host worker
    thread per slot inside the library (``ccp_batch_terms_device``)."""

    def __init__(self, model: Model, nm: int, box0: float, slots: int = 8, device: int = 0,
                 precision: str = "fp64"):
        prec = {"fp64": _lib.CCP_FP64, "mixed": _lib.CCP_MIXED}[precision]
        h = C.c_void_p()
        check(_lib.lib().ccp_batch_create(model.handle, nm, box0, slots, device, prec,
                                          C.byref(h)))
        self._h = h
        self.model = model
        self.nm = nm
        self.slots = slots
        self.device = device
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ccp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_option(self, name: str, value: int):
        check(_lib.lib().ccp_batch_set_option(self._h, name.encode(), int(value)))

    def set_fs3_params(self, cs_sr, cs_lr, bgr_sr, bgr_lr):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (cs_sr, cs_lr, bgr_sr, bgr_lr)]
        check(_lib.lib().ccp_batch_set_fs3_params(self._h, ptr(a[0]), ptr(a[1]), a[0].size,
                                                   ptr(a[2]), ptr(a[3])))

    def fs3_params(self):
        """The FS3 fit of slot 0 (every slot holds the same fit)."""
        h = C.c_void_p()
        check(_lib.lib().ccp_batch_context(self._h, 0, C.byref(h)))
        n = self.model.get_int("nclass")
        cs_sr, cs_lr = np.zeros(n), np.zeros(n)
        b_sr, b_lr = np.zeros((3, 289)), np.zeros((3, 289))
        check(_lib.lib().ccp_context_get_fs3_params(h, ptr(cs_sr), ptr(cs_lr), n, ptr(b_sr),
                                                     ptr(b_lr)))
        return cs_sr, cs_lr, b_sr, b_lr

    def terms_device(self, terms, box, x, y, z, xs, ys, zs, fxs=None, fys=None, fzs=None,
                     fxfs2=None, fyfs2=None, fzfs2=None, fxfs3=None, fyfs3=None, fzfs3=None,
                     idmx=None, idmy=None, idmz=None, pgrad=None) -> list:
        """The terms selected by ``terms`` for every frame.  x, y, z: (nframes, nm) and xs,
        ys, zs: (nframes, nm, ld) torch CUDA float64 tensors, outputs likewise; ``box`` is a
        sequence of nframes box lengths; ``pgrad`` an optional (nframes, 2 nclass + 1734)
        float64 numpy array for the per-frame FS3 parameter gradients.  Returns the
        per-frame energy dicts."""
        nf = int(x.shape[0]) if len(x.shape) == 2 else -1
        if nf < 1 or len(xs.shape) != 3:
            raise ValueError(f"x: expected (nframes, nm), xs: (nframes, nm, ld); got "
                             f"{tuple(x.shape)} and {tuple(xs.shape)}")
        nm, ld = _site_layout(xs[0], self.model.ns)
        if nm != self.nm:
            raise ValueError(f"xs: {nm} molecules per frame, the batch holds {self.nm}")
        d = self.device
        a = [_device_array(t, (nf, nm), n, d) for t, n in ((x, "x"), (y, "y"), (z, "z"))]
        a += [_device_array(t, (nf, nm, ld), n, d) for t, n in ((xs, "xs"), (ys, "ys"),
                                                                 (zs, "zs"))]
        shapes = [(nf, nm, ld)] * 3 + [(nf, nm)] * 6 + [(nf, nm, ld)] * 3
        names = ["fxs", "fys", "fzs", "fxfs2", "fyfs2", "fzfs2", "fxfs3", "fyfs3", "fzfs3",
                 "idmx", "idmy", "idmz"]
        outs = (fxs, fys, fzs, fxfs2, fyfs2, fzfs2, fxfs3, fyfs3, fzfs3, idmx, idmy, idmz)
        o = [_optional_device_array(t, sh, n, d) for t, sh, n in zip(outs, shapes, names)]
        boxes = np.ascontiguousarray(np.broadcast_to(np.asarray(box, dtype=np.float64), (nf,)))
        e = (CcpEnergies * max(nf, 1))()
        plen = 0
        if pgrad is not None:
            if pgrad.dtype != np.float64 or pgrad.ndim != 2 or pgrad.shape[0] != nf or \
                    not pgrad.flags.c_contiguous:
                raise ValueError("pgrad: expected a C-contiguous float64 (nframes, n) array")
            plen = pgrad.shape[1]
        check(_lib.lib().ccp_batch_terms_device(
            self._h, int(terms), nf, ptr(boxes), *a, ld, e, *o, ptr(pgrad), plen))
        return [_energies(e[f]) for f in range(nf)]

