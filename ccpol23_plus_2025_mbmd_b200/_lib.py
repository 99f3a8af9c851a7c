"""ctypes loader of the in-tree C-ABI library ``lib/libccpol23_b200.so``.

The library is the product; this module only declares argument types.  It raises
immediately when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("CCP_LIB_PATH") or
                Path(__file__).resolve().parent / "lib" / "libccpol23_b200.so")

CCP_OK = 0
CCP_ERR_BAD_INPUT = 1
CCP_ERR_NOT_CONVERGED = 2
CCP_ERR_CUDA = 3
CCP_ERR_NO_DEVICE = 4
CCP_ERR_IO = 5
CCP_ERR_CAPACITY = 6
CCP_FP64 = 0
CCP_MIXED = 1

# Every function declared in include/ccpol23_b200.h.
EXPORTS = [
    "ccp_last_error", "ccp_model_load", "ccp_model_free", "ccp_model_get_int",
    "ccp_model_get_double", "ccp_model_set_int", "ccp_model_set_double", "ccp_model_get_array",
    "ccp_sites", "ccp_ewald_setup", "ccp_context_create", "ccp_context_destroy",
    "ccp_context_set_ewald", "ccp_context_set_maxit", "ccp_context_set_stream",
    "ccp_ewald_self_correction", "ccp_rspace_ewald", "ccp_kspace_ewald", "ccp_nb_induction",
    "ccp_threebody_term", "ccp_hot_path", "ccp_hot_path_device", "ccp_context_last_launches",
    "ccp_context_set_timing", "ccp_context_phase_ms", "ccp_device_fma_peak",
    "ccp_kspace_ewald_fixed", "ccp_context_set_option", "ccp_context_get_option",
    "ccp_terms_device", "ccp_context_get_fs3_params", "ccp_context_set_fs3_params",
    "ccp_context_fs3_param_grad", "ccp_ccpol23plus", "ccp_md_set_state", "ccp_md_get_state",
    "ccp_md_nve", "ccp_md_get_dipoles", "ccp_batch_create", "ccp_batch_destroy",
    "ccp_batch_slots", "ccp_batch_context", "ccp_batch_set_option", "ccp_batch_set_fs3_params",
    "ccp_batch_terms_device", "ccp_md_set_equilibration", "ccp_md_get_stats",
    "ccp_md_set_ensemble", "ccp_md_run", "ccp_md_set_thermostat", "ccp_device_mufu_peak",
]

# term bits of ccp_terms_device (CCP_TERM_*)
TERM_SELF, TERM_RSPACE, TERM_KSPACE, TERM_INDUCTION, TERM_FS2, TERM_FS3 = 1, 2, 4, 8, 16, 32
TERM_VDW = 64

# ensembles of ccp_md_run (CCP_MD_*)
MD_ENSEMBLES = {"nve": 0, "nvt_b": 1, "npt_b": 2, "nvt_h": 3, "npt_h": 4,
                "npt_mtk": 5}
TERM_HOT = 63
TERM_ALL = 127


class CcpEnergies(C.Structure):
    _fields_ = [("scpe", C.c_double), ("rcpe", C.c_double), ("kcpe", C.c_double),
                ("indpe", C.c_double), ("fs2pe", C.c_double), ("fs3pe", C.c_double),
                ("vir", C.c_double), ("ind_iters", C.c_int), ("n_fs3_triples", C.c_int),
                ("n_fs3_blend", C.c_int), ("n_fs2_triples", C.c_int), ("vdwpe", C.c_double)]


class CcpMdStats(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("vdwpe", "cpe", "indpe", "pe3b", "pe", "tke", "rke", "te",
                                          "sys_temp", "vir", "pres")] + [("ind_iters", C.c_int)] + \
        [(k, C.c_double) for k in ("box", "volm", "chit", "chip", "consv")]


class CcpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[ccp status {code}] {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python -m ccpol23_plus_2025_mbmd_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    d, i, vp = C.c_double, C.c_int, C.c_void_p
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.ccp_last_error.restype = C.c_char_p
    L.ccp_model_load.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.ccp_model_free.argtypes = [vp]
    L.ccp_model_free.restype = None
    L.ccp_model_get_int.argtypes = [vp, C.c_char_p, pi]
    L.ccp_model_get_double.argtypes = [vp, C.c_char_p, pd]
    L.ccp_model_set_int.argtypes = [vp, C.c_char_p, i]
    L.ccp_model_set_double.argtypes = [vp, C.c_char_p, d]
    L.ccp_model_get_array.argtypes = [vp, C.c_char_p, vp, i]
    L.ccp_sites.argtypes = [vp, i, vp, i, vp, vp, vp]
    L.ccp_ewald_setup.argtypes = [d, d, d, pd, pi, pi, pi]
    L.ccp_context_create.argtypes = [vp, i, d, i, i, C.POINTER(vp)]
    L.ccp_context_destroy.argtypes = [vp]
    L.ccp_context_set_ewald.argtypes = [vp, d, i, i, i]
    L.ccp_context_set_maxit.argtypes = [vp, i]
    L.ccp_context_set_stream.argtypes = [vp, vp]
    L.ccp_context_last_launches.argtypes = [vp, pi]
    L.ccp_context_set_timing.argtypes = [vp, i]
    L.ccp_context_phase_ms.argtypes = [vp, vp, i]
    L.ccp_device_fma_peak.argtypes = [i, i, pd]
    L.ccp_device_mufu_peak.argtypes = [i, pd]
    L.ccp_ewald_self_correction.argtypes = [vp, d, d] + [vp] * 6 + [i, pd] + [vp] * 3 + [pd]
    L.ccp_rspace_ewald.argtypes = [vp] + [vp] * 6 + [i, d, d, pd] + [vp] * 3 + [pd]
    L.ccp_kspace_ewald.argtypes = [vp] + [vp] * 6 + [i, i, i, i, d, d, pd] + [vp] * 3 + [pd]
    L.ccp_nb_induction.argtypes = [vp] + [vp] * 6 + [i, d, pd] + [vp] * 6 + [pd, pi]
    L.ccp_threebody_term.argtypes = [vp] + [vp] * 6 + [i, d, pd, pd] + [vp] * 9 + [pd]
    L.ccp_hot_path.argtypes = [vp] + [vp] * 6 + [i, d, C.POINTER(CcpEnergies)] + [vp] * 12
    L.ccp_hot_path_device.argtypes = [vp] + [vp] * 6 + [i, d, C.POINTER(CcpEnergies)] + [vp] * 12
    L.ccp_ccpol23plus.argtypes = [vp] + [vp] * 6 + [i, d, pd] + [vp] * 3 + [pd]
    L.ccp_md_set_state.argtypes = [vp, d] + [vp] * 6
    L.ccp_md_get_state.argtypes = [vp] + [vp] * 6
    L.ccp_md_nve.argtypes = [vp, i, d, vp]
    L.ccp_md_get_dipoles.argtypes = [vp, i, vp, vp, vp]
    L.ccp_md_set_equilibration.argtypes = [vp, d, i]
    L.ccp_md_get_stats.argtypes = [vp, vp]
    L.ccp_md_set_ensemble.argtypes = [vp, i, d, d, d, d]
    L.ccp_md_run.argtypes = [vp, i, d, vp]
    L.ccp_md_set_thermostat.argtypes = [vp, d, d]
    L.ccp_terms_device.argtypes = [vp, C.c_uint] + [vp] * 6 + [i, d, C.POINTER(CcpEnergies)] + [vp] * 12
    L.ccp_context_get_fs3_params.argtypes = [vp, vp, vp, i, vp, vp]
    L.ccp_context_set_fs3_params.argtypes = [vp, vp, vp, i, vp, vp]
    L.ccp_context_fs3_param_grad.argtypes = [vp, vp, vp, i, vp, vp]
    L.ccp_context_set_option.argtypes = [vp, C.c_char_p, i]
    L.ccp_context_get_option.argtypes = [vp, C.c_char_p, pi]
    L.ccp_kspace_ewald_fixed.argtypes = [vp, i] + [vp] * 6 + [i, i, i, i, d, d] + [vp] * 5 + [vp]
    L.ccp_batch_create.argtypes = [vp, i, d, i, i, i, C.POINTER(vp)]
    L.ccp_batch_destroy.argtypes = [vp]
    L.ccp_batch_slots.argtypes = [vp, pi]
    L.ccp_batch_context.argtypes = [vp, i, C.POINTER(vp)]
    L.ccp_batch_set_option.argtypes = [vp, C.c_char_p, i]
    L.ccp_batch_set_fs3_params.argtypes = [vp, vp, vp, i, vp, vp]
    L.ccp_batch_terms_device.argtypes = ([vp, C.c_uint, i, vp] + [vp] * 6 + [i, vp] + [vp] * 12
                                         + [vp, i])
    _lib = L
    return L


def check(code: int) -> None:
    if code != CCP_OK:
        raise CcpError(code, lib().ccp_last_error().decode())


def ptr(a) -> int | None:
    """Address of a C-contiguous float64 numpy array (None passes NULL)."""
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
        raise ValueError("expected a C-contiguous float64 numpy array, got "
                         f"{type(a).__name__} {getattr(a, 'dtype', '')}")
    return a.ctypes.data
