"""B200-native CCpol23+(2025) force-evaluation hot path.

FS2/FS3 three-body terms with the SR/LR R_avg switch, the iterative induced-dipole solve
and the real/reciprocal Ewald sums, as hand-written sm_100a CUDA behind a C ABI
(``include/ccpol23_b200.h``) that mirrors the reference Fortran entry points.
"""
from .api import Batch, Context, HotPathResult, Model, data_dir, ewald_setup  # noqa: F401
from ._lib import CcpError  # noqa: F401

__all__ = ["Batch", "Context", "HotPathResult", "Model", "data_dir", "ewald_setup", "CcpError"]
