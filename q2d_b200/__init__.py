"""q2d_b200 — B200-native (sm_100a) explicit finite-volume residual and time-update path of
Q2D, behind the C ABI declared in include/q2d_gpu.h.

The compute path is hand-written CUDA in q2d_b200/csrc, built into q2d_b200/lib/libq2d_gpu.so.
This package is the host side: the ctypes binding (_abi), case generators (cases), the
Wrap_Setup/Wrap_Solve mirror (solver), the reference's case-directory formats (refio) and the
batched and served drivers.
"""
from . import _abi  # noqa: F401
from .cases import CaseSpec, BlockSpec  # noqa: F401
from .solver import Q2DSolver, Q2DError, make_options  # noqa: F401

__all__ = ["Q2DSolver", "Q2DError", "make_options", "CaseSpec", "BlockSpec"]
