"""B200-native xSPDE ensemble-integration path.

Public API mirrors the reference's control layer: ``xsim``/``xspde`` and
``xpreferences``; ``GpuPath`` is the p.path / p.method replacement of one input
struct.  The compute runs in libxspde_b200.so (C ABI in include/xspde_b200.h):
kernels generated per problem and compiled by NVRTC for sm_100a.
"""
from ._lib import XsError  # noqa: F401
from .xsim import GpuPath, Struct, xpreferences, xsim, xspde  # noqa: F401

__version__ = "0.1"
