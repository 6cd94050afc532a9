"""B200-native multi-fluid Hall-MHD step of MPCNS_Mercury.

The step runs as hand-written CUDA kernels for sm_100a in libmercury_mhd.so
behind a C ABI (include/mercury_mhd.h); this package holds the host-side
binding (capi), the physical-constant and case setup (setup) and the build.
"""
from . import capi  # noqa: F401
from .capi import Context, MhdError  # noqa: F401
from .constants import reference_constants  # noqa: F401
