"""B200-native data-parallel primitive library (AdaptiveCpp's
hipsycl::algorithms reduce / transform_reduce / inclusive_scan /
exclusive_scan / copy_if path, rebuilt as hand-written sm_100a CUDA behind a
C-ABI).  The C++ drop-in headers live in include/; this package holds the
CUDA sources (csrc/), the build script and the ctypes binding (capi)."""
from . import capi  # noqa: F401

__all__ = ["capi"]
