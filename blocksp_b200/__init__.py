"""blocksp_b200 — B200-native (sm_100a) implementation of BlockSp's solve path.

The compute lives in ``libblocksp_b200.so`` (hand-written CUDA behind the C ABI
declared in ``include/blocksp_b200.h``); this package holds the Python host
mirror of the reference interface, the seeded workload generator and the build
script.  Importing the package does not require a GPU; calling any compute
function does.
"""
from . import _lib
from ._lib import BspError
from .api import Handle, Matrix, bsmv, bsmv_dev, default_handle, dot_dev

__all__ = ["BspError", "Handle", "Matrix", "bsmv", "bsmv_dev", "default_handle", "dot_dev", "_lib"]
