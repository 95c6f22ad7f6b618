"""blocksp_b200 — B200-native (sm_100a) implementation of BlockSp's solve path.

The compute lives in ``libblocksp_b200.so`` (hand-written CUDA behind the C ABI
declared in ``include/blocksp_b200.h``); this package holds the Python host
mirror of the reference interface, the seeded workload generator and the build
script.  Importing the package does not require a GPU; calling any compute
function does.
"""
from . import _lib
from ._lib import BspError
from .api import (Batch, IChol0, IChol0_pCG, ILU0, ILU0_pGMRES, SOR, SOR_pCG, SOR_pGMRES, Diag, Handle, Matrix,
                  NoPre, Precond, Eigenvalues, arnoldi_eigenvalues, bs_id, bs_tr, bsmm, bsmv, bsmv_dev, default_handle, dot_dev, ez, matrix_add, pCG,
                  pGMRES)

__all__ = ["Batch", "BspError", "Handle", "Matrix", "Eigenvalues", "arnoldi_eigenvalues", "bs_id", "bs_tr", "bsmm", "matrix_add", "bsmv", "bsmv_dev", "default_handle", "dot_dev", "_lib",
           "Precond", "NoPre", "Diag", "SOR", "ILU0", "IChol0", "pCG", "pGMRES", "SOR_pGMRES",
           "SOR_pCG", "ILU0_pGMRES", "IChol0_pCG", "ez"]
