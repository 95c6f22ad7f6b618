"""MatrixMarket (.mtx) files to block CSR and solArray order (host side).

Mirrors the reference's converters mtxMatrix_to_BlockSp and
mtxArray_to_solArray (blocksp_tests.hpp:582-699) through the C ABI
(bsp_mtx_read_matrix / bsp_mtx_read_vector): same start_line, symmetric and
block-placement conventions, with two fixes: for D > 1 the reference puts
every vector value into dim 0 (in-block index i % B instead of i % (B*D),
blocksp_tests.hpp:679), and it ignores base_zero; here value i lands at flat
position i of the (element, dim, b) order and base_zero is honoured.
Reading needs the built library but no GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .systems import BSRSystem


def mtxMatrix_to_BlockSp(path: str, B: int, start_line: int = 0, symmetric: bool = False,
                         base_zero: bool = False) -> BSRSystem:
    """A .mtx coordinate matrix as block CSR with B x B blocks (blocks in order
    of first appearance within each block row)."""
    lib = _lib.load()
    n, m, nnzb = C.c_int(), C.c_int(), C.c_int64()
    args = (str(path).encode(), int(B), int(start_line), int(bool(symmetric)), int(bool(base_zero)),
            C.byref(n), C.byref(m), C.byref(nnzb))
    _lib.check(lib.bsp_mtx_read_matrix(*args, None, None, None), "bsp_mtx_read_matrix")
    row_ptr = np.zeros(n.value + 1, np.int32)
    col_idx = np.zeros(max(nnzb.value, 1), np.int32)
    vals = np.zeros((max(nnzb.value, 1), B, B))
    _lib.check(lib.bsp_mtx_read_matrix(*args, row_ptr.ctypes.data, col_idx.ctypes.data, vals.ctypes.data),
               "bsp_mtx_read_matrix")
    return BSRSystem(n=n.value, bs=int(B), row_ptr=row_ptr, col_idx=col_idx[:nnzb.value],
                     vals=vals[:nnzb.value], b=np.zeros(n.value * B), name=str(path))


def mtxArray_to_solArray(path: str, B: int, D: int = 1, start_line: int = 0) -> np.ndarray:
    """A .mtx M x 1 vector as the flat solArray<T, B, D> array (n * B * D values)."""
    lib = _lib.load()
    cnt = C.c_int64()
    _lib.check(lib.bsp_mtx_read_vector(str(path).encode(), int(start_line), int(B), int(D), C.byref(cnt), None),
               "bsp_mtx_read_vector")
    out = np.zeros(cnt.value)
    _lib.check(lib.bsp_mtx_read_vector(str(path).encode(), int(start_line), int(B), int(D), C.byref(cnt),
                                       out.ctypes.data), "bsp_mtx_read_vector")
    return out
