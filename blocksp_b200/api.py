"""Python host mirror of the BlockSp solve-path interface over the C ABI.

Names and argument meanings follow the reference library (BlockSp v1.0):
``bsmv`` (blocksp_multiply.hpp:364-404), ``pCG`` (blocksp_solvers.hpp:51-105),
``pGMRES`` (blocksp_solvers.hpp:156-295), the preconditioners ``Diag``, ``SOR``,
``ILU0``, ``IChol0`` (blocksp_preconditioners.hpp:75-538) and the solver structs
``SOR_pGMRES``, ``SOR_pCG``, ``ILU0_pGMRES``, ``IChol0_pCG`` with their ``ez``
one-call forms (blocksp_solvers.hpp:344-649).  Compute always runs through
``libblocksp_b200.so`` on the GPU; device vectors are torch CUDA tensors
(float64, the solArray layout flattened), host vectors are numpy arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import BspError, PrecondParams, SolveInfo, SolveOpts, check


def _ptr(a) -> int | None:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    raise TypeError(f"unsupported buffer {type(a)}")


class Handle:
    """A device + stream context (one per CUDA stream, not thread-safe)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.bsp_handle_create(device, stream, C.byref(h)), "bsp_handle_create")
        self.h = h
        self.device = device

    def sync(self) -> None:
        check(self.lib.bsp_handle_sync(self.h), "bsp_handle_sync", self.h)

    @property
    def stream(self) -> int:
        return self.lib.bsp_handle_stream(self.h) or 0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.bsp_handle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Handle | None = None


def default_handle() -> Handle:
    global _default
    if _default is None:
        _default = Handle(0)
    return _default


class Matrix:
    """A BSR matrix resident on the GPU (the packed form of BlockSp<T,N>)."""

    def __init__(self, row_ptr, col_idx, vals, bs: int, n_cols: int | None = None,
                 handle: Handle | None = None):
        self.handle = handle or default_handle()
        lib = self.handle.lib
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        col_idx = np.ascontiguousarray(col_idx, dtype=np.int32)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.n_rows = int(row_ptr.shape[0] - 1)
        self.n_cols = int(n_cols if n_cols is not None else self.n_rows)
        self.bs = int(bs)
        self.nnzb = int(col_idx.shape[0])
        m = C.c_void_p()
        check(lib.bsp_matrix_create(self.handle.h, self.n_rows, self.n_cols, self.bs, self.nnzb,
                                    _ptr(row_ptr), _ptr(col_idx), _ptr(vals), C.byref(m)),
              "bsp_matrix_create", self.handle.h)
        self.m = m

    @classmethod
    def from_system(cls, s, handle: Handle | None = None) -> "Matrix":
        return cls(s.row_ptr, s.col_idx, s.vals, s.bs, handle=handle)

    def make_lowp(self, dtype: int) -> None:
        check(self.handle.lib.bsp_matrix_make_lowp(self.m, dtype), "bsp_matrix_make_lowp",
              self.handle.h)

    def close(self) -> None:
        if getattr(self, "m", None):
            self.handle.lib.bsp_matrix_destroy(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bsmv_dev(A: Matrix, x, y, nrhs: int = 1, transpose: bool = False, alpha: float = 1.0,
             beta: float = 0.0, z=None, dtype: int = _lib.BSP_F64) -> None:
    """y = alpha*op(A)*x + beta*z on device tensors (z defaults to y)."""
    if z is None and beta != 0.0:
        z = y
    check(A.handle.lib.bsp_bsmv_dev(A.handle.h, A.m, nrhs, int(transpose), dtype, alpha, _ptr(x),
                                    beta, _ptr(z), _ptr(y)), "bsp_bsmv_dev", A.handle.h)


def bsmv(A: Matrix, x: np.ndarray, b: np.ndarray | None = None, nrhs: int = 1,
         transpose: bool = False) -> np.ndarray:
    """Host form of the reference bsmv.

    ``bsmv(A, x)`` returns A x (blocksp_multiply.hpp:377-390); with ``b`` given
    it accumulates into b like the void overloads ``bsmv(b, A, x)``.
    """
    x = np.ascontiguousarray(x, dtype=np.float64)
    m = (A.n_cols if transpose else A.n_rows) * A.bs * nrhs
    if b is None:
        y = np.zeros(m)
        beta = 0.0
    else:
        y = b
        beta = 1.0
    check(A.handle.lib.bsp_bsmv(A.handle.h, A.m, nrhs, int(transpose), 1.0, _ptr(x), beta, _ptr(y)),
          "bsp_bsmv", A.handle.h)
    return y


def dot_dev(handle: Handle, x, y) -> float:
    out = C.c_double()
    check(handle.lib.bsp_dot(handle.h, int(x.numel()), _ptr(x), _ptr(y), C.byref(out)), "bsp_dot",
          handle.h)
    return out.value
