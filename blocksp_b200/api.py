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
import weakref

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

    # cudaStreamLegacy: the legacy default stream, torch's default stream
    LEGACY_STREAM = 1

    def __init__(self, device: int = 0, stream: int | None = None):
        """stream: a CUDA stream handle (e.g. ``torch.cuda.Stream().cuda_stream``).
        By default the handle runs on torch's current stream of ``device``, so
        calls on torch tensors are ordered with the caller's torch work (a
        private stream would let torch read a tensor the library is still
        writing)."""
        self.lib = _lib.load()
        if stream is None:
            stream = self._torch_stream(device)
        h = C.c_void_p()
        check(self.lib.bsp_handle_create(device, stream, C.byref(h)), "bsp_handle_create")
        self.h = h
        self.device = device
        self._children = weakref.WeakSet()  # objects that must be released first

    @classmethod
    def _torch_stream(cls, device: int) -> int | None:
        try:
            import torch
            if not torch.cuda.is_available():
                return None
            s = torch.cuda.current_stream(device).cuda_stream
            return s if s else cls.LEGACY_STREAM
        except Exception:
            return None

    def adopt(self, obj) -> None:
        self._children.add(obj)

    def sync(self) -> None:
        check(self.lib.bsp_handle_sync(self.h), "bsp_handle_sync", self.h)

    def set_spin_limit(self, polls: int = 1 << 22) -> None:
        """Polls a device-side wait makes before it gives up with TIMEOUT
        (default 2^22); a small value makes waits run out on purpose."""
        check(self.lib.bsp_handle_set_spin_limit(self.h, int(polls)), "bsp_handle_set_spin_limit", self.h)

    @property
    def stream(self) -> int:
        return self.lib.bsp_handle_stream(self.h) or 0

    def close(self) -> None:
        if getattr(self, "h", None):
            for child in list(self._children):
                child.close()
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
    """A BSR matrix resident on the GPU (the packed form of BlockSp<T,N>).

    A complex matrix (``Matrix.from_complex``, T = std::complex<double>) is held
    as its real embedding: ``bs`` is twice the complex block size
    ``complex_bs``, and complex vectors (numpy complex128) are passed to the
    library as their interleaved (re, im) doubles."""

    complex_bs = 0

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
        self.handle.adopt(self)

    @classmethod
    def from_system(cls, s, handle: Handle | None = None) -> "Matrix":
        if np.iscomplexobj(s.vals):
            return cls.from_complex(s.row_ptr, s.col_idx, s.vals, handle=handle)
        return cls(s.row_ptr, s.col_idx, s.vals, s.bs, handle=handle)

    @classmethod
    def from_complex(cls, row_ptr, col_idx, vals, n_cols: int | None = None,
                     handle: Handle | None = None) -> "Matrix":
        """A complex block matrix: vals complex128 [nnzb, bs, bs] row-major."""
        handle = handle or default_handle()
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        col_idx = np.ascontiguousarray(col_idx, dtype=np.int32)
        vals = np.ascontiguousarray(vals, dtype=np.complex128)
        n = int(row_ptr.shape[0] - 1)
        cbs = int(vals.shape[1]) if vals.ndim == 3 else 1
        m = C.c_void_p()
        check(handle.lib.bsp_matrix_create_complex(handle.h, n, int(n_cols if n_cols is not None else n), cbs,
                                                   int(col_idx.shape[0]), _ptr(row_ptr), _ptr(col_idx),
                                                   _ptr(vals), C.byref(m)),
              "bsp_matrix_create_complex", handle.h)
        return cls._wrap(m, handle)

    @classmethod
    def _wrap(cls, m: C.c_void_p, handle: Handle) -> "Matrix":
        """A Matrix object owning the device matrix m made by the library."""
        obj = cls.__new__(cls)
        obj.handle = handle
        n, nc, bs, nnzb = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        check(handle.lib.bsp_matrix_info(m, C.byref(n), C.byref(nc), C.byref(bs), C.byref(nnzb)), "bsp_matrix_info")
        obj.n_rows, obj.n_cols, obj.bs, obj.nnzb = n.value, nc.value, bs.value, nnzb.value
        cb = C.c_int()
        check(handle.lib.bsp_matrix_complex_bs(m, C.byref(cb)), "bsp_matrix_complex_bs")
        obj.complex_bs = cb.value
        obj.m = m
        handle.adopt(obj)
        return obj

    def export(self):
        """(row_ptr, col_idx, vals) of the matrix, copied to the host."""
        rp = np.zeros(self.n_rows + 1, np.int32)
        ci = np.zeros(max(self.nnzb, 1), np.int32)
        va = np.zeros((max(self.nnzb, 1), self.bs, self.bs))
        check(self.handle.lib.bsp_matrix_export(self.m, _ptr(rp), _ptr(ci), _ptr(va)), "bsp_matrix_export")
        return rp, ci[:self.nnzb], va[:self.nnzb]

    def __add__(self, other: "Matrix") -> "Matrix":
        return matrix_add(1.0, self, 1.0, other)

    def __sub__(self, other: "Matrix") -> "Matrix":
        return matrix_add(1.0, self, -1.0, other)

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


def bs_id(size: int, bs: int, handle: Handle | None = None) -> Matrix:
    """bs_id<T, M>(size) (blocksp_multiply.hpp:335-336): the block identity."""
    h = handle or default_handle()
    m = C.c_void_p()
    check(h.lib.bsp_bs_id(h.h, int(size), int(bs), C.byref(m)), "bsp_bs_id", h.h)
    return Matrix._wrap(m, h)


def bs_tr(A: Matrix) -> Matrix:
    """bs_tr(A) (blocksp_multiply.hpp:339-340): block (j, i) = A_ij^T."""
    m = C.c_void_p()
    check(A.handle.lib.bsp_bs_tr(A.handle.h, A.m, C.byref(m)), "bsp_bs_tr", A.handle.h)
    return Matrix._wrap(m, A.handle)


def bsmm(A: Matrix, B: Matrix, *more, Atran: bool = False) -> Matrix:
    """bsmm(A, B[, C[, D]], Atran) (blocksp_multiply.hpp:343-362): op(A) B [C [D]]
    with op(A) = A^T when Atran; longer products nest to the right (:137-159)."""
    if more:
        B = bsmm(B, *more)
    m = C.c_void_p()
    check(A.handle.lib.bsp_bsmm(A.handle.h, A.m, B.m, int(bool(Atran)), C.byref(m)), "bsp_bsmm", A.handle.h)
    return Matrix._wrap(m, A.handle)


def matrix_add(alpha: float, A: Matrix, beta: float, B: Matrix) -> Matrix:
    """alpha A + beta B with the container's block order (A's blocks, then B's new ones)."""
    m = C.c_void_p()
    check(A.handle.lib.bsp_matrix_add(A.handle.h, float(alpha), A.m, float(beta), B.m, C.byref(m)),
          "bsp_matrix_add", A.handle.h)
    return Matrix._wrap(m, A.handle)


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
    cplx = bool(A.complex_bs)
    x = _as_real(x, cplx)
    m = (A.n_cols if transpose else A.n_rows) * A.bs * nrhs
    if b is None:
        y = np.zeros(m)
        beta = 0.0
    else:
        y = b.view(np.float64) if cplx else b
        beta = 1.0
    check(A.handle.lib.bsp_bsmv(A.handle.h, A.m, nrhs, int(transpose), 1.0, _ptr(x), beta, _ptr(y)),
          "bsp_bsmv", A.handle.h)
    return y.view(np.complex128) if cplx else y


def _as_real(v, cplx: bool) -> np.ndarray:
    """A host vector as the doubles the library reads: complex vectors as their
    interleaved (re, im) doubles."""
    if cplx:
        return np.ascontiguousarray(v, dtype=np.complex128).view(np.float64)
    return np.ascontiguousarray(v, dtype=np.float64)


def dot_dev(handle: Handle, x, y) -> float:
    out = C.c_double()
    check(handle.lib.bsp_dot(handle.h, int(x.numel()), _ptr(x), _ptr(y), C.byref(out)), "bsp_dot",
          handle.h)
    return out.value


# ---------------------------------------------------------------- preconditioners

class Precond:
    """A preconditioner built on the GPU (preConditioners::* in the reference).

    Calling it on a device tensor applies M^{-1} in place, like the reference's
    ``operator()(solArray&)`` (blocksp_preconditioners.hpp:541-556).
    """

    def __init__(self, A: Matrix, kind: int, w: float = 1.6, nu: int = 3, type_: int = 0,
                 precision: int = _lib.PREC_F64):
        self.A = A
        self.handle = A.handle
        self.kind = kind
        params = PrecondParams(kind, float(w), int(nu), int(type_), int(precision))
        p = C.c_void_p()
        check(self.handle.lib.bsp_precond_create(self.handle.h, A.m, C.byref(params), C.byref(p)),
              "bsp_precond_create", self.handle.h)
        self.p = p
        self.handle.adopt(self)

    @classmethod
    def wrap(cls, A: Matrix, ptr, kind: int) -> "Precond":
        """Adopts a preconditioner handle built by another entry point."""
        obj = cls.__new__(cls)
        obj.A = A
        obj.handle = A.handle
        obj.kind = kind
        obj.p = ptr
        obj.handle.adopt(obj)
        return obj

    def __call__(self, r) -> None:
        check(self.handle.lib.bsp_precond_apply_dev(self.handle.h, self.p, _ptr(r)),
              "bsp_precond_apply_dev", self.handle.h)

    def apply_host(self, r: np.ndarray) -> np.ndarray:
        cplx = bool(self.A.complex_bs)
        out = _as_real(r, cplx).copy()
        check(self.handle.lib.bsp_precond_apply(self.handle.h, self.p, _ptr(out)),
              "bsp_precond_apply", self.handle.h)
        return out.view(np.complex128) if cplx else out

    def info(self) -> dict:
        kind, lo, up, nnz = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        check(self.handle.lib.bsp_precond_info(self.p, C.byref(kind), C.byref(lo), C.byref(up),
                                               C.byref(nnz)), "bsp_precond_info")
        return {"kind": kind.value, "levels_lower": lo.value, "levels_upper": up.value,
                "factor_nnzb": nnz.value}

    def export(self) -> np.ndarray:
        inf = self.info()
        bs = self.A.bs
        nblk = inf["factor_nnzb"] if self.kind in (_lib.PC_ILU0, _lib.PC_ICHOL0, _lib.PC_LEARNED_LU) else self.A.n_rows
        out = np.zeros((nblk, bs, bs))
        check(self.handle.lib.bsp_precond_export(self.p, _ptr(out), out.size), "bsp_precond_export")
        return out

    def close(self) -> None:
        if getattr(self, "p", None):
            self.handle.lib.bsp_precond_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def NoPre(A: Matrix) -> None:
    """preConditioners::NoPre: no preconditioning (solvers take None)."""
    return None


def Diag(A: Matrix, inv: str = "LU", precision: int = _lib.PREC_F64) -> Precond:
    """Block-Jacobi: Diag<dense::LUFactor|CholeskyFactor> (preconditioners.hpp:75-111)."""
    return Precond(A, _lib.PC_DIAG_LU if inv == "LU" else _lib.PC_DIAG_CHOL, precision=precision)


def SOR(A: Matrix, w: float, nu: int, type_: int = 0, inv: str = "LU",
        precision: int = _lib.PREC_F64) -> Precond:
    """Block SOR from x = 0 (preconditioners.hpp:116-240); type <0 backward, 0 symmetric, >0 forward."""
    return Precond(A, _lib.PC_SOR_LU if inv == "LU" else _lib.PC_SOR_CHOL, w=w, nu=nu, type_=type_,
                   precision=precision)


def ILU0(A: Matrix, precision: int = _lib.PREC_F64) -> Precond:
    """Block ILU(0), natural order, no pivoting across blocks (preconditioners.hpp:246-357)."""
    return Precond(A, _lib.PC_ILU0, precision=precision)


def IChol0(A: Matrix, precision: int = _lib.PREC_F64) -> Precond:
    """Block IC(0) on A.lowTri() (preconditioners.hpp:364-538)."""
    return Precond(A, _lib.PC_ICHOL0, precision=precision)


# ---------------------------------------------------------------- solvers

def _opts(tol, max_iters, restart=-1, k=-1, print_iters=False, stop_rule=_lib.STOP_REFERENCE,
          precision=_lib.PREC_F64, inner_tol=1e-4, max_outer=50, print_eig_info=False) -> SolveOpts:
    return SolveOpts(float(tol), int(max_iters), int(restart), int(k), int(bool(print_iters)),
                     int(stop_rule), int(precision), float(inner_tol), int(max_outer), int(bool(print_eig_info)))


def _info_dict(info: SolveInfo) -> dict:
    return {f: getattr(info, f) for f, _ in SolveInfo._fields_}


def _solve(fn_dev, fn_host, A: Matrix, b, pc, opts: SolveOpts, return_info: bool):
    lib = A.handle.lib
    cap = max(4, opts.max_iters + 64 + (opts.max_iters // max(opts.restart, 1) if opts.restart > 0 else 0))
    hist = np.zeros(cap)
    info = SolveInfo()
    pcp = pc.p if pc is not None else None
    if hasattr(b, "data_ptr"):
        import torch
        x = torch.empty_like(b)
        st = getattr(lib, fn_dev)(A.handle.h, A.m, pcp, _ptr(b), _ptr(x), C.byref(opts), _ptr(hist),
                                  cap, C.byref(info))
    else:
        bb = _as_real(b, bool(A.complex_bs))
        x = np.zeros_like(bb)
        st = getattr(lib, fn_host)(A.handle.h, A.m, pcp, _ptr(bb), _ptr(x), C.byref(opts), _ptr(hist),
                                   cap, C.byref(info))
        if A.complex_bs:
            x = x.view(np.complex128)
    if st not in (_lib.BSP_OK, 4, 3, 5):  # MAXIT / BREAKDOWN / NAN still return x
        check(st, fn_dev, A.handle.h)
    if return_info:
        d = _info_dict(info)
        return x, d, hist[: info.n_hist].copy()
    return x


def pCG(A: Matrix, b, tol: float, preCond: Precond | None = None, maxIters: int = 1000,
        printIters: bool = False, return_info: bool = False, stop_rule: int = _lib.STOP_REFERENCE,
        precision: int = _lib.PREC_F64, inner_tol: float = 1e-6, max_outer: int = 50):
    """Preconditioned CG (blocksp_solvers.hpp:51-105); x_0 = 0.

    stop_rule=STOP_TRUE_RESIDUAL or precision != PREC_F64 wraps the solve in
    FP64 iterative refinement until ||b - A x|| / ||b|| <= tol."""
    return _solve("bsp_pcg_dev", "bsp_pcg", A, b, preCond,
                  _opts(tol, maxIters, print_iters=printIters, stop_rule=stop_rule,
                        precision=precision, inner_tol=inner_tol, max_outer=max_outer), return_info)


def pGMRES(A: Matrix, b, tol: float, preCond: Precond | None = None, maxIters: int = 500,
           restart: int = -1, k: int = -1, printIters: bool = False, return_info: bool = False,
           stop_rule: int = _lib.STOP_REFERENCE, precision: int = _lib.PREC_F64,
           inner_tol: float = 1e-6, max_outer: int = 50, printEigInfo: bool = False):
    """Left-preconditioned GMRES with optional deflated restart (blocksp_solvers.hpp:156-295).

    stop_rule / precision as for pCG.  printEigInfo prints the (harmonic, once
    restarted) Ritz value summary of the final Hessenberg matrix (:272-288)."""
    return _solve("bsp_pgmres_dev", "bsp_pgmres", A, b, preCond,
                  _opts(tol, maxIters, restart, k, printIters, stop_rule=stop_rule,
                        precision=precision, inner_tol=inner_tol, max_outer=max_outer,
                        print_eig_info=printEigInfo), return_info)


class Eigenvalues:
    """Eigenvalues_Arr (blocksp_dense_solvers.hpp:909-1000): real and imaginary
    parts, magnitudes and their statistics."""

    def __init__(self, wr: np.ndarray, wi: np.ndarray, harmonic_Ritz: bool = False):
        self.WR, self.WI = np.asarray(wr, float), np.asarray(wi, float)
        self.WM = np.sqrt(self.WR ** 2 + self.WI ** 2)
        self.harmonic_Ritz = harmonic_Ritz
        self.N = len(self.WR)

    def real(self): return self.WR
    def imag(self): return self.WI
    def mag(self): return self.WM
    def min_real(self): return float(self.WR.min())
    def max_real(self): return float(self.WR.max())
    def min_abs_real(self): return float(np.abs(self.WR).min())
    def max_abs_real(self): return float(np.abs(self.WR).max())
    def min_imag(self): return float(self.WI.min())
    def max_imag(self): return float(self.WI.max())
    def min_abs_imag(self): return float(np.abs(self.WI).min())
    def max_abs_imag(self): return float(np.abs(self.WI).max())
    def min_mag(self): return float(self.WM.min())
    def max_mag(self): return float(self.WM.max())
    def arg_min_mag(self): return int(np.argmin(self.WM))
    def arg_max_mag(self): return int(np.argmax(self.WM))
    def cond_number(self): return self.max_mag() / self.min_mag()

    def printEigInfo(self) -> None:
        print("Harmonic Ritz info" if self.harmonic_Ritz else "Eigenvalue info")
        print(f"min/max real eig {self.min_real():g} {self.max_real():g}")
        print(f"min/max img  eig {self.min_imag():g} {self.max_imag():g}")
        print(f"smallest magn eig {self.min_mag():g}")
        print(f"largest magn eig  {self.max_mag():g}")
        print(f"ratio/cond {self.cond_number():g}")

    def printEigVals(self) -> None:
        if self.harmonic_Ritz:
            print("Harmonic Ritz values")
        for title, v in (("real component", self.WR), ("imaginary component", self.WI), ("magnitude", self.WM)):
            print(f"Eigenvalues - {title}")
            print(" ".join(f"{x:g}" for x in v))


def arnoldi_eigenvalues(A: Matrix, iters: int = 30, preCond: Precond | None = None, printEigInfo: bool = False,
                        printEigVals: bool = False, harmonic_Ritz: bool = False) -> Eigenvalues:
    """arnoldi_eigenvalues (blocksp_solvers.hpp:306-334): Ritz (or harmonic Ritz)
    values of M^-1 A after `iters` Arnoldi steps from q_0 = e_0, on the GPU."""
    lib = A.handle.lib
    wr = np.zeros(max(1, iters))
    wi = np.zeros(max(1, iters))
    n = C.c_int()
    check(lib.bsp_arnoldi_eigenvalues(A.handle.h, A.m, preCond.p if preCond is not None else None, int(iters),
                                      int(bool(harmonic_Ritz)), int(bool(printEigInfo)), int(bool(printEigVals)),
                                      _ptr(wr), _ptr(wi), C.byref(n)), "bsp_arnoldi_eigenvalues", A.handle.h)
    return Eigenvalues(wr[:n.value], wi[:n.value], harmonic_Ritz)


class SOR_pGMRES:
    """pGMRES with block SOR / LU block inversion (blocksp_solvers.hpp:344-391)."""

    def __init__(self, A: Matrix, w: float = 1.6, nu: int = 3, SORtype: int = 0, tol: float = 1e-8,
                 maxIters: int = 5000, restart: int = -1, k: int = -1, printIters: bool = False):
        self.SOR_pre = SOR(A, w, nu, SORtype, "LU")
        self.tol, self.maxIters, self.restart, self.k, self.printIters = tol, maxIters, restart, k, printIters

    def solve(self, A: Matrix, b, return_info: bool = False):
        return pGMRES(A, b, self.tol, self.SOR_pre, self.maxIters, self.restart, self.k,
                      self.printIters, return_info)


class SOR_pCG:
    """pCG with symmetric block SOR / Cholesky block inversion (blocksp_solvers.hpp:395-431)."""

    def __init__(self, A: Matrix, w: float = 1.6, nu: int = 3, tol: float = 1e-8, maxIters: int = 5000,
                 printIters: bool = False):
        self.SOR_pre = SOR(A, w, nu, 0, "Chol")
        self.tol, self.maxIters, self.printIters = tol, maxIters, printIters

    def solve(self, A: Matrix, b, return_info: bool = False):
        return pCG(A, b, self.tol, self.SOR_pre, self.maxIters, self.printIters, return_info)


class ILU0_pGMRES:
    """pGMRES with block ILU0 (blocksp_solvers.hpp:434-467)."""

    def __init__(self, A: Matrix, tol: float = 1e-8, maxIters: int = 5000, restart: int = -1,
                 k: int = -1, printIters: bool = False):
        self.ILU0_pre = ILU0(A)
        self.tol, self.maxIters, self.restart, self.k, self.printIters = tol, maxIters, restart, k, printIters

    def solve(self, A: Matrix, b, return_info: bool = False):
        return pGMRES(A, b, self.tol, self.ILU0_pre, self.maxIters, self.restart, self.k,
                      self.printIters, return_info)


class IChol0_pCG:
    """pCG with block IChol0 (blocksp_solvers.hpp:471-498)."""

    def __init__(self, A: Matrix, tol: float = 1e-8, maxIters: int = 5000, printIters: bool = False):
        self.IChol0_pre = IChol0(A)
        self.tol, self.maxIters, self.printIters = tol, maxIters, printIters

    def solve(self, A: Matrix, b, return_info: bool = False):
        return pCG(A, b, self.tol, self.IChol0_pre, self.maxIters, self.printIters, return_info)


class ez:
    """One-call solvers with the reference's packaged defaults (blocksp_solvers.hpp:508-649):
    tolerance 1e-8 (FP64), maxIters 5000, SOR w = 1.6 (0.6 robust), nu = 3."""

    @staticmethod
    def sor_pGMRES(A, b, printIters=False):
        return SOR_pGMRES(A, 1.6, 3, 0, 1e-8, 5000, -1, -1, printIters).solve(A, b)

    @staticmethod
    def sor_pGMRES_robust(A, b, printIters=False):
        return SOR_pGMRES(A, 0.6, 3, 0, 1e-8, 5000, -1, -1, printIters).solve(A, b)

    @staticmethod
    def sor_pGMRES_dr(A, b, printIters=False):
        return SOR_pGMRES(A, 1.6, 3, 0, 1e-8, 5000, 30, 10, printIters).solve(A, b)

    @staticmethod
    def ilu0_pGMRES(A, b, printIters=False):
        return ILU0_pGMRES(A, 1e-8, 5000, -1, -1, printIters).solve(A, b)

    @staticmethod
    def ilu0_pGMRES_dr(A, b, printIters=False):
        return ILU0_pGMRES(A, 1e-8, 5000, 30, 10, printIters).solve(A, b)

    @staticmethod
    def sor_pCG(A, b, printIters=False):
        return SOR_pCG(A, 1.6, 3, 1e-8, 5000, printIters).solve(A, b)

    @staticmethod
    def ichol0_pCG(A, b, printIters=False):
        return IChol0_pCG(A, 1e-8, 5000, printIters).solve(A, b)


# ---------------------------------------------------------------- batched solver

class Batch:
    """Many independent SPD block systems solved together by block-IChol0 pCG.

    Equivalent to running ``IChol0_pCG<T,bs,1>(A_s, tol, maxIters).solve(A_s, b)``
    (blocksp_solvers.hpp:481-492) for every system s and every right-hand side,
    each (system, RHS) pair with its own alpha, beta and stopping test; the whole
    batch runs as one CUDA-graph launch.  ``systems`` are objects with
    ``row_ptr``, ``col_idx``, ``vals`` (n_blocks x bs x bs) and ``bs``.
    Vectors are the systems' solArray<T,bs,nrhs> blocks concatenated in order.
    """

    def __init__(self, systems, handle: Handle | None = None):
        self.handle = handle or default_handle()
        lib = self.handle.lib
        self.n_rows = np.array([len(s.row_ptr) - 1 for s in systems], dtype=np.int32)
        self.bs = np.array([s.bs for s in systems], dtype=np.int32)
        self.nnzb = np.array([len(s.col_idx) for s in systems], dtype=np.int64)
        rp = np.ascontiguousarray(np.concatenate([np.asarray(s.row_ptr, dtype=np.int32) for s in systems]))
        ci = np.ascontiguousarray(np.concatenate([np.asarray(s.col_idx, dtype=np.int32) for s in systems]))
        vals = np.ascontiguousarray(np.concatenate([np.asarray(s.vals, dtype=np.float64).ravel()
                                                    for s in systems]))
        b = C.c_void_p()
        check(lib.bsp_batch_create(self.handle.h, len(systems), _ptr(self.n_rows), _ptr(self.bs),
                                   _ptr(self.nnzb), _ptr(rp), _ptr(ci), _ptr(vals), C.byref(b)),
              "bsp_batch_create", self.handle.h)
        self.b = b
        self._last = (1, 0)
        self.handle.adopt(self)

    @property
    def n_sys(self) -> int:
        return int(self.n_rows.shape[0])

    def vector_size(self, nrhs: int) -> int:
        return int(np.sum(self.n_rows.astype(np.int64) * self.bs) * nrhs)

    def offsets(self, nrhs: int) -> np.ndarray:
        """Start of each system's block in a batch vector with nrhs right-hand sides."""
        sizes = self.n_rows.astype(np.int64) * self.bs * nrhs
        return np.concatenate([[0], np.cumsum(sizes)])

    def pcg(self, b, nrhs: int, tol: float = 1e-10, max_iters: int = 2000, mode: int = 0,
            check_every: int = 8, hist_cap: int = 0, retune: bool = False):
        """Solve; returns (x, info dict).  b is a device tensor or a host array."""
        lib = self.handle.lib
        opts = _lib.BatchOpts(float(tol), int(max_iters), int(mode), int(check_every), int(hist_cap),
                              int(bool(retune)))
        info = _lib.BatchInfo()
        if hasattr(b, "data_ptr"):
            import torch
            x = torch.empty_like(b)
            st = lib.bsp_batch_pcg_dev(self.handle.h, self.b, int(nrhs), _ptr(b), _ptr(x), C.byref(opts),
                                       C.byref(info))
        else:
            bb = np.ascontiguousarray(b, dtype=np.float64)
            x = np.zeros_like(bb)
            st = lib.bsp_batch_pcg(self.handle.h, self.b, int(nrhs), _ptr(bb), _ptr(x), C.byref(opts),
                                   C.byref(info))
        if st not in (_lib.BSP_OK, 4, 5):  # MAXIT / NAN still return x
            check(st, "bsp_batch_pcg", self.handle.h)
        self._last = (int(nrhs), int(hist_cap))
        return x, {f: getattr(info, f) for f, _ in _lib.BatchInfo._fields_}

    def results(self) -> dict:
        """Per-pair results of the last solve, arrays indexed [system, rhs]."""
        nrhs, hcap = self._last
        n = self.n_sys * nrhs
        iters = np.zeros(n, dtype=np.int32)
        state = np.zeros(n, dtype=np.int32)
        res = np.zeros(n)
        hist = np.zeros((n, hcap)) if hcap > 0 else None
        check(self.handle.lib.bsp_batch_results(self.b, nrhs, _ptr(iters), _ptr(state), _ptr(res),
                                                _ptr(hist) if hist is not None else None, hcap),
              "bsp_batch_results")
        out = {"iters": iters.reshape(self.n_sys, nrhs), "state": state.reshape(self.n_sys, nrhs),
               "final_res": res.reshape(self.n_sys, nrhs)}
        if hist is not None:
            out["hist"] = hist.reshape(self.n_sys, nrhs, hcap)
        return out

    def tuning(self) -> list[dict]:
        """Groups (one per block size) with the launch shapes the autotuner chose."""
        k = 4
        ng = C.c_int()
        arr = {n: np.zeros(k, dtype=np.int32) for n in ("bs", "systems", "tile_threads", "tile_ctas_per_sm",
                                                        "sweep_ctas_per_sm")}
        rows = np.zeros(k, dtype=np.int64)
        check(self.handle.lib.bsp_batch_tuning(self.b, C.byref(ng), _ptr(arr["bs"]), _ptr(arr["systems"]),
                                               _ptr(rows), _ptr(arr["tile_threads"]),
                                               _ptr(arr["tile_ctas_per_sm"]), _ptr(arr["sweep_ctas_per_sm"])),
              "bsp_batch_tuning")
        return [{**{n: int(v[i]) for n, v in arr.items()}, "rows": int(rows[i])} for i in range(ng.value)]

    def close(self) -> None:
        if getattr(self, "b", None):
            self.handle.lib.bsp_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
