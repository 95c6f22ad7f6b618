"""CPU oracle: a numpy/scipy restatement of BlockSp's solve path.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the GPU path is
compared against; it is imported by ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` and by nothing in the product package.

It restates, function by function, the reference library BlockSp v1.0 (file
paths are those of the reference project):

* ``bsmv``            blocksp_multiply.hpp:166-325 (both overloads, transpose)
* ``dot``/``two_norm``  blocksp_containers.hpp:974-1012
* ``LUFactor``        blocksp_dense_solvers.hpp:47-110 (getrf/getrs, small_solve for N<=3)
* ``CholeskyFactor``  blocksp_dense_solvers.hpp:123-190 (packed Cholesky)
* ``Diag``            blocksp_preconditioners.hpp:75-111 (+ makeADInv :22-63)
* ``SOR``             blocksp_preconditioners.hpp:116-240
* ``ILU0``            blocksp_preconditioners.hpp:246-357
* ``IChol0``          blocksp_preconditioners.hpp:364-538
* ``pcg``             blocksp_solvers.hpp:51-105
* ``pgmres``          blocksp_solvers.hpp:107-295
* ``deflated_restart``  blocksp_deflated_restart.hpp:38-269

The dense LAPACK steps (getrf, getrs, potrf, gels, gees, trsen, geqrf, orgqr)
are the third-party boundary of the reference (Intel MKL, no version pinned).
They are restated here by calling the same LAPACK routines through
``scipy.linalg.lapack`` (scipy's bundled OpenBLAS / reference-LAPACK
algorithms).  Pinning: this restatement is checked against the reference
itself, compiled from its own headers by ``oracle/Makefile`` (binaries in
``oracle/_ref/``), through the golden fixtures in ``tests/golden/``, and against
the reference's LDG known answer (infinity-norm error ~2.9e-4).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.linalg.lapack as lap

EPS = np.finfo(np.float64).eps


@dataclass
class BSR:
    """Block CSR in the reference's row-wise layout (columns in stored order)."""

    n: int
    bs: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    vals: np.ndarray  # [nnzb, bs, bs] row-major blocks
    n_cols: int | None = None

    def __post_init__(self):
        if self.n_cols is None:
            self.n_cols = self.n
        self._pos = None

    @classmethod
    def from_system(cls, s) -> "BSR":
        return cls(s.n, s.bs, np.asarray(s.row_ptr), np.asarray(s.col_idx),
                   np.array(s.vals, dtype=np.float64, copy=True))

    def cols(self, i: int) -> np.ndarray:
        return self.col_idx[self.row_ptr[i]:self.row_ptr[i + 1]]

    def pos(self, i: int, j: int) -> int:
        """Block index of (i, j) or -1 (CSR::scan, containers.hpp:211-216)."""
        if self._pos is None:
            self._pos = {}
            for r in range(self.n):
                for t in range(self.row_ptr[r], self.row_ptr[r + 1]):
                    self._pos[(r, int(self.col_idx[t]))] = t
        return self._pos.get((i, j), -1)

    def row_indices_by_col(self) -> list[list[int]]:
        """rowIndicesByCol (containers.hpp:410-417), rows in increasing order."""
        ind = [[] for _ in range(self.n_cols)]
        for i in range(self.n):
            for j in self.cols(i):
                ind[int(j)].append(i)
        return ind

    def low_tri(self) -> "BSR":
        """lowTri() (containers.hpp:277-285): blocks with col <= row, row order kept."""
        rp = [0]
        ci, vs = [], []
        for i in range(self.n):
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                if self.col_idx[t] <= i:
                    ci.append(self.col_idx[t])
                    vs.append(self.vals[t])
            rp.append(len(ci))
        return BSR(self.n, self.bs, np.array(rp, dtype=np.int32), np.array(ci, dtype=np.int32),
                   np.array(vs).reshape(-1, self.bs, self.bs), self.n_cols)


# ---------------------------------------------------------------- block algebra

class _Rows:
    """Row lists of (col, block) in creation order: the reference container's
    operator() appends a missing block at the end of its row
    (containers.hpp:147-164)."""

    def __init__(self, m: int, bs: int):
        self.bs = bs
        self.rows = [dict() for _ in range(m)]  # dicts keep insertion order

    def at(self, i: int, j: int) -> np.ndarray:
        r = self.rows[i]
        if j not in r:
            r[j] = np.zeros((self.bs, self.bs))
        return r[j]

    def to_bsr(self, n_cols: int) -> BSR:
        rp, ci, vs = [0], [], []
        for r in self.rows:
            for j, v in r.items():
                ci.append(j)
                vs.append(v)
            rp.append(len(ci))
        return BSR(len(self.rows), self.bs, np.array(rp, dtype=np.int32), np.array(ci, dtype=np.int32),
                   np.array(vs).reshape(-1, self.bs, self.bs), n_cols)


def bs_id(n: int, bs: int) -> BSR:
    """blkSpIdent (multiply.hpp:21-28)."""
    return BSR(n, bs, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
               np.repeat(np.eye(bs)[None], n, axis=0))


def bs_tr(A: BSR) -> BSR:
    """blkSpTranspose (multiply.hpp:31-42): tran(colInd, im) = A(im, colInd)^T,
    rows scanned in increasing order."""
    R = _Rows(A.n_cols, A.bs)
    for i in range(A.n):
        for t in range(A.row_ptr[i], A.row_ptr[i + 1]):
            R.at(int(A.col_idx[t]), i)[...] = A.vals[t].T
    return R.to_bsr(A.n)


def _mat_mat(a: np.ndarray, b: np.ndarray, a_trans: bool = False) -> np.ndarray:
    """dense::matMat (dense_multiply.hpp:130-190): loops im, ik, in with the
    inner index ascending (the nested-loop form the reference uses up to 8x8)."""
    if a_trans:
        a = a.T
    out = np.zeros((a.shape[0], b.shape[1]))
    for k in range(a.shape[1]):
        out += np.outer(a[:, k], b[k, :])
    return out


def bsmm(A: BSR, B: BSR, a_trans: bool = False) -> BSR:
    """blkSpMatMat (multiply.hpp:51-133): C(imA, colIndB) += A(imA, colIndA) B(colIndA, colIndB)
    or, transposed, C(colIndA, colIndB) += A(imA, colIndA)^T B(imA, colIndB)."""
    R = _Rows(A.n_cols if a_trans else A.n, A.bs)
    for i in range(A.n):
        for a in range(A.row_ptr[i], A.row_ptr[i + 1]):
            k = int(A.col_idx[a])
            src = i if a_trans else k
            for b in range(B.row_ptr[src], B.row_ptr[src + 1]):
                j = int(B.col_idx[b])
                row = k if a_trans else i
                blk = R.at(row, j)
                blk += _mat_mat(A.vals[a], B.vals[b], a_trans)
    return R.to_bsr(B.n_cols)


def matrix_add(alpha: float, A: BSR, beta: float, B: BSR) -> BSR:
    """alpha A + beta B as the container computes A1 += A2 after scaling
    (containers.hpp:302-318, 340-347): A's blocks, then B's new blocks."""
    R = _Rows(A.n, A.bs)
    for i in range(A.n):
        for t in range(A.row_ptr[i], A.row_ptr[i + 1]):
            R.at(i, int(A.col_idx[t]))[...] = alpha * A.vals[t] if alpha != 1.0 else A.vals[t]
        for t in range(B.row_ptr[i], B.row_ptr[i + 1]):
            R.at(i, int(B.col_idx[t]))[...] += beta * B.vals[t]
    return R.to_bsr(A.n_cols)


# ---------------------------------------------------------------- bsmv / vectors

def bsmv(A: BSR, x: np.ndarray, nrhs: int = 1, transpose: bool = False) -> np.ndarray:
    """y = op(A) x.  nrhs > 1: the BlockSp<T,B> x solArray<T,B,D> form, each
    dimension an independent right-hand side (multiply.hpp:170-205); nrhs == 1
    covers BlockSp<T,B*D> x solArray<T,B,D> (multiply.hpp:209-246) because the
    element layout equals tvConcat order (utility.hpp:257-265)."""
    bs = A.bs
    if not transpose:
        X = np.asarray(x, dtype=np.float64).reshape(A.n_cols, nrhs, bs)
        rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
        contrib = np.einsum("tab,trb->tra", A.vals, X[A.col_idx])
        Y = np.zeros((A.n, nrhs, bs))
        np.add.at(Y, rows, contrib)
    else:
        X = np.asarray(x, dtype=np.float64).reshape(A.n, nrhs, bs)
        rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
        contrib = np.einsum("tba,trb->tra", A.vals, X[rows])  # A_ij^T x_i
        Y = np.zeros((A.n_cols, nrhs, bs))
        np.add.at(Y, A.col_idx, contrib)
    return Y.reshape(-1)


def dot(x: np.ndarray, y: np.ndarray) -> float:
    """dot (containers.hpp:974-996), reals."""
    return float(np.dot(x, y))


def two_norm(x: np.ndarray) -> float:
    """twoNorm = sqrt(|dot(x,x)|) (containers.hpp:998-1012)."""
    return math.sqrt(abs(dot(x, x)))


# ---------------------------------------------------------------- dense blocks

def _explicit_small_inv(A: np.ndarray) -> np.ndarray:
    return np.linalg.inv(A)


class LUFactor:
    """dense::LUFactor<T,N> (dense_solvers.hpp:47-110)."""

    def __init__(self, A: np.ndarray):
        self.N = A.shape[0]
        self.A = np.array(A, dtype=np.float64)
        if self.N > 3:
            self.lu, self.piv, info = lap.dgetrf(self.A)
            self.info = info

    def invmul(self, x: np.ndarray) -> np.ndarray:
        """A^{-1} x (getrs 'N'; small_solve for N <= 3, dense_solvers.hpp:1029-1056)."""
        if self.N == 1:
            return x / self.A[0, 0]
        if self.N == 2:
            a = self.A
            det = a[0, 0] * a[1, 1] - a[0, 1] * a[1, 0]
            if x.ndim == 1:
                return np.array([(a[1, 1] * x[0] - a[0, 1] * x[1]) / det,
                                 (-a[1, 0] * x[0] + a[0, 0] * x[1]) / det])
            return np.linalg.solve(a, x)
        if self.N == 3:
            return _explicit_small_inv(self.A) @ x
        out, info = lap.dgetrs(self.lu, self.piv, x)
        return out

    def r_invmul(self, X: np.ndarray) -> np.ndarray:
        """X A^{-1} via A^T Y^T = X^T (dense_solvers.hpp:97-108)."""
        if self.N <= 3:
            return X @ np.linalg.inv(self.A)
        out, info = lap.dgetrs(self.lu, self.piv, X.T.copy(), trans=1)
        return out.T.copy()


class CholeskyFactor:
    """dense::CholeskyFactor<T,N> (dense_solvers.hpp:123-190): A = L L^T."""

    def __init__(self, A: np.ndarray):
        self.N = A.shape[0]
        self.A = np.array(A, dtype=np.float64)
        if self.N > 3:
            self.c, self.info = lap.dpotrf(self.A, lower=1, clean=1)

    def invmul(self, x: np.ndarray) -> np.ndarray:
        if self.N <= 3:
            return LUFactor(self.A).invmul(x) if self.N < 3 else np.linalg.inv(self.A) @ x
        out, info = lap.dpotrs(self.c, x, lower=1)
        return out


def make_ad_inv(A: BSR, inv=LUFactor) -> list:
    """makeADInv (preconditioners.hpp:22-63) with test_zero_eigenvalues = false."""
    out = []
    for i in range(A.n):
        t = A.pos(i, i)
        out.append(inv(A.vals[t] if t >= 0 else np.zeros((A.bs, A.bs))))
    return out


# ---------------------------------------------------------------- preconditioners

class Diag:
    """preConditioners::Diag (preconditioners.hpp:75-111)."""

    def __init__(self, A: BSR, inv=LUFactor):
        self.bs = A.bs
        self.AD_Inv = make_ad_inv(A, inv)

    def __call__(self, r: np.ndarray) -> np.ndarray:
        X = r.reshape(-1, self.bs)
        return np.concatenate([self.AD_Inv[i].invmul(X[i]) for i in range(len(self.AD_Inv))])


class SOR:
    """preConditioners::SOR (preconditioners.hpp:116-240): nu forward and/or
    backward block sweeps from x = 0 with damping w; type <0 backward only,
    0 symmetric, >0 forward only."""

    def __init__(self, A: BSR, w: float, nu: int, type_: int = 0, inv=LUFactor):
        self.A = A
        self.w, self.nu, self.type = w, nu, type_
        self.AD_Inv = make_ad_inv(A, inv)

    def _sweep(self, x: np.ndarray, b: np.ndarray, rows) -> None:
        A, bs, w = self.A, self.A.bs, self.w
        X = x.reshape(-1, bs)
        Bv = b.reshape(-1, bs)
        for im in rows:  # oneSORForw :131-166 / oneSORBack :171-202
            ph = np.zeros(bs)
            for t in range(A.row_ptr[im], A.row_ptr[im + 1]):
                c = A.col_idx[t]
                if c != im:
                    ph += A.vals[t] @ X[c]
            ph = Bv[im] - ph
            ph = self.AD_Inv[im].invmul(ph)
            X[im] += -w * X[im] + w * ph

    def __call__(self, r: np.ndarray) -> np.ndarray:
        n = self.A.n
        x = np.zeros_like(r)
        fwd, bwd = range(n), range(n - 1, -1, -1)
        if self.type < 0:
            for _ in range(self.nu):
                self._sweep(x, r, bwd)
        elif self.type == 0:
            for _ in range(self.nu):
                self._sweep(x, r, fwd)
            for _ in range(self.nu):
                self._sweep(x, r, bwd)
        else:
            for _ in range(self.nu):
                self._sweep(x, r, fwd)
        return x


class ILU0:
    """preConditioners::ILU0 (preconditioners.hpp:246-357)."""

    def __init__(self, A: BSR):
        self.LU = BSR(A.n, A.bs, A.row_ptr, A.col_idx, np.array(A.vals, copy=True), A.n_cols)
        self.n = A.n
        self.rowInd = A.row_indices_by_col()
        self._factor()
        self.D_Inv = make_ad_inv(self.LU, LUFactor)

    def _factor(self) -> None:
        """In-place right-looking block ILU(0), natural order (:274-291)."""
        A = self.LU
        rowset = [set(r) for r in self.rowInd]
        for i in range(self.n):
            AD_Inv = LUFactor(A.vals[A.pos(i, i)])
            for k in self.rowInd[i]:
                if k > i:
                    t = A.pos(k, i)
                    A.vals[t] = AD_Inv.r_invmul(A.vals[t])
            for k in self.rowInd[i]:
                if k > i:
                    Lki = A.vals[A.pos(k, i)]
                    for j in A.cols(k):
                        j = int(j)
                        if j > i and i in rowset[j]:
                            A.vals[A.pos(k, j)] -= Lki @ A.vals[A.pos(i, j)]

    def __call__(self, x: np.ndarray) -> np.ndarray:
        """invmul: unit-L forward then U backward (:294-349)."""
        LU, bs = self.LU, self.LU.bs
        X = np.array(x, dtype=np.float64).reshape(-1, bs)
        for im in range(1, self.n):
            for t in range(LU.row_ptr[im], LU.row_ptr[im + 1]):
                c = LU.col_idx[t]
                if c < im:
                    X[im] -= LU.vals[t] @ X[c]
        for im in range(self.n - 1, -1, -1):
            for t in range(LU.row_ptr[im], LU.row_ptr[im + 1]):
                c = LU.col_idx[t]
                if c > im:
                    X[im] -= LU.vals[t] @ X[c]
            X[im] = self.D_Inv[im].invmul(X[im])
        return X.reshape(-1)


class IChol0:
    """preConditioners::IChol0 (preconditioners.hpp:364-538): L L^T with the
    sparsity of A.lowTri()."""

    def __init__(self, A: BSR):
        self.n = A.n
        self.L = A.low_tri()
        self.rowInd = A.row_indices_by_col()
        self._factor()
        self.rowInd = self.L.row_indices_by_col()

    def _factor(self) -> None:
        L, bs = self.L, self.L.bs
        rowset = [set(r) for r in self.rowInd]
        for i in range(self.n):
            t = L.pos(i, i)
            c, info = lap.dpotrf(L.vals[t], lower=1, clean=1)  # potrf 'L' (:398-406)
            self.info = info
            L.vals[t] = c
            Lii = L.vals[t]
            for k in self.rowInd[i]:
                if k > i:  # L_ki = A_ki L_ii^{-T} (:411-421)
                    tk = L.pos(k, i)
                    Y = L.vals[tk].T.copy()
                    for r in range(bs):  # Lii_Inv_forward_subst on columns (:494-505)
                        Y[r] -= Lii[r, :r] @ Y[:r]
                        Y[r] /= Lii[r, r]
                    L.vals[tk] = Y.T
            for k in self.rowInd[i]:
                if k > i:
                    Lki = L.vals[L.pos(k, i)]
                    for j in L.cols(k):
                        j = int(j)
                        if i < j <= k and i in rowset[j]:
                            L.vals[L.pos(k, j)] -= Lki @ L.vals[L.pos(j, i)].T

    def __call__(self, x: np.ndarray) -> np.ndarray:
        """invmul: L forward then L^T backward (:432-489)."""
        L, bs = self.L, self.L.bs
        X = np.array(x, dtype=np.float64).reshape(-1, bs)
        for im in range(self.n):
            for t in range(L.row_ptr[im], L.row_ptr[im + 1]):
                c = L.col_idx[t]
                if c < im:
                    X[im] -= L.vals[t] @ X[c]
            Lii = L.vals[L.pos(im, im)]
            for r in range(bs):
                X[im, r] = (X[im, r] - Lii[r, :r] @ X[im, :r]) / Lii[r, r]
        for im in range(self.n - 1, -1, -1):
            for row in self.rowInd[im]:
                if row != im:
                    X[im] -= L.vals[L.pos(row, im)].T @ X[row]
            Lii = L.vals[L.pos(im, im)]
            for r in range(bs - 1, -1, -1):
                X[im, r] = (X[im, r] - Lii[r + 1:, r] @ X[im, r + 1:]) / Lii[r, r]
        return X.reshape(-1)


def no_pre(x: np.ndarray) -> np.ndarray:
    return x


# ---------------------------------------------------------------- solvers

@dataclass
class SolveResult:
    x: np.ndarray
    hist: list
    iters: int
    restarts: int = 0


def pcg(A: BSR, b: np.ndarray, tol: float, pre=no_pre, max_iters: int = 1000,
        matvec=None) -> SolveResult:
    """pCG (solvers.hpp:51-105), including its mixed stopping test: the first
    history entry is ||M^-1 b|| and later ones are the recursive ||r||.
    ``matvec`` (default: bsmv with A) lets tests perturb the product."""
    mv = matvec or (lambda v: bsmv(A, v))
    x = np.zeros_like(b)
    r = b.copy()
    p = pre(r.copy())
    z = p.copy()
    res = [math.sqrt(dot(p, p))]
    tolerance = res[-1] * tol
    it = 0
    while res[-1] > tolerance:
        Ap = mv(p)
        rz = dot(r, z)
        alpha = rz / dot(p, Ap)
        x += alpha * p
        r -= alpha * Ap
        res.append(math.sqrt(dot(r, r)))
        if res[-1] > tolerance:
            z = pre(r.copy())
            beta = dot(r, z) / rz
            p = z + beta * p
            it += 1
            if it > max_iters:
                break
    return SolveResult(x, res, it)


def _one_arnoldi(it, H, Qn, A, pre, zero_thresh):
    """one_arnoldi (solvers.hpp:109-136): MGS, H grown to (it+2, it+1)."""
    m, n = it + 2, it + 1
    Hn = np.zeros((m, n))
    Hn[:H.shape[0], :H.shape[1]] = H
    v = pre(bsmv(A, Qn[it]))
    for j in range(it + 1):
        Hn[j, it] = dot(Qn[j], v)
        v = v - Hn[j, it] * Qn[j]
    Hn[it + 1, it] = two_norm(v)
    if abs(Hn[it + 1, it]) < zero_thresh:
        return Hn
    Qn.append(v / Hn[it + 1, it])
    return Hn


def ritz_values(H: np.ndarray, harmonic: bool = False) -> np.ndarray:
    """Eigenvalues_Arr (dense_solvers.hpp:916-961) of H's square part H_s;
    harmonic: of H_s + h_mn^2 H_s^-T e_n e_n^T.  LAPACK gees stands for the
    reference's call through numpy."""
    n = H.shape[1]
    Hs = H[:n, :n].copy()
    if harmonic:
        e = np.zeros(n)
        e[-1] = 1.0
        Hs[:, -1] += H[n, n - 1] ** 2 * np.linalg.solve(Hs.T, e)
    return np.linalg.eigvals(Hs)


def arnoldi_eigenvalues(A: BSR, iters: int = 30, pre=no_pre, harmonic: bool = False) -> np.ndarray:
    """arnoldi_eigenvalues (solvers.hpp:306-334): iters Arnoldi steps of M^-1 A
    from q_0 = e_0 (stopping where the Krylov space is exhausted), then the
    (harmonic) Ritz values."""
    nv = A.n * A.bs
    q0 = np.zeros(nv)
    q0[0] = 1.0
    Qn = [q0]
    H = np.zeros((1, 0))
    zero_thresh = 10 * A.bs * A.bs * np.finfo(float).eps
    for it in range(min(iters, nv)):
        H = _one_arnoldi(it, H, Qn, A, pre, zero_thresh)
        if len(Qn) < it + 2:
            break
    return ritz_values(H, harmonic)


def deflated_restart(H, Qn, res_vec, res_mag, k):
    """Morgan's GMRES-DR restart (deflated_restart.hpp:38-269), real case.

    Returns (H_new, Qn_new, c_r, res_mag_new, k_eff)."""
    m, n = H.shape
    if k > n:
        k = n
    zero_thresh = 10 * n * n * EPS
    if k == 0:
        return np.zeros((0, 0)), [], np.zeros(1), [], 0
    Hn = H[:n, :n].copy()
    h_mn = H[n, n - 1]
    w = np.zeros(n)
    w[n - 1] = 1.0
    lu, piv, _ = lap.dgetrf(Hn.T.copy())
    w, _ = lap.dgetrs(lu, piv, w)
    Hn[:, n - 1] += h_mn * h_mn * w
    # (2) real Schur, select the k smallest |theta| (pairs kept together), reorder
    t, sdim, wr, wi, Z, _, info = lap.dgees(lambda a, b: False, Hn, compute_v=1, sort_t=0)
    mags = np.sqrt(wr * wr + wi * wi)
    perm = sorted(range(n), key=lambda i: mags[i])  # std::sort on magnitude
    select = np.zeros(n, dtype=np.int32)
    cnt = 0
    for i in range(n):
        if cnt >= k:
            break
        ip = perm[i]
        if select[ip]:
            continue
        select[ip] = 1
        cnt += 1
        if abs(wi[ip]) > zero_thresh:
            for j in range(n):
                if j != ip and abs(wr[j] - wr[ip]) < zero_thresh and abs(wi[j] + wi[ip]) < zero_thresh:
                    if not select[j]:
                        select[j] = 1
                        cnt += 1
                    break
    ts, qs, wr2, wi2, mk, s, sep, info = lap.dtrsen(select, t, Z, job="V", lwork=max(1, n * n),
                                                    liwork=max(1, n * n))
    k = int(mk)
    # (3) P_k = first k Schur vectors, orthonormalised by QR
    Pk = qs[:, :k].copy()
    qr, tau, _, _ = lap.dgeqrf(Pk)
    Pk, _, _ = lap.dorgqr(qr, tau)
    # (4) P_{k+1}
    Pk1 = np.zeros((n + 1, k + 1))
    Pk1[:n, :k] = Pk
    Pk1[:, k] = res_vec
    for i in range(k):
        d = float(np.dot(Pk1[:, i], Pk1[:, k]))
        Pk1[:, k] -= d * Pk1[:, i]
    Pk1[:, k] /= math.sqrt(float(np.dot(Pk1[:, k], Pk1[:, k])))
    # (5) c_r, (6) H_new, (7) Qn_new
    c_r = Pk1.T @ res_vec
    H_new = Pk1.T @ (H @ Pk)
    Qmat = np.stack(Qn[:m], axis=1)
    Qn_new = [Qmat @ Pk1[:, i] for i in range(k + 1)]
    return H_new, Qn_new, c_r, [res_mag[-1]], k


def pgmres(A: BSR, b: np.ndarray, tol: float, pre=no_pre, max_iters: int = 500,
           restart: int = -1, k: int = -1) -> SolveResult:
    """Left-preconditioned pGMRES with deflated restart (solvers.hpp:156-295).

    The returned history is every res_mag value in push order (after a
    restart the reference resets res_mag to its last entry; the same value is
    not repeated here)."""
    hist = []
    r0 = pre(b.copy())
    res_mag = [two_norm(r0)]
    hist.append(res_mag[0])
    Qn = [r0 / res_mag[0]]
    H = np.zeros((0, 0))
    x0 = np.zeros_like(b)
    zero_thresh = min(res_mag[0] * EPS, EPS)
    tolerance = res_mag[0] * tol
    it = tot = 0
    y = np.zeros(0)
    c_r = np.zeros(0)
    restarted = False
    n_restarts = 0
    while res_mag[-1] > tolerance:
        H = _one_arnoldi(it, H, Qn, A, pre, zero_thresh)
        m, n = it + 2, it + 1
        rhs = np.zeros(m)
        if not restarted:
            rhs[0] = res_mag[0]
        else:
            rhs[:len(c_r)] = c_r
        _, sol, info = lap.dgels(H.copy(), rhs.copy())
        y = sol[:n].copy()
        res_vec = rhs - H @ y
        res_mag.append(math.sqrt(float(np.sum(res_vec * res_vec))))
        hist.append(res_mag[-1])
        it += 1
        tot += 1
        if tot > max_iters:
            break
        if it == restart and res_mag[-1] > tolerance:
            x = x0.copy()
            for iy in range(len(y)):
                x += y[iy] * Qn[iy]
            x0 = x
            r0 = pre(b - bsmv(A, x0))
            H, Qn, c_r, res_mag, keff = deflated_restart(H, Qn, res_vec, res_mag, k)
            n_restarts += 1
            it = 0 if k == 0 else H.shape[1]
            if k == 0:
                res_mag.append(two_norm(r0))
                hist.append(res_mag[-1])
                c_r = np.array([res_mag[-1]])
                Qn = [r0 / res_mag[-1]]
            restarted = k != 0
    x = x0.copy()
    for iy in range(len(y)):
        x += y[iy] * Qn[iy]
    return SolveResult(x, hist, tot, n_restarts)


def true_rel_residual(A: BSR, b: np.ndarray, x: np.ndarray) -> float:
    r = b - bsmv(A, x)
    return float(np.linalg.norm(r) / np.linalg.norm(b))
