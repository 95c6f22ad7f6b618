"""CPU oracle of the solve path with T = std::complex<double> (numpy/scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker; never part of the
product path.

Restates the complex branches of the reference BlockSp v1.0 (paths are the
reference project's):

* ``bsmv``              blocksp_multiply.hpp:209-246 (complex blocks)
* ``dot``/``two_norm``  dot = sum conj(x_i) y_i (bdot, blocksp_utility.hpp:277-292);
                        twoNorm = sqrt(|dot(x, x)|) (blocksp_containers.hpp:998-1012)
* ``LUFactor``          blocksp_dense_solvers.hpp:47-110 with zgetrf / zgetrs
                        (explicit inverse for N <= 3, as the real oracle)
* ``Diag``, ``SOR``, ``ILU0``  blocksp_preconditioners.hpp:75-357 (the same
                        block algorithms in complex arithmetic)
* ``pgmres``            blocksp_solvers.hpp:107-295: zgels per step, |v|^2 as
                        conj(v) v (:206, :231)
* ``deflated_restart``  blocksp_deflated_restart.hpp:38-269, complex branch:
                        H_n^-H (conjugate transposes, blocksp_dense_multiply.hpp:206-216),
                        zgees + ztrsen on the k smallest |theta|, zgeqrf + zungqr,
                        Gram-Schmidt and c_r with conj, H_new = P^H H P_k

The LAPACK steps are scipy.linalg.lapack's z-routines, the ones the
reference calls through MKL.  Pinned against the reference itself, built with
T = std::complex<double> by oracle/Makefile (``_ref/ref_complex_hist``),
through the fixtures tests/golden/c_*.npz.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg.lapack as lap

from .blocksp_oracle import BSR, SolveResult

EPS = np.finfo(np.float64).eps


def bsmv(A: BSR, x: np.ndarray) -> np.ndarray:
    X = np.asarray(x, dtype=np.complex128).reshape(A.n_cols, A.bs)
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    contrib = np.einsum("tab,tb->ta", A.vals, X[A.col_idx])
    Y = np.zeros((A.n, A.bs), dtype=np.complex128)
    np.add.at(Y, rows, contrib)
    return Y.reshape(-1)


def dot(x: np.ndarray, y: np.ndarray) -> complex:
    return complex(np.vdot(x, y))


def two_norm(x: np.ndarray) -> float:
    return math.sqrt(abs(dot(x, x)))


class LUFactor:
    def __init__(self, A: np.ndarray):
        self.N = A.shape[0]
        self.A = np.array(A, dtype=np.complex128)
        if self.N > 3:
            self.lu, self.piv, self.info = lap.zgetrf(self.A)

    def invmul(self, x: np.ndarray) -> np.ndarray:
        if self.N <= 3:
            return np.linalg.inv(self.A) @ x
        out, info = lap.zgetrs(self.lu, self.piv, x)
        return out

    def r_invmul(self, X: np.ndarray) -> np.ndarray:
        """X A^{-1}"""
        if self.N <= 3:
            return X @ np.linalg.inv(self.A)
        out, info = lap.zgetrs(self.lu, self.piv, X.T.copy(), trans=1)
        return out.T.copy()


def make_ad_inv(A: BSR) -> list:
    return [LUFactor(A.vals[A.pos(i, i)]) for i in range(A.n)]


class Diag:
    def __init__(self, A: BSR):
        self.bs = A.bs
        self.inv = make_ad_inv(A)

    def __call__(self, r: np.ndarray) -> np.ndarray:
        X = np.asarray(r, dtype=np.complex128).reshape(-1, self.bs)
        return np.concatenate([self.inv[i].invmul(X[i]) for i in range(len(self.inv))])


class SOR:
    def __init__(self, A: BSR, w: float, nu: int, type_: int = 0):
        self.A, self.w, self.nu, self.type = A, w, nu, type_
        self.inv = make_ad_inv(A)

    def _sweep(self, X, Bv, rows) -> None:
        A, w = self.A, self.w
        for im in rows:
            ph = np.zeros(A.bs, dtype=np.complex128)
            for t in range(A.row_ptr[im], A.row_ptr[im + 1]):
                c = A.col_idx[t]
                if c != im:
                    ph += A.vals[t] @ X[c]
            X[im] += -w * X[im] + w * self.inv[im].invmul(Bv[im] - ph)

    def __call__(self, r: np.ndarray) -> np.ndarray:
        n, bs = self.A.n, self.A.bs
        X = np.zeros((n, bs), dtype=np.complex128)
        Bv = np.asarray(r, dtype=np.complex128).reshape(n, bs)
        fwd, bwd = range(n), range(n - 1, -1, -1)
        seq = ([bwd] * self.nu if self.type < 0 else
               [fwd] * self.nu + [bwd] * self.nu if self.type == 0 else [fwd] * self.nu)
        for rows in seq:
            self._sweep(X, Bv, rows)
        return X.reshape(-1)


class ILU0:
    def __init__(self, A: BSR):
        self.LU = BSR(A.n, A.bs, A.row_ptr, A.col_idx, np.array(A.vals, dtype=np.complex128, copy=True), A.n_cols)
        self.n = A.n
        LU = self.LU
        rowInd = A.row_indices_by_col()
        rowset = [set(r) for r in rowInd]
        for i in range(self.n):
            Dinv = LUFactor(LU.vals[LU.pos(i, i)])
            for k in rowInd[i]:
                if k > i:
                    t = LU.pos(k, i)
                    LU.vals[t] = Dinv.r_invmul(LU.vals[t])
            for k in rowInd[i]:
                if k > i:
                    Lki = LU.vals[LU.pos(k, i)]
                    for j in LU.cols(k):
                        j = int(j)
                        if j > i and i in rowset[j]:
                            LU.vals[LU.pos(k, j)] -= Lki @ LU.vals[LU.pos(i, j)]
        self.D_inv = make_ad_inv(LU)

    def __call__(self, x: np.ndarray) -> np.ndarray:
        LU, bs = self.LU, self.LU.bs
        X = np.array(x, dtype=np.complex128).reshape(-1, bs)
        for im in range(1, self.n):
            for t in range(LU.row_ptr[im], LU.row_ptr[im + 1]):
                if LU.col_idx[t] < im:
                    X[im] -= LU.vals[t] @ X[LU.col_idx[t]]
        for im in range(self.n - 1, -1, -1):
            for t in range(LU.row_ptr[im], LU.row_ptr[im + 1]):
                if LU.col_idx[t] > im:
                    X[im] -= LU.vals[t] @ X[LU.col_idx[t]]
            X[im] = self.D_inv[im].invmul(X[im])
        return X.reshape(-1)


def no_pre(x):
    return np.array(x, dtype=np.complex128, copy=True)


def _one_arnoldi(it, H, Qn, A, pre, zero_thresh):
    m, n = it + 2, it + 1
    Hn = np.zeros((m, n), dtype=np.complex128)
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


def deflated_restart(H, Qn, res_vec, res_mag, k):
    """Complex branch; returns (H_new, Qn_new, c_r, res_mag_new, k_eff)."""
    m, n = H.shape
    if k > n:
        k = n
    if k == 0:
        return np.zeros((0, 0), dtype=np.complex128), [], np.zeros(1, dtype=np.complex128), [], 0
    Hn = H[:n, :n].copy()
    h_mn = H[n, n - 1]
    e = np.zeros(n, dtype=np.complex128)
    e[n - 1] = 1.0
    lu, piv, _ = lap.zgetrf(Hn.conj().T.copy())
    w, _ = lap.zgetrs(lu, piv, e)
    Hn[:, n - 1] += np.conj(h_mn) * h_mn * w
    t, sdim, ev, Z, _, info = lap.zgees(lambda a: False, Hn, compute_v=1, sort_t=0)
    perm = sorted(range(n), key=lambda i: abs(ev[i]))
    select = np.zeros(n, dtype=np.int32)
    for i in range(k):
        select[perm[i]] = 1
    ts, qs, w2, mk, s, sep, info = lap.ztrsen(select, t, Z, job="V", lwork=max(1, n * n))
    k = int(mk)
    Pk = qs[:, :k].copy()
    qr, tau, _, _ = lap.zgeqrf(Pk)
    Pk, _, _ = lap.zungqr(qr, tau)
    Pk1 = np.zeros((n + 1, k + 1), dtype=np.complex128)
    Pk1[:n, :k] = Pk
    Pk1[:, k] = res_vec
    for i in range(k):
        d = np.vdot(Pk1[:, i], Pk1[:, k])
        Pk1[:, k] -= d * Pk1[:, i]
    Pk1[:, k] /= np.sqrt(np.vdot(Pk1[:, k], Pk1[:, k]))
    c_r = Pk1.conj().T @ res_vec
    H_new = Pk1.conj().T @ (H @ Pk)
    Qmat = np.stack(Qn[:m], axis=1)
    Qn_new = [Qmat @ Pk1[:, i] for i in range(k + 1)]
    return H_new, Qn_new, c_r, [res_mag[-1]], k


def pgmres(A: BSR, b: np.ndarray, tol: float, pre=no_pre, max_iters: int = 500,
           restart: int = -1, k: int = -1, deflate=None) -> SolveResult:
    """Complex pGMRES with deflated restart.  The history is the residuals the
    reference prints: res_mag[0], then one per iteration (the norm pushed at a
    pure restart is not printed).  ``deflate`` replaces deflated_restart (same
    arguments and results), so a test can run another implementation of it."""
    deflate = deflate or deflated_restart
    b = np.asarray(b, dtype=np.complex128)
    hist = []
    r0 = pre(b)
    res_mag = [two_norm(r0)]
    hist.append(res_mag[0])
    Qn = [r0 / res_mag[0]]
    H = np.zeros((1, 0), dtype=np.complex128)
    x0 = np.zeros_like(b)
    zero_thresh = min(res_mag[0] * EPS, EPS)
    tolerance = res_mag[0] * tol
    it = tot = 0
    y = np.zeros(0, dtype=np.complex128)
    c_r = np.zeros(0, dtype=np.complex128)
    restarted = False
    n_restarts = 0
    while res_mag[-1] > tolerance:
        H = _one_arnoldi(it, H, Qn, A, pre, zero_thresh)
        m, n = it + 2, it + 1
        rhs = np.zeros(m, dtype=np.complex128)
        if not restarted:
            rhs[0] = res_mag[0]
        else:
            rhs[:len(c_r)] = c_r
        _, sol, info = lap.zgels(H.copy(), rhs.copy())
        y = sol[:n].copy()
        res_vec = rhs - H @ y
        res_mag.append(math.sqrt(float(np.sum(np.abs(np.conj(res_vec) * res_vec)))))
        hist.append(res_mag[-1])
        it += 1
        tot += 1
        if tot > max_iters:
            break
        if it == restart and res_mag[-1] > tolerance:
            x0 = x0 + sum(y[i] * Qn[i] for i in range(len(y)))
            r0 = pre(b - bsmv(A, x0))
            H, Qn, c_r, res_mag, _ = deflate(H, Qn, res_vec, res_mag, k)
            n_restarts += 1
            it = 0 if k == 0 else H.shape[1]
            if k == 0:
                H = np.zeros((1, 0), dtype=np.complex128)
                res_mag.append(two_norm(r0))
                c_r = np.array([res_mag[-1]], dtype=np.complex128)
                Qn = [r0 / res_mag[-1]]
            restarted = k != 0
    x = x0 + sum((y[i] * Qn[i] for i in range(len(y))), np.zeros_like(b))
    return SolveResult(x, hist, tot, n_restarts)
