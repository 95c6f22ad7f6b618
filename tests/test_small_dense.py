"""CPU tests of the GPU solver's small dense routines (small_dense.h built for the host).

Checks the real Schur form, the invariant subspace used by the deflated
restart, the Givens least squares and the transposed LU solve against
scipy's LAPACK (gees/trsen, lstsq, solve) on random and Arnoldi-like matrices.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.linalg.lapack as lap

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "small_dense_harness.cpp"
LIB = ROOT / "_build" / "small_dense_harness.so"


@pytest.fixture(scope="module")
def sd():
    LIB.parent.mkdir(exist_ok=True)
    hdr = ROOT / "blocksp_b200" / "csrc" / "small_dense.h"
    if not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime, hdr.stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", str(SRC), "-o", str(LIB)], check=True)
    lib = C.CDLL(str(LIB))
    P = C.POINTER(C.c_double)
    lib.sd_schur.argtypes = [P, C.c_int, P, P, P, P]
    lib.sd_invariant.argtypes = [P, C.c_int, C.c_int, C.c_double, P, C.POINTER(C.c_int)]
    lib.sd_lstsq.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P]
    lib.sd_lstsq.restype = C.c_double
    lib.sd_solve_transposed.argtypes = [P, C.c_int, P]
    return lib


def ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def arnoldi_like(n, seed):
    """An upper-Hessenberg matrix plus a harmonic rank-one update, like H_tilde."""
    rng = np.random.default_rng(seed)
    H = np.triu(rng.standard_normal((n, n)), -1) + 2 * np.eye(n)
    return H


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (5, 2), (10, 3), (30, 4), (31, 5), (60, 6)])
def test_schur_matches_lapack(sd, n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) if seed % 2 else arnoldi_like(n, seed)
    A = np.ascontiguousarray(A)
    T = np.zeros((n, n)); Z = np.zeros((n, n)); wr = np.zeros(n); wi = np.zeros(n)
    assert sd.sd_schur(ptr(A), n, ptr(T), ptr(Z), ptr(wr), ptr(wi)) == 1
    assert np.abs(Z @ Z.T - np.eye(n)).max() < 1e-12
    assert np.abs(Z @ T @ Z.T - A).max() < 1e-11 * max(1, np.abs(A).max())
    assert np.abs(np.tril(T, -2)).max() == 0.0
    ev = np.sort_complex(wr + 1j * wi)
    ref = np.sort_complex(np.linalg.eigvals(A))
    assert np.abs(ev - ref).max() < 1e-9 * max(1, np.abs(ref).max())


def subspace_gap(P, Q):
    """Largest principal-angle sine between span(P) and span(Q)."""
    s = np.linalg.svd(P.T @ Q, compute_uv=False)
    return float(np.sqrt(max(0.0, 1 - s.min() ** 2)))


@pytest.mark.parametrize("n,k,seed", [(30, 10, 11), (30, 10, 12), (20, 5, 13), (31, 10, 14), (12, 11, 15)])
def test_invariant_subspace_matches_trsen(sd, n, k, seed):
    rng = np.random.default_rng(seed)
    A = np.ascontiguousarray(rng.standard_normal((n, n)) + 0.5 * np.diag(rng.standard_normal(n)))
    zt = 10 * n * n * np.finfo(float).eps
    P = np.zeros((n, n)); keff = C.c_int()
    assert sd.sd_invariant(ptr(A), n, k, zt, ptr(P), C.byref(keff)) == 1
    keff = keff.value
    Pk = P[:, :keff]
    # reference selection + reordering through LAPACK (deflated_restart.hpp:125-193)
    t, sdim, wr, wi, Z, _, info = lap.dgees(lambda a, b: False, A, compute_v=1, sort_t=0)
    mags = np.sqrt(wr * wr + wi * wi)
    perm = sorted(range(n), key=lambda i: mags[i])
    sel = np.zeros(n, dtype=np.int32); cnt = 0
    for i in range(n):
        if cnt >= k:
            break
        ip = perm[i]
        if sel[ip]:
            continue
        sel[ip] = 1; cnt += 1
        if abs(wi[ip]) > zt:
            for j in range(n):
                if j != ip and abs(wr[j] - wr[ip]) < zt and abs(wi[j] + wi[ip]) < zt:
                    if not sel[j]:
                        sel[j] = 1; cnt += 1
                    break
    ts, qs, _, _, m, *_ = lap.dtrsen(sel, t, Z, job="V", lwork=n * n, liwork=n * n)
    assert keff == m
    assert np.abs(Pk.T @ Pk - np.eye(keff)).max() < 1e-12
    # invariant to working accuracy and carrying exactly the selected spectrum
    assert np.linalg.norm(A @ Pk - Pk @ (Pk.T @ A @ Pk)) < 1e-12 * np.linalg.norm(A)
    got = np.sort_complex(np.linalg.eigvals(Pk.T @ A @ Pk))
    want = np.sort_complex((wr + 1j * wi)[sel.astype(bool)])
    assert np.abs(got - want).max() < 1e-9 * np.abs(want).max()
    # the same subspace as trsen's, up to its conditioning (close |theta| at
    # the selection boundary make the subspace itself sensitive at ~1e-8)
    assert subspace_gap(Pk, qs[:, :m]) < 1e-6


@pytest.mark.parametrize("m,ncols,dense", [(30, 30, 0), (30, 17, 0), (30, 25, 10), (8, 1, 0)])
def test_givens_lstsq(sd, m, ncols, dense):
    rng = np.random.default_rng(m + ncols)
    H = np.zeros((m + 1, m))
    for j in range(m):
        last = dense if j < dense else j + 1
        H[: last + 1, j] = rng.standard_normal(last + 1)
    rhs = np.zeros(m + 1)
    rhs[: (dense + 1 if dense else 1)] = rng.standard_normal(dense + 1 if dense else 1)
    y = np.zeros(m)
    res = sd.sd_lstsq(ptr(H), m, ncols, dense, ptr(rhs), ptr(y))
    Hs = H[: ncols + 1, :ncols]
    yref, *_ = np.linalg.lstsq(Hs, rhs[: ncols + 1], rcond=None)
    assert np.abs(y[:ncols] - yref).max() < 1e-10 * max(1, np.abs(yref).max())
    assert abs(res - np.linalg.norm(rhs[: ncols + 1] - Hs @ yref)) < 1e-12


def test_solve_transposed(sd):
    rng = np.random.default_rng(3)
    A = np.ascontiguousarray(rng.standard_normal((9, 9)))
    w = np.zeros(9); w[-1] = 1.0
    sd.sd_solve_transposed(ptr(A), 9, ptr(w))
    assert np.abs(A.T @ w - np.eye(9)[-1]).max() < 1e-12
