"""CPU tests of the complex pGMRES's host dense algebra (complex_dense.h built
for the host by g++).

* complex Schur form of general and Arnoldi-like matrices: Z unitary,
  Z T Z^H = A, T upper triangular, eigenvalues equal to numpy's;
* Householder least squares against numpy's lstsq;
* Ritz and harmonic Ritz values of an Arnoldi H (printEigInfo) against numpy;
* the deflated restart: the oracle's complex pGMRES run with the C++
  deflate_complex in place of its LAPACK one reproduces the reference's
  residual histories (tests/golden/c_*_dr_*.npz) within 1e-10 and its
  iteration counts, i.e. the C++ reordered Schur vectors span the same
  harmonic Ritz space.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle.blocksp_oracle import BSR
import oracle.complex_oracle as CO
from parity import arg
from test_complex_oracle import load_complex_golden, oracle_pre, rel

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "complex_dense_harness.cpp"
HDR = ROOT / "blocksp_b200" / "csrc" / "complex_dense.h"
LIB = ROOT / "_build" / "complex_dense_harness.so"


@pytest.fixture(scope="module")
def cd():
    LIB.parent.mkdir(exist_ok=True)
    if not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime, HDR.stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", str(SRC), "-o", str(LIB)], check=True)
    lib = C.CDLL(str(LIB))
    P = C.POINTER(C.c_double)
    lib.cd_schur.argtypes = [P, C.c_int, P, P]
    lib.cd_lstsq.argtypes = [P, C.c_int, C.c_int, P, P]
    lib.cd_deflate.argtypes = [P, C.c_int, P, C.c_int, P, P, P, C.POINTER(C.c_int)]
    lib.cd_ritz.argtypes = [P, C.c_int, C.c_int, P]
    return lib


def ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("n,seed,hess", [(1, 0, 0), (2, 1, 0), (5, 2, 1), (11, 3, 0), (30, 4, 1), (31, 5, 0)])
def test_complex_schur(cd, n, seed, hess):
    rng = np.random.default_rng(seed)
    A = crand(rng, n, n)
    if hess:
        A = np.triu(A, -1) + 2 * np.eye(n)
    A = np.ascontiguousarray(A)
    T = np.zeros((n, n), complex)
    Z = np.zeros((n, n), complex)
    assert cd.cd_schur(ptr(A), n, ptr(T), ptr(Z)) == 1
    assert np.abs(Z @ Z.conj().T - np.eye(n)).max() < 1e-12
    assert np.abs(Z @ T @ Z.conj().T - A).max() < 1e-11 * max(1, np.abs(A).max())
    assert np.abs(np.tril(T, -1)).max() == 0.0
    ev = np.sort_complex(np.diag(T))
    assert np.abs(ev - np.sort_complex(np.linalg.eigvals(A))).max() < 1e-9 * max(1, np.abs(ev).max())


@pytest.mark.parametrize("m,n,seed", [(2, 1, 0), (6, 5, 1), (31, 30, 2), (12, 7, 3)])
def test_complex_lstsq(cd, m, n, seed):
    rng = np.random.default_rng(seed)
    H = np.ascontiguousarray(crand(rng, m, n))
    r = np.ascontiguousarray(crand(rng, m))
    y = np.zeros(n, complex)
    cd.cd_lstsq(ptr(H), m, n, ptr(r), ptr(y))
    assert rel(y, np.linalg.lstsq(H, r, rcond=None)[0]) <= 1e-12


def cpp_deflate(cd):
    def deflate(H, Qn, res_vec, res_mag, k):
        m, n = H.shape
        k = min(k, n)
        Hc = np.ascontiguousarray(H, dtype=complex)
        rv = np.ascontiguousarray(res_vec, dtype=complex)
        P = np.zeros((n + 1) * (k + 1), complex)
        Hn = np.zeros((k + 1) * k, complex)
        cr = np.zeros(k + 1, complex)
        ke = C.c_int()
        assert cd.cd_deflate(ptr(Hc), n, ptr(rv), k, ptr(P), ptr(Hn), ptr(cr), C.byref(ke)) == 0
        ke = ke.value
        P = P[:(n + 1) * (ke + 1)].reshape(n + 1, ke + 1)
        Hn = Hn[:(ke + 1) * ke].reshape(ke + 1, ke)
        Qmat = np.stack(Qn[:m], axis=1)
        return Hn, [Qmat @ P[:, i] for i in range(ke + 1)], cr[:ke + 1], [res_mag[-1]], ke
    return deflate


@pytest.mark.parametrize("name", ["c_ilu0_pgmres_dr_3d_bs4", "c_ilu0_pgmres_dr_3d_bs8", "c_sor_pgmres_dr_2d_bs2"])
def test_cpp_deflate_reproduces_reference(cd, name):
    s, meta, x, hist, iters = load_complex_golden(name)
    Ao = BSR(s.n, s.bs, s.row_ptr, s.col_idx, s.vals)
    res = CO.pgmres(Ao, s.b, arg(meta, "--tol", 1e-10), oracle_pre(meta, Ao), arg(meta, "--maxit", 500),
                    arg(meta, "--restart", -1), arg(meta, "--k", -1), deflate=cpp_deflate(cd))
    assert abs(res.iters - iters) <= 1
    h, g = np.asarray(res.hist) / res.hist[0], np.asarray(hist) / hist[0]
    n = min(len(h), len(g))
    assert np.abs(h[:n] - g[:n]).max() <= 1e-10
    assert rel(res.x, x) <= 1e-8


@pytest.mark.parametrize("n,harmonic", [(1, 0), (6, 0), (6, 1), (20, 1)])
def test_complex_ritz_values(cd, n, harmonic):
    rng = np.random.default_rng(40 + n)
    H = np.triu(crand(rng, n + 1, n), -1) + np.vstack([2 * np.eye(n), np.zeros((1, n))])
    H = np.ascontiguousarray(H)
    ev = np.zeros(n, complex)
    assert cd.cd_ritz(ptr(H), n, harmonic, ptr(ev)) == n
    Hs = H[:n, :n].copy()
    if harmonic:
        e = np.zeros(n, complex)
        e[-1] = 1.0
        Hs[:, -1] += abs(H[n, n - 1]) ** 2 * np.linalg.solve(Hs.conj().T, e)
    ref = np.sort_complex(np.linalg.eigvals(Hs))
    assert np.abs(np.sort_complex(ev) - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())
