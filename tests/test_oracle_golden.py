"""Pinning the CPU oracle: the numpy restatement against the reference itself.

The golden fixtures in tests/golden/ were produced by the reference BlockSp
v1.0 headers compiled unmodified by oracle/Makefile (tests/golden/make_golden.py).
The restatement must reproduce them within the parity criteria of
tests/parity.py, and must reproduce the reference's own known answer on its LDG
fixture (infinity-norm error ~2.9e-4 against the exact solution).
"""
import numpy as np
import pytest

import oracle.blocksp_oracle as O
from parity import arg, cg_envelope, check_history, ldg_system, load_golden, rel

APPLY = ["ilu0_apply_3d_bs8", "ichol0_apply_2d_bs4", "sor_apply_2d_bs4", "diag_apply_3d_bs8"]
PCG = ["ichol0_pcg_2d_bs4", "sor_pcg_2d_bs4", "diag_pcg_2d_bs4"]
GMRES = ["ilu0_pgmres_3d_bs8", "ilu0_pgmres_dr_3d_bs8", "ilu0_pgmres_dr10_3d_bs8", "sor_pgmres_dr_2d_bs4",
         "ilu0_pgmres_3d_bs16"]


def oracle_pre(meta, Ao):
    sv = meta["solver"]
    if sv.startswith("ilu0"):
        return O.ILU0(Ao)
    if sv.startswith("ichol0"):
        return O.IChol0(Ao)
    if sv == "sor_apply":
        return O.SOR(Ao, arg(meta, "--w", 1.6), arg(meta, "--nu", 3), arg(meta, "--sortype", 0))
    if sv == "sor_pgmres":
        return O.SOR(Ao, arg(meta, "--w", 1.6), arg(meta, "--nu", 3), arg(meta, "--sortype", 0))
    if sv == "sor_pcg":
        return O.SOR(Ao, 1.6, 3, 0, O.CholeskyFactor)
    if sv == "diag_pcg":
        return O.Diag(Ao, O.CholeskyFactor)
    if sv == "diag_apply":
        return O.Diag(Ao, O.LUFactor)
    raise KeyError(sv)


@pytest.mark.parametrize("name", ["bsmv_2d_bs4", "bsmv_3d_bs8", "bsmv_3d_bs16", "bsmv_multi_bs4_d2"])
def test_bsmv_matches_reference(name):
    s, meta, x, _, _ = load_golden(name)
    nrhs = meta["D"] if meta["solver"] == "bsmv_multi" else 1
    y = O.bsmv(O.BSR.from_system(s), s.b, nrhs=nrhs)
    assert rel(y, x) <= 1e-14


@pytest.mark.parametrize("name", APPLY)
def test_preconditioner_apply_matches_reference(name):
    s, meta, x, _, _ = load_golden(name)
    Ao = O.BSR.from_system(s)
    assert rel(oracle_pre(meta, Ao)(s.b.copy()), x) <= 1e-11


@pytest.mark.parametrize("name", PCG)
def test_pcg_matches_reference(name):
    s, meta, x, hist, iters = load_golden(name)
    Ao = O.BSR.from_system(s)
    pre = oracle_pre(meta, Ao)
    tol, maxit = arg(meta, "--tol", 1e-10), arg(meta, "--maxit", 5000)
    r = O.pcg(Ao, s.b, tol, pre, maxit)
    assert abs(r.iters - iters) <= 1
    check_history(r.hist, hist, envelope=cg_envelope(Ao, s.b, tol, pre, maxit, hist))
    assert rel(r.x, x) <= 1e-8


@pytest.mark.parametrize("name", GMRES)
def test_pgmres_matches_reference(name):
    s, meta, x, hist, iters = load_golden(name)
    Ao = O.BSR.from_system(s)
    restart, k = arg(meta, "--restart", -1), arg(meta, "--k", -1)
    r = O.pgmres(Ao, s.b, arg(meta, "--tol", 1e-10), oracle_pre(meta, Ao), 5000, restart, k)
    assert abs(r.iters - iters) <= (2 if restart > 0 else 1)
    check_history(r.hist, hist)
    assert rel(r.x, x) <= 1e-8


def test_ldg_known_answer_reference_and_oracle():
    """The reference's only quantitative golden (blocksp_tests.hpp:304-318):
    infinity-norm error near 0.00029 against the exact solution at tol 1e-8."""
    s, sol, ref_err = ldg_system(4)
    for k, v in ref_err.items():
        assert 2.8e-4 < v < 3.0e-4, (k, v)
    Ao = O.BSR.from_system(s)
    r = O.pcg(Ao, s.b, 1e-8, O.IChol0(Ao), 5000)
    err = np.abs(r.x - sol).max()
    assert abs(err - ref_err["B4_ichol0_pcg"]) <= 1e-7
