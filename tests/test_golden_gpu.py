"""GPU against the reference itself: the golden fixtures made by the reference
BlockSp v1.0 build (tests/golden/make_golden.py), and its LDG known answer.

Criteria as in tests/parity.py: bsmv <= 1e-14; preconditioner application
<= 1e-11; iteration counts +-1 (+-2 with deflated restart); pGMRES normalised
history <= 1e-10 absolute; pCG history within the reference method's rounding
envelope; solutions <= 1e-8; LDG infinity-norm error within 1e-7 of the
reference's value for every solver and block size.
"""
import numpy as np
import pytest

import oracle.blocksp_oracle as O
from parity import arg, cg_envelope, check_history, ldg_system, load_golden, rel
from test_oracle_golden import APPLY, GMRES, PCG, oracle_pre

pytestmark = pytest.mark.gpu


def gpu_pre(bsp, meta, A):
    sv = meta["solver"]
    if sv.startswith("ilu0"):
        return bsp.ILU0(A)
    if sv.startswith("ichol0"):
        return bsp.IChol0(A)
    if sv in ("sor_apply", "sor_pgmres"):
        return bsp.SOR(A, arg(meta, "--w", 1.6), arg(meta, "--nu", 3), arg(meta, "--sortype", 0))
    if sv == "sor_pcg":
        return bsp.SOR(A, 1.6, 3, 0, "Chol")
    if sv == "diag_pcg":
        return bsp.Diag(A, "Chol")
    if sv == "diag_apply":
        return bsp.Diag(A, "LU")
    raise KeyError(sv)


@pytest.mark.parametrize("name", ["bsmv_2d_bs4", "bsmv_3d_bs8", "bsmv_3d_bs16", "bsmv_multi_bs4_d2"])
def test_bsmv_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, _, _ = load_golden(name)
    nrhs = meta["D"] if meta["solver"] == "bsmv_multi" else 1
    A = bsp.Matrix.from_system(s, handle)
    assert rel(bsp.bsmv(A, s.b, nrhs=nrhs), x) <= 1e-14


@pytest.mark.parametrize("name", APPLY)
def test_apply_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, _, _ = load_golden(name)
    A = bsp.Matrix.from_system(s, handle)
    assert rel(gpu_pre(bsp, meta, A).apply_host(s.b), x) <= 1e-11


@pytest.mark.parametrize("name", PCG)
def test_pcg_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, hist, iters = load_golden(name)
    A = bsp.Matrix.from_system(s, handle)
    tol, maxit = arg(meta, "--tol", 1e-10), arg(meta, "--maxit", 5000)
    xg, info, hg = bsp.pCG(A, s.b, tol, gpu_pre(bsp, meta, A), maxit, return_info=True)
    assert abs(info["iters"] - iters) <= 1
    Ao = O.BSR.from_system(s)
    check_history(hg, hist, envelope=cg_envelope(Ao, s.b, tol, oracle_pre(meta, Ao), maxit, hist))
    assert rel(xg, x) <= 1e-8


@pytest.mark.parametrize("name", GMRES)
def test_pgmres_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, hist, iters = load_golden(name)
    A = bsp.Matrix.from_system(s, handle)
    restart, k = arg(meta, "--restart", -1), arg(meta, "--k", -1)
    xg, info, hg = bsp.pGMRES(A, s.b, arg(meta, "--tol", 1e-10), gpu_pre(bsp, meta, A), 5000, restart, k,
                              return_info=True)
    assert abs(info["iters"] - iters) <= (2 if restart > 0 else 1)
    check_history(hg, hist)
    assert rel(xg, x) <= 1e-8


@pytest.mark.parametrize("B", [1, 2, 4])
def test_ldg_known_answer_on_gpu(handle, B):
    """blocksp_tests.hpp:304-342 on the GPU: the infinity-norm error against the
    exact solution matches the reference's (~2.946e-4) for each solver."""
    import blocksp_b200 as bsp
    s, sol, ref_err = ldg_system(B)
    A = bsp.Matrix.from_system(s, handle)
    runs = {
        "ichol0_pcg": lambda: bsp.IChol0_pCG(A, 1e-8, 5000).solve(A, s.b),
        "ilu0_pgmres": lambda: bsp.ILU0_pGMRES(A, 1e-8, 5000, -1, -1).solve(A, s.b),
        "ilu0_pgmres_dr": lambda: bsp.ILU0_pGMRES(A, 1e-8, 5000, 30, 10).solve(A, s.b),
        "sor_pcg": lambda: bsp.SOR_pCG(A, 1.6, 3, 1e-8, 5000).solve(A, s.b),
    }
    for name, run in runs.items():
        err = float(np.abs(run() - sol).max())
        assert abs(err - ref_err[f"B{B}_{name}"]) <= 1e-7, (name, err, ref_err[f"B{B}_{name}"])


@pytest.mark.parametrize("B, D", [(4, 2), (2, 2), (1, 2)])
def test_ldg_known_answer_d2_from_mtx(handle, tmp_path, B, D):
    """The LDG known answer at D = 2 through the library's .mtx readers (the
    reference's vector reader misplaces values for D > 1, blocksp_tests.hpp:679).
    Read as BlockSp<T, B*D> and solArray<T, B, D>, the system is the one the
    reference solves with block size B*D and D = 1, so the infinity-norm error
    must match the reference's run at that block size."""
    import blocksp_b200 as bsp
    from blocksp_b200.mtx import mtxArray_to_solArray, mtxMatrix_to_BlockSp
    from test_mtx import write_ldg
    write_ldg(tmp_path)
    s = mtxMatrix_to_BlockSp(tmp_path / "A.mtx", B * D, start_line=1, symmetric=True)
    b = mtxArray_to_solArray(tmp_path / "b.mtx", B, D, start_line=1)
    sol = mtxArray_to_solArray(tmp_path / "sol.mtx", B, D, start_line=1)
    s.b = b
    _, _, ref_err = ldg_system(B * D)
    A = bsp.Matrix.from_system(s, handle)
    for name, run in {"ichol0_pcg": lambda: bsp.IChol0_pCG(A, 1e-8, 5000).solve(A, b),
                      "ilu0_pgmres_dr": lambda: bsp.ILU0_pGMRES(A, 1e-8, 5000, 30, 10).solve(A, b)}.items():
        err = float(np.abs(run() - sol).max())
        assert abs(err - ref_err[f"B{B * D}_{name}"]) <= 1e-7, (name, err, ref_err[f"B{B * D}_{name}"])
