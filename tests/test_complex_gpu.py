"""The complex solve path (T = std::complex<double>) on the GPU.

Against the reference itself (tests/golden/c_*.npz, the reference built with
T = std::complex<double>): bsmv within 1e-14 relative; one Diag / SOR / ILU0
application within 1e-11; pGMRES with its iteration count +-1 (+-2 with
deflated restart), normalised residual history within 1e-10 absolute and the
solution within 1e-8 relative.  Against the complex oracle on a larger
system (12^3, 4x4 complex blocks, ILU0 pGMRES(20, k=6)), with the same
criteria.  IChol0, pCG and the learned preconditioner are refused for complex
matrices (real only in the reference).
"""
import numpy as np
import pytest

from blocksp_b200 import _lib, systems
from oracle.blocksp_oracle import BSR
import oracle.complex_oracle as CO
from parity import arg, check_history
from test_complex_oracle import APPLY, GMRES, load_complex_golden, rel

pytestmark = pytest.mark.gpu


def gpu_pre(bsp, meta, A):
    sv = meta["solver"]
    w, nu, ty = arg(meta, "--w", 1.6), arg(meta, "--nu", 3), arg(meta, "--sortype", 0)
    if sv.startswith("ilu0"):
        return bsp.ILU0(A)
    if sv.startswith("sor"):
        return bsp.SOR(A, w, nu, ty)
    if sv.startswith("diag"):
        return bsp.Diag(A, "LU")
    return None


@pytest.mark.parametrize("name", APPLY)
def test_complex_apply_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, _, _ = load_complex_golden(name)
    A = bsp.Matrix.from_system(s, handle)
    assert A.complex_bs == s.bs and A.bs == 2 * s.bs
    if meta["solver"] == "bsmv":
        out = bsp.bsmv(A, s.b)
        assert out.dtype == np.complex128
        assert rel(out, x) <= 1e-14
    else:
        pc = gpu_pre(bsp, meta, A)
        out = pc.apply_host(s.b)
        assert rel(out, x) <= 1e-11
        pc.close()
    A.close()


@pytest.mark.parametrize("name", GMRES)
def test_complex_pgmres_vs_reference(handle, name):
    import blocksp_b200 as bsp
    s, meta, x, hist, iters = load_complex_golden(name)
    A = bsp.Matrix.from_system(s, handle)
    pc = gpu_pre(bsp, meta, A)
    restart, k = arg(meta, "--restart", -1), arg(meta, "--k", -1)
    xg, info, hg = bsp.pGMRES(A, s.b, arg(meta, "--tol", 1e-10), pc, arg(meta, "--maxit", 500), restart, k,
                              return_info=True)
    assert xg.dtype == np.complex128
    assert abs(info["iters"] - iters) <= (2 if restart > 0 else 1)
    check_history(hg, hist)
    assert rel(xg, x) <= 1e-8
    for o in (pc, A):
        if o is not None:
            o.close()


def test_complex_pgmres_vs_oracle_larger(handle):
    import blocksp_b200 as bsp
    s = systems.complex_system((12, 12, 12), 4, 211)
    Ao = BSR(s.n, s.bs, s.row_ptr, s.col_idx, s.vals)
    ref = CO.pgmres(Ao, s.b, 1e-10, CO.ILU0(Ao), 500, 20, 6)
    A = bsp.Matrix.from_system(s, handle)
    pc = bsp.ILU0(A)
    xg, info, hg = bsp.pGMRES(A, s.b, 1e-10, pc, 500, 20, 6, return_info=True)
    assert abs(info["iters"] - ref.iters) <= 2
    check_history(hg, ref.hist)
    assert rel(xg, ref.x) <= 1e-8
    # the true complex residual of the solution
    r = s.b - CO.bsmv(Ao, xg)
    assert np.linalg.norm(r) / np.linalg.norm(s.b) <= 1e-7
    assert abs(info["true_rel_res"] - np.linalg.norm(r) / np.linalg.norm(s.b)) <= 1e-9
    pc.close()
    A.close()


def test_complex_refuses_real_only_methods(handle):
    import blocksp_b200 as bsp
    s = systems.complex_system((4, 4), 2, 7)
    A = bsp.Matrix.from_system(s, handle)
    with pytest.raises(_lib.BspError) as e:
        bsp.IChol0(A)
    assert e.value.status == 8
    with pytest.raises(_lib.BspError) as e:
        bsp.pCG(A, s.b, 1e-10, None, 100)
    assert e.value.status == 8
    A.close()
