"""Block algebra on the GPU against the reference (bs_id, bs_tr, bsmm, A + B).

Same fixtures and criteria as tests/test_algebra.py (the reference build's
own results): identical block structure, values within 1e-13 relative.  The
block_pseudo_heat operator I - delta A^T A (32x32 blocks) is then solved with
IChol0-pCG and ILU0-pGMRES(30, 10) as the reference's test engine does, and
compared with the reference's own solves of it: iteration counts +-1 (+-2
with deflated restart), solutions within 1e-8.
"""
import numpy as np
import pytest

from parity import check_history, rel
from test_algebra import CASES, check_pseudo_heat, check_same, load_case, pseudo_heat_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_gpu_block_algebra_vs_reference(handle, name):
    import blocksp_b200 as bsp
    d, meta, A = load_case(name)
    M = bsp.Matrix.from_system(A, handle)
    C = bsp.bs_tr(M) if meta["mode"] == "bs_tr" else bsp.bsmm(M, M, Atran=meta["args"][1] == "1")
    check_same(*C.export(), d)


def test_gpu_identity_and_sum(handle):
    import blocksp_b200 as bsp
    import oracle.blocksp_oracle as O
    from blocksp_b200 import systems
    A = systems.random_blocksp(10, 4, 3, 7)
    M = bsp.Matrix.from_system(A, handle)
    rp, ci, va = bsp.bs_id(10, 4, handle).export()
    assert np.array_equal(ci, np.arange(10)) and np.array_equal(va, np.repeat(np.eye(4)[None], 10, 0))
    ref = O.matrix_add(2.0, O.BSR.from_system(A), -0.5, O.bs_tr(O.BSR.from_system(A)))
    got = bsp.matrix_add(2.0, M, -0.5, bsp.bs_tr(M)).export()
    assert np.array_equal(got[0], ref.row_ptr) and np.array_equal(got[1], ref.col_idx)
    assert np.abs(got[2] - ref.vals).max() <= 1e-15 * np.abs(ref.vals).max()
    # triple product nests to the right: A (A A)
    rp3, ci3, va3 = bsp.bsmm(M, M, M).export()
    Ao = O.BSR.from_system(A)
    R3 = O.bsmm(Ao, O.bsmm(Ao, Ao))
    assert np.array_equal(ci3, R3.col_idx) and np.abs(va3 - R3.vals).max() <= 1e-13 * np.abs(R3.vals).max()


def test_gpu_pseudo_heat_operator_and_solves(handle):
    import blocksp_b200 as bsp
    d, ph, A, _ = pseudo_heat_oracle()
    M = bsp.Matrix.from_system(A, handle)
    # ASym = bs_id(l) - delta * bsmm(A, A, true)   (blocksp_tests.hpp:284)
    S = bsp.matrix_add(1.0, bsp.bs_id(ph["m"], ph["bs"], handle), -ph["delta"], bsp.bsmm(M, M, Atran=True))
    rp, ci, va = S.export()
    check_pseudo_heat(rp, ci, va, d)
    b = A.b
    x, info, hist = bsp.pCG(S, b, 1e-10, bsp.IChol0(S), 2000, return_info=True)
    assert abs(info["iters"] - int(d["pcg_iters"])) <= 1
    assert rel(x, d["pcg_x"]) <= 1e-8
    x, info, hist = bsp.pGMRES(S, b, 1e-10, bsp.ILU0(S), 5000, 30, 10, return_info=True)
    assert abs(info["iters"] - int(d["gmres_iters"])) <= 2
    check_history(hist, list(d["gmres_hist"]))
    assert rel(x, d["gmres_x"]) <= 1e-8


# ---- arnoldi_eigenvalues on the GPU (blocksp_solvers.hpp:306-334) ----
from test_algebra import EIG_CASES, load_eig, match_eigs  # noqa: E402


@pytest.mark.parametrize("name", EIG_CASES)
def test_gpu_arnoldi_eigenvalues_vs_reference(handle, name):
    import blocksp_b200 as bsp
    ref, meta, s = load_eig(name)
    A = bsp.Matrix.from_system(s, handle)
    e = bsp.arnoldi_eigenvalues(A, meta["iters"], harmonic_Ritz=bool(meta["harmonic"]))
    match_eigs(e.real() + 1j * e.imag(), ref, 1e-9)
    assert abs(e.cond_number() - np.abs(ref).max() / np.abs(ref).min()) <= 1e-6 * e.cond_number()


def test_gpu_arnoldi_eigenvalues_preconditioned_vs_oracle(handle):
    """With block ILU0 (the reference build's preconditioned form ends in a
    segmentation fault, so the oracle is the check): harmonic Ritz values of
    M^-1 A after 20 steps."""
    import blocksp_b200 as bsp
    import oracle.blocksp_oracle as O
    from blocksp_b200 import systems
    s = systems.grid_system((5, 5, 5), 8, seed=72, skew=0.3)
    A = bsp.Matrix.from_system(s, handle)
    e = bsp.arnoldi_eigenvalues(A, 20, bsp.ILU0(A), harmonic_Ritz=True)
    Ao = O.BSR.from_system(s)
    ref = O.arnoldi_eigenvalues(Ao, 20, O.ILU0(Ao), harmonic=True)
    match_eigs(e.real() + 1j * e.imag(), ref, 1e-8)


def test_gpu_pgmres_print_eig_info(handle, capfd):
    """pGMRES(printEigInfo) prints the harmonic Ritz summary after a restart."""
    import blocksp_b200 as bsp
    from blocksp_b200 import systems
    s = systems.grid_system((6, 6, 6), 8, seed=13, skew=0.3)
    A = bsp.Matrix.from_system(s, handle)
    bsp.pGMRES(A, s.b, 1e-10, bsp.ILU0(A), 5000, 10, 4, printIters=True, printEigInfo=True)
    out = capfd.readouterr().out
    assert "pGMRES iters" in out and "Harmonic Ritz info" in out and "ratio/cond" in out
