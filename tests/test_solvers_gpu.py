"""Solver parity: GPU pCG / pGMRES(-DR) against the CPU oracle on the same seeded systems.

Parity criteria (FP64): iteration count equal to the oracle's within +-1
(pCG, unrestarted pGMRES) or +-2 (deflated restart); the solution agrees within
1e-8 relative (infinity norm); the reported FP64 true residual matches the
oracle's x.  Residual history, normalised by its first entry:
  * pGMRES: within 1e-10 absolute at every step both histories have;
  * pCG: within 1e-10 absolute plus 10x the oracle's own rounding envelope
    (its running maximum up to that step).  CG's recursive residual is chaotic
    at rounding level: the oracle rerun with its matrix product and
    preconditioner output perturbed by 1e-15 relative already moves the
    normalised history by up to ~1e-7 with IChol0 (~5e-2 without a
    preconditioner) while x agrees to 1e-14, so a fixed 1e-10 bound would
    reject the reference against itself.  The envelope is measured from three
    such perturbed oracle runs.
"""
import numpy as np
import pytest

from blocksp_b200.systems import grid_system
import oracle.blocksp_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def check_parity(x, info, hist, ref, it_slack, x_tol=1e-8, h_tol=1e-10, envelope=None):
    assert abs(info["iters"] - ref.iters) <= it_slack, (info["iters"], ref.iters)
    h = np.asarray(hist) / hist[0]
    r = np.asarray(ref.hist) / ref.hist[0]
    n = min(len(h), len(r))
    assert n >= 2
    allowed = np.full(n, h_tol)
    if envelope is not None:
        m = min(n, len(envelope))
        run = np.maximum.accumulate(envelope) if len(envelope) else envelope
        allowed[:m] += 10.0 * run[:m]
        allowed[m:] += 10.0 * (run.max() if len(run) else 0.0)
    dev = np.abs(h[:n] - r[:n])
    assert np.all(dev <= allowed), (int(np.argmax(dev - allowed)), float(dev.max()))
    assert rel(x, ref.x) <= x_tol


def cg_envelope(Ao, b, tol, pre, max_iters, ref, trials=3, eps=1e-15):
    """Per-step spread of the oracle's normalised pCG history under
    rounding-level perturbations of its preconditioner output."""
    r = np.asarray(ref.hist) / ref.hist[0]
    env = np.zeros(len(r))
    for t in range(trials):
        rng = np.random.default_rng(100 + t)

        def jitter(y):
            return y * (1.0 + eps * rng.standard_normal(y.shape))
        o = O.pcg(Ao, b, tol, lambda v: jitter(pre(v)), max_iters,
                  matvec=lambda v: jitter(O.bsmv(Ao, v)))
        h = np.asarray(o.hist) / o.hist[0]
        n = min(len(h), len(r))
        env[:n] = np.maximum(env[:n], np.abs(h[:n] - r[:n]))
        if n < len(r):
            env[n:] = np.maximum(env[n:], r[n:])
    return env


def setup_system(handle, dims, bs, skew, seed):
    import blocksp_b200 as bsp
    s = grid_system(dims, bs, seed=seed, skew=skew)
    return s, bsp.Matrix.from_system(s, handle), O.BSR.from_system(s)


@pytest.mark.parametrize("dims,bs", [((16, 16), 4), ((10, 10), 2), ((6, 6, 6), 8), ((7, 7), 3)])
def test_pcg_ichol0(handle, dims, bs):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, dims, bs, 0.0, 21)
    x, info, hist = bsp.pCG(A, s.b, 1e-10, bsp.IChol0(A), 2000, return_info=True)
    ic = O.IChol0(Ao)
    ref = O.pcg(Ao, s.b, 1e-10, ic, 2000)
    assert info["status"] == 0
    check_parity(x, info, hist, ref, 1, envelope=cg_envelope(Ao, s.b, 1e-10, ic, 2000, ref))
    assert abs(info["true_rel_res"] - O.true_rel_residual(Ao, s.b, x)) <= 1e-12


@pytest.mark.parametrize("pre", ["none", "diag", "ssor_chol"])
def test_pcg_other_preconditioners(handle, pre):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (12, 12), 4, 0.0, 22)
    if pre == "none":
        pc, pr = None, O.no_pre
    elif pre == "diag":
        pc, pr = bsp.Diag(A, "Chol"), O.Diag(Ao, O.CholeskyFactor)
    else:
        pc, pr = bsp.SOR(A, 1.6, 3, 0, "Chol"), O.SOR(Ao, 1.6, 3, 0, O.CholeskyFactor)
    x, info, hist = bsp.pCG(A, s.b, 1e-10, pc, 2000, return_info=True)
    ref = O.pcg(Ao, s.b, 1e-10, pr, 2000)
    check_parity(x, info, hist, ref, 1, envelope=cg_envelope(Ao, s.b, 1e-10, pr, 2000, ref))


@pytest.mark.parametrize("restart,k,slack", [(-1, -1, 1), (30, 10, 2), (10, 4, 2), (8, 0, 1)])
def test_pgmres_ilu0(handle, restart, k, slack):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (6, 6, 6), 8, 0.3, 23)
    x, info, hist = bsp.pGMRES(A, s.b, 1e-10, bsp.ILU0(A), 5000, restart, k, return_info=True)
    ref = O.pgmres(Ao, s.b, 1e-10, O.ILU0(Ao), 5000, restart, k)
    assert info["status"] == 0
    assert info["n_restarts"] == ref.restarts or restart > 0 and abs(info["n_restarts"] - ref.restarts) <= 1
    check_parity(x, info, hist, ref, slack)


@pytest.mark.parametrize("restart,k", [(-1, -1), (12, 5)])
def test_pgmres_sor(handle, restart, k):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (8, 8), 4, 0.3, 24)
    x, info, hist = bsp.pGMRES(A, s.b, 1e-10, bsp.SOR(A, 1.6, 3, 0), 5000, restart, k, return_info=True)
    ref = O.pgmres(Ao, s.b, 1e-10, O.SOR(Ao, 1.6, 3, 0), 5000, restart, k)
    check_parity(x, info, hist, ref, 2)


def test_pgmres_bs16_dr(handle):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (4, 4, 4), 16, 0.3, 25)
    x, info, hist = bsp.pGMRES(A, s.b, 1e-10, bsp.ILU0(A), 5000, 10, 4, return_info=True)
    ref = O.pgmres(Ao, s.b, 1e-10, O.ILU0(Ao), 5000, 10, 4)
    check_parity(x, info, hist, ref, 2)


def test_device_and_host_paths_agree(handle, torch_cuda):
    import blocksp_b200 as bsp
    torch = torch_cuda
    s, A, Ao = setup_system(handle, (10, 10), 4, 0.0, 26)
    pc = bsp.IChol0(A)
    xh = bsp.pCG(A, s.b, 1e-10, pc, 1000)
    xd = bsp.pCG(A, torch.tensor(s.b, device="cuda"), 1e-10, pc, 1000)
    assert np.array_equal(xh, xd.cpu().numpy())  # deterministic reductions


def test_solver_structs_and_ez(handle):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (6, 6, 5), 8, 0.0, 27)
    for x in (bsp.ILU0_pGMRES(A, 1e-10, 5000, 30, 10).solve(A, s.b),
              bsp.IChol0_pCG(A, 1e-10).solve(A, s.b),
              bsp.SOR_pGMRES(A).solve(A, s.b), bsp.SOR_pCG(A).solve(A, s.b),
              bsp.ez.ilu0_pGMRES_dr(A, s.b), bsp.ez.sor_pGMRES_robust(A, s.b), bsp.ez.ichol0_pCG(A, s.b)):
        assert O.true_rel_residual(Ao, s.b, x) < 1e-7


def test_maxit_status_and_count(handle):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (16, 16), 4, 0.0, 28)
    x, info, hist = bsp.pCG(A, s.b, 1e-14, None, 5, return_info=True)
    ref = O.pcg(Ao, s.b, 1e-14, O.no_pre, 5)
    assert info["status"] == 4 and info["iters"] == ref.iters == 6
    x, info, hist = bsp.pGMRES(A, s.b, 1e-14, None, 7, return_info=True)
    ref = O.pgmres(Ao, s.b, 1e-14, O.no_pre, 7)
    assert info["status"] == 4 and info["iters"] == ref.iters


def test_nan_rhs_is_reported(handle):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (6, 6), 4, 0.0, 29)
    b = s.b.copy()
    b[5] = np.nan
    x, info, hist = bsp.pCG(A, b, 1e-10, bsp.IChol0(A), 100, return_info=True)
    assert info["status"] == 5  # BSP_NAN
    x, info, hist = bsp.pGMRES(A, b, 1e-10, bsp.ILU0(A), 100, return_info=True)
    assert info["status"] == 5


def test_zero_rhs_returns_zero(handle):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (6, 6), 4, 0.0, 30)
    x = bsp.pCG(A, np.zeros_like(s.b), 1e-10, bsp.IChol0(A), 100)
    assert not np.any(x)
    x = bsp.pGMRES(A, np.zeros_like(s.b), 1e-10, bsp.ILU0(A), 100)
    assert not np.any(x)


@pytest.mark.parametrize("precision", [0, 1, 2])  # PREC_F64, PREC_F32, PREC_BF16 factors
def test_true_residual_refinement_pgmres(handle, precision):
    """FP64 iterative refinement reaches the FP64 true residual 1e-10 with any
    inner operator precision; the solution error against the oracle's tight
    FP64 solve is stated and bounded by the conditioning (<= 1e-6 here)."""
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (6, 6, 6), 8, 0.3, 31)
    x, info, hist = bsp.pGMRES(A, s.b, 1e-10, bsp.ILU0(A), 5000, 30, 10, return_info=True,
                               stop_rule=1, precision=precision)
    assert info["status"] == 0
    assert info["true_rel_res"] <= 1e-10
    assert O.true_rel_residual(Ao, s.b, x) <= 1.5e-10
    ref = O.pgmres(Ao, s.b, 1e-13, O.ILU0(Ao), 5000, 30, 10)
    assert rel(x, ref.x) <= 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_true_residual_refinement_pcg(handle, precision):
    import blocksp_b200 as bsp
    s, A, Ao = setup_system(handle, (16, 16), 4, 0.0, 32)
    x, info, hist = bsp.pCG(A, s.b, 1e-10, bsp.IChol0(A), 2000, return_info=True, stop_rule=1,
                            precision=precision)
    assert info["status"] == 0 and info["true_rel_res"] <= 1e-10
    assert O.true_rel_residual(Ao, s.b, x) <= 1.5e-10


def test_refinement_applies_the_correction_after_a_breakdown(handle):
    """An inner pGMRES that breaks down (here the Krylov space of M^-1 A b is
    one-dimensional: A = 2I in 8x8 blocks, ILU0 exact) still holds the
    minimiser; the FP64 refinement applies it, recomputes the true residual
    and reports convergence instead of returning the previous iterate."""
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, systems
    n, bs = 10, 8
    s = systems.BSRSystem(n=n, bs=bs, row_ptr=np.arange(n + 1, dtype=np.int32), col_idx=np.arange(n, dtype=np.int32),
                          vals=np.repeat(2.0 * np.eye(bs)[None], n, 0), b=np.random.default_rng(3).random(n * bs))
    A = bsp.Matrix.from_system(s, handle)
    x, info, _ = bsp.pGMRES(A, s.b, 1e-10, bsp.ILU0(A), 100, 30, 10, return_info=True,
                           stop_rule=_lib.STOP_TRUE_RESIDUAL)
    assert info["status"] == 0 and info["true_rel_res"] <= 1e-14
    assert np.abs(x - s.b / 2).max() <= 1e-15
