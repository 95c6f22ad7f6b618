"""Learned preconditioner on the GPU against the oracle (oracle/learned_oracle.py).

* forward correction dF: FP64 kernels within 1e-12 relative of the oracle,
  FP32 kernels within 1e-4;
* loss (1/K) sum ||M^-1 A q - q||^2 and every parameter gradient: FP64 within
  1e-9 relative (per parameter tensor, max-norm), FP32 network within 2e-3
  (the triangular solves of the loss are FP64 in both);
* probes: orthonormal Arnoldi vectors of the ILU0-preconditioned operator,
  equal to the oracle's Arnoldi process within 1e-9;
* zero decoders reproduce block ILU0 bit for bit; with a relaxation they give
  ILU0's factors with the off-diagonal blocks scaled by 1 + relax;
* training steps lower the loss and the trained factors still solve;
* LearnedLU falls back to ILU0 when a model has not beaten it.
"""
import numpy as np
import pytest

from blocksp_b200 import _lib, learned, systems
import oracle.blocksp_oracle as O
import oracle.learned_oracle as LO

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def case(handle):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((5, 4, 3), 8, 31)
    A = bsp.Matrix.from_system(s, handle)
    Ao = O.BSR.from_system(s)
    ilu_o = O.ILU0(Ao)
    g = LO.graph_of(s.row_ptr, s.col_idx)
    rng = np.random.default_rng(5)
    p = LO.init_params(8, seed=9)
    for k in p:  # small decoders keep M = LU well conditioned
        p[k] = p[k] + (0.005 if k in ("Wo", "bo", "Wd", "bd") else 0.05) * rng.standard_normal(p[k].shape)
    yield s, A, Ao, ilu_o, g, p
    A.close()


@pytest.mark.parametrize("dtype,tol", [(_lib.BSP_F64, 1e-12), (_lib.BSP_F32, 1e-4)])
def test_forward_matches_oracle(handle, case, dtype, tol):
    s, A, _, _, g, p = case
    m = learned.LearnedModel(handle, 8, dtype, params=p)
    dF = m.forward(A).cpu().numpy()
    ref, _ = LO.forward(p, g, s.vals)
    assert rel(dF, ref) <= tol
    m.close()


@pytest.mark.parametrize("relax", [0.0, 0.4])
@pytest.mark.parametrize("dtype,ltol,gtol", [(_lib.BSP_F64, 1e-10, 1e-9), (_lib.BSP_F32, 1e-4, 2e-3)])
def test_loss_and_gradients_match_oracle(handle, case, torch_cuda, dtype, ltol, gtol, relax):
    torch = torch_cuda
    s, A, _, ilu_o, g, p = case
    import blocksp_b200 as bsp
    ilu = bsp.ILU0(A)
    F0 = learned.ilu_factors(A, ilu)
    assert rel(F0.cpu().numpy(), ilu_o.LU.vals) <= 1e-13
    rng = np.random.default_rng(6)
    Qh = np.linalg.qr(rng.standard_normal((s.n * 8, 3)))[0].T.copy()
    Q = torch.tensor(Qh, device="cuda")
    m = learned.LearnedModel(handle, 8, dtype, params=p, meta={"relax": relax})
    assert m.relax == relax
    loss = m.loss_grad(A, ilu, Q)
    ref_loss, ref_g = LO.loss_and_grads(p, g, s.vals, F0.cpu().numpy(), Qh, relax=relax)
    assert abs(loss - ref_loss) <= ltol * abs(ref_loss)
    gr = m.grads()
    for k in ref_g:
        assert rel(gr[k], ref_g[k]) <= gtol, (k, rel(gr[k], ref_g[k]))
    m.close()
    ilu.close()


def test_probes_are_the_arnoldi_vectors(handle, case, torch_cuda):
    s, A, Ao, ilu_o, _, _ = case
    import blocksp_b200 as bsp
    ilu = bsp.ILU0(A)
    K = 6
    Q = learned.probes(A, ilu, s.b, K).cpu().numpy()
    assert np.abs(Q @ Q.T - np.eye(K)).max() <= 1e-12
    v = ilu_o(s.b)
    ref = [v / np.linalg.norm(v)]
    for _ in range(1, K):
        w = ilu_o(O.bsmv(Ao, ref[-1]))
        for q in ref:
            w = w - (q @ w) * q
        ref.append(w / np.linalg.norm(w))
    assert rel(Q, np.array(ref)) <= 1e-9
    ilu.close()


def test_zero_decoders_reproduce_ilu0(handle, case, torch_cuda):
    torch = torch_cuda
    s, A, _, _, _, _ = case
    import blocksp_b200 as bsp
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32)  # decoders start at zero
    dF = m.forward(A).cpu().numpy()
    assert not np.any(dF)
    lp = m.precond(A)
    ilu = bsp.ILU0(A)
    f1, f2 = lp.export(), ilu.export()
    assert np.array_equal(f1, f2), float(np.abs(f1 - f2).max())
    r = torch.tensor(s.b, device="cuda")
    z1, z2, z3 = r.clone(), r.clone(), r.clone()
    lp(z1)
    ilu(z2)
    ilu(z3)
    assert torch.equal(z2, z3), "ILU0 apply not repeatable"
    assert torch.equal(z1, z2), float((z1 - z2).abs().max() / z2.abs().max())
    lp.close()
    ilu.close()
    m.close()


@pytest.mark.parametrize("relax", [0.25, 0.6])
def test_relaxation_scales_the_off_diagonal_factors(handle, case, torch_cuda, relax):
    """Zero decoders with a relaxation: the learned factors are ILU0's with
    every off-diagonal block scaled by 1 + relax (diagonal blocks bit for bit),
    and the preconditioner applies them like the oracle's ILU0 on those factors."""
    torch = torch_cuda
    s, A, Ao, _, g, _ = case
    import blocksp_b200 as bsp
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32, meta={"relax": relax})
    lp = m.precond(A)
    ilu = bsp.ILU0(A)
    f1, f0 = lp.export(), ilu.export()
    rows = np.repeat(np.arange(s.n), np.diff(s.row_ptr))
    off = s.col_idx != rows
    assert np.array_equal(f1[~off], f0[~off])
    assert rel(f1[off], f0[off] * (1 + relax)) <= 1e-15
    ref = O.ILU0(Ao)
    ref.LU.vals[:] = LO.relaxed(g, ref.LU.vals, relax)
    r = np.random.default_rng(7).uniform(-1, 1, s.n * 8)
    assert rel(lp.apply_host(r), ref(r)) <= 1e-11
    for o in (lp, ilu, m):
        o.close()
    with pytest.raises(_lib.BspError):
        learned.LearnedModel(handle, 8, _lib.BSP_F32, meta={"relax": -1.0})


def test_training_lowers_the_loss(handle, torch_cuda):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((12, 12, 12), 8, 41)
    A = bsp.Matrix.from_system(s, handle)
    ilu = bsp.ILU0(A)
    Q = learned.probes(A, ilu, s.b, 8)
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32)
    losses = []
    for _ in range(30):
        losses.append(m.loss_grad(A, ilu, Q))
        m.adam_step(1e-4)
    assert losses[-1] < losses[0], losses
    # the trained correction is applied by the same sweeps and still solves
    lp = m.precond(A)
    x, info, _ = bsp.pGMRES(A, s.b, 1e-10, lp, 2000, 30, 10, return_info=True,
                           stop_rule=_lib.STOP_TRUE_RESIDUAL)
    assert info["true_rel_res"] <= 1e-10
    for o in (lp, ilu, m, A):
        o.close()


def test_fallback_to_ilu0(handle, case):
    s, A, _, _, _, _ = case
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32, meta={"beats_ilu0": False})
    pc = learned.LearnedLU(A, m)
    assert pc.kind == _lib.PC_ILU0
    pc.close()
    pc = learned.LearnedLU(A, None)
    assert pc.kind == _lib.PC_ILU0
    pc.close()
    m.meta["beats_ilu0"] = True
    pc = learned.LearnedLU(A, m)
    assert pc.kind == _lib.PC_LEARNED_LU
    pc.close()
    m.close()
