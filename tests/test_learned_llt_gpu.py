"""The learned L L^T preconditioner (SPD systems, pCG) on the GPU against the
oracle's L L^T specification (oracle/learned_oracle.py, form="llt").

Same criteria as the LU form: forward correction FP64 within 1e-12 and FP32
within 1e-4 of the oracle; loss and every parameter gradient FP64 within 1e-9
(loss 1e-10), FP32 within 2e-3; zero decoders reproduce block IChol0 bit for
bit; training lowers the loss and the factors still solve with pCG; and
LearnedLLT falls back to IChol0 for a model that has not beaten it.
"""
import numpy as np
import pytest

from blocksp_b200 import _lib, learned, systems
import oracle.learned_oracle as LO
from test_learned_oracle import ichol0_in_a_order

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def spd_case(handle):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((5, 4, 3), 8, 33, speed=0.0)
    A = bsp.Matrix.from_system(s, handle)
    g = LO.graph_of(s.row_ptr, s.col_idx)
    rng = np.random.default_rng(15)
    p = LO.init_params(8, seed=19)
    for k in p:
        p[k] = p[k] + (0.005 if k in ("Wo", "bo", "Wd", "bd") else 0.05) * rng.standard_normal(p[k].shape)
    yield s, A, g, p
    A.close()


@pytest.mark.parametrize("dtype,tol", [(_lib.BSP_F64, 1e-12), (_lib.BSP_F32, 1e-4)])
def test_llt_forward_matches_oracle(handle, spd_case, dtype, tol):
    s, A, g, p = spd_case
    m = learned.LearnedModel(handle, 8, dtype, params=p, form="llt")
    dF = m.forward(A).cpu().numpy()
    ref, _ = LO.forward(p, g, s.vals, form="llt")
    assert rel(dF, ref) <= tol
    m.close()


@pytest.mark.parametrize("relax", [0.0, 0.4])
@pytest.mark.parametrize("dtype,ltol,gtol", [(_lib.BSP_F64, 1e-10, 1e-9), (_lib.BSP_F32, 1e-4, 2e-3)])
def test_llt_loss_and_gradients_match_oracle(handle, spd_case, torch_cuda, dtype, ltol, gtol, relax):
    torch = torch_cuda
    s, A, g, p = spd_case
    import blocksp_b200 as bsp
    ic = bsp.IChol0(A)
    F0 = learned.ilu_factors(A, ic).cpu().numpy()
    assert rel(F0, ichol0_in_a_order(s)) <= 1e-13
    rng = np.random.default_rng(16)
    Qh = np.linalg.qr(rng.standard_normal((s.n * 8, 3)))[0].T.copy()
    m = learned.LearnedModel(handle, 8, dtype, params=p, form="llt", meta={"relax": relax})
    loss = m.loss_grad(A, ic, torch.tensor(Qh, device="cuda"))
    ref_loss, ref_g = LO.loss_and_grads(p, g, s.vals, F0, Qh, form="llt", relax=relax)
    assert abs(loss - ref_loss) <= ltol * abs(ref_loss)
    gr = m.grads()
    for k in ref_g:
        assert rel(gr[k], ref_g[k]) <= gtol, (k, rel(gr[k], ref_g[k]))
    m.close()
    ic.close()


def test_llt_zero_decoders_reproduce_ichol0(handle, spd_case, torch_cuda):
    torch = torch_cuda
    s, A, _, _ = spd_case
    import blocksp_b200 as bsp
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32, form="llt")
    lp = m.precond(A)
    ic = bsp.IChol0(A)
    assert lp.kind == _lib.PC_LEARNED_LLT
    r = torch.tensor(s.b, device="cuda")
    z1, z2 = r.clone(), r.clone()
    lp(z1)
    ic(z2)
    # the learned factor's diagonal inverses are general inverses of the same
    # triangular blocks: equal to rounding
    assert float((z1 - z2).abs().max() / z2.abs().max()) <= 1e-12
    for o in (lp, ic, m):
        o.close()


def test_llt_training_lowers_the_loss_and_pcg_solves(handle, torch_cuda):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((12, 12, 12), 8, 43, speed=0.0)
    A = bsp.Matrix.from_system(s, handle)
    ic = bsp.IChol0(A)
    Q = learned.probes(A, ic, s.b, 8)
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32, form="llt")
    losses = []
    for _ in range(30):
        losses.append(m.loss_grad(A, ic, Q))
        m.adam_step(1e-4)
    assert losses[-1] < losses[0], losses
    lp = m.precond(A)
    x, info, _ = bsp.pCG(A, s.b, 1e-10, lp, 5000, return_info=True, stop_rule=_lib.STOP_TRUE_RESIDUAL)
    assert info["true_rel_res"] <= 1e-10
    for o in (lp, ic, m, A):
        o.close()


def test_llt_fallback_to_ichol0(handle, spd_case):
    s, A, _, _ = spd_case
    m = learned.LearnedModel(handle, 8, _lib.BSP_F32, meta={"beats_baseline": False}, form="llt")
    assert learned.LearnedLLT(A, m).kind == _lib.PC_ICHOL0
    assert learned.LearnedLLT(A, None).kind == _lib.PC_ICHOL0
    m.meta["beats_baseline"] = True
    assert learned.LearnedLLT(A, m).kind == _lib.PC_LEARNED_LLT
    m.close()
