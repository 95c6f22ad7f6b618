"""Ablation of the trained models against the methods without them.

LU form (blocksp_b200/weights/learned_convdiff_bs8.npz, trained on the GPU on
convection-diffusion systems at 64^3): on held-out seeds, pGMRES(30, k=10) to
the FP64 true residual 1e-10 runs with block ILU0, with the learned factors,
and with LearnedLU — which uses the learned factors only when the model's
recorded validation beat ILU0's total iteration count, and otherwise falls back
to ILU0.

L L^T form (blocksp_b200/weights/learned_diffusion_llt_bs8.npz, trained on SPD
diffusion systems at 64^3): on held-out seeds, pCG to the FP64 true residual
1e-10 with block IChol0 and with LearnedLLT.

Checked: every variant reaches 1e-10; the gate recorded in the weights matches
its own validation numbers; the gated preconditioner is exactly the baseline
(same kind, same iteration count) when the gate is closed, and takes fewer
iterations than the baseline when it is open.  The iteration counts are
printed (bench.py --workload learned / learned_llt measures the times).
"""
import pytest

from blocksp_b200 import _lib, learned, systems

pytestmark = pytest.mark.gpu


def test_weights_and_gate_are_consistent():
    assert learned.WEIGHTS.exists()
    m = learned.LearnedModel.load()
    val = m.meta["validation"]
    assert len(val) >= 2
    beats = sum(v["learned_iters"] for v in val) < sum(v["ilu0_iters"] for v in val) and \
        all(v["learned_res"] <= 1e-10 for v in val)
    assert bool(m.meta["beats_ilu0"]) == beats
    m.close()


@pytest.mark.parametrize("seed", [30100, 30101])
def test_ablation_held_out(handle, seed):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((24, 24, 24), 8, seed)
    A = bsp.Matrix.from_system(s, handle)
    m = learned.LearnedModel.load(handle=handle)
    ilu = bsp.ILU0(A)
    it0, r0 = learned.solve_iters(A, s.b, ilu)
    lp = m.precond(A)
    it1, r1 = learned.solve_iters(A, s.b, lp)
    gated = learned.LearnedLU(A, m)
    it2, r2 = learned.solve_iters(A, s.b, gated)
    print(f"seed {seed}: ILU0 {it0} iterations, learned {it1}, LearnedLU {it2} "
          f"(gate {'open' if m.meta['beats_ilu0'] else 'closed'})")
    assert max(r0, r1, r2) <= 1e-10
    if not m.meta["beats_ilu0"]:
        assert gated.kind == _lib.PC_ILU0 and it2 == it0
    else:
        assert gated.kind == _lib.PC_LEARNED_LU and it2 == it1
    for o in (gated, lp, ilu, m, A):
        o.close()


def test_llt_weights_and_gate_are_consistent():
    assert learned.WEIGHTS_LLT.exists()
    m = learned.LearnedModel.load(learned.WEIGHTS_LLT)
    assert m.form == "llt"
    assert m.relax == m.meta["relax"]
    val = m.meta["validation"]
    assert len(val) >= 2
    beats = sum(v["learned_iters"] for v in val) < sum(v["ilu0_iters"] for v in val) and \
        all(v["learned_res"] <= 1e-10 for v in val)
    assert bool(m.meta["beats_baseline"]) == beats
    m.close()


@pytest.mark.parametrize("seed", [30200, 30201])
def test_llt_ablation_held_out(handle, seed):
    import blocksp_b200 as bsp
    s = systems.convection_diffusion_system((32, 32, 32), 8, seed, speed=0.0)
    A = bsp.Matrix.from_system(s, handle)
    m = learned.LearnedModel.load(learned.WEIGHTS_LLT, handle=handle)
    ic = bsp.IChol0(A)
    it0, r0 = learned.solve_iters(A, s.b, ic, form="llt")
    gated = learned.LearnedLLT(A, m)
    it1, r1 = learned.solve_iters(A, s.b, gated, form="llt")
    print(f"seed {seed}: IChol0 {it0} iterations, LearnedLLT {it1} (relax {m.relax:g}, "
          f"gate {'open' if m.meta['beats_baseline'] else 'closed'})")
    assert max(r0, r1) <= 1e-10
    if m.meta["beats_baseline"]:
        assert gated.kind == _lib.PC_LEARNED_LLT and it1 < it0
    else:
        assert gated.kind == _lib.PC_ICHOL0 and it1 == it0
    for o in (gated, ic, m, A):
        o.close()
