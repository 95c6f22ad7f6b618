"""Batched block-IChol0 pCG: every (system, RHS) pair against the oracle.

The batched solve replaces the loop ``IChol0_pCG<T,bs,1>(A_s).solve(A_s, b)``
over systems and right-hand sides (blocksp_solvers.hpp:481-492); each pair is
checked like a single pCG solve, against the oracle and the oracle's own
spread when its matrix product and preconditioner output are perturbed at
rounding level (three runs): iteration count within that spread +-1, solution
within max(1e-8, 10x the spread) relative, residual history within 1e-10 plus
10x the history spread (the pCG criterion of test_solvers_gpu.py).  Slowly
converging pairs (the 16x16-block system needs ~115 iterations) move by a few
iterations under rounding-level perturbations, which the spread captures.
The batch mixes block sizes 4, 8 and 16 and uneven grid sizes, so systems
converge at different iterations and drop out of the batch at different times.
"""
import numpy as np
import pytest

from blocksp_b200 import systems
from parity import cg_spread, check_history, rel
import oracle.blocksp_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10
SPECS = [(6, 4, 501), (11, 8, 502), (9, 4, 503), (16, 8, 504), (5, 16, 505), (13, 4, 506), (8, 8, 507)]


def make_batch(specs, nrhs):
    return [systems.batch_system(side, bs, seed, nrhs=nrhs) for side, bs, seed in specs]


def column(s, v, nrhs, r):
    return v.reshape(s.n, nrhs, s.bs)[:, r, :].ravel()


def pack(sys_list):
    return np.concatenate([s.b for s in sys_list])


def within_spread(it, ref, its):
    allv = its + [ref.iters]
    return min(allv) - 1 <= it <= max(allv) + 1


@pytest.fixture(scope="module")
def batch4(handle):
    import blocksp_b200 as bsp
    sl = make_batch(SPECS, 4)
    B = bsp.Batch(sl, handle)
    yield sl, B
    B.close()


def test_batch_matches_oracle_per_pair(batch4):
    sl, B = batch4
    nrhs = 4
    x, info = B.pcg(pack(sl), nrhs, TOL, 2000, hist_cap=600)
    assert info["status"] == 0 and info["n_converged"] == info["n_pairs"] == len(sl) * nrhs
    res = B.results()
    off = B.offsets(nrhs)
    for si, s in enumerate(sl):
        Ao = O.BSR.from_system(s)
        ic = O.IChol0(Ao)
        xs = x[off[si]:off[si + 1]]
        for r in range(nrhs):
            bv = column(s, s.b, nrhs, r)
            ref = O.pcg(Ao, bv, TOL, ic, 2000)
            env, its, xdev = cg_spread(Ao, bv, TOL, ic, 2000, ref)
            it = int(res["iters"][si, r])
            assert within_spread(it, ref, its), (si, r, it, ref.iters, its)
            assert rel(column(s, xs, nrhs, r), ref.x) <= max(1e-8, 10 * max(xdev))
            hist = res["hist"][si, r, : it + 2]
            n = min(len(ref.hist), it + 2)
            check_history(hist[:n], ref.hist[:n], envelope=env)


def test_batch_matches_single_system_solver(handle, batch4):
    """Each pair equals the single-system GPU IChol0_pCG solve of that RHS
    within the oracle's own rounding spread."""
    import blocksp_b200 as bsp
    sl, B = batch4
    nrhs = 4
    x, _ = B.pcg(pack(sl), nrhs, TOL, 2000)
    res = B.results()
    off = B.offsets(nrhs)
    for si in (0, 3, 4):
        s = sl[si]
        A = bsp.Matrix.from_system(s, handle)
        pc = bsp.IChol0(A)
        Ao = O.BSR.from_system(s)
        ic = O.IChol0(Ao)
        for r in range(nrhs):
            bv = column(s, s.b, nrhs, r)
            xr, inf, _ = bsp.pCG(A, bv, TOL, pc, 2000, return_info=True)
            ref = O.pcg(Ao, bv, TOL, ic, 2000)
            _, its, xdev = cg_spread(Ao, bv, TOL, ic, 2000, ref)
            allv = its + [ref.iters]
            assert abs(inf["iters"] - res["iters"][si, r]) <= max(allv) - min(allv) + 1
            assert rel(column(s, x[off[si]:off[si + 1]], nrhs, r), xr) <= max(1e-8, 20 * max(xdev))
        pc.close()
        A.close()


def test_host_loop_mode_is_identical(batch4):
    sl, B = batch4
    nrhs = 4
    b = pack(sl)
    x0, i0 = B.pcg(b, nrhs, TOL, 2000, mode=0)
    x1, i1 = B.pcg(b, nrhs, TOL, 2000, mode=1, check_every=3)
    assert np.array_equal(x0, x1)
    assert i0["iters_total"] == i1["iters_total"]
    # the loop ran until the slowest pair finished
    assert i0["graph_iters"] == i0["iters_max"] + 1 == i1["graph_iters"]


def test_device_buffers_and_repeat_are_deterministic(batch4, torch_cuda):
    torch = torch_cuda
    sl, B = batch4
    nrhs = 4
    b = pack(sl)
    xh, _ = B.pcg(b, nrhs, TOL, 2000)
    bd = torch.tensor(b, device="cuda")
    xd, info = B.pcg(bd, nrhs, TOL, 2000)
    xd2, _ = B.pcg(bd, nrhs, TOL, 2000)
    assert np.array_equal(xd.cpu().numpy(), xh)
    assert torch.equal(xd, xd2)
    tun = B.tuning()
    assert [g["bs"] for g in tun] == [4, 8, 16]
    assert all(g["tile_threads"] in (128, 256, 512) and g["sweep_ctas_per_sm"] >= 1 for g in tun)
    assert sum(g["systems"] for g in tun) == len(sl)


@pytest.mark.parametrize("nrhs", [1, 2])
def test_fewer_rhs(handle, nrhs):
    import blocksp_b200 as bsp
    sl = make_batch(SPECS[:4], nrhs)
    B = bsp.Batch(sl, handle)
    x, info = B.pcg(pack(sl), nrhs, TOL, 2000)
    assert info["status"] == 0
    res = B.results()
    off = B.offsets(nrhs)
    for si, s in enumerate(sl):
        Ao = O.BSR.from_system(s)
        ic = O.IChol0(Ao)
        for r in range(nrhs):
            bv = column(s, s.b, nrhs, r)
            ref = O.pcg(Ao, bv, TOL, ic, 2000)
            _, its, xdev = cg_spread(Ao, bv, TOL, ic, 2000, ref)
            assert within_spread(int(res["iters"][si, r]), ref, its)
            assert rel(column(s, x[off[si]:off[si + 1]], nrhs, r), ref.x) <= max(1e-8, 10 * max(xdev))
    B.close()


def test_zero_rhs_pair_and_max_iters(handle):
    """A zero right-hand side converges at once with x = 0 (res_mag[0] = 0 is not
    above tol * 0); a small iteration limit ends pairs with the MAXIT state and
    the reference's count (it stops once it exceeds maxIters)."""
    import blocksp_b200 as bsp
    sl = make_batch(SPECS[:3], 2)
    sl[1].b.reshape(sl[1].n, 2, sl[1].bs)[:, 1, :] = 0.0
    B = bsp.Batch(sl, handle)
    b = pack(sl)
    x, info = B.pcg(b, 2, TOL, 2000)
    res = B.results()
    off = B.offsets(2)
    assert res["state"][1, 1] == 1 and res["iters"][1, 1] == 0
    assert not np.any(column(sl[1], x[off[1]:off[2]], 2, 1))
    x, info = B.pcg(b, 2, TOL, 5)
    res = B.results()
    assert info["status"] == 4
    live = res["state"] != 1
    assert np.all(res["state"][live] == 2) and np.all(res["iters"][live] == 6)
    Ao = O.BSR.from_system(sl[0])
    ref = O.pcg(Ao, column(sl[0], sl[0].b, 2, 0), TOL, O.IChol0(Ao), 5)
    assert ref.iters == 6
    assert rel(column(sl[0], x[:off[1]], 2, 0), ref.x) <= 1e-8
    B.close()
