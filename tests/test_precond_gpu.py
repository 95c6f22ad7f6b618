"""Preconditioner parity: GPU Diag / SOR / ILU0 / IChol0 against the CPU oracle.

Tolerances (FP64): factor blocks <= 1e-12 relative to the largest block entry;
one preconditioner application <= 1e-11 relative (infinity norm).  The GPU
inverts diagonal blocks explicitly where the reference calls getrs/pptrs, and
sums block rows in a different order, so agreement is to rounding, amplified
at most by the triangular solves' condition.
"""
import numpy as np
import pytest

from blocksp_b200.systems import grid_system
import oracle.blocksp_oracle as O

pytestmark = pytest.mark.gpu

SPD = [((10, 10), 4), ((7, 7), 2), ((5, 5), 3), ((4, 4, 4), 8), ((3, 3, 3), 16), ((6, 5), 1)]
NONSYM = [((4, 4, 4), 8), ((3, 3, 3), 16), ((6, 6), 4), ((5, 4), 3)]


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def build(handle, dims, bs, skew, seed=7):
    import blocksp_b200 as bsp
    s = grid_system(dims, bs, seed=seed, skew=skew)
    return s, bsp.Matrix.from_system(s, handle), O.BSR.from_system(s)


@pytest.mark.parametrize("dims,bs", SPD)
def test_ichol0_factor_and_apply(handle, dims, bs):
    import blocksp_b200 as bsp
    s, A, Ao = build(handle, dims, bs, 0.0)
    pc = bsp.IChol0(A)
    ref = O.IChol0(Ao)
    assert rel(pc.export(), ref.L.vals) <= 1e-12
    r = np.random.default_rng(1).uniform(-1, 1, s.n * bs)
    assert rel(pc.apply_host(r), ref(r)) <= 1e-11
    inf = pc.info()
    assert inf["levels_lower"] >= 1 and inf["levels_upper"] >= 1


@pytest.mark.parametrize("dims,bs", SPD + NONSYM)
def test_ilu0_factor_and_apply(handle, dims, bs):
    import blocksp_b200 as bsp
    skew = 0.3 if len(dims) == 3 or bs in (3,) else 0.0
    s, A, Ao = build(handle, dims, bs, skew)
    pc = bsp.ILU0(A)
    ref = O.ILU0(Ao)
    assert rel(pc.export(), ref.LU.vals) <= 1e-12
    r = np.random.default_rng(2).uniform(-1, 1, s.n * bs)
    assert rel(pc.apply_host(r), ref(r)) <= 1e-11


@pytest.mark.parametrize("dims,bs", SPD[:4] + NONSYM[:2])
@pytest.mark.parametrize("inv", ["LU", "Chol"])
def test_diag(handle, dims, bs, inv):
    import blocksp_b200 as bsp
    s, A, Ao = build(handle, dims, bs, 0.0)
    pc = bsp.Diag(A, inv)
    ref = O.Diag(Ao, O.LUFactor if inv == "LU" else O.CholeskyFactor)
    r = np.random.default_rng(3).uniform(-1, 1, s.n * bs)
    assert rel(pc.apply_host(r), ref(r)) <= 1e-11


@pytest.mark.parametrize("dims,bs,skew", [((8, 8), 4, 0.0), ((4, 4, 4), 8, 0.3), ((5, 5), 3, 0.0),
                                          ((3, 3, 3), 16, 0.3)])
@pytest.mark.parametrize("w,nu,typ", [(1.6, 3, 0), (1.2, 2, 1), (0.6, 1, -1), (1.0, 1, 0)])
def test_sor(handle, dims, bs, skew, w, nu, typ):
    import blocksp_b200 as bsp
    s, A, Ao = build(handle, dims, bs, skew)
    pc = bsp.SOR(A, w, nu, typ)
    ref = O.SOR(Ao, w, nu, typ)
    r = np.random.default_rng(4).uniform(-1, 1, s.n * bs)
    assert rel(pc.apply_host(r), ref(r)) <= 1e-11


def test_device_apply_in_place(handle, torch_cuda):
    import blocksp_b200 as bsp
    torch = torch_cuda
    s, A, Ao = build(handle, (12, 12), 4, 0.0)
    pc = bsp.IChol0(A)
    r = np.random.default_rng(5).uniform(-1, 1, s.n * 4)
    rd = torch.tensor(r, device="cuda")
    pc(rd)
    handle.sync()
    assert rel(rd.cpu().numpy(), O.IChol0(Ao)(r)) <= 1e-11


def test_zero_diagonal_block_is_reported(handle):
    import blocksp_b200 as bsp
    # row 0 has no lower neighbours, so its ILU0 pivot block is A_00 itself
    s = grid_system((5, 5), 4, seed=2)
    d = [t for t in range(s.row_ptr[0], s.row_ptr[1]) if s.col_idx[t] == 0][0]
    s.vals[d] = 0.0
    A = bsp.Matrix.from_system(s, handle)
    for make in (bsp.ILU0, lambda M: bsp.Diag(M, "LU"), lambda M: bsp.SOR(M, 1.0, 1)):
        with pytest.raises(bsp.BspError) as e:
            make(A)
        assert e.value.status == 1  # BSP_ZERO_PIVOT


def test_not_spd_is_reported(handle):
    import blocksp_b200 as bsp
    s = grid_system((5, 5), 4, seed=2)
    d = [t for t in range(s.row_ptr[3], s.row_ptr[4]) if s.col_idx[t] == 3][0]
    s.vals[d] = -np.eye(4)
    A = bsp.Matrix.from_system(s, handle)
    with pytest.raises(bsp.BspError) as e:
        bsp.IChol0(A)
    assert e.value.status == 2  # BSP_NOT_SPD


def test_missing_diagonal_block_is_reported(handle):
    import blocksp_b200 as bsp
    from blocksp_b200.systems import BSRSystem
    # 2 block rows, row 1 has no diagonal block
    s = BSRSystem(n=2, bs=2, row_ptr=np.array([0, 1, 2], np.int32), col_idx=np.array([0, 0], np.int32),
                  vals=np.stack([np.eye(2), np.eye(2)]), b=np.ones(4))
    A = bsp.Matrix.from_system(s, handle)
    with pytest.raises(bsp.BspError) as e:
        bsp.ILU0(A)
    assert e.value.status == 1


def long_row_system(n, bs, band, seed):
    """Block rows holding every block column in [i - band, i + 2] (clipped):
    rows past `band` have more lower entries than the factorisation stages per
    row, so both the staged and the global-memory elimination plans run.
    Diagonal blocks dominate, so ILU0 exists and is well conditioned."""
    from blocksp_b200.systems import BSRSystem
    rng = np.random.default_rng(seed)
    rp, ci, vs = [0], [], []
    for i in range(n):
        cols = list(range(max(0, i - band), min(n, i + 3)))
        blocks = {j: rng.uniform(-1, 1, (bs, bs)) / (bs * len(cols)) for j in cols if j != i}
        blocks[i] = np.eye(bs) * 2.0 + rng.uniform(-0.1, 0.1, (bs, bs))
        for j in cols:
            ci.append(j)
            vs.append(blocks[j])
        rp.append(len(ci))
    return BSRSystem(n=n, bs=bs, row_ptr=np.array(rp, dtype=np.int32), col_idx=np.array(ci, dtype=np.int32),
                     vals=np.array(vs).reshape(-1, bs, bs), b=rng.uniform(-1, 1, n * bs), name=f"band{band}")


@pytest.mark.parametrize("bs", [4, 8, 16])
def test_ilu0_long_rows(handle, bs):
    """Rows with 40 lower blocks (more than the staged plan holds) against the oracle."""
    import blocksp_b200 as bsp
    s = long_row_system(72, bs, 40, seed=bs)
    A = bsp.Matrix.from_system(s, handle)
    pc = bsp.ILU0(A)
    ref = O.ILU0(O.BSR.from_system(s))
    assert rel(pc.export(), ref.LU.vals) <= 1e-12
    r = np.random.default_rng(3).uniform(-1, 1, s.n * bs)
    assert rel(pc.apply_host(r), ref(r)) <= 1e-11
    pc.close()
    A.close()
