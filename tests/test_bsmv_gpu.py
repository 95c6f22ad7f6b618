"""bsmv parity: the CUDA kernels against the CPU oracle (blocksp_multiply.hpp:166-325).

FP64 tolerance: relative infinity-norm error <= 1e-14 (the summation order of a
block row differs from the reference's only at the ulp level).  FP32 values
and vectors: <= 1e-5 relative.  BF16 storage with FP32 accumulation: the
stored matrix is the BF16 rounding of A, so the product is compared with the
oracle applied to that rounded matrix at <= 1e-5.
"""
import numpy as np
import pytest

from blocksp_b200.systems import BSRSystem, grid_system
import oracle.blocksp_oracle as O

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b)).max()
    return d / max(np.abs(b).max(), 1e-300)


def random_bsr(n, bs, density, seed, empty_rows=(), n_cols=None):
    rng = np.random.default_rng(seed)
    n_cols = n_cols or n
    rp, ci = [0], []
    for i in range(n):
        if i in empty_rows:
            rp.append(len(ci))
            continue
        cols = np.flatnonzero(rng.random(n_cols) < density)
        rng.shuffle(cols)  # insertion order, as the reference container keeps it
        ci.extend(cols.tolist())
        rp.append(len(ci))
    vals = rng.standard_normal((len(ci), bs, bs))
    return BSRSystem(n=n, bs=bs, row_ptr=np.array(rp, np.int32), col_idx=np.array(ci, np.int32),
                     vals=vals, b=rng.uniform(-1, 1, n_cols * bs))


@pytest.mark.parametrize("bs", [1, 2, 3, 4, 5, 8, 16, 32])
@pytest.mark.parametrize("nrhs", [1, 2, 4, 5])
def test_bsmv_fp64_random(handle, torch_cuda, bs, nrhs):
    import blocksp_b200 as bsp
    torch = torch_cuda
    s = random_bsr(57, bs, 0.12, seed=bs * 31 + nrhs, empty_rows=(3, 40))
    A = bsp.Matrix.from_system(s, handle)
    x = np.random.default_rng(bs + nrhs).uniform(-1, 1, s.n * bs * nrhs)
    ref = O.bsmv(O.BSR.from_system(s), x, nrhs=nrhs)
    xd = torch.tensor(x, device="cuda")
    yd = torch.full((s.n * bs * nrhs,), float("nan"), dtype=torch.float64, device="cuda")
    bsp.bsmv_dev(A, xd, yd, nrhs=nrhs)
    handle.sync()
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-14
    # accumulate form (void bsmv(b, A, x) adds into b)
    y0 = np.random.default_rng(7).uniform(-1, 1, s.n * bs * nrhs)
    yd = torch.tensor(y0, device="cuda")
    bsp.bsmv_dev(A, xd, yd, nrhs=nrhs, beta=1.0)
    handle.sync()
    assert rel_err(yd.cpu().numpy(), y0 + ref) <= 1e-14
    # transposed form
    reft = O.bsmv(O.BSR.from_system(s), x, nrhs=nrhs, transpose=True)
    yt = torch.zeros(s.n * bs * nrhs, dtype=torch.float64, device="cuda")
    bsp.bsmv_dev(A, xd, yt, nrhs=nrhs, transpose=True)
    handle.sync()
    assert rel_err(yt.cpu().numpy(), reft) <= 1e-14


@pytest.mark.parametrize("dims,bs,skew", [((16, 16), 4, 0.0), ((8, 8, 8), 8, 0.3), ((6, 6, 6), 16, 0.3)])
def test_bsmv_stencil_host_api(handle, dims, bs, skew):
    import blocksp_b200 as bsp
    s = grid_system(dims, bs, seed=11, skew=skew)
    A = bsp.Matrix.from_system(s, handle)
    ref = O.bsmv(O.BSR.from_system(s), s.b)
    y = bsp.bsmv(A, s.b)
    assert rel_err(y, ref) <= 1e-14
    acc = np.ones_like(ref)
    bsp.bsmv(A, s.b, b=acc)
    assert rel_err(acc, ref + 1.0) <= 1e-14


@pytest.mark.parametrize("bs,dtype", [(4, "f32"), (8, "f32"), (16, "f32"), (8, "bf16"), (16, "bf16")])
def test_bsmv_low_precision(handle, torch_cuda, bs, dtype):
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib
    torch = torch_cuda
    s = grid_system((6, 6, 5), bs, seed=5, skew=0.3)
    A = bsp.Matrix.from_system(s, handle)
    code = _lib.BSP_F32 if dtype == "f32" else _lib.BSP_BF16
    A.make_lowp(code)
    x = np.random.default_rng(3).uniform(-1, 1, s.n * bs).astype(np.float32)
    if dtype == "f32":
        vals = s.vals.astype(np.float32).astype(np.float64)
    else:
        vals = torch.tensor(s.vals).to(torch.bfloat16).to(torch.float64).numpy()
    sr = O.BSR(s.n, bs, s.row_ptr, s.col_idx, vals)
    ref = O.bsmv(sr, x.astype(np.float64))
    xd = torch.tensor(x, device="cuda")
    yd = torch.zeros(s.n * bs, dtype=torch.float32, device="cuda")
    bsp.bsmv_dev(A, xd, yd, dtype=code)
    handle.sync()
    assert rel_err(yd.cpu().numpy().astype(np.float64), ref) <= 1e-5


def test_bsmv_empty_matrix(handle, torch_cuda):
    import blocksp_b200 as bsp
    torch = torch_cuda
    s = BSRSystem(n=4, bs=8, row_ptr=np.zeros(5, np.int32), col_idx=np.zeros(0, np.int32),
                  vals=np.zeros((0, 8, 8)), b=np.ones(32))
    A = bsp.Matrix.from_system(s, handle)
    y = torch.full((32,), 5.0, dtype=torch.float64, device="cuda")
    bsp.bsmv_dev(A, torch.ones(32, dtype=torch.float64, device="cuda"), y)
    handle.sync()
    assert float(y.abs().max()) == 0.0
