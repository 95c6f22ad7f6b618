"""The vector kernels on their own: bsp_dot, bsp_dot_dev and bsp_axpy_dev
(the reference's dot / axpy on solArrays, blocksp_utility.hpp) against numpy.

Criteria: a dot product within 1e-14 of numpy's, relative to sum |x_i y_i|
(the rounding of any summation order); the same call twice gives the same bits
(the partial sums are combined in index order); the device-result form equals
the host-result form; axpy y += a x within 2 ulp-scale (1e-15 relative to
|a x| + |y|) of numpy, elementwise.  Sizes cover the empty vector, sizes
around one CTA's chunk and a vector of the benchmark's length.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 5, 4097, 8192, 8193, 1_000_003, 2_097_152]


@pytest.fixture(scope="module")
def lib():
    from blocksp_b200 import _lib
    return _lib.load()


def vectors(torch, n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, max(n, 1))
    y = rng.uniform(-1, 1, max(n, 1))
    return x, y, torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")


@pytest.mark.parametrize("n", SIZES)
def test_dot_matches_numpy_and_repeats(lib, handle, torch_cuda, n):
    torch = torch_cuda
    x, y, xd, yd = vectors(torch, n, n + 11)
    out = [C.c_double(), C.c_double()]
    for o in out:
        assert lib.bsp_dot(handle.h, n, xd.data_ptr(), yd.data_ptr(), C.byref(o)) == 0
    ref = float(np.dot(x[:n], y[:n])) if n else 0.0
    scale = float(np.abs(x[:n] * y[:n]).sum()) if n else 0.0
    assert abs(out[0].value - ref) <= 1e-14 * max(scale, 1e-300)
    assert out[0].value == out[1].value  # bit for bit
    # the device-result form gives the same value
    dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.bsp_dot_dev(handle.h, n, xd.data_ptr(), yd.data_ptr(), dev.data_ptr()) == 0
    assert lib.bsp_handle_sync(handle.h) == 0
    assert float(dev.item()) == out[0].value


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("a", [0.0, 1.0, -2.5e-3])
def test_axpy_matches_numpy(lib, handle, torch_cuda, n, a):
    torch = torch_cuda
    x, y, xd, yd = vectors(torch, n, 3 * n + 1)
    assert lib.bsp_axpy_dev(handle.h, n, a, xd.data_ptr(), yd.data_ptr()) == 0
    assert lib.bsp_handle_sync(handle.h) == 0
    got = yd.cpu().numpy()[:n]
    ref = y[:n] + a * x[:n]
    tol = 1e-15 * (np.abs(a * x[:n]) + np.abs(y[:n])) + 1e-300
    assert np.all(np.abs(got - ref) <= tol)
    # entries past n are untouched
    if n == 0:
        assert yd.cpu().numpy()[0] == y[0]
