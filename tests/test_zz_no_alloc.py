"""bsp_dot_noalloc: the dot product for callers that cannot allocate device memory.

A caller that is handed a stream and device pointers by another framework (a
plugin or callback that does not own the allocator), or that runs where an
allocation is not allowed, cannot create a handle, because a handle allocates
its reduction workspace.  This entry point takes only a stream and device
pointers and keeps its scratch in a fixed device array.  The test calls it
through the C ABI twice in a row and checks both results against the existing
handle-based entry point, bsp_dot, within the FP64 reduction tolerance used
elsewhere in the suite (1e-14 relative to sum |x_i y_i|), and checks that a
size beyond the scratch limit is rejected with BSP_INVALID.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 8192 * 4096  # the documented limit: one CTA of 8,192 elements per scratch slot


@pytest.fixture(scope="module")
def lib():
    from blocksp_b200 import _lib
    return _lib.load()


@pytest.mark.parametrize("n", [0, 1, 777, 8192, 8193, 2_097_152, MAX_N])
def test_noalloc_dot_matches_handle_dot(lib, handle, torch_cuda, n):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(n + 1)
    x = torch.rand(max(n, 1), dtype=torch.float64, device="cuda", generator=g) - 0.25
    y = torch.rand(max(n, 1), dtype=torch.float64, device="cuda", generator=g) - 0.25
    torch.cuda.synchronize()
    ref = C.c_double()
    assert lib.bsp_dot(handle.h, n, x.data_ptr(), y.data_ptr(), C.byref(ref)) == 0
    scale = float((x[:n].abs() * y[:n].abs()).sum()) if n else 0.0
    stream = torch.cuda.current_stream()
    for _ in range(2):  # two calls in a row share the scratch
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.bsp_dot_noalloc(C.c_void_p(stream.cuda_stream), n, x.data_ptr(), y.data_ptr(),
                                 out.data_ptr())
        assert st == 0, lib.bsp_last_error(None)
        stream.synchronize()
        got = float(out.item())
        assert abs(got - ref.value) <= 1e-14 * max(scale, 1e-300) or (n == 0 and got == 0.0)


def test_noalloc_dot_rejects_size_beyond_scratch(lib, torch_cuda):
    torch = torch_cuda
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.bsp_dot_noalloc(C.c_void_p(torch.cuda.current_stream().cuda_stream), MAX_N + 1,
                             x.data_ptr(), x.data_ptr(), out.data_ptr())
    assert st == 8  # BSP_INVALID
    assert b"exceeds the maximum" in lib.bsp_last_error(None)
