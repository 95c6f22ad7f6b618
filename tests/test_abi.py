"""The C ABI boundary without a GPU: the library loads, exports every entry point
declared in include/*.h, the ctypes table covers them, and compute calls fail
loudly (BSP_NO_DEVICE) instead of falling back to the CPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bsp_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "bsp_bsmv_dev" in names and "bsp_pgmres" in names and len(names) >= 25


def test_library_exports_every_declared_symbol():
    from blocksp_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared_functions() if getattr(lib, n, None) is None]
    assert not missing, f"declared but not exported: {missing}"


def test_ctypes_table_covers_header():
    from blocksp_b200 import _lib
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, f"no ctypes signature for: {missing}"


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible; the no-device path is tested on CPU hosts")
    from blocksp_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.bsp_handle_create(0, None, C.byref(h)) == 9  # BSP_NO_DEVICE
    assert b"no CPU fallback" in lib.bsp_last_error(None)
    cnt = C.c_int(-1)
    assert lib.bsp_device_count(C.byref(cnt)) == 9 and cnt.value == 0
    assert lib.bsp_abi_version() == 1
    assert lib.bsp_status_string(2) == b"block Cholesky met a non-positive pivot"


def test_python_mirror_raises_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import blocksp_b200 as bsp
    with pytest.raises(bsp.BspError):
        bsp.Handle(0)
