"""Failure detection on the GPU: the bounded device waits give up.

Every device-side wait of the sync-free factorisation and sweeps polls at most
the handle's spin limit before it records TIMEOUT (with the block row) and
returns, so the launch completes and the host reads the status; nothing
hangs or faults.  These tests set the limit to one re-poll on a 3D system
large enough that waits certainly occur (32^3 block rows, 8x8 blocks), check
that the call reports TIMEOUT, then restore the default limit and check that
the same handle still computes the oracle's result (the status word was
cleared and the context is intact).
"""
import numpy as np
import pytest

import oracle.blocksp_oracle as O
from blocksp_b200 import systems
from parity import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    return systems.grid_system((32, 32, 32), 8, seed=41, skew=0.3)


def _timeout(exc) -> bool:
    from blocksp_b200 import _lib
    return isinstance(exc, _lib.BspError) and exc.status == 6


def test_factorisation_wait_times_out(handle, system):
    import blocksp_b200 as bsp
    A = bsp.Matrix.from_system(system, handle)
    handle.set_spin_limit(1)
    try:
        with pytest.raises(Exception) as ei:
            bsp.ILU0(A)
        assert _timeout(ei.value), repr(ei.value)
        assert "block row" in str(ei.value)
    finally:
        handle.set_spin_limit()
    # the handle is still usable and the status word is clear
    pc = bsp.ILU0(A)
    z = pc.apply_host(system.b)
    assert np.isfinite(z).all()
    pc.close()
    A.close()


@pytest.mark.parametrize("kind", ["ILU0", "IChol0"])
def test_sweep_wait_times_out_then_recovers(handle, system, kind):
    import blocksp_b200 as bsp
    s = system if kind == "ILU0" else systems.grid_system((32, 32, 32), 8, seed=42)
    A = bsp.Matrix.from_system(s, handle)
    pc = getattr(bsp, kind)(A)
    handle.set_spin_limit(1)
    try:
        with pytest.raises(Exception) as ei:
            pc.apply_host(s.b)
        assert _timeout(ei.value), repr(ei.value)
    finally:
        handle.set_spin_limit()
    Ao = O.BSR.from_system(s)
    ref = (O.ILU0(Ao) if kind == "ILU0" else O.IChol0(Ao))(s.b.copy())
    assert rel(pc.apply_host(s.b), ref) <= 1e-11
    pc.close()
    A.close()


def test_spin_limit_rejects_zero(handle):
    from blocksp_b200 import _lib
    with pytest.raises(_lib.BspError):
        handle.set_spin_limit(0)
