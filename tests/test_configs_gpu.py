"""GPU against the reference at the full benchmark sizes.

The fixtures are the reference BlockSp v1.0 build's own solves of the three
full-size systems (tests/golden/make_golden.py, ``CONFIG_CASES``):

* 2D 64x64, 5-point, 4x4 blocks (4,096 block rows), IChol0_pCG(A, 1e-10, 2000);
* 3D 64^3, 7-point, 8x8 blocks, skew 0.3 (262,144 block rows, 1,810,432
  blocks), ILU0_pGMRES(A, 1e-10, 5000, 30, 10);
* 3D 48^3, 7-point, 16x16 blocks, skew 0.3 (110,592 block rows),
  ILU0_pGMRES(A, 1e-10, 5000, 30, 10).

At these sizes the sweep scheduler runs its full-size shape (4,096 chains in
256 super-tasks of 4 x 4 chains and 31 super-task levels per sweep at 64^3),
which the small fixtures do not reach.  Criteria as in tests/parity.py: iteration counts +-1 (+-2 with
deflated restart); pGMRES normalised residual history within 1e-10 absolute
at every step; pCG history within 1e-10 plus 10x the oracle's own rounding
envelope (stored in the fixture); solutions within 1e-8 relative (the whole x
for the 2D system; the norm and a fixed strided sample of x for the 3D ones).
"""
import json

import numpy as np
import pytest

from blocksp_b200 import systems
from parity import GOLDEN, check_history

pytestmark = pytest.mark.gpu


def load(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(d["meta"]))
    return d, meta, getattr(systems, meta["system"])()


def check_x(x, d):
    """x against the reference's solution: whole vector or norm + sample."""
    x = np.asarray(x)
    if "x" in d:
        ref = d["x"]
        assert np.abs(x - ref).max() / np.abs(ref).max() <= 1e-8
    idx, sample = d["x_sample_idx"], d["x_sample"]
    assert np.abs(x[idx] - sample).max() / np.abs(sample).max() <= 1e-8
    assert abs(np.linalg.norm(x) - float(d["x_norm"])) / float(d["x_norm"]) <= 1e-8


def test_cfg0_ichol0_pcg_vs_reference(handle):
    import blocksp_b200 as bsp
    d, meta, s = load("cfg0_ichol0_pcg_2d64_bs4")
    assert (s.n, s.bs) == (4096, 4)
    A = bsp.Matrix.from_system(s, handle)
    pc = bsp.IChol0(A)
    x, info, hist = bsp.pCG(A, s.b, 1e-10, pc, 2000, return_info=True)
    assert info["status"] == 0
    assert abs(info["iters"] - int(d["iters"])) <= 1, (info["iters"], int(d["iters"]))
    check_history(hist, list(d["hist"]), envelope=d["hist_envelope"])
    check_x(x, d)
    pc.close()
    A.close()


@pytest.mark.parametrize("name, n, bs", [("cfg1_ilu0_pgmres_dr_3d64_bs8", 262144, 8),
                                         ("cfg2b_ilu0_pgmres_dr_3d48_bs16", 110592, 16)])
def test_3d_ilu0_pgmres_dr_vs_reference(handle, name, n, bs):
    import blocksp_b200 as bsp
    d, meta, s = load(name)
    assert (s.n, s.bs) == (n, bs)
    A = bsp.Matrix.from_system(s, handle)
    pc = bsp.ILU0(A)
    x, info, hist = bsp.pGMRES(A, s.b, 1e-10, pc, 5000, 30, 10, return_info=True)
    assert info["status"] == 0
    assert abs(info["iters"] - int(d["iters"])) <= 2, (info["iters"], int(d["iters"]))
    check_history(hist, list(d["hist"]))
    check_x(x, d)
    pc.close()
    A.close()
