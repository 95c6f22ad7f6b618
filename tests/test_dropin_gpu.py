"""The C++ drop-in header (include/blocksp_b200.hpp) against the reference.

oracle/_ref/dropin_test is one program that builds BlockSp<double,B*D> and
solArray<double,B,D> with the reference's own headers and solves with both
BlockSp::<solver> (the reference, CPU) and blocksp_b200::<solver> (this
library, GPU) — the same names, template arguments and call shapes — and
prints how far apart the answers are.  Criteria: bsmv <= 1e-14 relative;
solutions within 1e-8 relative; iteration counts within +-2 (the reference's
own printed counts, "pGMRES iters N" / "pCG iters N").  A complex system
(T = std::complex<double>) runs bsmv, ILU0_pGMRES(30, 10) and SOR_pGMRES with
the same criteria.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from blocksp_b200 import systems


pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "oracle" / "_ref" / "dropin_test"


def run(tmp_path, s, B, D, spd):
    if np.iscomplexobj(s.vals):
        f = tmp_path / "sys.bspc"
        systems.write_complex_bsr(f, s)
    else:
        f = tmp_path / "sys.bsps"
        systems.write_bsr(f, s)
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    if spd:
        env["DROPIN_SPD"] = "1"
    r = subprocess.run([str(EXE), str(f), str(B), str(D)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {}
    for line in r.stdout.splitlines():
        if line.startswith("CHECK "):
            _, name, d, it_ref, it_gpu = line.split()
            out[name] = (float(d), int(it_ref), int(it_gpu))
    return out


def test_dropin_binary_is_built():
    assert EXE.exists(), "build with __graft_entry__.build() (oracle/Makefile target _ref/dropin_test)"


def check_algebra(out):
    """bsmm / bs_tr / bs_id: same block order per row and values within 1e-13;
    Arnoldi Ritz values (12 steps) within 1e-8 of the reference's."""
    for name in ("bsmm", "bsmm_t", "bs_tr", "bs_id"):
        assert out[name][0] <= 1e-13, (name, out[name])
    d, n_ref, n_gpu = out["arnoldi_eig"]
    assert d <= 1e-8 and n_ref == n_gpu, out["arnoldi_eig"]


def test_dropin_spd_2d(tmp_path):
    out = run(tmp_path, systems.grid_system((12, 12), 4, seed=61), 2, 2, True)
    assert out["bsmv"][0] <= 1e-14
    check_algebra(out)
    for name in ("ilu0_pgmres_dr", "sor_pgmres", "ichol0_pcg", "sor_pcg"):
        d, ir, ig = out[name]
        assert d <= 1e-8 and abs(ir - ig) <= 2, (name, out[name])


def test_dropin_nonsymmetric_3d(tmp_path):
    out = run(tmp_path, systems.grid_system((6, 6, 6), 8, seed=62, skew=0.3), 4, 2, False)
    assert out["bsmv"][0] <= 1e-14
    check_algebra(out)
    for name in ("ilu0_pgmres_dr", "sor_pgmres"):
        d, ir, ig = out[name]
        assert d <= 1e-8 and abs(ir - ig) <= 2, (name, out[name])


@pytest.mark.parametrize("dims,B", [((6, 6, 6), 4), ((10, 10), 2)])
def test_dropin_complex(tmp_path, dims, B):
    out = run(tmp_path, systems.complex_system(dims, B, 63 + B), B, 1, False)
    assert out["c_bsmv"][0] <= 1e-14
    for name in ("c_ilu0_pgmres_dr", "c_sor_pgmres"):
        d, ir, ig = out[name]
        assert d <= 1e-8 and abs(ir - ig) <= 2, (name, out[name])
