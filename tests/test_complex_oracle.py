"""CPU checks of the complex (T = std::complex<double>) oracle and fixtures.

* the oracle (oracle/complex_oracle.py) against the reference itself, built
  with T = std::complex<double> (tests/golden/c_*.npz, made by
  tests/golden/make_golden_complex.py): bsmv and one preconditioner
  application within 1e-13 relative; pGMRES (with and without deflated
  restart, pure restart, SOR / Diag / no preconditioner) with the same
  iteration count, normalised residual history within 1e-12 absolute and the
  solution within 1e-12 relative;
* the real embedding used by the library (systems.complex_embedding) computes
  the complex block product.
"""
import json

import numpy as np
import pytest

from blocksp_b200 import systems
from oracle.blocksp_oracle import BSR
import oracle.complex_oracle as CO
from parity import GOLDEN, arg

APPLY = ["c_bsmv_3d_bs4", "c_ilu0_apply_3d_bs4", "c_sor_apply_2d_bs2", "c_diag_apply_3d_bs8"]
GMRES = ["c_ilu0_pgmres_3d_bs4", "c_ilu0_pgmres_dr_3d_bs4", "c_ilu0_pgmres_dr_3d_bs8", "c_sor_pgmres_dr_2d_bs2",
         "c_diag_pgmres_restart_2d_bs1", "c_nopre_pgmres_2d_bs2"]


def load_complex_golden(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(d["meta"]))
    s = systems.complex_system(tuple(meta["dims"]), meta["bs"], meta["seed"])
    return s, meta, d["x"], list(d["hist"]), int(d["iters"])


def oracle_pre(meta, Ao):
    w, nu, ty = arg(meta, "--w", 1.6), arg(meta, "--nu", 3), arg(meta, "--sortype", 0)
    sv = meta["solver"]
    if sv.startswith("ilu0"):
        return CO.ILU0(Ao)
    if sv.startswith("sor"):
        return CO.SOR(Ao, w, nu, ty)
    if sv.startswith("diag"):
        return CO.Diag(Ao)
    return CO.no_pre


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", APPLY)
def test_oracle_apply_matches_reference(name):
    s, meta, x, _, _ = load_complex_golden(name)
    Ao = BSR(s.n, s.bs, s.row_ptr, s.col_idx, s.vals)
    out = CO.bsmv(Ao, s.b) if meta["solver"] == "bsmv" else oracle_pre(meta, Ao)(s.b)
    assert rel(out, x) <= 1e-13


@pytest.mark.parametrize("name", GMRES)
def test_oracle_pgmres_matches_reference(name):
    s, meta, x, hist, iters = load_complex_golden(name)
    Ao = BSR(s.n, s.bs, s.row_ptr, s.col_idx, s.vals)
    res = CO.pgmres(Ao, s.b, arg(meta, "--tol", 1e-10), oracle_pre(meta, Ao), arg(meta, "--maxit", 500),
                    arg(meta, "--restart", -1), arg(meta, "--k", -1))
    assert res.iters == iters
    h, g = np.asarray(res.hist) / res.hist[0], np.asarray(hist) / hist[0]
    assert len(h) == len(g)
    assert np.abs(h - g).max() <= 1e-12
    assert rel(res.x, x) <= 1e-12


def test_embedding_is_the_complex_product():
    s = systems.complex_system((3, 3), 2, 5)
    Ao = BSR(s.n, s.bs, s.row_ptr, s.col_idx, s.vals)
    E = BSR(s.n, 2 * s.bs, s.row_ptr, s.col_idx, systems.complex_embedding(s.vals))
    x = np.random.default_rng(0).standard_normal(s.n * 2) + 1j * np.random.default_rng(1).standard_normal(s.n * 2)
    from oracle.blocksp_oracle import bsmv as real_bsmv
    y = real_bsmv(E, x.view(np.float64)).view(np.complex128)
    assert rel(y, CO.bsmv(Ao, x)) <= 1e-15
