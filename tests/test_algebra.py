"""Block algebra of the oracle against the reference (CPU).

The fixtures are the reference's own bsmm (A B and A^T B), bs_tr and
block_pseudo_heat operator I - delta A^T A (blocksp_multiply.hpp:21-159,
blocksp_tests.hpp:269-300) on seeded random block matrices, written by the
reference build (tests/golden/make_golden.py).  Structure (block order within
each row) must be identical; values within 1e-13 relative.
"""
import json

import numpy as np
import pytest

import oracle.blocksp_oracle as O
from blocksp_b200 import systems
from parity import GOLDEN

CASES = ["bsmm_rand_bs4", "bsmm_t_rand_bs4", "bs_tr_rand_bs4", "bsmm_t_rand_bs8"]


def load_case(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(d["meta"]))
    A = systems.random_blocksp(meta["m"], meta["bs"], meta["n_col"], meta["seed"])
    return d, meta, A


def oracle_result(meta, A):
    Ao = O.BSR.from_system(A)
    if meta["mode"] == "bs_tr":
        return O.bs_tr(Ao)
    return O.bsmm(Ao, Ao, meta["args"][1] == "1")


def check_same(got_rp, got_ci, got_vals, d, tol=1e-13):
    assert np.array_equal(got_rp, d["row_ptr"]) and np.array_equal(got_ci, d["col_idx"])
    ref = d["vals"]
    assert np.abs(np.asarray(got_vals) - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("name", CASES)
def test_oracle_block_algebra_vs_reference(name):
    d, meta, A = load_case(name)
    C = oracle_result(meta, A)
    check_same(C.row_ptr, C.col_idx, C.vals, d)


def pseudo_heat_oracle():
    d = np.load(GOLDEN / "pseudo_heat_bs32.npz")
    ph = json.loads(str(d["meta"]))
    A = systems.random_blocksp(ph["m"], ph["bs"], ph["n_col"], ph["seed"])
    Ao = O.BSR.from_system(A)
    S = O.matrix_add(1.0, O.bs_id(ph["m"], ph["bs"]), -ph["delta"], O.bsmm(Ao, Ao, True))
    return d, ph, A, S


def check_pseudo_heat(rp, ci, vals, d, tol=1e-13):
    assert np.array_equal(rp, d["row_ptr"]) and np.array_equal(ci, d["col_idx"])
    flat = np.asarray(vals).reshape(-1)
    sample = d["vals_sample"]
    assert np.abs(flat[d["vals_sample_idx"]] - sample).max() <= tol * np.abs(sample).max()
    assert abs(np.linalg.norm(flat) - float(d["vals_norm"])) <= tol * float(d["vals_norm"])


def test_oracle_pseudo_heat_operator_vs_reference():
    d, ph, A, S = pseudo_heat_oracle()
    check_pseudo_heat(S.row_ptr, S.col_idx, S.vals, d)


# ---- arnoldi_eigenvalues (blocksp_solvers.hpp:306-334) ----
EIG_CASES = ["arnoldi_eig_3d_bs8", "arnoldi_eig_harm_3d_bs8"]


def load_eig(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(d["meta"]))
    s = systems.grid_system(tuple(meta["dims"]), meta["bs"], seed=meta["seed"], skew=meta["skew"])
    return d["wr"] + 1j * d["wi"], meta, s


def match_eigs(got, ref, tol):
    """Every reference value has a computed value within tol * max |lambda| (and vice versa)."""
    got, ref = np.asarray(got), np.asarray(ref)
    assert len(got) == len(ref)
    scale = np.abs(ref).max()
    d1 = np.abs(got[:, None] - ref[None, :]).min(axis=0)
    d2 = np.abs(got[:, None] - ref[None, :]).min(axis=1)
    assert max(d1.max(), d2.max()) <= tol * scale, (d1.max(), d2.max())


@pytest.mark.parametrize("name", EIG_CASES)
def test_oracle_arnoldi_eigenvalues_vs_reference(name):
    ref, meta, s = load_eig(name)
    got = O.arnoldi_eigenvalues(O.BSR.from_system(s), meta["iters"], harmonic=bool(meta["harmonic"]))
    match_eigs(got, ref, 1e-9)
