"""MatrixMarket readers (host code of the library; no GPU needed).

The reference's LDG fixture (stored as arrays in tests/golden/ldg_2d_veclap.npz)
is written back out as .mtx files in the reference's layout (size line first,
symmetric lower triangle, 1-based) and read by the library's readers; the
result must equal the fixture's block matrix for every block size, and a
vector read with D > 1 must keep every value in place (the reference's reader
puts them all into dim 0, blocksp_tests.hpp:679).
"""
import numpy as np
import pytest

from blocksp_b200 import BspError
from blocksp_b200.mtx import mtxArray_to_solArray, mtxMatrix_to_BlockSp
from parity import GOLDEN, ldg_system


def write_ldg(tmp_path):
    d = np.load(GOLDEN / "ldg_2d_veclap.npz")
    n = int(d["n"])
    lines = [f"{n} {n} {len(d['vals'])}"]
    lines += [f"{int(i) + 1} {int(j) + 1} {float(v)!r}" for i, j, v in zip(d["rows"], d["cols"], d["vals"])]
    (tmp_path / "A.mtx").write_text("\n".join(lines) + "\n")
    (tmp_path / "b.mtx").write_text("\n".join([f"{n} 1"] + [repr(float(v)) for v in d["b"]]) + "\n")
    (tmp_path / "sol.mtx").write_text("\n".join([f"{n} 1"] + [repr(float(v)) for v in d["sol"]]) + "\n")
    return d


def as_blocks(s):
    out = {}
    for i in range(s.n):
        for t in range(s.row_ptr[i], s.row_ptr[i + 1]):
            out[(i, int(s.col_idx[t]))] = np.asarray(s.vals[t])
    return out


@pytest.mark.parametrize("B", [1, 2, 4, 8])
def test_ldg_matrix_roundtrip(tmp_path, B):
    write_ldg(tmp_path)
    got = mtxMatrix_to_BlockSp(tmp_path / "A.mtx", B, start_line=1, symmetric=True)
    ref, _, _ = ldg_system(B)
    assert (got.n, got.bs) == (ref.n, B)
    g, r = as_blocks(got), as_blocks(ref)
    assert g.keys() == r.keys()
    assert all(np.array_equal(g[k], r[k]) for k in r)


@pytest.mark.parametrize("B, D", [(1, 1), (4, 1), (4, 2), (2, 2), (1, 2)])
def test_vector_keeps_every_value_in_place(tmp_path, B, D):
    d = write_ldg(tmp_path)
    x = mtxArray_to_solArray(tmp_path / "b.mtx", B, D, start_line=1)
    assert np.array_equal(x, d["b"])


def test_first_appearance_order_base_zero_and_overwrite(tmp_path):
    # 4x4 with 2x2 blocks; entries listed so that block (0, 1) appears before (0, 0)
    (tmp_path / "m.mtx").write_text("% comment\n4 4 4\n0 3 1.5\n1 0 2.0\n0 3 2.5\n3 3 4.0\n")
    s = mtxMatrix_to_BlockSp(tmp_path / "m.mtx", 2, start_line=2, base_zero=True)
    assert s.n == 2 and list(s.row_ptr) == [0, 2, 3] and list(s.col_idx) == [1, 0, 1]
    assert s.vals[0][0, 1] == 2.5  # a repeated entry overwrites
    assert s.vals[1][1, 0] == 2.0 and s.vals[2][1, 1] == 4.0


def test_bad_block_size_and_missing_file(tmp_path):
    (tmp_path / "m.mtx").write_text("3 3 1\n1 1 1.0\n")
    with pytest.raises(BspError):
        mtxMatrix_to_BlockSp(tmp_path / "m.mtx", 2)
    with pytest.raises(BspError):
        mtxMatrix_to_BlockSp(tmp_path / "absent.mtx", 1)
    (tmp_path / "v.mtx").write_text("6 1\n" + "1\n" * 6)
    with pytest.raises(BspError):
        mtxArray_to_solArray(tmp_path / "v.mtx", 4, 1)
