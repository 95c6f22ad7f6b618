"""Host-side logic on CPU: the synthetic system generators, the exchange
format read by the reference driver, and the learned model's parameter
packing.  No GPU is used."""
import numpy as np
import pytest

from blocksp_b200 import systems
from blocksp_b200 import learned


def _sym_part_min_eig(s):
    D = s.to_dense()
    return float(np.linalg.eigvalsh(0.5 * (D + D.T)).min()), D


def test_grid_system_structure_and_definiteness():
    dims, bs = (4, 3, 5), 8
    s = systems.grid_system(dims, bs, seed=7, skew=0.3)
    n = int(np.prod(dims))
    edges = sum(int(np.prod(dims)) // dims[a] * (dims[a] - 1) for a in range(3))
    assert s.n == n and s.nnzb == n + 2 * edges
    assert s.row_ptr[0] == 0 and s.row_ptr[-1] == s.nnzb
    # every block row holds its diagonal block exactly once
    rows = np.repeat(np.arange(n), np.diff(s.row_ptr))
    assert np.array_equal(np.sort(rows[s.col_idx == rows]), np.arange(n))
    lo, D = _sym_part_min_eig(s)
    assert lo > 0.0                       # symmetric part SPD
    assert np.abs(D - D.T).max() > 1e-3   # the skew term makes A nonsymmetric


def test_grid_system_without_skew_is_spd():
    s = systems.grid_system((6, 5), 4, seed=3)
    lo, D = _sym_part_min_eig(s)
    assert np.abs(D - D.T).max() == 0.0 and lo > 0.0


def test_generators_are_deterministic():
    a = systems.grid_system((3, 3, 3), 8, seed=11, skew=0.3)
    b = systems.grid_system((3, 3, 3), 8, seed=11, skew=0.3)
    c = systems.grid_system((3, 3, 3), 8, seed=12, skew=0.3)
    assert np.array_equal(a.vals, b.vals) and np.array_equal(a.b, b.b)
    assert not np.array_equal(a.vals, c.vals)


def test_convection_diffusion_system():
    dims, bs = (5, 4, 3), 8
    s0 = systems.convection_diffusion_system(dims, bs, seed=5, speed=0.0)
    lo, D0 = _sym_part_min_eig(s0)
    assert np.abs(D0 - D0.T).max() < 1e-12 and lo > 0.0   # pure diffusion: SPD
    s1 = systems.convection_diffusion_system(dims, bs, seed=5)
    lo1, D1 = _sym_part_min_eig(s1)
    assert np.abs(D1 - D1.T).max() > 1e-6 and lo1 > 0.0   # upwind convection: nonsymmetric
    # the velocity only enters through the upwind terms: same sparsity
    assert np.array_equal(s0.col_idx, s1.col_idx)


def test_batch_specs_ranges():
    sp = systems.batch_specs(seed=3, count=256)
    sides = np.array([x[0] for x in sp])
    assert len(sp) == 256 and sides.min() >= 32 and sides.max() <= 256
    assert set(x[1] for x in sp) == {4, 8}
    assert len({x[2] for x in sp}) == 256   # distinct seeds


def test_bsr_exchange_round_trip(tmp_path):
    s = systems.grid_system((3, 4), 4, seed=2, nrhs=2)
    f = tmp_path / "s.bsps"
    systems.write_bsr(f, s)
    t = systems.read_bsr(f)
    assert (t.n, t.bs, t.nnzb, t.nrhs) == (s.n, s.bs, s.nnzb, s.nrhs)
    for a, b in ((s.row_ptr, t.row_ptr), (s.col_idx, t.col_idx), (s.vals, t.vals), (s.b, t.b)):
        assert np.array_equal(np.asarray(a).ravel(), np.asarray(b).ravel())


@pytest.mark.parametrize("bs", [4, 8])
def test_learned_parameter_packing(bs):
    shapes = learned.param_shapes(bs)
    total = sum(int(np.prod(v)) for v in shapes.values())
    if bs == 8:
        assert total == 24992
    p = learned.init_params(bs, seed=1)
    flat = learned.flatten(p, bs)
    assert flat.shape == (total,)
    q = learned.unflatten(flat, bs)
    assert set(q) == set(shapes)
    for k in shapes:
        assert q[k].shape == tuple(shapes[k]) and np.array_equal(q[k], p[k])
    # the decoders start at zero, so the initial preconditioner is exactly ILU0
    assert not np.any(p["Wo"]) and not np.any(p["Wd"])
