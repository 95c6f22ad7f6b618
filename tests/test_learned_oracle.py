"""CPU checks of the learned-preconditioner specification (oracle/learned_oracle.py)
and of the convection-diffusion generator it trains on.

* the oracle's analytic gradients agree with central finite differences
  (relative error <= 1e-5 on sampled entries of every parameter);
* with zero decoders the network's correction is exactly zero (the initial
  preconditioner is block ILU0) and the loss is ILU0's;
* the relaxation scales exactly the off-diagonal factor blocks, and the
  gradients stay exact (finite differences) with it in place;
* the generator follows its stated conventions (velocity magnitude, harmonic
  edge conductivities, upwind blocks, SPD coupling, unit-variance field).
"""
import numpy as np

from blocksp_b200 import learned, systems
import oracle.blocksp_oracle as O
import oracle.learned_oracle as LO


def small_case(seed=7, dims=(4, 3, 3)):
    s = systems.convection_diffusion_system(dims, 8, seed)
    g = LO.graph_of(s.row_ptr, s.col_idx)
    F0 = O.ILU0(O.BSR.from_system(s)).LU.vals
    return s, g, F0


def test_oracle_gradients_match_finite_differences():
    s, g, F0 = small_case()
    rng = np.random.default_rng(1)
    p = LO.init_params(8, seed=3)
    for k in p:  # small decoders keep M = LU well conditioned
        p[k] = p[k] + (0.005 if k in ("Wo", "bo", "Wd", "bd") else 0.05) * rng.standard_normal(p[k].shape)
    Q = np.linalg.qr(rng.standard_normal((s.n * 8, 3)))[0].T
    _, gr = LO.loss_and_grads(p, g, s.vals, F0, Q)
    worst = 0.0
    for name in p:
        for _ in range(2):
            idx = tuple(int(rng.integers(0, d)) for d in p[name].shape)
            fd = LO.finite_difference(p, g, s.vals, F0, Q, name, idx, h=1e-5)
            an = gr[name][idx]
            worst = max(worst, abs(fd - an) / max(1e-8, abs(fd) + abs(an)))
    assert worst <= 1e-5, worst


def test_zero_decoders_give_ilu0():
    s, g, F0 = small_case()
    p = LO.init_params(8, seed=0)
    dF, _ = LO.forward(p, g, s.vals)
    assert not np.any(dF)
    rng = np.random.default_rng(2)
    Q = np.linalg.qr(rng.standard_normal((s.n * 8, 2)))[0].T
    loss, _ = LO.loss_and_factor_grad(g, s.vals, F0, Q)
    # ILU0's M^-1 A differs from I only through the dropped fill-in
    assert 0.0 < loss < 2.0


def test_host_parameter_layout_matches_oracle():
    assert learned.param_shapes(8) == LO.param_shapes(8)
    assert list(learned.param_shapes(8)) == list(LO.param_shapes(8))
    p = learned.init_params(8, seed=4)
    back = learned.unflatten(learned.flatten(p))
    assert all(np.array_equal(p[k], back[k]) for k in p)


def test_generator_conventions():
    dims = (5, 4, 3)
    sp = systems.convection_diffusion_spec(dims, 8, 11)
    assert abs(np.linalg.norm(sp.velocity) - 0.5) < 1e-15
    assert np.all(np.linalg.eigvalsh(sp.M) > 0.0)
    s = systems.convection_diffusion_system(dims, 8, 11, spec=sp)
    A = s.to_dense()
    nx, ny, _ = dims
    kap = sp.kappa
    # edge (p, q = p + 1) along x
    ke = 2.0 * kap[0] * kap[1] / (kap[0] + kap[1])
    c = sp.velocity[0]
    assert np.allclose(A[0:8, 8:16], -ke * sp.M - max(-c, 0.0) * np.eye(8), rtol=0, atol=1e-14)
    assert np.allclose(A[8:16, 0:8], -ke * sp.M - max(c, 0.0) * np.eye(8), rtol=0, atol=1e-14)
    # corner cell 0: one edge towards +axis per axis, plus the shift
    D = 0.01 * np.eye(8)
    for ax, q in enumerate((1, nx, nx * ny)):
        ke = 2.0 * kap[0] * kap[q] / (kap[0] + kap[q])
        D = D + ke * sp.M + max(-sp.velocity[ax], 0.0) * np.eye(8)
    assert np.allclose(A[:8, :8], D, rtol=0, atol=1e-12)


def test_gaussian_field_statistics():
    rng = systems.rng_for(5)
    f = systems.gaussian_field(rng, (64, 64, 16), 8.0).reshape(16, 64, 64)
    assert abs(f.std() - 1.0) < 0.35
    # correlation at lag 8 along x near exp(-1/2)
    a = (f * np.roll(f, 8, axis=2)).mean() / f.var()
    assert 0.3 < a < 0.9


# ---- the L L^T form (SPD systems, pCG) ----
def ichol0_in_a_order(s):
    """The block-IChol0 factor of s in A's block order (upper blocks zero)."""
    L = O.IChol0(O.BSR.from_system(s)).L
    F = np.zeros_like(s.vals)
    for i in range(s.n):
        lo = [t for t in range(s.row_ptr[i], s.row_ptr[i + 1]) if s.col_idx[t] <= i]
        F[lo] = L.vals[L.row_ptr[i]:L.row_ptr[i + 1]]
    return F


def small_spd_case(seed=9, dims=(4, 3, 3)):
    s = systems.convection_diffusion_system(dims, 8, seed, speed=0.0)
    return s, LO.graph_of(s.row_ptr, s.col_idx), ichol0_in_a_order(s)


def test_llt_oracle_gradients_match_finite_differences():
    s, g, F0 = small_spd_case()
    rng = np.random.default_rng(5)
    p = LO.init_params(8, seed=6)
    for k in p:
        p[k] = p[k] + (0.005 if k in ("Wo", "bo", "Wd", "bd") else 0.05) * rng.standard_normal(p[k].shape)
    Q = np.linalg.qr(rng.standard_normal((s.n * 8, 3)))[0].T
    _, gr = LO.loss_and_grads(p, g, s.vals, F0, Q, form="llt")
    worst = 0.0
    for name in p:
        for _ in range(2):
            idx = tuple(int(rng.integers(0, d)) for d in p[name].shape)
            fd = LO.finite_difference(p, g, s.vals, F0, Q, name, idx, h=1e-5, form="llt")
            an = gr[name][idx]
            worst = max(worst, abs(fd - an) / max(1e-8, abs(fd) + abs(an)))
    assert worst <= 1e-5, worst


def test_llt_form_keeps_the_factor_lower_and_spd():
    s, g, F0 = small_spd_case()
    rng = np.random.default_rng(8)
    p = LO.init_params(8, seed=2)
    p["Wd"] += 0.01 * rng.standard_normal(p["Wd"].shape)
    p["Wo"] += 0.01 * rng.standard_normal(p["Wo"].shape)
    dF, _ = LO.forward(p, g, s.vals, form="llt")
    rows = np.repeat(np.arange(s.n), np.diff(s.row_ptr))
    assert not np.any(dF[s.col_idx > rows])                        # no upper corrections
    assert not np.any(np.triu(dF[s.col_idx == rows], 1))           # triangular diagonal corrections
    Ld = LO.llt_dense(g, F0 + dF)
    assert np.all(np.linalg.eigvalsh(Ld @ Ld.T) > 0)
    # with zero decoders the factor is IChol0's: L L^T = the reference's IC(0)
    dF0, _ = LO.forward(LO.init_params(8, seed=2), g, s.vals, form="llt")
    assert not np.any(dF0)


# ---- the relaxation of the baseline factors ----

def test_relaxed_scales_off_diagonal_blocks_only():
    for s, g, F0 in (small_case(), small_spd_case()):
        rows = np.repeat(np.arange(s.n), np.diff(s.row_ptr))
        off = s.col_idx != rows
        R = LO.relaxed(g, F0, 0.35)
        assert np.array_equal(R[~off], F0[~off])
        assert np.array_equal(R[off], F0[off] * 1.35)
        assert np.array_equal(LO.relaxed(g, F0, 0.0), F0)
    # the L L^T factor stays lower: its upper blocks are zero before and after
    s, g, F0 = small_spd_case()
    rows = np.repeat(np.arange(s.n), np.diff(s.row_ptr))
    assert not np.any(LO.relaxed(g, F0, 0.5)[s.col_idx > rows])


def test_gradients_with_relaxation_match_finite_differences():
    rng = np.random.default_rng(12)
    for form, (s, g, F0) in (("lu", small_case()), ("llt", small_spd_case())):
        p = LO.init_params(8, seed=13)
        for k in p:
            p[k] = p[k] + (0.005 if k in ("Wo", "bo", "Wd", "bd") else 0.05) * rng.standard_normal(p[k].shape)
        Q = np.linalg.qr(rng.standard_normal((s.n * 8, 3)))[0].T
        _, gr = LO.loss_and_grads(p, g, s.vals, F0, Q, form=form, relax=0.4)
        worst = 0.0
        for name in p:
            idx = tuple(int(rng.integers(0, d)) for d in p[name].shape)
            fd = LO.finite_difference(p, g, s.vals, F0, Q, name, idx, h=1e-5, form=form, relax=0.4)
            an = gr[name][idx]
            worst = max(worst, abs(fd - an) / max(1e-8, abs(fd) + abs(an)))
        assert worst <= 1e-5, (form, worst)


def test_relaxation_choice_rule():
    # the committed L L^T fit: 0.7 has the fewest iterations but 0.8 fails
    # within the margin, so 0.65 is chosen
    table = {0.0: 891, 0.5: 469, 0.6: 398, 0.65: 374, 0.7: 372, 0.75: 428, 0.8: None}
    assert learned.choose_relax(table) == 0.65
    # without failures the minimum wins; ties go to the smaller value
    assert learned.choose_relax({0.0: 10, 0.1: 8, 0.2: 8, 0.3: 9}) == 0.1
    # everything failing but 0 -> 0; a fully failing table -> 0
    assert learned.choose_relax({0.0: 5, 0.05: None, 0.1: None}) == 0.0
    assert learned.choose_relax({0.0: None}) == 0.0
    # the committed weights record their own fit consistently
    import json
    import numpy as np
    for w in (learned.WEIGHTS, learned.WEIGHTS_LLT):
        meta = json.loads(str(np.load(w)["meta"]))
        tab = {float(k): v for k, v in meta["relax_fit"]["grid_total_iters"].items()}
        assert learned.choose_relax(tab) == meta["relax"]
