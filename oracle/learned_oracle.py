"""CPU oracle (numpy, FP64) of the learned block preconditioner's network.

TEST INFRASTRUCTURE ONLY: imported by tests/ to verify the GPU forward /
backward kernels; never part of the product path.

The reference has no learned component (it is new on this solve path); this
module is the specification the CUDA kernels implement, written as plainly as
possible, plus a finite-difference gradient check of the specification itself.

Model (message passing over the block graph of A: nodes = block rows, one
directed edge k = (i, j) per off-diagonal block A_ij, in CSR order):
    s_i   = sqrt(mean(A_ii * A_ii))                        node scale
    x_i   = [A_ii / s_i (bs*bs values), log s_i]            node input
    a_k   = A_ij / sqrt(s_i s_j)                            edge input
    h_i   = relu(Wn x_i + bn)                               node encoder
    e_k   = relu(We a_k + be)                               edge encoder
    L layers:  msg_k = relu(Wm [h_j; e_k] + bm)
               m_i   = sum over edges k of row i of msg_k   (CSR order)
               h_i  <- h_i + relu(Wu [h_i; m_i] + bu)
    dF_k  = alpha c_k (Wo [h_i; h_j; e_k] + bo)             off-diagonal block
    dF_ii = alpha s_i (Wd h_i + bd)                         diagonal block
with c_k = sqrt(s_i s_j) for an upper block (j > i, the scale of U_ij ~ A_ij)
and c_k = sqrt(s_i / s_j) for a lower block (j < i, the scale of
L_ij ~ A_ij U_jj^-1).
The preconditioner is M = L U with L = unit lower + strict-lower blocks and U
the upper blocks (diagonal included) of F = R(F_ILU0) + dF (A's pattern), where
R scales every off-diagonal block by 1 + relax (a fixed scalar of the model,
fitted to the training systems' iteration counts; 0 leaves F_ILU0 as it is).

Loss over orthonormal probe vectors q_1..q_K (Arnoldi vectors of the
ILU0-preconditioned operator, generated by the solver): the distance of the
left-preconditioned operator from the identity on them,
    loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2.
With z = M^-1 A q, g = (2/K)(z - q), w = U^-T g, lam = L^-T w, y = U z:
    d loss / d L_ij = -sum_k lam_k[i] y_k[j]^T  (strictly lower blocks)
    d loss / d U_ij = -sum_k   w_k[i] z_k[j]^T  (upper blocks)
Here written with dense matrices (small test systems only).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

ALPHA = 0.01


@dataclass
class Graph:
    n: int
    row_ptr: np.ndarray   # CSR of A (all blocks)
    col_idx: np.ndarray
    diag_pos: np.ndarray  # block index of A_ii per row
    e_blk: np.ndarray     # block index of each edge (off-diagonal blocks, CSR order)
    e_row: np.ndarray
    e_col: np.ndarray


def graph_of(row_ptr, col_idx) -> Graph:
    n = len(row_ptr) - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    blk = np.arange(len(col_idx))
    off = col_idx != rows
    diag_pos = np.zeros(n, dtype=np.int64)
    diag_pos[rows[~off]] = blk[~off]
    return Graph(n, np.asarray(row_ptr), np.asarray(col_idx), diag_pos, blk[off], rows[off],
                 np.asarray(col_idx)[off])


def param_shapes(bs: int, H: int = 32, L: int = 3) -> dict[str, tuple]:
    Fn, Fe, B2 = bs * bs + 1, bs * bs, bs * bs
    shp = {"Wn": (H, Fn), "bn": (H,), "We": (H, Fe), "be": (H,)}
    for l in range(L):
        shp[f"Wm{l}"] = (H, 2 * H)
        shp[f"bm{l}"] = (H,)
        shp[f"Wu{l}"] = (H, 2 * H)
        shp[f"bu{l}"] = (H,)
    shp.update({"Wo": (B2, 3 * H), "bo": (B2,), "Wd": (B2, H), "bd": (B2,)})
    return shp


def init_params(bs: int, seed: int = 0, H: int = 32, L: int = 3) -> dict[str, np.ndarray]:
    """He-style initial weights; the decoders start at zero so the initial
    preconditioner is exactly ILU0."""
    rng = np.random.default_rng(seed)
    out = {}
    for k, s in param_shapes(bs, H, L).items():
        if k.startswith("W") and k not in ("Wo", "Wd"):
            out[k] = rng.standard_normal(s) * np.sqrt(2.0 / s[1])
        else:
            out[k] = np.zeros(s)
    return out


def relu(x):
    return np.maximum(x, 0.0)


def features(g: Graph, vals: np.ndarray):
    bs = vals.shape[1]
    D = vals[g.diag_pos].reshape(g.n, bs * bs)
    s = np.sqrt(np.mean(D * D, axis=1))
    x = np.concatenate([D / s[:, None], np.log(s)[:, None]], axis=1)
    a = vals[g.e_blk].reshape(-1, bs * bs) / np.sqrt(s[g.e_row] * s[g.e_col])[:, None]
    return s, x, a


def forward(p: dict, g: Graph, vals: np.ndarray, L: int = 3, form: str = "lu"):
    """Returns dF (nnzb, bs, bs) in A's block order and the cache for backward.

    form "llt" (the L L^T variant for SPD systems): the output scales are
    alpha sqrt(s_i) for lower blocks (the scale of L_ij = A_ij L_jj^-T) and for
    the diagonal (L_ii ~ A_ii^1/2), upper blocks get no correction, and the
    diagonal correction is kept lower triangular."""
    bs = vals.shape[1]
    s, x, a = features(g, vals)
    h = relu(x @ p["Wn"].T + p["bn"])
    e = relu(a @ p["We"].T + p["be"])
    hs, msgs, ms, us = [h], [], [], []
    for l in range(L):
        msg = relu(np.concatenate([h[g.e_col], e], axis=1) @ p[f"Wm{l}"].T + p[f"bm{l}"])
        m = np.zeros_like(h)
        np.add.at(m, g.e_row, msg)
        u = relu(np.concatenate([h, m], axis=1) @ p[f"Wu{l}"].T + p[f"bu{l}"])
        h = h + u
        msgs.append(msg)
        ms.append(m)
        us.append(u)
        hs.append(h)
    si, sj = s[g.e_row], s[g.e_col]
    if form == "llt":
        se = ALPHA * np.where(g.e_col < g.e_row, np.sqrt(si), 0.0)
        sd = ALPHA * np.sqrt(s)
        dmask = np.tril(np.ones((bs, bs))).reshape(-1)
    else:
        se = ALPHA * np.where(g.e_col < g.e_row, np.sqrt(si / sj), np.sqrt(si * sj))
        sd = ALPHA * s
        dmask = np.ones(bs * bs)
    din = np.concatenate([h[g.e_row], h[g.e_col], e], axis=1)
    dF = np.zeros((len(g.col_idx), bs * bs))
    dF[g.e_blk] = se[:, None] * (din @ p["Wo"].T + p["bo"])
    dF[g.diag_pos] = sd[:, None] * (h @ p["Wd"].T + p["bd"]) * dmask
    cache = dict(s=s, x=x, a=a, e=e, hs=hs, msgs=msgs, ms=ms, us=us, se=se, sd=sd, dmask=dmask, din=din)
    return dF.reshape(-1, bs, bs), cache


def dense_of(g: Graph, blocks: np.ndarray) -> np.ndarray:
    n, bs = g.n, blocks.shape[1]
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    D = np.zeros((n * bs, n * bs))
    for b, (i, j) in enumerate(zip(rows, g.col_idx)):
        D[i * bs:(i + 1) * bs, j * bs:(j + 1) * bs] = blocks[b]
    return D


def lu_dense(g: Graph, F: np.ndarray):
    """L (unit lower, strict-lower blocks of F) and U (upper blocks of F)."""
    n, bs = g.n, F.shape[1]
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    lower = g.col_idx < rows
    Fl = np.where(lower[:, None, None], F, 0.0)
    Fu = np.where(lower[:, None, None], 0.0, F)
    return np.eye(n * bs) + dense_of(g, Fl), dense_of(g, Fu)


def loss_and_factor_grad(g: Graph, vals: np.ndarray, F: np.ndarray, Q: np.ndarray):
    """loss and d loss / d F (nnzb, bs, bs) for probes Q (K, n*bs)."""
    n, bs = g.n, vals.shape[1]
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    K = Q.shape[0]
    A = dense_of(g, vals)
    L, U = lu_dense(g, F)
    Z = np.linalg.solve(L @ U, A @ Q.T)          # (N, K)
    E = Z - Q.T
    loss = float(np.sum(E * E)) / K
    G = 2.0 * E / K
    W = np.linalg.solve(U.T, G)
    Lam = np.linalg.solve(L.T, W)
    Y = U @ Z
    gF = np.zeros_like(F)
    for b, (i, j) in enumerate(zip(rows, g.col_idx)):
        si, sj = slice(i * bs, (i + 1) * bs), slice(j * bs, (j + 1) * bs)
        if j < i:
            gF[b] = -Lam[si] @ Y[sj].T
        else:
            gF[b] = -W[si] @ Z[sj].T
    return loss, gF


def llt_dense(g: Graph, F: np.ndarray) -> np.ndarray:
    """L: the lower blocks of F (diagonal blocks lower triangular), dense."""
    n, bs = g.n, F.shape[1]
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    diag = g.col_idx == rows
    lower = g.col_idx < rows
    Fl = np.where(lower[:, None, None], F, 0.0) + np.where(diag[:, None, None], np.tril(F), 0.0)
    return dense_of(g, Fl)


def loss_and_factor_grad_llt(g: Graph, vals: np.ndarray, F: np.ndarray, Q: np.ndarray):
    """L L^T form: loss = (1/K) sum ||M^-1 A q - q||^2, M = L L^T, and d loss / d F
    (nnzb, bs, bs): with z = M^-1 A q, g = (2/K)(z - q), w = M^-1 g, y = L^T z,
    u = L^T w,  d loss / d L_ij = -(w_i y_j^T + z_i u_j^T) for j <= i (lower
    triangle of the diagonal blocks), zero for upper blocks."""
    n, bs = g.n, vals.shape[1]
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    K = Q.shape[0]
    A = dense_of(g, vals)
    Ld = llt_dense(g, F)
    M = Ld @ Ld.T
    Z = np.linalg.solve(M, A @ Q.T)
    E = Z - Q.T
    loss = float(np.sum(E * E)) / K
    W = np.linalg.solve(M, 2.0 * E / K)
    Y, U = Ld.T @ Z, Ld.T @ W
    gF = np.zeros_like(F)
    for b, (i, j) in enumerate(zip(rows, g.col_idx)):
        if j > i:
            continue
        si, sj = slice(i * bs, (i + 1) * bs), slice(j * bs, (j + 1) * bs)
        gb = -(W[si] @ Y[sj].T + Z[si] @ U[sj].T)
        gF[b] = np.tril(gb) if i == j else gb
    return loss, gF


def backward(p: dict, g: Graph, cache: dict, gdF: np.ndarray, L: int = 3) -> dict:
    """Parameter gradients given d loss / d dF (nnzb, bs, bs)."""
    B2 = gdF.shape[1] * gdF.shape[2]
    gdF = gdF.reshape(-1, B2)
    H = p["bn"].shape[0]
    s, x, a, e, hs = cache["s"], cache["x"], cache["a"], cache["e"], cache["hs"]
    grads = {}
    # decoders
    go = cache["se"][:, None] * gdF[g.e_blk]                 # (E, B2)
    grads["Wo"] = go.T @ cache["din"]
    grads["bo"] = go.sum(0)
    gdin = go @ p["Wo"]                                      # (E, 3H)
    gd = cache["sd"][:, None] * gdF[g.diag_pos] * cache["dmask"]  # (n, B2)
    grads["Wd"] = gd.T @ hs[-1]
    grads["bd"] = gd.sum(0)
    dh = gd @ p["Wd"]
    np.add.at(dh, g.e_row, gdin[:, :H])
    np.add.at(dh, g.e_col, gdin[:, H:2 * H])
    de = gdin[:, 2 * H:].copy()
    # message-passing layers, last first
    for l in reversed(range(L)):
        h_in, m, u, msg = hs[l], cache["ms"][l], cache["us"][l], cache["msgs"][l]
        gu = dh * (u > 0)
        grads[f"Wu{l}"] = gu.T @ np.concatenate([h_in, m], axis=1)
        grads[f"bu{l}"] = gu.sum(0)
        gin = gu @ p[f"Wu{l}"]
        dh_new = dh + gin[:, :H]
        dm = gin[:, H:]
        gpm = dm[g.e_row] * (msg > 0)
        grads[f"Wm{l}"] = gpm.T @ np.concatenate([h_in[g.e_col], e], axis=1)
        grads[f"bm{l}"] = gpm.sum(0)
        gmi = gpm @ p[f"Wm{l}"]
        np.add.at(dh_new, g.e_col, gmi[:, :H])
        de += gmi[:, H:]
        dh = dh_new
    ge = de * (e > 0)
    grads["We"] = ge.T @ a
    grads["be"] = ge.sum(0)
    gh = dh * (hs[0] > 0)
    grads["Wn"] = gh.T @ x
    grads["bn"] = gh.sum(0)
    return grads


def _factor_loss(form: str):
    return loss_and_factor_grad_llt if form == "llt" else loss_and_factor_grad


def relaxed(g: Graph, F0: np.ndarray, relax: float) -> np.ndarray:
    """The baseline factors with every off-diagonal block scaled by 1 + relax
    (the learned factors' relaxation; F0's upper blocks are zero in the L L^T
    form).  The learned factors are relaxed(F0) + dF."""
    F = F0 * (1.0 + relax)
    F[g.diag_pos] = F0[g.diag_pos]
    return F


def loss_fn(p: dict, g: Graph, vals: np.ndarray, F0: np.ndarray, Q: np.ndarray, L: int = 3,
            form: str = "lu", relax: float = 0.0) -> float:
    dF, _ = forward(p, g, vals, L, form)
    return _factor_loss(form)(g, vals, relaxed(g, F0, relax) + dF, Q)[0]


def loss_and_grads(p: dict, g: Graph, vals: np.ndarray, F0: np.ndarray, Q: np.ndarray, L: int = 3,
                   form: str = "lu", relax: float = 0.0):
    dF, cache = forward(p, g, vals, L, form)
    loss, gF = _factor_loss(form)(g, vals, relaxed(g, F0, relax) + dF, Q)
    return loss, backward(p, g, cache, gF, L)


def finite_difference(p: dict, g: Graph, vals, F0, Q, name: str, idx: tuple, h: float = 1e-6,
                      L: int = 3, form: str = "lu", relax: float = 0.0) -> float:
    """Central difference of the loss in one parameter entry."""
    q = {k: v.copy() for k, v in p.items()}
    q[name][idx] += h
    lp = loss_fn(q, g, vals, F0, Q, L, form, relax)
    q[name][idx] -= 2 * h
    lm = loss_fn(q, g, vals, F0, Q, L, form, relax)
    return (lp - lm) / (2 * h)
