"""Parity helpers shared by the CPU oracle tests and the GPU parity tests.

Criteria (FP64), as stated in the test modules:
  bsmv <= 1e-14 relative; one preconditioner application <= 1e-11; solutions
  <= 1e-8; iteration counts +-1 (+-2 with deflated restart); normalised
  residual histories <= 1e-10 absolute (pGMRES) or <= 1e-10 plus 10x the
  reference method's own rounding envelope (pCG, whose recursive residual is
  chaotic at rounding level).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from blocksp_b200 import systems
import oracle.blocksp_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel(a, b) -> float:
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def load_golden(name: str):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(d["meta"]))
    nrhs = meta["D"] if meta["solver"] == "bsmv_multi" else 1
    s = systems.grid_system(tuple(meta["dims"]), meta["bs"], seed=meta["seed"], skew=meta["skew"], nrhs=nrhs)
    return s, meta, d["x"], list(d["hist"]), int(d["iters"])


def arg(meta, key, default):
    a = meta["args"]
    return type(default)(a[a.index(key) + 1]) if key in a else default


def cg_spread(Ao, b, tol, pre, max_iters, ref, trials=3, eps=1e-15):
    """The oracle's pCG rerun with its matrix product and preconditioner output
    perturbed at rounding level (relative 1e-15): per-step spread of the
    normalised history, the iteration counts and the solutions' relative
    distance from the unperturbed run ``ref``."""
    r = np.asarray(ref.hist) / ref.hist[0]
    env = np.zeros(len(r))
    iters, xdev = [], []
    for t in range(trials):
        rng = np.random.default_rng(100 + t)

        def jitter(y):
            return y * (1.0 + eps * rng.standard_normal(y.shape))
        o = O.pcg(Ao, b, tol, lambda v: jitter(pre(v)), max_iters, matvec=lambda v: jitter(O.bsmv(Ao, v)))
        h = np.asarray(o.hist) / o.hist[0]
        n = min(len(h), len(r))
        env[:n] = np.maximum(env[:n], np.abs(h[:n] - r[:n]))
        if n < len(r):
            env[n:] = np.maximum(env[n:], r[n:])
        iters.append(o.iters)
        xdev.append(rel(o.x, ref.x))
    return env, iters, xdev


def cg_envelope(Ao, b, tol, pre, max_iters, ref_hist, trials=3, eps=1e-15):
    """Per-step spread of the oracle's normalised pCG history when its matrix
    product and preconditioner output are perturbed at rounding level."""
    class _Ref:
        hist = list(ref_hist)
        x = np.zeros_like(b)
    return cg_spread(Ao, b, tol, pre, max_iters, _Ref, trials, eps)[0]


def check_history(hist, ref_hist, h_tol=1e-10, envelope=None):
    h = np.asarray(hist) / hist[0]
    r = np.asarray(ref_hist) / ref_hist[0]
    n = min(len(h), len(r))
    assert n >= 2
    allowed = np.full(n, h_tol)
    if envelope is not None and len(envelope):
        run = np.maximum.accumulate(envelope)
        m = min(n, len(run))
        allowed[:m] += 10.0 * run[:m]
        allowed[m:] += 10.0 * run.max()
    dev = np.abs(h[:n] - r[:n])
    assert np.all(dev <= allowed), (int(np.argmax(dev - allowed)), float(dev.max()))


def ldg_system(B: int):
    """The reference's LDG fixture as a BlockSp<double, B> (symmetric fill,
    blocktests.hpp mtxMatrix_to_BlockSp with symmetric = true) and b, sol."""
    d = np.load(GOLDEN / "ldg_2d_veclap.npz")
    n = int(d["n"])
    r, c, v = d["rows"], d["cols"], d["vals"]
    off = r != c
    rr = np.concatenate([r, c[off]])
    cc = np.concatenate([c, r[off]])
    vv = np.concatenate([v, v[off]])
    nb = n // B
    br, bc = rr // B, cc // B
    key = br.astype(np.int64) * nb + bc
    uniq, inv = np.unique(key, return_inverse=True)
    vals = np.zeros((len(uniq), B, B))
    np.add.at(vals, (inv, rr % B, cc % B), vv)
    row_of = (uniq // nb).astype(np.int32)
    col_idx = (uniq % nb).astype(np.int32)
    row_ptr = np.zeros(nb + 1, np.int32)
    np.add.at(row_ptr, row_of + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    s = systems.BSRSystem(n=nb, bs=B, row_ptr=row_ptr, col_idx=col_idx, vals=vals, b=d["b"].copy(),
                          name=f"ldg_B{B}")
    return s, d["sol"].copy(), json.loads(str(d["ref_errinf"]))
