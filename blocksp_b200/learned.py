"""Learned block preconditioner: host side of the network in learned.cu.

The network (a 3-layer message-passing network, hidden width 32, over the block
graph of A) is trained on the GPU by the library's own forward and backward
kernels; this module drives it: parameter I/O, probe generation, the training
loop, and the preconditioners it builds, in two factor forms:

* LU form (``LearnedLU``, pGMRES): corrects the block-ILU0 factors; falls back
  to block ILU0 when the model did not beat ILU0's iteration count on its
  held-out validation systems;
* L L^T form (``LearnedLLT``, pCG on SPD systems): corrects the block-IChol0
  factor; falls back to block IChol0 the same way.

Both forms first scale the baseline factors' off-diagonal blocks by 1 + relax,
a scalar of the model fitted to the training systems' iteration counts (a
compensation for the fill-in that the incomplete factorisation drops, in the
spirit of modified ILU), and add the network's correction to that.

No reference counterpart (the reference's preconditioners end at IChol0,
blocksp_preconditioners.hpp:364-538); the produced factors keep A's sparsity
and are applied by the same triangular sweeps as ILU0 (ILU0::invmul order).
"""
from __future__ import annotations

import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check
from .api import Handle, Matrix, Precond, _ptr, default_handle

LAYERS = 3
HIDDEN = 32
WEIGHTS = Path(__file__).resolve().parent / "weights" / "learned_convdiff_bs8.npz"
WEIGHTS_LLT = Path(__file__).resolve().parent / "weights" / "learned_diffusion_llt_bs8.npz"
FORMS = {"lu": _lib.LEARNED_LU, "llt": _lib.LEARNED_LLT}


def param_shapes(bs: int = 8, H: int = HIDDEN, layers: int = LAYERS) -> dict[str, tuple]:
    b2 = bs * bs
    shp = {"Wn": (H, b2 + 1), "bn": (H,), "We": (H, b2), "be": (H,)}
    for l in range(layers):
        shp.update({f"Wm{l}": (H, 2 * H), f"bm{l}": (H,), f"Wu{l}": (H, 2 * H), f"bu{l}": (H,)})
    shp.update({"Wo": (b2, 3 * H), "bo": (b2,), "Wd": (b2, H), "bd": (b2,)})
    return shp


def flatten(params: dict[str, np.ndarray], bs: int = 8) -> np.ndarray:
    return np.concatenate([np.asarray(params[k], dtype=np.float64).ravel() for k in param_shapes(bs)])


def unflatten(flat: np.ndarray, bs: int = 8) -> dict[str, np.ndarray]:
    out, off = {}, 0
    for k, s in param_shapes(bs).items():
        n = int(np.prod(s))
        out[k] = np.array(flat[off:off + n]).reshape(s)
        off += n
    return out


def init_params(bs: int = 8, seed: int = 0) -> dict[str, np.ndarray]:
    """He-scaled encoders and message layers; zero decoders, so the initial
    preconditioner is exactly block ILU0."""
    rng = np.random.default_rng(seed)
    out = {}
    for k, s in param_shapes(bs).items():
        if k.startswith("W") and k not in ("Wo", "Wd"):
            out[k] = rng.standard_normal(s) * np.sqrt(2.0 / s[1])
        else:
            out[k] = np.zeros(s)
    return out


class LearnedModel:
    """Device-resident network parameters with their Adam state."""

    def __init__(self, handle: Handle | None = None, bs: int = 8, dtype: int = _lib.BSP_F32,
                 params=None, meta: dict | None = None, form: str = "lu"):
        self.handle = handle or default_handle()
        self.bs = bs
        self.dtype = dtype
        self.form = form
        m = C.c_void_p()
        check(self.handle.lib.bsp_learned_create(self.handle.h, bs, dtype, C.byref(m)), "bsp_learned_create",
              self.handle.h)
        self.m = m
        self.handle.adopt(self)
        check(self.handle.lib.bsp_learned_set_form(self.m, FORMS[form]), "bsp_learned_set_form")
        cnt = C.c_int64()
        check(self.handle.lib.bsp_learned_param_count(self.m, C.byref(cnt)), "bsp_learned_param_count")
        self.n_params = cnt.value
        self.meta = dict(meta or {})
        self.set_params(params if params is not None else init_params(bs))
        self.set_relax(float(self.meta.get("relax", 0.0)))

    # -------------------------------------------------------------- parameters
    def set_params(self, params) -> None:
        flat = flatten(params, self.bs) if isinstance(params, dict) else np.asarray(params, dtype=np.float64)
        flat = np.ascontiguousarray(flat, dtype=np.float64)
        if flat.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {flat.size}")
        check(self.handle.lib.bsp_learned_set_params(self.m, _ptr(flat), flat.size), "bsp_learned_set_params")

    def set_relax(self, relax: float) -> None:
        """Scale the off-diagonal blocks of the baseline factors by 1 + relax
        before the network's correction is added (0 keeps them as they are)."""
        check(self.handle.lib.bsp_learned_set_relax(self.m, float(relax)), "bsp_learned_set_relax")

    @property
    def relax(self) -> float:
        r = C.c_double()
        check(self.handle.lib.bsp_learned_get_relax(self.m, C.byref(r)), "bsp_learned_get_relax")
        return r.value

    def params(self) -> dict[str, np.ndarray]:
        flat = np.zeros(self.n_params)
        check(self.handle.lib.bsp_learned_get_params(self.m, _ptr(flat), flat.size), "bsp_learned_get_params")
        return unflatten(flat, self.bs)

    def grads(self) -> dict[str, np.ndarray]:
        flat = np.zeros(self.n_params)
        check(self.handle.lib.bsp_learned_get_grads(self.m, _ptr(flat), flat.size), "bsp_learned_get_grads")
        return unflatten(flat, self.bs)

    def save(self, path: str | Path) -> None:
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, params=flatten(self.params(), self.bs), meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path: str | Path = WEIGHTS, handle: Handle | None = None, dtype: int = _lib.BSP_F32):
        d = np.load(path)
        meta = json.loads(str(d["meta"]))
        return cls(handle, int(meta.get("bs", 8)), dtype, params=d["params"], meta=meta,
                   form=meta.get("form", "lu"))

    # -------------------------------------------------------------- kernels
    def forward(self, A: Matrix):
        """dF (nnzb, bs, bs) in A's block order, as a device tensor."""
        import torch
        dF = torch.empty((A.nnzb, self.bs, self.bs), dtype=torch.float64, device="cuda")
        check(self.handle.lib.bsp_learned_forward(self.handle.h, self.m, A.m, _ptr(dF)), "bsp_learned_forward",
              self.handle.h)
        return dF

    def loss_grad(self, A: Matrix, ilu: Precond, probes) -> float:
        """loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2 for M = the ILU0 factors of
        ``ilu`` corrected by the network; keeps the parameter gradient."""
        loss = C.c_double()
        check(self.handle.lib.bsp_learned_loss_grad(self.handle.h, self.m, A.m, ilu.p, int(probes.shape[0]),
                                                    _ptr(probes), C.byref(loss)), "bsp_learned_loss_grad",
              self.handle.h)
        return loss.value

    def adam_step(self, lr: float = 1e-4, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        check(self.handle.lib.bsp_learned_adam_step(self.handle.h, self.m, lr, beta1, beta2, eps),
              "bsp_learned_adam_step", self.handle.h)

    def precond(self, A: Matrix, precision: int = _lib.PREC_F64) -> Precond:
        p = C.c_void_p()
        check(self.handle.lib.bsp_learned_precond(self.handle.h, self.m, A.m, precision, C.byref(p)),
              "bsp_learned_precond", self.handle.h)
        return Precond.wrap(A, p, _lib.PC_LEARNED_LLT if self.form == "llt" else _lib.PC_LEARNED_LU)

    def close(self) -> None:
        if getattr(self, "m", None):
            self.handle.lib.bsp_learned_destroy(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ilu_factors(A: Matrix, ilu: Precond):
    """Block-ILU0 factors in A's block order (device tensor, FP64)."""
    import torch
    F0 = torch.empty((A.nnzb, A.bs, A.bs), dtype=torch.float64, device="cuda")
    check(A.handle.lib.bsp_learned_ilu_factors(A.handle.h, ilu.p, _ptr(F0)), "bsp_learned_ilu_factors",
          A.handle.h)
    return F0


def probes(A: Matrix, pc: Precond | None, b, K: int):
    """K orthonormal Arnoldi vectors of M^-1 A started from M^-1 b (device)."""
    import torch
    bd = b if hasattr(b, "data_ptr") else torch.tensor(np.asarray(b, dtype=np.float64), device="cuda")
    Q = torch.empty((K, A.n_rows * A.bs), dtype=torch.float64, device="cuda")
    check(A.handle.lib.bsp_learned_probes(A.handle.h, A.m, pc.p if pc is not None else None, _ptr(bd), int(K),
                                          _ptr(Q)), "bsp_learned_probes", A.handle.h)
    return Q


def smooth_probes(A: Matrix, pc: Precond, K: int, steps: int, seed: int = 0):
    """K orthonormal smoothed error vectors: random vectors after `steps`
    iterations of e <- e - M^-1 A e (the slow modes of the preconditioned
    iteration, which dominate the Krylov solve's iteration count)."""
    import torch
    rng = np.random.default_rng(seed)
    V = torch.tensor(rng.standard_normal((K, A.n_rows * A.bs)), device="cuda")
    check(A.handle.lib.bsp_learned_smooth(A.handle.h, A.m, pc.p, int(K), int(steps), _ptr(V)),
          "bsp_learned_smooth", A.handle.h)
    return V


def training_probes(A: Matrix, ilu: Precond, b, n_arnoldi: int, n_smooth: int, smooth_steps: int, seed: int):
    """Probe set of a training step: Arnoldi vectors of the ILU0-preconditioned
    operator from M0^-1 b plus smoothed error vectors (each set orthonormal)."""
    import torch
    parts = []
    if n_arnoldi:
        parts.append(probes(A, ilu, b, n_arnoldi))
    if n_smooth:
        parts.append(smooth_probes(A, ilu, n_smooth, smooth_steps, seed))
    return torch.cat(parts).contiguous()


def LearnedLU(A: Matrix, model: LearnedModel | None, precision: int = _lib.PREC_F64) -> Precond:
    """The learned preconditioner, or block ILU0 when the model is absent or its
    validation showed no gain over ILU0's iteration count (the fallback)."""
    from .api import ILU0
    if model is None or model.form != "lu" or not model.meta.get("beats_ilu0", False):
        return ILU0(A, precision)
    return model.precond(A, precision)


def LearnedLLT(A: Matrix, model: LearnedModel | None, precision: int = _lib.PREC_F64) -> Precond:
    """The learned L L^T preconditioner for pCG on SPD systems, or block IChol0
    when the model is absent or its validation showed no gain over IChol0's
    iteration count (the fallback)."""
    from .api import IChol0
    if model is None or model.form != "llt" or not model.meta.get("beats_baseline", False):
        return IChol0(A, precision)
    return model.precond(A, precision)


# ------------------------------------------------------------------ training

def solve_iters(A: Matrix, b, pc, tol: float = 1e-10, restart: int = 30, k: int = 10,
                form: str = "lu") -> tuple[int, float]:
    """Iterations to the FP64 true residual tol, and that residual: pGMRES(restart,
    k) for the LU form, pCG for the L L^T form."""
    from .api import pCG, pGMRES
    if form == "llt":
        _, info, _ = pCG(A, b, tol, pc, 20000, return_info=True, stop_rule=_lib.STOP_TRUE_RESIDUAL)
    else:
        _, info, _ = pGMRES(A, b, tol, pc, 5000, restart, k, return_info=True, stop_rule=_lib.STOP_TRUE_RESIDUAL)
    return int(info["iters"]), float(info["true_rel_res"])


def training_system(dims, seed: int, form: str = "lu"):
    """A training / validation system: 3D convection-diffusion (LU form) or the
    same heterogeneous diffusion without convection, which is SPD (L L^T form)."""
    from . import systems
    return systems.convection_diffusion_system(dims, 8, int(seed), speed=0.0 if form == "llt" else 0.5)


RELAX_GRID = tuple(round(0.05 * i, 2) for i in range(17))  # 0, 0.05, ..., 0.8


def fit_relax(model: LearnedModel, seeds, dims, form: str = "lu", grid=RELAX_GRID, log=print,
              margin: float = 0.1):
    """Fit the model's relaxation to systems: the grid value with the fewest
    total solver iterations to the FP64 true residual 1e-10 (ties: the smaller
    value).  A value whose factors break down or miss 1e-10 on any system is
    out, and so is every value within ``margin`` below one that is out: the
    iteration count falls up to the point where the relaxed factors stop
    converging, and unseen systems may reach that point a little earlier.
    Leaves the model at the chosen value; returns it and the table."""
    h = model.handle
    table = {float(r): 0 for r in grid}
    for sd in seeds:
        sysm = training_system(dims, sd, form)
        A = Matrix.from_system(sysm, h)
        row = {}
        for r in grid:
            if table[float(r)] is None:
                continue
            model.set_relax(r)
            try:
                lp = model.precond(A)
            except _lib.BspError as e:
                if e.status not in (1, 2, 5):
                    raise
                table[float(r)] = None
                continue
            it, res = solve_iters(A, sysm.b, lp, form=form)
            lp.close()
            row[float(r)] = it
            table[float(r)] = table[float(r)] + it if res <= 1e-10 else None
        A.close()
        log(f"relaxation fit seed {sd}: " + " ".join(f"{r:g}:{it}" for r, it in row.items()))
    best = choose_relax(table, margin)
    model.set_relax(best)
    return best, table


def choose_relax(table: dict, margin: float = 0.1) -> float:
    """The fit's rule on a table {relax: total iterations, or None where some
    system broke down or missed the tolerance}: the value with the fewest
    iterations among those with no failing value in (relax, relax + margin];
    ties go to the smaller value; 0 when nothing qualifies."""
    bad = [r for r, t in table.items() if t is None]
    ok = {r: t for r, t in table.items() if t is not None and not any(r < q <= r + margin + 1e-9 for q in bad)}
    return min(ok, key=lambda r: (ok[r], r)) if ok else 0.0


def train(train_seeds, val_seeds, dims=(64, 64, 64), steps_per_system: int = 4, epochs: int = 1,
          n_probes: int = 16, lr: float = 1e-4, handle: Handle | None = None, seed: int = 0,
          n_smooth: int = 8, smooth_steps: int = 20, log=print, form: str = "lu", fit_seeds=(),
          relax_grid=RELAX_GRID) -> LearnedModel:
    """Train on convection-diffusion systems (LU form; SPD diffusion for the L L^T
    form) with the GPU kernels: first fit the relaxation of the baseline
    factors on ``fit_seeds`` (none: relaxation 0), then train the network with
    that relaxation in place, and keep the network only if it lowers the
    iteration count on the fit systems (else its decoders are zeroed); then
    validate against the baseline (ILU0 / IChol0) on held-out seeds, with the
    relaxation alone and with the whole model, and record whether the model
    beats the baseline's iteration count (the fallback gate)."""
    import torch
    from .api import IChol0, ILU0
    h = handle or default_handle()
    base = IChol0 if form == "llt" else ILU0
    model = LearnedModel(h, 8, _lib.BSP_F32, params=init_params(8, seed), form=form)
    t0 = time.time()
    relax, relax_table = 0.0, {}
    if len(fit_seeds):
        relax, relax_table = fit_relax(model, fit_seeds, dims, form, relax_grid, log)
        log(f"relaxation {relax:g} ({time.time() - t0:.0f}s)")
    history = []
    prev, reverts, lr0 = None, 0, lr
    for ep in range(epochs):
        for si, s in enumerate(train_seeds):
            sysm = training_system(dims, s, form)
            A = Matrix.from_system(sysm, h)
            ilu = base(A)
            Q = training_probes(A, ilu, torch.tensor(sysm.b, device="cuda"), n_probes - n_smooth, n_smooth,
                                smooth_steps, int(s))
            for _ in range(steps_per_system):
                # a step whose factors break down (zero pivot, not SPD, NaN)
                # is undone and the learning rate halved
                try:
                    loss = model.loss_grad(A, ilu, Q)
                    ok = np.isfinite(loss)
                except _lib.BspError as e:
                    if e.status not in (1, 2, 5):
                        raise
                    ok = False
                if not ok:
                    if prev is None:
                        raise RuntimeError("the initial factors break down")
                    model.set_params(prev)
                    lr *= 0.5
                    reverts += 1
                    continue
                prev = flatten(model.params(), 8)
                model.adam_step(lr)
                history.append(loss)
            ilu.close()
            A.close()
            if si % 20 == 0:
                log(f"epoch {ep} system {si} loss {history[-1]:.6e} ({time.time() - t0:.0f}s)")
    # the relaxation alone: zero decoders, so the network adds nothing
    relax_only = LearnedModel(h, 8, _lib.BSP_F32, params=init_params(8, seed), meta={"relax": relax}, form=form)
    # keep the network only if it lowers the iteration count on the fit systems
    # (training data); otherwise zero its decoders (the relaxation alone)
    network_fit = None
    if len(fit_seeds) and history:
        tot = [0, 0]
        for sd in fit_seeds:
            sysm = training_system(dims, sd, form)
            A = Matrix.from_system(sysm, h)
            for k, mm in enumerate((relax_only, model)):
                try:
                    pc = mm.precond(A)
                    it, res = solve_iters(A, sysm.b, pc, form=form)
                    pc.close()
                except _lib.BspError as e:
                    if e.status not in (1, 2, 5):
                        raise
                    it, res = 10**9, np.inf
                tot[k] += it if res <= 1e-10 else 10**9
            A.close()
        network_fit = {"relax_only_iters": tot[0], "with_network_iters": tot[1]}
        log(f"fit systems: relaxation only {tot[0]} iterations, with the network {tot[1]}")
        if tot[1] >= tot[0]:
            model.set_params(init_params(8, seed))
    network_used = network_fit is not None and network_fit["with_network_iters"] < network_fit["relax_only_iters"]
    val = []
    for s in val_seeds:
        sysm = training_system(dims, s, form)
        A = Matrix.from_system(sysm, h)
        ilu = base(A)
        it0, r0 = solve_iters(A, sysm.b, ilu, form=form)
        rp = relax_only.precond(A)
        itr, rr = solve_iters(A, sysm.b, rp, form=form)
        lp = model.precond(A)
        it1, r1 = solve_iters(A, sysm.b, lp, form=form)
        val.append({"seed": int(s), "ilu0_iters": it0, "learned_iters": it1, "ilu0_res": r0, "learned_res": r1,
                    "relax_only_iters": itr, "relax_only_res": rr})
        for o in (rp, lp, ilu, A):
            o.close()
        log(f"validation seed {s}: {base.__name__} {it0} iterations, relaxation only {itr}, learned {it1}")
    relax_only.close()
    beats = bool(val) and sum(v["learned_iters"] for v in val) < sum(v["ilu0_iters"] for v in val) and \
        all(v["learned_res"] <= 1e-10 for v in val)
    model.meta = {"bs": 8, "hidden": HIDDEN, "layers": LAYERS, "dims": list(dims), "form": form,
                  "baseline": base.__name__, "beats_baseline": beats, "relax": relax,
                  "relax_fit": {"seeds": [int(s) for s in fit_seeds], "grid_total_iters": relax_table},
                  "network_used": bool(network_used), "network_fit": network_fit,
                  "train_seeds": [int(s) for s in train_seeds], "val_seeds": [int(s) for s in val_seeds],
                  "steps_per_system": steps_per_system, "epochs": epochs, "n_probes": n_probes, "lr": lr0,
                  "lr_final": lr, "reverted_steps": reverts,
                  "n_smooth": n_smooth, "smooth_steps": smooth_steps,
                  "loss_first": history[0] if history else None, "loss_last": history[-1] if history else None,
                  "loss_history": history[:: max(1, len(history) // 200)], "validation": val,
                  "beats_ilu0": beats and form == "lu", "train_seconds": time.time() - t0}
    return model


if __name__ == "__main__":  # pragma: no cover - the training run itself
    import argparse
    ap = argparse.ArgumentParser(description="train the learned preconditioner on the GPU")
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--train", type=int, default=200)
    ap.add_argument("--val", type=int, default=4)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--probes", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-4)
    ap.add_argument("--smooth", type=int, default=8)
    ap.add_argument("--smooth-steps", type=int, default=20)
    ap.add_argument("--form", default="lu", choices=["lu", "llt"])
    ap.add_argument("--fit", type=int, default=4, help="systems the relaxation is fitted on")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    tr = [10_000 + i for i in range(a.train)]
    va = [20_000 + i for i in range(a.val)]
    fit = [15_000 + i for i in range(a.fit)]
    m = train(tr, va, (a.side,) * 3, a.steps, a.epochs, a.probes, a.lr, n_smooth=a.smooth,
              smooth_steps=a.smooth_steps, form=a.form, fit_seeds=fit)
    a.out = a.out or str(WEIGHTS_LLT if a.form == "llt" else WEIGHTS)
    m.save(a.out)
    print(json.dumps({k: v for k, v in m.meta.items() if k != "loss_history"}))
