"""Benchmark of the BlockSp B200 solve path.

Workload (one GPU, the configuration the headline metric is quoted on): the 3D
64^3 7-point block stencil with 8x8 blocks (262,144 block rows, 1,810,432
blocks, nonsymmetric), solved by pGMRES(30) with deflated restart k = 10 and
block ILU0 — the plain GPU drop-in of ILU0_pGMRES — until the FP64 true
relative residual ||b - A x|| / ||b|| <= 1e-10.  A "step" is one complete
solve: ILU0 set-up on the device plus the refined pGMRES solve, timed with CUDA
events on the solver's stream.  Variants measured per step: plain FP64 and the
mixed-precision inner operator (FP32 storage of A and of the ILU0 factors,
FP64 vectors, FP64 refinement); ``value`` is the faster one (both reach the
same FP64 true residual).  The standalone bsmv and one ILU0 application of the
same matrix are timed too and carry the roofline.

``--impl reference`` times the reference's own CPU implementation of the path
on this host instead (the reference library compiled from its headers by
oracle/Makefile; single-threaded by construction).  Multi-GPU: the path does
not shard (replicas only): ``--gpus N`` runs N independent replicas, one per
rank, and reports the max-over-ranks time with ``value`` = N solves / time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time-to-1e-10 FP64 residual: learned/mixed vs plain GPU Krylov; bsmv HBM GB/s"
FALLBACK_HBM_GBS = 6650.0
TOL = 1e-10
GOLDEN = ROOT / "tests" / "golden"
# ncu DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one ILU0
# application at 64^3 with 8x8 FP64 blocks (its two streamed sweeps), from the
# committed capture summarised in profiles/sweep_stream_ilu0_64cube_bs8.md
ILU_APPLY_TRAFFIC_64 = 1_013_952_512  # 439.6 MB forward + 574.3 MB backward


def reference_golden(side: int) -> dict | None:
    """The reference's own solve of the default system (seed 1, side^3):
    ILU0_pGMRES(A, 1e-10, 5000, 30, 10) run to completion by the reference
    build, stored as a test fixture (iterations and residual history)."""
    f = GOLDEN / "cfg1_ilu0_pgmres_dr_3d64_bs8.npz"
    if side != 64 or not f.exists():
        return None
    d = np.load(f)
    return {"iters": int(d["iters"]), "hist": d["hist"]}


def read_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.out.flush()
        rows = []
        for line in Path(self.out.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        loaded = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def dist_setup(backend: str = "nccl"):
    """Process group of a torchrun launch (one rank per GPU).  The path does
    not shard, so the group only carries the barrier and the max-over-ranks
    timing; ``gloo`` runs the same host logic without GPUs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def pinned_copy(a: np.ndarray) -> np.ndarray:
    """numpy view of a page-locked host copy of a (host<->device copies from
    pinned memory run at link speed and do not stage through a bounce buffer)."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def bsmv_bytes(n: int, bs: int, nnzb: int, nrhs: int = 1, val_bytes: int = 8, vec_bytes: int = 8) -> int:
    """Algorithmic bytes of y = A x: blocks + indices + x read once + y written."""
    return nnzb * bs * bs * val_bytes + nnzb * 4 + (n + 1) * 4 + 2 * n * bs * nrhs * vec_bytes


def ilu_apply_bytes(n: int, bs: int, nnzb: int, val_bytes: int = 8) -> int:
    """Algorithmic bytes of one ILU0 application (forward + backward sweep):
    the strictly-lower blocks (forward) and strictly-upper blocks plus the
    inverted diagonal blocks (backward) once each (the diagonal U blocks are
    not read: their inverses replace them), one column index per strict
    block, a row pointer per row and sweep, and in each sweep the right-hand
    side read and the result written."""
    strict = nnzb - n
    return (strict + n) * bs * bs * val_bytes + strict * 4 + 2 * (n + 1) * 4 + 4 * n * bs * 8


# --------------------------------------------------------------------- GPU arm

def target_comparison(results: dict) -> dict | None:
    """The target comparison: the learned (with its ILU0 fallback) mixed-precision
    solver against plain FP64 ILU0-pGMRES on the same system, wall time to the
    FP64 true residual."""
    from blocksp_b200 import learned
    if "plain_f64" not in results or "learned_mixed_f32" not in results:
        return None
    meta = json.loads(str(np.load(learned.WEIGHTS)["meta"])) if learned.WEIGHTS.exists() else {}
    plain, lm = results["plain_f64"]["total_s"], results["learned_mixed_f32"]["total_s"]
    return {"plain_f64_s": plain, "learned_mixed_f32_s": lm, "speedup": plain / lm,
            "plain_f64_iters": results["plain_f64"]["iters"],
            "learned_mixed_f32_iters": results["learned_mixed_f32"]["iters"],
            "learned_gate_open": meta.get("beats_ilu0"), "learned_relax": meta.get("relax"),
            "learned_network_used": meta.get("network_used"),
            "preconditioner_used": results["learned_mixed_f32"].get("preconditioner")}


def pc_name(pc) -> str:
    from blocksp_b200 import _lib
    return {_lib.PC_ILU0: "ILU0", _lib.PC_LEARNED_LU: "learned LU"}.get(pc.kind, str(pc.kind))


def run_gpu(args, world, rank, local):
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, systems

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    h = bsp.Handle(local, stream=stream.cuda_stream)
    lib = _lib.load()
    sysm = systems.config1(seed=1 + rank, side=args.side)
    n, bs, nnzb = sysm.n, sysm.bs, sysm.nnzb
    A = bsp.Matrix.from_system(sysm, h)
    b = torch.tensor(sysm.b, device="cuda")
    y = torch.empty_like(b)
    peak, peak_kind = read_peaks()

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    # the learned preconditioner with its ILU0 fallback (the committed model's
    # own validation decides which one runs)
    from blocksp_b200 import learned
    model = learned.LearnedModel.load(handle=h) if learned.WEIGHTS.exists() else None
    makers = {"plain_f64": (lambda: bsp.ILU0(A), _lib.PREC_F64),
              "mixed_f32": (lambda: bsp.ILU0(A), _lib.PREC_F32),
              "learned_mixed_f32": (lambda: learned.LearnedLU(A, model), _lib.PREC_F32)}

    # ---- one solve: preconditioner set-up + refined pGMRES-DR to the true residual ----
    def solve_once(name):
        make_pc, precision = makers[name]
        e0 = ev()
        pc = make_pc()
        e1 = ev()
        x, info, hist = bsp.pGMRES(A, b, TOL, pc, 5000, 30, 10, return_info=True,
                                   stop_rule=_lib.STOP_TRUE_RESIDUAL, precision=precision,
                                   inner_tol=1e-6)
        e2 = ev()
        e2.synchronize()
        pc.close()
        return {"setup_s": e0.elapsed_time(e1) / 1e3, "solve_s": e1.elapsed_time(e2) / 1e3,
                "total_s": e0.elapsed_time(e2) / 1e3, "iters": info["iters"], "preconditioner": pc_name(pc),
                "refinements": info["n_outer"], "restarts": info["n_restarts"],
                "true_rel_res": info["true_rel_res"], "status": info["status"]}

    # parity run (untimed): the reference's method and stopping rule, whose
    # residual history is compared with the reference's own solve of this system
    pc = bsp.ILU0(A)
    _, pinfo, phist = bsp.pGMRES(A, b, TOL, pc, 5000, 30, 10, return_info=True)
    pc.close()
    variants = {k: makers[k][1] for k in args.variants.split(",") if k in makers}
    results = {}
    launches = 0
    with ClockSampler(local) as clk:
        for name in variants:
            for _ in range(max(args.warmup, 3)):
                solve_once(name)
            torch.cuda.synchronize()
            barrier(world)
            l0 = lib.bsp_launch_count()
            steps = [solve_once(name) for _ in range(args.steps)]
            launches += lib.bsp_launch_count() - l0
            tot = max_over_ranks(statistics.mean(s["total_s"] for s in steps), world)
            results[name] = {**steps[-1], "total_s": tot,
                             "setup_s": statistics.mean(s["setup_s"] for s in steps),
                             "solve_s": statistics.mean(s["solve_s"] for s in steps)}

        # ---- standalone bsmv and ILU0 apply (roofline legs) ----
        for _ in range(3):
            bsp.bsmv_dev(A, b, y)
        torch.cuda.synchronize()
        e0 = ev()
        for _ in range(args.bsmv_reps):
            bsp.bsmv_dev(A, b, y)
        e1 = ev()
        e1.synchronize()
        bsmv_ms = max_over_ranks(e0.elapsed_time(e1) / args.bsmv_reps, world)
        pc = bsp.ILU0(A)
        z = b.clone()
        for _ in range(3):
            pc(z)
        torch.cuda.synchronize()
        reps = max(5, args.bsmv_reps // 5)
        e0 = ev()
        for _ in range(reps):
            pc(z)
        e1 = ev()
        e1.synchronize()
        ilu_ms = max_over_ranks(e0.elapsed_time(e1) / reps, world)
        levels = pc.info()
        pc.close()
    clocks = clk.summary()

    # ---- e2e: the drop-in call with host buffers (matrix, b in; x out) ----
    best = min(results, key=lambda k: results[k]["total_s"])
    xh = np.zeros_like(sysm.b)
    if args.no_e2e:
        if model is not None:
            model.close()
        A.close()
        h.close()
        return {"n": n, "bs": bs, "nnzb": nnzb, "results": results, "best": best, "e2e_s": float("nan"),
                "bsmv_ms": bsmv_ms, "ilu_ms": ilu_ms, "levels": levels, "peak": peak,
                "peak_kind": peak_kind, "clocks": clocks, "launches": launches, "x_norm": 0.0,
                "hist_f64": list(phist), "iters_f64": pinfo["iters"]}
    # Inputs in pinned host memory (numpy views of page-locked tensors); one
    # untimed call, then the mean over the timed calls.  Each call uploads the
    # matrix and right-hand side, builds ILU0, solves and reads x back.
    rp_h, ci_h, va_h, b_h = (
        pinned_copy(a) for a in (sysm.row_ptr.astype(np.int32), sysm.col_idx.astype(np.int32), sysm.vals, sysm.b))

    parts = {"matrix_create_s": 0.0, "precond_create_s": 0.0, "solve_s": 0.0, "release_s": 0.0}

    def e2e_call():
        t = [time.perf_counter()]
        A2 = bsp.Matrix(rp_h, ci_h, va_h, bs, handle=h)
        t.append(time.perf_counter())
        pc2 = learned.LearnedLU(A2, model) if best == "learned_mixed_f32" else bsp.ILU0(A2)
        t.append(time.perf_counter())
        out = bsp.pGMRES(A2, b_h, TOL, pc2, 5000, 30, 10, stop_rule=_lib.STOP_TRUE_RESIDUAL,
                         precision=variants[best])
        t.append(time.perf_counter())
        pc2.close()
        A2.close()
        t.append(time.perf_counter())
        for k, key in enumerate(parts):
            parts[key] += t[k + 1] - t[k]
        return out

    e2e_call()
    for key in parts:
        parts[key] = 0.0
    e2e_steps = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        xh = e2e_call()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, world)
    e2e_parts = {k: v / e2e_steps for k, v in parts.items()}
    if model is not None:
        model.close()
    A.close()
    h.close()
    return {
        "n": n, "bs": bs, "nnzb": nnzb, "results": results, "best": best, "e2e_s": e2e_s,
        "bsmv_ms": bsmv_ms, "ilu_ms": ilu_ms, "levels": levels, "peak": peak, "peak_kind": peak_kind,
        "clocks": clocks, "launches": launches, "x_norm": float(np.linalg.norm(xh)),
        "hist_f64": list(phist), "iters_f64": pinfo["iters"], "e2e_parts": e2e_parts,
    }


# --------------------------------------------------------------------- CPU arms

def ref_binary() -> Path | None:
    p = ROOT / "oracle" / "_ref" / "ref_solve"
    return p if p.exists() else None


def cpu_reference_full(side: int, runs: int = 1, budget_s: float = 150.0) -> dict | None:
    """The reference's CPU ILU0_pGMRES(A, 1e-10, 5000, 30, 10) on the same
    system, run to completion by the reference build (its own set-up and
    solve timers): at least one full run, more while the budget lasts, up to
    `runs`.  Returns the mean set-up, solve and total seconds, the iteration
    count and the number of runs."""
    exe = ref_binary()
    if exe is None:
        return None
    from blocksp_b200 import systems
    s = systems.config1(seed=1, side=side)
    done = []
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "sys.bsps"
        systems.write_bsr(f, s)
        cmd = [str(exe), str(f), "--B", "4", "--D", "2", "--solver", "ilu0_pgmres", "--tol", "1e-10",
               "--maxit", "5000", "--restart", "30", "--k", "10", "--time", "--print-iters"]
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        t_start = time.time()
        while len(done) < max(1, runs):
            r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
            out = {}
            for line in r.stdout.splitlines():
                if line.startswith("TIME "):
                    k, v = line.split()[1:3]
                    out[k] = float(v)
                elif line.startswith("pGMRES iters"):
                    out["iters"] = int(line.split()[2])
            if "setup_s" not in out or "solve_s" not in out:
                break
            done.append(out)
            per = (time.time() - t_start) / len(done)
            if time.time() - t_start + per > budget_s:
                break
    if not done:
        return None
    mean = lambda k: float(np.mean([o[k] for o in done]))  # noqa: E731
    return {"setup_s": mean("setup_s"), "solve_s": mean("solve_s"), "total_s": mean("setup_s") + mean("solve_s"),
            "iters": done[-1].get("iters"), "runs": len(done)}


# ----------------------------------------------------------------- batch workload

BATCH_METRIC = "batched pCG+IChol0: time to FP64 relative residual 1e-10 for every system x RHS"


def batch_bytes_per_iter(n: int, bs: int, nnzb: int, R: int) -> int:
    """Algorithmic bytes of one batched pCG iteration of one system: A's blocks
    and indices once (spmv), the strictly-lower IChol0 blocks and inverted
    diagonals twice (forward and backward sweep), and 19 passes over an
    n x R x bs vector (spmv 2, update 8 incl. sentinel refills, sweeps 4,
    r.z 2, p update 3)."""
    b2 = bs * bs * 8
    lower = (nnzb - n) // 2
    return nnzb * b2 + nnzb * 4 + (n + 1) * 4 + 2 * (lower * b2 + n * b2 + lower * 8) + 19 * n * R * bs * 8


def batch_cpu_sample(specs, iters, budget_s: float = 25.0) -> dict | None:
    """The reference's IChol0_pCG (one call per system per RHS, D = 1) timed on
    a bounded sample of the batch's systems: the smallest systems of each block
    size, first right-hand side; returns the per-(row x iteration) solve cost
    and per-row set-up cost per block size."""
    exe = ref_binary()
    if exe is None:
        return None
    from blocksp_b200 import systems
    out = {}
    spent = 0.0
    for bs in (4, 8):
        cand = sorted((side, i) for i, (side, b, _) in enumerate(specs) if b == bs)[:2]
        costs, setups = [], []
        for side, i in cand:
            if spent > budget_s:
                break
            s = systems.batch_system(side, bs, specs[i][2], nrhs=1)
            with tempfile.TemporaryDirectory() as d:
                f = Path(d) / "sys.bsps"
                systems.write_bsr(f, s)
                cmd = [str(exe), str(f), "--B", str(bs), "--D", "1", "--solver", "ichol0_pcg", "--tol", "1e-10",
                       "--maxit", "2000", "--time"]
                env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
                t0 = time.time()
                r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=600)
                spent += time.time() - t0
            tm = {ln.split()[1]: float(ln.split()[2]) for ln in r.stdout.splitlines() if ln.startswith("TIME ")}
            if "solve_s" not in tm:
                continue
            it = int(iters[i][0]) + 1
            costs.append(tm["solve_s"] / (s.n * it))
            setups.append(tm["setup_s"] / s.n)
        if costs:
            out[bs] = {"solve_per_row_iter_s": float(np.mean(costs)), "setup_per_row_s": float(np.mean(setups)),
                       "systems": len(costs)}
    return out or None


def run_batch(args):
    print(json.dumps(batch_measure(args, args.steps, max(args.warmup, 3), not args.no_cpu_baseline)), flush=True)


def batch_summary(args) -> dict:
    """cfg3 inside the default line: one warm-up and one timed batched solve
    (the standalone `--workload batch` run is the full measurement)."""
    line = batch_measure(args, 1, 1, False)
    it = line["iterations"]
    return {"metric": line["metric"], "value": line["value"], "unit": "s", "steps": 1, "warmup": 1,
            "systems": line["config"]["systems"], "rhs": line["config"]["rhs"],
            "iterations_max": it["max"], "converged_pairs": it["converged_pairs"], "pairs": it["pairs"],
            "achieved_gbs": line["roofline"]["achieved"], "frac_of_peak": line["roofline"]["frac"],
            "e2e_s": line["e2e"]["value"], "gpu_launches": line["gpu_launches"],
            "launch": "one CUDA graph launch per solve; its device-side while node replays one pCG "
                      "iteration of every block-size group (several kernels) until every pair converges"}


def batch_measure(args, steps: int, warmup: int, with_cpu: bool) -> dict:
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, systems

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    lib = _lib.load()
    specs = systems.batch_specs(seed=3, count=args.batch_count)
    R = 4
    t0 = time.time()
    sl = [systems.batch_system(side, bs, seed, nrhs=R) for side, bs, seed in specs]
    gen_s = time.time() - t0
    t0 = time.time()
    B = bsp.Batch(sl, h)
    create_s = time.time() - t0
    bh = pinned_copy(np.concatenate([s.b for s in sl]))
    bd = torch.tensor(bh, device="cuda")
    peak, peak_kind = read_peaks()

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    first = None
    for _ in range(warmup):
        x, info = B.pcg(bd, R, TOL, 2000)
        first = first or info
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        l0 = lib.bsp_launch_count()
        e0 = ev()
        for _ in range(steps):
            x, info = B.pcg(bd, R, TOL, 2000)
        e1 = ev()
        e1.synchronize()
        launches = lib.bsp_launch_count() - l0
    clocks = clk.summary()
    solve_s = e0.elapsed_time(e1) / 1e3 / steps
    res = B.results()
    # algorithmic bytes: every system active for (its slowest pair's iterations + 1)
    total_bytes = 0
    for i, s in enumerate(sl):
        total_bytes += batch_bytes_per_iter(s.n, s.bs, s.nnzb, R) * (int(res["iters"][i].max()) + 1)
    gbs = total_bytes / solve_s / 1e9
    # e2e through the host-buffer entry point
    t0 = time.perf_counter()
    xh, _ = B.pcg(bh, R, TOL, 2000)
    e2e_s = time.perf_counter() - t0
    tun = B.tuning()
    cpu = None
    if with_cpu:
        cs = batch_cpu_sample(specs, res["iters"])
        if cs is not None and all(bs in cs for bs in (4, 8)):
            est = 0.0
            for i, s in enumerate(sl):
                c = cs[s.bs]
                est += c["setup_per_row_s"] * s.n + c["solve_per_row_iter_s"] * s.n * float(
                    np.sum(res["iters"][i] + 1))
            cpu = {"value": est, "unit": "s", "cores": 1, "cores_available": os.cpu_count() or 1,
                   "kind": "reference",
                   "sample": "reference IChol0_pCG<T,bs,1> on the two smallest systems of each block size "
                             f"(first RHS), per-row-iteration cost {cs[4]['solve_per_row_iter_s']:.3e} s (bs 4) / "
                             f"{cs[8]['solve_per_row_iter_s']:.3e} s (bs 8), extrapolated over all "
                             f"{len(sl)} systems x {R} RHS with the iteration counts of this solve"}
    n_rows = int(sum(s.n for s in sl))
    nnzb = int(sum(s.nnzb for s in sl))
    line = {
        "metric": BATCH_METRIC, "value": solve_s, "unit": "s", "higher_is_better": False, "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": solve_s * 1e3, "dtype": "f64",
        "data": "synthetic (seeded 2D 5-point block stencils)", "vs_baseline": None, "scaling": "weak",
        "config": {"workload": f"{len(sl)} SPD 2D block systems, sides log-uniform 32..256, bs 4/8 by seed, "
                               f"{R} RHS each; batched pCG + block IChol0, FP64, tol 1e-10",
                   "systems": len(sl), "rhs": R, "block_rows": n_rows, "nnzb": nnzb,
                   "matrix_gb": sum(s.vals.nbytes for s in sl) / 1e9,
                   "l2": "inputs larger than L2"},
        "iterations": {"max": int(res["iters"].max()), "mean": float(res["iters"].mean()),
                       "graph_iters": info["graph_iters"], "converged_pairs": info["n_converged"],
                       "pairs": info["n_pairs"]},
        "setup": {"generate_s": gen_s, "create_s": create_s, "first_solve_autotune_capture_ms": first["setup_ms"]},
        "tuning": tun,
        "roofline": {"bound": "hbm", "kernel": "whole batched iteration (spmv + sweeps + vector passes)",
                     "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes": total_bytes},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": bh.nbytes, "d2h_bytes_per_step": bh.nbytes},
        "gpu_launches": launches // steps, "clocks": clocks, "cpu_baseline": cpu,
    }
    B.close()
    h.close()
    return line


# ----------------------------------------------------------------- mixed / learned workloads

def _solve_variant(bsp, _lib, A, b, stream, make_pc, precision, solver="pgmres"):
    """One timed solve: preconditioner set-up + refined pGMRES(30, k=10) (or
    pCG) to the FP64 true relative residual 1e-10."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pc = make_pc()
    e1.record(stream)
    if solver == "pcg":
        x, info, _ = bsp.pCG(A, b, TOL, pc, 20000, return_info=True, stop_rule=_lib.STOP_TRUE_RESIDUAL,
                             precision=precision, inner_tol=1e-6)
    else:
        x, info, _ = bsp.pGMRES(A, b, TOL, pc, 20000, 30, 10, return_info=True,
                                stop_rule=_lib.STOP_TRUE_RESIDUAL, precision=precision, inner_tol=1e-6)
    e2.record(stream)
    e2.synchronize()
    kind = pc.kind
    pc.close()
    return x, {"setup_s": e0.elapsed_time(e1) / 1e3, "solve_s": e1.elapsed_time(e2) / 1e3,
               "total_s": e0.elapsed_time(e2) / 1e3, "iters": info["iters"], "refinements": info["n_outer"],
               "true_rel_res": info["true_rel_res"], "status": info["status"], "precond_kind": kind}


def reference_x(s, B, D, budget_s=900.0):
    """The reference's own FP64 solve (ILU0_pGMRES(30, 10) to 1e-10, the build
    without fast-math) of system s on this host, for solution errors."""
    exe = ROOT / "oracle" / "_ref" / "ref_solve_hist"
    if not exe.exists():
        return None, None
    from blocksp_b200 import systems
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "sys.bsps"
        xo = Path(d) / "x.vec"
        systems.write_bsr(f, s)
        cmd = [str(exe), str(f), "--B", str(B), "--D", str(D), "--solver", "ilu0_pgmres", "--tol", "1e-10",
               "--maxit", "20000", "--restart", "30", "--k", "10", "--x", str(xo), "--time"]
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        t0 = time.time()
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=budget_s)
        el = time.time() - t0
        if r.returncode != 0 or not xo.exists():
            return None, el
        raw = xo.read_bytes()
        return np.frombuffer(raw[8:], dtype="<f8").copy(), el


def run_mixed(args):
    """cfg2: the 64^3 bs-8 system and the 48^3 bs-16 system, pGMRES-DR + ILU0 to
    the FP64 true residual 1e-10 with the inner work in FP64, FP32 storage or
    BF16 storage (FP64 vectors, refinement, Arnoldi and least squares), and each
    result's relative error against the reference's FP64 CPU solution."""
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, systems
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    out = {}
    with ClockSampler(0) as clk:
        for name, s, B, D in (("3d64_bs8", systems.config1(seed=1, side=64), 4, 2),
                              ("3d48_bs16", systems.config2b(seed=2, side=48), 8, 2)):
            A = bsp.Matrix.from_system(s, h)
            b = torch.tensor(s.b, device="cuda")
            res = {}
            xs = {}
            for vname, prec in (("f64", _lib.PREC_F64), ("f32_storage", _lib.PREC_F32),
                                ("bf16_storage", _lib.PREC_BF16)):
                for _ in range(max(args.warmup, 1)):
                    _solve_variant(bsp, _lib, A, b, stream, lambda: bsp.ILU0(A), prec)
                runs = [_solve_variant(bsp, _lib, A, b, stream, lambda: bsp.ILU0(A), prec) for _ in range(args.steps)]
                xs[vname] = runs[-1][0].cpu().numpy()
                r = runs[-1][1]
                r["total_s"] = statistics.mean(v[1]["total_s"] for v in runs)
                res[vname] = r
            xref, ref_s = (reference_x(s, B, D) if not args.no_cpu_baseline else (None, None))
            for vname in res:
                res[vname]["rel_err_vs_gpu_f64"] = float(np.abs(xs[vname] - xs["f64"]).max() /
                                                         np.abs(xs["f64"]).max())
                if xref is not None:
                    res[vname]["rel_err_vs_reference_f64"] = float(np.abs(xs[vname] - xref).max() /
                                                                   np.abs(xref).max())
            out[name] = {"n_block_rows": s.n, "bs": s.bs, "nnzb": s.nnzb, "variants": res,
                         "reference_solve_wall_s": ref_s}
            A.close()
    best = min(out["3d64_bs8"]["variants"].items(), key=lambda kv: kv[1]["total_s"])
    line = {"metric": "mixed precision: time to FP64 true relative residual 1e-10 (pGMRES-DR + ILU0)",
            "value": best[1]["total_s"], "unit": "s", "higher_is_better": False, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "dtype": "f64 outer / f32 or bf16 inner storage",
            "data": "synthetic (seeded 3D 7-point block stencils)", "vs_baseline": None,
            "config": {"workload": "cfg2: 64^3 8x8 and 48^3 16x16 block systems, skew 0.3",
                       "best_variant_3d64": best[0]},
            "systems": out, "clocks": clk.summary()}
    h.close()
    print(json.dumps(line), flush=True)


def run_learned(args):
    """cfg4 ablation: held-out 3D convection-diffusion systems (8x8 blocks,
    log-normal conductivity, random velocity) at side^3, pGMRES(30, k=10) to the
    FP64 true residual 1e-10 with block ILU0, with the trained network's
    factors (forced), and with LearnedLU (the learned factors only when the
    model's validation beat ILU0, else ILU0), in FP64 and with FP32 storage."""
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, learned, systems
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    model = learned.LearnedModel.load(handle=h)
    seeds = [30000 + i for i in range(args.learned_seeds)]
    dims = (args.learned_side,) * 3
    per = []
    with ClockSampler(0) as clk:
        for sd in seeds:
            s = systems.convection_diffusion_system(dims, 8, sd)
            A = bsp.Matrix.from_system(s, h)
            b = torch.tensor(s.b, device="cuda")
            row = {"seed": sd}
            for vname, mk, prec in (
                    ("ilu0_f64", lambda: bsp.ILU0(A), _lib.PREC_F64),
                    ("ilu0_f32", lambda: bsp.ILU0(A), _lib.PREC_F32),
                    ("learned_forced_f64", lambda: model.precond(A), _lib.PREC_F64),
                    ("learned_forced_f32", lambda: model.precond(A), _lib.PREC_F32),
                    ("learned_with_fallback_f64", lambda: learned.LearnedLU(A, model), _lib.PREC_F64)):
                _solve_variant(bsp, _lib, A, b, stream, mk, prec)  # warm-up
                row[vname] = _solve_variant(bsp, _lib, A, b, stream, mk, prec)[1]
            per.append(row)
            A.close()
    names = [k for k in per[0] if k != "seed"]
    summary = {k: {"total_s": float(np.mean([r[k]["total_s"] for r in per])),
                   "iters": float(np.mean([r[k]["iters"] for r in per]))} for k in names}
    line = {"metric": "learned preconditioner ablation: time to FP64 true relative residual 1e-10",
            "value": summary["learned_with_fallback_f64"]["total_s"], "unit": "s", "higher_is_better": False,
            "n_gpus": 1, "dtype": "f64 (f32 storage variants marked)", "vs_baseline": None,
            "data": f"synthetic held-out seeds {seeds} (training used 10000-10199, validation 20000-20003)",
            "config": {"workload": f"cfg4: 3D {dims[0]}^3 convection-diffusion, 8x8 blocks, pGMRES(30, k=10)",
                       "model_beats_ilu0_on_validation": bool(model.meta.get("beats_ilu0", False)),
                       "model_validation": model.meta.get("validation")},
            "summary": summary, "per_seed": per, "clocks": clk.summary()}
    model.close()
    h.close()
    print(json.dumps(line), flush=True)


def llt_measure(args, warmup: int, steps: int) -> dict:
    """The learned L L^T preconditioner against block IChol0: held-out SPD 3D
    diffusion systems (8x8 blocks, log-normal conductivity), pCG to the FP64
    true relative residual 1e-10; per variant the mean set-up + solve time over
    `steps` timed solves after `warmup`, on each seed."""
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, learned, systems
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    model = learned.LearnedModel.load(learned.WEIGHTS_LLT, handle=h) if learned.WEIGHTS_LLT.exists() else None
    seeds = [30200 + i for i in range(args.learned_seeds)]
    dims = (args.llt_side,) * 3
    variants = (("ichol0_f64", lambda A: bsp.IChol0(A), _lib.PREC_F64),
                ("ichol0_f32", lambda A: bsp.IChol0(A, _lib.PREC_F32), _lib.PREC_F32),
                ("learned_llt_f64", lambda A: learned.LearnedLLT(A, model), _lib.PREC_F64),
                ("learned_llt_f32", lambda A: learned.LearnedLLT(A, model, _lib.PREC_F32), _lib.PREC_F32))
    per = []
    launches = 0
    lib = _lib.load()
    with ClockSampler(0) as clk:
        for sd in seeds:
            s = systems.convection_diffusion_system(dims, 8, sd, speed=0.0)
            A = bsp.Matrix.from_system(s, h)
            b = torch.tensor(s.b, device="cuda")
            row = {"seed": sd}
            for vname, mk, prec in variants:
                for _ in range(warmup):
                    _solve_variant(bsp, _lib, A, b, stream, lambda: mk(A), prec, "pcg")
                l0 = lib.bsp_launch_count()
                runs = [_solve_variant(bsp, _lib, A, b, stream, lambda: mk(A), prec, "pcg")[1] for _ in range(steps)]
                launches += lib.bsp_launch_count() - l0
                row[vname] = {**runs[-1], "total_s": float(np.mean([r["total_s"] for r in runs])),
                              "setup_s": float(np.mean([r["setup_s"] for r in runs])),
                              "solve_s": float(np.mean([r["solve_s"] for r in runs]))}
            per.append(row)
            A.close()
    names = [v[0] for v in variants]
    summary = {k: {"total_s": float(np.mean([r[k]["total_s"] for r in per])),
                   "setup_s": float(np.mean([r[k]["setup_s"] for r in per])),
                   "iters": float(np.mean([r[k]["iters"] for r in per])),
                   "max_true_rel_res": float(max(r[k]["true_rel_res"] for r in per))} for k in names}
    gate = bool(model is not None and model.meta.get("beats_baseline", False))
    out = {"metric": "learned L L^T vs block IChol0: pCG time to FP64 true relative residual 1e-10",
           "value": summary["learned_llt_f32"]["total_s"], "unit": "s", "higher_is_better": False,
           "speedup_vs_ichol0_f64": summary["ichol0_f64"]["total_s"] / summary["learned_llt_f32"]["total_s"],
           "iteration_ratio_f64": summary["learned_llt_f64"]["iters"] / summary["ichol0_f64"]["iters"],
           "seeds": seeds, "side": dims[0], "steps": steps, "warmup": warmup, "gate_open": gate,
           "relax": model.relax if model is not None else None,
           "network_used": model.meta.get("network_used") if model is not None else None,
           "summary": summary, "per_seed": per, "gpu_launches": launches, "clocks": clk.summary()}
    if model is not None:
        model.close()
    h.close()
    return out


def run_learned_llt(args):
    m = llt_measure(args, max(args.warmup, 3), args.steps)
    line = {**m, "n_gpus": 1, "dtype": "f64 (f32 storage variants marked)", "vs_baseline": None,
            "data": f"synthetic held-out seeds {m['seeds']} (training used 10000-10099, relaxation fit "
                    "15000-15003, validation 20000-20003)",
            "config": {"workload": f"SPD 3D {m['side']}^3 diffusion, 8x8 blocks, pCG + IChol0 / learned L L^T"}}
    print(json.dumps(line), flush=True)


def llt_summary(args) -> dict:
    """The learned L L^T comparison inside the default line: one warm-up and
    one timed solve per variant and seed (`--workload learned_llt` is the full
    measurement)."""
    m = llt_measure(args, 1, 1)
    return {k: m[k] for k in ("metric", "value", "unit", "speedup_vs_ichol0_f64", "iteration_ratio_f64", "seeds",
                              "side", "gate_open", "relax", "network_used", "summary", "gpu_launches")}


def run_complex(args):
    """The complex solve path (T = std::complex<double>): 3D side^3 7-point
    complex 4x4 block system (the real embedding is 8x8), block ILU0 +
    pGMRES(30, k=10) with the reference's stopping rule 1e-10, host vectors in
    and out; per step the ILU0 set-up and the solve.  The reference's own
    complex build (oracle/_ref/ref_complex_hist, single-threaded) times one
    full solve of the same system on the host."""
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import _lib, systems
    side = args.complex_side
    s = systems.complex_system((side,) * 3, 4, 5)
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    lib = _lib.load()
    A = bsp.Matrix.from_system(s, h)

    def one():
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        pc = bsp.ILU0(A)
        e[1].record(stream)
        x, info, hist = bsp.pGMRES(A, s.b, TOL, pc, 5000, 30, 10, return_info=True)
        e[2].record(stream)
        e[2].synchronize()
        pc.close()
        return x, info, hist, e[0].elapsed_time(e[1]) / 1e3, e[1].elapsed_time(e[2]) / 1e3
    with ClockSampler(0) as clk:
        for _ in range(max(args.warmup, 3)):
            one()
        l0 = lib.bsp_launch_count()
        runs = [one() for _ in range(args.steps)]
        launches = lib.bsp_launch_count() - l0
    x, info, hist, _, _ = runs[-1]
    setup = float(np.mean([r[3] for r in runs]))
    solve = float(np.mean([r[4] for r in runs]))
    cpu = None
    ref_iters = None
    exe = ROOT / "oracle" / "_ref" / "ref_complex_hist"
    if exe.exists() and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            f = Path(td) / "c.bspc"
            systems.write_complex_bsr(f, s)
            t0 = time.perf_counter()
            out = subprocess.run([str(exe), str(f), "--B", "4", "--solver", "ilu0_pgmres", "--restart", "30",
                                  "--k", "10", "--tol", repr(TOL)], capture_output=True, text=True,
                                 env=dict(os.environ, OPENBLAS_NUM_THREADS="1"), timeout=1800).stdout
            wall = time.perf_counter() - t0
        t = {ln.split()[1]: float(ln.split()[2]) for ln in out.splitlines() if ln.startswith("TIME ")}
        ref_iters = next((int(ln.split()[2]) for ln in out.splitlines() if ln.startswith("pGMRES iters")), None)
        cpu = {"value": t.get("setup_s", 0.0) + t.get("solve_s", 0.0), "unit": "s", "cores": 1, "kind": "reference",
               "sample": f"one full reference ILU0_pGMRES<std::complex<double>,4,1>(A, 1e-10, 5000, 30, 10) solve of "
                         f"the same system ({ref_iters} iterations): set-up {t.get('setup_s', 0):.2f} s + solve "
                         f"{t.get('solve_s', 0):.2f} s, timed inside the reference build (process wall {wall:.1f} s)"}
    line = {"metric": "complex ILU0-pGMRES(30, k=10): time to relative preconditioned residual 1e-10",
            "value": setup + solve, "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "dtype": "complex f64", "vs_baseline": None,
            "data": f"synthetic (seeded {side}^3 7-point complex block stencil)",
            "config": {"workload": f"complex T: 3D {side}^3, 4x4 complex blocks (8x8 real embedding), ILU0 + "
                                   "pGMRES(30, k=10), reference stopping rule", "n_block_rows": s.n,
                       "nnzb": int(s.row_ptr[-1])},
            "setup_s": setup, "solve_s": solve, "iters": info["iters"], "reference_iters": ref_iters,
            "restarts": info["n_restarts"], "true_rel_res": info["true_rel_res"],
            "gpu_launches": launches, "clocks": clk.summary(), "cpu_baseline": cpu}
    A.close()
    h.close()
    print(json.dumps(line), flush=True)


def run_apply(args):
    """The ILU0 application alone (forward + backward streamed sweeps) on the
    64^3 8x8 system, `steps` times after `warmup`: the kernel the solve's
    roofline is quoted on, in a short program that profilers can capture."""
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import systems
    stream = torch.cuda.Stream()
    h = bsp.Handle(0, stream=stream.cuda_stream)
    s = systems.config1(seed=1, side=args.side)
    A = bsp.Matrix.from_system(s, h)
    pc = bsp.ILU0(A)
    b = torch.tensor(s.b, device="cuda")
    z = torch.empty_like(b)
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 1)):
            z.copy_(b)
            pc(z)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(args.steps):
            z.copy_(b)
            e0.record(stream)
            pc(z)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    peak, kind = read_peaks()
    nbytes = ilu_apply_bytes(s.n, s.bs, s.nnzb)
    t = statistics.mean(ms)
    print(json.dumps({"metric": "ILU0 application (two streamed sweeps) GB/s", "value": nbytes / (t * 1e-3) / 1e9,
                      "unit": "GB/s", "ms_per_apply": t, "steps": args.steps, "warmup": args.warmup,
                      "algorithmic_bytes": nbytes, "peak": peak, "peak_source": kind,
                      "levels": [pc.info()["levels_lower"], pc.info()["levels_upper"]]}), flush=True)
    pc.close()
    A.close()
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--bsmv-reps", type=int, default=50)
    ap.add_argument("--cpu-budget", type=float, default=150.0,
                    help="reference arm: seconds of full CPU solves to run (at least one)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", default="plain_f64,mixed_f32,learned_mixed_f32")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="leave the cfg3 batch summary out of the default line")
    ap.add_argument("--no-llt", action="store_true",
                    help="leave the learned L L^T vs IChol0 summary out of the default line")
    ap.add_argument("--workload", default="cfg1",
                    choices=["cfg1", "batch", "mixed", "learned", "learned_llt", "complex", "apply"],
                    help="cfg1: the headline line; batch: 256-system batched pCG; mixed: cfg2 precision "
                         "variants; learned: cfg4 ablation; learned_llt: learned L L^T vs IChol0 with pCG; "
                         "apply: the ILU0 application alone (profiling)")
    ap.add_argument("--llt-side", type=int, default=64)
    ap.add_argument("--complex-side", type=int, default=48)
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--learned-side", type=int, default=96)
    ap.add_argument("--learned-seeds", type=int, default=2)
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend under torchrun (gloo: the rank logic on CPU only)")
    args = ap.parse_args()
    if args.workload != "cfg1":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": f"the {args.workload} leg reports its CPU "
                              "reference inside its own line"}))
            return
        {"batch": run_batch, "mixed": run_mixed, "learned": run_learned, "learned_llt": run_learned_llt,
         "complex": run_complex, "apply": run_apply}[args.workload](args)
        return
    world, rank, local = dist_setup(args.dist_backend)
    workload = (f"pGMRES(30, deflated restart k=10) + block ILU0 to FP64 true relative residual "
                f"1e-10; 3D {args.side}^3 7-point block stencil, 8x8 FP64 blocks, skew c=0.3")
    cores = os.cpu_count() or 1
    n_rows = args.side ** 3
    nnzb = n_rows + 2 * 3 * (args.side - 1) * args.side ** 2
    config = {"workload": workload, "n_block_rows": n_rows, "nnzb": nnzb, "bs": 8,
              "l2": f"inputs larger than L2 ({nnzb * 64 * 8 / 1e6:.0f} MB of matrix blocks)",
              "parallelism": "replicas"}

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_reference_full(args.side, runs=args.steps, budget_s=args.cpu_budget)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference build oracle/_ref/ref_solve missing (run make -C oracle)"}))
            return
        sample = (f"full run{'s' if cb['runs'] > 1 else ''}: {cb['runs']} complete reference ILU0_pGMRES(A, 1e-10, "
                  f"5000, 30, 10) solve{'s' if cb['runs'] > 1 else ''} ({cb['iters']} iterations), mean set-up "
                  f"{cb['setup_s']:.2f} s + solve {cb['solve_s']:.2f} s; single-threaded by construction, so one "
                  "core; runs stop once the time budget is spent, so steps counts the runs made")
        line = {"metric": METRIC, "impl": "reference", "value": cb["total_s"], "unit": "s",
                "higher_is_better": False, "n_gpus": args.gpus, "steps": cb["runs"],
                "warmup": 0, "ms_per_step": cb["total_s"] * 1e3, "config": config,
                "iterations": cb["iters"],
                "cpu_baseline": {"value": cb["total_s"], "unit": "s", "cores": 1, "cores_available": cores,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": cb["total_s"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    r = run_gpu(args, world, rank, local)
    if rank != 0:
        return
    best = r["results"][r["best"]]
    n, bs, nnzb = r["n"], r["bs"], r["nnzb"]
    bsmv_gbs = bsmv_bytes(n, bs, nnzb) / (r["bsmv_ms"] * 1e-3) / 1e9
    ilu_b = ilu_apply_bytes(n, bs, nnzb)
    ilu_gbs = ilu_b / (r["ilu_ms"] * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cb = cpu_reference_full(args.side, runs=1)
        if cb is not None:
            cpu = {"value": cb["total_s"], "unit": "s", "cores": 1, "cores_available": cores, "kind": "reference",
                   "sample": f"full run: one complete reference ILU0_pGMRES(A, 1e-10, 5000, 30, 10) solve of "
                             f"the same system ({cb['iters']} iterations), set-up {cb['setup_s']:.2f} s + solve "
                             f"{cb['solve_s']:.2f} s; single-threaded by construction"}
    gold = reference_golden(args.side)
    parity = None
    if gold is not None:
        h = np.asarray(r["hist_f64"])
        g = gold["hist"]
        k = min(len(h), len(g))
        parity = {"reference_iters": gold["iters"], "gpu_iters": r["iters_f64"],
                  "history_max_abs_dev": float(np.abs(h[:k] / h[0] - g[:k] / g[0]).max())}
    xbytes = n * bs * 8
    traffic = ILU_APPLY_TRAFFIC_64 if args.side == 64 else None
    line = {
        "metric": METRIC,
        "value": best["total_s"] / args.gpus if args.gpus > 1 else best["total_s"],
        "unit": "s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": best["total_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": f"synthetic (seeded {args.side}^3 7-point block stencil)",
        "config": {**config, "best_variant": r["best"]},
        "variants": r["results"],
        "target_comparison": target_comparison(r["results"]),
        "parity_vs_reference": parity,
        "bsmv": {"kernel": "k_bsmv<8,double,double,1>", "ms": r["bsmv_ms"], "gbs": bsmv_gbs,
                 "frac_of_peak": bsmv_gbs / r["peak"], "algorithmic_bytes": bsmv_bytes(n, bs, nnzb)},
        "ilu0_apply": {"ms": r["ilu_ms"], "gbs": ilu_gbs, "frac_of_peak": ilu_gbs / r["peak"],
                       "algorithmic_bytes": ilu_b,
                       "levels": [r["levels"]["levels_lower"], r["levels"]["levels_upper"]]},
        "roofline": {"bound": "hbm",
                     "kernel": "k_ssweep<8,double> x2 (one ILU0 application: forward + backward streamed sweeps)",
                     "achieved": ilu_gbs, "peak": r["peak"], "unit": "GB/s", "frac": ilu_gbs / r["peak"],
                     "traffic": traffic, "algorithmic_bytes": ilu_b, "peak_source": r["peak_kind"]},
        "e2e": {"value": r["e2e_s"], "unit": "s", "h2d_bytes_per_step": nnzb * bs * bs * 8 + nnzb * 4
                + (n + 1) * 4 + xbytes, "d2h_bytes_per_step": xbytes, "parts": r.get("e2e_parts")},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "cpu_baseline": cpu,
    }
    if not args.no_batch and args.gpus == 1:
        line["batch"] = batch_summary(args)
    if not args.no_llt and args.gpus == 1:
        line["learned_llt"] = llt_summary(args)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
