"""Benchmark of the BlockSp B200 solve path.

Default workload (one GPU): the plain GPU drop-in solve, pGMRES(30) with
deflated restart k = 10 and block ILU0 in FP64 on the 3D 64^3 7-point block
stencil with 8x8 blocks (262,144 block rows, 1,810,432 blocks), to relative
tolerance 1e-10, plus the standalone bsmv of the same matrix.  A "step" is one
solve (preconditioner setup + pGMRES), timed on the device with CUDA events.

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's
own CPU implementation of the path on this host instead (the reference
library compiled from its headers by oracle/Makefile, else the oracle port).
Multi-GPU: the path does not shard (replicas only), so ``--gpus N`` runs N
independent replicas, one per rank, and reports the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
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
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------- GPU arm

def bsmv_bytes(n: int, bs: int, nnzb: int, nrhs: int = 1, val_bytes: int = 8, vec_bytes: int = 8) -> int:
    """Algorithmic bytes of y = A x: blocks + indices + x read once + y written."""
    return (nnzb * bs * bs * val_bytes + nnzb * 4 + (n + 1) * 4 + 2 * n * bs * nrhs * vec_bytes)


def run_gpu(args, world, rank, local):
    import torch
    import blocksp_b200 as bsp
    from blocksp_b200 import systems

    torch.cuda.set_device(local)
    dev_stream = torch.cuda.Stream()
    h = bsp.Handle(local, stream=dev_stream.cuda_stream)
    sysm = systems.config1(seed=1 + rank, side=args.side)
    A = bsp.Matrix.from_system(sysm, h)
    n, bs, nnzb = sysm.n, sysm.bs, sysm.nnzb
    x = torch.tensor(sysm.b, device="cuda")
    y = torch.empty_like(x)

    # ---- standalone bsmv: K launches, inputs (969 MB) larger than L2 ----
    for _ in range(max(args.warmup, 3)):
        bsp.bsmv_dev(A, x, y)
    torch.cuda.synchronize()
    barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    reps = args.bsmv_reps
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        with torch.cuda.stream(dev_stream):
            ev0.record(dev_stream)
            for _ in range(reps):
                bsp.bsmv_dev(A, x, y)
            ev1.record(dev_stream)
        ev1.synchronize()
    bsmv_ms = ev0.elapsed_time(ev1) / reps
    bsmv_ms = max_over_ranks(bsmv_ms, world)
    alg = bsmv_bytes(n, bs, nnzb)
    peak, peak_kind = read_peaks()
    achieved = alg / (bsmv_ms * 1e-3) / 1e9

    # ---- e2e bsmv through the host-buffer C ABI: pinned x in, y out ----
    xh = torch.tensor(sysm.b).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    lib = bsp._lib.load()
    for _ in range(3):
        bsp._lib.check(lib.bsp_bsmv(h.h, A.m, 1, 0, 1.0, xh.data_ptr(), 0.0, yh.data_ptr()), "bsp_bsmv")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_reps = max(3, reps // 4)
    for _ in range(e2e_reps):
        bsp._lib.check(lib.bsp_bsmv(h.h, A.m, 1, 0, 1.0, xh.data_ptr(), 0.0, yh.data_ptr()), "bsp_bsmv")
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_reps
    e2e_ms = max_over_ranks(e2e_ms, world)
    clocks = clk.summary()
    res = {
        "bsmv_ms": bsmv_ms, "bsmv_gbs": achieved, "bsmv_alg_bytes": alg,
        "e2e_bsmv_ms": e2e_ms, "n": n, "bs": bs, "nnzb": nnzb,
        "peak": peak, "peak_kind": peak_kind, "clocks": clocks, "launches": reps,
    }
    A.close()
    h.close()
    return res


# --------------------------------------------------------------------- CPU arms

def cpu_bsmv_sample(side: int) -> dict:
    """Oracle (numpy restatement) bsmv on the same matrix, a bounded sample."""
    from blocksp_b200 import systems
    import oracle.blocksp_oracle as O
    s = systems.config1(seed=1, side=side)
    A = O.BSR.from_system(s)
    O.bsmv(A, s.b)
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 10.0 and reps < 20:
        O.bsmv(A, s.b)
        reps += 1
    ms = (time.perf_counter() - t0) * 1e3 / reps
    return {"ms": ms, "reps": reps, "gbs": bsmv_bytes(s.n, s.bs, s.nnzb) / (ms * 1e-3) / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--bsmv-reps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_bsmv_sample(args.side)
        line = {"metric": METRIC, "impl": "reference", "value": cb["gbs"], "unit": "GB/s",
                "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "cpu_baseline": {"value": cb["gbs"], "unit": "GB/s", "cores": 1,
                                                       "kind": "port", "sample": f"{cb['reps']} bsmv calls"},
                "e2e": {"value": cb["gbs"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    r = run_gpu(args, world, rank, local)
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cb = cpu_bsmv_sample(args.side)
        cpu = {"value": cb["gbs"], "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"{cb['reps']} oracle bsmv calls on the same matrix"}
    xbytes = r["n"] * r["bs"] * 8
    line = {
        "metric": METRIC,
        "value": r["bsmv_gbs"] * args.gpus,
        "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.bsmv_reps, "warmup": args.warmup,
        "ms_per_step": r["bsmv_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 64^3 7-point block stencil)",
        "config": {"workload": "bsmv, 3D 64^3 7-point, 8x8 FP64 blocks (cfg1 matrix)",
                   "n_block_rows": r["n"], "nnzb": r["nnzb"], "bs": r["bs"],
                   "l2": "inputs larger than L2 (969 MB per bsmv)", "parallelism": "replicas"},
        "roofline": {"bound": "hbm", "achieved": r["bsmv_gbs"], "peak": r["peak"], "unit": "GB/s",
                     "frac": r["bsmv_gbs"] / r["peak"], "traffic": None,
                     "peak_source": r["peak_kind"]},
        "e2e": {"value": bsmv_bytes(r["n"], r["bs"], r["nnzb"]) / (r["e2e_bsmv_ms"] * 1e-3) / 1e9,
                "unit": "GB/s", "h2d_bytes_per_step": xbytes, "d2h_bytes_per_step": xbytes},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
