"""Generate the complex (T = std::complex<double>) golden fixtures in tests/golden/.

TEST INFRASTRUCTURE.  Runs oracle/_ref/ref_complex_hist (the reference BlockSp
v1.0 headers with T = std::complex<double>, residual prints enabled, built by
oracle/Makefile) on small seeded complex systems from
blocksp_b200.systems.complex_system and stores, per case, the reference's
outputs: the result vector (complex), the residual history it prints and the
printed iteration count.  The systems are regenerated from their parameters
by the tests.

Run from the repository root:
    python tests/golden/make_golden_complex.py
"""
from __future__ import annotations

import json
import struct
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from blocksp_b200 import systems  # noqa: E402

OUT = Path(__file__).resolve().parent
EXE = ROOT / "oracle" / "_ref" / "ref_complex_hist"

# name: (dims, complex bs, seed, solver, extra args)
CASES = {
    "c_bsmv_3d_bs4": ((4, 4, 4), 4, 101, "bsmv", []),
    "c_ilu0_apply_3d_bs4": ((4, 4, 4), 4, 102, "ilu0_apply", []),
    "c_sor_apply_2d_bs2": ((8, 8), 2, 103, "sor_apply", ["--w", "1.6", "--nu", "3", "--sortype", "0"]),
    "c_diag_apply_3d_bs8": ((3, 3, 3), 8, 104, "diag_apply", []),
    "c_ilu0_pgmres_3d_bs4": ((5, 5, 5), 4, 105, "ilu0_pgmres", ["--tol", "1e-10", "--maxit", "500"]),
    "c_ilu0_pgmres_dr_3d_bs4": ((6, 6, 6), 4, 106, "ilu0_pgmres",
                                ["--tol", "1e-10", "--maxit", "500", "--restart", "10", "--k", "4"]),
    "c_ilu0_pgmres_dr_3d_bs8": ((4, 4, 4), 8, 107, "ilu0_pgmres",
                                ["--tol", "1e-10", "--maxit", "500", "--restart", "15", "--k", "5"]),
    "c_sor_pgmres_dr_2d_bs2": ((10, 10), 2, 108, "sor_pgmres",
                               ["--tol", "1e-10", "--maxit", "500", "--restart", "10", "--k", "3",
                                "--w", "1.2", "--nu", "2", "--sortype", "0"]),
    "c_diag_pgmres_restart_2d_bs1": ((12, 12), 1, 109, "diag_pgmres",
                                     ["--tol", "1e-10", "--maxit", "120", "--restart", "10", "--k", "0"]),
    "c_nopre_pgmres_2d_bs2": ((6, 6), 2, 110, "nopre_pgmres", ["--tol", "1e-10", "--maxit", "500"]),
}


def read_complex_vec(path: Path) -> np.ndarray:
    raw = path.read_bytes()
    m = struct.unpack("<q", raw[:8])[0]
    return np.frombuffer(raw[8:8 + 8 * m], dtype=np.complex128).copy()


def run_case(name, spec, tmp: Path) -> dict:
    dims, bs, seed, solver, extra = spec
    s = systems.complex_system(dims, bs, seed)
    f = tmp / f"{name}.bspc"
    systems.write_complex_bsr(f, s)
    xo = tmp / f"{name}.x"
    cmd = [str(EXE), str(f), "--B", str(bs), "--solver", solver, "--x", str(xo), *extra]
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
    hist, iters = [], -1
    for line in out.splitlines():
        p = line.split()
        if not p:
            continue
        if p[0] == "RES0":
            hist.append(float(p[1]))
        elif p[0] == "RES":
            hist.append(float(p[2]))
        elif line.startswith("pGMRES iters"):
            iters = int(p[2])
    meta = {"dims": list(dims), "bs": bs, "seed": seed, "solver": solver, "args": extra}
    np.savez_compressed(OUT / f"{name}.npz", x=read_complex_vec(xo), hist=np.array(hist), iters=np.array(iters),
                        meta=np.array(json.dumps(meta)))
    return {"name": name, "iters": iters, "hist_len": len(hist)}


def main():
    if not EXE.exists():
        sys.exit(f"{EXE} missing: build it with `make -C oracle REF=<reference sources>`")
    with tempfile.TemporaryDirectory() as td:
        for name, spec in CASES.items():
            print(run_case(name, spec, Path(td)), flush=True)


if __name__ == "__main__":
    main()
