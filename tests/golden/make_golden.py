"""Generate the golden fixtures in tests/golden/ by running the reference itself.

TEST INFRASTRUCTURE.  Runs oracle/_ref/ref_solve_hist (the reference BlockSp
v1.0 headers compiled by oracle/Makefile, residual prints enabled) on small
seeded systems from blocksp_b200.systems and stores, per case, the reference's
outputs: the result vector, the residual history it prints, and the printed
iteration count.  The systems are regenerated from their parameters by the
tests (the generator is deterministic), so only outputs are stored.

Also stores the LDG fixture (the reference's test_mats/LDG_2D_vecLap*.mtx,
converted to arrays) and the reference's infinity-norm errors on it, so the GPU
can be checked against the reference's only known answer where the reference
sources are not present.

Also stores the reference's solves of three full-size benchmark systems
(``CONFIG_CASES``: the 64^2 bs4 IChol0-pCG system, the 64^3 bs8 ILU0-pGMRES(30)
deflated-restart system and the 48^3 bs16 one): their residual histories,
iteration counts, the norm of x and a fixed strided sample of x (the whole x
for the 64^2 system), so the GPU solver is checked at full size.

Run from the repository root:
    python tests/golden/make_golden.py [--configs-only [NAME ...] | --ldg-only | --algebra-only]
The reference sources are read from $BLOCKSP_REFERENCE (the LDG matrices under
its test_mats/); the checker binary must have been built by oracle/Makefile.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from blocksp_b200 import systems  # noqa: E402

OUT = Path(__file__).resolve().parent
EXE = ROOT / "oracle" / "_ref" / "ref_solve_hist"
REF_MATS = Path(os.environ.get("BLOCKSP_REFERENCE", "")) / "test_mats"

# Full-size systems: name -> (system factory, B, D, solver, extra args, full x?)
CONFIG_CASES = {
    "cfg0_ichol0_pcg_2d64_bs4": ("config0", 2, 2, "ichol0_pcg", ["--tol", "1e-10", "--maxit", "2000"], True),
    "cfg1_ilu0_pgmres_dr_3d64_bs8": ("config1", 4, 2, "ilu0_pgmres",
                                     ["--tol", "1e-10", "--maxit", "5000", "--restart", "30", "--k", "10"],
                                     False),
    "cfg2b_ilu0_pgmres_dr_3d48_bs16": ("config2b", 8, 2, "ilu0_pgmres",
                                       ["--tol", "1e-10", "--maxit", "5000", "--restart", "30", "--k", "10"],
                                       False),
}
X_SAMPLE_STRIDE = 997  # a prime stride, so the sample visits every block-row position

# Block algebra on seeded random block matrices (systems.random_blocksp):
# name -> (m, bs, n_col, seed, B, D, driver mode, extra args)
ALGEBRA_CASES = {
    "bsmm_rand_bs4": (24, 4, 4, 31, 4, 1, "bsmm", ["--atran", "0"]),
    "bsmm_t_rand_bs4": (24, 4, 4, 31, 4, 1, "bsmm", ["--atran", "1"]),
    "bs_tr_rand_bs4": (24, 4, 4, 31, 4, 1, "bs_tr", []),
    "bsmm_t_rand_bs8": (16, 8, 3, 33, 8, 1, "bsmm", ["--atran", "1"]),
}
# arnoldi_eigenvalues: name -> (dims, bs, seed, skew, B, D, mode, iters, harmonic).
# Without a preconditioner only: the reference build's arnoldi_eigenvalues
# with an ILU0 preconditioner pointer ends in SIGSEGV (the driver's
# arnoldi_eig_ilu0 mode), so that case is checked against the oracle only.
EIG_CASES = {
    "arnoldi_eig_3d_bs8": ((5, 5, 5), 8, 71, 0.3, 8, 1, "arnoldi_eig", 30, 0),
    "arnoldi_eig_harm_3d_bs8": ((5, 5, 5), 8, 72, 0.3, 8, 1, "arnoldi_eig", 20, 1),
}
# block_pseudo_heat (blocksp_tests.hpp:269-300): ASym = I - delta A^T A with
# A random, 32x32 blocks (B = 16, D = 2), then the reference's solvers on it
PSEUDO_HEAT = {"m": 64, "bs": 32, "n_col": 4, "seed": 32, "delta": 2e-4, "B": 16, "D": 2}

# name: (dims, bs, seed, skew, B, D, solver, extra args)
CASES = {
    "bsmv_2d_bs4": ((8, 8), 4, 1, 0.0, 2, 2, "bsmv", []),
    "bsmv_3d_bs8": ((4, 4, 4), 8, 2, 0.3, 4, 2, "bsmv", []),
    "bsmv_3d_bs16": ((3, 3, 3), 16, 3, 0.3, 8, 2, "bsmv", []),
    "bsmv_multi_bs4_d2": ((6, 6), 4, 4, 0.0, 4, 2, "bsmv_multi", []),
    "ilu0_apply_3d_bs8": ((4, 4, 4), 8, 5, 0.3, 4, 2, "ilu0_apply", []),
    "ichol0_apply_2d_bs4": ((8, 8), 4, 6, 0.0, 2, 2, "ichol0_apply", []),
    "sor_apply_2d_bs4": ((8, 8), 4, 7, 0.3, 2, 2, "sor_apply", ["--w", "1.6", "--nu", "3", "--sortype", "0"]),
    "diag_apply_3d_bs8": ((4, 4, 4), 8, 8, 0.3, 4, 2, "diag_apply", []),
    "ichol0_pcg_2d_bs4": ((16, 16), 4, 9, 0.0, 2, 2, "ichol0_pcg", ["--tol", "1e-10", "--maxit", "2000"]),
    "sor_pcg_2d_bs4": ((12, 12), 4, 10, 0.0, 2, 2, "sor_pcg", ["--tol", "1e-10", "--maxit", "2000"]),
    "diag_pcg_2d_bs4": ((12, 12), 4, 11, 0.0, 2, 2, "diag_pcg", ["--tol", "1e-10", "--maxit", "2000"]),
    "ilu0_pgmres_3d_bs8": ((6, 6, 6), 8, 12, 0.3, 4, 2, "ilu0_pgmres", ["--tol", "1e-10"]),
    "ilu0_pgmres_dr_3d_bs8": ((6, 6, 6), 8, 13, 0.3, 4, 2, "ilu0_pgmres",
                              ["--tol", "1e-10", "--restart", "30", "--k", "10"]),
    "ilu0_pgmres_dr10_3d_bs8": ((6, 6, 6), 8, 14, 0.3, 4, 2, "ilu0_pgmres",
                                ["--tol", "1e-10", "--restart", "10", "--k", "4"]),
    "sor_pgmres_dr_2d_bs4": ((10, 10), 4, 15, 0.3, 2, 2, "sor_pgmres",
                             ["--tol", "1e-10", "--restart", "12", "--k", "5"]),
    "ilu0_pgmres_3d_bs16": ((4, 4, 4), 16, 16, 0.3, 8, 2, "ilu0_pgmres", ["--tol", "1e-10"]),
}


def system_for(dims, bs, seed, skew, nrhs=1):
    return systems.grid_system(dims, bs, seed=seed, skew=skew, nrhs=nrhs)


def run_ref(s, name, B, D, solver, extra, tmp: Path):
    """Run the reference on system s; returns (x, residual history, iterations)."""
    f = tmp / f"{name}.bsps"
    systems.write_bsr(f, s)
    xo = tmp / f"{name}.x"
    cmd = [str(EXE), str(f), "--B", str(B), "--D", str(D), "--solver", solver, "--x", str(xo),
           "--print-iters", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, check=True)
    hist, iters = [], -1
    for line in r.stdout.splitlines():
        p = line.split()
        if not p:
            continue
        if p[0] == "RES0":
            hist.append(float(p[1]))
        elif p[0] == "RES":
            hist.append(float(p[2]))
        elif line.startswith("pCG iters") or line.startswith("pGMRES iters"):
            iters = int(p[2])
    return systems.read_vec(xo), np.array(hist), iters


def run_case(name, spec, tmp: Path) -> dict:
    dims, bs, seed, skew, B, D, solver, extra = spec
    nrhs = D if solver == "bsmv_multi" else 1
    s = system_for(dims, bs, seed, skew, nrhs)
    x, hist, iters = run_ref(s, name, B, D, solver, extra, tmp)
    meta = {"dims": list(dims), "bs": bs, "seed": seed, "skew": skew, "B": B, "D": D,
            "solver": solver, "args": extra}
    np.savez_compressed(OUT / f"{name}.npz", x=x, hist=hist, iters=np.array(iters),
                        meta=np.array(json.dumps(meta)))
    return {"name": name, "iters": iters, "hist_len": len(hist)}


def run_config_case(name, spec, tmp: Path) -> dict:
    factory, B, D, solver, extra, full_x = spec
    s = getattr(systems, factory)()
    x, hist, iters = run_ref(s, name, B, D, solver, extra, tmp)
    sample_idx = np.arange(0, x.size, X_SAMPLE_STRIDE, dtype=np.int64)
    out = {"hist": hist, "iters": np.array(iters), "x_norm": np.array(np.linalg.norm(x)),
           "x_sample_idx": sample_idx, "x_sample": x[sample_idx],
           "meta": np.array(json.dumps({"system": factory, "n": s.n, "bs": s.bs, "B": B, "D": D,
                                        "solver": solver, "args": extra}))}
    if full_x:
        out["x"] = x
    if solver == "ichol0_pcg":
        # pCG's recursive residual is chaotic at rounding level: the oracle's
        # per-step spread under 1e-15 relative perturbations (three trials) is
        # stored with the history, since recomputing it takes minutes of numpy
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle.blocksp_oracle as O
        from parity import cg_envelope
        Ao = O.BSR.from_system(s)
        tol, maxit = float(extra[extra.index("--tol") + 1]), int(extra[extra.index("--maxit") + 1])
        out["hist_envelope"] = cg_envelope(Ao, s.b, tol, O.IChol0(Ao), maxit, hist)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    return {"name": name, "iters": iters, "hist_len": len(hist), "x_norm": float(np.linalg.norm(x))}


def run_algebra(A, name, B, D, mode, extra, tmp: Path):
    """The reference's block algebra on A (the driver writes the result matrix)."""
    f = tmp / f"{name}.bsps"
    systems.write_bsr(f, A)
    out = tmp / f"{name}.out.bsps"
    subprocess.run([str(EXE), str(f), "--B", str(B), "--D", str(D), "--solver", mode, "--x", str(out), *extra],
                   capture_output=True, text=True, check=True)
    return systems.read_bsr(out)


def eig_fixtures(tmp: Path) -> None:
    for name, (dims, bs, seed, skew, B, D, mode, iters, harm) in EIG_CASES.items():
        s = system_for(dims, bs, seed, skew)
        f = tmp / f"{name}.bsps"
        systems.write_bsr(f, s)
        r = subprocess.run([str(EXE), str(f), "--B", str(B), "--D", str(D), "--solver", mode, "--maxit", str(iters),
                            "--k", str(harm)], capture_output=True, text=True, check=True)
        ev = np.array([[float(v) for v in ln.split()[1:3]] for ln in r.stdout.splitlines() if ln.startswith("EIG ")])
        meta = {"dims": list(dims), "bs": bs, "seed": seed, "skew": skew, "mode": mode, "iters": iters,
                "harmonic": harm}
        np.savez_compressed(OUT / f"{name}.npz", wr=ev[:, 0], wi=ev[:, 1], meta=np.array(json.dumps(meta)))
        print({"name": name, "n": len(ev)})


def algebra_fixtures(tmp: Path) -> None:
    for name, (m, bs, nc, seed, B, D, mode, extra) in ALGEBRA_CASES.items():
        C = run_algebra(systems.random_blocksp(m, bs, nc, seed), name, B, D, mode, extra, tmp)
        meta = {"m": m, "bs": bs, "n_col": nc, "seed": seed, "mode": mode, "args": extra}
        np.savez_compressed(OUT / f"{name}.npz", row_ptr=C.row_ptr, col_idx=C.col_idx, vals=C.vals,
                            meta=np.array(json.dumps(meta)))
        print({"name": name, "nnzb": C.nnzb})
    ph = PSEUDO_HEAT
    A = systems.random_blocksp(ph["m"], ph["bs"], ph["n_col"], ph["seed"])
    S = run_algebra(A, "pseudo_heat", ph["B"], ph["D"], "pseudo_heat", ["--delta", repr(ph["delta"])], tmp)
    S.b = A.b
    flat = S.vals.reshape(-1)
    idx = np.arange(0, flat.size, X_SAMPLE_STRIDE, dtype=np.int64)
    out = {"row_ptr": S.row_ptr, "col_idx": S.col_idx, "vals_norm": np.array(np.linalg.norm(flat)),
           "vals_sample_idx": idx, "vals_sample": flat[idx], "meta": np.array(json.dumps(ph))}
    for tag, solver, args in (("pcg", "ichol0_pcg", ["--tol", "1e-10", "--maxit", "2000"]),
                              ("gmres", "ilu0_pgmres",
                               ["--tol", "1e-10", "--maxit", "5000", "--restart", "30", "--k", "10"])):
        x, hist, iters = run_ref(S, f"pseudo_heat_{tag}", ph["B"], ph["D"], solver, args, tmp)
        out[f"{tag}_x"], out[f"{tag}_hist"], out[f"{tag}_iters"] = x, hist, np.array(iters)
        print({"name": f"pseudo_heat_{tag}", "iters": iters})
    np.savez_compressed(OUT / "pseudo_heat_bs32.npz", **out)


def ldg_fixture() -> None:
    """The reference's LDG fixture as arrays plus its known-answer errors."""
    if not REF_MATS.exists():
        print("reference test_mats not present; LDG fixture not regenerated")
        return

    # these files start directly with the size line (the reference reads them
    # with start_line = 1, i.e. from the first line: blocksp_tests.hpp:326-336)
    def read_vec(path):
        lines = path.read_text().split("\n")
        n = int(lines[0].split()[0])
        return np.array([float(v) for v in lines[1:1 + n]])

    lines = (REF_MATS / "LDG_2D_vecLap.mtx").read_text().split("\n")
    m, n, nnz = map(int, lines[0].split())
    rows = np.empty(nnz, np.int32)
    cols = np.empty(nnz, np.int32)
    vals = np.empty(nnz)
    for k in range(nnz):
        i, j, v = lines[1 + k].split()
        rows[k], cols[k], vals[k] = int(i) - 1, int(j) - 1, float(v)
    b = read_vec(REF_MATS / "LDG_2D_vecLap_b.mtx")
    sol = read_vec(REF_MATS / "LDG_2D_vecLap_sol.mtx")
    errs = {}
    for B in (1, 2, 4, 8):
        r = subprocess.run([str(EXE), "--ldg", str(REF_MATS), "--B", str(B)], capture_output=True,
                           text=True, check=True)
        for line in r.stdout.splitlines():
            if line.startswith("ERRINF"):
                _, name, v = line.split()
                errs[f"B{B}_{name}"] = float(v)
    np.savez_compressed(OUT / "ldg_2d_veclap.npz", n=np.array(m), rows=rows, cols=cols, vals=vals, b=b,
                        sol=sol, ref_errinf=np.array(json.dumps(errs)))
    print("LDG errors", errs)


def main():
    if not EXE.exists():
        sys.exit("build the reference checker first: make -C oracle")
    if "--ldg-only" in sys.argv:
        ldg_fixture()
        return
    if "--algebra-only" in sys.argv:
        with tempfile.TemporaryDirectory() as d:
            algebra_fixtures(Path(d))
            eig_fixtures(Path(d))
        return
    configs_only = "--configs-only" in sys.argv
    with tempfile.TemporaryDirectory() as d:
        if not configs_only:
            for name, spec in CASES.items():
                print(run_case(name, spec, Path(d)))
            algebra_fixtures(Path(d))
        only = [a for a in sys.argv[1:] if not a.startswith("--")]
        for name, spec in CONFIG_CASES.items():
            if not only or name in only:
                print(run_config_case(name, spec, Path(d)), flush=True)
    if not configs_only:
        ldg_fixture()


if __name__ == "__main__":
    main()
