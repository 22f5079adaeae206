"""Runs the compiled reference oracle (oracle/_ref/ref_<NS>x<NT>_l<LEVELS>) on given inputs.

TEST INFRASTRUCTURE ONLY: imported by tests/, by tests/golden/make_golden.py and by the
CPU-baseline leg of bench.py; never by the product package.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"


def binary(ns: int, nt: int, levels: int) -> Path:
    return REF_DIR / f"ref_{ns}x{nt}_l{levels}"


# The reference checkout: AMG_REFERENCE_DIR, else a directory named `reference` beside this
# repository's root.
DEFAULT_REFDIR = os.environ.get("AMG_REFERENCE_DIR", str(HERE.parent.parent / "reference"))


def available(ns: int, nt: int, levels: int, refdir: str = DEFAULT_REFDIR) -> bool:
    """The binary exists, or the reference sources to build it do."""
    return binary(ns, nt, levels).exists() or (Path(refdir) / "src" / "amg.cpp").exists()


def build(ns: int, nt: int, levels: int, refdir: str = DEFAULT_REFDIR) -> Path:
    b = binary(ns, nt, levels)
    # (re)built when missing or older than the harness or the MPI stand-in
    newest = max((HERE / f).stat().st_mtime for f in ("ref_harness.cpp", "mpi_shim/mpi.h", "build_ref.sh"))
    if not b.exists() or b.stat().st_mtime < newest:
        subprocess.run([str(HERE / "build_ref.sh"), str(ns), str(nt), str(levels), refdir],
                       check=True, capture_output=True)
    return b


def params_text(rows) -> str:
    return "\n".join(" ".join(str(int(v)) for v in r) for r in rows) + "\n"


def read_outputs(workdir: Path) -> dict:
    out = {}
    man = workdir / "manifest.txt"
    if man.exists():
        for line in man.read_text().split("\n"):
            if not line.strip():
                continue
            name, dt, *shape = line.split()
            dtype = {"c16": np.complex128, "i4": np.int32}[dt]
            a = np.fromfile(workdir / f"{name}.bin", dtype=dtype)
            out[name] = a.reshape([int(s) for s in shape])
    info = workdir / "info.txt"
    if info.exists():
        for line in info.read_text().split("\n"):
            if line.strip():
                k, v = line.split()
                out["info:" + k] = float(v)
    return out


def run(ns: int, nt: int, rows, gauge: np.ndarray, rhs: np.ndarray, *, m0: float,
        cycle: int = 1, nit: int = 0, sap_tv_iters: int = 4, nu1: int = 0, nu2: int = 2,
        solve: int = 1, phases: int = 0, dump_hierarchy: int = 1, dphi_reps: int = 0,
        dphi_only: int = 0, outer_iteration_reps: int = 0, hierarchy: dict | None = None, probes=None,
        workdir: str | None = None, timeout: float = 3600, krylov: int = 0, ranks: int = 1,
        ranks_after_setup: int = 0, drill_exit_rank: int = -1, solve_reps: int = 0,
        solve_budget_seconds: float = 0.0) -> dict:
    """Writes the job, runs the binary for (ns, nt, len(rows)+1 levels), returns its dumps
    (rank 0's).  ranks > 1 runs the reference's MPI layout as that many processes on this
    host (oracle/mpi_shim/mpi.h): its SAP block solves split among them; with
    ranks_after_setup = 1 the ranks start after the set-up, just before the timed outer
    iterations (they then share the set-up's memory).  solve_reps = R > 0 runs the complete
    FGMRES_AMG solve up to R times on the one set-up (or on a loaded `hierarchy`), timing each
    (info:solve_seconds_<r>, info:iterations_<r>, info:solves_done), stopping early once
    another solve would take rank 0's total past solve_budget_seconds (0: no budget); 0 runs
    one solve (no per-solve keys) or, with a loaded hierarchy, the outer-iteration sample.
    drill_exit_rank = r > 0 makes rank r leave before its first collective (the stand-in's
    failure drill)."""
    levels = len(rows) + 1
    b = binary(ns, nt, levels)
    if not b.exists():
        raise FileNotFoundError(f"{b} not built (oracle/build_ref.sh {ns} {nt} {levels})")
    tmp = None
    if workdir is None:
        tmp = tempfile.TemporaryDirectory(prefix="oracle_")
        workdir = tmp.name
    wd = Path(workdir)
    wd.mkdir(parents=True, exist_ok=True)
    (wd / "params.dat").write_text(params_text(rows))
    job = dict(m0=repr(float(m0)), cycle=cycle, nit=nit, sap_tv_iters=sap_tv_iters, nu1=nu1,
               nu2=nu2, solve=solve, phases=phases, dump_hierarchy=dump_hierarchy,
               dphi_reps=dphi_reps, dphi_only=dphi_only,
               outer_iteration_reps=outer_iteration_reps, krylov=krylov, ranks=ranks,
               ranks_after_setup=ranks_after_setup, drill_exit_rank=drill_exit_rank, solve_reps=solve_reps,
               solve_budget_seconds=solve_budget_seconds)
    (wd / "job.txt").write_text("".join(f"{k} {v}\n" for k, v in job.items()))
    np.ascontiguousarray(gauge, dtype=np.complex128).tofile(wd / "gauge.bin")
    np.ascontiguousarray(rhs, dtype=np.complex128).tofile(wd / "rhs.bin")
    if hierarchy is not None:
        # {"tv": {l: W[Ntest][N_l][DOF_l]}, "links": {l: (G1, G2, G3)}} in the reference layouts
        job["load_hierarchy"] = 1
        (wd / "job.txt").write_text("".join(f"{k} {v}\n" for k, v in job.items()))
        for l, W in hierarchy["tv"].items():
            np.ascontiguousarray(W, dtype=np.complex128).tofile(wd / f"hier_tv_l{l}.bin")
        for l, gs in hierarchy["links"].items():
            for name, G in zip(("g1", "g2", "g3"), gs):
                np.ascontiguousarray(G, dtype=np.complex128).tofile(wd / f"hier_{name}_l{l}.bin")
    for l, p in (probes or {}).items():
        np.ascontiguousarray(p, dtype=np.complex128).tofile(wd / f"probe_l{l}.bin")
    proc = subprocess.run([str(b), str(wd)], cwd=str(wd), capture_output=True, text=True,
                          timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"oracle failed ({proc.returncode}): {proc.stderr[-2000:]}")
    out = read_outputs(wd)
    out["stdout"] = proc.stdout
    res = list(wd.glob("Residuals_FGMRES_*.res"))
    if res:
        out["residual_history"] = np.loadtxt(res[0])[:, 1].reshape(-1)
    if tmp is not None:
        tmp.cleanup()
    return out
