"""Generates the golden fixtures in this directory from the compiled reference oracle.

Run in a container that has the reference sources (it builds oracle/_ref binaries with
oracle/build_ref.sh) from the repository root:

    python tests/golden/make_golden.py

Each fixture is one .npz holding the inputs (gauge field, source, probe vectors) and the
reference's outputs on them: index maps, D_phi / D_dagger_phi, the set-up hierarchy (test
vectors and coarse links), per-level operator / P / P^dagger / SAP / GMRES probes, one
preconditioner application, and the outer solve (x, iteration count, residual history).
Large arrays are dropped for the bigger lattices to keep the files small.

The Krylov fixture (KRYLOV) holds the reference's comparison solvers on one source: the
conjugate_gradient solution of D D^dagger y = phi, the bi_cgstab solution of D x = phi, the
unpreconditioned FGMRES_fine_level(20, 50) solution and the FGMRES_SAP(20, 50) solution (the
global SAP object given the gauge field by its set_params), with their iteration counts.

The solve fixtures (SOLVES) hold complete reference solves at the workload sizes (256x256,
512x512, 1024x1024), stored small: the iteration count, the true residual, the residual
history, |x| and x and D_phi(b) on a strided subsample of the sites; the gauge field and the
source are regenerated from the seeds in their meta.

The adjoint fixture (ADJOINT) holds the reference's two solves behind the gradient of
L = Re(eta^dagger D^{-1} b): x = D^{-1} b and y = D^{-1} gamma5 eta (so lambda = gamma5 y),
each a full FGMRES_AMG run of the reference; the gauge field and the two sources are
regenerated from the seeds in its meta.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from amg_schwingermodel_b200.inputs import gauge_angles, gauge_field, gaussian_spinor  # noqa: E402
from oracle import ref_runner  # noqa: E402
from oracle.restatement import read_parameters  # noqa: E402

CONFIGS = {
    # name: (ns, rows, beta, m0, seed, job overrides, keep large arrays)
    "c16_l2_k": (16, [[0, 4, 4, 4, 2, 2]], 2.0, -0.1, 11, {}, True),
    "c32_l3_k": (32, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], 3.0, -0.1, 12, {}, True),
    "c32_l3_v_nu1": (32, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], 3.0, -0.1, 13,
                     {"cycle": 0, "nu1": 1}, False),
    "c32_l3_k_nit1": (32, [[0, 4, 4, 6, 2, 2], [1, 2, 2, 6, 2, 2]], 2.0, -0.1, 14, {"nit": 1}, False),
    "c64_l2_k": (64, [[0, 8, 8, 10, 4, 4]], 2.0, -0.1, 1, {}, False),
    "c64_l4_k": (64, [[0, 8, 8, 8, 4, 4], [1, 4, 4, 8, 4, 4], [2, 2, 2, 8, 2, 2]], 4.0, -0.05, 15, {}, False),
    # SAP blocks of 32x32 and 16x32 sites (the block shapes of the 1024x1024 benchmark rows)
    "c64_l3_sap1024": (64, [[0, 8, 8, 8, 2, 2], [1, 4, 4, 8, 2, 2]], 3.0, -0.1, 16, {}, False),
    "c64_l2_sap512": (64, [[0, 8, 8, 8, 4, 2]], 4.0, -0.05, 17, {}, False),
}

# name: (ns, rows, beta, m0, seed); inputs: theta = gauge_angles(ns, ns, beta, seed),
# b = gaussian_spinor(N, 2, seed + 1000), eta = gaussian_spinor(N, 2, seed + 3000)
ADJOINT = {
    "adj128_l3": (128, [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]], 2.0, -0.1, 21),
}

# The comparison solvers conjugate_gradient (on D D^dagger), bi_cgstab and the
# unpreconditioned FGMRES_fine_level of the reference (src/conjugate_gradient.cpp:5-65,
# src/bi_cgstab.cpp:5-89, include/fgmres.h:126-148) on one source:
# name: (ns, rows, beta, m0, seed); U = gauge_field(ns, ns, beta, seed),
# phi = gaussian_spinor(N, 2, seed + 1); iteration counts from the reference's own output.
KRYLOV = {
    "krylov32": (32, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], 3.0, -0.1, 31),
    "krylov64": (64, [[0, 8, 8, 8, 4, 4]], 2.0, -0.05, 43),
}

# Complete FGMRES_AMG solves (src/tests.cpp:67-82) at the workload configurations:
# name: (ns, rows, beta, m0, seed); U = gauge_field(ns, ns, beta, seed),
# b = gaussian_spinor(N, 2, seed + 1000).
SOLVES = {
    # 256x256, 3 levels, aggregation 8x8 then 4x4 blocks, Nv = 12, 4x4 SAP blocks, beta = 3
    "solve256_l3": (256, [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]], 3.0, -0.05, 51),
    # 1024x1024, 4 levels, Nv = 16, beta = 4, with the benchmark rows (32x32-site SAP blocks)
    "solve1024_l4": (1024, [[0, 8, 8, 16, 32, 32], [1, 4, 4, 16, 4, 4], [2, 2, 2, 16, 2, 2]], 4.0, -0.05, 52),
    # ... and with the reference-style rows (4x4 SAP blocks of 256x256 sites)
    "solve1024_l4_refrows": (1024, [[0, 8, 8, 16, 4, 4], [1, 4, 4, 16, 4, 4], [2, 2, 2, 16, 2, 2]], 4.0, -0.05, 53),
    # one configuration per lattice size of the uneven batch (128^2 at beta 2, 256^2 at 3,
    # 512^2 at 4): 32x32-site SAP blocks, aggregation 8x8 then 4x4 blocks, Nv = 12
    "solve128_l3_b2": (128, [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]], 2.0, -0.05, 54),
    "solve256_l3_b3": (256, [[0, 8, 8, 12, 8, 8], [1, 4, 4, 12, 4, 4]], 3.0, -0.05, 55),
    "solve512_l3_b4": (512, [[0, 8, 8, 12, 16, 16], [1, 4, 4, 12, 4, 4]], 4.0, -0.05, 56),
}
# sites kept of x and D_phi(b) in a solve fixture (every (N // SAMPLE_SITES)-th site)
SAMPLE_SITES = 16384

SMALL_KEYS_ALWAYS = ("dphi", "ddagphi", "x", "cycle0_rhs")


def make(name: str, cfg) -> dict:
    ns, rows, beta, m0, seed, over, keep_large = cfg
    lps = read_parameters(ns, ns, rows)
    L = len(lps)
    ref_runner.build(ns, ns, L)
    U = gauge_field(ns, ns, beta, seed)
    b = gaussian_spinor(ns * ns, 2, seed + 1000)
    probes = {l: gaussian_spinor(lp.n, lp.dof, seed + 2000 + l) for l, lp in enumerate(lps)}
    job = dict(cycle=1, nit=0, nu1=0, nu2=2, sap_tv_iters=4)
    job.update(over)
    out = ref_runner.run(ns, ns, rows, U, b, m0=m0, phases=1, probes=probes, **job)
    arrays = {"gauge": U, "rhs": b}
    for l, p in probes.items():
        arrays[f"probe_l{l}"] = p
    for k, v in out.items():
        if not isinstance(v, np.ndarray) or k.startswith("init_tv"):
            continue
        if not keep_large and k.startswith("tv_l"):
            continue
        if not keep_large and k.startswith(("g1_l", "g2_l", "g3_l")) and v.nbytes > 300_000:
            continue
        arrays[k] = v
    meta = dict(ns=ns, nt=ns, rows=rows, beta=beta, m0=m0, seed=seed, job=job,
                iterations=int(out["info:iterations"]),
                true_rel_residual=out["info:true_rel_residual"],
                sap_ret={l: int(out.get(f"info:sap_ret_l{l}", -1)) for l in range(L - 1)},
                gmres_iters={l: int(out.get(f"info:gmres_iters_l{l}", -1)) for l in range(1, L)},
                kfgmres1_iters=int(out.get("info:kfgmres1_iters", -1)))
    arrays["meta"] = np.array(json.dumps(meta))
    return arrays


def sample_sites(n: int) -> np.ndarray:
    """The site indices a solve fixture keeps: every (n // SAMPLE_SITES)-th site."""
    return np.arange(0, n, max(1, n // SAMPLE_SITES))


def make_solve(name: str, cfg) -> dict:
    ns, rows, beta, m0, seed = cfg
    ref_runner.build(ns, ns, len(rows) + 1)
    N = ns * ns
    U = gauge_field(ns, ns, beta, seed)
    b = gaussian_spinor(N, 2, seed + 1000)
    job = dict(cycle=1, nit=0, nu1=0, nu2=2, sap_tv_iters=4, dump_hierarchy=0)
    out = ref_runner.run(ns, ns, rows, U, b, m0=m0, timeout=4 * 3600, **job)
    idx = sample_sites(N)
    meta = dict(ns=ns, nt=ns, rows=rows, beta=beta, m0=m0, seed=seed, job=job,
                iterations=int(out["info:iterations"]), true_rel_residual=out["info:true_rel_residual"],
                setup_seconds=out["info:setup_seconds"], solve_seconds=out["info:solve_seconds"],
                x_norm=float(np.linalg.norm(out["x"])))
    return {"sites": idx, "x_sample": out["x"][idx], "dphi_sample": out["dphi"][idx],
            "residual_history": out["residual_history"], "meta": np.array(json.dumps(meta))}


def make_adjoint(name: str, cfg) -> dict:
    ns, rows, beta, m0, seed = cfg
    L = len(rows) + 1
    ref_runner.build(ns, ns, L)
    N = ns * ns
    U = np.exp(1j * gauge_angles(ns, ns, beta, seed))
    b = gaussian_spinor(N, 2, seed + 1000)
    eta = gaussian_spinor(N, 2, seed + 3000)
    g5eta = eta.copy()
    g5eta[:, 1] *= -1
    job = dict(cycle=1, nit=0, nu1=0, nu2=2, sap_tv_iters=4, dump_hierarchy=0)
    ox = ref_runner.run(ns, ns, rows, U, b, m0=m0, **job)
    oy = ref_runner.run(ns, ns, rows, U, g5eta, m0=m0, **job)
    meta = dict(ns=ns, nt=ns, rows=rows, beta=beta, m0=m0, seed=seed, job=job,
                iterations_x=int(ox["info:iterations"]), iterations_y=int(oy["info:iterations"]),
                true_rel_residual_x=ox["info:true_rel_residual"], true_rel_residual_y=oy["info:true_rel_residual"])
    return {"x": ox["x"], "y": oy["x"], "meta": np.array(json.dumps(meta))}


def make_krylov(name: str, cfg) -> dict:
    ns, rows, beta, m0, seed = cfg
    ref_runner.build(ns, ns, len(rows) + 1)
    U = gauge_field(ns, ns, beta, seed)
    phi = gaussian_spinor(ns * ns, 2, seed + 1)
    out = ref_runner.run(ns, ns, rows, U, phi, m0=m0, krylov=1, dump_hierarchy=0)
    cg = re.search(r"^Converged in (\d+) iterations", out["stdout"], re.M)
    bi = re.search(r"^Bi-CG-stab for D converged in (\d+) iterations", out["stdout"], re.M)
    meta = dict(ns=ns, nt=ns, rows=rows, beta=beta, m0=m0, seed=seed,
                cg_iterations=int(cg.group(1)), bicg_iterations=int(bi.group(1)),
                gmres_iterations=int(out["info:gmres_iterations"]),
                sap_iterations=int(out["info:sap_iterations"]))
    return {"cg_x": out["cg_x"], "bicg_x": out["bicg_x"], "gmres_x": out["gmres_x"], "sap_x": out["sap_x"],
            "meta": np.array(json.dumps(meta))}


def main(names=None):
    here = Path(__file__).resolve().parent
    for name, cfg in SOLVES.items():
        if names and name not in names:
            continue
        arrays = make_solve(name, cfg)
        np.savez_compressed(here / f"{name}.npz", **arrays)
        print(name, (here / f"{name}.npz").stat().st_size // 1024, "KiB")
    for name, cfg in KRYLOV.items():
        if names and name not in names:
            continue
        arrays = make_krylov(name, cfg)
        np.savez_compressed(here / f"{name}.npz", **arrays)
        print(name, (here / f"{name}.npz").stat().st_size // 1024, "KiB")
    for name, cfg in ADJOINT.items():
        if names and name not in names:
            continue
        arrays = make_adjoint(name, cfg)
        np.savez_compressed(here / f"{name}.npz", **arrays)
        print(name, (here / f"{name}.npz").stat().st_size // 1024, "KiB")
    for name, cfg in CONFIGS.items():
        if names and name not in names:
            continue
        arrays = make(name, cfg)
        np.savez_compressed(here / f"{name}.npz", **arrays)
        print(name, (here / f"{name}.npz").stat().st_size // 1024, "KiB")


if __name__ == "__main__":
    main(sys.argv[1:])
