#!/usr/bin/env python
"""Benchmark: 1024x1024 Schwinger-model DD-alpha-AMG solves per second to FP64 relative
residual <= 1e-10 (4 levels, Nv = 16, beta = 4, m0 = -0.05), mixed precision with batched
sources against the plain FP64 drop-in, plus the fine D-apply bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--rhs R] [--precision mixed|f64] [--no-cpu] [--no-extras] [--transfers]

One step = one batched solve of R seeded complex-Gaussian sources on one seeded gauge
field per GPU (inputs resident in HBM; the working set of a step is far above the 126 MB
L2).  With N GPUs every rank solves its own gauge field and sources (replicas, weak
scaling); timing is CUDA events on the solver's stream, max over ranks.  Rank 0 prints one
JSON line.  At N = 1 the line also carries the FP64 forms (one source and the same batch),
the reference-style blocking at 1024^2, the 256^2 FP64-vs-mixed comparison, and the uneven
batch of 24 configurations (128^2 / 256^2 / 512^2) x 32 sources.

`--impl reference` times the reference's own CPU code (compiled from its unmodified sources
into oracle/_ref) on the same workload: its own complete set-up, then complete FGMRES_AMG
solves (one untimed, then up to K timed within a time budget), run in the reference's MPI
layout on up to 8 host cores; `steps` states how many solves were timed.
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

NX = NT = 1024
ROWS = [[0, 8, 8, 16, 32, 32], [1, 4, 4, 16, 4, 4], [2, 2, 2, 16, 2, 2]]
# the reference-style rows at 1024^2: 4x4 SAP blocks of 256x256 sites
REF_ROWS = [[0, 8, 8, 16, 4, 4], [1, 4, 4, 16, 4, 4], [2, 2, 2, 16, 2, 2]]
BETA, M0, TOL = 4.0, -0.05, 1e-10
METRIC = "1024^2 solves/s at FP64 resid <=1e-10: mixed+batched vs FP64 GPU; D-apply GB/s"
UNIT = "solves/s"
WORKLOAD = "schwinger_wilson_1024x1024_L4_Nv16_beta4_m0-0.05"
# 256x256, 3 levels, aggregation 8x8 then 4x4 blocks, Nv = 12, 4x4 SAP blocks, beta = 3
C2_NS, C2_ROWS, C2_BETA, C2_SEED = 256, [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]], 3.0, 51
# the uneven batch: 8 configurations each at 128^2, 256^2 and 512^2 (beta cycling through 2, 3,
# 4), 32 sources each, 32x32-site SAP blocks, aggregation 8x8 then 4x4 blocks, Nv = 12
BATCH_ROWS = {128: [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]],
              256: [[0, 8, 8, 12, 8, 8], [1, 4, 4, 12, 4, 4]],
              512: [[0, 8, 8, 12, 16, 16], [1, 4, 4, 12, 4, 4]]}
BATCH_PER_SIZE, BATCH_RHS = 8, 32

# Algorithmic FP32 flops of one fine SAP block solve, per site: GMRES(5) restarted 5 times
# from x0 = b (include/sap.h:27-47; the 1e-3 tolerance is never met on these blocks, so all
# 25 Arnoldi steps run).  With F_D = 60 flops per site for the block operator (the fine D
# apply's count), 16 per site for an axpy or a dot over the two spin components, 8 for a
# norm and 4 for a real scaling: the initial residual b - D_B b with its norm, 72; per
# restart cycle the Arnoldi steps j = 0..4, sum_j (60 + 32 (j + 1) + 8 + 4) = 840, the update
# x += sum_j y_j V_j, 80, and the residual with its norm, 72.  72 + 5 * 992 = 5032.
SAP_FLOPS_PER_SITE = 5032
# DRAM bytes (read + write) of one fine SAP launch per (block, source) it solves, from an ncu
# capture (dram__bytes_read.sum, dram__bytes_write.sum) of this workload's SAP kernel at 32
# sources: 542.37 MB read + 227.01 MB written by a launch of 16384 block-sources.
SAP_DRAM_BYTES_PER_BLOCK_SOURCE = (542.37e6 + 227.01e6) / 16384
FP32_LANES_PER_SM = 128


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.flush()
        lines = [l.split(",") for l in Path(self.f.name).read_text().strip().split("\n") if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in lines:
            if len(l) < 9:
                continue
            try:
                sm.append(float(l[1]))
                mx.append(float(l[2]))
            except ValueError:
                continue
            for n, v in zip(names, l[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    """One process per GPU (torchrun env).  NCCL between GPUs; gloo when CUDA is absent
    (the multi-rank plumbing is tested that way on CPU)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    """The largest of the ranks' values (device times are reported as the max over ranks)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seeds(rank: int) -> tuple[int, int]:
    """Seeds of the gauge field and the sources of one rank: every rank solves its own
    configuration (replicas, no data exchanged)."""
    return 1000 + rank, 2000 + rank


def hierarchy_for_reference(ctx) -> dict:
    """The set-up hierarchy in the reference's layouts (test vectors, coarse links)."""
    tv = {l: ctx.test_vectors(l) for l in range(ctx.levels - 1)}
    links = {l: ctx.coarse_links(l) for l in range(1, ctx.levels)}
    return {"tv": tv, "links": links}


def _read(path):
    try:
        return Path(path).read_text().split()
    except OSError:
        return None


def host_cores() -> int:
    """Usable host cores: the affinity mask, bounded by a cgroup CPU quota (v2, then v1)."""
    cores = len(os.sched_getaffinity(0))
    q = _read("/sys/fs/cgroup/cpu.max")
    if q and q[0] != "max":
        cores = min(cores, max(1, int(q[0]) // int(q[1])))
    q, per = _read("/sys/fs/cgroup/cpu/cpu.cfs_quota_us"), _read("/sys/fs/cgroup/cpu/cpu.cfs_period_us")
    if q and per and int(q[0]) > 0:
        cores = min(cores, max(1, int(q[0]) // int(per[0])))
    return cores


def host_available_bytes() -> int:
    """MemAvailable, bounded by a cgroup memory limit (v2, then v1); 0 if unknown."""
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) * 1024 for l in f if l.startswith("MemAvailable:"))
    except (OSError, StopIteration, ValueError):
        return 0
    for lim, use in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        a, b = _read(lim), _read(use)
        if a and b and a[0] != "max" and int(a[0]) < (1 << 60):
            avail = min(avail, int(a[0]) - int(b[0]))
    return avail


def reference_layout() -> tuple[int, bool]:
    """Ranks for the reference's CPU runs (its MPI layout as processes on this host, the SAP
    block solves split among them) and whether they start before the set-up.  A 1024x1024
    4-level run of the reference holds about 13 GB per rank when every rank runs the set-up;
    ranks started after the set-up share its pages, about 20 GB for the first and 6 GB for
    each further one.  Up to 8 ranks (the usable cores), within half the available memory;
    the ranks start before the set-up (which it then splits too) when all of them fit that
    way.  AMG_REF_RANKS overrides the count (ranks then start after the set-up)."""
    if os.environ.get("AMG_REF_RANKS"):
        return max(1, int(os.environ["AMG_REF_RANKS"])), False
    cores = min(host_cores(), 8)
    avail = host_available_bytes()
    if avail <= 0:
        return 1, False
    early = int((0.5 * avail) // 13e9)
    if early >= cores:
        return cores, True
    late = int((0.5 * avail - 20e9) // 6e9) + 1
    return max(1, min(cores, late)), False


def run_reference_job(ranks: int, early: bool, rows=ROWS, **kw):
    """ref_runner.run on the bench lattice with `ranks` ranks (started before the set-up if
    `early`, else after it); if that run fails (a rank lost, e.g. to memory pressure) it is
    repeated with one rank.  Returns (outputs, ranks used)."""
    from oracle import ref_runner
    if ranks > 1:
        try:
            return ref_runner.run(NX, NT, rows, ranks=ranks, ranks_after_setup=0 if early else 1, **kw), ranks
        except RuntimeError as e:
            print(f"reference with {ranks} ranks failed ({str(e)[:200]}); one rank", file=sys.stderr)
    return ref_runner.run(NX, NT, rows, **kw), 1


def run_reference(args, world, rank):
    """The reference's own CPU code on this workload: its complete set-up (test-vector
    smoothing included, as FGMRES_AMG's constructor runs it), then complete FGMRES_AMG solves
    from x0 = 0: one untimed, then up to `steps` timed, stopping early once another solve
    would exceed the time budget (AMG_REF_SOLVE_BUDGET_S, default 150 s).  solves/s = timed
    solves / their summed time."""
    if rank != 0:
        return
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    from oracle import ref_runner
    if not ref_runner.binary(NX, NT, len(ROWS) + 1).exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref binary for 1024x1024 L4 not built"}))
        return
    gseed, bseed = replica_seeds(0)
    U = gauge_field(NX, NT, BETA, gseed)
    b0 = gaussian_spinor(NX * NT, 2, bseed)
    budget = float(os.environ.get("AMG_REF_SOLVE_BUDGET_S", "150"))
    ranks, early = reference_layout()
    t0 = time.time()
    out, ranks = run_reference_job(ranks, early, gauge=U, rhs=b0, m0=M0, solve=1, dump_hierarchy=0, dphi_reps=20,
                                   solve_reps=1 + args.steps, solve_budget_seconds=budget, timeout=3 * 3600)
    done = int(out["info:solves_done"])
    times = [out[f"info:solve_seconds_{r}"] for r in range(done)]
    iters = [int(out[f"info:iterations_{r}"]) for r in range(done)]
    warm = 1 if done > 1 else 0
    timed = times[warm:]
    value = len(timed) / sum(timed)
    sample = (f"complete reference FGMRES_AMG solves (x0 = 0 to FP64 relative residual 1e-10) at {NX}x{NT}, 4 levels, "
              f"after its own complete set-up ({out['info:setup_seconds']:.1f} s); {warm} untimed + {len(timed)} timed "
              f"within a {budget:.0f} s budget: {statistics.mean(timed):.2f} s per solve, {iters[-1]} iterations; "
              f"{ranks} rank(s) of its MPI layout, one core each (SAP blocks split among them"
              f"{', set-up included' if early and ranks > 1 else '; ranks started after the set-up'})")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": len(timed),
            "warmup": warm, "ms_per_step": 1e3 * statistics.mean(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "lattice": [NX, NT], "levels": 4, "rows": ROWS, "nrhs": 1,
                       "steps_requested": args.steps, "solve_budget_s": budget},
            "iterations": iters, "true_rel_residual": out.get("info:true_rel_residual"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ranks, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "dphi_s_per_apply": out.get("info:dphi_seconds_per_apply"),
            "ref_setup_s": out.get("info:setup_seconds"), "wall_s": time.time() - t0}
    print(json.dumps(line))


def cpu_reference_solve(U, b0, hierarchy, timeout: float = 900) -> dict:
    """Times complete FGMRES_AMG solves of the reference's own code (oracle/_ref) on this
    workload, on the hierarchy the GPU FP64 set-up built (loaded into the reference's
    AlgebraicMG, its own set-up skipped): one solve, a second one if both fit 30 s."""
    from oracle import ref_runner
    b = ref_runner.binary(NX, NT, len(ROWS) + 1)
    if not b.exists():
        return {"error": f"{b.name} not built"}
    ranks, _ = reference_layout()
    out, used = run_reference_job(ranks, False, gauge=U, rhs=b0, m0=M0, solve=1, dump_hierarchy=0, dphi_reps=20,
                                  hierarchy=hierarchy, solve_reps=2, solve_budget_seconds=30, timeout=timeout)
    done = int(out["info:solves_done"])
    return dict(t=out[f"info:solve_seconds_{done - 1}"], iterations=int(out["info:iterations"]),
                residual=out["info:true_rel_residual"], dphi_s=out.get("info:dphi_seconds_per_apply"), ranks=used,
                solves=done)


def timed_solves(ctx, b_ptr, x_ptr, nrhs, steps, warmup):
    """warmup + steps batched solves on device buffers; returns (ms per step, last infos)."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    infos = None
    for _ in range(warmup):
        infos = ctx.solve_dev(b_ptr, x_ptr, nrhs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        infos = ctx.solve_dev(b_ptr, x_ptr, nrhs)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, infos


def line_config2(local):
    """256x256, 3 levels (aggregation 8x8 then 4x4 blocks, Nv = 12, beta = 3, m0 = -0.05), one
    source: the FP64 drop-in against the mixed form, iterations beside the reference's."""
    import torch

    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    N = C2_NS * C2_NS
    U = gauge_field(C2_NS, C2_NS, C2_BETA, C2_SEED)
    b = torch.from_numpy(gaussian_spinor(N, 2, C2_SEED + 1000).view(np.float64).copy()).to(f"cuda:{local}")
    res, xs = {}, {}
    for name, prec in (("f64", 0), ("mixed", 1)):
        with AMGContext(C2_NS, C2_NS, C2_ROWS, M0, precision=prec, max_rhs=1, device=local) as ctx:
            ctx.set_gauge(U)
            setup_ms = ctx.setup()
            x = torch.empty_like(b)
            ms, infos = timed_solves(ctx, b.data_ptr(), x.data_ptr(), 1, 10, 3)
            xs[name] = x.cpu().numpy()
            res[name] = {"value": 1e3 / ms, "unit": UNIT, "iterations": infos[0]["iterations"],
                         "rel_residual": infos[0]["rel_residual"], "setup_s": setup_ms / 1e3}
    res["mixed"]["err_vs_fp64"] = float(np.linalg.norm(xs["mixed"] - xs["f64"]) / np.linalg.norm(xs["f64"]))
    fx = ROOT / "tests" / "golden" / "solve256_l3.npz"
    ref_it = json.loads(str(np.load(fx)["meta"]))["iterations"] if fx.exists() else None
    return {"workload": "schwinger_wilson_256x256_L3_Nv12_beta3_m0-0.05", "rows": C2_ROWS, "nrhs": 1,
            "reference_iterations": ref_it, **res, "speedup_mixed_vs_f64": res["mixed"]["value"] / res["f64"]["value"]}


def line_reference_rows(local, R):
    """1024x1024 with the reference-style rows (SAP blocks of 256x256 sites, solved by the
    any-shape block kernel), mixed precision, R sources: iterations and solves/s."""
    import torch

    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field
    N = NX * NT
    U = gauge_field(NX, NT, BETA, replica_seeds(0)[0])
    g = torch.Generator(device=f"cuda:{local}").manual_seed(7)
    b = torch.randn(R, N, 2, 2, dtype=torch.float64, device=f"cuda:{local}", generator=g)
    x = torch.empty_like(b)
    with AMGContext(NX, NT, REF_ROWS, M0, precision=1, max_rhs=R, device=local) as ctx:
        ctx.set_gauge(U)
        setup_ms = ctx.setup()
        ms, infos = timed_solves(ctx, b.data_ptr(), x.data_ptr(), R, 1, 1)
        tuned = ctx.autotune_info()
    fx = ROOT / "tests" / "golden" / "solve1024_l4_refrows.npz"
    ref_it = json.loads(str(np.load(fx)["meta"]))["iterations"] if fx.exists() else None
    return {"rows": REF_ROWS, "nrhs": R, "precision": "mixed", "value": R * 1e3 / ms, "unit": UNIT,
            "iterations": sorted({i["iterations"] for i in infos}),
            "max_rel_residual": max(i["rel_residual"] for i in infos), "setup_s": setup_ms / 1e3,
            "reference_iterations_fp64_one_source": ref_it, "autotune": tuned}


def line_uneven_batch(local, steps):
    """24 configurations (8 each at 128^2, 256^2 and 512^2, beta cycling through 2, 3, 4,
    m0 = -0.05), 32 sources each, mixed precision, solved together by amg_solve_many_dev."""
    import torch

    from amg_schwingermodel_b200 import AMGContext, solve_many_dev
    from amg_schwingermodel_b200.inputs import gauge_field
    dev = f"cuda:{local}"
    ctxs, bufs = [], []
    setup_s = 0.0
    try:
        k = 0
        for ns, rows in BATCH_ROWS.items():
            for i in range(BATCH_PER_SIZE):
                beta = (2.0, 3.0, 4.0)[i % 3]
                ctx = AMGContext(ns, ns, rows, M0, precision=1, max_rhs=BATCH_RHS, device=local)
                ctxs.append(ctx)
                ctx.set_gauge(gauge_field(ns, ns, beta, 3000 + k))
                setup_s += ctx.setup() / 1e3
                g = torch.Generator(device=dev).manual_seed(4000 + k)
                b = torch.randn(BATCH_RHS, ns * ns, 2, 2, dtype=torch.float64, device=dev, generator=g)
                bufs.append((b, torch.empty_like(b)))
                k += 1
        bp = [b.data_ptr() for b, _ in bufs]
        xp = [x.data_ptr() for _, x in bufs]
        nr = [BATCH_RHS] * len(ctxs)
        infos = solve_many_dev(ctxs, bp, xp, nr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            infos = solve_many_dev(ctxs, bp, xp, nr)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / steps
    finally:
        for c in ctxs:
            c.close()
    allinfo = [i for inf in infos for i in inf]
    per_size = {}
    for (ns, _), inf in zip([(ns, i) for ns in BATCH_ROWS for i in range(BATCH_PER_SIZE)], infos):
        per_size.setdefault(str(ns), set()).update(i["iterations"] for i in inf)
    return {"configurations": len(ctxs), "sizes": list(BATCH_ROWS), "nrhs_each": BATCH_RHS,
            "rows": {str(k): v for k, v in BATCH_ROWS.items()}, "precision": "mixed",
            "value": len(allinfo) / dt, "unit": UNIT, "s_per_step": dt, "steps": steps,
            "iterations_by_size": {k: sorted(v) for k, v in per_size.items()},
            "max_rel_residual": max(i["rel_residual"] for i in allinfo),
            "converged": all(i["converged"] for i in allinfo), "setup_s_total": setup_s,
            "timing": "host clock around amg_solve_many_dev calls (the contexts run on their own streams; the call "
                      "returns after every context's solve has finished)"}


def run_transfers(args, local):
    """The mixed form's level-0 transfers alone at the benchmark's shape (1024^2, 8x8
    aggregation blocks of 128x128 sites, 16 test vectors, R sources): restriction and
    prolongation through amg_restrict0_mixed_dev / amg_prolong0_mixed_dev on device buffers,
    warm-up then timed launches with CUDA events on the context's stream; a few GB on the
    device (no solve buffers), the size an ncu capture of these kernels takes."""
    import ctypes as C

    import torch

    from amg_schwingermodel_b200 import AMGContext, _lib
    from amg_schwingermodel_b200.inputs import gauge_field
    torch.cuda.set_device(local)
    R, N = args.rhs, NX * NT
    ctx = AMGContext(NX, NT, ROWS, M0, precision=1, max_rhs=R, device=local)
    ctx.set_gauge(gauge_field(NX, NT, BETA, replica_seeds(0)[0]))
    ctx.setup()
    nblk, ntest = ROWS[0][1] * ROWS[0][2], ROWS[0][3]
    g = torch.Generator(device=f"cuda:{local}").manual_seed(3)
    v = torch.randn(R, N, 2, dtype=torch.complex64, device=f"cuda:{local}", generator=g)
    vc = torch.randn(R, nblk, 2 * ntest, dtype=torch.complex64, device=f"cuda:{local}", generator=g)
    out = torch.empty_like(vc)
    psi = torch.zeros_like(v)
    lib = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream())
    hbm, kind = peaks()
    res = {}
    for name, fn, a, b, nbytes in (
            ("restrict", lib.amg_restrict0_mixed_dev, v, out, ntest * N * 2 * 4 + R * N * 2 * 8 + R * nblk * 2 * ntest * 8),
            ("prolong", lib.amg_prolong0_mixed_dev, vc, psi, ntest * N * 2 * 4 + 2 * R * N * 2 * 8)):
        def call():
            rc = fn(ctx._h, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), R)
            if rc != 0:
                raise RuntimeError(f"{name}: {lib.amg_last_error()}")
        for _ in range(3):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # each call synchronises its stream, so the events bracket the launches alone
        ms = 0.0
        for _ in range(args.steps):
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms /= args.steps
        res[name] = {"ms_per_launch": ms, "algorithmic_bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9,
                     "frac": nbytes / (ms * 1e-3) / 1e9 / hbm}
    ctx.close()
    print(json.dumps({"kernels": "level-0 transfers, mixed form", "tensor_cores": os.environ.get("AMG_TC_TRANSFER", "1") != "0",
                      "lattice": [NX, NT], "nrhs": R, "ntest": ntest, "peak_gbs": hbm, "peak": kind, **res}))


def run_ours(args, world, rank, local):
    import torch

    from amg_schwingermodel_b200 import AMGContext, dirac_apply_raw, launch_count
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor

    torch.cuda.set_device(local)
    R = args.rhs
    prec = 1 if args.precision == "mixed" else 0
    N = NX * NT
    gseed, bseed = replica_seeds(rank)
    U = gauge_field(NX, NT, BETA, gseed)
    b_host = gaussian_spinor(N, 2, bseed, nrhs=R)
    extras = world == 1 and not args.no_extras
    # ---- the chosen form: mixed precision, R sources per solve
    ctx = AMGContext(NX, NT, ROWS, M0, precision=prec, max_rhs=R, device=local)
    ctx.set_gauge(U)
    setup_ms = ctx.setup()
    setup_split = ctx.setup_timings()
    stream = torch.cuda.ExternalStream(ctx.stream())
    b_dev = torch.from_numpy(b_host.view(np.float64).copy()).to(f"cuda:{local}")
    x_dev = torch.empty_like(b_dev)
    for _ in range(args.warmup):
        infos = ctx.solve_dev(b_dev.data_ptr(), x_dev.data_ptr(), R)
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    e0.record(stream)
    for _ in range(args.steps):
        infos = ctx.solve_dev(b_dev.data_ptr(), x_dev.data_ptr(), R)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = launch_count() - l0
    clocks = sampler.stop()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = world * R * args.steps / (ms / 1e3)
    iters = [i["iterations"] for i in infos]
    resid = max(i["rel_residual"] for i in infos)
    converged = all(i["converged"] for i in infos)
    x_chosen = x_dev.cpu().numpy().view(np.complex128).reshape(R, N, 2)
    tuned = ctx.autotune_info()

    # ---- per-kernel-class device time inside the same kind of step (profiled pass)
    ctx.profile(True)
    ctx.solve_dev(b_dev.data_ptr(), x_dev.data_ptr(), R)
    prof = ctx.profile_report()
    ctx.profile(False)

    # ---- end to end through the C ABI from pinned host buffers: amg_solve_stream, one batch
    # of R sources per step; every step copies its sources in and its solutions out (a
    # batch's copies overlap the neighbouring batches' solves).  amg_solve once per step
    # (copy in, solve, copy out, in series) is timed beside it.
    b_pin = torch.from_numpy(b_host.view(np.float64).copy()).pin_memory()
    x_pins = [torch.empty_like(b_pin).pin_memory() for _ in range(2)]
    bptrs = [b_pin.data_ptr()] * args.steps
    xptrs = [x_pins[k % 2].data_ptr() for k in range(args.steps)]
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.solve_stream_ptrs(bptrs[:2], xptrs[:2], R)
    barrier(world)
    torch.cuda.synchronize()
    e2.record(stream)
    infos_e2e = ctx.solve_stream_ptrs(bptrs, xptrs, R)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3), world)
    e2e_value = world * R * args.steps / (ms_e2e / 1e3)
    x_e2e = x_pins[(args.steps - 1) % 2].numpy().view(np.complex128).reshape(R, N, 2)
    e2e_matches = bool(np.array_equal(x_e2e, x_chosen)) and all(i["converged"] for b in infos_e2e for i in b)
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e4.record(stream)
    for _ in range(args.steps):
        ctx.solve_host_ptr(b_pin.data_ptr(), x_pins[0].data_ptr(), R)
    e5.record(stream)
    torch.cuda.synchronize()
    e2e_call_value = world * R * args.steps / (max_over_ranks(e4.elapsed_time(e5), world) / 1e3)
    ctx.close()
    del b_pin, x_pins

    # ---- the plain FP64 drop-in on one source, same gauge field (>= 10 timed solves)
    ctx64 = AMGContext(NX, NT, ROWS, M0, precision=0, max_rhs=1, device=local)
    ctx64.set_gauge(U)
    setup64_ms = ctx64.setup()
    b1 = b_dev[0:1].contiguous()
    x1 = torch.empty_like(b1)
    n64 = max(10, min(args.steps, 20))
    ms64, info64 = timed_solves(ctx64, b1.data_ptr(), x1.data_ptr(), 1, n64, max(3, args.warmup))
    ms64 = max_over_ranks(ms64, world)
    fp64_value = world * 1e3 / ms64
    x64 = x1.cpu().numpy().view(np.complex128).reshape(N, 2)
    tuned64 = ctx64.autotune_info()
    err_vs_fp64 = float(np.linalg.norm(x_chosen[0] - x64) / np.linalg.norm(x64))
    hierarchy = hierarchy_for_reference(ctx64) if (rank == 0 and extras and not args.no_cpu) else None
    ctx64.close()
    fp64_batched = None
    if extras:
        # ---- FP64 on the same batch of R sources: splits the gain into batching and precision
        with AMGContext(NX, NT, ROWS, M0, precision=0, max_rhs=R, device=local) as ctx64b:
            ctx64b.set_gauge(U)
            ctx64b.setup()
            ms64b, info64b = timed_solves(ctx64b, b_dev.data_ptr(), x_dev.data_ptr(), R, 3, 1)
            fp64_batched = {"value": R * 1e3 / ms64b, "unit": UNIT, "nrhs": R, "steps": 3,
                            "iterations": sorted({i["iterations"] for i in info64b}),
                            "max_rel_residual": max(i["rel_residual"] for i in info64b),
                            "autotune": ctx64b.autotune_info()}

    link_lines = None
    if extras:
        # ---- storage of the mixed cycle's fine links: FP16 (the default: the line above), FP32,
        # BF16
        link_lines = {"f16": {"value": value, "unit": UNIT, "iterations": sorted(set(iters)),
                              "max_rel_residual": resid, "err_vs_fp64": err_vs_fp64, "default": True}}
        for name, code in (("f32", 0), ("bf16", 1)):
            with AMGContext(NX, NT, ROWS, M0, precision=1, max_rhs=R, device=local, link_storage=code) as ctxl:
                ctxl.set_gauge(U)
                ctxl.setup()
                msl, infl = timed_solves(ctxl, b_dev.data_ptr(), x_dev.data_ptr(), R, 3, 1)
                xl = x_dev[0].cpu().numpy().view(np.complex128).reshape(N, 2)
                link_lines[name] = {"value": R * 1e3 / msl, "unit": UNIT, "steps": 3,
                                    "iterations": sorted({i["iterations"] for i in infl}),
                                    "max_rel_residual": max(i["rel_residual"] for i in infl),
                                    "err_vs_fp64": float(np.linalg.norm(xl - x64) / np.linalg.norm(x64))}

    # ---- fine D-apply bandwidth (FP64, 8 sources per launch: 768 MB of spinors > L2)
    nd = 8
    Ud = torch.from_numpy(U.view(np.float64).copy()).cuda()
    vin = torch.randn(nd, N, 2, 2, dtype=torch.float64, device="cuda")
    vout = torch.empty_like(vin)
    ds = torch.cuda.current_stream()
    for _ in range(3):
        dirac_apply_raw(Ud.data_ptr(), vin.data_ptr(), vout.data_ptr(), NX, NT, nd, M0, False, ds.cuda_stream)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nrep = 30
    torch.cuda.nvtx.range_push("dapply")
    g0.record(ds)
    for _ in range(nrep):
        dirac_apply_raw(Ud.data_ptr(), vin.data_ptr(), vout.data_ptr(), NX, NT, nd, M0, False, ds.cuda_stream)
    g1.record(ds)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    d_ms = g0.elapsed_time(g1) / nrep
    d_bytes = N * (32 + nd * 64)
    hbm, peak_kind = peaks()
    d_gbs = d_bytes / (d_ms * 1e-3) / 1e9
    del vin, vout, Ud

    po = prof.get("outer_op", {})
    outer_op = None
    if po.get("launches"):
        ms_l = po["ms"] / po["launches"]
        by_l = po["bytes"] / po["launches"]
        outer_op = {"gbs": by_l / (ms_l * 1e-3) / 1e9, "frac": by_l / (ms_l * 1e-3) / 1e9 / hbm, "peak": peak_kind,
                    "ms_per_launch": ms_l, "bytes_per_launch": by_l, "nrhs": R}

    # ---- roofline of the dominant kernel class of the step
    dom = max(prof, key=lambda k: prof[k]["ms"])
    pd = prof[dom]
    per_launch_ms = pd["ms"] / max(pd["launches"], 1)
    per_launch_bytes = pd["bytes"] / max(pd["launches"], 1)
    achieved_gbs = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    tot_prof = sum(v["ms"] for v in prof.values())
    share = pd["ms"] / tot_prof if tot_prof else None
    if dom == "sap":
        # block solves live in shared memory and registers: bound by FP32 issue, not HBM
        ncol = ROWS[0][4] * ROWS[0][5] // 2
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        peak_tf = sms * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
        flops = SAP_FLOPS_PER_SITE * (N // 2) * R
        tf = flops / (per_launch_ms * 1e-3) / 1e12
        roofline = {"kernel": "sap", "bound": "fp32", "achieved": tf, "peak": peak_tf, "unit": "TFLOP/s",
                    "frac": tf / peak_tf, "traffic": SAP_DRAM_BYTES_PER_BLOCK_SOURCE * ncol * R,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at 32 sources",
                    "peak_kind": (f"nominal FP32 CUDA-core peak: {sms} SMs x {FP32_LANES_PER_SM} lanes x 2 flop x "
                                  f"{sm_mhz:.0f} MHz (sampled); no measured FP32 peak exists on this pool"),
                    "flops_per_launch": flops, "bytes_per_launch": per_launch_bytes,
                    "ms_per_launch": per_launch_ms, "achieved_gbs": achieved_gbs, "hbm_frac": achieved_gbs / hbm,
                    "share_of_step": share}
    else:
        roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                    "frac": achieved_gbs / hbm, "traffic": None, "peak_kind": peak_kind,
                    "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms, "share_of_step": share}

    extra = {}
    if extras:
        torch.cuda.empty_cache()
        for key, fn in (("config2_256", lambda: line_config2(local)),
                        ("reference_rows", lambda: line_reference_rows(local, R)),
                        ("uneven_batch", lambda: line_uneven_batch(local, 2))):
            try:
                extra[key] = fn()
            except Exception as e:  # noqa: BLE001 -- a failed side line must not lose the headline
                extra[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()

    # ---- CPU baseline: complete reference solves on this workload (rank 0, N = 1)
    cpu = None
    if hierarchy is not None:
        try:
            res = cpu_reference_solve(U, b_host[0], hierarchy)
            if "error" not in res:
                cpu = {"value": 1.0 / res["t"], "unit": UNIT, "cores": res["ranks"], "kind": "reference",
                       "sample": (f"complete reference FGMRES_AMG solve (its FGMRES, K-cycle, SAP and D_phi code) "
                                  f"at {NX}x{NT} L4 on the hierarchy the GPU FP64 set-up built, {res['ranks']} rank(s) "
                                  f"of its MPI layout: {res['t']:.2f} s, {res['iterations']} iterations, FP64 "
                                  f"residual {res['residual']:.1e} (solve {res['solves']} of {res['solves']}); "
                                  f"D_phi {res['dphi_s'] * 1e3:.1f} ms/apply")}
            else:
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": res["error"]}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 inner (bf16 test vectors, f16 links), f64 outer" if prec else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "lattice": [NX, NT], "levels": 4, "rows": ROWS, "nrhs_per_step": R,
                       "precision": args.precision, "beta": BETA, "m0": M0, "tol": TOL,
                       "l2": "working set > L2 (126 MB)", "parallelism": f"replicas x{world}",
                       "autotune": tuned},
            "iterations": iters, "max_rel_residual": resid, "converged": converged,
            "err_vs_fp64": err_vs_fp64,
            "setup_s": setup_ms / 1e3,
            "setup_split_ms": setup_split,
            "fp64_dropin": {"value": fp64_value, "unit": UNIT, "nrhs": 1, "steps": n64,
                            "iterations": info64[0]["iterations"], "rel_residual": info64[0]["rel_residual"],
                            "setup_s": setup64_ms / 1e3, "autotune": tuned64},
            "speedup_vs_fp64_dropin": value / fp64_value,
            "dapply": {"gbs": d_gbs, "frac": d_gbs / hbm, "peak_gbs": hbm, "peak": peak_kind,
                       "ms_per_launch": d_ms, "nrhs": nd, "bytes_per_launch": d_bytes},
            # the D apply inside the solve: the outer step's w = D z_j from the FP32 z_j, with
            # z_j's FP64 promotion written by the same pass (R sources per launch)
            "dapply_outer": outer_op,
            "roofline": roofline,
            "kernels": prof,
            "e2e": {"value": e2e_value, "unit": UNIT, "api": "amg_solve_stream", "same_x_as_device_run": e2e_matches,
                    "per_call": {"value": e2e_call_value, "api": "amg_solve"},
                    "h2d_bytes_per_step": int(R * N * 32),
                    "d2h_bytes_per_step": int(R * N * 32)},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        if link_lines is not None:
            line["link_storage"] = link_lines
        if fp64_batched is not None:
            line["fp64_batched"] = fp64_batched
            line["speedup_split"] = {"batching_f64": fp64_batched["value"] / fp64_value,
                                     "precision_at_batch": value / fp64_batched["value"]}
        line.update(extra)
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rhs", type=int, default=32, help="sources per batched solve (one step)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the side lines (FP64 batch, reference rows, 256^2, uneven batch)")
    ap.add_argument("--transfers", action="store_true",
                    help="time the mixed form's level-0 restriction and prolongation alone (no solve)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.transfers:
        run_transfers(args, local)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
