#!/usr/bin/env python
"""Benchmark: 1024x1024 Schwinger-model DD-alpha-AMG solves per second to FP64 relative
residual <= 1e-10 (4 levels, Nv = 16, beta = 4, m0 = -0.05), mixed precision with batched
sources against the plain FP64 drop-in, plus the fine D-apply bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--rhs R] [--precision mixed|f64]

One step = one batched solve of R seeded complex-Gaussian sources on one seeded gauge
field per GPU (inputs resident in HBM; the working set of a step is far above the 126 MB
L2).  With N GPUs every rank solves its own gauge field and sources (replicas, weak
scaling); timing is CUDA events on the solver's stream, max over ranks.  Rank 0 prints one
JSON line.  `--impl reference` times the reference's own CPU code (compiled from its
sources into oracle/_ref) on the same workload: the reference's set-up with its test-vector
smoothing skipped, then a bounded sample of outer FGMRES iterations (one K-cycle from the
fine level plus D_phi each) scaled to the workload's iteration count, run in the
reference's MPI layout on up to 8 host cores (reference_ranks).
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
# DRAM bytes (read + write) of one fine SAP launch per (block, source) it solves, from an ncu
# capture of this workload at 2 sources (42.02 MB read + 0.37 MB written for 512 blocks x 2
# sources); the traffic grows with the blocks x sources a launch solves.
SAP_DRAM_BYTES_PER_BLOCK_SOURCE = 42.391808e6 / 1024
BETA, M0, TOL = 4.0, -0.05, 1e-10
METRIC = "1024^2 solves/s at FP64 resid <=1e-10: mixed+batched vs FP64 GPU; D-apply GB/s"
UNIT = "solves/s"
WORKLOAD = "schwinger_wilson_1024x1024_L4_Nv16_beta4_m0-0.05"


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


def reference_ranks() -> int:
    """Ranks for the reference's CPU runs (its MPI layout as processes on this host, the SAP
    block solves split among them): the usable cores, at most 8, and no more than half the
    available memory holds -- a 1024x1024 4-level run of the reference takes about 20 GB
    for its first rank and about 6 GB for each further rank started after the set-up.
    AMG_REF_RANKS overrides."""
    if os.environ.get("AMG_REF_RANKS"):
        return max(1, int(os.environ["AMG_REF_RANKS"]))

    def read(path):
        try:
            return Path(path).read_text().split()
        except OSError:
            return None

    cores = len(os.sched_getaffinity(0))
    # a CPU quota of this container (cgroup v2, then v1) bounds the cores too
    q = read("/sys/fs/cgroup/cpu.max")
    if q and q[0] != "max":
        cores = min(cores, max(1, int(q[0]) // int(q[1])))
    q, per = read("/sys/fs/cgroup/cpu/cpu.cfs_quota_us"), read("/sys/fs/cgroup/cpu/cpu.cfs_period_us")
    if q and per and int(q[0]) > 0:
        cores = min(cores, max(1, int(q[0]) // int(per[0])))
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) * 1024 for l in f if l.startswith("MemAvailable:"))
    except (OSError, StopIteration, ValueError):
        return 1
    # and so does a memory limit of this container (cgroup v2, then v1)
    for lim, use in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        a, b = read(lim), read(use)
        if a and b and a[0] != "max" and int(a[0]) < (1 << 60):
            avail = min(avail, int(a[0]) - int(b[0]))
    by_mem = int((0.5 * avail - 20e9) // 6e9) + 1
    return max(1, min(cores, 8, by_mem))


def run_reference_job(ranks: int, **kw):
    """ref_runner.run on the bench workload with `ranks` ranks started after the set-up; if
    that run fails (a rank lost, e.g. to memory pressure) it is repeated with one rank.
    Returns (outputs, ranks used)."""
    from oracle import ref_runner
    if ranks > 1:
        try:
            return ref_runner.run(NX, NT, ROWS, ranks=ranks, ranks_after_setup=1, **kw), ranks
        except RuntimeError as e:
            print(f"reference with {ranks} ranks failed ({str(e)[:200]}); one rank", file=sys.stderr)
    return ref_runner.run(NX, NT, ROWS, **kw), 1


def cpu_reference_sample(U, b0, hierarchy, reps: int, ranks: int = 1, timeout: float = 900):
    """Times outer FGMRES iterations of the reference's own code (oracle/_ref) on this workload:
    one preconditioner application (K-cycle from the fine level) plus D_phi per repetition,
    on `ranks` ranks."""
    from oracle import ref_runner
    b = ref_runner.binary(NX, NT, len(ROWS) + 1)
    if not b.exists():
        return None, f"{b.name} not built"
    kw = dict(m0=M0, solve=1, dump_hierarchy=0, dphi_reps=20, outer_iteration_reps=reps, sap_tv_iters=0)
    if hierarchy is not None:
        kw["hierarchy"] = hierarchy
    out, used = run_reference_job(ranks, gauge=U, rhs=b0, timeout=timeout, **kw)
    if hierarchy is not None:
        times = [out[f"info:outer_iteration_seconds_{r}"] for r in range(reps)]
    else:
        times = [out["info:outer_iteration_seconds"]]
    return dict(times=times, dphi_s=out.get("info:dphi_seconds_per_apply"),
                setup_s=out.get("info:setup_seconds"), ranks=used), None


def run_reference(args, world, rank):
    """The reference's own CPU code on this workload: its set-up (test-vector smoothing
    skipped to bound the run), then warmup + steps outer FGMRES iterations (K-cycle from the
    fine level + D_phi), each a bounded sample of one solve; solves/s scales the per-iteration
    time by the outer iteration count of the reference algorithm on this workload."""
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
    reps = args.warmup + args.steps
    t0 = time.time()
    out, ranks = run_reference_job(reference_ranks(), gauge=U, rhs=b0, m0=M0, solve=1, dump_hierarchy=0,
                                   dphi_reps=20, outer_iteration_reps=reps, sap_tv_iters=0, timeout=3600)
    times = [out[f"info:outer_iteration_seconds_{r}"] for r in range(reps)][args.warmup:]
    it_s = statistics.mean(times)
    iters = args.ref_iterations
    value = 1.0 / (iters * it_s)
    sample = (f"reference outer FGMRES iterations (K-cycle from the fine level + D_phi) at {NX}x{NT}, 4 levels, "
              f"after its own set-up with test-vector smoothing skipped; mean of {len(times)} timed of {reps}: "
              f"{it_s:.2f} s/iteration; solves/s = 1/({iters} iterations x that); {ranks} rank(s) of its MPI "
              f"layout, one core each (SAP blocks split among them)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * iters * it_s, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "lattice": [NX, NT], "levels": 4, "rows": ROWS, "nrhs": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ranks, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "dphi_s_per_apply": out.get("info:dphi_seconds_per_apply"),
            "ref_setup_s": out.get("info:setup_seconds"), "wall_s": time.time() - t0}
    print(json.dumps(line))


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
    # ---- the chosen form: mixed precision, R sources per solve
    ctx = AMGContext(NX, NT, ROWS, M0, precision=prec, max_rhs=R, device=local)
    ctx.set_gauge(U)
    setup_ms = ctx.setup()
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

    # ---- end to end through the C ABI from pinned host buffers
    b_pin = torch.from_numpy(b_host.view(np.float64).copy()).pin_memory()
    x_pin = torch.empty_like(b_pin).pin_memory()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.solve_host_ptr(b_pin.data_ptr(), x_pin.data_ptr(), R)
    barrier(world)
    torch.cuda.synchronize()
    e2.record(stream)
    for _ in range(args.steps):
        ctx.solve_host_ptr(b_pin.data_ptr(), x_pin.data_ptr(), R)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3), world)
    e2e_value = world * R * args.steps / (ms_e2e / 1e3)
    ctx.close()

    # ---- the plain FP64 drop-in on one source, same gauge field
    ctx64 = AMGContext(NX, NT, ROWS, M0, precision=0, max_rhs=1, device=local)
    ctx64.set_gauge(U)
    setup64_ms = ctx64.setup()
    b1 = b_dev[0:1].contiguous()
    x1 = torch.empty_like(b1)
    for _ in range(max(2, args.warmup)):
        info64 = ctx64.solve_dev(b1.data_ptr(), x1.data_ptr(), 1)
    torch.cuda.synchronize()
    s64 = torch.cuda.ExternalStream(ctx64.stream())
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n64 = max(2, min(args.steps, 3))
    f0.record(s64)
    for _ in range(n64):
        info64 = ctx64.solve_dev(b1.data_ptr(), x1.data_ptr(), 1)
    f1.record(s64)
    torch.cuda.synchronize()
    ms64 = max_over_ranks(f0.elapsed_time(f1), world)
    fp64_value = world * n64 / (ms64 / 1e3)
    x64 = x1.cpu().numpy().view(np.complex128).reshape(N, 2)
    tuned64 = ctx64.autotune_info()
    err_vs_fp64 = float(np.linalg.norm(x_chosen[0] - x64) / np.linalg.norm(x64))
    hierarchy = hierarchy_for_reference(ctx64) if (rank == 0 and world == 1 and not args.no_cpu) else None
    ctx64.close()

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

    # ---- roofline of the dominant kernel class of the step
    dom = max(prof, key=lambda k: prof[k]["ms"])
    pd = prof[dom]
    per_launch_ms = pd["ms"] / max(pd["launches"], 1)
    per_launch_bytes = pd["bytes"] / max(pd["launches"], 1)
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    tot_prof = sum(v["ms"] for v in prof.values())
    ncol = ROWS[0][4] * ROWS[0][5] // 2
    sap_traffic = SAP_DRAM_BYTES_PER_BLOCK_SOURCE * ncol * R

    # ---- CPU baseline: the reference's own outer iteration on this workload (rank 0, N = 1)
    cpu = None
    if hierarchy is not None:
        try:
            ranks = reference_ranks()
            # with several ranks the first iteration also pays the first touch of the shared
            # all-reduce buffers: time two and keep the second
            res, err = cpu_reference_sample(U, b_host[0], hierarchy, 2 if ranks > 1 else 1, ranks)
            if res:
                it_s = res["times"][-1]
                it_count = info64[0]["iterations"]
                cpu = {"value": 1.0 / (it_count * it_s), "unit": UNIT, "cores": res["ranks"], "kind": "reference",
                       "sample": (f"reference K-cycle + D_phi (one outer FGMRES iteration) at {NX}x{NT} L4 on "
                                  f"this hierarchy, {res['ranks']} rank(s) of its MPI layout: {it_s:.2f} s; "
                                  f"x {it_count} iterations; D_phi {res['dphi_s'] * 1e3:.1f} ms/apply")}
            else:
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": err}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+bf16 inner, f64 outer" if prec else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "lattice": [NX, NT], "levels": 4, "rows": ROWS, "nrhs_per_step": R,
                       "precision": args.precision, "beta": BETA, "m0": M0, "tol": TOL,
                       "l2": "working set > L2 (126 MB)", "parallelism": f"replicas x{world}",
                       "autotune": tuned},
            "iterations": iters, "max_rel_residual": resid, "converged": converged,
            "err_vs_fp64": err_vs_fp64,
            "setup_s": setup_ms / 1e3,
            "fp64_dropin": {"value": fp64_value, "unit": UNIT, "iterations": info64[0]["iterations"],
                            "rel_residual": info64[0]["rel_residual"], "setup_s": setup64_ms / 1e3,
                            "autotune": tuned64},
            "speedup_vs_fp64_dropin": value / fp64_value,
            "dapply": {"gbs": d_gbs, "frac": d_gbs / hbm, "peak_gbs": hbm, "peak": peak_kind,
                       "ms_per_launch": d_ms, "nrhs": nd, "bytes_per_launch": d_bytes},
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": sap_traffic if dom == "sap" else None,
                         "traffic_source": "ncu capture at 2 sources, scaled by blocks x sources" if dom == "sap" else None,
                         "peak_kind": peak_kind,
                         "share_of_step": pd["ms"] / tot_prof if tot_prof else None,
                         "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms},
            "kernels": prof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(R * N * 32),
                    "d2h_bytes_per_step": int(R * N * 32)},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
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
    ap.add_argument("--ref-iterations", type=int, default=10,
                    help="outer iterations of the reference algorithm on this workload (FP64 drop-in count)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
