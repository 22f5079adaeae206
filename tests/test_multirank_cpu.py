"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the path a torchrun launch on
N GPUs takes, with NCCL there).  Every rank solves its own configuration (replicas), so the
only collectives are the barrier around the timed region and the max over ranks of the
device time; the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    top = bench.max_over_ranks(1.5 + rank, w)
    seeds = bench.replica_seeds(r)
    # the reference arm prints nothing on ranks other than 0 and does no work there
    ref_noop = rank != 0 and bench.run_reference(None, w, r) is None
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((rank, top, seeds, ref_noop))


def test_two_gloo_ranks_barrier_max_and_replica_seeds():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [t for _, t, _, _ in res] == [2.5, 2.5]
    seeds = [s for _, _, s, _ in res]
    assert len(set(seeds)) == world
    assert res[1][3] is True


def test_reference_rank_count(monkeypatch):
    """The reference's CPU runs take 1..8 ranks, no more than the usable cores; they start
    before the set-up only when every rank fits in memory that way; AMG_REF_RANKS overrides
    the count (ranks then start after the set-up)."""
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.delenv("AMG_REF_RANKS", raising=False)
    n, early = bench.reference_layout()
    assert 1 <= n <= min(8, len(os.sched_getaffinity(0)))
    if early:
        assert n * 13e9 <= 0.5 * bench.host_available_bytes()
    # memory for every rank to run the set-up: all usable cores, started early
    monkeypatch.setattr(bench, "host_available_bytes", lambda: int(2 * 8 * 13e9) + 1)
    monkeypatch.setattr(bench, "host_cores", lambda: 16)
    assert bench.reference_layout() == (8, True)
    # memory for 3 ranks started after the set-up only (20 GB + 2 x 6 GB in half of it)
    monkeypatch.setattr(bench, "host_available_bytes", lambda: int(2 * 32e9) + 1)
    assert bench.reference_layout() == (3, False)
    monkeypatch.setattr(bench, "host_available_bytes", lambda: 0)
    assert bench.reference_layout() == (1, False)
    monkeypatch.setenv("AMG_REF_RANKS", "5")
    assert bench.reference_layout() == (5, False)
    monkeypatch.setenv("AMG_REF_RANKS", "0")
    assert bench.reference_layout() == (1, False)
