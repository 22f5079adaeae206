"""The compiled reference as several ranks on the host's cores (oracle/mpi_shim/mpi.h): the
reference's MPI layout, its SAP block solves of each colour split among the ranks
(src/sap.cpp:77-78) and summed by the all-reduce (src/sap.cpp:113,149), gives the one-rank
run's results exactly -- the solution, the iteration count and the residual history -- for
2, 3 and 4 ranks (an uneven split of the 8 blocks per colour included), with the ranks
started at the beginning or after the set-up (the timed-sample mode the CPU baseline
uses).  A rank that leaves before its first collective ends the job with an error within
seconds instead of leaving the others waiting.  Needs the reference sources to build
oracle/_ref/ref_32x32_l3; skipped without."""
import numpy as np
import pytest

from oracle import ref_runner

NS, ROWS, M0 = 32, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], -0.1


@pytest.fixture(scope="module")
def oracle_binary():
    if not ref_runner.available(NS, NS, 3):
        pytest.skip("reference sources absent and oracle/_ref/ref_32x32_l3 not built")
    return ref_runner.build(NS, NS, 3)


def _inputs():
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    return gauge_field(NS, NS, 3.0, 31), gaussian_spinor(NS * NS, 2, 32)


def test_ranks_give_the_one_rank_solve(oracle_binary, tmp_path):
    U, b = _inputs()
    one = ref_runner.run(NS, NS, ROWS, U, b, m0=M0, nit=1, dump_hierarchy=0)
    for ranks in (2, 3, 4):
        wd = tmp_path / f"r{ranks}"
        out = ref_runner.run(NS, NS, ROWS, U, b, m0=M0, nit=1, dump_hierarchy=0, ranks=ranks, workdir=str(wd))
        assert out["info:iterations"] == one["info:iterations"]
        assert np.array_equal(out["x"], one["x"])
        assert np.array_equal(out["residual_history"], one["residual_history"])
        # every rank ran the job; the others wrote under rank<r>/
        assert sorted(p.name for p in wd.glob("rank*")) == [f"rank{r}" for r in range(1, ranks)]


def test_ranks_started_after_setup_give_the_one_rank_cycle(oracle_binary):
    U, b = _inputs()
    one = ref_runner.run(NS, NS, ROWS, U, b, m0=M0, dump_hierarchy=1)
    hier = {"tv": {l: np.stack([one[f"tv_l{l}_{i}"] for i in range(ROWS[l][3])]) for l in range(2)},
            "links": {l: tuple(one[f"{g}_l{l}"] for g in ("g1", "g2", "g3")) for l in (1, 2)}}
    z = {}
    for ranks, late in ((1, 0), (4, 1), (3, 1)):
        out = ref_runner.run(NS, NS, ROWS, U, b, m0=M0, dump_hierarchy=0, outer_iteration_reps=2,
                             hierarchy=hier, ranks=ranks, ranks_after_setup=late)
        z[ranks] = out["sample_z"]
        assert all(out[f"info:outer_iteration_seconds_{r}"] > 0 for r in range(2))
    assert np.array_equal(z[4], z[1]) and np.array_equal(z[3], z[1])
    assert np.linalg.norm(z[1]) > 0


def test_a_lost_rank_ends_the_job_with_an_error(oracle_binary):
    import time
    U, b = _inputs()
    t0 = time.time()
    with pytest.raises(RuntimeError, match="exited inside a collective"):
        ref_runner.run(NS, NS, ROWS, U, b, m0=M0, dump_hierarchy=0, ranks=3, drill_exit_rank=2, timeout=120)
    assert time.time() - t0 < 60


def test_ranks_started_after_the_reference_setup_give_the_one_rank_cycle(oracle_binary):
    """The reference arm's mode: the reference's own set-up (with test-vector smoothing),
    then the ranks, then the timed outer iterations."""
    U, b = _inputs()
    z = {}
    for ranks in (1, 4):
        out = ref_runner.run(NS, NS, ROWS, U, b, m0=M0, dump_hierarchy=0, outer_iteration_reps=2,
                             sap_tv_iters=2, ranks=ranks, ranks_after_setup=1)
        z[ranks] = out["sample_z"]
        assert out["info:outer_iteration_seconds"] > 0
    assert np.array_equal(z[4], z[1]) and np.linalg.norm(z[1]) > 0
