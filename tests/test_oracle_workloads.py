"""The solve fixtures at the workload sizes (tests/golden/solve*.npz: complete solves of the
compiled reference at 128^2 .. 1024^2) are self-consistent and pin the restatement:

* the inputs regenerate from the seeds in their meta: the restatement's D_phi of the
  regenerated source equals the reference's D_phi(b) on the fixture's site sample to 1e-13
  (src/dirac_operator.cpp:3-27);
* each reference solve met its tolerance (FP64 true residual <= 1e-10) and its residual
  history ends below 1e-10 |b|;
* at 128^2 the restatement's whole set-up and FGMRES_AMG solve reproduce the reference's
  iteration count and solution (1e-12 on the sample).
"""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel
from oracle import restatement as R

SOLVES = sorted(p.stem for p in GOLDEN.glob("solve*.npz"))


def inputs(m):
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    ns = m["ns"]
    return gauge_field(ns, m["nt"], m["beta"], m["seed"]), gaussian_spinor(ns * m["nt"], 2, m["seed"] + 1000)


def test_solve_fixtures_present():
    assert {"solve256_l3", "solve1024_l4", "solve1024_l4_refrows", "solve128_l3_b2", "solve256_l3_b3",
            "solve512_l3_b4"} <= set(SOLVES)


@pytest.mark.parametrize("name", SOLVES)
def test_solve_fixture_inputs_and_convergence(name):
    g = load_golden(name)
    m = g["meta"]
    U, b = inputs(m)
    idx = g["sites"]
    assert rel(R.d_phi(U, b, m["m0"], m["ns"], m["nt"])[idx], g["dphi_sample"]) < 1e-13
    assert m["true_rel_residual"] <= 1e-10
    hist = g["residual_history"]
    assert hist[-1] < 1e-10 * np.linalg.norm(b)
    assert m["iterations"] == len(hist)


def test_restatement_solve_matches_reference_128():
    g = load_golden("solve128_l3_b2")
    m = g["meta"]
    U, b = inputs(m)
    job = m["job"]
    sp_ = R.SolverParams(m0=m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"], nit=job["nit"],
                         sap_tv_iters=job["sap_tv_iters"])
    amg = R.AMG(U, m["ns"], m["nt"], m["rows"], sp_)
    amg.setup_from(R.reference_initial_test_vectors(amg.lps))
    x, it = amg.solve(b)
    assert it == m["iterations"]
    assert rel(x[g["sites"]], g["x_sample"]) < 1e-12
