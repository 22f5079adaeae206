"""Pins the numpy restatement of the reference (oracle/restatement.py) against the golden
fixtures the compiled reference produced (tests/golden/make_golden.py).

Integer index maps must be bit-exact; FP64 results agree to rounding (the reference sums
in a different order).  Iteration counts must be equal.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel
from oracle import restatement as R

NAMES = golden_names()


def _setup(g):
    m = g["meta"]
    lps = R.read_parameters(m["ns"], m["nt"], m["rows"])
    job = m["job"]
    sp_ = R.SolverParams(m0=m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                         nit=job["nit"], sap_tv_iters=job["sap_tv_iters"])
    return m, lps, sp_


@pytest.mark.parametrize("name", NAMES)
def test_index_maps_bit_exact(name):
    g = load_golden(name)
    m, lps, _ = _setup(g)
    for l, lp in enumerate(lps):
        Rt, Lt, sR, sL = R.boundary(lp)
        assert np.array_equal(g[f"rightpb_l{l}"], Rt.reshape(-1))
        assert np.array_equal(g[f"leftpb_l{l}"], Lt.reshape(-1))
        assert np.array_equal(g[f"signr_l{l}"], sR.reshape(-1))
        assert np.array_equal(g[f"signl_l{l}"], sL.reshape(-1))
        blocks, red, black = R.schwarz_blocks(lp)
        assert np.array_equal(g[f"sapblocks_l{l}"], blocks.reshape(-1))
        assert np.array_equal(g[f"sapred_l{l}"], red)
        assert np.array_equal(g[f"sapblack_l{l}"], black)
        if l < len(lps) - 1:
            assert np.array_equal(g[f"latblocks_l{l}"], R.lattice_blocks(lp).reshape(-1))
            agg, nc, sc, cc = R.aggregates(lp)
            assert np.array_equal(g[f"agg_l{l}"], agg.reshape(-1))
            assert np.array_equal(g[f"ncoords_l{l}"], nc)
            assert np.array_equal(g[f"scoords_l{l}"], sc)
            assert np.array_equal(g[f"ccoords_l{l}"], cc)


@pytest.mark.parametrize("name", NAMES)
def test_dirac_operator(name):
    g = load_golden(name)
    m = g["meta"]
    U, b = g["gauge"], g["rhs"]
    assert rel(R.d_phi(U, b, m["m0"], m["ns"], m["nt"]), g["dphi"]) < 1e-14
    assert rel(R.d_dagger_phi(U, b, m["m0"], m["ns"], m["nt"]), g["ddagphi"]) < 1e-14


def test_initial_test_vectors_reproduce_reference_rng():
    """Level-0 test vectors of setUpPhase regenerate bit-exactly (src/amg.cpp:8-19); the
    set-up built from them reproduces the reference's final test vectors."""
    g = load_golden("c16_l2_k")
    m, lps, sp_ = _setup(g)
    init = R.reference_initial_test_vectors(lps)
    amg = R.AMG(g["gauge"], m["ns"], m["nt"], m["rows"], sp_)
    amg.setup_from(init)
    for i in range(lps[0].ntest):
        assert rel(amg.levels[0].W[i], g[f"tv_l0_{i}"]) < 1e-12


@pytest.mark.parametrize("name", NAMES)
def test_setup_probes_and_solve(name):
    g = load_golden(name)
    m, lps, sp_ = _setup(g)
    L = len(lps)
    amg = R.AMG(g["gauge"], m["ns"], m["nt"], m["rows"], sp_)
    amg.setup_from(R.reference_initial_test_vectors(lps))
    for l in range(L - 1):
        for i in range(lps[l].ntest):
            if f"tv_l{l}_{i}" in g:
                assert rel(amg.levels[l].W[i], g[f"tv_l{l}_{i}"]) < 1e-10
    for l in range(1, L):
        for k, G in (("g1", amg.levels[l].G1), ("g2", amg.levels[l].G2), ("g3", amg.levels[l].G3)):
            if f"{k}_l{l}" in g:
                assert rel(G.reshape(-1), g[f"{k}_l{l}"]) < 1e-10
    for l in range(L):
        p = g[f"probe_l{l}"]
        assert rel(amg.levels[l].apply(p), g[f"dop_l{l}"]) < 1e-10
        if l < L - 1:
            Lv = amg.levels[l]
            c = R.pt_v(Lv.W, p, Lv.lp)
            assert rel(c, g[f"pt_l{l}"]) < 1e-10
            assert rel(R.p_v(Lv.W, c, Lv.lp), g[f"ppt_l{l}"]) < 1e-10
            xs, ret = amg.sap(l, p, np.zeros_like(p), 2)
            assert rel(xs, g[f"sap_l{l}"]) < 1e-9
            assert ret == m["sap_ret"][str(l)]
        else:
            xg, it = R.fgmres(Lv_apply := amg.levels[l].apply, lambda v, z: v, p, p, 20, 20, 0.1)
            assert rel(xg, g[f"gmres_l{l}"]) < 1e-9
            assert it == m["gmres_iters"][str(l)]
    z = amg.precondition(g["rhs"])
    assert rel(z, g["cycle0_rhs"]) < 1e-9
    hist = []
    x, it = amg.solve(g["rhs"], hist)
    assert it == m["iterations"]
    assert rel(x, g["x"]) < 1e-9
    np.testing.assert_allclose(hist, g["residual_history"], rtol=1e-6, atol=1e-12 * hist[0])
    assert R.true_residual(g["gauge"], x, g["rhs"], m["m0"], m["ns"], m["nt"]) < 1e-10
