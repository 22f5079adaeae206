"""GPU parity at the workload sizes, against complete solves of the reference
(tests/golden/solve*.npz, made from the compiled reference by tests/golden/make_golden.py):

* 256x256, 3 levels, aggregation 8x8 then 4x4 blocks, Nv = 12, 4x4 SAP blocks, beta = 3,
  m0 = -0.05: the FP64 drop-in and the mixed form;
* 1024x1024, 4 levels, Nv = 16, beta = 4, m0 = -0.05, with the benchmark rows (32x32-site SAP
  blocks) and with the reference-style rows (4x4 SAP blocks of 256x256 sites);
* one configuration per lattice size of the uneven batch (128^2, 256^2, 512^2 at beta 2, 3, 4),
  solved together through amg_solve_many with 32 sources each, the fixture's source first.

The gauge field and the source are regenerated from each fixture's seeds; a fixture keeps x
and D_phi(b) on a strided subsample of the sites.  Bars: D within 1e-13 on the sample; FP64
solve: the reference's iteration count, x within 1e-8 on the sample, the residual history
within rtol 1e-5, FP64 true residual <= 1e-10; mixed solve: at most one outer iteration more
than the reference, x within 1e-8 on the sample, FP64 true residual <= 1e-10.
"""
import numpy as np
import pytest

from conftest import load_golden, rel

pytestmark = pytest.mark.gpu

SOLVES = ["solve128_l3_b2", "solve256_l3", "solve256_l3_b3", "solve512_l3_b4", "solve1024_l4",
          "solve1024_l4_refrows"]
BATCH = ["solve128_l3_b2", "solve256_l3_b3", "solve512_l3_b4"]


def inputs(m):
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    ns = m["ns"]
    return gauge_field(ns, m["nt"], m["beta"], m["seed"]), gaussian_spinor(ns * m["nt"], 2, m["seed"] + 1000)


def make_ctx(m, **over):
    from amg_schwingermodel_b200 import AMGContext
    job = m["job"]
    return AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                      nit=job["nit"], sap_tv_iters=job["sap_tv_iters"], **over)


@pytest.mark.parametrize("name", SOLVES)
def test_workload_fp64_matches_reference(name):
    g = load_golden(name)
    m, idx = g["meta"], g["sites"]
    U, b = inputs(m)
    with make_ctx(m) as ctx:
        ctx.set_gauge(U)
        assert rel(ctx.dirac(b)[idx], g["dphi_sample"]) < 1e-13
        ctx.setup()
        x, info = ctx.solve(b)
        hist = ctx.residual_history()
    print(f"{name} FP64: {info[0]['iterations']} iterations (reference {m['iterations']}), "
          f"residual {info[0]['rel_residual']:.2e}, |x - x_ref|/|x_ref| on the sample {rel(x[idx], g['x_sample']):.2e}")
    assert info[0]["iterations"] == m["iterations"]
    assert info[0]["converged"] and info[0]["rel_residual"] < 1e-10
    assert rel(x[idx], g["x_sample"]) < 1e-8
    assert abs(np.linalg.norm(x) / m["x_norm"] - 1) < 1e-8
    np.testing.assert_allclose(hist, g["residual_history"], rtol=1e-5, atol=1e-11 * hist[0])


@pytest.mark.parametrize("name", SOLVES)
def test_workload_mixed_against_reference(name):
    g = load_golden(name)
    m, idx = g["meta"], g["sites"]
    U, b = inputs(m)
    with make_ctx(m, precision=1) as ctx:
        ctx.set_gauge(U)
        ctx.setup()
        x, info = ctx.solve(b)
    err = rel(x[idx], g["x_sample"])
    print(f"{name} mixed: {info[0]['iterations']} iterations (reference {m['iterations']}), "
          f"residual {info[0]['rel_residual']:.2e}, |x - x_ref|/|x_ref| on the sample {err:.2e}")
    assert info[0]["iterations"] <= m["iterations"] + 1
    assert info[0]["converged"] and info[0]["rel_residual"] < 1e-10
    assert err < 1e-8


def test_uneven_batch_32_sources_matches_reference():
    """128^2, 256^2 and 512^2 configurations with 32 sources each, mixed precision, solved
    together (amg_solve_many); each configuration's first source is the fixture's."""
    from amg_schwingermodel_b200 import solve_many
    from amg_schwingermodel_b200.inputs import gaussian_spinor
    ctxs, bs, gs = [], [], []
    try:
        for name in BATCH:
            g = load_golden(name)
            m = g["meta"]
            U, b = inputs(m)
            N = m["ns"] * m["nt"]
            ctx = make_ctx(m, precision=1, max_rhs=32)
            ctxs.append(ctx)
            ctx.set_gauge(U)
            ctx.setup()
            bs.append(np.concatenate([b[None], gaussian_spinor(N, 2, m["seed"] + 5000, nrhs=31)]))
            gs.append(g)
        xs, infos = solve_many(ctxs, bs)
    finally:
        for c in ctxs:
            c.close()
    for g, x, info in zip(gs, xs, infos):
        m = g["meta"]
        assert len(info) == 32
        assert all(i["converged"] and i["rel_residual"] < 1e-10 for i in info), info
        assert info[0]["iterations"] <= m["iterations"] + 1, (m["ns"], info[0], m["iterations"])
        assert rel(x[0][g["sites"]], g["x_sample"]) < 1e-8
