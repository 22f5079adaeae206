"""Several configurations of uneven lattice sizes solved together (amg_solve_many): each
context's outer FGMRES advances in turn on its own stream.  The results equal the
contexts' own amg_solve results (same kernels, same order: within 1e-12), and on the
reference's fixtures the iteration counts and solutions are the reference's."""
import numpy as np
import pytest

from conftest import load_golden, rel

pytestmark = pytest.mark.gpu


def test_many_fixtures_match_reference_fp64():
    from amg_schwingermodel_b200 import AMGContext, solve_many
    names = ["c32_l3_k", "c64_l2_k", "c64_l3_sap1024", "c16_l2_k"]
    ctxs, bs, gs = [], [], []
    for name in names:
        g = load_golden(name)
        m = g["meta"]
        job = m["job"]
        ctx = AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                         nit=job["nit"], sap_tv_iters=job["sap_tv_iters"])
        ctx.set_gauge(g["gauge"])
        ctx.setup()
        ctxs.append(ctx)
        bs.append(g["rhs"])
        gs.append(g)
    xs, infos = solve_many(ctxs, bs)
    for g, x, info in zip(gs, xs, infos):
        assert info[0]["iterations"] == g["meta"]["iterations"], (g["meta"], info)
        assert info[0]["converged"] and info[0]["rel_residual"] < 1e-10
        assert rel(x, g["x"]) < 1e-8
    for c in ctxs:
        c.close()


def test_many_uneven_mixed_batches_equal_single_solves():
    from amg_schwingermodel_b200 import AMGContext, solve_many
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    # three lattice sizes, beta in {2, 3, 4}, m0 = -0.05, several sources each, mixed precision
    specs = [(32, [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]], 2.0, 3),
             (64, [[0, 8, 8, 8, 2, 2], [1, 4, 4, 8, 2, 2]], 3.0, 2),
             (128, [[0, 8, 8, 12, 4, 4], [1, 4, 4, 12, 4, 4]], 4.0, 4)]
    ctxs, bs = [], []
    for i, (ns, rows, beta, nrhs) in enumerate(specs):
        ctx = AMGContext(ns, ns, rows, -0.05, precision=1, max_rhs=nrhs)
        ctx.set_gauge(gauge_field(ns, ns, beta, 50 + i))
        ctx.setup()
        ctxs.append(ctx)
        bs.append(gaussian_spinor(ns * ns, 2, 60 + i, nrhs=nrhs))
    xs, infos = solve_many(ctxs, bs)
    for ctx, b, x, info in zip(ctxs, bs, xs, infos):
        x1, info1 = ctx.solve(b)
        assert rel(x, x1) < 1e-12
        assert [i["iterations"] for i in info] == [i["iterations"] for i in info1]
        assert all(i["converged"] and i["rel_residual"] < 1e-10 for i in info)
    for c in ctxs:
        c.close()
