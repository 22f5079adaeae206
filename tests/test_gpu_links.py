"""Low-precision storage of the fine links in the mixed form (amg_params.link_storage: BF16 or
FP16 pairs, FP32 arithmetic): complete solves at 256x256 (3 levels) and 1024x1024 (4 levels,
the benchmark rows) against the reference's solves (tests/golden/solve*.npz).

Bars, as for the mixed form with FP32 links: at most one outer iteration more than the
reference, FP64 true residual <= 1e-10, x within 1e-8 of the reference's on the fixture's site
sample.  The storage is also checked to be in effect: the preconditioner output of one cycle
changes the solve's residual history by more than FP32 rounding would.
"""
import numpy as np
import pytest

from conftest import load_golden, rel

pytestmark = pytest.mark.gpu


def inputs(m):
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    return gauge_field(m["ns"], m["nt"], m["beta"], m["seed"]), gaussian_spinor(m["ns"] * m["nt"], 2, m["seed"] + 1000)


@pytest.mark.parametrize("name", ["solve256_l3", "solve1024_l4"])
@pytest.mark.parametrize("storage", [1, 2])
def test_low_precision_links_solve_matches_reference(name, storage):
    from amg_schwingermodel_b200 import AMGContext
    g = load_golden(name)
    m, idx = g["meta"], g["sites"]
    job = m["job"]
    U, b = inputs(m)
    with AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                    nit=job["nit"], sap_tv_iters=job["sap_tv_iters"], precision=1, link_storage=storage) as ctx:
        ctx.set_gauge(U)
        ctx.setup()
        x, info = ctx.solve(b)
    err = rel(x[idx], g["x_sample"])
    print(f"{name} links={'bf16' if storage == 1 else 'f16'}: {info[0]['iterations']} iterations "
          f"(reference {m['iterations']}), residual {info[0]['rel_residual']:.2e}, x error {err:.2e}")
    assert info[0]["iterations"] <= m["iterations"] + 1
    assert info[0]["converged"] and info[0]["rel_residual"] < 1e-10
    assert err < 1e-8


def test_link_storage_is_in_effect():
    """The mixed solves' residual histories (|g_{j+1}| per Arnoldi step) carry the rounding of
    their cycles, so BF16 or FP16 links move them away from the FP32-link solve's."""
    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    ns = 64
    rows = [[0, 8, 8, 8, 2, 2], [1, 4, 4, 8, 2, 2]]
    U = gauge_field(ns, ns, 3.0, 7)
    b = gaussian_spinor(ns * ns, 2, 8)
    hist = {}
    for storage in (0, 1, 2):
        with AMGContext(ns, ns, rows, -0.05, precision=1, link_storage=storage) as ctx:
            ctx.set_gauge(U)
            ctx.setup()
            x, info = ctx.solve(b)
            assert info[0]["converged"]
            hist[storage] = ctx.residual_history()
    n = min(len(h) for h in hist.values())
    d_bf = np.max(np.abs(hist[1][:n] / hist[0][:n] - 1))
    d_h = np.max(np.abs(hist[2][:n] / hist[0][:n] - 1))
    # the residual estimates move by more than FP32 rounding would move them
    assert d_bf > 1e-6 and d_h > 1e-7
