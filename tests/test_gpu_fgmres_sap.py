"""The reference's comparison solver FGMRES_SAP (include/sap.h:194-225): the outer FGMRES with
one fine-level SAP sweep as its preconditioner, selected by amg_set_preconditioner.  The
oracle is the restatement (oracle/restatement.py AMG.solve_sap), which gives the reference's
own FGMRES_SAP runs exactly (tests/golden/krylov*.npz, tests/test_oracle_krylov.py).
Lattices with 4 x 4 SAP blocks, the blocking the reference's FGMRES_SAP uses
(SAPV::sap_block_x/t = 4, include/variables.h:35-36).
Bars: FP64 within one iteration of the restatement (the outer Gram-Schmidt is CGS2 here, MGS
there, so rounding may move the stopping step), mixed precision at most one more; x within
1e-8 and FP64 true residual <= 1e-10 for both; switching back to the multigrid
preconditioner gives the same iteration count as before."""
import pytest

from conftest import rel
from oracle import restatement as R

pytestmark = pytest.mark.gpu

CASES = [(32, [[0, 4, 4, 8, 4, 4]], -0.1, 3.0), (64, [[0, 8, 8, 10, 4, 4]], -0.05, 4.0)]


@pytest.mark.parametrize("ns,rows,m0,beta", CASES)
def test_fgmres_sap_matches_restatement(ns, rows, m0, beta):
    from amg_schwingermodel_b200 import AMGContext, _lib
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    U = gauge_field(ns, ns, beta, 91)
    b = gaussian_spinor(ns * ns, 2, 92)
    amg = R.AMG(U, ns, ns, rows, R.SolverParams(m0=m0))
    x_ref, it_ref = amg.solve_sap(b)
    for prec in (0, 1):
        with AMGContext(ns, ns, rows, m0, precision=prec, autotune=0) as ctx:
            ctx.set_gauge(U)
            ctx.setup()
            _, info_mg = ctx.solve(b)
            ctx.set_preconditioner(_lib.AMG_PRECOND_SAP)
            x, info = ctx.solve(b)
            assert info[0]["converged"] and info[0]["rel_residual"] <= 1e-10, info
            assert R.true_residual(U, x, b, m0, ns, ns) <= 1e-10
            if prec == 0:
                assert abs(info[0]["iterations"] - it_ref) <= 1, (info, it_ref)
            else:
                assert info[0]["iterations"] <= it_ref + 1, (info, it_ref)
            assert rel(x, x_ref) < 1e-8
            ctx.set_preconditioner(_lib.AMG_PRECOND_MG)
            _, info_back = ctx.solve(b)
            assert info_back[0]["iterations"] == info_mg[0]["iterations"]
    with pytest.raises(Exception):
        with AMGContext(ns, ns, rows, m0) as ctx:
            ctx.set_preconditioner(7)
