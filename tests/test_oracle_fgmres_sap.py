"""The restated FGMRES_SAP (include/sap.h:194-225; oracle/restatement.py AMG.solve_sap), the
oracle of the FGMRES+SAP comparison solver: on a 32x32 lattice with 4 x 4 SAP blocks it
converges to the FP64 tolerance (checked with the restated D_phi), and one SAP sweep is a
useful preconditioner (far fewer outer iterations than the unpreconditioned FGMRES(20))."""
import numpy as np

from oracle import restatement as R


def test_restated_fgmres_sap_converges():
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    ns, rows, m0 = 32, [[0, 4, 4, 8, 4, 4]], -0.1
    U = gauge_field(ns, ns, 3.0, 91)
    b = gaussian_spinor(ns * ns, 2, 92)
    amg = R.AMG(U, ns, ns, rows, R.SolverParams(m0=m0))
    x, it = amg.solve_sap(b)
    assert R.true_residual(U, x, b, m0, ns, ns) <= 1e-10
    func = lambda z: R.d_phi(U, z, m0, ns, ns)
    _, it_plain = R.fgmres(func, lambda v, z: v, b, np.zeros_like(b), 20, 50, 1e-10)
    assert it < it_plain / 2, (it, it_plain)
