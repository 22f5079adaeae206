"""The comparison solvers on the GPU stencil through the C ABI (amg_cg_normal, amg_bicgstab,
amg_solve with AMG_PRECOND_NONE) against the reference's own runs (tests/golden/krylov32.npz):
conjugate_gradient on D D^dagger (src/conjugate_gradient.cpp:5-65), bi_cgstab
(src/bi_cgstab.cpp:5-89) and FGMRES_fine_level(20, 50) (include/fgmres.h:126-148).
Bars: the solutions within 1e-8 of the reference's; iteration counts within 2 of the
reference's (the device sums the dots in another order, which moves the Krylov recurrences
in their last bits); the true residual of D D^dagger y = phi and D x = phi at the 1e-10
tolerance (checked with the restated operator, x10 for the accumulated recurrence drift).
Unpreconditioned GMRES: iterations within 1 of the reference's (CGS2 here, MGS there),
solution within 1e-8, in both context precisions (the mixed context runs it in FP64)."""
import numpy as np
import pytest

from conftest import load_golden, rel
from oracle import restatement as R

pytestmark = pytest.mark.gpu


def test_gpu_cg_and_bicgstab_match_reference():
    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    g = load_golden("krylov32")
    m = g["meta"]
    ns, m0 = m["ns"], m["m0"]
    U = gauge_field(ns, ns, m["beta"], m["seed"])
    phi = gaussian_spinor(ns * ns, 2, m["seed"] + 1)
    with AMGContext(ns, ns, m["rows"], m0) as ctx:
        ctx.set_gauge(U)
        y, k, ok = ctx.cg_normal(phi)
        x, k2, ok2 = ctx.bicgstab(phi)
        xz, k3, ok3 = ctx.bicgstab(phi, x0=np.zeros_like(phi))
    assert ok and abs(k - m["cg_iterations"]) <= 2, (k, m["cg_iterations"])
    assert rel(y, g["cg_x"]) < 1e-8
    ddag = R.d_phi(U, R.d_dagger_phi(U, y, m0, ns, ns), m0, ns, ns)
    assert np.linalg.norm(phi - ddag) / np.linalg.norm(phi) < 1e-9
    assert ok2 and abs(k2 - m["bicg_iterations"]) <= 2, (k2, m["bicg_iterations"])
    assert rel(x, g["bicg_x"]) < 1e-8
    assert R.true_residual(U, x, phi, m0, ns, ns) < 1e-9
    assert ok3 and k3 == k2 and rel(xz, x) == 0.0


@pytest.mark.parametrize("prec", [0, 1])
def test_gpu_unpreconditioned_gmres_matches_reference(prec):
    from amg_schwingermodel_b200 import AMGContext, _lib
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    g = load_golden("krylov32")
    m = g["meta"]
    ns, m0 = m["ns"], m["m0"]
    U = gauge_field(ns, ns, m["beta"], m["seed"])
    phi = gaussian_spinor(ns * ns, 2, m["seed"] + 1)
    with AMGContext(ns, ns, m["rows"], m0, precision=prec) as ctx:
        ctx.set_gauge(U)
        ctx.setup()
        ctx.set_preconditioner(_lib.AMG_PRECOND_NONE)
        x, info = ctx.solve(phi)
        ctx.set_preconditioner(_lib.AMG_PRECOND_MG)
        _, info_mg = ctx.solve(phi)
    assert info[0]["converged"] and info[0]["rel_residual"] <= 1e-10, info
    assert abs(info[0]["iterations"] - m["gmres_iterations"]) <= 1, (info, m["gmres_iterations"])
    assert rel(x, g["gmres_x"]) < 1e-8
    assert R.true_residual(U, x, phi, m0, ns, ns) <= 1e-10
    assert info_mg[0]["converged"] and info_mg[0]["iterations"] < m["gmres_iterations"] // 4
