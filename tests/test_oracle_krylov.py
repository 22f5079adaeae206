"""The restated comparison solvers against the reference's own runs (tests/golden/krylov32.npz
and krylov64.npz, made by tests/golden/make_golden.py from the compiled reference): conjugate_gradient on
D D^dagger (src/conjugate_gradient.cpp:5-65), bi_cgstab (src/bi_cgstab.cpp:5-89) and the
unpreconditioned FGMRES_fine_level(20, 50) (include/fgmres.h:126-148) give the reference's
iteration counts exactly and its solutions to 1e-10."""
import numpy as np
import pytest

from conftest import load_golden, rel
from oracle import restatement as R


CASES = ["krylov32", "krylov64"]


@pytest.mark.parametrize("name", CASES)
def test_restated_cg_and_bicgstab_match_reference(name):
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    g = load_golden(name)
    m = g["meta"]
    ns, m0 = m["ns"], m["m0"]
    U = gauge_field(ns, ns, m["beta"], m["seed"])
    phi = gaussian_spinor(ns * ns, 2, m["seed"] + 1)
    y, k, ok = R.cg_normal(U, phi, m0, ns, ns)
    assert ok and k == m["cg_iterations"], (k, m["cg_iterations"])
    assert rel(y, g["cg_x"]) < 1e-10
    x, k2, ok2 = R.bicgstab(U, phi, np.zeros_like(phi), m0, ns, ns)
    assert ok2 and k2 == m["bicg_iterations"], (k2, m["bicg_iterations"])
    assert rel(x, g["bicg_x"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_restated_unpreconditioned_gmres_matches_reference(name):
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    g = load_golden(name)
    m = g["meta"]
    ns, m0 = m["ns"], m["m0"]
    U = gauge_field(ns, ns, m["beta"], m["seed"])
    phi = gaussian_spinor(ns * ns, 2, m["seed"] + 1)
    x, it = R.gmres_fine(U, phi, np.zeros_like(phi), m0, ns, ns)
    assert it == m["gmres_iterations"], (it, m["gmres_iterations"])
    assert rel(x, g["gmres_x"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_restated_fgmres_sap_matches_reference(name):
    """FGMRES_SAP (include/sap.h:194-225) as Tests::FGMRES_sap runs it, with the global SAP
    object given the gauge field by its set_params: the restatement (4 x 4 SAP blocks, the
    global object's SAPV::sap_block_x/t) takes the reference's iteration count and solution."""
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
    g = load_golden(name)
    m = g["meta"]
    ns, m0 = m["ns"], m["m0"]
    U = gauge_field(ns, ns, m["beta"], m["seed"])
    phi = gaussian_spinor(ns * ns, 2, m["seed"] + 1)
    rows4 = [list(r) for r in m["rows"]]
    rows4[0][4] = rows4[0][5] = 4
    x, it = R.AMG(U, ns, ns, rows4, R.SolverParams(m0=m0)).solve_sap(phi)
    assert it == m["sap_iterations"], (it, m["sap_iterations"])
    assert rel(x, g["sap_x"]) < 1e-10
