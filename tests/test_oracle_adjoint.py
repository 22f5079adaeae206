"""CPU checks of the adjoint restatement (the checker of the GPU adjoint solve and force).

* gamma5-hermiticity: gamma5 D_phi gamma5 equals the reference's own D_dagger_phi output
  stored in the golden fixtures.
* force(): the restated dL/dtheta of L = Re(eta^dagger D^{-1} b) equals central finite
  differences (h = 1e-6) of L over every link of an 8x8 lattice, with exact sparse solves.
* the adjoint fixture: the reference's two FGMRES_AMG solves (x = D^{-1} b and
  y = D^{-1} gamma5 eta) solve the restated D to the reference's tolerance, and the gradient
  built from them agrees with the exact (sparse LU) gradient.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as sla

from conftest import golden_names, load_golden, rel
from oracle import restatement as R


@pytest.mark.parametrize("name", golden_names())
def test_gamma5_hermiticity_against_reference(name):
    g = load_golden(name)
    m = g["meta"]
    out = R.gamma5(R.d_phi(g["gauge"], R.gamma5(g["rhs"]), m["m0"], m["ns"], m["nt"]))
    assert rel(out, g["ddagphi"]) < 1e-14


def test_force_matches_central_differences():
    from amg_schwingermodel_b200.inputs import gauge_angles, gaussian_spinor
    nx = nt = 8
    m0 = -0.1
    th = gauge_angles(nx, nt, 2.0, 3)
    b = gaussian_spinor(nx * nt, 2, 4).reshape(-1)
    eta = gaussian_spinor(nx * nt, 2, 5).reshape(-1)
    D = R.dirac_matrix(np.exp(1j * th), m0, nx, nt).tocsc()
    x = sla.spsolve(D, b)
    lam = sla.spsolve(D.conj().T.tocsc(), eta)
    F = R.force(np.exp(1j * th), lam.reshape(-1, 2), x.reshape(-1, 2), nx, nt)

    def loss(t):
        Dt = R.dirac_matrix(np.exp(1j * t), m0, nx, nt).tocsc()
        return np.real(np.vdot(eta, sla.spsolve(Dt, b)))

    h = 1e-6
    fd = np.zeros_like(F)
    for n in range(nx * nt):
        for mu in range(2):
            tp, tm = th.copy(), th.copy()
            tp[n, mu] += h
            tm[n, mu] -= h
            fd[n, mu] = (loss(tp) - loss(tm)) / (2 * h)
    assert rel(F, fd) < 1e-6


def test_adjoint_fixture_two_solve_gradient():
    from amg_schwingermodel_b200.inputs import gauge_angles, gaussian_spinor
    g = load_golden("adj128_l3")
    m = g["meta"]
    ns, seed = m["ns"], m["seed"]
    N = ns * ns
    U = np.exp(1j * gauge_angles(ns, ns, m["beta"], seed))
    b = gaussian_spinor(N, 2, seed + 1000)
    eta = gaussian_spinor(N, 2, seed + 3000)
    assert R.true_residual(U, g["x"], b, m["m0"], ns, ns) < 1e-10
    assert R.true_residual(U, g["y"], R.gamma5(eta), m["m0"], ns, ns) < 1e-10
    F_ref = R.force(U, R.gamma5(g["y"]), g["x"], ns, ns)
    lu = sla.splu(R.dirac_matrix(U, m["m0"], ns, ns).tocsc())
    x = lu.solve(b.reshape(-1)).reshape(-1, 2)
    lam = lu.solve(eta.reshape(-1), trans="H").reshape(-1, 2)
    assert rel(F_ref, R.force(U, lam, x, ns, ns)) < 1e-8
