"""CPU checks of the arithmetic behind the FP32 SAP kernel's Gram-Schmidt forms, on the
block operator D_B of a 32x32-site Schwarz block (the bench's block shape) of a beta = 4,
m0 = -0.05 U(1) field, in FP64 numpy:

* the classical Gram-Schmidt step with the norm by Pythagoras (|w - V h|^2 = |w|^2 - |h|^2)
  and a second projection when |w_perp| < |w| / 8 gives the block GMRES(5) x 5 restarts
  iterate of the modified Gram-Schmidt form (src/fgmres.cpp:24-32) to 1e-12;
* the modified form with the last projection's norm by Pythagoras does too;
* on these blocks the cancellation ratio |w_perp| / |w| stays well above 1/8 (the kernel's
  second projection is the rare path), for rough and for smooth right-hand sides.
"""
import numpy as np

from oracle import restatement as R

NS, M0, BLK = 64, -0.05, 32


def _block_operator():
    from amg_schwingermodel_b200.inputs import gauge_field
    U = gauge_field(NS, NS, 4.0, 3)
    D = R.dirac_matrix(U, M0, NS, NS).tocsr()
    idx = np.array([(x * NS + t) * 2 + s for x in range(16, 16 + BLK) for t in range(16, 16 + BLK)
                    for s in range(2)])
    return D[idx][:, idx].toarray()


def _gmres(A, b, form, ratios=None, m=5, restarts=5):
    """Block GMRES(m) x restarts from x0 = b, Givens least squares, as the SAP block solve."""
    x = b.copy()
    r = b - A @ x
    for _ in range(restarts):
        beta = np.linalg.norm(r)
        V = [r / beta]
        H = np.zeros((m + 1, m), dtype=complex)
        for j in range(m):
            w = A @ V[j]
            if form == "mgs":
                for i in range(j + 1):
                    H[i, j] = np.vdot(V[i], w)
                    w = w - H[i, j] * V[i]
                hn = np.linalg.norm(w)
            elif form == "mgs_pyth":
                for i in range(j):
                    H[i, j] = np.vdot(V[i], w)
                    w = w - H[i, j] * V[i]
                ww = np.vdot(w, w).real
                H[j, j] = np.vdot(V[j], w)
                w = w - H[j, j] * V[j]
                hn2 = ww - abs(H[j, j]) ** 2
                hn = np.sqrt(hn2) if hn2 >= ww / 64 else np.linalg.norm(w)
            else:   # "cgs": batched dots, Pythagorean norm, second projection on cancellation
                h = np.array([np.vdot(v, w) for v in V])
                ww = np.vdot(w, w).real
                w = w - sum(hi * v for hi, v in zip(h, V))
                hn2 = ww - np.sum(abs(h) ** 2)
                if ratios is not None:
                    ratios.append(np.sqrt(max(hn2, 0.0) / ww))
                if hn2 < ww / 64:
                    h2 = np.array([np.vdot(v, w) for v in V])
                    w = w - sum(hi * v for hi, v in zip(h2, V))
                    h = h + h2
                    hn2 = np.vdot(w, w).real
                H[: j + 1, j] = h
                hn = np.sqrt(max(hn2, 0.0))
            H[j + 1, j] = hn
            V.append(w / hn)
        Vm = np.array(V[:m]).T
        g = np.zeros(m + 1, dtype=complex)
        g[0] = beta
        y = np.linalg.lstsq(H, g, rcond=None)[0]
        x = x + Vm @ y
        r = b - A @ x
    return x


def test_gram_schmidt_forms_give_the_same_block_solve():
    A = _block_operator()
    rng = np.random.default_rng(5)
    for smooth in (False, True):
        b = rng.standard_normal(A.shape[0]) + 1j * rng.standard_normal(A.shape[0])
        if smooth:
            b = np.linalg.solve(A, b)
        ratios = []
        x_mgs = _gmres(A, b, "mgs")
        x_cgs = _gmres(A, b, "cgs", ratios)
        x_pyth = _gmres(A, b, "mgs_pyth")
        assert np.linalg.norm(x_cgs - x_mgs) / np.linalg.norm(x_mgs) < 1e-12
        assert np.linalg.norm(x_pyth - x_mgs) / np.linalg.norm(x_mgs) < 1e-12
        # the second projection (ratio below 1/8) is the rare path on these blocks
        assert min(ratios) > 0.25, min(ratios)
