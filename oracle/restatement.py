"""CPU restatement of the reference's DD-alpha-AMG solve path in numpy (FP64).

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA library is compared
against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
it.  It is pinned against the compiled reference (oracle/_ref, built from the unmodified
reference sources by oracle/build_ref.sh) and against the golden fixtures under
tests/golden/ that the reference produced.

Every function cites the reference file:line it restates (Fabian2598/AMG_SchwingerModel).
Layouts follow the reference: a level-l vector is v[n][dof] with n = x*Nt_l + t and
dof = 2*c + spin; gauge links U[n][mu] with mu = 0 the time direction.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp


# --------------------------------------------------------------------------------------
# Parameters and geometry
# --------------------------------------------------------------------------------------
@dataclass
class LevelParams:
    """One level's sizes, as readParameters fills LevelV (include/params.h:30-62)."""
    l: int
    nx: int
    nt: int
    colors: int
    # aggregation to level l+1 (absent on the coarsest level)
    bx: int = 1
    bt: int = 1
    ntest: int = 1
    # SAP blocking (1x1 on the coarsest level, include/params.h:60-61)
    sbx: int = 1
    sbt: int = 1

    @property
    def n(self) -> int:
        return self.nx * self.nt

    @property
    def dof(self) -> int:
        return 2 * self.colors

    @property
    def xe(self) -> int:  # sites per aggregation block in x (include/level.h:147)
        return self.nx // self.bx

    @property
    def te(self) -> int:
        return self.nt // self.bt

    @property
    def sxe(self) -> int:  # SAP block extent (include/params.h:44-45)
        return self.nx // self.sbx

    @property
    def ste(self) -> int:
        return self.nt // self.sbt


def read_parameters(ns: int, nt: int, rows) -> list[LevelParams]:
    """readParameters (include/params.h:17-69): rows 'level bx bt ntest sbx sbt'."""
    rows = sorted([list(map(int, r)) for r in rows])
    L = len(rows) + 1
    levels = []
    for r in rows:
        l, bx, bt, ntest, sbx, sbt = r
        if l == 0:
            nx_l, nt_l, col = ns, nt, 1
        else:
            p = rows[l - 1]
            nx_l, nt_l, col = p[1], p[2], p[3]
        levels.append(LevelParams(l, nx_l, nt_l, col, bx, bt, ntest, sbx, sbt))
    p = rows[-1]
    levels.append(LevelParams(L - 1, p[1], p[2], p[3]))
    return levels


def boundary(lp: LevelParams):
    """Neighbour and sign tables of one level (include/boundary.h:24-46).

    Returns right[n][mu], left[n][mu] (periodic), signr[n][mu], signl[n][mu]: the time
    direction (mu = 0) is antiperiodic, the sign is -1 on the hop across t = Nt-1 -> 0.
    """
    x, t = np.divmod(np.arange(lp.n), lp.nt)
    right = np.stack([x * lp.nt + (t + 1) % lp.nt, ((x + 1) % lp.nx) * lp.nt + t], axis=1)
    left = np.stack([x * lp.nt + (t - 1) % lp.nt, ((x - 1) % lp.nx) * lp.nt + t], axis=1)
    signr = np.ones((lp.n, 2), dtype=np.int32)
    signl = np.ones((lp.n, 2), dtype=np.int32)
    signr[t == lp.nt - 1, 0] = -1
    signl[t == 0, 0] = -1
    return right.astype(np.int32), left.astype(np.int32), signr, signl


def lattice_blocks(lp: LevelParams) -> np.ndarray:
    """Level::makeBlocks (src/level.cpp:53-73): [NBlocks][sites], block = bx*BlocksT + bt."""
    out = np.empty((lp.bx * lp.bt, lp.xe * lp.te), dtype=np.int32)
    for X in range(lp.bx):
        for T in range(lp.bt):
            xs = np.arange(X * lp.xe, (X + 1) * lp.xe)[:, None]
            ts = np.arange(T * lp.te, (T + 1) * lp.te)[None, :]
            out[X * lp.bt + T] = (xs * lp.nt + ts).reshape(-1)
    return out


def aggregates(lp: LevelParams):
    """Level::makeAggregates (src/level.cpp:3-34).

    Returns agg[2*NBlocks][sites*colors] (element index i = n*colors*2 + c*2 + s) and the
    coordinate tables ncoords, scoords, ccoords indexed by i.
    """
    col = lp.colors
    agg = np.empty((2 * lp.bx * lp.bt, lp.xe * lp.te * col), dtype=np.int32)
    for X in range(lp.bx):
        for T in range(lp.bt):
            for s in range(2):
                a = X * lp.bt * 2 + T * 2 + s
                xs = np.arange(X * lp.xe, (X + 1) * lp.xe)[:, None, None]
                ts = np.arange(T * lp.te, (T + 1) * lp.te)[None, :, None]
                cs = np.arange(col)[None, None, :]
                agg[a] = (xs * lp.nt * col * 2 + ts * col * 2 + cs * 2 + s).reshape(-1)
    i = np.arange(lp.n * 2 * col)
    ncoords = (i // (2 * col)).astype(np.int32)
    ccoords = ((i // 2) % col).astype(np.int32)
    scoords = (i % 2).astype(np.int32)
    return agg, ncoords, scoords, ccoords


def schwarz_blocks(lp: LevelParams):
    """SAP_C::SchwarzBlocks (src/sap.cpp:3-39): block site lists and red/black sets.

    With an even number of blocks in t the colours form a checkerboard over (x, t); with
    an odd number the colour is the block-id parity.  A single block appears in both
    colour lists (the black list keeps its zero initialisation, include/sap.h:68,76-77).
    """
    nb = lp.sbx * lp.sbt
    ncol = nb // 2 if nb != 1 else 1
    blocks = np.empty((nb, lp.sxe * lp.ste), dtype=np.int32)
    red = np.zeros(ncol, dtype=np.int32)
    black = np.zeros(ncol, dtype=np.int32)
    for X in range(lp.sbx):
        for T in range(lp.sbt):
            b = X * lp.sbt + T
            xs = np.arange(X * lp.sxe, (X + 1) * lp.sxe)[:, None]
            ts = np.arange(T * lp.ste, (T + 1) * lp.ste)[None, :]
            blocks[b] = (xs * lp.nt + ts).reshape(-1)
            if lp.sbt % 2 == 0:
                is_red = (b % 2 == 0) if X % 2 == 0 else (b % 2 == 1)
            else:
                is_red = b % 2 == 0
            if b // 2 < ncol:
                (red if is_red else black)[b // 2] = b
    return blocks, red, black


# --------------------------------------------------------------------------------------
# Fine-level Wilson-Dirac operator
# --------------------------------------------------------------------------------------
def d_phi(U: np.ndarray, phi: np.ndarray, m0: float, nx: int, nt: int) -> np.ndarray:
    """D_phi (src/dirac_operator.cpp:3-27)."""
    lp = LevelParams(0, nx, nt, 1)
    R, Lf, sR, sL = boundary(lp)
    p0, p1 = phi[:, 0], phi[:, 1]
    ur0 = U[:, 0] * sR[:, 0]
    ur1 = U[:, 1] * sR[:, 1]
    ul0 = np.conj(U[Lf[:, 0], 0]) * sL[:, 0]
    ul1 = np.conj(U[Lf[:, 1], 1]) * sL[:, 1]
    a, b = p0[R[:, 0]], p1[R[:, 0]]
    c, d = p0[R[:, 1]], p1[R[:, 1]]
    e, f = p0[Lf[:, 0]], p1[Lf[:, 0]]
    g, h = p0[Lf[:, 1]], p1[Lf[:, 1]]
    out = np.empty_like(phi)
    out[:, 0] = (m0 + 2) * p0 - 0.5 * (ur0 * (a - b) + ur1 * (c + 1j * d) + ul0 * (e + f) + ul1 * (g - 1j * h))
    out[:, 1] = (m0 + 2) * p1 - 0.5 * (ur0 * (-a + b) + ur1 * (-1j * c + d) + ul0 * (e + f) + ul1 * (1j * g + h))
    return out


def d_dagger_phi(U: np.ndarray, phi: np.ndarray, m0: float, nx: int, nt: int) -> np.ndarray:
    """D_dagger_phi (src/dirac_operator.cpp:30-54): the spin projectors of D swapped."""
    lp = LevelParams(0, nx, nt, 1)
    R, Lf, sR, sL = boundary(lp)
    p0, p1 = phi[:, 0], phi[:, 1]
    ur0 = U[:, 0] * sR[:, 0]
    ur1 = U[:, 1] * sR[:, 1]
    ul0 = np.conj(U[Lf[:, 0], 0]) * sL[:, 0]
    ul1 = np.conj(U[Lf[:, 1], 1]) * sL[:, 1]
    a, b = p0[R[:, 0]], p1[R[:, 0]]
    c, d = p0[R[:, 1]], p1[R[:, 1]]
    e, f = p0[Lf[:, 0]], p1[Lf[:, 0]]
    g, h = p0[Lf[:, 1]], p1[Lf[:, 1]]
    out = np.empty_like(phi)
    out[:, 0] = (m0 + 2) * p0 - 0.5 * (ul0 * (e - f) + ul1 * (g + 1j * h) + ur0 * (a + b) + ur1 * (c - 1j * d))
    out[:, 1] = (m0 + 2) * p1 - 0.5 * (ul0 * (-e + f) + ul1 * (-1j * g + h) + ur0 * (a + b) + ur1 * (1j * c + d))
    return out


# --------------------------------------------------------------------------------------
# Level operator from link tensors
# --------------------------------------------------------------------------------------
_M = np.array([[[1, -1], [-1, 1]], [[1, 1j], [-1j, 1]]], dtype=np.complex128)   # 1 - sigma_mu
_P = np.array([[[1, 1], [1, 1]], [[1, -1j], [1j, 1]]], dtype=np.complex128)     # 1 + sigma_mu


def make_dirac(U: np.ndarray, lp: LevelParams):
    """Level::makeDirac (src/level.cpp:87-125): level-0 G1 = 0, G2, G3 in the reference's
    index order G[x][alf][bet][c][b][mu] (c = b = 0)."""
    R, Lf, _, _ = boundary(lp)
    N = lp.n
    G1 = np.zeros((N, 2, 2, 1, 1), dtype=np.complex128)
    G2 = np.zeros((N, 2, 2, 1, 1, 2), dtype=np.complex128)
    G3 = np.zeros((N, 2, 2, 1, 1, 2), dtype=np.complex128)
    for mu in range(2):
        G2[:, :, :, 0, 0, mu] = 0.5 * _M[mu][None] * U[:, mu][:, None, None]
        G3[:, :, :, 0, 0, mu] = 0.5 * _P[mu][None] * np.conj(U[Lf[:, mu], mu])[:, None, None]
    return G1, G2, G3


def link_matrices(G1, G2, G3):
    """Reference link tensors -> dense per-site matrices acting on dof = 2c + alf:
    self[x][i][j] = G1[x][alf][bet][c][b], hop[x][mu][i][j] for G2 (right) / G3 (left)."""
    N, _, _, c, _ = G1.shape
    K = 2 * c
    self_m = G1.transpose(0, 3, 1, 4, 2).reshape(N, K, K)
    g2 = G2.transpose(0, 5, 3, 1, 4, 2).reshape(N, 2, K, K)
    g3 = G3.transpose(0, 5, 3, 1, 4, 2).reshape(N, 2, K, K)
    return self_m, g2, g3


def level_operator_matrix(G1, G2, G3, lp: LevelParams, m0: float) -> sp.csr_matrix:
    """Level::D_operator (src/level.cpp:161-180) as a sparse matrix:
    out = (m0+2) v - G1 v - sum_mu (G2 signR v(x+mu) + G3 signL v(x-mu))."""
    R, Lf, sR, sL = boundary(lp)
    self_m, g2, g3 = link_matrices(G1, G2, G3)
    N, K = lp.n, lp.dof
    rows, cols, vals = [], [], []
    base_r = (np.arange(N)[:, None, None] * K + np.arange(K)[None, :, None])
    ii = np.broadcast_to(base_r, (N, K, K))

    def add(mat, nbr):
        jj = np.broadcast_to(nbr[:, None, None] * K + np.arange(K)[None, None, :], (N, K, K))
        rows.append(ii.reshape(-1))
        cols.append(jj.reshape(-1))
        vals.append(mat.reshape(-1))

    add(-self_m, np.arange(N))
    for mu in range(2):
        add(-g2[:, mu] * sR[:, mu][:, None, None], R[:, mu])
        add(-g3[:, mu] * sL[:, mu][:, None, None], Lf[:, mu])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(N * K, N * K))
    A = A + (m0 + 2) * sp.identity(N * K, dtype=np.complex128, format="csr")
    A.sum_duplicates()
    return A.tocsr()


# --------------------------------------------------------------------------------------
# Adjoint: gamma5, the fine operator as a sparse matrix, and the fermion force
# (no reference code; derived from the reference's operator, src/level.cpp:87-180)
# --------------------------------------------------------------------------------------
def gamma5(v: np.ndarray) -> np.ndarray:
    """gamma5 = diag(1, -1) on the spin index of a fine vector [..., N, 2];
    D_dagger_phi = gamma5 D_phi gamma5 (src/dirac_operator.cpp:3-54)."""
    out = np.array(v, dtype=np.complex128, copy=True)
    out[..., 1] *= -1
    return out


def dirac_matrix(U: np.ndarray, m0: float, nx: int, nt: int) -> sp.csr_matrix:
    """The fine Wilson-Dirac operator D (= Level::D_operator at level 0, built from
    Level::makeDirac's links, src/level.cpp:87-180) as a sparse matrix on [N][2]."""
    lp = LevelParams(0, nx, nt, 1)
    G1, G2, G3 = make_dirac(U, lp)
    return level_operator_matrix(G1, G2, G3, lp, m0)


def force(U: np.ndarray, lam: np.ndarray, x: np.ndarray, nx: int, nt: int) -> np.ndarray:
    """F[n][mu] = -sum_r Re(lam_r^dagger (dD/dtheta_mu(n)) x_r) for U = exp(i theta).

    theta_mu(m) enters D (src/level.cpp:161-180 with the level-0 links of :87-125) through
    G2[m][.][.][mu] = 1/2 (1 - sigma_mu) U_mu(m), applied with signR(m, mu) to x(m + mu), and
    G3[m + mu][.][.][mu] = 1/2 (1 + sigma_mu) conj(U_mu(m)), applied with signL(m + mu, mu) to
    x(m); d/dtheta multiplies the first by i and the second by -i.  Since D = (m0+2) - hops,
    F = Re(lam(m)^dag i G2 signR x(m+mu)) + Re(lam(m+mu)^dag (-i) G3 signL x(m))."""
    lp = LevelParams(0, nx, nt, 1)
    R, Lf, sR, sL = boundary(lp)
    _, G2, G3 = make_dirac(U, lp)
    lam = np.asarray(lam).reshape(-1, lp.n, 2)
    x = np.asarray(x).reshape(-1, lp.n, 2)
    F = np.zeros((lp.n, 2))
    for mu in range(2):
        g2 = G2[:, :, :, 0, 0, mu]                       # [m][alf][bet]
        fwd = R[:, mu]                                   # m + mu
        g3 = G3[fwd, :, :, 0, 0, mu]                     # G3 of the row m + mu
        t2 = np.einsum("rma,mab,rmb->m", np.conj(lam), g2, x[:, fwd])
        t3 = np.einsum("rma,mab,rmb->m", np.conj(lam[:, fwd]), g3, x)
        F[:, mu] = np.real(1j * t2 * sR[:, mu]) + np.real(-1j * t3 * sL[fwd, mu])
    return F


# --------------------------------------------------------------------------------------
# Interpolation
# --------------------------------------------------------------------------------------
def site_block(lp: LevelParams) -> np.ndarray:
    """Level::getLatticeBlock (include/level.h:267-278) for every site."""
    x, t = np.divmod(np.arange(lp.n), lp.nt)
    return ((x // lp.xe) * lp.bt + (t // lp.te)).astype(np.int64)


def pt_v(W: np.ndarray, v: np.ndarray, lp: LevelParams) -> np.ndarray:
    """Level::Pt_v (src/level.cpp:212-237): out[nc][2cc+s] = sum_{n in nc, c}
    conj(W[cc][n][2c+s]) v[n][2c+s].  W is [Ntest][N][DOF]."""
    nb = lp.bx * lp.bt
    blk = site_block(lp)
    col = lp.colors
    prod = np.conj(W) * v[None]                       # [Ntest][N][DOF]
    prod = prod.reshape(lp.ntest, lp.n, col, 2).sum(axis=2)   # sum over c -> [Ntest][N][2]
    out = np.zeros((nb, lp.ntest, 2), dtype=np.complex128)
    np.add.at(out, blk, prod.transpose(1, 0, 2))
    return out.reshape(nb, 2 * lp.ntest)


def p_v(W: np.ndarray, vc: np.ndarray, lp: LevelParams) -> np.ndarray:
    """Level::P_v (src/level.cpp:182-209): out[n][2c+s] = sum_cc W[cc][n][2c+s] vc[nc][2cc+s]."""
    blk = site_block(lp)
    col = lp.colors
    vcs = vc.reshape(-1, lp.ntest, 2)[blk]                            # [N][Ntest][2]
    Wr = W.reshape(lp.ntest, lp.n, col, 2)
    out = np.einsum("knca,nka->nca", Wr, vcs)
    return out.reshape(lp.n, lp.dof)


def orthonormalize(W: np.ndarray, lp: LevelParams) -> np.ndarray:
    """Level::orthonormalize (src/level.cpp:373-417): modified Gram-Schmidt of the Ntest
    pieces of every aggregate (block x spin), in the reference's order."""
    W = W.copy()
    blk = site_block(lp)
    nb = lp.bx * lp.bt
    col = lp.colors
    Wr = W.reshape(lp.ntest, lp.n, col, 2)
    order = np.argsort(blk, kind="stable")
    spb = lp.xe * lp.te
    # [Ntest][block][site-in-block][c][s] -> aggregate vectors [block][s][Ntest][spb*c]
    A = Wr[:, order].reshape(lp.ntest, nb, spb, col, 2).transpose(1, 4, 0, 2, 3).reshape(nb, 2, lp.ntest, spb * col)
    for nt in range(lp.ntest):
        for ntt in range(nt):
            proj = np.sum(A[:, :, nt] * np.conj(A[:, :, ntt]), axis=-1)
            A[:, :, nt] -= proj[..., None] * A[:, :, ntt]
        norm = np.sqrt(np.real(np.sum(A[:, :, nt] * np.conj(A[:, :, nt]), axis=-1)))
        A[:, :, nt] /= norm[..., None]
    back = A.reshape(nb, 2, lp.ntest, spb, col).transpose(2, 0, 3, 4, 1).reshape(lp.ntest, lp.n, col, 2)
    Wr[:, order] = back
    return Wr.reshape(lp.ntest, lp.n, lp.dof)


def make_coarse_links(W: np.ndarray, G1, G2, G3, lp: LevelParams, lpn: LevelParams):
    """Level::makeCoarseLinks (src/level.cpp:242-301).

    A(x) collects hops that stay inside block x, B_mu(x) hops from x into block x+mu,
    C_mu(x) hops into block x-mu; no fermionic sign is applied here (the next level's
    operator applies its own).  Returns the next level's G1, G2, G3 in reference layout.
    """
    R, Lf, _, _ = boundary(lp)
    Rn, Ln, _, _ = boundary(lpn)
    blk = site_block(lp)
    col, nts = lp.colors, lp.ntest
    nb = lp.bx * lp.bt
    Wr = W.reshape(nts, lp.n, col, 2)                     # [s][n][b][bet]
    Wc = np.conj(Wr)                                      # [p][n][c][alf]
    A = np.zeros((nb, 2, 2, nts, nts), dtype=np.complex128)
    B = np.zeros((nb, 2, 2, nts, nts, 2), dtype=np.complex128)
    C = np.zeros((nb, 2, 2, nts, nts, 2), dtype=np.complex128)

    def contrib(G, nbr):
        # Y[n][alf][bet][c][s] = sum_b G[n][alf][bet][c][b] W_s[nbr][b][bet]
        Y = np.einsum("nabcd,sndb->nabcs", G, Wr[:, nbr])
        # per-site contribution [n][alf][bet][p][s] = sum_c conj(W_p[n][c][alf]) Y
        return np.einsum("pnca,nabcs->nabps", Wc, Y)

    np.add.at(A, blk, contrib(G1, np.arange(lp.n)))
    for mu in range(2):
        br, bl = blk[R[:, mu]], blk[Lf[:, mu]]
        cr = contrib(G2[..., mu], R[:, mu])
        cl = contrib(G3[..., mu], Lf[:, mu])
        inA = br == blk
        np.add.at(A, blk[inA], cr[inA])
        inB = (~inA) & (br == Rn[blk, mu])
        np.add.at(B[..., mu], blk[inB], cr[inB])
        inA = bl == blk
        np.add.at(A, blk[inA], cl[inA])
        inC = (~inA) & (bl == Ln[blk, mu])
        np.add.at(C[..., mu], blk[inC], cl[inC])
    return A, B, C


# --------------------------------------------------------------------------------------
# Krylov solver
# --------------------------------------------------------------------------------------
def fgmres(func, precond, phi: np.ndarray, x0: np.ndarray, m: int, restarts: int, tol: float,
           history: list | None = None):
    """FGMRES::fgmres (src/fgmres.cpp:5-88) with rotation (:90-104) and the triangular
    solve (:107-115).  Modified Gram-Schmidt; Arnoldi stops when |g_{j+1}| < tol*||phi||;
    a true-residual test after every cycle.  `maxIt` keeps the value of the last early
    exit across restart cycles exactly as the reference does.  The preconditioner is
    called as precond(v_j, z_j) with the Z column's current content: the K-cycle's
    inner FGMRES passes ZmT[j] straight into k_cycle (include/amg.h:37-39), which adds its
    correction to it, and ZmT is only zeroed at the start of a call (include/fgmres.h:93-120),
    so a second restart cycle starts from the previous cycle's z_j.  Returns
    (x, iterations) with iterations = k*m + maxIt, or restarts*m when not converged."""
    shape = phi.shape
    b = phi.reshape(-1)
    n = b.size
    V = np.zeros((m + 1, n), dtype=np.complex128)
    Z = np.zeros((m, n), dtype=np.complex128)
    H = np.zeros((m + 1, m), dtype=np.complex128)
    g = np.zeros(m + 1, dtype=np.complex128)
    sn = np.zeros(m, dtype=np.complex128)
    cn = np.zeros(m, dtype=np.complex128)
    x = x0.reshape(-1).astype(np.complex128).copy()
    r = b - func(x.reshape(shape)).reshape(-1)
    norm_phi = np.sqrt(np.real(np.vdot(b, b)))
    err = np.sqrt(np.real(np.vdot(r, r)))
    max_it = m
    for k in range(restarts):
        beta = err
        V[0] = r / beta
        g[0] = beta
        for j in range(m):
            Z[j] = precond(V[j].reshape(shape), Z[j].reshape(shape)).reshape(-1)
            w = func(Z[j].reshape(shape)).reshape(-1).copy()
            for i in range(j + 1):
                H[i, j] = np.sum(w * np.conj(V[i]))
                w -= H[i, j] * V[i]
            H[j + 1, j] = np.sqrt(np.real(np.vdot(w, w)))
            if np.real(H[j + 1, j]) > 0:
                V[j + 1] = w / H[j + 1, j]
            for i in range(j):
                temp = np.conj(cn[i]) * H[i, j] + np.conj(sn[i]) * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cn[i] * H[i + 1, j]
                H[i, j] = temp
            den = np.sqrt(np.conj(H[j, j]) * H[j, j] + np.conj(H[j + 1, j]) * H[j + 1, j])
            sn[j] = H[j + 1, j] / den
            cn[j] = H[j, j] / den
            H[j, j] = np.conj(cn[j]) * H[j, j] + np.conj(sn[j]) * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = np.conj(cn[j]) * g[j]
            if history is not None:
                history.append(abs(g[j + 1]))
            if abs(g[j + 1]) < tol * norm_phi:
                max_it = j + 1
                break
        eta = np.zeros(m, dtype=np.complex128)
        for i in range(max_it - 1, -1, -1):
            eta[i] = g[i]
            for jj in range(i + 1, max_it):
                eta[i] -= H[i, jj] * eta[jj]
            eta[i] /= H[i, i]
        x += eta[:max_it] @ Z[:max_it]
        r = b - func(x.reshape(shape)).reshape(-1)
        err = np.sqrt(np.real(np.vdot(r, r)))
        if err < tol * norm_phi:
            return x.reshape(shape), k * m + max_it
    return x.reshape(shape), restarts * m


# --------------------------------------------------------------------------------------
# Initial test vectors
# --------------------------------------------------------------------------------------
class ReferenceUniform:
    """The draw `distribution(randomInt) + I_number * distribution(randomInt)` of
    AlgebraicMG::setUpPhase (src/amg.cpp:8-16) with a std::mt19937(50) and
    std::uniform_real_distribution<double>(-1, 1) from libstdc++: each double takes two
    32-bit outputs, u = (x1 + x2 * 2^32) / 2^64, value = -1 + 2u.  g++ evaluates the
    imaginary operand first, so the first double of a pair is the imaginary part.
    numpy's legacy RandomState seeds MT19937 with the same init_genrand."""

    def __init__(self, seed: int = 50):
        self._bg = np.random.RandomState(seed)._bit_generator

    def complex(self, count: int) -> np.ndarray:
        raw = self._bg.random_raw(4 * count).astype(np.float64)
        d = -1.0 + 2.0 * ((raw[0::2] + raw[1::2] * 4294967296.0) / 18446744073709551616.0)
        return d[1::2] + 1j * d[0::2]


def reference_initial_test_vectors(lps: list) -> list:
    """The test vectors setUpPhase starts from (src/amg.cpp:8-35): level 0 uniform draws in
    [i][n][dof] order; level l >= 1 column i < Ntest[l-1] is P^dagger of level l-1 column i
    built with the still-random level l-1 interpolator, later columns are fresh draws."""
    rng = ReferenceUniform(50)
    out = []
    lp0 = lps[0]
    out.append(rng.complex(lp0.ntest * lp0.n * lp0.dof).reshape(lp0.ntest, lp0.n, lp0.dof))
    for l in range(1, len(lps) - 1):
        lp, lpp = lps[l], lps[l - 1]
        W = np.empty((lp.ntest, lp.n, lp.dof), dtype=np.complex128)
        for i in range(lp.ntest):
            if i < lpp.ntest:
                W[i] = pt_v(out[l - 1], out[l - 1][i], lpp)
            else:
                W[i] = rng.complex(lp.n * lp.dof).reshape(lp.n, lp.dof)
        out.append(W)
    return out


# --------------------------------------------------------------------------------------
# Hierarchy, SAP and the cycles
# --------------------------------------------------------------------------------------
@dataclass
class SolverParams:
    """Solver knobs with the reference's defaults (src/variables.cpp:46-87) and the values
    its main sets (src/main.cpp:61-65, :129)."""
    m0: float = -0.1
    cycle: int = 1              # 1 = K-cycle, 0 = V-cycle (AMGV::cycle)
    nu1: int = 0
    nu2: int = 2
    nit: int = 0
    sap_tv_iters: int = 4
    sap_gmres_m: int = 5
    sap_gmres_restarts: int = 5
    sap_gmres_tol: float = 1e-3
    sap_tol: float = 1e-10
    kcycle_m: int = 5
    kcycle_restarts: int = 2
    kcycle_tol: float = 0.1
    coarse_m: int = 20          # LevelV::GMRES_*[maxLevel] (include/params.h:63-65)
    coarse_restarts: int = 20
    coarse_tol: float = 0.1
    outer_m: int = 20
    outer_restarts: int = 50
    outer_tol: float = 1e-10


@dataclass
class Level:
    lp: LevelParams
    G1: np.ndarray
    G2: np.ndarray
    G3: np.ndarray
    W: np.ndarray | None = None          # interpolator columns [Ntest][N][DOF]
    D: sp.csr_matrix | None = None
    sap_blocks: np.ndarray | None = None
    sap_red: np.ndarray | None = None
    sap_black: np.ndarray | None = None
    local_ops: dict = field(default_factory=dict)

    def apply(self, v):
        return (self.D @ v.reshape(-1)).reshape(v.shape)


class AMG:
    """AlgebraicMG (include/amg.h:8-94, src/amg.cpp) over numpy levels."""

    def __init__(self, U: np.ndarray, ns: int, nt: int, rows, sp_: SolverParams):
        self.p = sp_
        self.lps = read_parameters(ns, nt, rows)
        self.U = U
        self.ns, self.nt = ns, nt
        G1, G2, G3 = make_dirac(U, self.lps[0])
        self.levels = [Level(self.lps[0], G1, G2, G3)]
        for lp in self.lps[1:]:
            self.levels.append(Level(lp, None, None, None))
        self._finish_level(0)

    # -- per-level operator state
    def _finish_level(self, l: int):
        L = self.levels[l]
        L.D = level_operator_matrix(L.G1, L.G2, L.G3, L.lp, self.p.m0)
        L.sap_blocks, L.sap_red, L.sap_black = schwarz_blocks(L.lp)
        L.local_ops = {}

    def local_op(self, l: int, block: int):
        """SAP_level_l::D_local (src/level.cpp:304-368): the level operator restricted to
        one SAP block, neighbours outside the block dropped."""
        L = self.levels[l]
        if block not in L.local_ops:
            K = L.lp.dof
            idx = (L.sap_blocks[block][:, None] * K + np.arange(K)[None, :]).reshape(-1)
            L.local_ops[block] = (L.D[idx][:, idx].tocsr(), idx)
        return L.local_ops[block]

    def sap(self, l: int, v: np.ndarray, x: np.ndarray, nu: int) -> tuple[np.ndarray, int]:
        """SAP_C::SAP (src/sap.cpp:64-174) with every block of a colour solved."""
        L = self.levels[l]
        p = self.p
        K = L.lp.dof
        x = x.copy()
        vf = v.reshape(-1)
        v_norm = np.sqrt(np.real(np.vdot(vf, vf)))
        r = vf - L.D @ x.reshape(-1)
        err = None
        for _ in range(nu):
            for colour in (L.sap_red, L.sap_black):
                upd = np.zeros_like(vf)
                for blk in colour:
                    A, idx = self.local_op(l, int(blk))
                    rb = r[idx]
                    xb, _ = fgmres(lambda z: A @ z, lambda v, z: v, rb, rb, p.sap_gmres_m,
                                   p.sap_gmres_restarts, p.sap_gmres_tol)
                    upd[idx] = xb
                x = (x.reshape(-1) + upd).reshape(x.shape)
                r = vf - L.D @ x.reshape(-1)
            err = np.sqrt(np.real(np.vdot(r, r)))
            if err < p.sap_tol * v_norm:
                return x, 1
        return x, 0

    def setup_from(self, init_tv: list):
        """setUpPhase (src/amg.cpp:3-88) after its random draw: SAP-smooth each test
        vector on D x = 0, orthonormalise, build the next level's links; then Nit
        bootstrap passes.  init_tv[l] is [Ntest_l][N_l][DOF_l]."""
        p = self.p
        nl = len(self.levels)
        for l in range(nl - 1):
            L = self.levels[l]
            W = np.array(init_tv[l], dtype=np.complex128).copy()
            zero = np.zeros((L.lp.n, L.lp.dof), dtype=np.complex128)
            for i in range(L.lp.ntest):
                W[i], _ = self.sap(l, zero, W[i], p.sap_tv_iters)
            L.W = orthonormalize(W, L.lp)
            self._coarsen(l)
        for _ in range(p.nit):
            for l in range(nl - 1):
                L = self.levels[l]
                newW = np.empty_like(L.W)
                for i in range(L.lp.ntest):
                    v = L.W[i]
                    rhs = v - L.apply(v)
                    z = np.zeros_like(v)
                    z = self.k_cycle(l, rhs, z) if p.cycle == 1 else self.v_cycle(l, rhs, z)
                    newW[i] = z + v
                L.W = orthonormalize(newW, L.lp)
                self._coarsen(l)

    def _coarsen(self, l: int):
        L, Ln = self.levels[l], self.levels[l + 1]
        A, B, C = make_coarse_links(L.W, L.G1, L.G2, L.G3, L.lp, Ln.lp)
        Ln.G1, Ln.G2, Ln.G3 = A, B, C
        self._finish_level(l + 1)

    def coarsest_solve(self, eta):
        """Level::GMRES_level_l on the coarsest level, x0 = rhs (src/amg.cpp:136-139)."""
        p = self.p
        L = self.levels[-1]
        x, _ = fgmres(L.apply, lambda v, z: v, eta, eta, p.coarse_m, p.coarse_restarts, p.coarse_tol)
        return x

    def k_cycle(self, l: int, eta: np.ndarray, psi: np.ndarray) -> np.ndarray:
        """AlgebraicMG::k_cycle (src/amg.cpp:135-178)."""
        p = self.p
        if l == len(self.levels) - 1:
            return self.coarsest_solve(eta)
        L = self.levels[l]
        if p.nu1 > 0:
            psi, _ = self.sap(l, eta, psi, p.nu1)
        r = eta - L.apply(psi)
        eta_c = pt_v(L.W, r, L.lp)
        psi_c, _ = fgmres(self.levels[l + 1].apply, lambda v, z: self.k_cycle(l + 1, v, z),
                          eta_c, eta_c, p.kcycle_m, p.kcycle_restarts, p.kcycle_tol)
        psi = psi + p_v(L.W, psi_c, L.lp)
        if p.nu2 > 0:
            psi, _ = self.sap(l, eta, psi, p.nu2)
        return psi

    def v_cycle(self, l: int, eta: np.ndarray, psi: np.ndarray) -> np.ndarray:
        """AlgebraicMG::v_cycle (src/amg.cpp:90-132)."""
        p = self.p
        if l == len(self.levels) - 1:
            return self.coarsest_solve(eta)
        L = self.levels[l]
        if p.nu1 > 0:
            psi, _ = self.sap(l, eta, psi, p.nu1)
        r = eta - L.apply(psi)
        eta_c = pt_v(L.W, r, L.lp)
        psi_c = self.v_cycle(l + 1, eta_c, np.zeros_like(eta_c))
        psi = psi + p_v(L.W, psi_c, L.lp)
        if p.nu2 > 0:
            psi, _ = self.sap(l, eta, psi, p.nu2)
        return psi

    def precondition(self, v: np.ndarray, z_old=None) -> np.ndarray:
        """FGMRES_AMG::preconditioner (include/amg.h:134-144): zero, then one cycle."""
        z = np.zeros_like(v)
        return self.k_cycle(0, v, z) if self.p.cycle == 1 else self.v_cycle(0, v, z)

    def solve(self, b: np.ndarray, history: list | None = None):
        """FGMRES_AMG::fgmres(b, x0 = 0, x) (include/amg.h:99-145, src/fgmres.cpp:5-88)
        with func = D_phi."""
        p = self.p
        func = lambda z: d_phi(self.U, z, p.m0, self.ns, self.nt)
        return fgmres(func, self.precondition, b, np.zeros_like(b), p.outer_m, p.outer_restarts,
                      p.outer_tol, history)


    def solve_sap(self, b: np.ndarray, history: list | None = None):
        """FGMRES_SAP::fgmres(b, x0 = 0, x) (include/sap.h:194-225, run by Tests::FGMRES_sap,
        src/tests.cpp:33-46): func = D_phi; the preconditioner zeroes z and applies
        SAP_C::SAP(v, z, nu = 1) on the fine level."""
        p = self.p
        func = lambda z: d_phi(self.U, z, p.m0, self.ns, self.nt)
        precond = lambda v, z: self.sap(0, v, np.zeros_like(v), 1)[0]
        return fgmres(func, precond, b, np.zeros_like(b), p.outer_m, p.outer_restarts, p.outer_tol, history)


def gmres_fine(U, phi, x0, m0, nx, nt, m: int = 20, restarts: int = 50, tol: float = 1e-10,
               history: list | None = None):
    """FGMRES_fine_level::fgmres (include/fgmres.h:126-148, run by Tests::GMRES,
    src/tests.cpp:13-22): func = D_phi, the identity as preconditioner; returns (x, iterations)."""
    func = lambda z: d_phi(U, z, m0, nx, nt)
    return fgmres(func, lambda v, z: v.copy(), phi, x0, m, restarts, tol, history)


def cg_normal(U, phi, m0, nx, nt, max_iter: int = 100000, tol: float = 1e-10):
    """conjugate_gradient (src/conjugate_gradient.cpp:5-65): x = (D D^dagger)^{-1} phi from
    x = phi; returns (x, k, converged) with k the reference's iteration count at convergence."""
    ddag = lambda v: d_phi(U, d_dagger_phi(U, v, m0, nx, nt), m0, nx, nt)
    x = phi.astype(np.complex128).copy()
    r = phi - ddag(x)
    d = r.copy()
    r_norm2 = np.sum(r * np.conj(r))
    phi_norm = np.sqrt(np.real(np.sum(phi * np.conj(phi))))
    k = 0
    while k < max_iter:
        Ad = ddag(d)
        alpha = r_norm2 / np.sum(d * np.conj(Ad))
        x = x + alpha * d
        r = r - alpha * Ad
        err_sqr = np.real(np.sum(r * np.conj(r)))
        if np.sqrt(err_sqr) < tol * phi_norm:
            return x, k, True
        beta = err_sqr / r_norm2
        d = d * beta + r
        r_norm2 = err_sqr
        k += 1
    return x, k, False


def bicgstab(U, phi, x0, m0, nx, nt, max_iter: int = 100000, tol: float = 1e-10):
    """bi_cgstab (src/bi_cgstab.cpp:5-89) with func = D_phi: D x = phi from x0; returns
    (x, iterations, converged) with iterations = k + 1 at convergence."""
    A = lambda v: d_phi(U, v, m0, nx, nt)
    x = x0.astype(np.complex128).copy()
    r = phi - A(x)
    r_tilde = r.copy()
    norm_phi = np.sqrt(np.real(np.sum(phi * np.conj(phi))))
    k = 0
    alpha = omega = rho_i_2 = 0.0
    d = np.zeros_like(r)
    Ad = np.zeros_like(r)
    while k < max_iter:
        rho_i = np.sum(r * np.conj(r_tilde))
        if k == 0:
            d = r.copy()
        else:
            beta = alpha * rho_i / (omega * rho_i_2)
            d = r + beta * (d - omega * Ad)
        Ad = A(d)
        alpha = rho_i / np.sum(Ad * np.conj(r_tilde))
        s = r - alpha * Ad
        if np.sqrt(np.real(np.sum(s * np.conj(s)))) < tol * norm_phi:
            return x + alpha * d, k + 1, True
        t = A(s)
        omega = np.sum(s * np.conj(t)) / np.sum(t * np.conj(t))
        r = s - omega * t
        x = x + alpha * d + omega * s
        rho_i_2 = rho_i
        k += 1
    return x, k, False


def true_residual(U, x, b, m0, nx, nt) -> float:
    r = b - d_phi(U, x, m0, nx, nt)
    return float(np.linalg.norm(r) / np.linalg.norm(b))
