"""B200-native DD-alpha-AMG for the 2-D Schwinger-model Wilson-Dirac operator.

Python host API over the C ABI of libschwinger_amg.so (include/schwinger_amg.h).  The
C++ drop-in classes mirroring the reference (FGMRES_AMG, AlgebraicMG, Level, SAP_C, ...)
live in include/amg_b200/; this module mirrors the same operations for Python callers,
tests and the torch.autograd wrapper (amg_schwingermodel_b200.autograd).

Arrays use the reference's layouts: spinors psi[N][2] complex128 with n = x*Nt + t, gauge
links U[N][2], level-l vectors v[N_l][DOF_l].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import AmgError, AmgParams, AmgSolveInfo, check, default_params, lib  # noqa: F401

__all__ = ["AMGContext", "AmgError", "AmgParams", "default_params", "read_parameters", "dirac_apply_raw",
           "solve_many", "solve_many_dev"]


def _cptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _c128(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if shape is not None:
        a = a.reshape(shape)
    return a


def launch_count() -> int:
    """Kernels launched by the library so far (all contexts)."""
    return int(lib().amg_launch_count())


def read_parameters(path: str) -> list:
    """readParameters (include/params.h:17-69): the rows of a parameters.dat file."""
    rows = np.zeros((64, 6), dtype=np.int32)
    n = C.c_int(0)
    check(lib().amg_read_parameters(str(path).encode(), _cptr(rows), 64, C.byref(n)), "amg_read_parameters")
    return rows[: n.value].tolist()


def dirac_apply_raw(U_ptr: int, in_ptr: int, out_ptr: int, nx: int, nt: int, nrhs: int, m0: float,
                    dagger: bool = False, stream: int = 0) -> None:
    """The stand-alone FP64 stencil on caller-owned device memory (raw device pointers)."""
    check(lib().amg_dirac_apply_raw(C.c_void_p(U_ptr), C.c_void_p(in_ptr), C.c_void_p(out_ptr), nx, nt, nrhs,
                                    float(m0), int(dagger), C.c_void_p(stream)), "amg_dirac_apply_raw")


def solve_many(ctxs, bs):
    """amg_solve_many: the solves of several contexts (any lattice sizes) driven together.
    bs[i] is [N_i][2] or [nrhs_i][N_i][2]; returns (xs, infos) per context."""
    n = len(ctxs)
    bs = [_c128(b) for b in bs]
    xs = [np.empty_like(b) for b in bs]
    nrhs = (C.c_int * n)(*[1 if b.ndim == 2 else b.shape[0] for b in bs])
    infos = [(AmgSolveInfo * nrhs[i])() for i in range(n)]
    hs = (C.c_void_p * n)(*[c._h.value for c in ctxs])
    bp = (C.c_void_p * n)(*[b.ctypes.data for b in bs])
    xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    ip = (C.c_void_p * n)(*[C.cast(i, C.c_void_p).value for i in infos])
    check(lib().amg_solve_many(n, hs, bp, xp, nrhs, ip), "amg_solve_many")
    return xs, [[dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                 for i in inf] for inf in infos]


def solve_many_dev(ctxs, b_ptrs, x_ptrs, nrhs):
    """amg_solve_many_dev: as solve_many, on device buffers (one [nrhs_i][N_i][2] complex128
    source and solution buffer per context, on that context's device).  Returns the infos."""
    n = len(ctxs)
    nr = (C.c_int * n)(*[int(r) for r in nrhs])
    infos = [(AmgSolveInfo * nr[i])() for i in range(n)]
    hs = (C.c_void_p * n)(*[c._h.value for c in ctxs])
    bp = (C.c_void_p * n)(*[int(p) for p in b_ptrs])
    xp = (C.c_void_p * n)(*[int(p) for p in x_ptrs])
    ip = (C.c_void_p * n)(*[C.cast(i, C.c_void_p).value for i in infos])
    check(lib().amg_solve_many_dev(n, hs, bp, xp, nr, ip), "amg_solve_many_dev")
    return [[dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual) for i in inf]
            for inf in infos]


class AMGContext:
    """One lattice, gauge field and multigrid hierarchy on one GPU.

    Mirrors the reference's solve path: the constructor takes what FGMRES_AMG and
    AlgebraicMG take (lattice NS x NT, the parameters.dat rows, m0, solver knobs);
    setup() is AlgebraicMG::setUpPhase; solve() is FGMRES_AMG::fgmres(b, 0, x).
    """

    def __init__(self, nx: int, nt: int, rows, m0: float, params: AmgParams | None = None, device: int = 0,
                 **param_over):
        self.nx, self.nt = int(nx), int(nt)
        self.rows = [list(map(int, r)) for r in rows]
        self.levels = len(self.rows) + 1
        self.m0 = float(m0)
        self.device = int(device)
        p = params if params is not None else default_params(**param_over)
        self.params = p
        r = np.ascontiguousarray(np.array(self.rows, dtype=np.int32).reshape(-1))
        h = C.c_void_p()
        check(lib().amg_create(C.byref(h), self.nx, self.nt, self.levels, _cptr(r), self.m0, C.byref(p), device),
              "amg_create")
        self._h = h
        self.info = [self.level_info(l) for l in range(self.levels)]

    def close(self):
        if getattr(self, "_h", None):
            lib().amg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- geometry
    def level_info(self, level: int) -> dict:
        o = np.zeros(6, dtype=np.int32)
        check(lib().amg_level_info(self._h, level, _cptr(o)), "amg_level_info")
        return dict(n=int(o[0]), nx=int(o[1]), nt=int(o[2]), dof=int(o[3]), colors=int(o[4]), ntest=int(o[5]))

    @property
    def N(self) -> int:
        return self.nx * self.nt

    def _vshape(self, level: int):
        i = self.info[level]
        return (i["n"], i["dof"])

    # ---- operator
    def set_gauge(self, U) -> None:
        U = _c128(U, (self.N, 2))
        check(lib().amg_set_gauge(self._h, _cptr(U)), "amg_set_gauge")

    def set_mass(self, m0: float) -> None:
        self.m0 = float(m0)
        check(lib().amg_set_mass(self._h, self.m0), "amg_set_mass")

    def cg_normal(self, phi, max_iter: int = 100000, tol: float = 1e-10):
        """conjugate_gradient (src/conjugate_gradient.cpp:5-65): x = (D D^dagger)^{-1} phi.
        Returns (x, iterations, converged)."""
        phi = _c128(phi, (self.nx * self.nt, 2))
        x = np.empty_like(phi)
        it = C.c_int(0)
        st = check(lib().amg_cg_normal(self._h, _cptr(phi), _cptr(x), int(max_iter), float(tol), C.byref(it)),
                   "amg_cg_normal")
        return x, it.value, st == _lib.AMG_OK

    def bicgstab(self, phi, x0=None, max_iter: int = 100000, tol: float = 1e-10):
        """bi_cgstab (src/bi_cgstab.cpp:5-89): D x = phi from x0 (zero when None).
        Returns (x, iterations, converged)."""
        phi = _c128(phi, (self.nx * self.nt, 2))
        x = np.empty_like(phi)
        it = C.c_int(0)
        x0a = None if x0 is None else _c128(x0, (self.nx * self.nt, 2))
        x0p = None if x0a is None else _cptr(x0a)
        st = check(lib().amg_bicgstab(self._h, _cptr(phi), x0p, _cptr(x), int(max_iter), float(tol), C.byref(it)),
                   "amg_bicgstab")
        return x, it.value, st == _lib.AMG_OK

    def set_preconditioner(self, kind: int) -> None:
        """amg_set_preconditioner: _lib.AMG_PRECOND_MG (FGMRES_AMG, default),
        _lib.AMG_PRECOND_SAP (the reference's FGMRES_SAP, include/sap.h:194-225) or
        _lib.AMG_PRECOND_NONE (FGMRES_fine_level, include/fgmres.h:126-148)."""
        check(lib().amg_set_preconditioner(self._h, int(kind)), "amg_set_preconditioner")

    def dirac(self, psi, dagger: bool = False) -> np.ndarray:
        """D_phi / D_dagger_phi on [N][2] or [nrhs][N][2]."""
        psi = _c128(psi)
        nrhs = 1 if psi.ndim == 2 else psi.shape[0]
        out = np.empty_like(psi)
        check(lib().amg_dirac_apply(self._h, _cptr(psi), _cptr(out), nrhs, int(dagger)), "amg_dirac_apply")
        return out

    # ---- set-up
    def set_initial_test_vectors(self, level: int, W) -> None:
        i = self.info[level]
        W = _c128(W, (i["ntest"], i["n"], i["dof"]))
        check(lib().amg_set_initial_test_vectors(self._h, level, _cptr(W)), "amg_set_initial_test_vectors")

    def setup(self) -> float:
        check(lib().amg_setup(self._h), "amg_setup")
        return self.timings()[0]

    def test_vectors(self, level: int) -> np.ndarray:
        i = self.info[level]
        W = np.empty((i["ntest"], i["n"], i["dof"]), dtype=np.complex128)
        check(lib().amg_get_test_vectors(self._h, level, _cptr(W)), "amg_get_test_vectors")
        return W

    def coarse_links(self, level: int):
        """Level::G1/G2/G3 of level >= 1 in the reference's layout (flattened)."""
        i = self.info[level]
        n, c = i["n"], i["colors"]
        G1 = np.empty(n * 4 * c * c, dtype=np.complex128)
        G2 = np.empty(n * 8 * c * c, dtype=np.complex128)
        G3 = np.empty(n * 8 * c * c, dtype=np.complex128)
        check(lib().amg_get_coarse_links(self._h, level, _cptr(G1), _cptr(G2), _cptr(G3)), "amg_get_coarse_links")
        return G1, G2, G3

    # ---- level operations
    def level_apply(self, level: int, v) -> np.ndarray:
        v = _c128(v, self._vshape(level))
        out = np.empty_like(v)
        check(lib().amg_level_apply(self._h, level, _cptr(v), _cptr(out)), "amg_level_apply")
        return out

    def restrict(self, level: int, v) -> np.ndarray:
        v = _c128(v, self._vshape(level))
        out = np.empty(self._vshape(level + 1), dtype=np.complex128)
        check(lib().amg_restrict(self._h, level, _cptr(v), _cptr(out)), "amg_restrict")
        return out

    def prolong(self, level: int, vc) -> np.ndarray:
        vc = _c128(vc, self._vshape(level + 1))
        out = np.empty(self._vshape(level), dtype=np.complex128)
        check(lib().amg_prolong(self._h, level, _cptr(vc), _cptr(out)), "amg_prolong")
        return out

    def sap(self, level: int, v, x=None, nu: int = 1):
        """SAP_C::SAP: returns (x, converged)."""
        v = _c128(v, self._vshape(level))
        x = np.zeros_like(v) if x is None else _c128(x, self._vshape(level)).copy()
        st = check(lib().amg_sap(self._h, level, _cptr(v), _cptr(x), int(nu)), "amg_sap")
        return x, st == _lib.AMG_OK

    def level_gmres(self, level: int, b):
        b = _c128(b, self._vshape(level))
        x = np.empty_like(b)
        it = C.c_int(0)
        check(lib().amg_level_gmres(self._h, level, _cptr(b), _cptr(x), C.byref(it)), "amg_level_gmres")
        return x, it.value

    def cycle(self, level: int, eta, psi=None) -> np.ndarray:
        eta = _c128(eta, self._vshape(level))
        psi = np.zeros_like(eta) if psi is None else _c128(psi, self._vshape(level)).copy()
        check(lib().amg_cycle(self._h, level, _cptr(eta), _cptr(psi)), "amg_cycle")
        return psi

    def kcycle_fgmres(self, level: int, b):
        b = _c128(b, self._vshape(level))
        x = np.empty_like(b)
        it = C.c_int(0)
        check(lib().amg_kcycle_fgmres(self._h, level, _cptr(b), _cptr(x), C.byref(it)), "amg_kcycle_fgmres")
        return x, it.value

    # ---- solve
    def solve(self, b):
        """FGMRES_AMG::fgmres(b, x0 = 0, x) for [N][2] or [nrhs][N][2] sources.
        Returns (x, infos) with infos a list of dicts (iterations, converged, rel_residual)."""
        b = _c128(b)
        nrhs = 1 if b.ndim == 2 else b.shape[0]
        x = np.empty_like(b)
        infos = (AmgSolveInfo * nrhs)()
        check(lib().amg_solve(self._h, _cptr(b), _cptr(x), nrhs, infos), "amg_solve")
        return x, [dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                   for i in infos]

    def solve_dev(self, b_ptr: int, x_ptr: int, nrhs: int):
        infos = (AmgSolveInfo * nrhs)()
        check(lib().amg_solve_dev(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), nrhs, infos), "amg_solve_dev")
        return [dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                for i in infos]

    def solve_host_ptr(self, b_ptr: int, x_ptr: int, nrhs: int):
        """amg_solve on raw host pointers (e.g. pinned buffers): copies in, solves, copies out."""
        infos = (AmgSolveInfo * nrhs)()
        check(lib().amg_solve(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), nrhs, infos), "amg_solve")
        return [dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                for i in infos]

    def solve_stream_ptrs(self, b_ptrs, x_ptrs, nrhs: int):
        """amg_solve_stream: batches of nrhs sources at raw host pointers (page-locked for the
        copies to overlap the solves), solved one after another; one info list per batch."""
        nb = len(b_ptrs)
        if nb != len(x_ptrs) or nb < 1:
            raise ValueError("need as many output as input batches, at least one")
        bp = (C.c_void_p * nb)(*b_ptrs)
        xp = (C.c_void_p * nb)(*x_ptrs)
        infos = [(AmgSolveInfo * nrhs)() for _ in range(nb)]
        ip = (C.c_void_p * nb)(*[C.cast(i, C.c_void_p) for i in infos])
        check(lib().amg_solve_stream(self._h, nb, bp, xp, nrhs, ip), "amg_solve_stream")
        return [[dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                 for i in inf] for inf in infos]

    # ---- adjoint
    def solve_adjoint(self, g):
        """lambda = D^{-dagger} g on the same hierarchy; returns (lambda, infos)."""
        g = _c128(g)
        nrhs = 1 if g.ndim == 2 else g.shape[0]
        lam = np.empty_like(g)
        infos = (AmgSolveInfo * nrhs)()
        check(lib().amg_solve_adjoint(self._h, _cptr(g), _cptr(lam), nrhs, infos), "amg_solve_adjoint")
        return lam, [dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                     for i in infos]

    def solve_adjoint_dev(self, g_ptr: int, lam_ptr: int, nrhs: int):
        infos = (AmgSolveInfo * nrhs)()
        check(lib().amg_solve_adjoint_dev(self._h, C.c_void_p(g_ptr), C.c_void_p(lam_ptr), nrhs, infos),
              "amg_solve_adjoint_dev")
        return [dict(iterations=i.iterations, converged=bool(i.converged), rel_residual=i.rel_residual)
                for i in infos]

    def force(self, lam, x) -> np.ndarray:
        """F[n][mu] = -sum_r Re(lam_r^dagger dD/dtheta_mu(n) x_r), float64 [N][2]."""
        lam = _c128(lam)
        x = _c128(x, lam.shape)
        nrhs = 1 if lam.ndim == 2 else lam.shape[0]
        F = np.empty((self.N, 2), dtype=np.float64)
        check(lib().amg_force(self._h, _cptr(lam), _cptr(x), nrhs, _cptr(F)), "amg_force")
        return F

    def force_dev(self, lam_ptr: int, x_ptr: int, nrhs: int, F_ptr: int) -> None:
        check(lib().amg_force_dev(self._h, C.c_void_p(lam_ptr), C.c_void_p(x_ptr), nrhs, C.c_void_p(F_ptr)),
              "amg_force_dev")

    def autotune_info(self) -> dict:
        """The autotuner's choice (amg_autotune_info_n)."""
        o = np.zeros(5, dtype=np.int32)
        check(lib().amg_autotune_info_n(self._h, _cptr(o), 5), "amg_autotune_info_n")
        names = {-1: "default", 0: "generic", 1: "lean", 2: "paired_f32", 3: "ca_f32", 4: "cgs_f32", 5: "half_basis",
                 6: "bf16_basis", 7: "paired_f32_spt2"}
        return dict(tuned=bool(o[0]), sap_kernel=names.get(int(o[1]), str(o[1])), engine_cluster=int(o[2]),
                    engine_sap_teams=int(o[4]), tuned_cycle_us=int(o[3]))

    def residual_history(self) -> np.ndarray:
        n = C.c_int(0)
        check(lib().amg_residual_history(self._h, None, 0, C.byref(n)), "amg_residual_history")
        out = np.zeros(max(n.value, 1), dtype=np.float64)
        check(lib().amg_residual_history(self._h, _cptr(out), n.value, C.byref(n)), "amg_residual_history")
        return out[: n.value]

    def stream(self) -> int:
        """The cudaStream_t (as an integer) all calls on this context run on."""
        return lib().amg_get_stream(self._h) or 0

    def profile(self, enable: bool = True) -> None:
        check(lib().amg_profile(self._h, int(enable)), "amg_profile")

    def profile_report(self) -> dict:
        out = {}
        for name, slot in _lib.PROF_SLOTS.items():
            ms, n, b = C.c_double(0), C.c_longlong(0), C.c_double(0)
            check(lib().amg_profile_query(self._h, slot, C.byref(ms), C.byref(n), C.byref(b)), "amg_profile_query")
            out[name] = dict(ms=ms.value, launches=n.value, bytes=b.value)
        return out

    def engine_counters(self) -> dict:
        """Coarse-level operation counts since the previous call, per level."""
        o = np.zeros(6 * 6, dtype=np.int64)
        check(lib().amg_engine_counters(self._h, _cptr(o), o.size), "amg_engine_counters")
        names = ("apply", "local_apply", "kfgmres_steps", "gmres_steps", "sap_steps", "sap_calls")
        return {l: dict(zip(names, map(int, o[6 * l: 6 * l + 6]))) for l in range(1, self.levels)}

    def setup_timings(self) -> dict:
        """The last set-up's device milliseconds by phase (amg_setup_timings)."""
        o = np.zeros(_lib.AMG_SETUP_PHASES, dtype=np.float64)
        check(lib().amg_setup_timings(self._h, _cptr(o), o.size), "amg_setup_timings")
        return dict(zip(("initial_vectors", "smoothing", "orthonormalisation", "coarse_links", "bootstrap",
                         "mixed_copies"), map(float, o)))

    def timings(self):
        s, v = C.c_double(0), C.c_double(0)
        check(lib().amg_last_timings(self._h, C.byref(s), C.byref(v)), "amg_last_timings")
        return s.value, v.value
