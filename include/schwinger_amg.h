/*
 * schwinger_amg.h -- C ABI of the B200 DD-alpha-AMG solver for the 2-D Schwinger-model
 * Wilson-Dirac operator (libschwinger_amg.so).
 *
 * Every entry point returns an int status: AMG_OK (0), AMG_NOT_CONVERGED (1) when an
 * iteration limit was reached, or a negative AMG_ERR_* code; amg_last_error() gives the
 * message.  No entry point exits the process or traps on the device (the reference calls
 * exit(1) on bad input, include/params.h:21-24, src/gauge_conf.cpp:20-23).
 *
 * Layouts at this boundary are the reference's, as contiguous interleaved complex128
 * arrays:
 *   fine spinor / source      psi[N][2]           n = x*Nt + t (src/variables.cpp:10-16)
 *   gauge field               U[N][2]             U[n][mu], mu = 0 time, mu = 1 space
 *   level-l vector            v[N_l][DOF_l]       dof = 2*c + spin (src/level.cpp:166)
 *   test vectors of level l   W[Ntest_l][N_l][DOF_l]   (interpolator_columns, include/level.h:144)
 *   coarse links of level l   G1[N_l][2][2][c][c], G2/G3[N_l][2][2][c][c][2]
 *                             (include/level.h:126-128, 162-164, 169-185)
 * Arrays with a trailing "nrhs" dimension are [nrhs][...] (one full vector per source).
 * Pointers are host pointers unless the function name ends in _dev (device pointers).
 */
#ifndef SCHWINGER_AMG_H
#define SCHWINGER_AMG_H

#if defined(__GNUC__)
#define AMG_API __attribute__((visibility("default")))
#else
#define AMG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define AMG_OK 0
#define AMG_NOT_CONVERGED 1
#define AMG_ERR_INVALID (-1)     /* bad argument or parameter */
#define AMG_ERR_CUDA (-2)        /* CUDA runtime error */
#define AMG_ERR_STATE (-3)       /* call order (e.g. solve before set-up) */
#define AMG_ERR_NOMEM (-4)       /* device allocation failed */
#define AMG_ERR_DEVICE_WAIT (-5) /* a bounded device-side wait gave up */
#define AMG_ERR_UNSUPPORTED (-6) /* configuration outside what the kernels support */

#define AMG_PREC_F64 0           /* everything FP64: the plain drop-in */
#define AMG_PREC_MIXED 1         /* FP32 cycle (SAP, P, P^dagger, coarse levels) with BF16
                                    test vectors inside the FP64 outer FGMRES */

#define AMG_LINKS_F32 0          /* amg_params.link_storage: fine links of the mixed cycle */
#define AMG_LINKS_BF16 1
#define AMG_LINKS_F16 2

#define AMG_CYCLE_V 0            /* AMGV::cycle = 0 (include/variables.h:64) */
#define AMG_CYCLE_K 1

/* preconditioner of the outer FGMRES (amg_set_preconditioner) */
#define AMG_PRECOND_MG 0         /* FGMRES_AMG: the K- or V-cycle (include/amg.h:99-145) */
#define AMG_PRECOND_SAP 1        /* FGMRES_SAP: one fine-level SAP sweep (include/sap.h:194-225) */
#define AMG_PRECOND_NONE 2       /* FGMRES_fine_level: no preconditioner (include/fgmres.h:126-148) */

typedef struct amg_context* amg_ctx;

/* Solver knobs.  Defaults (amg_params_default) are the reference's:
 * src/variables.cpp:46-87 and include/params.h:63-65, with the values its main sets
 * (K-cycle, Nit = 0, 4 SAP iterations on the test vectors; src/main.cpp:61-65, :129). */
typedef struct amg_params {
    int cycle;                 /* AMGV::cycle */
    int nu1, nu2;              /* AMGV::nu1 / nu2: pre/post SAP iterations */
    int nit;                   /* AMGV::Nit: bootstrap passes of the set-up */
    int sap_tv_iters;          /* AMGV::SAP_test_vectors_iterations */
    int sap_gmres_m;           /* SAPV::sap_gmres_restart_length */
    int sap_gmres_restarts;    /* SAPV::sap_gmres_restarts */
    double sap_gmres_tol;      /* SAPV::sap_gmres_tolerance */
    double sap_tol;            /* SAPV::sap_tolerance */
    int kcycle_m;              /* AMGV::fgmres_k_cycle_restart_length */
    int kcycle_restarts;       /* AMGV::fgmres_k_cycle_restarts */
    double kcycle_tol;         /* AMGV::fgmres_k_cycle_tol */
    int coarse_m;              /* LevelV::GMRES_restart_len[maxLevel] */
    int coarse_restarts;       /* LevelV::GMRES_restarts[maxLevel] */
    double coarse_tol;         /* LevelV::GMRES_tol[maxLevel] */
    int outer_m;               /* FGMRESV::fgmres_restart_length */
    int outer_restarts;        /* FGMRESV::fgmres_restarts */
    double outer_tol;          /* FGMRESV::fgmres_tolerance */
    int precision;             /* AMG_PREC_F64 or AMG_PREC_MIXED */
    int max_rhs;               /* largest number of sources per solve call (buffers) */
    unsigned long long tv_seed;/* 0: the reference's draw (mt19937(50), src/amg.cpp:8-16) */
    int autotune;              /* 1 (default): the first solve of a context times the fine SAP
                                  kernel variants and the coarse-engine cluster sizes on its own
                                  data and keeps the fastest; 0: fixed defaults */
    int link_storage;          /* mixed form: storage of the fine links its cycle reads,
                                  AMG_LINKS_F16 (default: unit-modulus links in 10 mantissa bits),
                                  AMG_LINKS_BF16 or AMG_LINKS_F32 (FP32 arithmetic either way);
                                  the FP64 operator keeps FP64 links */
} amg_params;

/* Per-source result of a solve. */
typedef struct amg_solve_info {
    int iterations;            /* FGMRES::fgmres return value (src/fgmres.cpp:80, :87) */
    int converged;             /* 1 if the FP64 true residual met the tolerance */
    double rel_residual;       /* ||b - D x|| / ||b|| in FP64 */
} amg_solve_info;

/* ---- errors, version ------------------------------------------------------------- */
AMG_API const char* amg_status_string(int status);
AMG_API const char* amg_last_error(void);
AMG_API int amg_version(void);

/* ---- parameters ------------------------------------------------------------------ */
AMG_API void amg_params_default(amg_params* p);

/* readParameters (include/params.h:17-69): reads "level bx bt ntest sbx sbt" rows from a
 * parameters.dat file into rows[max_rows][6]; *nrows receives the row count. */
AMG_API int amg_read_parameters(const char* path, int* rows, int max_rows, int* nrows);

/* ---- context ---------------------------------------------------------------------- */
/* Replaces AlgebraicMG(GConf, m0, nu1, nu2) (include/amg.h:42-64) plus the lattice size
 * and level count the reference fixes at compile time (include/config.h.in:3-5):
 * nx = NS, nt = NT, levels = LEVELS, rows = the parameters.dat rows [levels-1][6]. */
AMG_API int amg_create(amg_ctx* ctx, int nx, int nt, int levels, const int* rows, double m0,
               const amg_params* params, int device);
AMG_API int amg_destroy(amg_ctx ctx);
AMG_API int amg_get_params(amg_ctx ctx, amg_params* out);
/* mass::m0 (include/variables.h:20-22) */
AMG_API int amg_set_mass(amg_ctx ctx, double m0);
/* Replaces assigning AMGV::cycle (include/variables.h:64) after creation: AMG_CYCLE_K or
 * AMG_CYCLE_V for the amg_cycle, amg_solve and bootstrap calls that follow. */
AMG_API int amg_set_cycle(amg_ctx ctx, int cycle);
/* Chooses the outer FGMRES's preconditioner for the amg_solve* calls that follow:
 * AMG_PRECOND_MG (default, FGMRES_AMG); AMG_PRECOND_SAP, the reference's comparison solver
 * FGMRES_SAP (include/sap.h:194-225, run by Tests::FGMRES_sap, src/tests.cpp:33-46): each
 * preconditioner call zeroes z and applies SAP_C::SAP(v, z, nu = 1) on the fine level, with
 * the fine SAP kernels of the context's precision; or AMG_PRECOND_NONE, GMRES without
 * preconditioning (FGMRES_fine_level, include/fgmres.h:126-148, run by Tests::GMRES,
 * src/tests.cpp:13-22; FP64 whatever the context's precision; amg_params.outer_m /
 * outer_restarts give its restart length and count).  The solve still needs amg_setup (the
 * work buffers live with the hierarchy). */
AMG_API int amg_set_preconditioner(amg_ctx ctx, int kind);
/* Level sizes as LevelV fills them: out[l] = {Nsites, NxSites, NtSites, DOF, Colors, Ntest}. */
AMG_API int amg_level_info(amg_ctx ctx, int level, int* out6);

/* GaugeConf::setGconf / read_conf (include/gauge_conf.h:34, src/gauge_conf.cpp:18-32):
 * U[N][2] complex128.  Invalidates the set-up. */
AMG_API int amg_set_gauge(amg_ctx ctx, const double* U);

/* ---- fine operator ------------------------------------------------------------------ */
/* D_phi / D_dagger_phi (src/dirac_operator.cpp:3-54; include/dirac_operator.h:14-24):
 * out = D in (dagger = 0) or D^dagger in (dagger = 1), for nrhs sources. */
AMG_API int amg_dirac_apply(amg_ctx ctx, const double* in, double* out, int nrhs, int dagger);
AMG_API int amg_dirac_apply_dev(amg_ctx ctx, const void* in, void* out, int nrhs, int dagger);
/* Stand-alone FP64 stencil on caller-owned device memory (no context): U_dev [N][2],
 * in_dev / out_dev [nrhs][N][2] complex128, launched on `stream` (a cudaStream_t). */
AMG_API int amg_dirac_apply_raw(const void* U_dev, const void* in_dev, void* out_dev, int nx, int nt,
                        int nrhs, double m0, int dagger, void* stream);
/* Comparison solvers on the fine stencil (FP64, one source, host arrays; they need the gauge
 * field, not the set-up):
 * amg_cg_normal: conjugate_gradient (src/conjugate_gradient.cpp:5-65, run by Tests::CG,
 *   src/tests.cpp:24-31): x = (D D^dagger)^{-1} phi from x = phi, CG until |r| < tol |phi|
 *   (the reference's CG::tol = 1e-10, CG::max_iter = 100000, src/variables.cpp:84-87);
 *   iterations = the reference's k at convergence.
 * amg_bicgstab: bi_cgstab (src/bi_cgstab.cpp:5-89, run by Tests::BiCG with tol 1e-10): D x =
 *   phi from x0 (NULL: zero); iterations = k + 1 at convergence.
 * Both return AMG_OK when converged, AMG_NOT_CONVERGED after max_iter. */
AMG_API int amg_cg_normal(amg_ctx ctx, const double* phi, double* x, int max_iter, double tol, int* iterations);
AMG_API int amg_bicgstab(amg_ctx ctx, const double* phi, const double* x0, double* x, int max_iter, double tol,
                         int* iterations);
/* Self-test of the bounded device waits (no reference counterpart): runs the bulk-copy D apply
 * on caller-owned device memory (nt a multiple of 256, nx of 4, 16-byte aligned, distinct
 * in/out) without issuing its copies, so its first wait gives up after a short poll limit
 * with nothing in flight.  Returns AMG_ERR_DEVICE_WAIT when the kernel reported that (the
 * expected outcome), AMG_OK if it did not, AMG_ERR_INVALID for a lattice the kernel does not
 * take.  out is left undefined; the device stays usable. */
AMG_API int amg_debug_dirac_wait_test(const void* U_dev, const void* in_dev, void* out_dev, int nx, int nt, int nrhs);
/* Stand-alone FP64 stencil on host arrays, no context: D_phi / D_dagger_phi
 * (src/dirac_operator.cpp:3-54) with the reference's signature data (U[N][2], in/out
 * [nrhs][N][2]); device buffers are allocated and freed inside the call. */
AMG_API int amg_dirac_apply_host(const double* U, const double* in, double* out, int nx, int nt, int nrhs,
                                 double m0, int dagger);
/* Stand-alone FP64 level-0 restriction out = P^dagger v that allocates no device memory, for
 * callers that may not allocate while they run (an application that owns all device memory
 * through its own pool, or code inside a region where an allocation would synchronise or
 * fail).  No counterpart in the reference: it computes what Level::Pt_v does at level 0
 * (src/level.cpp:212-237) and what amg_restrict(ctx, 0, ...) returns.
 *   W_dev   [ntest][N][2] complex128 test vectors (amg_get_test_vectors layout)
 *   v_dev   [nrhs][N][2] complex128, out_dev [nrhs][bx*bt][2*ntest] complex128
 *   bx, bt  aggregate counts along x and t (nx % bx == nt % bt == 0), ntest in [1, 32]
 * Chunk partial sums go to a 4 MiB array owned by the library on every device; calls with
 * nrhs * bx * bt * 2 * ntest * 16 > 4 MiB are rejected with AMG_ERR_INVALID.  The buffers
 * belong to the current device.  The first call on a device looks up that array's address
 * (make that first call before any stream capture).  All calls on a device share the array,
 * so calls that overlap on the GPU (other streams, other host threads) race; serialise them.
 * The looked-up address does not survive cudaDeviceReset: do not call this again on a device
 * after resetting it.  A CUDA error already pending on the calling thread is reported (and
 * left pending) as AMG_ERR_CUDA, with nothing launched.  nx * nt * 2 must fit in an int. */
AMG_API int amg_restrict_raw_noalloc(const void* W_dev, const void* v_dev, void* out_dev, int nx, int nt,
                                     int bx, int bt, int ntest, int nrhs, void* stream);

/* ---- set-up ------------------------------------------------------------------------ */
/* Optional: the test vectors the set-up starts from on level l, W[Ntest_l][N_l][DOF_l]
 * (the columns setUpPhase draws, src/amg.cpp:8-35).  Without it the set-up draws them. */
AMG_API int amg_set_initial_test_vectors(amg_ctx ctx, int level, const double* W);
/* AlgebraicMG::setUpPhase(Nit) (src/amg.cpp:3-88): smooth, orthonormalise, build the
 * coarse links of every level, then params.nit bootstrap passes. */
AMG_API int amg_setup(amg_ctx ctx);
/* Level::interpolator_columns after set-up (include/level.h:144). */
AMG_API int amg_get_test_vectors(amg_ctx ctx, int level, double* W);
/* Level::G1/G2/G3 of level l >= 1 (built by makeCoarseLinks, src/level.cpp:242-301). */
AMG_API int amg_get_coarse_links(amg_ctx ctx, int level, double* G1, double* G2, double* G3);

/* ---- level operators (one source) -------------------------------------------------- */
/* Level::D_operator (src/level.cpp:161-180) of level l. */
AMG_API int amg_level_apply(amg_ctx ctx, int level, const double* in, double* out);
/* Level::Pt_v (src/level.cpp:212-237): level l -> l+1. */
AMG_API int amg_restrict(amg_ctx ctx, int level, const double* in, double* out);
/* Level::P_v (src/level.cpp:182-209): level l+1 -> l. */
AMG_API int amg_prolong(amg_ctx ctx, int level, const double* in, double* out);
/* The mixed form's level-0 Level::Pt_v / Level::P_v (src/level.cpp:182-237) on device buffers
 * of complex64 values, as its cycles run them (BF16 test vectors, FP32 sources; the tensor-core
 * kernels where the lattice allows, AMG_TC_TRANSFER=0 for the CUDA-core ones):
 *   restriction:  out[nrhs][bx*bt][2*Ntest] = P^dagger in[nrhs][N][2]
 *   prolongation: out[nrhs][N][2] += P in[nrhs][bx*bt][2*Ntest]
 * The context must be in the mixed form with its set-up done; synchronises its stream. */
AMG_API int amg_restrict0_mixed_dev(amg_ctx ctx, const void* in_dev, void* out_dev, int nrhs);
AMG_API int amg_prolong0_mixed_dev(amg_ctx ctx, const void* in_dev, void* out_dev, int nrhs);
/* SAP_C::SAP (src/sap.cpp:64-174) on level l: nu iterations on D x = v, x in/out.
 * Returns AMG_OK if the SAP tolerance was met, AMG_NOT_CONVERGED otherwise (the
 * reference returns 1 / 0). */
AMG_API int amg_sap(amg_ctx ctx, int level, const double* v, double* x, int nu);
/* Level::GMRES_level_l::fgmres(b, b, x) on level l >= 1 with the coarsest-level knobs
 * (include/level.h:66-85); *iterations receives the FGMRES count. */
AMG_API int amg_level_gmres(amg_ctx ctx, int level, const double* b, double* x, int* iterations);
/* One cycle from level l: AlgebraicMG::k_cycle / v_cycle(l, eta, psi) (src/amg.cpp:90-178),
 * psi in/out (the caller zeroes it for a fresh cycle). */
AMG_API int amg_cycle(amg_ctx ctx, int level, const double* eta, double* psi);
/* FGMRES_k_cycle of level l >= 1 (include/amg.h:19-40): fgmres(b, x0 = b, x). */
AMG_API int amg_kcycle_fgmres(amg_ctx ctx, int level, const double* b, double* x, int* iterations);

/* ---- solve --------------------------------------------------------------------------- */
/* FGMRES_AMG::fgmres(b, x0 = 0, x) (include/amg.h:99-145, src/fgmres.cpp:5-88) for nrhs
 * sources at once: b, x [nrhs][N][2] host arrays; info[nrhs] optional. */
AMG_API int amg_solve(amg_ctx ctx, const double* b, double* x, int nrhs, amg_solve_info* info);
/* Same on device arrays (no host copies). */
AMG_API int amg_solve_dev(amg_ctx ctx, const void* b_dev, void* x_dev, int nrhs, amg_solve_info* info);
/* nbatch batches of nrhs sources from host memory, solved one after another (each as
 * amg_solve): b[i], x[i] are [nrhs][N][2] host arrays, info[i] (optional) [nrhs].  The copies
 * run on a second stream through two device slots, so batch i+1's sources go in and batch
 * i-1's solutions come out while batch i is solved; with page-locked host arrays only the
 * first batch's input and the last batch's output copies are not hidden.  Replaces calling
 * FGMRES_AMG::fgmres once per right-hand side (src/tests.cpp:67-82).  Returns
 * AMG_NOT_CONVERGED if any source of any batch did not converge. */
AMG_API int amg_solve_stream(amg_ctx ctx, int nbatch, const double* const* b, double* const* x, int nrhs,
                             amg_solve_info* const* info);
/* Solves on several contexts at once (uneven lattice sizes, different gauge fields): the
 * outer FGMRES of every context advances in turn, each on its context's stream, so one
 * context's kernels run while the host does another's Givens rotations.  Context i solves
 * nrhs[i] sources b[i] -> x[i] ([nrhs][N_i][2] complex128; device pointers for _dev);
 * info[i] (optional, or info == NULL) receives nrhs[i] results.  Every context appears at
 * most once.  Same results as amg_solve on each context alone.  No reference counterpart:
 * the reference solves one configuration per run (src/main.cpp:130). */
AMG_API int amg_solve_many(int count, const amg_ctx* ctx, const double* const* b, double* const* x, const int* nrhs,
                           amg_solve_info* const* info);
AMG_API int amg_solve_many_dev(int count, const amg_ctx* ctx, const void* const* b_dev, void* const* x_dev,
                               const int* nrhs, amg_solve_info* const* info);
/* Residual history of source 0 of the last solve: |g_{j+1}| per Arnoldi step
 * (the reference's Residuals_FGMRES_*.res, src/fgmres.cpp:45, :70-79). */
AMG_API int amg_residual_history(amg_ctx ctx, double* out, int max_len, int* len);

/* ---- adjoint (no reference counterpart beyond D_dagger_phi) ------------------------- */
/* lambda = D^{-dagger} g through the same hierarchy: lambda = gamma5 D^{-1} gamma5 g
 * (D_dagger_phi = gamma5 D_phi gamma5, src/dirac_operator.cpp:3-54).  info[i].rel_residual
 * is ||g - D^dagger lambda|| / ||g||. */
AMG_API int amg_solve_adjoint(amg_ctx ctx, const double* g, double* lambda, int nrhs, amg_solve_info* info);
AMG_API int amg_solve_adjoint_dev(amg_ctx ctx, const void* g_dev, void* lambda_dev, int nrhs, amg_solve_info* info);
/* Fermion force: F[n][mu] = -sum_r Re(lambda_r^dagger dD/dtheta_mu(n) x_r) for U = exp(i theta),
 * F[N][2] float64.  With x = D^{-1} b and lambda = D^{-dagger} eta this is dL/dtheta of
 * L = Re(eta^dagger D^{-1} b); twice it with x = (D^dagger D)^{-1} phi and lambda = D x is the
 * derivative of phi^dagger (D^dagger D)^{-1} phi. */
AMG_API int amg_force(amg_ctx ctx, const double* lambda, const double* x, int nrhs, double* F);
AMG_API int amg_force_dev(amg_ctx ctx, const void* lambda_dev, const void* x_dev, int nrhs, void* F_dev);

/* ---- timing and profiling ---------------------------------------------------------- */
/* Kernel classes timed by amg_profile (CUDA events on the context's stream around each
 * launch): the fine SAP block solves, the coarse-level engine, fine restriction and
 * prolongation, the fine stencil / residual inside the cycle, the outer FGMRES
 * orthogonalisation, and the outer step's operator w = D z_j. */
#define AMG_PROF_SAP 0
#define AMG_PROF_ENGINE 1
#define AMG_PROF_RESTRICT 2
#define AMG_PROF_PROLONG 3
#define AMG_PROF_FINE_OP 4
#define AMG_PROF_BLAS 5
#define AMG_PROF_OUTER_OP 6
#define AMG_PROF_SLOTS 7
/* Enables (1) or disables (0) per-class timing and clears the accumulated values. */
AMG_API int amg_profile(amg_ctx ctx, int enable);
/* Accumulated device milliseconds, launch count and algorithmic bytes of one class. */
AMG_API int amg_profile_query(amg_ctx ctx, int slot, double* ms, long long* launches, double* bytes);
/* Coarse-level operation counts since the last call (then reset), out[level*6 + k] for
 * k = operator applies, block-local applies, K-cycle FGMRES steps, level GMRES steps, SAP
 * block GMRES steps, SAP calls (a tracing aid; the reference keeps no such counts). */
AMG_API int amg_engine_counters(amg_ctx ctx, long long* out, int len);
/* Number of CUDA kernels the library has launched so far (all contexts). */
AMG_API long long amg_launch_count(void);
/* The cudaStream_t every call on this context runs on (for callers that time or order work). */
AMG_API void* amg_get_stream(amg_ctx ctx);
/* Device milliseconds of the last amg_setup / solve call (CUDA events). */
AMG_API int amg_last_timings(amg_ctx ctx, double* setup_ms, double* solve_ms);
/* The last amg_setup by phase (device milliseconds between CUDA events at the phase
 * boundaries): the initial test vectors and the fine operator's hop table, the test-vector
 * smoothing (SAP), the orthonormalisation, the coarse links (all levels), the bootstrap
 * passes, and the mixed form's FP32/BF16/FP16 copies with its engine.  ms[i] for
 * i < min(n, AMG_SETUP_PHASES). */
#define AMG_SETUP_INIT 0
#define AMG_SETUP_SMOOTH 1
#define AMG_SETUP_ORTHO 2
#define AMG_SETUP_LINKS 3
#define AMG_SETUP_BOOT 4
#define AMG_SETUP_MIXED 5
#define AMG_SETUP_PHASES 6
AMG_API int amg_setup_timings(amg_ctx ctx, double* ms, int n);
/* The autotuner's choice: out[0] = 1 once tuned, out[1] = fine SAP kernel (0 generic,
 * 1 lean, 2 paired FP32, 3 communication-avoiding FP32, 4 classical Gram-Schmidt FP32,
 * 5 FP16 basis, 6 BF16 basis, 7 paired FP32 with two sites per thread; -1 default),
 * out[2] = engine cluster size (0 default), out[3] = the tuned preconditioner time in
 * microseconds. */
AMG_API int amg_autotune_info(amg_ctx ctx, int* out4);
/* The same plus out[4] = the coarse SAP teams per engine CTA (1, 2 or 4); writes the first
 * min(n, 5) values. */
AMG_API int amg_autotune_info_n(amg_ctx ctx, int* out, int n);

#ifdef __cplusplus
}
#endif
#endif
