// Launchers of the CUDA kernels (host side).  All take a stream; none synchronises.
#pragma once
#include "common.cuh"
#include "engine.cuh"

namespace amgb {

void set_last_error(const char* msg, const char* file, int line);

// number of kernels this library has launched (all contexts); read by amg_launch_count
extern long long g_launches;
inline void count_launch(int n = 1) { __atomic_add_fetch(&g_launches, (long long)n, __ATOMIC_RELAXED); }

// ---- fine lattice (fine.cu) ----
template <typename T>
void launch_dirac(const cx<T>* U, const cx<T>* in, cx<T>* out, int nx, int nt, int nrhs, T m0, int dagger,
                  cudaStream_t s);
// out = D in (FP64) for FP32 spinors in (promoted exactly), and in_copy = in (FP32)
void launch_dirac_promote(const double2* U, const float2* in, double2* out, float2* in_copy, int nx, int nt,
                          int nrhs, double m0, cudaStream_t s);
// reads and clears the fine kernels' device error flag (bit 0: a bulk-copy wait of the D
// apply gave up); synchronises the stream; -1 on a CUDA error
int fine_error_check(cudaStream_t s);
// runs the bulk-copy D apply with waits that cannot complete and returns the device flag
int dirac_tma_wait_test(const double2* U, const double2* in, double2* out, int nx, int nt, int nrhs, cudaStream_t s);
template <typename T>
void launch_residual(const Links<T> U, const cx<T>* b, long long bstride, const cx<T>* x, cx<T>* r, int nx, int nt,
                     int nrhs, T m0, double* partial, double* norm2_out, const int* act, cudaStream_t s);
template <typename T>
void launch_norm2(const cx<T>* v, long long len, long long stride, int nrhs, double* partial, double* out,
                  cudaStream_t s);
int residual_partials(int nx, int nt);
template <typename T, typename TW>
cudaError_t launch_restrict0(const TW* W, const cx<T>* v, cx<T>* out, cx<T>* partial, int nx, int nt, int bx,
                             int bt, int ntest, int nrhs, int nchunk, cudaStream_t s);
int smem_optin_bytes();
// psi += P vc at level 0, or psi = P vc with add = false (psi is then written, never read)
template <typename T, typename TW>
void launch_prolong0_add(const TW* W, const cx<T>* vc, cx<T>* psi, int nx, int nt, int bx, int bt, int ntest,
                         int nrhs, cudaStream_t s, bool add = true);
template <typename T>
int sap0_smem_bytes(int S, int m, int use_smem);
int sap0_warp_enabled();
void set_sap0_warp(int on);
// fine-level SAP block solvers: generic (any block), lean (MGS, one CTA per block), paired
// (FP32 MGS with two-wide arithmetic, four sites per thread; paired2: two, twice the
// threads), ca (FP32 communication-avoiding GMRES), cgs (the paired kernel with classical
// Gram-Schmidt and re-orthogonalisation on demand), half / bf16b (16-bit Krylov basis)
enum { SAP_VARIANT_GENERIC = 0, SAP_VARIANT_LEAN = 1, SAP_VARIANT_PAIRED = 2, SAP_VARIANT_CA = 3, SAP_VARIANT_CGS = 4,
       SAP_VARIANT_HALF = 5, SAP_VARIANT_BF16B = 6, SAP_VARIANT_PAIRED2 = 7 };
template <typename T>
// vfuse (optional): the SAP right-hand side v; r = v - D x is then formed for the colour's
// blocks inside the launch (in a separate residual launch where the chosen kernel cannot)
// and r is written there, instead of r being read as given
cudaError_t launch_sap0(const Links<T> U, cx<T>* r, cx<T>* x, const int* blocks, int ncol, int nrhs, int nx,
                        int nt, int sbt, int sxe, int ste, T m0, int m, int restarts, T tol, int use_smem,
                        cx<T>* gscratch, int* iters, const int* act, cudaStream_t s, int variant = -1,
                        const cx<T>* vfuse = nullptr, long long vstride = 0);
// One lattice's share of a grouped launch of the 16-bit-basis SAP kernel: its FP16 links, SAP
// residual r, iterate x, the colour's block list and its per-source active flags.
struct SapTask {
    const void* U;
    float2* r;
    float2* x;
    const int* blocks;
    const int* act;
    int ncol, nrhs, nx, nt, sbt, sxe, ste, restarts;
    float m0, tol;
};
// The block solves of one colour on several lattices with blocks of S = 256, 512 or 1024
// sites in one launch: column c of the grid solves block col_seg[c] of task col_task[c]
// (tasks and both column tables in device memory), row y its source y.
cudaError_t launch_sap0_h_group(const SapTask* tasks, const int* col_task, const int* col_seg, int ncols,
                                int max_rhs, int S, bool bf, cudaStream_t s);
void launch_multidot(const double2* w, const double2* V, long long len, long long vstride, int nv, int nrhs,
                     double2* partial, int nparts, double2* out, const int* act, cudaStream_t s);
void launch_axpy_multidot(double2* w, const double2* V, long long len, long long vstride, int nv, const double2* h,
                          int hstride, int nd, const int* act, int nrhs, double2* partial, int nparts, double2* out,
                          cudaStream_t s);
void launch_multiaxpy(double2* w, const double2* V, long long len, long long vstride, int nv, const double2* h,
                      int hstride, const int* act, int nrhs, cudaStream_t s);
// x += sum_k c_k Z_k with Z in FP64 (double2) or FP32 (float2, promoted exactly)
template <typename TZ>
void launch_multiaxpy_add(double2* x, const TZ* Z, long long len, long long vstride, int nv, const double2* c,
                          int cstride, const int* nvr, const int* act, int nrhs, cudaStream_t s);
// y = (w - sum_{k<nv} h[k] V_k) * sc for the sources with act (w unchanged; partial receives
// unused |w|^2 partials)
void launch_axpy_scale_to(double2* y, const double2* w, const double2* V, long long len, long long vstride, int nv,
                          const double2* h, int hstride, const double* sc, const int* act, int nrhs, double2* partial,
                          int nparts, cudaStream_t s, float2* yf = nullptr);
// y = sc[rhs] x for the sources with act; yf (optional) receives the FP32 copy of y
void launch_scale(double2* y, const double2* x, long long len, const double* sc, const int* act, int nrhs,
                  cudaStream_t s, float2* yf = nullptr);
void launch_d2f(float2* y, const double2* x, long long n, cudaStream_t s);
void launch_d2h(__half2* y, const double2* x, long long n, cudaStream_t s);
void launch_f2d(double2* y, const float2* x, long long n, cudaStream_t s);
void launch_d2bf(__nv_bfloat162* y, const double2* x, long long n, cudaStream_t s);

void launch_gamma5(double2* y, const double2* x, long long nsites, cudaStream_t s);
void launch_force(const double2* U, const double2* lam, const double2* x, double2* F, int nx, int nt, int nrhs,
                  cudaStream_t s);

// ---- coarse engine (coarse.cu) ----
enum EngOp {
    ENG_KFGMRES = 0,   // FGMRES_k_cycle of level l: x = fgmres(b, x0 = b)
    ENG_KCYCLE = 1,    // k_cycle(l, b, x) accumulating into x
    ENG_VCYCLE = 2,    // v_cycle(l, b, x) accumulating into x
    ENG_SAP = 3,       // SAP(l, b, x, nu) with x in/out
    ENG_APPLY = 4,     // x = D_l b
    ENG_GMRES = 5,     // coarsest-style GMRES on level l: x = gmres(b, x0 = b)
    ENG_RESTRICT = 6,  // x (level l+1) = P_l^dagger b
    ENG_PROLONG = 7,   // x (level l) = P_l b (level l+1)
};
template <typename T>
cudaError_t launch_engine_dev(const EngArgs<T>* dev_args, int op, int level, int nu, const cx<T>* in,
                              long long in_stride, cx<T>* out, long long out_stride, int nsrc, int smem_bytes,
                              int csize, cudaStream_t s);
template <typename T>
int engine_max_clusters(int csize, int smem_bytes);

// ---- set-up (setup.cu) ----
template <typename T>
void launch_fine_hops(const cx<T>* U, cx<T>* hops, int nx, int nt, cudaStream_t s);
template <typename T>
void launch_coarse_links(const cx<T>* W, const cx<T>* hops, cx<T>* out, int nx, int nt, int K, int bx, int bt,
                         int ntest, cx<T>* partial, int nchunk, cudaStream_t s);
template <typename T>
void launch_orthonormalize(cx<T>* W, int nx, int nt, int K, int bx, int bt, int ntest, cudaStream_t s);

}  // namespace amgb
