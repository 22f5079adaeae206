// Host side of libschwinger_amg.so: the solver context, the set-up phase, the fine-level
// cycle, the outer FGMRES and the C ABI declared in include/schwinger_amg.h.
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <condition_variable>
#include <map>
#include <mutex>
#include <thread>
#include <memory>
#include <tuple>
#include <random>
#include <string>
#include <vector>

#include "kernels.h"
#include "../../include/schwinger_amg.h"

namespace amgb {

long long g_launches = 0;
static thread_local std::string g_last_error;
void set_last_error(const char* msg, const char* file, int line) {
    g_last_error = std::string(msg) + " (" + file + ":" + std::to_string(line) + ")";
}
static int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CK(expr)                                                                   \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            set_last_error(cudaGetErrorString(_e), __FILE__, __LINE__);            \
            return _e == cudaErrorMemoryAllocation ? AMG_ERR_NOMEM : AMG_ERR_CUDA; \
        }                                                                          \
    } while (0)
#define CKR(expr)              \
    do {                       \
        int _r = (expr);       \
        if (_r < 0) return _r; \
    } while (0)
#define CKL()  CK(cudaGetLastError())

// ---------------------------------------------------------------------------------
// level geometry (readParameters, include/params.h:17-69; Level, include/level.h:147-157;
// SAP_C::SchwarzBlocks, src/sap.cpp:3-39)
// ---------------------------------------------------------------------------------
struct LevelHost {
    int nx, nt, n, colors, K;
    int coarsest;
    int bx = 1, bt = 1, xe = 1, te = 1, ntest = 1;
    int sbx = 1, sbt = 1, sxe = 1, ste = 1, ncol = 1;
    std::vector<int> red, black;
};

static int build_levels(int nx, int nt, int L, const int* rows, std::vector<LevelHost>& lv) {
    if (L < 2 || L > kMaxLevels) return fail(AMG_ERR_INVALID, "levels must be in [2, %d], got %d", kMaxLevels, L);
    if (nx < 2 || nt < 2) return fail(AMG_ERR_INVALID, "lattice %dx%d too small", nx, nt);
    if (!rows) return fail(AMG_ERR_INVALID, "no parameter rows");
    std::vector<std::array<int, 6>> r(L - 1);
    std::vector<int> seen(L - 1, 0);
    for (int i = 0; i < L - 1; i++) {
        int l = rows[6 * i];
        if (l < 0 || l >= L - 1) return fail(AMG_ERR_INVALID, "parameter row %d names level %d", i, l);
        for (int k = 0; k < 6; k++) r[l][k] = rows[6 * i + k];
        seen[l]++;
    }
    for (int l = 0; l < L - 1; l++)
        if (seen[l] != 1) return fail(AMG_ERR_INVALID, "level %d needs exactly one parameter row", l);
    lv.assign(L, LevelHost{});
    for (int l = 0; l < L; l++) {
        LevelHost& h = lv[l];
        h.nx = l == 0 ? nx : r[l - 1][1];
        h.nt = l == 0 ? nt : r[l - 1][2];
        h.colors = l == 0 ? 1 : r[l - 1][3];
        h.K = 2 * h.colors;
        h.n = h.nx * h.nt;
        h.coarsest = (l == L - 1);
        if (h.coarsest) continue;
        h.bx = r[l][1]; h.bt = r[l][2]; h.ntest = r[l][3]; h.sbx = r[l][4]; h.sbt = r[l][5];
        if (h.bx <= 0 || h.bt <= 0 || h.ntest <= 0 || h.sbx <= 0 || h.sbt <= 0)
            return fail(AMG_ERR_INVALID, "level %d: non-positive blocking", l);
        if (h.nx % h.bx || h.nt % h.bt)
            return fail(AMG_ERR_INVALID, "level %d: %dx%d lattice not divisible into %dx%d blocks", l, h.nx, h.nt, h.bx, h.bt);
        if (h.nx % h.sbx || h.nt % h.sbt)
            return fail(AMG_ERR_INVALID, "level %d: %dx%d lattice not divisible into %dx%d SAP blocks", l, h.nx, h.nt,
                        h.sbx, h.sbt);
        if (h.ntest > 32) return fail(AMG_ERR_UNSUPPORTED, "level %d: at most 32 test vectors", l);
        h.xe = h.nx / h.bx; h.te = h.nt / h.bt;
        h.sxe = h.nx / h.sbx; h.ste = h.nt / h.sbt;
        const int nb = h.sbx * h.sbt;
        if (nb != 1 && nb % 2)
            return fail(AMG_ERR_UNSUPPORTED,
                        "level %d: an odd number of SAP blocks (%d) leaves one block unsolved in the reference "
                        "(include/sap.h:68)", l, nb);
        h.ncol = nb == 1 ? 1 : nb / 2;
        h.red.assign(h.ncol, 0);
        h.black.assign(h.ncol, 0);
        for (int X = 0; X < h.sbx; X++)
            for (int T = 0; T < h.sbt; T++) {
                const int b = X * h.sbt + T;
                bool is_red;
                if (h.sbt % 2 == 0) is_red = (X % 2 == 0) ? (b % 2 == 0) : (b % 2 == 1);
                else is_red = (b % 2 == 0);
                if (b / 2 < h.ncol) (is_red ? h.red : h.black)[b / 2] = b;
            }
    }
    return AMG_OK;
}

// ---------------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t b) {
        if (p && bytes >= b) return AMG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(AMG_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
        }
        bytes = b;
        return AMG_OK;
    }
    template <typename X> X* as() const { return reinterpret_cast<X*>(p); }
};

// page-locked host memory, so device-to-host copies of the outer FGMRES stay asynchronous
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
    int alloc(size_t b) {
        if (p && bytes >= b) return AMG_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMallocHost(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(AMG_ERR_NOMEM, "cudaMallocHost(%zu) failed: %s", b, cudaGetErrorString(e));
        }
        bytes = b;
        return AMG_OK;
    }
};

// per-precision state of the fine-level cycle and the engine
template <typename T>
struct PrecSet {
    DevBuf U;                      // [N][2]
    DevBuf W0;                     // level-0 test vectors [ntest][N][2] (BF16 in the mixed form)
    int w0_bf16 = 0;
    std::vector<DevBuf> W;         // levels >= 1: [ntest][n][K]
    std::vector<DevBuf> links;     // levels >= 1: [n][5][K][K]
    DevBuf eng_args, eng_work, eng_status, red_black;
    EngArgs<T> eh{};
    int eng_smem = 0, eng_cap = 0;
    int max_cluster = 1;             // largest engine cluster the slabs are sized for
    int cluster_cache[17] = {0};     // engine_max_clusters(c) + 1, 0 = not queried
    int cluster_pick = 0;            // the autotuner's cluster size (0: largest single-wave size)
    int sap_teams = 0;               // the autotuner's coarse SAP teams per engine CTA (0: default)
    DevBuf r0, eta1, psi1, rpart, sap_r, sap_scratch;
    int ready = 0;
};

}  // namespace amgb

using namespace amgb;

struct amg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    amg_params p{};
    double m0 = 0;
    int nx = 0, nt = 0, N = 0, L = 0;
    std::vector<LevelHost> lv;
    PrecSet<double> d;             // FP64 hierarchy (master)
    PrecSet<float> f;              // FP32 / BF16 copy for the mixed form
    DevBuf hops0, linkpart, zero, boot_a, boot_b, adj;
    std::vector<int> have_init;
    int gauge_set = 0, setup_done = 0;
    // outer FGMRES
    DevBuf V, Z, w, x, b, partial, dots, scal, masks, etab, vf, zf, vd, zd, sap_flags, norms;
    PinnedBuf hpin;                // host staging of the outer FGMRES (dots, norms, masks)
    char* hpin_dev = nullptr;      // hpin's device mapping (null: copy through the copy engines)
    cudaEvent_t ev_host = nullptr; // marks the end of each queued piece of the outer FGMRES
    int Rcap = 0;
    std::vector<double> history;
    double last_setup_ms = 0, last_solve_ms = 0;
    double setup_phase_ms[AMG_SETUP_PHASES] = {0};   // the last set-up by phase (amg_setup_timings)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // per-kernel-class timing with CUDA events on the context's stream (amg_profile)
    struct ProfSlot { double ms = 0; long long n = 0; double bytes = 0; };
    int prof_on = 0;
    ProfSlot prof[AMG_PROF_SLOTS];
    struct Pending { int slot; cudaEvent_t a, b; double bytes; };
    std::vector<Pending> prof_pending;
    std::vector<cudaEvent_t> ev_pool;
    // the preconditioner (one K- or V-cycle from the fine level) as CUDA graphs, one per
    // (precision path, sources, input, output); built on a key's second use, replayed after
    struct GraphEntry { int uses = 0; cudaGraphExec_t exec = nullptr; long long launches = 0; };
    std::map<std::tuple<int, int, const void*, void*>, GraphEntry> graphs;
    int graphs_off = 0;            // capture failed once: run eagerly from then on
    // autotuner state: the fine SAP kernel variant (-1: default) and whether it ran
    int sap_variant = -1, tuned = 0;
    int precond = AMG_PRECOND_MG;   // amg_set_preconditioner
    // the FP64 vector whose FP32 copy the mixed preconditioner's input buffer vf holds (the
    // outer FGMRES writes that copy while it normalises the basis vector), or null
    const void* vf_src = nullptr;
    double tuned_us = 0;
    // amg_solve_stream: the copy stream and the second device slot of b and x (the first is
    // b, x), created on first use; per slot: inputs copied, solve done, outputs copied
    cudaStream_t copy_stream = nullptr;
    DevBuf b1, x1;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_solved[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
    cudaEvent_t ev_piece[2] = {nullptr, nullptr};   // the batch copies' pieces in flight
    void drop_graphs() {
        for (auto& kv : graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
    }
    ~amg_context() {
        drop_graphs();
        for (auto& p : prof_pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        for (auto e : ev_pool) cudaEventDestroy(e);
    }
};

namespace {

using cd = std::complex<double>;

cudaEvent_t prof_event(amg_context* c) {
    if (!c->ev_pool.empty()) { cudaEvent_t e = c->ev_pool.back(); c->ev_pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
// Records an event pair around the launches of one kernel class when profiling is on.
struct ProfScope {
    amg_context* c;
    int slot;
    double bytes;
    cudaEvent_t a = nullptr;
    ProfScope(amg_context* c_, int slot_, double bytes_) : c(c_), slot(slot_), bytes(bytes_) {
        if (c->prof_on) { a = prof_event(c); cudaEventRecord(a, c->stream); }
    }
    ~ProfScope() {
        if (!a) return;
        cudaEvent_t b = prof_event(c);
        cudaEventRecord(b, c->stream);
        c->prof_pending.push_back({slot, a, b, bytes});
    }
};
void prof_harvest(amg_context* c) {
    if (c->prof_pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto& p : c->prof_pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        c->prof[p.slot].ms += ms;
        c->prof[p.slot].n += 1;
        c->prof[p.slot].bytes += p.bytes;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->prof_pending.clear();
}

long long vlen0(const amg_context* c) { return 2LL * c->N; }

// elementwise helpers on FP64 [n] complex arrays
__global__ void k_sub_d(double2* d, const double2* a, const double2* b, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] = a[e] - b[e];
}
__global__ void k_add_d(double2* d, const double2* a, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] += a[e];
}
// Copies of a few kilobytes between device memory and the outer FGMRES's page-locked staging,
// through the staging's device mapping by one CTA, so they never queue on the copy engines
// behind large transfers of other streams (the batches amg_solve_stream moves while a solve
// runs); the host reads the staging only after an event recorded behind the copy.  Loads
// are volatile: a host-side source is read where it lies, never from a cached copy.
__global__ void k_stage_words(unsigned* dst, const volatile unsigned* src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    __threadfence_system();
}

__global__ void k_set_int(int* p, int v, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}
__global__ void k_sap_check(const double* norm2, const double* vnorm2, double tol, int* act, int* conv, int R) {
    const int i = threadIdx.x;
    if (i >= R || !act[i]) return;
    if (sqrt(norm2[i]) < tol * sqrt(vnorm2[i])) { act[i] = 0; conv[i] = 1; }
}
// Re-orthogonalise a source only when the first Gram-Schmidt pass cancelled more than half of
// |w|^2 ("twice is enough": |w'| < |w| / sqrt(2)); d1[r][nv] = |w|^2, d2[r][nv] = |w'|^2.
__global__ void k_reorth_flag(const double2* d1, const double2* d2, int nv, const int* arn, int* flag, int R) {
    const int i = threadIdx.x;
    if (i >= R) return;
    flag[i] = (arn[i] && d2[i * (nv + 1) + nv].x < 0.5 * d1[i * (nv + 1) + nv].x) ? 1 : 0;
}
// |w_final|^2 of source r from the second pass: d2[r][nv] = |w'|^2 and, where a third pass
// projects again (flag), minus its coefficients' |d2[r][k]|^2 (Pythagoras; they are the
// small re-orthogonalisation corrections, so nothing cancels)
__host__ __device__ inline double final_norm2(const double2* d2r, int nv, int proj) {
    double v = d2r[nv].x;
    if (proj)
        for (int k = 0; k < nv; k++) v -= d2r[k].x * d2r[k].x + d2r[k].y * d2r[k].y;
    return v > 0 ? v : 0.0;
}
// scale[r] = 1/|w_final|, wmask[r] = arn[r] && |w_final| > 0, split into pmask (projected
// again on the way into V_{j+1}) and smask (only scaled)
__global__ void k_inv_norm2(const double2* d2, const int* flag, int nv, double* scale, const int* arn, int* wmask,
                            int* pmask, int* smask, int R) {
    const int i = threadIdx.x;
    if (i >= R) return;
    const double h = sqrt(final_norm2(d2 + (size_t)i * (nv + 1), nv, flag[i]));
    scale[i] = h > 0 ? 1.0 / h : 0.0;
    const int wm = (arn[i] && h > 0) ? 1 : 0;
    wmask[i] = wm;
    pmask[i] = wm && flag[i];
    smask[i] = wm && !flag[i];
}

int ensure_capacity(amg_context* c, int R);

// AMG_SAP_FUSE=1 forms the SAP residual before each red colour (and the first) inside the
// block solves instead of as a launch of its own.  It saves the residual launches (fine
// operator 15.1 -> 8.6 ms per 32-source step) but the D apply from global memory at the start
// of every block solve costs the SAP kernel more (154 -> 171 ms), so it is off by default.
bool sap_fuse_enabled() {
    static const int on = [] {
        const char* e = getenv("AMG_SAP_FUSE");
        return (e && e[0] == '1') ? 1 : 0;
    }();
    return on != 0;
}

// the D apply's bounded bulk-copy waits (k_dirac_tma): AMG_ERR_DEVICE_WAIT if one gave up
int check_fine_waits(cudaStream_t s) {
    const int e = fine_error_check(s);
    if (e < 0) return fail(AMG_ERR_CUDA, "reading the device error flag: %s", cudaGetErrorString(cudaGetLastError()));
    if (e > 0) return fail(AMG_ERR_DEVICE_WAIT, "a bulk-copy wait of the Dirac apply gave up");
    return AMG_OK;
}

// Teams (concurrent coarse SAP block solves) per engine CTA for blocks of up to 1024 dof,
// before the autotuner picks (or fixed by AMG_ENGINE_SAP_TEAMS = 1, 2 or 4): fewer, larger
// teams keep a block's links in L1 across its GMRES steps and split each step over more
// threads, at the price of more rounds per colour
int engine_sap_teams() {
    static const int n = [] {
        const char* e = getenv("AMG_ENGINE_SAP_TEAMS");
        const int v = e ? atoi(e) : 2;
        return (v == 1 || v == 4) ? v : 2;
    }();
    return n;
}

int engine_cluster_limit() {
    const char* e = getenv("AMG_ENGINE_CLUSTER");
    int v = e ? atoi(e) : 16;
    int p = 1;
    while (p * 2 <= v && p < 16) p *= 2;
    return p;
}

// ---------------------------------------------------------------------------------
// engine arguments for one precision
// ---------------------------------------------------------------------------------
template <typename T>
int build_engine(amg_context* c, PrecSet<T>& ps, int nsrc) {
    c->drop_graphs();   // captured cycles hold the old engine arguments
    const amg_params& p = c->p;
    EngArgs<T>& a = ps.eh;
    memset(&a, 0, sizeof a);
    a.nlev = c->L;
    a.p.m0 = (T)c->m0;
    a.p.cycle = p.cycle; a.p.nu1 = p.nu1; a.p.nu2 = p.nu2;
    a.p.sap_m = p.sap_gmres_m; a.p.sap_restarts = p.sap_gmres_restarts;
    a.p.sap_gmres_tol = (T)p.sap_gmres_tol; a.p.sap_tol = (T)p.sap_tol;
    a.p.k_m = p.kcycle_m; a.p.k_restarts = p.kcycle_restarts; a.p.k_tol = (T)p.kcycle_tol;
    a.p.c_m = p.coarse_m; a.p.c_restarts = p.coarse_restarts; a.p.c_tol = (T)p.coarse_tol;
    std::vector<int> rb;
    std::vector<int> rb_off(c->L, 0);
    for (int l = 0; l < c->L; l++) {
        rb_off[l] = (int)rb.size();
        rb.insert(rb.end(), c->lv[l].red.begin(), c->lv[l].red.end());
        rb.insert(rb.end(), c->lv[l].black.begin(), c->lv[l].black.end());
    }
    CKR(ps.red_black.alloc(std::max<size_t>(rb.size(), 1) * sizeof(int)));
    if (!rb.empty())
        CK(cudaMemcpyAsync(ps.red_black.p, rb.data(), rb.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    long long off = 0;
    int sm = 0;
    auto al = [](long long v) { return (v + 1) & ~1LL; };
    for (int l = 1; l < c->L; l++) {
        const LevelHost& h = c->lv[l];
        EngLevel<T>& e = a.lv[l];
        e.level = l;
        e.nx = h.nx; e.nt = h.nt; e.n = h.n; e.K = h.K; e.coarsest = h.coarsest;
        e.bx = h.bx; e.bt = h.bt; e.xe = h.xe; e.te = h.te; e.ntest = h.ntest;
        e.W = h.coarsest ? nullptr : ps.W[l].template as<cx<T>>();
        e.links = ps.links[l].template as<cx<T>>();
        e.sbx = h.sbx; e.sbt = h.sbt; e.sxe = h.sxe; e.ste = h.ste; e.ncol = h.ncol;
        e.red = ps.red_black.template as<int>() + rb_off[l];
        e.black = e.red + h.ncol;
        // Level::gmres_l: GMRES(20, 20, 1e-10) below the coarsest level, the coarse knobs on it
        e.gm_m = h.coarsest ? p.coarse_m : 20;
        e.gm_restarts = h.coarsest ? p.coarse_restarts : 20;
        e.gm_tol = h.coarsest ? (T)p.coarse_tol : (T)1e-10;
        const long long nvec = (long long)h.n * h.K;
        e.off_kfg = off; off += al((2LL * p.kcycle_m + 2) * nvec);
        e.off_cg = off; off += al((long long)(e.gm_m + 2) * nvec);
        e.sm_kfg = sm; sm += gm_state_bytes(1, p.kcycle_m, sizeof(T));
        e.sm_cg = sm; sm += gm_state_bytes(1, e.gm_m, sizeof(T));
        if (!h.coarsest) {
            const LevelHost& hn = c->lv[l + 1];
            const long long ncv = (long long)hn.n * hn.K;
            e.off_cyc = off; off += al(nvec + 2 * ncv);
            const long long seglen = (long long)h.sxe * h.ste * h.K;
            e.off_sap = off; off += al(nvec + (long long)h.ncol * seglen);
            // (team areas are sized for 4 teams, so the autotuner may change the count in place)
            e.sap_nteam = seglen <= 1024 ? (ps.sap_teams ? ps.sap_teams : engine_sap_teams()) : 1;
            e.sap_vec_smem = 0;
            e.off_sapteam = off; off += al(4LL * (p.sap_gmres_m + 4) * seglen);
        }
    }
    // whole-CTA reduction scratch and the team area of the SAP block solves
    auto al16 = [](int v) { return (v + 15) & ~15; };
    sm = al16(sm);
    a.smem_red = sm;
    sm += al16(2 * 2 * (kEngineThreads / 32) * (int)sizeof(T));
    a.smem_team = sm;
    const int tb_state = al16(gm_state_bytes(1, p.sap_gmres_m, sizeof(T)) + 64 * (int)sizeof(T));
    int tb = tb_state;
    for (int l = 1; l < c->L; l++) {
        const LevelHost& h = c->lv[l];
        if (h.coarsest) continue;
        EngLevel<T>& e = a.lv[l];
        const int seglen = h.sxe * h.ste * h.K;
        const int with_vec = al16(tb_state + (p.sap_gmres_m + 4) * seglen * (int)sizeof(cx<T>));
        if (sm + (seglen <= 1024 ? 4 : 1) * std::max(tb, with_vec) <= 200 * 1024) {
            e.sap_vec_smem = 1;
            tb = std::max(tb, with_vec);
        }
    }
    a.team_bytes = tb;
    sm += 4 * tb;
    long long io = 2;
    for (int l = 1; l < c->L; l++) io = std::max<long long>(io, (long long)c->lv[l].n * c->lv[l].K);
    a.off_io = off;
    a.io_len = al(io);
    off += 2 * a.io_len;
    sm += 64;
    if (sm > 227 * 1024) return fail(AMG_ERR_UNSUPPORTED, "engine shared memory needs %d bytes", sm);
    ps.eng_smem = sm;
    a.slab = std::max<long long>(off, 2);
    ps.eng_cap = std::max(nsrc, 1);
    ps.max_cluster = engine_cluster_limit();
    CKR(ps.eng_work.alloc((size_t)a.slab * ps.eng_cap * ps.max_cluster * sizeof(cx<T>)));
    CKR(ps.eng_status.alloc(sizeof(int) * (ps.eng_cap + 4) + sizeof(unsigned long long) * kMaxLevels * ENG_NCOUNT));
    a.work = ps.eng_work.template as<cx<T>>();
    a.status = ps.eng_status.template as<int>();
    a.flags = a.status + ps.eng_cap;
    a.counters = reinterpret_cast<unsigned long long*>(a.status + ps.eng_cap + 4);
    CK(cudaMemsetAsync(a.flags, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(a.counters, 0, sizeof(unsigned long long) * kMaxLevels * ENG_NCOUNT, c->stream));
    CKR(ps.eng_args.alloc(sizeof(EngArgs<T>)));
    CK(cudaMemcpyAsync(ps.eng_args.p, &a, sizeof a, cudaMemcpyHostToDevice, c->stream));
    return AMG_OK;
}

// Cluster size for `nsrc` concurrent engine sources: the largest power of two up to the
// configured limit (AMG_ENGINE_CLUSTER, default 16) whose clusters all fit on the device at
// once, so one launch serves every source in a single wave.
template <typename T>
int pick_cluster(PrecSet<T>& ps, int nsrc) {
    if (ps.cluster_pick > 0 && ps.cluster_pick <= ps.max_cluster) return ps.cluster_pick;
    for (int cs = ps.max_cluster; cs > 1; cs >>= 1) {
        if (!ps.cluster_cache[cs]) ps.cluster_cache[cs] = engine_max_clusters<T>(cs, ps.eng_smem) + 1;
        if (ps.cluster_cache[cs] - 1 >= nsrc) return cs;
    }
    return 1;
}

template <typename T>
int run_engine(amg_context* c, PrecSet<T>& ps, int op, int level, int nu, const cx<T>* in, long long in_stride,
               cx<T>* out, long long out_stride, int nsrc) {
    if (nsrc > ps.eng_cap) return fail(AMG_ERR_INVALID, "engine capacity %d < %d sources", ps.eng_cap, nsrc);
    const int cs = pick_cluster(ps, nsrc);
    ProfScope ps_(c, AMG_PROF_ENGINE, 0.0);
    CK(launch_engine_dev<T>(ps.eng_args.template as<EngArgs<T>>(), op, level, nu, in, in_stride, out, out_stride,
                            nsrc, ps.eng_smem, cs, c->stream));
    return AMG_OK;
}

template <typename T>
int alloc_fine(amg_context* c, PrecSet<T>& ps, int R) {
    const LevelHost& h0 = c->lv[0];
    const LevelHost& h1 = c->lv[1];
    const long long len = vlen0(c);
    CKR(ps.r0.alloc((size_t)R * len * sizeof(cx<T>)));
    CKR(ps.sap_r.alloc((size_t)R * len * sizeof(cx<T>)));
    CKR(ps.eta1.alloc((size_t)R * h1.n * h1.K * sizeof(cx<T>)));
    CKR(ps.psi1.alloc((size_t)R * h1.n * h1.K * sizeof(cx<T>)));
    const int nblk = h0.bx * h0.bt;
    const int spb = h0.xe * h0.te;
    int nchunk = std::max(1, std::min(std::max(1, spb / 128), (1184 + nblk - 1) / nblk));
    CKR(ps.rpart.alloc((size_t)R * nblk * nchunk * 2 * h0.ntest * sizeof(cx<T>)));
    return AMG_OK;
}

template <typename T>
int restrict_chunks(amg_context* c, int R) {
    const LevelHost& h0 = c->lv[0];
    const int nblk = h0.bx * h0.bt;
    const int spb = h0.xe * h0.te;
    (void)R;
    return std::max(1, std::min(std::max(1, spb / 128), (1184 + nblk - 1) / nblk));
}

// The fine links of a precision set as its kernels read them: FP64, or in the mixed form FP32,
// BF16 or FP16 pairs (amg_params.link_storage)
template <typename T>
Links<T> fine_links(amg_context* c, PrecSet<T>& ps) {
    if constexpr (sizeof(T) == 8) {
        (void)c;
        return Links<T>(ps.U.template as<cx<T>>());
    } else {
        return Links<T>(ps.U.p, c->p.link_storage == AMG_LINKS_BF16 ? LINK_BF16
                                : c->p.link_storage == AMG_LINKS_F16 ? LINK_F16
                                                                     : LINK_NATIVE);
    }
}

template <typename T>
void fine_restrict(amg_context* c, PrecSet<T>& ps, const cx<T>* v, cx<T>* out, int R) {
    const LevelHost& h0 = c->lv[0];
    ProfScope ps_(c, AMG_PROF_RESTRICT,
                  (double)h0.ntest * c->N * 2 * (ps.w0_bf16 ? 4.0 : (double)sizeof(cx<T>)) +
                      (double)R * c->N * 2 * sizeof(cx<T>));
    const int nchunk = restrict_chunks<T>(c, R);
    if (ps.w0_bf16)
        launch_restrict0<float, __nv_bfloat162>(ps.W0.template as<__nv_bfloat162>(), (const cx<float>*)v,
                                                 (cx<float>*)out, ps.rpart.template as<cx<float>>(), c->nx, c->nt,
                                                 h0.bx, h0.bt, h0.ntest, R, nchunk, c->stream);
    else
        launch_restrict0<T, cx<T>>(ps.W0.template as<cx<T>>(), v, out, ps.rpart.template as<cx<T>>(), c->nx, c->nt,
                                    h0.bx, h0.bt, h0.ntest, R, nchunk, c->stream);
}

// psi += P vc, or psi = P vc with add = false (psi not read: the cycle's first write of it)
template <typename T>
void fine_prolong_add(amg_context* c, PrecSet<T>& ps, const cx<T>* vc, cx<T>* psi, int R, bool add = true) {
    const LevelHost& h0 = c->lv[0];
    ProfScope ps_(c, AMG_PROF_PROLONG,
                  (double)h0.ntest * c->N * 2 * (ps.w0_bf16 ? 4.0 : (double)sizeof(cx<T>)) +
                      (double)R * c->N * 2 * (add ? 2 : 1) * sizeof(cx<T>));
    if (ps.w0_bf16)
        launch_prolong0_add<float, __nv_bfloat162>(ps.W0.template as<__nv_bfloat162>(), (const cx<float>*)vc,
                                                    (cx<float>*)psi, c->nx, c->nt, h0.bx, h0.bt, h0.ntest, R,
                                                    c->stream, add);
    else
        launch_prolong0_add<T, cx<T>>(ps.W0.template as<cx<T>>(), vc, psi, c->nx, c->nt, h0.bx, h0.bt, h0.ntest, R,
                                       c->stream, add);
}

// ---------------------------------------------------------------------------------
// SAP_C::SAP on the fine level (src/sap.cpp:64-174) for R sources, x in/out; v has stride
// vstride (0: the same source for all).  Every block of a colour is solved in one launch.
// Per-source early exit on ||v - D x|| < sap_tol ||v|| through device flags.  When
// need_ret is 0 the residual after the last sweep is skipped: the reference computes it
// only for the convergence test, whose result the cycles ignore.
// ---------------------------------------------------------------------------------
template <typename T>
int fine_sap(amg_context* c, PrecSet<T>& ps, const cx<T>* v, long long vstride, cx<T>* x, int nu, int R,
             int need_ret) {
    const LevelHost& h = c->lv[0];
    const amg_params& p = c->p;
    const long long len = vlen0(c);
    int* act = c->sap_flags.as<int>();
    int* conv = act + c->Rcap;
    double* vnorm2 = c->norms.as<double>();
    double* norm2 = vnorm2 + c->Rcap;
    double* partial = c->partial.as<double>();
    cx<T>* r = ps.sap_r.template as<cx<T>>();
    const Links<T> U = fine_links<T>(c, ps);
    const T m0 = (T)c->m0;
    k_set_int<<<1, 256, 0, c->stream>>>(act, 1, R);
    k_set_int<<<1, 256, 0, c->stream>>>(conv, 0, R);
    count_launch(2);
    launch_norm2<T>(v, len, vstride, R, partial, vnorm2, c->stream);
    // r = v - D x before every colour (src/sap.cpp:64-174).  With fusion (opt-in) the SAP
    // launch forms it for its own blocks (launch_sap0's vfuse); the residual after the black
    // colour stays a launch of its own because the early exit needs its norm over the whole
    // lattice.
    const bool fuse = sap_fuse_enabled();
    bool r_fresh = false;
    if (!fuse) {
        launch_residual<T>(U, v, vstride, x, r, c->nx, c->nt, R, m0, nullptr, nullptr, nullptr, c->stream);
        r_fresh = true;
    }
    const int S = h.sxe * h.ste;
    const int use_smem = sap0_smem_bytes<T>(S, p.sap_gmres_m, 1) <= 200 * 1024;
    if (!use_smem) CKR(ps.sap_scratch.alloc((size_t)h.ncol * R * (p.sap_gmres_m + 5) * 2 * S * sizeof(cx<T>)));
    cx<T>* scratch = use_smem ? nullptr : ps.sap_scratch.template as<cx<T>>();
    const int* d_red = ps.red_black.template as<int>();
    const int* d_black = d_red + h.ncol;
    for (int it = 0; it < nu; it++) {
        for (int colour = 0; colour < 2; colour++) {
            {
                ProfScope ps_(c, AMG_PROF_SAP, (double)h.ncol * S * (2.0 + 6.0 * R) * sizeof(cx<T>));
                CK(launch_sap0<T>(U, r, x, colour == 0 ? d_red : d_black, h.ncol, R, c->nx, c->nt, h.sbt, h.sxe,
                                  h.ste, m0, p.sap_gmres_m, p.sap_gmres_restarts, (T)p.sap_gmres_tol, use_smem,
                                  scratch, nullptr, act, c->stream, c->sap_variant, r_fresh ? nullptr : v,
                                  vstride));
            }
            r_fresh = false;
            const bool last = (colour == 1) && (it == nu - 1);
            if (last && !need_ret) break;
            if (colour == 1 || !fuse) {
                ProfScope ps_(c, AMG_PROF_FINE_OP, (double)c->N * (2.0 + 6.0 * R) * sizeof(cx<T>));
                launch_residual<T>(U, v, vstride, x, r, c->nx, c->nt, R, m0, partial,
                                   colour == 1 ? norm2 : nullptr, act, c->stream);
                r_fresh = true;
            }
            if (colour == 1) {
                k_sap_check<<<1, 256, 0, c->stream>>>(norm2, vnorm2, p.sap_tol, act, conv, R);
                count_launch(1);
            }
        }
    }
    CKL();
    return AMG_OK;
}

// ---------------------------------------------------------------------------------
// AlgebraicMG::k_cycle / v_cycle from the fine level (src/amg.cpp:90-178) for R sources:
// psi is added into.  psi_zero tells that psi is zero on entry (FGMRES_AMG zeroes it,
// include/amg.h:135-139), so r = eta - D psi is eta exactly.
// ---------------------------------------------------------------------------------
template <typename T>
int fine_cycle(amg_context* c, PrecSet<T>& ps, const cx<T>* eta, cx<T>* psi, int R, bool psi_zero) {
    const amg_params& p = c->p;
    const LevelHost& h1 = c->lv[1];
    const long long len = vlen0(c);
    const long long n1 = (long long)h1.n * h1.K;
    if (p.nu1 > 0) {
        CKR(fine_sap<T>(c, ps, eta, len, psi, p.nu1, R, 0));
        psi_zero = false;
    }
    const cx<T>* r = eta;
    if (!psi_zero) {
        launch_residual<T>(fine_links<T>(c, ps), eta, len, psi, ps.r0.template as<cx<T>>(), c->nx, c->nt, R,
                           (T)c->m0, nullptr, nullptr, nullptr, c->stream);
        r = ps.r0.template as<cx<T>>();
    }
    cx<T>* eta1 = ps.eta1.template as<cx<T>>();
    cx<T>* psi1 = ps.psi1.template as<cx<T>>();
    fine_restrict<T>(c, ps, r, eta1, R);
    if (p.cycle == AMG_CYCLE_K) {
        CKR(run_engine<T>(c, ps, ENG_KFGMRES, 1, 0, eta1, n1, psi1, n1, R));
    } else {
        CK(cudaMemsetAsync(psi1, 0, (size_t)R * n1 * sizeof(cx<T>), c->stream));
        CKR(run_engine<T>(c, ps, ENG_VCYCLE, 1, 0, eta1, n1, psi1, n1, R));
    }
    // with psi = 0 on entry and no pre-smoothing psi has not been read yet: the prolongation
    // stores into it (the caller need not clear it)
    fine_prolong_add<T>(c, ps, psi1, psi, R, !psi_zero);
    if (p.nu2 > 0) CKR(fine_sap<T>(c, ps, eta, len, psi, p.nu2, R, 0));
    CKL();
    return AMG_OK;
}

// FGMRES_AMG::preconditioner (include/amg.h:134-144): out = 0, then one cycle
// AMG_GRAPHS=0 runs the cycles eagerly (A/B tests)
int graphs_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("AMG_GRAPHS");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on;
}

// Runs body() (launches on c->stream only, no host synchronisation) through the graph cache
// entry `key`: eagerly on its first use (lazy allocations and attributes happen then),
// captured into a graph on the second, replayed afterwards.  Profiling runs eagerly.
template <class Body>
int run_graph(amg_context* c, const std::tuple<int, int, const void*, void*>& key, Body&& body) {
    if (!graphs_enabled() || c->graphs_off || c->prof_on) return body();
    amg_context::GraphEntry& e = c->graphs[key];
    if (e.exec) {
        count_launch((int)e.launches);
        CK(cudaGraphLaunch(e.exec, c->stream));
        return AMG_OK;
    }
    if (e.uses++ == 0) return body();
    const long long l0 = amg_launch_count();
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = (rc >= 0 && ec == cudaSuccess && g) ? cudaGraphInstantiate(&exec, g, 0) : cudaErrorUnknown;
    if (g) cudaGraphDestroy(g);
    if (rc < 0 || ec != cudaSuccess || ei != cudaSuccess) {
        // capture did not work here: fall back to eager launches for this context
        cudaGetLastError();
        c->graphs_off = 1;
        if (rc < 0) return rc;
        return body();
    }
    e.exec = exec;
    e.launches = amg_launch_count() - l0;
    CK(cudaGraphLaunch(e.exec, c->stream));
    return AMG_OK;
}

// z = M v for R sources.  Mixed precision with want_z = false leaves the FP32 result in c->zf
// for the caller (the outer step promotes it while applying D), instead of converting it
// into z.
int precondition(amg_context* c, const double2* v, double2* z, int R, bool want_z = true) {
    const long long len = vlen0(c);
    if (c->precond == AMG_PRECOND_NONE) {   // FGMRES_fine_level::preconditioner: z = v
        CK(cudaMemcpyAsync(z, v, (size_t)R * len * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        return AMG_OK;
    }
    if (c->p.precision == AMG_PREC_F64) {
        // staged through fixed buffers, so one graph serves every Krylov slot
        double2* vs = c->vd.as<double2>();
        double2* zs = c->zd.as<double2>();
        CK(cudaMemcpyAsync(vs, v, (size_t)R * len * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        CKR(run_graph(c, std::make_tuple(0, R, (const void*)vs, (void*)zs), [&]() -> int {
            // the cycle without pre-smoothing writes z before reading it
            if (c->precond == AMG_PRECOND_SAP || c->p.nu1 > 0)
                CK(cudaMemsetAsync(zs, 0, (size_t)R * len * sizeof(double2), c->stream));
            if (c->precond == AMG_PRECOND_SAP) return fine_sap<double>(c, c->d, vs, len, zs, 1, R, 0);
            return fine_cycle<double>(c, c->d, vs, zs, R, true);
        }));
        CK(cudaMemcpyAsync(z, zs, (size_t)R * len * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        return AMG_OK;
    }
    float2* vf = c->vf.as<float2>();
    float2* zf = c->zf.as<float2>();
    if (c->vf_src != v) {
        launch_d2f(vf, v, R * len, c->stream);
        c->vf_src = v;
    }
    CKR(run_graph(c, std::make_tuple(1, R, (const void*)vf, (void*)zf), [&]() -> int {
        if (c->precond == AMG_PRECOND_SAP || c->p.nu1 > 0)
            CK(cudaMemsetAsync(zf, 0, (size_t)R * len * sizeof(float2), c->stream));
        if (c->precond == AMG_PRECOND_SAP) return fine_sap<float>(c, c->f, vf, len, zf, 1, R, 0);
        return fine_cycle<float>(c, c->f, vf, zf, R, true);
    }));
    if (want_z) launch_f2d(z, zf, R * len, c->stream);
    CKL();
    return AMG_OK;
}

// ---------------------------------------------------------------------------------
// The many-configuration solve's preconditioner (amg_solve_many): contexts whose fine SAP
// runs the 16-bit-basis kernel on blocks of one size go through their K- or V-cycles in
// lock step, and each colour's block solves of all of them are one launch over a table of
// (lattice, block) columns instead of one launch per lattice.  Everything else a context
// launches stays on its own stream; the shared launch runs on the first context's stream,
// which waits for every context's residual before it, and every stream waits for it after.
// AMG_SAP_GROUP=0 keeps one launch per lattice (A/B tests).
// ---------------------------------------------------------------------------------
bool sap_group_enabled() {
    static const int on = [] {
        const char* e = getenv("AMG_SAP_GROUP");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on != 0;
}

// block size of the context's fine SAP if the group can run it, else 0
int group_block_size(const amg_context* c) {
    const amg_params& p = c->p;
    const LevelHost& h = c->lv[0];
    const int S = h.sxe * h.ste;
    if (p.precision != AMG_PREC_MIXED || c->precond != AMG_PRECOND_MG || p.nu1 != 0 || c->L < 2 ||
        p.link_storage != AMG_LINKS_F16 || p.sap_gmres_m != 5 || h.ste % 4 != 0 || sap_fuse_enabled() ||
        c->prof_on || !sap0_warp_enabled())
        return 0;
    return (S == 256 || S == 512 || S == 1024) ? S : 0;
}

struct SapGroup {
    std::vector<amg_context*> cs;
    std::vector<int> R;
    int S = 0, ncols = 0, max_rhs = 0;
    bool bf = true;
    DevBuf tasks, cols;              // SapTask [2][n]; col_task [2][ncols] then col_seg [2][ncols]
    std::vector<cudaEvent_t> ev;     // per context: its work up to the shared launch
    cudaEvent_t join = nullptr;      // the shared launch
    SapGroup() = default;
    SapGroup(const SapGroup&) = delete;
    SapGroup& operator=(const SapGroup&) = delete;
    ~SapGroup() {
        for (auto e : ev) if (e) cudaEventDestroy(e);
        if (join) cudaEventDestroy(join);
    }

    int build(const std::vector<amg_context*>& cs_, const std::vector<int>& R_) {
        cs = cs_;
        R = R_;
        const int n = (int)cs.size();
        S = group_block_size(cs[0]);
        bf = false;
        for (auto* c : cs) bf |= c->sap_variant != SAP_VARIANT_HALF;   // FP16 basis only if every context chose it
        std::vector<SapTask> t(2 * n);
        std::vector<int> col_task, col_seg;
        ncols = 0;
        max_rhs = 0;
        for (int i = 0; i < n; i++) ncols += cs[i]->lv[0].ncol;
        col_task.resize(2 * ncols);
        col_seg.resize(2 * ncols);
        for (int q = 0; q < 2; q++) {
            int col = q * ncols;
            for (int i = 0; i < n; i++) {
                amg_context* c = cs[i];
                const LevelHost& h = c->lv[0];
                const Links<float> U = fine_links<float>(c, c->f);
                const int* red = c->f.red_black.template as<int>();
                SapTask& k = t[q * n + i];
                k.U = U.p;
                k.r = c->f.sap_r.as<float2>();
                k.x = c->zf.as<float2>();
                k.blocks = q == 0 ? red : red + h.ncol;
                k.act = c->sap_flags.as<int>();
                k.ncol = h.ncol;
                k.nrhs = R[i];
                k.nx = c->nx;
                k.nt = c->nt;
                k.sbt = h.sbt;
                k.sxe = h.sxe;
                k.ste = h.ste;
                k.restarts = c->p.sap_gmres_restarts;
                k.m0 = (float)c->m0;
                k.tol = (float)c->p.sap_gmres_tol;
                for (int s = 0; s < h.ncol; s++, col++) {
                    col_task[col] = q * n + i;
                    col_seg[col] = s;
                }
                max_rhs = std::max(max_rhs, R[i]);
            }
        }
        amg_context* c0 = cs[0];
        CKR(tasks.alloc(t.size() * sizeof(SapTask)));
        CKR(cols.alloc(4 * (size_t)ncols * sizeof(int)));
        CK(cudaMemcpyAsync(tasks.p, t.data(), t.size() * sizeof(SapTask), cudaMemcpyHostToDevice, c0->stream));
        CK(cudaMemcpyAsync(cols.p, col_task.data(), 2 * (size_t)ncols * sizeof(int), cudaMemcpyHostToDevice,
                           c0->stream));
        CK(cudaMemcpyAsync(cols.as<int>() + 2 * ncols, col_seg.data(), 2 * (size_t)ncols * sizeof(int),
                           cudaMemcpyHostToDevice, c0->stream));
        ev.assign(n, nullptr);
        for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        CK(cudaStreamSynchronize(c0->stream));   // the host tables may go
        return AMG_OK;
    }

    // one colour's block solves of every context (src/sap.cpp:64-174, the colour loop)
    int shared_launch(int colour) {
        const int n = (int)cs.size();
        cudaStream_t s0 = cs[0]->stream;
        for (int i = 1; i < n; i++) {
            CK(cudaEventRecord(ev[i], cs[i]->stream));
            CK(cudaStreamWaitEvent(s0, ev[i], 0));
        }
        const int* ct = cols.as<int>() + colour * ncols;
        CK(launch_sap0_h_group(tasks.as<SapTask>(), ct, ct + 2 * ncols, ncols, max_rhs, S, bf, s0));
        CK(cudaEventRecord(join, s0));
        for (int i = 1; i < n; i++) CK(cudaStreamWaitEvent(cs[i]->stream, join, 0));
        return AMG_OK;
    }

    // fine_sap<float>(c, c->f, v, len, x, nu, R, 0) of every context, the block solves shared
    int sap(const std::vector<const float2*>& v, const std::vector<float2*>& x, int nu) {
        const int n = (int)cs.size();
        for (int i = 0; i < n; i++) {
            amg_context* c = cs[i];
            const long long len = vlen0(c);
            int* act = c->sap_flags.as<int>();
            double* vnorm2 = c->norms.as<double>();
            k_set_int<<<1, 256, 0, c->stream>>>(act, 1, R[i]);
            k_set_int<<<1, 256, 0, c->stream>>>(act + c->Rcap, 0, R[i]);
            count_launch(2);
            launch_norm2<float>(v[i], len, len, R[i], c->partial.as<double>(), vnorm2, c->stream);
            launch_residual<float>(fine_links<float>(c, c->f), v[i], len, x[i], c->f.sap_r.as<float2>(), c->nx, c->nt,
                                   R[i], (float)c->m0, nullptr, nullptr, nullptr, c->stream);
        }
        for (int it = 0; it < nu; it++) {
            for (int colour = 0; colour < 2; colour++) {
                CKR(shared_launch(colour));
                if (colour == 1 && it == nu - 1) break;
                for (int i = 0; i < n; i++) {
                    amg_context* c = cs[i];
                    int* act = c->sap_flags.as<int>();
                    double* vnorm2 = c->norms.as<double>();
                    double* norm2 = vnorm2 + c->Rcap;
                    launch_residual<float>(fine_links<float>(c, c->f), v[i], vlen0(c), x[i], c->f.sap_r.as<float2>(),
                                           c->nx, c->nt, R[i], (float)c->m0, c->partial.as<double>(),
                                           colour == 1 ? norm2 : nullptr, act, c->stream);
                    if (colour == 1) {
                        k_sap_check<<<1, 256, 0, c->stream>>>(norm2, vnorm2, c->p.sap_tol, act, act + c->Rcap, R[i]);
                        count_launch(1);
                    }
                }
            }
        }
        for (auto* c : cs) CKL();
        return AMG_OK;
    }

    // z = M v (FGMRES_AMG::preconditioner, include/amg.h:134-144) for every context in the
    // mixed form, the FP32 result left in each context's zf (as precondition(.., false))
    int precondition(const std::vector<const double2*>& v) {
        const int n = (int)cs.size();
        std::vector<const float2*> vf(n);
        std::vector<float2*> zf(n);
        for (int i = 0; i < n; i++) {
            amg_context* c = cs[i];
            const long long len = vlen0(c);
            vf[i] = c->vf.as<float2>();
            zf[i] = c->zf.as<float2>();
            if (c->vf_src != v[i]) {
                launch_d2f(c->vf.as<float2>(), v[i], R[i] * len, c->stream);
                c->vf_src = v[i];
            }
            // fine_cycle<float> with psi = 0 on entry and no pre-smoothing: r = eta, and the
            // prolongation is the first write of z
            const LevelHost& h1 = c->lv[1];
            const long long n1 = (long long)h1.n * h1.K;
            float2* eta1 = c->f.eta1.as<float2>();
            float2* psi1 = c->f.psi1.as<float2>();
            fine_restrict<float>(c, c->f, vf[i], eta1, R[i]);
            if (c->p.cycle == AMG_CYCLE_K) {
                CKR(run_engine<float>(c, c->f, ENG_KFGMRES, 1, 0, eta1, n1, psi1, n1, R[i]));
            } else {
                CK(cudaMemsetAsync(psi1, 0, (size_t)R[i] * n1 * sizeof(float2), c->stream));
                CKR(run_engine<float>(c, c->f, ENG_VCYCLE, 1, 0, eta1, n1, psi1, n1, R[i]));
            }
            fine_prolong_add<float>(c, c->f, psi1, zf[i], R[i], false);
        }
        if (cs[0]->p.nu2 > 0) CKR(sap(vf, zf, cs[0]->p.nu2));
        for (auto* c : cs) CKL();
        return AMG_OK;
    }
};

// Coarse SAP teams per engine CTA (1, 2 or 4) for the levels whose block vectors allow more
// than one, in the active precision's engine arguments (host copy and device block).
int set_sap_teams(amg_context* c, int t) {
    auto apply = [&](auto& ps) -> int {
        if (!ps.eng_args.p) return AMG_OK;
        ps.sap_teams = t;
        for (int l = 1; l < c->L; l++)
            if (!c->lv[l].coarsest && ps.eh.lv[l].sap_nteam > 0 &&
                (long long)c->lv[l].sxe * c->lv[l].ste * c->lv[l].K <= 1024)
                ps.eh.lv[l].sap_nteam = t;
        CK(cudaMemcpyAsync(ps.eng_args.p, &ps.eh, sizeof ps.eh, cudaMemcpyHostToDevice, c->stream));
        return AMG_OK;
    };
    return c->p.precision == AMG_PREC_MIXED ? apply(c->f) : apply(c->d);
}

// ---------------------------------------------------------------------------------
// Autotuner: on a context's first solve, time one preconditioner application (the first
// Krylov vector, R sources) for every fine SAP kernel variant that applies (FP32: paired
// MGS with four or two sites per thread, paired CGS, communication-avoiding, lean, and with
// FP16 links the FP16- and BF16-basis kernels at three CTAs per SM; FP64: lean) and every
// engine cluster size
// the device can schedule, and keep the fastest; then, at that choice, the coarse SAP teams
// per engine CTA (4, 2, 1).  An environment override (AMG_SAP_KERNEL, AMG_ENGINE_CLUSTER,
// AMG_ENGINE_SAP_TEAMS) fixes that dimension instead.
// ---------------------------------------------------------------------------------
int autotune(amg_context* c, const double2* v, double2* z, int R) {
    c->tuned = 1;
    if (!c->p.autotune) return AMG_OK;
    const bool mixed = c->p.precision == AMG_PREC_MIXED;
    std::vector<int> variants{-1};
    if (!getenv("AMG_SAP_KERNEL") && mixed) {
        variants = {SAP_VARIANT_PAIRED, SAP_VARIANT_PAIRED2, SAP_VARIANT_CGS, SAP_VARIANT_CA, SAP_VARIANT_LEAN};
        if (c->p.link_storage == AMG_LINKS_F16) {
            variants.push_back(SAP_VARIANT_HALF);
            variants.push_back(SAP_VARIANT_BF16B);
        }
    }
    int* pick = mixed ? &c->f.cluster_pick : &c->d.cluster_pick;
    const int maxc = mixed ? c->f.max_cluster : c->d.max_cluster;
    const int smem = mixed ? c->f.eng_smem : c->d.eng_smem;
    std::vector<int> clusters{0};
    if (!getenv("AMG_ENGINE_CLUSTER")) {
        clusters.clear();
        for (int cs = maxc; cs >= 1; cs >>= 1) {
            const int n = cs == 1 ? 1 : (mixed ? engine_max_clusters<float>(cs, smem) : engine_max_clusters<double>(cs, smem));
            if (n > 0) clusters.push_back(cs);
        }
        if (clusters.empty()) clusters.push_back(0);
    }
    const int graphs_was = c->graphs_off;
    c->graphs_off = 1;
    cudaEvent_t a = nullptr, b = nullptr;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float best = 1e30f;
    int bv = -1, bc = 0;
    int rc = AMG_OK;
    for (int vv : variants) {
        for (int cs : clusters) {
            c->sap_variant = vv;
            *pick = cs;
            if ((rc = precondition(c, v, z, R, false)) < 0) break;   // warm-up (attributes, lazy buffers)
            cudaEventRecord(a, c->stream);
            if ((rc = precondition(c, v, z, R, false)) < 0) break;
            cudaEventRecord(b, c->stream);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (ms < best) { best = ms; bv = vv; bc = cs; }
        }
        if (rc < 0) break;
    }
    c->sap_variant = bv;
    *pick = bc;
    // then the coarse SAP teams per engine CTA at that choice (the engine reads the count
    // from its argument block, so each candidate is one upload)
    if (rc >= 0 && !getenv("AMG_ENGINE_SAP_TEAMS")) {
        int bt = 0;
        float best_t = 1e30f;
        for (int t : {4, 2, 1}) {
            if ((rc = set_sap_teams(c, t)) < 0) break;
            if ((rc = precondition(c, v, z, R, false)) < 0) break;
            cudaEventRecord(a, c->stream);
            if ((rc = precondition(c, v, z, R, false)) < 0) break;
            cudaEventRecord(b, c->stream);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (ms < best_t) { best_t = ms; bt = t; }
        }
        if (rc >= 0 && bt) {
            rc = set_sap_teams(c, bt);
            best = best_t;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    c->graphs_off = graphs_was;
    c->tuned_us = best < 1e29f ? 1e3 * best : 0;
    c->drop_graphs();
    return rc;
}

// ---------------------------------------------------------------------------------
// Outer FGMRES (FGMRES::fgmres, src/fgmres.cpp:5-115) with func = D_phi and the AMG
// preconditioner, x0 = 0, for R sources with independent Krylov spaces.  Arnoldi uses
// classical Gram-Schmidt with one re-orthogonalisation on the device; the Hessenberg
// rotations, the triangular solve and every control decision run on the host in FP64,
// per source exactly as the reference (maxIt carried over restart cycles).
//
// The solve is a state machine: issue() queues device work on the context's stream that
// ends with a device-to-host copy into pinned memory and an event; advance() runs once that
// event has completed, does the host part and queues the next piece.  One solve drives it
// to the end (outer_fgmres); amg_solve_many drives several contexts in turn, so the GPU
// runs one context's kernels while the host handles another's Givens rotations.
// ---------------------------------------------------------------------------------
// dst = src for `bytes` (a multiple of 4) where one side lies in c->hpin: by k_stage_words
// through hpin's device mapping, or by cudaMemcpyAsync if there is none
int stage_copy(amg_context* c, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (!c->hpin_dev || bytes % 4 || bytes > (size_t(1) << 30)) {
        CK(cudaMemcpyAsync(dst, src, bytes, kind, c->stream));
        return AMG_OK;
    }
    char* h0 = static_cast<char*>(c->hpin.p);
    auto dev = [&](const void* hp) { return c->hpin_dev + (static_cast<const char*>(hp) - h0); };
    unsigned* d = static_cast<unsigned*>(kind == cudaMemcpyDeviceToHost ? static_cast<void*>(dev(dst)) : dst);
    const unsigned* s =
        static_cast<const unsigned*>(kind == cudaMemcpyHostToDevice ? static_cast<const void*>(dev(src)) : src);
    k_stage_words<<<1, 256, 0, c->stream>>>(d, s, (int)(bytes / 4));
    count_launch(1);
    CK(cudaGetLastError());
    return AMG_OK;
}

struct OuterSolve {
    // PRECOND: a step waits for its preconditioner, which the caller runs for several
    // contexts together (defer set: amg_solve_many's grouped SAP), then issue_step_post
    enum Phase { INIT, STEP, RESTART, PRECOND, DONE };
    bool defer = false;
    amg_context* c = nullptr;
    const double2* b = nullptr;
    double2* x = nullptr;
    int R = 0;
    amg_solve_info* info = nullptr;
    int m = 0, np = 0;
    long long len = 0, vstride = 0;
    std::vector<cd> H, g, cn, sn, eta;
    std::vector<double> err, normb;
    std::vector<int> maxit, act, arn, iters;
    int k = 0, j = 0;
    Phase phase = DONE;
    int rc = AMG_OK;
    // pinned host staging (views into c->hpin)
    double* h_norm = nullptr;      // [2R]
    double2* h_dots = nullptr;     // [R * (2m + 3)]
    int* h_ro = nullptr;           // [R]
    int* h_mask = nullptr;         // [2R]  act, arn
    double* h_scal = nullptr;      // [R]
    double2* h_eta = nullptr;      // [R * m]
    int* h_nvr = nullptr;          // [R]

    int* act_d() const { return c->masks.as<int>(); }
    int* arn_d() const { return act_d() + c->Rcap; }
    int* wm_d() const { return arn_d() + c->Rcap; }
    int* nvr_d() const { return wm_d() + c->Rcap; }
    int* ro_d() const { return nvr_d() + c->Rcap; }
    int* pm_d() const { return ro_d() + c->Rcap; }   // wm && ro: projected again into V_{j+1}
    int* sm_d() const { return pm_d() + c->Rcap; }   // wm && !ro: only scaled into V_{j+1}

    int init(amg_context* c_, const double2* b_, double2* x_, int R_, amg_solve_info* info_) {
        c = c_; b = b_; x = x_; R = R_; info = info_;
        c->vf_src = nullptr;
        const amg_params& p = c->p;
        m = p.outer_m;
        len = vlen0(c);
        vstride = (long long)R * len;
        np = (int)std::min<long long>(592, (len + 255) / 256);
        H.assign((size_t)R * (m + 1) * m, cd(0));
        g.assign((size_t)R * (m + 1), cd(0));
        cn.assign((size_t)R * m, cd(0));
        sn.assign((size_t)R * m, cd(0));
        eta.assign((size_t)R * m, cd(0));
        err.assign(R, 0);
        normb.assign(R, 0);
        maxit.assign(R, m);
        act.assign(R, 1);
        arn.assign(R, 0);
        iters.assign(R, p.outer_restarts * m);
        char* hp = static_cast<char*>(c->hpin.p);
        auto take = [&](size_t bytes) { char* q = hp; hp += (bytes + 15) & ~size_t(15); return q; };
        h_norm = reinterpret_cast<double*>(take(2 * R * sizeof(double)));
        h_dots = reinterpret_cast<double2*>(take((size_t)R * (2 * m + 3) * sizeof(double2)));
        h_ro = reinterpret_cast<int*>(take(R * sizeof(int)));
        h_mask = reinterpret_cast<int*>(take(2 * R * sizeof(int)));
        h_scal = reinterpret_cast<double*>(take(R * sizeof(double)));
        h_eta = reinterpret_cast<double2*>(take((size_t)R * m * sizeof(double2)));
        h_nvr = reinterpret_cast<int*>(take(R * sizeof(int)));
        c->history.clear();
        // x = x0 = 0; r = b - D x into V0; |r|^2 and |b|^2 to the host
        double2* V = c->V.as<double2>();
        double* n2 = c->norms.as<double>();
        double* partial = c->partial.as<double>();
        CK(cudaMemsetAsync(x, 0, (size_t)R * len * sizeof(double2), c->stream));
        launch_residual<double>(c->d.U.as<double2>(), b, len, x, V, c->nx, c->nt, R, c->m0, partial, n2, nullptr,
                                c->stream);
        launch_norm2<double>(b, len, len, R, partial, n2 + c->Rcap, c->stream);
        CKR(stage_copy(c, h_norm, n2, R * sizeof(double), cudaMemcpyDeviceToHost));
        CKR(stage_copy(c, h_norm + R, n2 + c->Rcap, R * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaEventRecord(c->ev_host, c->stream));
        phase = INIT;
        return AMG_OK;
    }

    int upload_masks() {
        for (int r = 0; r < R; r++) { h_mask[r] = act[r]; h_mask[R + r] = arn[r]; }
        CKR(stage_copy(c, act_d(), h_mask, R * sizeof(int), cudaMemcpyHostToDevice));
        CKR(stage_copy(c, arn_d(), h_mask + R, R * sizeof(int), cudaMemcpyHostToDevice));
        return AMG_OK;
    }

    // a new restart cycle: V0 = r / |r| for the active sources, then Arnoldi step 0
    int begin_cycle() {
        bool any = false;
        for (int r = 0; r < R; r++) any |= act[r] != 0;
        if (!any || k >= c->p.outer_restarts) return finish();
        for (int r = 0; r < R; r++) {
            arn[r] = act[r];
            h_scal[r] = act[r] ? 1.0 / err[r] : 0.0;
            if (act[r]) g[(size_t)r * (m + 1)] = cd(err[r], 0);
        }
        CKR(upload_masks());
        CKR(stage_copy(c, c->scal.p, h_scal, R * sizeof(double), cudaMemcpyHostToDevice));
        double2* V = c->V.as<double2>();
        float2* yf = c->p.precision == AMG_PREC_MIXED ? c->vf.as<float2>() : nullptr;
        launch_scale(V, V, len, c->scal.as<double>(), act_d(), R, c->stream, yf);
        c->vf_src = yf ? V : nullptr;
        j = 0;
        return issue_step();
    }

    // Arnoldi step j on the device: Z_j = M V_j, w = D Z_j, CGS2 against V_0..V_j,
    // V_{j+1} = w / |w|; the Hessenberg column goes to the host
    int issue_step() {
        double2* V = c->V.as<double2>();
        double2* Z = c->Z.as<double2>();
        double2* Vj = V + (long long)j * vstride;
        double2* Zj = Z + (long long)j * vstride;
        if (!c->tuned && !c->prof_on && c->precond != AMG_PRECOND_NONE) CKR(autotune(c, Vj, Zj, R));
        if (defer && group_block_size(c)) {
            phase = PRECOND;
            return AMG_OK;
        }
        const bool mixed = c->p.precision == AMG_PREC_MIXED && c->precond != AMG_PRECOND_NONE;
        CKR(precondition(c, Vj, Zj, R, !mixed));
        return issue_step_post();
    }
    // the basis vector step j preconditions (the grouped preconditioner's input)
    const double2* step_input() const { return c->V.as<double2>() + (long long)j * vstride; }
    // the mixed form keeps Z_k = M V_k as the preconditioner wrote it, in FP32 (its FP64 value
    // is the exact promotion), in the first half of the Z buffer with the FP64 slots' strides
    float2* zslot_f32(int k) const { return c->Z.as<float2>() + (long long)k * vstride; }

    // the rest of Arnoldi step j once z_j is in c->zf (mixed) or Z_j: w = D z_j, CGS2, V_{j+1}
    int issue_step_post() {
        double2* V = c->V.as<double2>();
        double2* Z = c->Z.as<double2>();
        double2* w = c->w.as<double2>();
        double2* dpart = c->partial.as<double2>();
        double2* dots = c->dots.as<double2>();
        double2* Zj = Z + (long long)j * vstride;
        const bool mixed = c->p.precision == AMG_PREC_MIXED && c->precond != AMG_PRECOND_NONE;
        {
            // algorithmic bytes per site: the links (2 x 16 B) and per source z_j in (FP32:
            // 16 B, FP64: 32 B) and w out (32 B), plus Z_j out (FP32, 16 B) in the mixed form
            ProfScope ps_(c, AMG_PROF_OUTER_OP, (double)c->N * (32.0 + 64.0 * R));
            if (mixed)   // w = D z_j from the FP32 preconditioner output, copied into Z_j (FP32)
                launch_dirac_promote(c->d.U.as<double2>(), c->zf.as<float2>(), w, zslot_f32(j), c->nx, c->nt, R,
                                     c->m0, c->stream);
            else
                launch_dirac<double>(c->d.U.as<double2>(), Zj, w, c->nx, c->nt, R, c->m0, 0, c->stream);
        }
        const int nv = j + 1;
        double2* d1 = dots;
        double2* d2 = dots + (size_t)R * (nv + 1);
        {
            // classical Gram-Schmidt, re-orthogonalised only where the first pass cancelled; the
            // second projection and the normalisation are one pass writing V_{j+1}
            ProfScope ps_(c, AMG_PROF_BLAS, (double)R * len * sizeof(double2) * (3.0 * nv + 5.0));
            launch_multidot(w, V, len, vstride, nv, R, dpart, np, d1, arn_d(), c->stream);
            launch_axpy_multidot(w, V, len, vstride, nv, d1, nv + 1, nv, arn_d(), R, dpart, np, d2, c->stream);
            k_reorth_flag<<<1, 256, 0, c->stream>>>(d1, d2, nv, arn_d(), ro_d(), R);
            k_inv_norm2<<<1, 256, 0, c->stream>>>(d2, ro_d(), nv, c->scal.as<double>(), arn_d(), wm_d(), pm_d(),
                                                  sm_d(), R);
            count_launch(2);
            double2* Vn = V + (long long)(j + 1) * vstride;
            // (mixed precision: the FP32 copy of V_{j+1} for the next preconditioner call too)
            float2* yf = c->p.precision == AMG_PREC_MIXED ? c->vf.as<float2>() : nullptr;
            launch_axpy_scale_to(Vn, w, V, len, vstride, nv, d2, nv + 1, c->scal.as<double>(), pm_d(), R, dpart, np,
                                 c->stream, yf);
            launch_scale(Vn, w, len, c->scal.as<double>(), sm_d(), R, c->stream, yf);
            c->vf_src = yf ? Vn : nullptr;
        }
        CKR(stage_copy(c, h_dots, dots, (size_t)R * 2 * (nv + 1) * sizeof(double2), cudaMemcpyDeviceToHost));
        CKR(stage_copy(c, h_ro, ro_d(), R * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaEventRecord(c->ev_host, c->stream));
        phase = STEP;
        return AMG_OK;
    }

    // the host part of Arnoldi step j: Hessenberg column, rotation(j) (src/fgmres.cpp:90-104)
    int finish_step() {
        const int nv = j + 1;
        const double2* hd = h_dots;
        for (int r = 0; r < R; r++) {
            if (!arn[r]) continue;
            cd* Hr = &H[(size_t)r * (m + 1) * m];
            cd* cnr = &cn[(size_t)r * m];
            cd* snr = &sn[(size_t)r * m];
            cd* gr = &g[(size_t)r * (m + 1)];
            for (int i = 0; i <= j; i++) {
                const double2 a = hd[(size_t)r * (nv + 1) + i];
                const double2 bq = hd[(size_t)R * (nv + 1) + (size_t)r * (nv + 1) + i];
                Hr[i * m + j] = h_ro[r] ? cd(a.x + bq.x, a.y + bq.y) : cd(a.x, a.y);
            }
            const double hn2 = final_norm2(hd + (size_t)R * (nv + 1) + (size_t)r * (nv + 1), nv, h_ro[r]);
            Hr[(j + 1) * m + j] = cd(std::sqrt(hn2), 0);
            for (int i = 0; i < j; i++) {
                cd temp = std::conj(cnr[i]) * Hr[i * m + j] + std::conj(snr[i]) * Hr[(i + 1) * m + j];
                Hr[(i + 1) * m + j] = -snr[i] * Hr[i * m + j] + cnr[i] * Hr[(i + 1) * m + j];
                Hr[i * m + j] = temp;
            }
            cd den = std::sqrt(std::conj(Hr[j * m + j]) * Hr[j * m + j] +
                               std::conj(Hr[(j + 1) * m + j]) * Hr[(j + 1) * m + j]);
            snr[j] = Hr[(j + 1) * m + j] / den;
            cnr[j] = Hr[j * m + j] / den;
            Hr[j * m + j] = std::conj(cnr[j]) * Hr[j * m + j] + std::conj(snr[j]) * Hr[(j + 1) * m + j];
            Hr[(j + 1) * m + j] = 0.0;
            gr[j + 1] = -snr[j] * gr[j];
            gr[j] = std::conj(cnr[j]) * gr[j];
            if (r == 0) c->history.push_back(std::abs(gr[j + 1]));
            if (std::abs(gr[j + 1]) < c->p.outer_tol * normb[r]) {
                maxit[r] = j + 1;
                arn[r] = 0;
            }
        }
        CKR(upload_masks());
        bool anyarn = false;
        for (int r = 0; r < R; r++) anyarn |= arn[r] != 0;
        if (anyarn && j + 1 < m) {
            j++;
            return issue_step();
        }
        return end_cycle();
    }

    // solve_upper_triangular (src/fgmres.cpp:107-115), x += sum eta_j Z_j, true residual
    int end_cycle() {
        for (int r = 0; r < R; r++) {
            h_nvr[r] = 0;
            if (!act[r]) continue;
            const cd* Hr = &H[(size_t)r * (m + 1) * m];
            const cd* gr = &g[(size_t)r * (m + 1)];
            cd* er = &eta[(size_t)r * m];
            const int n = maxit[r];
            for (int i = n - 1; i >= 0; i--) {
                er[i] = gr[i];
                for (int jj = i + 1; jj < n; jj++) er[i] -= Hr[i * m + jj] * er[jj];
                er[i] /= Hr[i * m + i];
            }
            for (int i = 0; i < m; i++) h_eta[(size_t)r * m + i] = i < n ? make_double2(er[i].real(), er[i].imag())
                                                                        : make_double2(0, 0);
            h_nvr[r] = n;
        }
        double2* eta_d = c->etab.as<double2>();
        CKR(stage_copy(c, eta_d, h_eta, (size_t)R * m * sizeof(double2), cudaMemcpyHostToDevice));
        CKR(stage_copy(c, nvr_d(), h_nvr, R * sizeof(int), cudaMemcpyHostToDevice));
        if (c->p.precision == AMG_PREC_MIXED && c->precond != AMG_PRECOND_NONE)
            launch_multiaxpy_add(x, zslot_f32(0), len, vstride, m, eta_d, m, nvr_d(), act_d(), R, c->stream);
        else
            launch_multiaxpy_add(x, c->Z.as<double2>(), len, vstride, m, eta_d, m, nvr_d(), act_d(), R, c->stream);
        double* n2 = c->norms.as<double>();
        launch_residual<double>(c->d.U.as<double2>(), b, len, x, c->V.as<double2>(), c->nx, c->nt, R, c->m0,
                                c->partial.as<double>(), n2, act_d(), c->stream);
        CKR(stage_copy(c, h_norm, n2, R * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaEventRecord(c->ev_host, c->stream));
        phase = RESTART;
        return AMG_OK;
    }

    int finish() {
        CKL();
        prof_harvest(c);
        if (info)
            for (int r = 0; r < R; r++) {
                info[r].iterations = iters[r];
                info[r].rel_residual = normb[r] > 0 ? err[r] / normb[r] : err[r];
                info[r].converged = err[r] < c->p.outer_tol * normb[r];
            }
        rc = AMG_OK;
        for (int r = 0; r < R; r++)
            if (act[r]) rc = AMG_NOT_CONVERGED;
        phase = DONE;
        return AMG_OK;
    }

    // called once the event of the queued piece has completed
    int advance() {
        switch (phase) {
            case INIT:
                for (int r = 0; r < R; r++) { err[r] = std::sqrt(h_norm[r]); normb[r] = std::sqrt(h_norm[R + r]); }
                k = 0;
                return begin_cycle();
            case STEP:
                return finish_step();
            case RESTART:
                for (int r = 0; r < R; r++) {
                    if (!act[r]) continue;
                    err[r] = std::sqrt(h_norm[r]);
                    if (err[r] < c->p.outer_tol * normb[r]) {
                        iters[r] = k * m + maxit[r];
                        act[r] = 0;
                    }
                }
                k++;
                return begin_cycle();
            default:
                return AMG_OK;
        }
    }
};

int outer_fgmres(amg_context* c, const double2* b, double2* x, int R, amg_solve_info* info) {
    OuterSolve s;
    CKR(s.init(c, b, x, R, info));
    while (s.phase != OuterSolve::DONE) {
        CK(cudaEventSynchronize(c->ev_host));
        CKR(s.advance());
    }
    return s.rc;
}

int ensure_capacity(amg_context* c, int R) {
    if (R <= c->Rcap && c->V.p) return AMG_OK;
    c->drop_graphs();
    const int Rn = std::max(R, c->Rcap);
    const long long len = vlen0(c);
    const int m = c->p.outer_m;
    CKR(c->V.alloc((size_t)(m + 1) * Rn * len * sizeof(double2)));
    CKR(c->Z.alloc((size_t)m * Rn * len * sizeof(double2)));
    CKR(c->w.alloc((size_t)Rn * len * sizeof(double2)));
    CKR(c->x.alloc((size_t)Rn * len * sizeof(double2)));
    CKR(c->b.alloc((size_t)Rn * len * sizeof(double2)));
    const size_t np = 592;
    CKR(c->partial.alloc(np * Rn * 24 * sizeof(double2)));
    CKR(c->dots.alloc((size_t)Rn * 3 * 24 * sizeof(double2)));
    CKR(c->scal.alloc((size_t)Rn * sizeof(double)));
    CKR(c->masks.alloc((size_t)7 * Rn * sizeof(int)));
    CKR(c->etab.alloc((size_t)Rn * m * sizeof(double2)));
    CKR(c->sap_flags.alloc((size_t)2 * Rn * sizeof(int)));
    CKR(c->norms.alloc((size_t)2 * Rn * sizeof(double)));
    CKR(c->hpin.alloc((size_t)Rn * (2 * sizeof(double) + (2 * m + 3) * sizeof(double2) + 4 * sizeof(int) +
                                     sizeof(double) + m * sizeof(double2)) + 8 * 16));
    {
        void* d = nullptr;
        c->hpin_dev = cudaHostGetDevicePointer(&d, c->hpin.p, 0) == cudaSuccess ? static_cast<char*>(d) : nullptr;
        cudaGetLastError();
    }
    c->Rcap = Rn;
    CKR(alloc_fine<double>(c, c->d, Rn));
    if (c->p.precision == AMG_PREC_F64) {
        CKR(c->vd.alloc((size_t)Rn * len * sizeof(double2)));
        CKR(c->zd.alloc((size_t)Rn * len * sizeof(double2)));
    }
    if (c->p.precision == AMG_PREC_MIXED) {
        c->vf_src = nullptr;
        CKR(c->vf.alloc((size_t)Rn * len * sizeof(float2)));
        CKR(c->zf.alloc((size_t)Rn * len * sizeof(float2)));
        CKR(alloc_fine<float>(c, c->f, Rn));
    }
    return AMG_OK;
}

// ---------------------------------------------------------------------------------
// set-up (AlgebraicMG::setUpPhase, src/amg.cpp:3-88)
// ---------------------------------------------------------------------------------
struct Draw {
    // The reference draws `distribution(randomInt) + I_number * distribution(randomInt)` with
    // std::mt19937(50) and uniform(-1, 1) (src/amg.cpp:8-16); g++ evaluates the imaginary
    // operand first, which this generator reproduces.  A non-zero seed selects a 64-bit
    // Mersenne twister instead.
    std::mt19937 g32;
    std::mt19937_64 g64;
    bool use64;
    std::uniform_real_distribution<double> dist{-1.0, 1.0};
    explicit Draw(unsigned long long seed) : g32(50), g64(seed), use64(seed != 0) {}
    double next() { return use64 ? dist(g64) : dist(g32); }
    void fill(std::vector<double2>& v) {
        for (auto& z : v) {
            const double im = next();
            const double re = next();
            z = make_double2(re, im);
        }
    }
};

int coarse_links(amg_context* c, int l) {
    const LevelHost& h = c->lv[l];
    const int nblk = h.bx * h.bt, spb = h.xe * h.te;
    const int nchunk = std::max(1, std::min(std::max(1, spb / 64), (592 + nblk - 1) / nblk));
    const int Kc = 2 * h.ntest;
    CKR(c->linkpart.alloc((size_t)nblk * nchunk * 5 * Kc * Kc * sizeof(double2)));
    const double2* hops = l == 0 ? c->hops0.as<double2>() : c->d.links[l].as<double2>();
    const double2* W = l == 0 ? c->d.W0.as<double2>() : c->d.W[l].as<double2>();
    launch_coarse_links<double>(W, hops, c->d.links[l + 1].as<double2>(), h.nx, h.nt, h.K, h.bx, h.bt, h.ntest,
                                c->linkpart.as<double2>(), nchunk, c->stream);
    CKL();
    return AMG_OK;
}

int orthonormalize(amg_context* c, int l) {
    const LevelHost& h = c->lv[l];
    double2* W = l == 0 ? c->d.W0.as<double2>() : c->d.W[l].as<double2>();
    launch_orthonormalize<double>(W, h.nx, h.nt, h.K, h.bx, h.bt, h.ntest, c->stream);
    CKL();
    return AMG_OK;
}

int build_mixed(amg_context* c) {
    PrecSet<float>& f = c->f;
    const long long len = vlen0(c);
    // fine links: FP32, or BF16 / FP16 pairs (amg_params.link_storage)
    if (c->p.link_storage == AMG_LINKS_BF16) {
        CKR(f.U.alloc((size_t)len * sizeof(__nv_bfloat162)));
        launch_d2bf(f.U.as<__nv_bfloat162>(), c->d.U.as<double2>(), len, c->stream);
    } else if (c->p.link_storage == AMG_LINKS_F16) {
        CKR(f.U.alloc((size_t)len * sizeof(__half2)));
        launch_d2h(f.U.as<__half2>(), c->d.U.as<double2>(), len, c->stream);
    } else {
        CKR(f.U.alloc((size_t)len * sizeof(float2)));
        launch_d2f(f.U.as<float2>(), c->d.U.as<double2>(), len, c->stream);
    }
    const LevelHost& h0 = c->lv[0];
    CKR(f.W0.alloc((size_t)h0.ntest * len * sizeof(__nv_bfloat162)));
    launch_d2bf(f.W0.as<__nv_bfloat162>(), c->d.W0.as<double2>(), h0.ntest * len, c->stream);
    f.w0_bf16 = 1;
    f.W.resize(c->L);
    f.links.resize(c->L);
    for (int l = 1; l < c->L; l++) {
        const LevelHost& h = c->lv[l];
        const long long nl = (long long)h.n * 5 * h.K * h.K;
        CKR(f.links[l].alloc((size_t)nl * sizeof(float2)));
        launch_d2f(f.links[l].as<float2>(), c->d.links[l].as<double2>(), nl, c->stream);
        if (!h.coarsest) {
            const long long nw = (long long)h.ntest * h.n * h.K;
            CKR(f.W[l].alloc((size_t)nw * sizeof(float2)));
            launch_d2f(f.W[l].as<float2>(), c->d.W[l].as<double2>(), nw, c->stream);
        }
    }
    CKR(build_engine<float>(c, f, c->d.eng_cap));
    CKR(alloc_fine<float>(c, f, c->Rcap));
    c->vf_src = nullptr;
    CKR(c->vf.alloc((size_t)c->Rcap * len * sizeof(float2)));
    CKR(c->zf.alloc((size_t)c->Rcap * len * sizeof(float2)));
    f.ready = 1;
    CKL();
    return AMG_OK;
}

// Device time of the set-up's phases: events recorded on the context's stream at each phase
// boundary; the time from one mark to the next is charged to the phase that just ended.
struct SetupClock {
    amg_context* c;
    std::vector<std::pair<int, cudaEvent_t>> marks;   // (phase ended at this mark, event)
    explicit SetupClock(amg_context* c_) : c(c_) {}
    ~SetupClock() { for (auto& m : marks) cudaEventDestroy(m.second); }
    void mark(int phase) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
        cudaEventRecord(e, c->stream);
        marks.emplace_back(phase, e);
    }
    void harvest() {
        for (double& v : c->setup_phase_ms) v = 0;
        if (marks.empty() || cudaEventSynchronize(marks.back().second) != cudaSuccess) return;
        for (size_t i = 1; i < marks.size(); i++) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second) == cudaSuccess)
                c->setup_phase_ms[marks[i].first] += ms;
        }
    }
};

int do_setup(amg_context* c) {
    SetupClock clk(c);
    clk.mark(AMG_SETUP_INIT);
    c->drop_graphs();
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "set the gauge field before the set-up");
    const amg_params& p = c->p;
    const int L = c->L;
    int cap = c->Rcap;
    for (int l = 0; l < L - 1; l++) cap = std::max(cap, c->lv[l].ntest);
    CKR(ensure_capacity(c, cap));
    CKR(build_engine<double>(c, c->d, cap));
    const long long len = vlen0(c);
    long long zlen = len;
    for (int l = 1; l < L; l++) zlen = std::max<long long>(zlen, (long long)c->lv[l].n * c->lv[l].K);
    CKR(c->zero.alloc((size_t)zlen * sizeof(double2)));
    CK(cudaMemsetAsync(c->zero.p, 0, (size_t)zlen * sizeof(double2), c->stream));

    // initial test vectors (src/amg.cpp:8-35)
    Draw rng(p.tv_seed);
    const LevelHost& h0 = c->lv[0];
    if (!c->have_init[0]) {
        std::vector<double2> host((size_t)h0.ntest * len);
        rng.fill(host);
        CK(cudaMemcpyAsync(c->d.W0.p, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    for (int l = 1; l < L - 1; l++) {
        if (c->have_init[l]) continue;
        const LevelHost& h = c->lv[l];
        const LevelHost& hp = c->lv[l - 1];
        const long long nv = (long long)h.n * h.K;
        double2* W = c->d.W[l].as<double2>();
        for (int i = 0; i < h.ntest; i++) {
            if (i < hp.ntest) {
                if (l == 1) {
                    fine_restrict<double>(c, c->d, c->d.W0.as<double2>() + (long long)i * len, W + i * nv, 1);
                } else {
                    const long long nvp = (long long)hp.n * hp.K;
                    CKR(run_engine<double>(c, c->d, ENG_RESTRICT, l - 1, 0, c->d.W[l - 1].as<double2>() + i * nvp, 0,
                                           W + i * nv, 0, 1));
                }
            } else {
                std::vector<double2> host((size_t)nv);
                rng.fill(host);
                CK(cudaMemcpyAsync(W + i * nv, host.data(), nv * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
        }
    }
    CKR(c->hops0.alloc((size_t)c->N * 20 * sizeof(double2)));
    launch_fine_hops<double>(c->d.U.as<double2>(), c->hops0.as<double2>(), c->nx, c->nt, c->stream);
    clk.mark(AMG_SETUP_INIT);
    // smoothing, orthonormalisation and coarse links, level by level
    for (int l = 0; l < L - 1; l++) {
        const LevelHost& h = c->lv[l];
        if (p.sap_tv_iters > 0) {
            if (l == 0) {
                CKR(fine_sap<double>(c, c->d, c->zero.as<double2>(), 0, c->d.W0.as<double2>(), p.sap_tv_iters,
                                     h.ntest, 0));
            } else {
                const long long nv = (long long)h.n * h.K;
                CKR(run_engine<double>(c, c->d, ENG_SAP, l, p.sap_tv_iters, c->zero.as<double2>(), 0,
                                       c->d.W[l].as<double2>(), nv, h.ntest));
            }
        }
        clk.mark(AMG_SETUP_SMOOTH);
        CKR(orthonormalize(c, l));
        clk.mark(AMG_SETUP_ORTHO);
        CKR(coarse_links(c, l));
        clk.mark(AMG_SETUP_LINKS);
    }
    // bootstrap passes (src/amg.cpp:52-84)
    for (int it = 0; it < p.nit; it++) {
        for (int l = 0; l < L - 1; l++) {
            const LevelHost& h = c->lv[l];
            const long long nv = (long long)h.n * h.K;
            const long long tot = nv * h.ntest;
            CKR(c->boot_a.alloc((size_t)tot * sizeof(double2)));
            CKR(c->boot_b.alloc((size_t)tot * sizeof(double2)));
            double2* rhs = c->boot_a.as<double2>();
            double2* z = c->boot_b.as<double2>();
            double2* W = l == 0 ? c->d.W0.as<double2>() : c->d.W[l].as<double2>();
            if (l == 0) {
                launch_dirac<double>(c->d.U.as<double2>(), W, rhs, c->nx, c->nt, h.ntest, c->m0, 0, c->stream);
            } else {
                CKR(run_engine<double>(c, c->d, ENG_APPLY, l, 0, W, nv, rhs, nv, h.ntest));
            }
            k_sub_d<<<592, 256, 0, c->stream>>>(rhs, W, rhs, tot);
            CK(cudaMemsetAsync(z, 0, (size_t)tot * sizeof(double2), c->stream));
            if (l == 0) {
                CKR(fine_cycle<double>(c, c->d, rhs, z, h.ntest, true));
            } else {
                CKR(run_engine<double>(c, c->d, p.cycle == AMG_CYCLE_K ? ENG_KCYCLE : ENG_VCYCLE, l, 0, rhs, nv, z,
                                       nv, h.ntest));
            }
            k_add_d<<<592, 256, 0, c->stream>>>(W, z, tot);
            CKR(orthonormalize(c, l));
            CKR(coarse_links(c, l));
        }
    }
    clk.mark(AMG_SETUP_BOOT);
    CK(cudaStreamSynchronize(c->stream));
    int flags = 0;
    CK(cudaMemcpy(&flags, c->d.eh.flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) return fail(AMG_ERR_UNSUPPORTED, "engine reported flags %d", flags);
    c->f.ready = 0;
    if (p.precision == AMG_PREC_MIXED) CKR(build_mixed(c));
    clk.mark(AMG_SETUP_MIXED);
    c->setup_done = 1;
    CK(cudaStreamSynchronize(c->stream));
    clk.harvest();
    return AMG_OK;
}

// copy helpers for the single-source probes
int to_dev(DevBuf& b, const double* h, long long ncplx, cudaStream_t s) {
    CKR(b.alloc((size_t)ncplx * sizeof(double2)));
    if (h) CK(cudaMemcpyAsync(b.p, h, (size_t)ncplx * sizeof(double2), cudaMemcpyHostToDevice, s));
    return AMG_OK;
}
int to_host(double* h, const DevBuf& b, long long ncplx, cudaStream_t s) {
    CK(cudaMemcpyAsync(h, b.p, (size_t)ncplx * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return AMG_OK;
}

int check_ready(amg_ctx c, int level, bool need_setup) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    if (level < 0 || level >= c->L) return fail(AMG_ERR_INVALID, "level %d out of range", level);
    if (need_setup && !c->setup_done) return fail(AMG_ERR_STATE, "set-up not done");
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "gauge field not set");
    return AMG_OK;
}

int select_device(amg_ctx c) {
    CK(cudaSetDevice(c->device));
    return AMG_OK;
}

}  // namespace

// =================================================================================
// C ABI
// =================================================================================
extern "C" {

const char* amg_status_string(int s) {
    switch (s) {
        case AMG_OK: return "ok";
        case AMG_NOT_CONVERGED: return "not converged";
        case AMG_ERR_INVALID: return "invalid argument";
        case AMG_ERR_CUDA: return "CUDA error";
        case AMG_ERR_STATE: return "wrong call order";
        case AMG_ERR_NOMEM: return "out of device memory";
        case AMG_ERR_DEVICE_WAIT: return "device-side wait gave up";
        case AMG_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}
const char* amg_last_error(void) { return g_last_error.c_str(); }
int amg_version(void) { return 100; }

void amg_params_default(amg_params* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->cycle = AMG_CYCLE_K;
    p->nu1 = 0;
    p->nu2 = 2;
    p->nit = 0;
    p->sap_tv_iters = 4;
    p->sap_gmres_m = 5;
    p->sap_gmres_restarts = 5;
    p->sap_gmres_tol = 1e-3;
    p->sap_tol = 1e-10;
    p->kcycle_m = 5;
    p->kcycle_restarts = 2;
    p->kcycle_tol = 0.1;
    p->coarse_m = 20;
    p->coarse_restarts = 20;
    p->coarse_tol = 0.1;
    p->outer_m = 20;
    p->outer_restarts = 50;
    p->outer_tol = 1e-10;
    p->precision = AMG_PREC_F64;
    p->max_rhs = 1;
    p->tv_seed = 0;
    p->autotune = 1;
    p->link_storage = AMG_LINKS_F16;
}

int amg_read_parameters(const char* path, int* rows, int max_rows, int* nrows) {
    if (!path || !rows || !nrows) return fail(AMG_ERR_INVALID, "null argument");
    std::ifstream f(path);
    if (!f) return fail(AMG_ERR_INVALID, "parameters file %s not found", path);
    int v[6], n = 0;
    while (f >> v[0] >> v[1] >> v[2] >> v[3] >> v[4] >> v[5]) {
        if (n >= max_rows) return fail(AMG_ERR_INVALID, "more than %d parameter rows", max_rows);
        for (int k = 0; k < 6; k++) rows[6 * n + k] = v[k];
        n++;
    }
    if (!f.eof()) return fail(AMG_ERR_INVALID, "malformed parameters file %s (6 integers per row)", path);
    *nrows = n;
    return AMG_OK;
}

int amg_create(amg_ctx* out, int nx, int nt, int levels, const int* rows, double m0, const amg_params* params,
               int device) {
    if (!out) return fail(AMG_ERR_INVALID, "null context pointer");
    *out = nullptr;
    amg_params p;
    if (params) p = *params; else amg_params_default(&p);
    if (p.sap_gmres_m < 1 || p.kcycle_m < 1 || p.coarse_m < 1 || p.outer_m < 1 || p.outer_m > 22)
        return fail(AMG_ERR_INVALID, "restart lengths must be >= 1 (outer <= 22)");
    if (p.sap_gmres_restarts < 1 || p.kcycle_restarts < 1 || p.coarse_restarts < 1 || p.outer_restarts < 1)
        return fail(AMG_ERR_INVALID, "restart counts must be >= 1");
    if (p.precision != AMG_PREC_F64 && p.precision != AMG_PREC_MIXED) return fail(AMG_ERR_INVALID, "precision");
    if (p.cycle != AMG_CYCLE_K && p.cycle != AMG_CYCLE_V) return fail(AMG_ERR_INVALID, "cycle");
    if (p.link_storage != AMG_LINKS_F32 && p.link_storage != AMG_LINKS_BF16 && p.link_storage != AMG_LINKS_F16)
        return fail(AMG_ERR_INVALID, "link_storage");
    if (p.max_rhs < 1) p.max_rhs = 1;
    std::vector<LevelHost> lv;
    CKR(build_levels(nx, nt, levels, rows, lv));
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(AMG_ERR_INVALID, "device %d of %d", device, ndev);
    CK(cudaSetDevice(device));
    amg_context* c = new amg_context();
    c->device = device;
    c->p = p;
    c->m0 = m0;
    c->nx = nx; c->nt = nt; c->N = nx * nt; c->L = levels;
    c->lv = lv;
    c->have_init.assign(levels, 0);
    int rc = AMG_OK;
    auto bail = [&](int r) { delete c; return r; };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_host, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(AMG_ERR_CUDA, "stream/event creation failed"));
    const long long len = vlen0(c);
    if ((rc = c->d.U.alloc((size_t)len * sizeof(double2))) < 0) return bail(rc);
    if ((rc = c->d.W0.alloc((size_t)lv[0].ntest * len * sizeof(double2))) < 0) return bail(rc);
    c->d.W.resize(levels);
    c->d.links.resize(levels);
    for (int l = 1; l < levels; l++) {
        const LevelHost& h = lv[l];
        if ((rc = c->d.links[l].alloc((size_t)h.n * 5 * h.K * h.K * sizeof(double2))) < 0) return bail(rc);
        if (!h.coarsest && (rc = c->d.W[l].alloc((size_t)h.ntest * h.n * h.K * sizeof(double2))) < 0) return bail(rc);
    }
    if ((rc = ensure_capacity(c, p.max_rhs)) < 0) return bail(rc);
    *out = c;
    return AMG_OK;
}

int amg_destroy(amg_ctx c) {
    if (!c) return AMG_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev_host) cudaEventDestroy(c->ev_host);
    for (int k = 0; k < 2; k++) {
        if (c->ev_in[k]) cudaEventDestroy(c->ev_in[k]);
        if (c->ev_solved[k]) cudaEventDestroy(c->ev_solved[k]);
        if (c->ev_out[k]) cudaEventDestroy(c->ev_out[k]);
        if (c->ev_piece[k]) cudaEventDestroy(c->ev_piece[k]);
    }
    cudaStream_t s = c->stream, cs = c->copy_stream;
    delete c;
    if (s) cudaStreamDestroy(s);
    if (cs) cudaStreamDestroy(cs);
    return AMG_OK;
}

int amg_get_params(amg_ctx c, amg_params* out) {
    if (!c || !out) return fail(AMG_ERR_INVALID, "null argument");
    *out = c->p;
    return AMG_OK;
}

int amg_set_mass(amg_ctx c, double m0) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    c->m0 = m0;
    c->setup_done = 0;
    c->drop_graphs();
    return AMG_OK;
}

int amg_set_cycle(amg_ctx c, int cycle) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    if (cycle != AMG_CYCLE_K && cycle != AMG_CYCLE_V) return fail(AMG_ERR_INVALID, "cycle must be AMG_CYCLE_K or AMG_CYCLE_V");
    c->p.cycle = cycle;
    c->drop_graphs();
    return AMG_OK;
}

int amg_set_preconditioner(amg_ctx c, int kind) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    if (kind != AMG_PRECOND_MG && kind != AMG_PRECOND_SAP && kind != AMG_PRECOND_NONE)
        return fail(AMG_ERR_INVALID, "preconditioner must be AMG_PRECOND_MG, AMG_PRECOND_SAP or AMG_PRECOND_NONE");
    c->precond = kind;
    c->drop_graphs();
    return AMG_OK;
}

int amg_level_info(amg_ctx c, int level, int* o) {
    if (!c || !o) return fail(AMG_ERR_INVALID, "null argument");
    if (level < 0 || level >= c->L) return fail(AMG_ERR_INVALID, "level %d out of range", level);
    const LevelHost& h = c->lv[level];
    o[0] = h.n; o[1] = h.nx; o[2] = h.nt; o[3] = h.K; o[4] = h.colors; o[5] = h.coarsest ? 0 : h.ntest;
    return AMG_OK;
}

int amg_set_gauge(amg_ctx c, const double* U) {
    if (!c || !U) return fail(AMG_ERR_INVALID, "null argument");
    CKR(select_device(c));
    CK(cudaMemcpyAsync(c->d.U.p, U, (size_t)vlen0(c) * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->gauge_set = 1;
    c->setup_done = 0;
    c->drop_graphs();
    return AMG_OK;
}

int amg_dirac_apply_dev(amg_ctx c, const void* in, void* out, int nrhs, int dagger) {
    if (!c || !in || !out || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "gauge field not set");
    CKR(select_device(c));
    launch_dirac<double>(c->d.U.as<double2>(), (const double2*)in, (double2*)out, c->nx, c->nt, nrhs, c->m0,
                         dagger ? 1 : 0, c->stream);
    CKL();
    CK(cudaStreamSynchronize(c->stream));
    return check_fine_waits(c->stream);
}

// ---------------------------------------------------------------------------------
// Comparison solvers on the fine stencil (FP64, one source): conjugate_gradient
// (src/conjugate_gradient.cpp:5-65) on D D^dagger and bi_cgstab (src/bi_cgstab.cpp:5-89),
// each a host loop over device kernels; every vector update evaluates the reference's
// expression in its order, and every dot is the reference's dot(x, y) = sum x conj(y).
// ---------------------------------------------------------------------------------
namespace {
// y += a x
__global__ void k_cs_xpay(double2* __restrict__ y, const double2* __restrict__ x, double2 a, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = y[e] + cmul(a, x[e]);
}
// y = r - a q
__global__ void k_cs_rmaq(double2* __restrict__ y, const double2* __restrict__ r, const double2* __restrict__ q,
                          double2 a, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = r[e] - cmul(a, q[e]);
}
// d = d beta + r (CG)
__global__ void k_cs_dbr(double2* __restrict__ d, const double2* __restrict__ r, double2 beta, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] = cmul(d[e], beta) + r[e];
}
// d = r + beta (d - omega Ad) (BiCGStab)
__global__ void k_cs_bicg_d(double2* __restrict__ d, const double2* __restrict__ r, const double2* __restrict__ Ad,
                            double2 beta, double2 omega, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] = r[e] + cmul(beta, d[e] - cmul(omega, Ad[e]));
}
// x = x + alpha d + omega s (BiCGStab)
__global__ void k_cs_x3(double2* __restrict__ x, const double2* __restrict__ d, const double2* __restrict__ s,
                        double2 alpha, double2 omega, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        x[e] = x[e] + cmul(alpha, d[e]) + cmul(omega, s[e]);
}

struct FineKrylov {
    amg_context* c;
    long long n;          // complex entries of one fine vector
    int np;
    DevBuf part, out;
    std::complex<double> hdot[2];
    int init(amg_context* c_) {
        c = c_;
        n = vlen0(c);
        np = (int)std::min<long long>(592, (n + 255) / 256);
        CKR(part.alloc((size_t)np * 2 * sizeof(double2)));
        CKR(out.alloc(2 * sizeof(double2)));
        return AMG_OK;
    }
    dim3 grid() const { return dim3((unsigned)std::min<long long>(592, (n + 255) / 256)); }
    // dot(a, b) = sum a conj(b) (include/lin_alg_op.h:32-40)
    int dot(const double2* a, const double2* b, std::complex<double>& r) {
        launch_axpy_multidot(const_cast<double2*>(a), b, n, n, 0, nullptr, 0, 1, nullptr, 1, part.as<double2>(), np,
                             out.as<double2>(), c->stream);
        CK(cudaMemcpyAsync(hdot, out.p, 2 * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        r = hdot[0];
        return AMG_OK;
    }
    void dirac(const double2* in, double2* o, int dagger) {
        launch_dirac<double>(c->d.U.as<double2>(), in, o, c->nx, c->nt, 1, c->m0, dagger, c->stream);
    }
};
inline double2 d2(std::complex<double> z) { return make_double2(z.real(), z.imag()); }
}  // namespace

int amg_cg_normal(amg_ctx c, const double* phi, double* x, int max_iter, double tol, int* iterations) {
    CKR(check_ready(c, 0, false));
    if (!phi || !x || max_iter < 0 || !(tol > 0)) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    FineKrylov K;
    CKR(K.init(c));
    const long long n = K.n;
    DevBuf P, X, R, D, AD, T;
    CKR(to_dev(P, phi, n, c->stream));
    CKR(to_dev(X, phi, n, c->stream));   // x = phi
    CKR(to_dev(R, nullptr, n, c->stream));
    CKR(to_dev(D, nullptr, n, c->stream));
    CKR(to_dev(AD, nullptr, n, c->stream));
    CKR(to_dev(T, nullptr, n, c->stream));
    double2 *p = P.as<double2>(), *xv = X.as<double2>(), *r = R.as<double2>(), *d = D.as<double2>(),
            *ad = AD.as<double2>(), *t = T.as<double2>();
    const dim3 g = K.grid();
    auto ddag = [&](const double2* in, double2* o) {   // D_D_dagger_phi (src/dirac_operator.cpp:57-61)
        K.dirac(in, t, 1);
        K.dirac(t, o, 0);
    };
    ddag(xv, ad);
    k_cs_rmaq<<<g, 256, 0, c->stream>>>(r, p, ad, make_double2(1.0, 0.0), n);
    CK(cudaMemcpyAsync(d, r, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    std::complex<double> r_norm2, pp, dad, rr;
    CKR(K.dot(r, r, r_norm2));
    CKR(K.dot(p, p, pp));
    const double phi_norm = std::sqrt(pp.real());
    int k = 0, conv = 0;
    while (k < max_iter) {
        ddag(d, ad);
        CKR(K.dot(d, ad, dad));
        const std::complex<double> alpha = r_norm2 / dad;
        k_cs_xpay<<<g, 256, 0, c->stream>>>(xv, d, d2(alpha), n);
        k_cs_xpay<<<g, 256, 0, c->stream>>>(r, ad, d2(-alpha), n);
        CKR(K.dot(r, r, rr));
        const double err_sqr = rr.real();
        if (std::sqrt(err_sqr) < tol * phi_norm) {
            conv = 1;
            break;
        }
        const std::complex<double> beta = err_sqr / r_norm2;
        k_cs_dbr<<<g, 256, 0, c->stream>>>(d, r, d2(beta), n);
        r_norm2 = err_sqr;
        k++;
    }
    CKL();
    CKR(to_host(x, X, n, c->stream));
    if (iterations) *iterations = k;
    CKR(check_fine_waits(c->stream));
    return conv ? AMG_OK : AMG_NOT_CONVERGED;
}

int amg_bicgstab(amg_ctx c, const double* phi, const double* x0, double* x, int max_iter, double tol,
                 int* iterations) {
    CKR(check_ready(c, 0, false));
    if (!phi || !x || max_iter < 0 || !(tol > 0)) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    FineKrylov K;
    CKR(K.init(c));
    const long long n = K.n;
    DevBuf P, X, R, RT, D, S, T, AD;
    CKR(to_dev(P, phi, n, c->stream));
    CKR(to_dev(X, x0, n, c->stream));
    if (!x0) CK(cudaMemsetAsync(X.p, 0, (size_t)n * sizeof(double2), c->stream));
    CKR(to_dev(R, nullptr, n, c->stream));
    CKR(to_dev(RT, nullptr, n, c->stream));
    CKR(to_dev(D, nullptr, n, c->stream));
    CKR(to_dev(S, nullptr, n, c->stream));
    CKR(to_dev(T, nullptr, n, c->stream));
    CKR(to_dev(AD, nullptr, n, c->stream));
    double2 *p = P.as<double2>(), *xv = X.as<double2>(), *r = R.as<double2>(), *rt = RT.as<double2>(),
            *d = D.as<double2>(), *sv = S.as<double2>(), *t = T.as<double2>(), *ad = AD.as<double2>();
    const dim3 g = K.grid();
    K.dirac(xv, ad, 0);
    k_cs_rmaq<<<g, 256, 0, c->stream>>>(r, p, ad, make_double2(1.0, 0.0), n);   // r = b - A x
    CK(cudaMemcpyAsync(rt, r, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    std::complex<double> pp, rho_i, rho_i_2, alpha, beta, omega, tmp, st, tt, ss;
    CKR(K.dot(p, p, pp));
    const double norm_phi = std::sqrt(pp.real());
    int k = 0, conv = 0;
    while (k < max_iter) {
        CKR(K.dot(r, rt, rho_i));
        if (k == 0) {
            CK(cudaMemcpyAsync(d, r, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        } else {
            beta = alpha * rho_i / (omega * rho_i_2);
            k_cs_bicg_d<<<g, 256, 0, c->stream>>>(d, r, ad, d2(beta), d2(omega), n);
        }
        K.dirac(d, ad, 0);
        CKR(K.dot(ad, rt, tmp));
        alpha = rho_i / tmp;
        k_cs_rmaq<<<g, 256, 0, c->stream>>>(sv, r, ad, d2(alpha), n);
        CKR(K.dot(sv, sv, ss));
        if (std::sqrt(ss.real()) < tol * norm_phi) {
            k_cs_xpay<<<g, 256, 0, c->stream>>>(xv, d, d2(alpha), n);
            conv = 1;
            k++;
            break;
        }
        K.dirac(sv, t, 0);
        CKR(K.dot(sv, t, st));
        CKR(K.dot(t, t, tt));
        omega = st / tt;
        k_cs_rmaq<<<g, 256, 0, c->stream>>>(r, sv, t, d2(omega), n);
        k_cs_x3<<<g, 256, 0, c->stream>>>(xv, d, sv, d2(alpha), d2(omega), n);
        rho_i_2 = rho_i;
        k++;
    }
    CKL();
    CKR(to_host(x, X, n, c->stream));
    if (iterations) *iterations = k;
    CKR(check_fine_waits(c->stream));
    return conv ? AMG_OK : AMG_NOT_CONVERGED;
}

int amg_dirac_apply(amg_ctx c, const double* in, double* out, int nrhs, int dagger) {
    if (!c || !in || !out || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "gauge field not set");
    CKR(select_device(c));
    DevBuf a, b;
    const long long n = (long long)nrhs * vlen0(c);
    CKR(to_dev(a, in, n, c->stream));
    CKR(to_dev(b, nullptr, n, c->stream));
    launch_dirac<double>(c->d.U.as<double2>(), a.as<double2>(), b.as<double2>(), c->nx, c->nt, nrhs, c->m0,
                         dagger ? 1 : 0, c->stream);
    CKL();
    CKR(to_host(out, b, n, c->stream));
    return check_fine_waits(c->stream);
}

int amg_dirac_apply_raw(const void* U_dev, const void* in_dev, void* out_dev, int nx, int nt, int nrhs, double m0,
                        int dagger, void* stream) {
    if (!U_dev || !in_dev || !out_dev || nx < 2 || nt < 2 || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    launch_dirac<double>((const double2*)U_dev, (const double2*)in_dev, (double2*)out_dev, nx, nt, nrhs, m0,
                         dagger ? 1 : 0, (cudaStream_t)stream);
    CKL();
    return AMG_OK;
}

int amg_debug_dirac_wait_test(const void* U_dev, const void* in_dev, void* out_dev, int nx, int nt, int nrhs) {
    if (!U_dev || !in_dev || !out_dev || nx < 2 || nt < 2 || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    const int r = dirac_tma_wait_test((const double2*)U_dev, (const double2*)in_dev, (double2*)out_dev, nx, nt, nrhs,
                                      0);
    if (r < 0) return fail(AMG_ERR_INVALID, "lattice or buffers outside the bulk-copy kernel, or a CUDA error: %s",
                           cudaGetErrorString(cudaGetLastError()));
    if (r > 0) return fail(AMG_ERR_DEVICE_WAIT, "a bulk-copy wait of the Dirac apply gave up (self-test)");
    return AMG_OK;
}

int amg_dirac_apply_host(const double* U, const double* in, double* out, int nx, int nt, int nrhs, double m0,
                         int dagger) {
    if (!U || !in || !out || nx < 2 || nt < 2 || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    const long long N = (long long)nx * nt;
    DevBuf u, a, b;
    CKR(to_dev(u, U, 2 * N, 0));
    CKR(to_dev(a, in, 2 * N * nrhs, 0));
    CKR(to_dev(b, nullptr, 2 * N * nrhs, 0));
    launch_dirac<double>(u.as<double2>(), a.as<double2>(), b.as<double2>(), nx, nt, nrhs, m0, dagger ? 1 : 0, 0);
    CKL();
    CKR(to_host(out, b, 2 * N * nrhs, 0));
    return check_fine_waits(0);
}

int amg_set_initial_test_vectors(amg_ctx c, int level, const double* W) {
    if (!c || !W) return fail(AMG_ERR_INVALID, "null argument");
    if (level < 0 || level >= c->L - 1) return fail(AMG_ERR_INVALID, "level %d has no test vectors", level);
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const size_t bytes = (size_t)h.ntest * h.n * h.K * sizeof(double2);
    void* dst = level == 0 ? c->d.W0.p : c->d.W[level].p;
    CK(cudaMemcpyAsync(dst, W, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->have_init[level] = 1;
    c->setup_done = 0;
    return AMG_OK;
}

int amg_setup(amg_ctx c) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    CKR(select_device(c));
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = do_setup(c);
    if (rc < 0) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_setup_ms = ms;
    // imported initial vectors are consumed by one set-up
    std::fill(c->have_init.begin(), c->have_init.end(), 0);
    return AMG_OK;
}

int amg_get_test_vectors(amg_ctx c, int level, double* W) {
    CKR(check_ready(c, level, true));
    if (level >= c->L - 1) return fail(AMG_ERR_INVALID, "level %d has no test vectors", level);
    const LevelHost& h = c->lv[level];
    const void* src = level == 0 ? c->d.W0.p : c->d.W[level].p;
    CK(cudaMemcpyAsync(W, src, (size_t)h.ntest * h.n * h.K * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return AMG_OK;
}

int amg_get_coarse_links(amg_ctx c, int level, double* G1, double* G2, double* G3) {
    CKR(check_ready(c, level, true));
    if (level < 1) return fail(AMG_ERR_INVALID, "coarse links exist for levels >= 1");
    const LevelHost& h = c->lv[level];
    const int K = h.K, col = h.colors;
    std::vector<double2> lk((size_t)h.n * 5 * K * K);
    CK(cudaMemcpyAsync(lk.data(), c->d.links[level].p, lk.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // links[x][h][j = 2b+bet][i = 2c+alf] -> G1[x][alf][bet][c][b], G2/G3[x][alf][bet][c][b][mu]
    for (int x = 0; x < h.n; x++)
        for (int alf = 0; alf < 2; alf++)
            for (int bet = 0; bet < 2; bet++)
                for (int cc = 0; cc < col; cc++)
                    for (int bb = 0; bb < col; bb++) {
                        const int i = 2 * cc + alf, j = 2 * bb + bet;
                        auto at = [&](int hop) { return lk[(((size_t)x * 5 + hop) * K + j) * K + i]; };
                        const size_t g1 = (((((size_t)x * 2 + alf) * 2 + bet) * col + cc) * col + bb);
                        if (G1) { G1[2 * g1] = at(0).x; G1[2 * g1 + 1] = at(0).y; }
                        for (int mu = 0; mu < 2; mu++) {
                            const size_t g2 = g1 * 2 + mu;
                            if (G2) { G2[2 * g2] = at(1 + mu).x; G2[2 * g2 + 1] = at(1 + mu).y; }
                            if (G3) { G3[2 * g2] = at(3 + mu).x; G3[2 * g2 + 1] = at(3 + mu).y; }
                        }
                    }
    return AMG_OK;
}

int amg_level_apply(amg_ctx c, int level, const double* in, double* out) {
    CKR(check_ready(c, level, level > 0));
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const long long nv = (long long)h.n * h.K;
    DevBuf a, b;
    CKR(to_dev(a, in, nv, c->stream));
    CKR(to_dev(b, nullptr, nv, c->stream));
    if (level == 0)
        launch_dirac<double>(c->d.U.as<double2>(), a.as<double2>(), b.as<double2>(), c->nx, c->nt, 1, c->m0, 0,
                             c->stream);
    else
        CKR(run_engine<double>(c, c->d, ENG_APPLY, level, 0, a.as<double2>(), 0, b.as<double2>(), 0, 1));
    CKL();
    return to_host(out, b, nv, c->stream);
}

int amg_restrict(amg_ctx c, int level, const double* in, double* out) {
    CKR(check_ready(c, level, true));
    if (level >= c->L - 1) return fail(AMG_ERR_INVALID, "no coarser level below %d", level);
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const LevelHost& hn = c->lv[level + 1];
    DevBuf a, b;
    CKR(to_dev(a, in, (long long)h.n * h.K, c->stream));
    CKR(to_dev(b, nullptr, (long long)hn.n * hn.K, c->stream));
    if (level == 0) fine_restrict<double>(c, c->d, a.as<double2>(), b.as<double2>(), 1);
    else CKR(run_engine<double>(c, c->d, ENG_RESTRICT, level, 0, a.as<double2>(), 0, b.as<double2>(), 0, 1));
    CKL();
    return to_host(out, b, (long long)hn.n * hn.K, c->stream);
}

int amg_prolong(amg_ctx c, int level, const double* in, double* out) {
    CKR(check_ready(c, level, true));
    if (level >= c->L - 1) return fail(AMG_ERR_INVALID, "no coarser level below %d", level);
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const LevelHost& hn = c->lv[level + 1];
    DevBuf a, b;
    CKR(to_dev(a, in, (long long)hn.n * hn.K, c->stream));
    CKR(to_dev(b, nullptr, (long long)h.n * h.K, c->stream));
    if (level == 0) {
        CK(cudaMemsetAsync(b.p, 0, (size_t)h.n * h.K * sizeof(double2), c->stream));
        fine_prolong_add<double>(c, c->d, a.as<double2>(), b.as<double2>(), 1);
    } else {
        CKR(run_engine<double>(c, c->d, ENG_PROLONG, level, 0, a.as<double2>(), 0, b.as<double2>(), 0, 1));
    }
    CKL();
    return to_host(out, b, (long long)h.n * h.K, c->stream);
}

// The mixed form's level-0 transfers on device buffers (complex64), the kernels its cycles run
static int transfer0_mixed(amg_ctx c, int op, const void* in_dev, void* out_dev, int nrhs) {
    CKR(check_ready(c, 0, true));
    if (c->p.precision != AMG_PREC_MIXED) return fail(AMG_ERR_STATE, "the context is not in the mixed form");
    if (c->L < 2) return fail(AMG_ERR_INVALID, "one level: no transfer");
    if (nrhs < 1) return fail(AMG_ERR_INVALID, "nrhs < 1");
    if (!in_dev || !out_dev) return fail(AMG_ERR_INVALID, "null device pointer");
    CKR(select_device(c));
    // only the mixed set's fine buffers (grow-only; captured cycles are dropped first when
    // they might move)
    if (nrhs > c->Rcap) c->drop_graphs();
    CKR(alloc_fine<float>(c, c->f, nrhs));
    if (op == 0)
        fine_restrict<float>(c, c->f, static_cast<const float2*>(in_dev), static_cast<float2*>(out_dev), nrhs);
    else
        fine_prolong_add<float>(c, c->f, static_cast<const float2*>(in_dev), static_cast<float2*>(out_dev), nrhs);
    CKL();
    const int e = fine_error_check(c->stream);
    if (e < 0) return fail(AMG_ERR_CUDA, "transfer: %s", cudaGetErrorString(cudaGetLastError()));
    if (e) return fail(AMG_ERR_DEVICE_WAIT, "transfer: a device wait gave up (flag %d)", e);
    return AMG_OK;
}

int amg_restrict0_mixed_dev(amg_ctx c, const void* in_dev, void* out_dev, int nrhs) {
    return transfer0_mixed(c, 0, in_dev, out_dev, nrhs);
}

int amg_prolong0_mixed_dev(amg_ctx c, const void* in_dev, void* out_dev, int nrhs) {
    return transfer0_mixed(c, 1, in_dev, out_dev, nrhs);
}

int amg_sap(amg_ctx c, int level, const double* v, double* x, int nu) {
    CKR(check_ready(c, level, level > 0));
    if (level >= c->L - 1) return fail(AMG_ERR_INVALID, "no SAP on the coarsest level");
    if (nu < 0) return fail(AMG_ERR_INVALID, "nu < 0");
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const long long nv = (long long)h.n * h.K;
    DevBuf a, b;
    CKR(to_dev(a, v, nv, c->stream));
    CKR(to_dev(b, x, nv, c->stream));
    int conv = 0;
    if (level == 0) {
        if (!c->d.eng_args.p) CKR(build_engine<double>(c, c->d, c->Rcap));
        CKR(fine_sap<double>(c, c->d, a.as<double2>(), nv, b.as<double2>(), nu, 1, 1));
        CK(cudaMemcpyAsync(&conv, c->sap_flags.as<int>() + c->Rcap, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    } else {
        CKR(run_engine<double>(c, c->d, ENG_SAP, level, nu, a.as<double2>(), 0, b.as<double2>(), 0, 1));
        CK(cudaMemcpyAsync(&conv, c->d.eh.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    CKR(to_host(x, b, nv, c->stream));
    return conv ? AMG_OK : AMG_NOT_CONVERGED;
}

int amg_level_gmres(amg_ctx c, int level, const double* bh, double* xh, int* iterations) {
    CKR(check_ready(c, level, true));
    if (level < 1) return fail(AMG_ERR_UNSUPPORTED, "level GMRES is provided for levels >= 1");
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const long long nv = (long long)h.n * h.K;
    DevBuf a, b;
    CKR(to_dev(a, bh, nv, c->stream));
    CKR(to_dev(b, nullptr, nv, c->stream));
    CKR(run_engine<double>(c, c->d, ENG_GMRES, level, 0, a.as<double2>(), 0, b.as<double2>(), 0, 1));
    int it = 0;
    CK(cudaMemcpyAsync(&it, c->d.eh.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CKR(to_host(xh, b, nv, c->stream));
    if (iterations) *iterations = it;
    return AMG_OK;
}

int amg_cycle(amg_ctx c, int level, const double* eta, double* psi) {
    CKR(check_ready(c, level, true));
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const long long nv = (long long)h.n * h.K;
    DevBuf a, b;
    CKR(to_dev(a, eta, nv, c->stream));
    CKR(to_dev(b, psi, nv, c->stream));
    if (level == 0) {
        CKR(fine_cycle<double>(c, c->d, a.as<double2>(), b.as<double2>(), 1, false));
    } else {
        CKR(run_engine<double>(c, c->d, c->p.cycle == AMG_CYCLE_K ? ENG_KCYCLE : ENG_VCYCLE, level, 0,
                               a.as<double2>(), 0, b.as<double2>(), 0, 1));
    }
    CKL();
    return to_host(psi, b, nv, c->stream);
}

int amg_kcycle_fgmres(amg_ctx c, int level, const double* bh, double* xh, int* iterations) {
    CKR(check_ready(c, level, true));
    if (level < 1) return fail(AMG_ERR_INVALID, "the K-cycle FGMRES exists for levels >= 1");
    CKR(select_device(c));
    const LevelHost& h = c->lv[level];
    const long long nv = (long long)h.n * h.K;
    DevBuf a, b;
    CKR(to_dev(a, bh, nv, c->stream));
    CKR(to_dev(b, nullptr, nv, c->stream));
    CKR(run_engine<double>(c, c->d, ENG_KFGMRES, level, 0, a.as<double2>(), 0, b.as<double2>(), 0, 1));
    int it = 0;
    CK(cudaMemcpyAsync(&it, c->d.eh.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CKR(to_host(xh, b, nv, c->stream));
    if (iterations) *iterations = it;
    return AMG_OK;
}

int amg_solve_dev(amg_ctx c, const void* b_dev, void* x_dev, int nrhs, amg_solve_info* info) {
    CKR(check_ready(c, 0, true));
    if (!b_dev || !x_dev || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    if (nrhs > c->Rcap) {
        CKR(ensure_capacity(c, nrhs));
        CKR(build_engine<double>(c, c->d, std::max(c->d.eng_cap, nrhs)));
        if (c->p.precision == AMG_PREC_MIXED) CKR(build_engine<float>(c, c->f, std::max(c->f.eng_cap, nrhs)));
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    int rc = outer_fgmres(c, (const double2*)b_dev, (double2*)x_dev, nrhs, info);
    if (rc < 0) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_solve_ms = ms;
    int flags = 0;
    CK(cudaMemcpy(&flags, c->d.eh.flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) return fail(AMG_ERR_UNSUPPORTED, "engine reported flags %d", flags);
    CKR(check_fine_waits(c->stream));
    return rc;
}

int amg_solve(amg_ctx c, const double* b, double* x, int nrhs, amg_solve_info* info) {
    CKR(check_ready(c, 0, true));
    if (!b || !x || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    if (nrhs > c->Rcap) {
        CKR(ensure_capacity(c, nrhs));
        CKR(build_engine<double>(c, c->d, std::max(c->d.eng_cap, nrhs)));
        if (c->p.precision == AMG_PREC_MIXED) CKR(build_engine<float>(c, c->f, std::max(c->f.eng_cap, nrhs)));
    }
    const long long n = (long long)nrhs * vlen0(c);
    CK(cudaMemcpyAsync(c->b.p, b, (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    int rc = amg_solve_dev(c, c->b.p, c->x.p, nrhs, info);
    if (rc < 0) return rc;
    CK(cudaMemcpyAsync(x, c->x.p, (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return rc;
}

// Batches of host-resident sources solved one after another with the copies hidden: batch i's
// solve runs on the context's stream while the copy stream brings batch i+1's sources in and
// takes batch i-1's solutions out, through two device slots (b/x and b1/x1).  Slot k's
// inputs may be overwritten once the solve that read them is done (ev_solved), and its
// output once the copy that read it is done (ev_out).
int amg_solve_stream(amg_ctx c, int nbatch, const double* const* b, double* const* x, int nrhs,
                     amg_solve_info* const* info) {
    CKR(check_ready(c, 0, true));
    if (nbatch < 1 || !b || !x || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    for (int i = 0; i < nbatch; i++)
        if (!b[i] || !x[i]) return fail(AMG_ERR_INVALID, "null vector for batch %d", i);
    CKR(select_device(c));
    if (nrhs > c->Rcap) {
        CKR(ensure_capacity(c, nrhs));
        CKR(build_engine<double>(c, c->d, std::max(c->d.eng_cap, nrhs)));
        if (c->p.precision == AMG_PREC_MIXED) CKR(build_engine<float>(c, c->f, std::max(c->f.eng_cap, nrhs)));
    }
    if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
        if (!c->ev_in[k]) CK(cudaEventCreateWithFlags(&c->ev_in[k], cudaEventDisableTiming));
        if (!c->ev_solved[k]) CK(cudaEventCreateWithFlags(&c->ev_solved[k], cudaEventDisableTiming));
        if (!c->ev_out[k]) CK(cudaEventCreateWithFlags(&c->ev_out[k], cudaEventDisableTiming));
        if (!c->ev_piece[k]) CK(cudaEventCreateWithFlags(&c->ev_piece[k], cudaEventDisableTiming));
    }
    const long long n = (long long)nrhs * vlen0(c);
    const size_t bytes = (size_t)n * sizeof(double2);
    CKR(c->b1.alloc(bytes));
    CKR(c->x1.alloc(bytes));
    void* bs[2] = {c->b.p, c->b1.p};
    void* xs[2] = {c->x.p, c->x1.p};
    cudaStream_t cs = c->copy_stream;
    // both slots free: nothing of an earlier call may still read or write them
    CK(cudaStreamSynchronize(c->stream));

    // The copies are enqueued by a helper thread, in pieces of kPiece bytes with at most two
    // in flight (the helper waits for the older one before it enqueues the next): a whole
    // gigabyte queued at once holds the driver long enough to delay the solve's own launches.
    // Host-side counters order each event's recording before every wait that refers to it:
    //   in_done   batches whose input copy (ev_in) is enqueued    (helper -> solver)
    //   solved    batches whose ev_solved is recorded            (solver -> helper)
    //   out_done  batches whose output copy (ev_out) is enqueued  (helper -> solver)
    std::mutex mu;
    std::condition_variable cv;
    int in_done = 0, solved = 0, out_done = 0;
    bool stop = false;
    cudaError_t copy_err = cudaSuccess;
    auto wait_for = [&](const int& counter, int need) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || counter >= need; });
        return !stop;
    };
    auto publish = [&](int& counter, int value) {
        {
            std::lock_guard<std::mutex> lk(mu);
            counter = value;
        }
        cv.notify_all();
    };
    auto halt = [&]() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
    };
    const int device = c->device;
    constexpr size_t kPiece = size_t(64) << 20;
    auto copy_loop = [&] {
        cudaSetDevice(device);
        auto ok = [&](cudaError_t e) {
            if (e != cudaSuccess && copy_err == cudaSuccess) copy_err = e;
            return e == cudaSuccess;
        };
        long long piece = 0;
        auto paced = [&](void* dst, const void* src, cudaMemcpyKind kind) {
            for (size_t o = 0; o < bytes; o += kPiece, piece++) {
                cudaEvent_t ev = c->ev_piece[piece & 1];
                if (piece >= 2 && !ok(cudaEventSynchronize(ev))) return false;
                if (!ok(cudaMemcpyAsync(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o,
                                        std::min(kPiece, bytes - o), kind, cs)) ||
                    !ok(cudaEventRecord(ev, cs)))
                    return false;
            }
            return true;
        };
        for (int s = 0; s <= nbatch; s++) {
            if (s < nbatch) {
                // batch s's sources into slot s&1 once batch s-2's solve stopped reading it
                if (s >= 2) {
                    if (!wait_for(solved, s - 1)) return;
                    if (!ok(cudaStreamWaitEvent(cs, c->ev_solved[s & 1], 0))) break;
                }
                if (!paced(bs[s & 1], b[s], cudaMemcpyHostToDevice) || !ok(cudaEventRecord(c->ev_in[s & 1], cs)))
                    break;
                publish(in_done, s + 1);
            }
            if (s >= 1) {
                // batch s-1's solutions out once its solve is done
                if (!wait_for(solved, s)) return;
                if (!ok(cudaStreamWaitEvent(cs, c->ev_solved[(s - 1) & 1], 0)) ||
                    !paced(x[s - 1], xs[(s - 1) & 1], cudaMemcpyDeviceToHost) ||
                    !ok(cudaEventRecord(c->ev_out[(s - 1) & 1], cs)))
                    break;
                publish(out_done, s);
            }
        }
        if (copy_err != cudaSuccess) halt();
    };
    std::thread helper;
    try {
        helper = std::thread(copy_loop);
    } catch (const std::exception& ex) {
        return fail(AMG_ERR_UNSUPPORTED, "no copy thread: %s", ex.what());
    }
    int rc = AMG_OK;
    for (int i = 0; i < nbatch && rc >= 0; i++) {
        const int k = i & 1;
        if (!wait_for(in_done, i + 1)) break;
        cudaError_t e = cudaStreamWaitEvent(c->stream, c->ev_in[k], 0);
        if (e == cudaSuccess && i >= 2) {   // batch i-2's solutions copied out of slot k
            if (!wait_for(out_done, i - 1)) break;
            e = cudaStreamWaitEvent(c->stream, c->ev_out[k], 0);
        }
        if (e != cudaSuccess) {
            rc = fail(AMG_ERR_CUDA, "%s", cudaGetErrorString(e));
            break;
        }
        const int r = amg_solve_dev(c, bs[k], xs[k], nrhs, info ? info[i] : nullptr);
        if (r < 0) {
            rc = r;
            break;
        }
        if (r == AMG_NOT_CONVERGED) rc = r;
        if ((e = cudaEventRecord(c->ev_solved[k], c->stream)) != cudaSuccess) {
            rc = fail(AMG_ERR_CUDA, "%s", cudaGetErrorString(e));
            break;
        }
        publish(solved, i + 1);
    }
    if (rc < 0) halt();
    helper.join();
    const cudaError_t es = cudaStreamSynchronize(cs);
    if (rc < 0) return rc;
    if (copy_err != cudaSuccess) return fail(AMG_ERR_CUDA, "batch copy: %s", cudaGetErrorString(copy_err));
    if (stop) return fail(AMG_ERR_CUDA, "batch copies stopped");
    if (es != cudaSuccess) return fail(AMG_ERR_CUDA, "%s", cudaGetErrorString(es));
    return rc;
}

namespace {
// capacity and engines of a context for nrhs sources (amg_solve_dev's preamble)
int prepare_solve(amg_ctx c, int nrhs) {
    CKR(check_ready(c, 0, true));
    if (nrhs < 1) return fail(AMG_ERR_INVALID, "nrhs must be >= 1");
    CKR(select_device(c));
    if (nrhs > c->Rcap) {
        CKR(ensure_capacity(c, nrhs));
        CKR(build_engine<double>(c, c->d, std::max(c->d.eng_cap, nrhs)));
        if (c->p.precision == AMG_PREC_MIXED) CKR(build_engine<float>(c, c->f, std::max(c->f.eng_cap, nrhs)));
    }
    return AMG_OK;
}

// several contexts' outer FGMRES solves driven in turn (see OuterSolve)
int solve_many(int count, const amg_ctx* ctx, const double2* const* b, double2* const* x, const int* nrhs,
               amg_solve_info* const* info) {
    std::vector<OuterSolve> S(count);
    for (int i = 0; i < count; i++) {
        CKR(select_device(ctx[i]));
        CK(cudaEventRecord(ctx[i]->ev0, ctx[i]->stream));
        CKR(S[i].init(ctx[i], b[i], x[i], nrhs[i], info ? info[i] : nullptr));
    }
    // grouped preconditioners (SapGroup): contexts whose steps wait in PRECOND, keyed by
    // device, block size and post-smoothing count, share their SAP launches
    const bool group = count > 1 && sap_group_enabled();
    for (int i = 0; i < count; i++) S[i].defer = group;
    std::map<std::vector<amg_context*>, std::unique_ptr<SapGroup>> groups;
    for (bool busy = true; busy;) {
        busy = false;
        for (int i = 0; i < count; i++) {
            if (S[i].phase == OuterSolve::DONE) continue;
            busy = true;
            if (S[i].phase == OuterSolve::PRECOND) continue;
            CKR(select_device(ctx[i]));
            CK(cudaEventSynchronize(ctx[i]->ev_host));
            CKR(S[i].advance());
        }
        std::map<std::tuple<int, int, int>, std::vector<int>> waiting;
        for (int i = 0; i < count; i++)
            if (S[i].phase == OuterSolve::PRECOND)
                waiting[std::make_tuple(ctx[i]->device, group_block_size(ctx[i]), ctx[i]->p.nu2)].push_back(i);
        for (auto& kv : waiting) {
            const std::vector<int>& ids = kv.second;
            CKR(select_device(ctx[ids[0]]));
            if (ids.size() == 1) {
                // nobody to share with: the context's own (graph-captured) preconditioner
                OuterSolve& s = S[ids[0]];
                CKR(precondition(s.c, s.step_input(), nullptr, s.R, false));
            } else {
                std::vector<amg_context*> cs;
                std::vector<int> R;
                std::vector<const double2*> v;
                for (int i : ids) {
                    cs.push_back(ctx[i]);
                    R.push_back(S[i].R);
                    v.push_back(S[i].step_input());
                }
                std::unique_ptr<SapGroup>& g = groups[cs];
                if (!g) {
                    g.reset(new SapGroup());
                    CKR(g->build(cs, R));
                }
                CKR(g->precondition(v));
            }
            for (int i : ids) CKR(S[i].issue_step_post());
        }
    }
    int rc = AMG_OK;
    for (int i = 0; i < count; i++) {
        amg_ctx c = ctx[i];
        CKR(select_device(c));
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaEventSynchronize(c->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->last_solve_ms = ms;
        int flags = 0;
        CK(cudaMemcpy(&flags, c->d.eh.flags, sizeof(int), cudaMemcpyDeviceToHost));
        if (flags) return fail(AMG_ERR_UNSUPPORTED, "engine of context %d reported flags %d", i, flags);
        CKR(check_fine_waits(c->stream));
        if (S[i].rc == AMG_NOT_CONVERGED) rc = AMG_NOT_CONVERGED;
    }
    return rc;
}

int check_many(int count, const amg_ctx* ctx, const void* const* b, void* const* x, const int* nrhs) {
    if (count < 1 || !ctx || !b || !x || !nrhs) return fail(AMG_ERR_INVALID, "bad argument");
    for (int i = 0; i < count; i++) {
        if (!b[i] || !x[i]) return fail(AMG_ERR_INVALID, "null vector for context %d", i);
        for (int k = 0; k < i; k++)
            if (ctx[k] == ctx[i]) return fail(AMG_ERR_INVALID, "context %d appears twice", i);
        CKR(prepare_solve(ctx[i], nrhs[i]));
    }
    return AMG_OK;
}
}  // namespace

int amg_solve_many_dev(int count, const amg_ctx* ctx, const void* const* b_dev, void* const* x_dev, const int* nrhs,
                       amg_solve_info* const* info) {
    CKR(check_many(count, ctx, b_dev, x_dev, nrhs));
    std::vector<const double2*> b(count);
    std::vector<double2*> x(count);
    for (int i = 0; i < count; i++) {
        b[i] = static_cast<const double2*>(b_dev[i]);
        x[i] = static_cast<double2*>(x_dev[i]);
    }
    return solve_many(count, ctx, b.data(), x.data(), nrhs, info);
}

int amg_solve_many(int count, const amg_ctx* ctx, const double* const* b, double* const* x, const int* nrhs,
                   amg_solve_info* const* info) {
    CKR(check_many(count, ctx, reinterpret_cast<const void* const*>(b), reinterpret_cast<void* const*>(x), nrhs));
    std::vector<const double2*> bd(count);
    std::vector<double2*> xd(count);
    for (int i = 0; i < count; i++) {
        amg_ctx c = ctx[i];
        CKR(select_device(c));
        const long long n = (long long)nrhs[i] * vlen0(c);
        CK(cudaMemcpyAsync(c->b.p, b[i], (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        bd[i] = c->b.as<double2>();
        xd[i] = c->x.as<double2>();
    }
    const int rc = solve_many(count, ctx, bd.data(), xd.data(), nrhs, info);
    if (rc < 0) return rc;
    for (int i = 0; i < count; i++) {
        amg_ctx c = ctx[i];
        CKR(select_device(c));
        const long long n = (long long)nrhs[i] * vlen0(c);
        CK(cudaMemcpyAsync(x[i], c->x.p, (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return rc;
}

int amg_residual_history(amg_ctx c, double* out, int max_len, int* len) {
    if (!c || !len) return fail(AMG_ERR_INVALID, "null argument");
    const int n = (int)c->history.size();
    *len = n;
    if (out)
        for (int i = 0; i < std::min(n, max_len); i++) out[i] = c->history[i];
    return AMG_OK;
}

// D^dagger lambda = g through the solve of D: lambda = gamma5 D^{-1} gamma5 g.  The FP64
// true residual reported for D y = gamma5 g equals ||g - D^dagger lambda|| / ||g|| because
// gamma5 is unitary.
int amg_solve_adjoint_dev(amg_ctx c, const void* g, void* lambda, int nrhs, amg_solve_info* info) {
    CKR(check_ready(c, 0, true));
    if (!g || !lambda || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    const long long n = (long long)nrhs * vlen0(c);
    CKR(c->adj.alloc((size_t)n * sizeof(double2)));
    launch_gamma5(c->adj.as<double2>(), (const double2*)g, n / 2, c->stream);
    CKL();
    const int rc = amg_solve_dev(c, c->adj.p, lambda, nrhs, info);
    if (rc < 0) return rc;
    launch_gamma5((double2*)lambda, (const double2*)lambda, n / 2, c->stream);
    CKL();
    CK(cudaStreamSynchronize(c->stream));
    return rc;
}

int amg_solve_adjoint(amg_ctx c, const double* g, double* lambda, int nrhs, amg_solve_info* info) {
    CKR(check_ready(c, 0, true));
    if (!g || !lambda || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    CKR(select_device(c));
    if (nrhs > c->Rcap) {
        CKR(ensure_capacity(c, nrhs));
        CKR(build_engine<double>(c, c->d, std::max(c->d.eng_cap, nrhs)));
        if (c->p.precision == AMG_PREC_MIXED) CKR(build_engine<float>(c, c->f, std::max(c->f.eng_cap, nrhs)));
    }
    const long long n = (long long)nrhs * vlen0(c);
    CK(cudaMemcpyAsync(c->b.p, g, (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    const int rc = amg_solve_adjoint_dev(c, c->b.p, c->x.p, nrhs, info);
    if (rc < 0) return rc;
    CK(cudaMemcpyAsync(lambda, c->x.p, (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return rc;
}

int amg_force_dev(amg_ctx c, const void* lambda, const void* x, int nrhs, void* F) {
    if (!c || !lambda || !x || !F || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "gauge field not set");
    CKR(select_device(c));
    launch_force(c->d.U.as<double2>(), (const double2*)lambda, (const double2*)x, (double2*)F, c->nx, c->nt, nrhs,
                 c->stream);
    CKL();
    CK(cudaStreamSynchronize(c->stream));
    return AMG_OK;
}

int amg_force(amg_ctx c, const double* lambda, const double* x, int nrhs, double* F) {
    if (!c || !lambda || !x || !F || nrhs < 1) return fail(AMG_ERR_INVALID, "bad argument");
    if (!c->gauge_set) return fail(AMG_ERR_STATE, "gauge field not set");
    CKR(select_device(c));
    DevBuf a, b, f;
    const long long n = (long long)nrhs * vlen0(c);
    CKR(to_dev(a, lambda, n, c->stream));
    CKR(to_dev(b, x, n, c->stream));
    CKR(to_dev(f, nullptr, c->N, c->stream));
    launch_force(c->d.U.as<double2>(), a.as<double2>(), b.as<double2>(), f.as<double2>(), c->nx, c->nt, nrhs,
                 c->stream);
    CKL();
    return to_host(F, f, c->N, c->stream);
}

int amg_engine_counters(amg_ctx c, long long* out, int len) {
    if (!c || !out) return fail(AMG_ERR_INVALID, "null argument");
    PrecSet<double>& d = c->d;
    std::vector<unsigned long long> v(kMaxLevels * ENG_NCOUNT, 0), w(kMaxLevels * ENG_NCOUNT, 0);
    if (d.eh.counters) CK(cudaMemcpy(v.data(), d.eh.counters, v.size() * 8, cudaMemcpyDeviceToHost));
    if (c->f.ready && c->f.eh.counters) CK(cudaMemcpy(w.data(), c->f.eh.counters, w.size() * 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < len && i < (int)v.size(); i++) out[i] = (long long)(v[i] + w[i]);
    if (d.eh.counters) CK(cudaMemset(d.eh.counters, 0, v.size() * 8));
    if (c->f.ready && c->f.eh.counters) CK(cudaMemset(c->f.eh.counters, 0, w.size() * 8));
    return AMG_OK;
}

long long amg_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

void* amg_get_stream(amg_ctx c) { return c ? (void*)c->stream : nullptr; }

int amg_profile(amg_ctx c, int enable) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    prof_harvest(c);
    c->prof_on = enable ? 1 : 0;
    for (auto& s : c->prof) s = amg_context::ProfSlot{};
    return AMG_OK;
}

int amg_profile_query(amg_ctx c, int slot, double* ms, long long* launches, double* bytes) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    if (slot < 0 || slot >= AMG_PROF_SLOTS) return fail(AMG_ERR_INVALID, "profile slot %d", slot);
    prof_harvest(c);
    if (ms) *ms = c->prof[slot].ms;
    if (launches) *launches = c->prof[slot].n;
    if (bytes) *bytes = c->prof[slot].bytes;
    return AMG_OK;
}

int amg_autotune_info(amg_ctx c, int* out) {
    if (!c || !out) return fail(AMG_ERR_INVALID, "null argument");
    const bool mixed = c->p.precision == AMG_PREC_MIXED;
    out[0] = c->tuned;
    out[1] = c->sap_variant;
    out[2] = mixed ? c->f.cluster_pick : c->d.cluster_pick;
    out[3] = (int)c->tuned_us;
    return AMG_OK;
}

int amg_autotune_info_n(amg_ctx c, int* out, int n) {
    if (!c || !out || n < 0) return fail(AMG_ERR_INVALID, "bad argument");
    int v[5];
    CKR(amg_autotune_info(c, v));
    const int t = c->p.precision == AMG_PREC_MIXED ? c->f.sap_teams : c->d.sap_teams;
    v[4] = t ? t : engine_sap_teams();
    for (int i = 0; i < std::min(n, 5); i++) out[i] = v[i];
    return AMG_OK;
}

int amg_setup_timings(amg_ctx c, double* ms, int n) {
    if (!c || !ms || n < 0) return fail(AMG_ERR_INVALID, "bad argument");
    for (int i = 0; i < std::min(n, (int)AMG_SETUP_PHASES); i++) ms[i] = c->setup_phase_ms[i];
    return AMG_OK;
}

int amg_last_timings(amg_ctx c, double* setup_ms, double* solve_ms) {
    if (!c) return fail(AMG_ERR_INVALID, "null context");
    if (setup_ms) *setup_ms = c->last_setup_ms;
    if (solve_ms) *solve_ms = c->last_solve_ms;
    return AMG_OK;
}

}  // extern "C"
