// Coarse-level engine: the whole multigrid work below the fine level runs inside one CTA
// per source.  Every function here is called by all threads of the CTA and ends with the
// CTA synchronised, so its results are visible to every thread.
//
// Levels l >= 1 use the generic level operator of the reference (Level::D_operator,
// src/level.cpp:161-180) with dense per-site link matrices; vectors are v[n][dof] with
// dof = 2c + spin, exactly as the reference stores them.  The fine level (l = 0) is
// handled by the fine-lattice kernels and only enters here through its coarse image.
#pragma once
#include "common.cuh"

namespace amgb {

constexpr int kMaxLevels = 6;
constexpr int kEngineThreads = 512;

// Hop order of the stored link matrices: self (G1), right mu=0, right mu=1 (G2),
// left mu=0, left mu=1 (G3).
enum { HOP_SELF = 0, HOP_R0 = 1, HOP_R1 = 2, HOP_L0 = 3, HOP_L1 = 4 };

// Per-level description used by the engine (device copy lives in kernel parameters).
template <typename T>
struct EngLevel {
    int level;                  // index of this level in the hierarchy
    int nx, nt, n, K;           // lattice and dof per site
    int coarsest;
    // aggregation to level l+1
    int bx, bt, xe, te, ntest;
    const cx<T>* W;             // [ntest][n][K]
    // operator: links[x][hop][j][i] (column-major K x K), reference G without sign
    const cx<T>* links;
    // SAP blocking
    int sbx, sbt, sxe, ste, ncol;
    const int* red;             // [ncol]
    const int* black;           // [ncol]
    // per-source work vectors (offsets in elements of cx<T> inside the source's slab)
    long long off_kfg;          // K-cycle FGMRES: V[m+1], Z[m], w    (all levels)
    long long off_cg;           // coarsest GMRES: V[m+1], w           (coarsest)
    long long off_cyc;          // cycle: r, eta_c, psi_c, ppsi        (non-coarsest)
    long long off_sap;          // SAP: r, upd, V[m+1] (colour), w, b, x (non-coarsest)
    // shared-memory scalar blocks (byte offsets)
    int sm_kfg, sm_cg, sm_sap;
    // Level::gmres_l knobs of this level (LevelV::GMRES_*, include/params.h:51-53, 63-65)
    int gm_m, gm_restarts;
    T gm_tol;
    // SAP block solves: teams per CTA, and whether a team's block vectors fit in shared memory
    int sap_nteam, sap_vec_smem;
    long long off_sapteam;      // slab offset of the team block vectors when not in shared memory
};

template <typename T>
struct EngParams {
    T m0;
    int cycle, nu1, nu2;
    int sap_m, sap_restarts;
    T sap_gmres_tol, sap_tol;
    int k_m, k_restarts;
    T k_tol;
    int c_m, c_restarts;
    T c_tol;
};

template <typename T>
struct EngArgs {
    EngLevel<T> lv[kMaxLevels];
    int nlev;
    EngParams<T> p;
    cx<T>* work;                 // per-source slabs
    long long slab;              // elements per slab
    int smem_red;                // byte offset of the whole-CTA reduction scratch (2*2*16 reals)
    int smem_team;               // byte offset of the team area (SAP block solves)
    int team_bytes;              // bytes per team in that area
    long long off_io;            // slab offset of the entry op's input / output copies
    long long io_len;            // elements of each copy
    int* status;                 // [nsrc] per-source result code / iteration count
    int* flags;                  // error flag (bit 0: recursion bound, bit 1: unsupported)
    unsigned long long* counters;  // [kMaxLevels][ENG_NCOUNT] operation counts (tracing)
};

// engine operation counters, per level
enum { CNT_APPLY = 0, CNT_LOCAL_APPLY = 1, CNT_KFG_STEP = 2, CNT_GMRES_STEP = 3, CNT_SAP_STEP = 4, CNT_SAP_CALL = 5,
       ENG_NCOUNT = 6 };

// ---------------------------------------------------------------------------------
// FGMRES scalar state for nseg independent segments
// ---------------------------------------------------------------------------------
template <typename T>
struct GmState {
    cx<T>* H;      // [nseg][(m+1)*m]   H[i][j] at i*m + j
    cx<T>* g;      // [nseg][m+1]
    cx<T>* cn;     // [nseg][m]
    cx<T>* sn;     // [nseg][m]
    cx<T>* eta;    // [nseg][m]
    T* err;        // [nseg]
    T* normb;      // [nseg]
    cx<T>* red;    // [nseg] reduction results
    int* maxit;    // [nseg]
    int* act;      // [nseg] 1 while in the restart loop
    int* arn;      // [nseg] 1 while in the Arnoldi loop
    int* iters;    // [nseg]
};

// bytes of the shared-memory block for a GmState
__host__ __device__ inline int gm_state_bytes(int nseg, int m, int real_bytes) {
    int c = 2 * real_bytes;
    int nc = nseg * ((m + 1) * m + (m + 1) + 3 * m + 1);
    int b = nc * c + 2 * nseg * real_bytes + 4 * nseg * 4;
    return (b + 15) & ~15;
}

template <typename T>
__device__ inline GmState<T> gm_state_at(char* base, int nseg, int m) {
    GmState<T> s;
    cx<T>* c = reinterpret_cast<cx<T>*>(base);
    s.H = c; c += nseg * (m + 1) * m;
    s.g = c; c += nseg * (m + 1);
    s.cn = c; c += nseg * m;
    s.sn = c; c += nseg * m;
    s.eta = c; c += nseg * m;
    s.red = c; c += nseg;
    T* r = reinterpret_cast<T*>(c);
    s.err = r; r += nseg;
    s.normb = r; r += nseg;
    int* i = reinterpret_cast<int*>(r);
    s.maxit = i; i += nseg;
    s.act = i; i += nseg;
    s.arn = i; i += nseg;
    s.iters = i;
    return s;
}

// ---------------------------------------------------------------------------------
// whole-CTA elementwise helpers (end synchronised)
// ---------------------------------------------------------------------------------
template <typename T>
__device__ void v_copy(cx<T>* d, const cx<T>* s, int n) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) d[e] = s[e];
    __syncthreads();
}
template <typename T>
__device__ void v_zero(cx<T>* d, int n) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) d[e] = czero<T>();
    __syncthreads();
}
// d = a - b
template <typename T>
__device__ void v_sub(cx<T>* d, const cx<T>* a, const cx<T>* b, int n) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) d[e] = a[e] - b[e];
    __syncthreads();
}
// d += s
template <typename T>
__device__ void v_add(cx<T>* d, const cx<T>* s, int n) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) d[e] += s[e];
    __syncthreads();
}

// ---------------------------------------------------------------------------------
// engine context per CTA (one source)
// ---------------------------------------------------------------------------------
template <typename T>
struct Eng {
    const EngArgs<T>* a;
    cx<T>* slab;
    char* smem;
    T* red;
    int crank, csize;           // rank in the thread-block cluster serving this source, cluster size

    __device__ const EngLevel<T>& L(int l) const { return a->lv[l]; }
    __device__ cx<T>* work(long long off) const { return slab + off; }
};

template <typename T>
__device__ __forceinline__ void eng_count(const Eng<T>& E, int level, int what, unsigned long long n = 1) {
    if (E.a->counters && E.crank == 0 && threadIdx.x == 0)
        atomicAdd(&E.a->counters[level * ENG_NCOUNT + what], n);
}

// ---------------------------------------------------------------------------------
// level geometry helpers
// ---------------------------------------------------------------------------------
__device__ __forceinline__ int nb_site(int x, int t, int nx, int nt, int hop) {
    switch (hop) {
        case HOP_R0: t = (t + 1 == nt) ? 0 : t + 1; break;
        case HOP_R1: x = (x + 1 == nx) ? 0 : x + 1; break;
        case HOP_L0: t = (t == 0) ? nt - 1 : t - 1; break;
        case HOP_L1: x = (x == 0) ? nx - 1 : x - 1; break;
        default: break;
    }
    return x * nt + t;
}
// SignR_l / SignL_l (include/boundary.h:37-38): -1 on the time hop across t = Nt-1 -> 0
__device__ __forceinline__ int hop_sign(int t, int nt, int hop) {
    if (hop == HOP_R0 && t == nt - 1) return -1;
    if (hop == HOP_L0 && t == 0) return -1;
    return 1;
}

// Hardware barrier over the thread-block cluster with release/acquire ordering of every
// memory access before it (global stores into other CTAs' slabs included).
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Rows [e0, e1) of a partitioned operator output computed by this CTA, and the distance
// (in elements) from this CTA's slab to the slab of cluster rank q.
template <typename T>
__device__ __forceinline__ void part_range(const Eng<T>& E, int tot, int& e0, int& e1) {
    const int per = (tot + E.csize - 1) / E.csize;
    e0 = min(tot, E.crank * per);
    e1 = min(tot, e0 + per);
}
// The cluster split as plain values, read once per operator call: inside the row loops the
// fields of the engine context would otherwise be re-read from the caller's stack frame
// after every store (the stores go through generic pointers that may alias it).
struct Part {
    int csize, crank;
    long long slab;
};
template <typename T>
__device__ __forceinline__ Part part_of(const Eng<T>& E) {
    return Part{E.csize, E.crank, E.a->slab};
}
template <typename T>
__device__ __forceinline__ void part_store(const Part& P, cx<T>* out, int e, cx<T> v) {
    if (P.csize == 1) { out[e] = v; return; }
    for (int q = 0; q < P.csize; q++) out[(long long)(q - P.crank) * P.slab + e] = v;
}
template <typename T>
__device__ __forceinline__ void part_begin(const Eng<T>& E) {
    if (E.csize > 1) cluster_barrier();
    else __syncthreads();
}
template <typename T>
__device__ __forceinline__ void part_end(const Eng<T>& E) {
    if (E.csize > 1) cluster_barrier();
    else __syncthreads();
}

// Threads cooperating on one output row of a dense coarse operator: every row's K columns
// are split over TPR consecutive lanes so each thread keeps several independent L2 loads in
// flight; the partial sums are combined with shuffles.
constexpr int kTPR = 8;
template <typename T>
__device__ __forceinline__ cx<T> tpr_sum(cx<T> a) {
#pragma unroll
    for (int o = kTPR / 2; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
        a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
    }
    return a;
}

// Level::D_operator (src/level.cpp:161-180) for l >= 1:
// out = (m0+2) in - sum_hop sign * G_hop in(neighbour).  With a cluster, every CTA computes
// a slice of the rows and stores it into every CTA's copy of `out`.
template <typename T>
__device__ __noinline__ void dc_apply(const Eng<T>& E, const EngLevel<T>& L, T m0, const cx<T>* in, cx<T>* out) {
    const int K = L.K, tot = L.n * K, lnx = L.nx, lnt = L.nt;
    const cx<T>* const links = L.links;
    const Part P = part_of(E);
    const T mass = m0 + T(2);
    int e0, e1;
    eng_count(E, L.level, CNT_APPLY);
    part_range(E, tot, e0, e1);
    part_begin(E);
    const int g = threadIdx.x % kTPR, rows_per_pass = blockDim.x / kTPR;
    for (int rb = e0; rb < e1; rb += rows_per_pass) {
        const int e = rb + threadIdx.x / kTPR;
        const bool on = e < e1;
        cx<T> acc = czero<T>();
        if (on) {
            const int xs = e / K, i = e - xs * K;
            const int x = xs / lnt, t = xs - x * lnt;
            const cx<T>* lk = links + (long long)xs * 5 * K * K + i;
#pragma unroll 1
            for (int h = 0; h < 5; h++) {
                const int nbs = nb_site(x, t, lnx, lnt, h);
                const cx<T>* v = in + (long long)nbs * K;
                const cx<T>* a = lk + (long long)h * K * K;
                cx<T> s = czero<T>();
#pragma unroll 4
                for (int j = g; j < K; j += kTPR) cfma(s, __ldg(a + (long long)j * K), v[j]);
                if (hop_sign(t, lnt, h) < 0) acc -= s; else acc += s;
            }
        }
        acc = tpr_sum<T>(acc);
        if (on && g == 0) part_store<T>(P, out, e, mass * in[e] - acc);
    }
    part_end(E);
}

// SAP block bookkeeping (SAP_C::SchwarzBlocks, src/sap.cpp:3-39): block b covers
// x in [bx*sxe, (bx+1)*sxe), t in [bt*ste, (bt+1)*ste), b = bx*sbt + bt; local site
// index m = mx*ste + mt.
template <typename T>
__device__ __forceinline__ int sap_site(const EngLevel<T>& L, int block, int m, int* xo, int* to) {
    const int bxi = block / L.sbt, bti = block - bxi * L.sbt;
    const int mx = m / L.ste, mt = m - mx * L.ste;
    const int x = bxi * L.sxe + mx, t = bti * L.ste + mt;
    *xo = x; *to = t;
    return x * L.nt + t;
}

// Level::Pt_v (src/level.cpp:212-237): out[nc][2cc+s] = sum_{n in nc, c} conj(W_cc[n][2c+s]) v[n][2c+s]
template <typename T>
__device__ __noinline__ void restrict_v(const Eng<T>& E, const EngLevel<T>& L, const cx<T>* v, cx<T>* out) {
    const int K = L.K, col = K / 2, nblk = L.bx * L.bt, ntest = L.ntest, tot = nblk * 2 * ntest;
    const int xe = L.xe, te = L.te, lbt = L.bt, lnt = L.nt, nterm = xe * te * col;
    const long long wstride = (long long)L.n * K;
    const cx<T>* const W = L.W;
    const Part P = part_of(E);
    int e0, e1;
    part_range(E, tot, e0, e1);
    part_begin(E);
    const int g = threadIdx.x % kTPR, rows_per_pass = blockDim.x / kTPR;
    for (int rb = e0; rb < e1; rb += rows_per_pass) {
        const int o = rb + threadIdx.x / kTPR;
        const bool on = o < e1;
        cx<T> acc = czero<T>();
        if (on) {
            const int nc = o / (2 * ntest), r = o - nc * 2 * ntest, cc = r >> 1, s = r & 1;
            const int bxi = nc / lbt, bti = nc - bxi * lbt;
            const cx<T>* w = W + (long long)cc * wstride;
#pragma unroll 4
            for (int q = g; q < nterm; q += kTPR) {
                const int site = q / col, c = q - site * col;
                const int mx = site / te, mt = site - mx * te;
                const long long n = (long long)(bxi * xe + mx) * lnt + (bti * te + mt);
                cfmac(acc, __ldg(w + n * K + 2 * c + s), v[n * K + 2 * c + s]);
            }
        }
        acc = tpr_sum<T>(acc);
        if (on && g == 0) part_store<T>(P, out, o, acc);
    }
    part_end(E);
}

// out (+)= P vc: Level::P_v (src/level.cpp:182-209), out[n][2c+s] = sum_cc W_cc[n][2c+s] vc[nc][2cc+s]
template <typename T>
__device__ __noinline__ void prolong_v(const Eng<T>& E, const EngLevel<T>& L, const cx<T>* vc, cx<T>* out,
                                       int accumulate) {
    const int K = L.K, tot = L.n * K, lnt = L.nt, xe = L.xe, te = L.te, lbt = L.bt, ntest = L.ntest;
    const long long wstride = (long long)L.n * K;
    const cx<T>* const W = L.W;
    const Part P = part_of(E);
    int e0, e1;
    part_range(E, tot, e0, e1);
    part_begin(E);
    const int g = threadIdx.x % kTPR, rows_per_pass = blockDim.x / kTPR;
    for (int rb = e0; rb < e1; rb += rows_per_pass) {
        const int e = rb + threadIdx.x / kTPR;
        const bool on = e < e1;
        cx<T> acc = czero<T>();
        if (on) {
            const int n = e / K, d = e - n * K, s = d & 1;
            const int x = n / lnt, t = n - x * lnt;
            const int nc = (x / xe) * lbt + (t / te);
            const cx<T>* pv = vc + (long long)nc * 2 * ntest + s;
#pragma unroll 2
            for (int cc = g; cc < ntest; cc += kTPR) cfma(acc, __ldg(W + (long long)cc * wstride + e), pv[2 * cc]);
        }
        acc = tpr_sum<T>(acc);
        if (on && g == 0) part_store<T>(P, out, e, accumulate ? out[e] + acc : acc);
    }
    part_end(E);
}

// ---------------------------------------------------------------------------------
// Teams: a whole CTA (hardware barrier 0) or a slice of it with its own named barrier.
// ---------------------------------------------------------------------------------
struct Team {
    int tid, size, nw, bar;     // thread index in the team, threads, warps, barrier id
};
__device__ __forceinline__ Team whole_cta() { return Team{(int)threadIdx.x, (int)blockDim.x, (int)(blockDim.x >> 5), 0}; }
__device__ __forceinline__ void team_sync(const Team& tm) {
    if (tm.bar == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(tm.bar), "r"(tm.size) : "memory");
}
// Sum of (ax, ay) over the team; every thread receives it.  `part` holds 2*2*nw reals used as
// two alternating buffers, so one barrier per reduction suffices.
template <typename T>
__device__ __forceinline__ cx<T> team_sum2(const Team& tm, T* part, int& buf, T ax, T ay) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (tm.nw == 1) return mk<T>(ax, ay);
    T* pb = part + buf * tm.nw * 2;
    const int lane = tm.tid & 31, wid = tm.tid >> 5;
    if (lane == 0) { pb[2 * wid] = ax; pb[2 * wid + 1] = ay; }
    team_sync(tm);
    T sx = 0, sy = 0;
    for (int k = 0; k < tm.nw; k++) { sx += pb[2 * k]; sy += pb[2 * k + 1]; }
    buf ^= 1;
    return mk<T>(sx, sy);
}

// ---------------------------------------------------------------------------------
// FGMRES (src/fgmres.cpp:5-115) of one team on one vector of n entries with x0 = b (the
// only start the multigrid uses below the fine level: src/amg.cpp:138, :161,
// src/sap.cpp:61).  op(in, out) and pre(j, V_j, Z_j) are collective operations that start by
// synchronising (so earlier writes to their input are visible) and end synchronised;
// between them every thread only touches its own entries e = tid, tid + size, ...  The
// arithmetic is the reference's: modified Gram-Schmidt, Givens rotations, Arnoldi exit on
// |g_{j+1}| < tol*||b||, a true residual after each cycle, and maxIt carried over restart
// cycles.  Z may alias V (identity preconditioner).  Returns k*m + maxIt or restarts*m.
// ---------------------------------------------------------------------------------
template <typename T, class Op, class Pre>
__device__ int team_fgmres(const Team& tm, T* part, const Eng<T>* E, int cnt_level, int cnt_what, Op& op, Pre& pre,
                           const cx<T>* b, cx<T>* x, cx<T>* V, cx<T>* Z, cx<T>* w, const GmState<T>& st, int n,
                           int m, int restarts, T tol) {
    int buf = 0;
    const int tid = tm.tid, ts = tm.size;
    // setZeros (include/fgmres.h:93-120)
    for (long long e = tid; e < (long long)(m + 1) * n; e += ts) V[e] = czero<T>();
    if (Z != V)
        for (long long e = tid; e < (long long)m * n; e += ts) Z[e] = czero<T>();
    if (tid == 0) {
        for (int q = 0; q < (m + 1) * m; q++) st.H[q] = czero<T>();
        for (int q = 0; q <= m; q++) st.g[q] = czero<T>();
        for (int q = 0; q < m; q++) { st.cn[q] = czero<T>(); st.sn[q] = czero<T>(); st.eta[q] = czero<T>(); }
    }
    for (int e = tid; e < n; e += ts) x[e] = b[e];
    op(x, w);
    T rr = 0, bb = 0;
    for (int e = tid; e < n; e += ts) {
        const cx<T> r = b[e] - w[e];
        V[e] = r;
        rr += cnorm2(r);
        bb += cnorm2(b[e]);
    }
    cx<T> s2 = team_sum2(tm, part, buf, rr, bb);
    T err = sqrt(s2.x);
    const T normb = sqrt(s2.y);
    int maxit = m, ret = restarts * m;
    for (int k = 0; k < restarts; k++) {
        {
            const T inv = T(1) / err;
            for (int e = tid; e < n; e += ts) V[e] = inv * V[e];
        }
        if (tid == 0) st.g[0] = mk<T>(err, T(0));
        for (int j = 0; j < m; j++) {
            if (E) eng_count(*E, cnt_level, cnt_what);
            cx<T>* Vj = V + (long long)j * n;
            cx<T>* Zj = (Z == V) ? Vj : Z + (long long)j * n;
            pre(j, Vj, Zj);
            op(Zj, w);
            for (int i = 0; i <= j; i++) {
                const cx<T>* Vi = V + (long long)i * n;
                T ax = 0, ay = 0;
                for (int e = tid; e < n; e += ts) {
                    const cx<T> u = w[e], vv = Vi[e];
                    ax += u.x * vv.x + u.y * vv.y;
                    ay += u.y * vv.x - u.x * vv.y;
                }
                const cx<T> h = team_sum2(tm, part, buf, ax, ay);
                if (tid == 0) st.H[i * m + j] = h;
                for (int e = tid; e < n; e += ts) {
                    cx<T> ww = w[e];
                    cfma(ww, -h, Vi[e]);
                    w[e] = ww;
                }
            }
            T nn = 0;
            for (int e = tid; e < n; e += ts) nn += cnorm2(w[e]);
            const T hn = sqrt(team_sum2(tm, part, buf, nn, T(0)).x);
            if (hn > T(0)) {
                const T inv = T(1) / hn;
                cx<T>* Vn = V + (long long)(j + 1) * n;
                for (int e = tid; e < n; e += ts) Vn[e] = inv * w[e];
            }
            // rotation(j) (src/fgmres.cpp:90-104) by the team's first thread
            if (tid == 0) {
                cx<T>* H = st.H;
                H[(j + 1) * m + j] = mk<T>(hn, T(0));
                for (int i = 0; i < j; i++) {
                    const cx<T> hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
                    const cx<T> temp = cmulc(st.cn[i], hij) + cmulc(st.sn[i], hi1);
                    H[(i + 1) * m + j] = cmul(st.cn[i], hi1) - cmul(st.sn[i], hij);
                    H[i * m + j] = temp;
                }
                const cx<T> hjj = H[j * m + j], hj1 = H[(j + 1) * m + j];
                const T den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                st.sn[j] = mk<T>(hj1.x / den, hj1.y / den);
                st.cn[j] = mk<T>(hjj.x / den, hjj.y / den);
                H[j * m + j] = cmulc(st.cn[j], hjj) + cmulc(st.sn[j], hj1);
                H[(j + 1) * m + j] = czero<T>();
                const cx<T> gj = st.g[j];
                st.g[j + 1] = -cmul(st.sn[j], gj);
                st.g[j] = cmulc(st.cn[j], gj);
                st.arn[0] = (sqrt(cnorm2(st.g[j + 1])) < tol * normb) ? 0 : 1;
            }
            team_sync(tm);
            if (st.arn[0] == 0) {
                maxit = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115)
        if (tid == 0) {
            for (int i = maxit - 1; i >= 0; i--) {
                cx<T> o = st.g[i];
                for (int jj = i + 1; jj < maxit; jj++) o -= cmul(st.H[i * m + jj], st.eta[jj]);
                st.eta[i] = cdiv(o, st.H[i * m + i]);
            }
        }
        team_sync(tm);
        for (int e = tid; e < n; e += ts) {
            cx<T> acc = x[e];
            for (int jj = 0; jj < maxit; jj++) {
                const cx<T>* Zq = (Z == V) ? V + (long long)jj * n : Z + (long long)jj * n;
                cfma(acc, st.eta[jj], Zq[e]);
            }
            x[e] = acc;
        }
        // true residual into V0
        op(x, w);
        rr = 0;
        for (int e = tid; e < n; e += ts) {
            const cx<T> r = b[e] - w[e];
            V[e] = r;
            rr += cnorm2(r);
        }
        err = sqrt(team_sum2(tm, part, buf, rr, T(0)).x);
        if (err < tol * normb) {
            ret = k * m + maxit;
            break;
        }
    }
    return ret;
}

// SAP_level_l::D_local (src/level.cpp:304-368) for one block, by one team: out[m][i] for the
// block's sites m (local order) from in[m][j]; neighbours outside the block are dropped.
template <typename T>
__device__ void dlocal_block(const Team& tm, const EngLevel<T>& L, T m0, int block, const cx<T>* in, cx<T>* out) {
    const int K = L.K, sxe = L.sxe, ste = L.ste, sbt = L.sbt, lnx = L.nx, lnt = L.nt, spb = sxe * ste, n = spb * K;
    const cx<T>* const links = L.links;
    const T mass = m0 + T(2);
    const int bxi = block / sbt, bti = block - bxi * sbt;
    const int g = tm.tid % kTPR, rows_per_pass = tm.size / kTPR;
    for (int rb = 0; rb < n; rb += rows_per_pass) {
        const int e = rb + tm.tid / kTPR;
        const bool on = e < n;
        cx<T> acc = czero<T>();
        if (on) {
            const int m = e / K, i = e - m * K;
            const int mx = m / ste, mt = m - mx * ste;
            const int x = bxi * sxe + mx, t = bti * ste + mt;
            const int xs = x * lnt + t;
            const cx<T>* lk = links + (long long)xs * 5 * K * K + i;
#pragma unroll 1
            for (int h = 0; h < 5; h++) {
                int nx_ = x, nt_ = t;
                switch (h) {
                    case HOP_R0: nt_ = (t + 1 == lnt) ? 0 : t + 1; break;
                    case HOP_R1: nx_ = (x + 1 == lnx) ? 0 : x + 1; break;
                    case HOP_L0: nt_ = (t == 0) ? lnt - 1 : t - 1; break;
                    case HOP_L1: nx_ = (x == 0) ? lnx - 1 : x - 1; break;
                    default: break;
                }
                const int nbx = nx_ / sxe, nbt = nt_ / ste;
                if (nbx * sbt + nbt != block) continue;
                const int ml = (nx_ - nbx * sxe) * ste + (nt_ - nbt * ste);
                const cx<T>* v = in + (long long)ml * K;
                const cx<T>* a = lk + (long long)h * K * K;
                cx<T> s = czero<T>();
#pragma unroll 4
                for (int j = g; j < K; j += kTPR) cfma(s, __ldg(a + (long long)j * K), v[j]);
                if (hop_sign(t, lnt, h) < 0) acc -= s; else acc += s;
            }
        }
        acc = tpr_sum<T>(acc);
        if (on && g == 0) out[e] = mass * in[e] - acc;
    }
}

// SAP_C::SAP (src/sap.cpp:64-174) on coarse level l: nu red/black sweeps; the blocks of a
// colour are spread over the teams of every CTA of the cluster (first one per CTA), each
// team runs the block GMRES with its vectors in its own shared-memory area, the block
// solutions are broadcast to every CTA, and the residual update is shared.  Returns 1 if
// ||v - D x|| < sap_tol * ||v||.
template <typename T>
__device__ __noinline__ int eng_sap(const Eng<T>& E, int l, const cx<T>* v, cx<T>* x, int nu) {
    const EngLevel<T>& L = E.L(l);
    const EngParams<T>& p = E.a->p;
    const int nvec = L.n * L.K;
    const int spb = L.sxe * L.ste, seglen = spb * L.K, ncol = L.ncol, m = p.sap_m;
    cx<T>* r = E.work(L.off_sap);
    cx<T>* xall = r + nvec;                                   // [ncol][seglen]
    const Team cta = whole_cta();
    T* cpart = E.red;
    int cbuf = 0;
    const int nteam = L.sap_nteam, tsize = blockDim.x / nteam, team = threadIdx.x / tsize;
    const Team tm{(int)threadIdx.x - team * tsize, tsize, tsize >> 5, team + 1};
    char* tsm = E.smem + E.a->smem_team + team * E.a->team_bytes;
    const GmState<T> st = gm_state_at<T>(tsm, 1, m);
    T* tpart = reinterpret_cast<T*>(tsm + gm_state_bytes(1, m, sizeof(T)));
    cx<T>* tv = L.sap_vec_smem ? reinterpret_cast<cx<T>*>(tsm + gm_state_bytes(1, m, sizeof(T)) + 64 * sizeof(T))
                               : E.work(L.off_sapteam) + (long long)team * (m + 4) * seglen;
    cx<T>* bv = tv;
    cx<T>* xv = bv + seglen;
    cx<T>* wv = xv + seglen;
    cx<T>* Vv = wv + seglen;

    eng_count(E, l, CNT_SAP_CALL);
    T vv = 0;
    for (int e = threadIdx.x; e < nvec; e += blockDim.x) vv += cnorm2(v[e]);
    const T vnorm = sqrt(team_sum2(cta, cpart, cbuf, vv, T(0)).x);
    dc_apply(E, L, p.m0, x, r);
    for (int e = threadIdx.x; e < nvec; e += blockDim.x) r[e] = v[e] - r[e];
    const int nslot = E.csize * nteam, slot = team * E.csize + E.crank;
    for (int it = 0; it < nu; it++) {
        for (int colour = 0; colour < 2; colour++) {
            const int* blocks = colour == 0 ? L.red : L.black;
            __syncthreads();                                  // r complete before the gathers
            for (int bi = slot; bi < ncol; bi += nslot) {
                const int block = blocks[bi];
                const int bxi = block / L.sbt, bti = block - bxi * L.sbt;
                for (int e = tm.tid; e < seglen; e += tm.size) {
                    const int mm = e / L.K, i = e - mm * L.K;
                    const int mx = mm / L.ste, mt = mm - mx * L.ste;
                    bv[e] = r[(long long)((bxi * L.sxe + mx) * L.nt + bti * L.ste + mt) * L.K + i];
                }
                auto lop = [&](const cx<T>* in, cx<T>* out) {
                    team_sync(tm);
                    dlocal_block(tm, L, p.m0, block, in, out);
                    team_sync(tm);
                };
                auto ident = [](int, const cx<T>*, cx<T>*) {};
                team_fgmres(tm, tpart, &E, l, CNT_SAP_STEP, lop, ident, bv, xv, Vv, Vv, wv, st, seglen, m,
                            p.sap_restarts, p.sap_gmres_tol);
                // broadcast the block solution to every CTA of the cluster
                const Part P = part_of(E);
                for (int e = tm.tid; e < seglen; e += tm.size) part_store<T>(P, xall + (long long)bi * seglen, e, xv[e]);
                team_sync(tm);
            }
            if (E.csize > 1) cluster_barrier(); else __syncthreads();
            // x += solutions of this colour (every CTA, its own copy)
            for (int e = threadIdx.x; e < ncol * seglen; e += blockDim.x) {
                const int s = e / seglen, q = e - s * seglen, mm = q / L.K, i = q - mm * L.K;
                const int block = blocks[s];
                const int bxi = block / L.sbt, bti = block - bxi * L.sbt;
                const int mx = mm / L.ste, mt = mm - mx * L.ste;
                x[(long long)((bxi * L.sxe + mx) * L.nt + bti * L.ste + mt) * L.K + i] += xall[e];
            }
            dc_apply(E, L, p.m0, x, r);
            for (int e = threadIdx.x; e < nvec; e += blockDim.x) r[e] = v[e] - r[e];
        }
        T rr = 0;
        for (int e = threadIdx.x; e < nvec; e += blockDim.x) rr += cnorm2(r[e]);
        const T err = sqrt(team_sum2(cta, cpart, cbuf, rr, T(0)).x);
        if (err < p.sap_tol * vnorm) return 1;
    }
    __syncthreads();
    return 0;
}

// Level::GMRES_level_l::fgmres(eta, eta, psi) (include/level.h:66-85); on the coarsest level
// this is the coarse solve of the cycles (src/amg.cpp:136-139)
template <typename T>
__device__ __noinline__ int eng_coarse_gmres(const Eng<T>& E, int l, const cx<T>* b, cx<T>* x) {
    const EngLevel<T>& L = E.L(l);
    const EngParams<T>& p = E.a->p;
    const int nvec = L.n * L.K;
    cx<T>* V = E.work(L.off_cg);
    cx<T>* w = V + (long long)(L.gm_m + 1) * nvec;
    const GmState<T> st = gm_state_at<T>(E.smem + L.sm_cg, 1, L.gm_m);
    const Team cta = whole_cta();
    auto op = [&](const cx<T>* in, cx<T>* out) { dc_apply(E, L, p.m0, in, out); };
    auto ident = [](int, const cx<T>*, cx<T>*) {};
    const int it = team_fgmres(cta, E.red, &E, l, CNT_GMRES_STEP, op, ident, b, x, V, V, w, st, nvec, L.gm_m,
                               L.gm_restarts, L.gm_tol);
    __syncthreads();
    return it;
}

template <typename T, int D> struct Cycles;

template <typename T>
struct Cycles<T, 0> {
    __device__ static void kcycle(const Eng<T>& E, int, const cx<T>*, cx<T>*) { if (threadIdx.x == 0) atomicOr(E.a->flags, 1); __syncthreads(); }
    __device__ static int kfgmres(const Eng<T>& E, int, const cx<T>*, cx<T>*) { if (threadIdx.x == 0) atomicOr(E.a->flags, 1); __syncthreads(); return 0; }
    __device__ static void vcycle(const Eng<T>& E, int, const cx<T>*, cx<T>*) { if (threadIdx.x == 0) atomicOr(E.a->flags, 1); __syncthreads(); }
};

template <typename T, int D>
struct Cycles {
    // AlgebraicMG::k_cycle (src/amg.cpp:135-178); psi is accumulated into
    __device__ static void kcycle(const Eng<T>& E, int l, const cx<T>* eta, cx<T>* psi) {
        if (E.L(l).coarsest) { eng_coarse_gmres(E, l, eta, psi); return; }
        const EngLevel<T>& L = E.L(l);
        const EngLevel<T>& Ln = E.L(l + 1);
        const EngParams<T>& p = E.a->p;
        const int nvec = L.n * L.K, ncv = Ln.n * Ln.K;
        cx<T>* r = E.work(L.off_cyc);
        cx<T>* etac = r + nvec;
        cx<T>* psic = etac + ncv;
        if (p.nu1 > 0) eng_sap(E, l, eta, psi, p.nu1);
        dc_apply(E, L, p.m0, psi, r);
        v_sub<T>(r, eta, r, nvec);
        restrict_v(E, L, r, etac);
        Cycles<T, D - 1>::kfgmres(E, l + 1, etac, psic);
        prolong_v(E, L, psic, psi, 1);
        if (p.nu2 > 0) eng_sap(E, l, eta, psi, p.nu2);
    }
    // AlgebraicMG::v_cycle (src/amg.cpp:90-132)
    __device__ static void vcycle(const Eng<T>& E, int l, const cx<T>* eta, cx<T>* psi) {
        if (E.L(l).coarsest) { eng_coarse_gmres(E, l, eta, psi); return; }
        const EngLevel<T>& L = E.L(l);
        const EngLevel<T>& Ln = E.L(l + 1);
        const EngParams<T>& p = E.a->p;
        const int nvec = L.n * L.K, ncv = Ln.n * Ln.K;
        cx<T>* r = E.work(L.off_cyc);
        cx<T>* etac = r + nvec;
        cx<T>* psic = etac + ncv;
        if (p.nu1 > 0) eng_sap(E, l, eta, psi, p.nu1);
        dc_apply(E, L, p.m0, psi, r);
        v_sub<T>(r, eta, r, nvec);
        restrict_v(E, L, r, etac);
        v_zero<T>(psic, ncv);
        Cycles<T, D - 1>::vcycle(E, l + 1, etac, psic);
        prolong_v(E, L, psic, psi, 1);
        if (p.nu2 > 0) eng_sap(E, l, eta, psi, p.nu2);
    }
    // FGMRES_k_cycle of level l (include/amg.h:19-40): fgmres(b, x0 = b, x) with
    // func = D_l and preconditioner k_cycle(l, V_j, Z_j) accumulating into Z_j.
    __device__ static int kfgmres(const Eng<T>& E, int l, const cx<T>* b, cx<T>* x) {
        const EngLevel<T>& L = E.L(l);
        const EngParams<T>& p = E.a->p;
        const int nvec = L.n * L.K;
        cx<T>* V = E.work(L.off_kfg);
        cx<T>* Z = V + (long long)(p.k_m + 1) * nvec;
        cx<T>* w = Z + (long long)p.k_m * nvec;
        const GmState<T> st = gm_state_at<T>(E.smem + L.sm_kfg, 1, p.k_m);
        const Team cta = whole_cta();
        auto op = [&](const cx<T>* in, cx<T>* out) { dc_apply(E, L, p.m0, in, out); };
        auto pre = [&](int, const cx<T>* v, cx<T>* z) { Cycles<T, D>::kcycle(E, l, v, z); };
        const int it = team_fgmres(cta, E.red, &E, l, CNT_KFG_STEP, op, pre, b, x, V, Z, w, st, nvec, p.k_m,
                                   p.k_restarts, p.k_tol);
        __syncthreads();
        return it;
    }
};

}  // namespace amgb
