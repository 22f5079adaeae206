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
    int smem_red;                // byte offset of the reduction scratch
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
// segmented vector space: nseg segments of seglen complex entries, contiguous
// ---------------------------------------------------------------------------------
template <typename T>
struct Seg {
    int nseg, seglen, tps;       // threads per segment (power of two)
    T* red;                      // shared scratch [2 * blockDim.x / 32]
};

template <typename T>
__device__ inline Seg<T> make_seg(int nseg, int seglen, T* red) {
    Seg<T> s;
    s.nseg = nseg; s.seglen = seglen; s.red = red;
    int tps = blockDim.x / nseg;
    int p = 1;
    while (p * 2 <= tps) p *= 2;
    s.tps = p;
    return s;
}

// res[s] = sum_e a[e] * conj(b[e]) over segment s (the reference's dot, include/lin_alg_op.h:32-40)
template <typename T>
__device__ void seg_dot(const Seg<T>& sp, const cx<T>* a, const cx<T>* b, cx<T>* res) {
    const int tid = threadIdx.x;
    const int grp = tid / sp.tps, q = tid % sp.tps;
    T ax = 0, ay = 0;
    if (grp < sp.nseg) {
        const cx<T>* pa = a + (long long)grp * sp.seglen;
        const cx<T>* pb = b + (long long)grp * sp.seglen;
        for (int e = q; e < sp.seglen; e += sp.tps) {
            cx<T> u = pa[e], v = pb[e];
            ax += u.x * v.x + u.y * v.y;
            ay += u.y * v.x - u.x * v.y;
        }
    }
    const int w = (sp.tps < 32) ? sp.tps : 32;
    for (int o = w / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (sp.tps <= 32) {
        __syncthreads();
        if (grp < sp.nseg && q == 0) res[grp] = mk<T>(ax, ay);
        __syncthreads();
        return;
    }
    const int lane = tid & 31, wid = tid >> 5;
    __syncthreads();
    if (lane == 0) { sp.red[2 * wid] = ax; sp.red[2 * wid + 1] = ay; }
    __syncthreads();
    if (grp < sp.nseg && q == 0) {
        const int wpg = sp.tps / 32;
        T sx = 0, sy = 0;
        for (int k = 0; k < wpg; k++) { sx += sp.red[2 * (grp * wpg + k)]; sy += sp.red[2 * (grp * wpg + k) + 1]; }
        res[grp] = mk<T>(sx, sy);
    }
    __syncthreads();
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
template <typename T>
__device__ __forceinline__ void part_store(const Eng<T>& E, cx<T>* out, int e, cx<T> v) {
    if (E.csize == 1) { out[e] = v; return; }
    const long long slab = E.a->slab;
    for (int q = 0; q < E.csize; q++) out[(long long)(q - E.crank) * slab + e] = v;
}
template <typename T>
__device__ __forceinline__ void part_begin(const Eng<T>& E) {
    if (E.csize > 1) cluster_barrier();
}
template <typename T>
__device__ __forceinline__ void part_end(const Eng<T>& E) {
    if (E.csize > 1) cluster_barrier();
    else __syncthreads();
}

// Level::D_operator (src/level.cpp:161-180) for l >= 1:
// out = (m0+2) in - sum_hop sign * G_hop in(neighbour).  With a cluster, every CTA computes
// a slice of the rows and stores it into every CTA's copy of `out`.
template <typename T>
__device__ __noinline__ void dc_apply(const Eng<T>& E, const EngLevel<T>& L, T m0, const cx<T>* in, cx<T>* out) {
    const int K = L.K, tot = L.n * K;
    const T mass = m0 + T(2);
    int e0, e1;
    eng_count(E, L.level, CNT_APPLY);
    part_range(E, tot, e0, e1);
    part_begin(E);
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int xs = e / K, i = e - xs * K;
        const int x = xs / L.nt, t = xs - x * L.nt;
        cx<T> acc = czero<T>();
        const cx<T>* lk = L.links + (long long)xs * 5 * K * K + i;
#pragma unroll 1
        for (int h = 0; h < 5; h++) {
            const int nbs = nb_site(x, t, L.nx, L.nt, h);
            const cx<T>* v = in + (long long)nbs * K;
            const cx<T>* a = lk + (long long)h * K * K;
            cx<T> s = czero<T>();
            for (int j = 0; j < K; j++) cfma(s, a[(long long)j * K], v[j]);
            if (hop_sign(t, L.nt, h) < 0) acc -= s; else acc += s;
        }
        cx<T> self = in[e];
        part_store(E, out, e, mass * self - acc);
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

// SAP_level_l::D_local (src/level.cpp:304-368) on all blocks of one colour at once:
// in/out are [ncol][spb][K]; neighbours outside the block are dropped.
template <typename T>
__device__ __noinline__ void dlocal_apply(const Eng<T>& E, const EngLevel<T>& L, T m0, const int* blocks, int nblk,
                                          const cx<T>* in, cx<T>* out) {
    const int K = L.K, spb = L.sxe * L.ste, seglen = spb * K, tot = nblk * seglen;
    const T mass = m0 + T(2);
    int e0, e1;
    eng_count(E, L.level, CNT_LOCAL_APPLY);
    part_range(E, tot, e0, e1);
    part_begin(E);
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int seg = e / seglen, r = e - seg * seglen;
        const int m = r / K, i = r - m * K;
        const int block = blocks[seg];
        int x, t;
        const int xs = sap_site(L, block, m, &x, &t);
        const cx<T>* lk = L.links + (long long)xs * 5 * K * K + i;
        const cx<T>* base = in + (long long)seg * seglen;
        cx<T> acc = czero<T>();
#pragma unroll 1
        for (int h = 0; h < 5; h++) {
            int nx_ = x, nt_ = t;
            switch (h) {
                case HOP_R0: nt_ = (t + 1 == L.nt) ? 0 : t + 1; break;
                case HOP_R1: nx_ = (x + 1 == L.nx) ? 0 : x + 1; break;
                case HOP_L0: nt_ = (t == 0) ? L.nt - 1 : t - 1; break;
                case HOP_L1: nx_ = (x == 0) ? L.nx - 1 : x - 1; break;
                default: break;
            }
            const int nbx = nx_ / L.sxe, nbt = nt_ / L.ste;
            if (nbx * L.sbt + nbt != block) continue;
            const int ml = (nx_ - nbx * L.sxe) * L.ste + (nt_ - nbt * L.ste);
            const cx<T>* v = base + (long long)ml * K;
            const cx<T>* a = lk + (long long)h * K * K;
            cx<T> s = czero<T>();
            for (int j = 0; j < K; j++) cfma(s, a[(long long)j * K], v[j]);
            if (hop_sign(t, L.nt, h) < 0) acc -= s; else acc += s;
        }
        part_store(E, out, e, mass * base[r] - acc);
    }
    part_end(E);
}

// gather / scatter between a level vector and the colour's block segments
template <typename T>
__device__ void sap_gather(const EngLevel<T>& L, const int* blocks, int nblk, const cx<T>* v, cx<T>* seg) {
    const int K = L.K, spb = L.sxe * L.ste, seglen = spb * K, tot = nblk * seglen;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int s = e / seglen, r = e - s * seglen, m = r / K, i = r - m * K;
        int x, t;
        const int xs = sap_site(L, blocks[s], m, &x, &t);
        seg[e] = v[(long long)xs * K + i];
    }
    __syncthreads();
}
template <typename T>
__device__ void sap_scatter_add(const EngLevel<T>& L, const int* blocks, int nblk, const cx<T>* seg, cx<T>* v) {
    const int K = L.K, spb = L.sxe * L.ste, seglen = spb * K, tot = nblk * seglen;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int s = e / seglen, r = e - s * seglen, m = r / K, i = r - m * K;
        int x, t;
        const int xs = sap_site(L, blocks[s], m, &x, &t);
        v[(long long)xs * K + i] += seg[e];
    }
    __syncthreads();
}

// Level::Pt_v (src/level.cpp:212-237): out[nc][2cc+s] = sum_{n in nc, c} conj(W_cc[n][2c+s]) v[n][2c+s]
template <typename T>
__device__ __noinline__ void restrict_v(const Eng<T>& E, const EngLevel<T>& L, const cx<T>* v, cx<T>* out) {
    const int K = L.K, col = K / 2, nblk = L.bx * L.bt, tot = nblk * 2 * L.ntest;
    int e0, e1;
    part_range(E, tot, e0, e1);
    part_begin(E);
    for (int o = e0 + threadIdx.x; o < e1; o += blockDim.x) {
        const int nc = o / (2 * L.ntest), r = o - nc * 2 * L.ntest, cc = r >> 1, s = r & 1;
        const int bxi = nc / L.bt, bti = nc - bxi * L.bt;
        const cx<T>* w = L.W + (long long)cc * L.n * K;
        cx<T> acc = czero<T>();
        for (int mx = 0; mx < L.xe; mx++)
            for (int mt = 0; mt < L.te; mt++) {
                const long long n = (long long)(bxi * L.xe + mx) * L.nt + (bti * L.te + mt);
                for (int c = 0; c < col; c++) cfmac(acc, w[n * K + 2 * c + s], v[n * K + 2 * c + s]);
            }
        part_store(E, out, o, acc);
    }
    part_end(E);
}

// out (+)= P vc: Level::P_v (src/level.cpp:182-209), out[n][2c+s] = sum_cc W_cc[n][2c+s] vc[nc][2cc+s]
template <typename T>
__device__ __noinline__ void prolong_v(const Eng<T>& E, const EngLevel<T>& L, const cx<T>* vc, cx<T>* out,
                                       int accumulate) {
    const int K = L.K, tot = L.n * K;
    int e0, e1;
    part_range(E, tot, e0, e1);
    part_begin(E);
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int n = e / K, d = e - n * K, s = d & 1;
        const int x = n / L.nt, t = n - x * L.nt;
        const int nc = (x / L.xe) * L.bt + (t / L.te);
        const cx<T>* pv = vc + (long long)nc * 2 * L.ntest + s;
        cx<T> acc = czero<T>();
        for (int cc = 0; cc < L.ntest; cc++) cfma(acc, L.W[(long long)cc * L.n * K + e], pv[2 * cc]);
        part_store(E, out, e, accumulate ? out[e] + acc : acc);
    }
    part_end(E);
}

// ---------------------------------------------------------------------------------
// FGMRES (src/fgmres.cpp:5-115) for nseg independent segments, x0 = b (the only start the
// multigrid uses below the fine level: src/amg.cpp:138, :161, src/sap.cpp:61).
// op(in, out) applies the operator to all segments; pre(j) fills Z_j from V_j (Z may
// alias V for the identity preconditioner).  Per segment it follows the reference:
// modified Gram-Schmidt, Givens rotations, Arnoldi exit on |g_{j+1}| < tol*||b||, a true
// residual after each cycle, and maxIt carried over restart cycles.
// Returns in st.iters[s] the reference's return value (k*m + maxIt or restarts*m).
// ---------------------------------------------------------------------------------
template <typename T, class Op, class Pre>
__device__ void seg_fgmres(const Eng<T>* E, int cnt_level, int cnt_what, const Seg<T>& sp, Op& op, Pre& pre,
                           const cx<T>* b, cx<T>* x, cx<T>* V, cx<T>* Z, cx<T>* w, const GmState<T>& st, int m,
                           int restarts, T tol) {
    const int nseg = sp.nseg, seglen = sp.seglen, tot = nseg * seglen;
    const long long vstride = tot;
    const int tid = threadIdx.x;
    // setZeros (include/fgmres.h:93-120): H, g, V, Z are zero at the start of every call
    for (int e = tid; e < nseg * (m + 1) * m; e += blockDim.x) st.H[e] = czero<T>();
    for (int e = tid; e < nseg * (m + 1); e += blockDim.x) st.g[e] = czero<T>();
    for (int e = tid; e < nseg * m; e += blockDim.x) { st.cn[e] = czero<T>(); st.sn[e] = czero<T>(); st.eta[e] = czero<T>(); }
    for (long long e = tid; e < (long long)(m + 1) * vstride; e += blockDim.x) V[e] = czero<T>();
    if (Z != V)
        for (long long e = tid; e < (long long)m * vstride; e += blockDim.x) Z[e] = czero<T>();
    // x = x0 = b; r = b - A x into V0
    for (int e = tid; e < tot; e += blockDim.x) x[e] = b[e];
    __syncthreads();
    op(x, w);
    for (int e = tid; e < tot; e += blockDim.x) V[e] = b[e] - w[e];
    __syncthreads();
    seg_dot(sp, V, V, st.red);
    for (int s = tid; s < nseg; s += blockDim.x) {
        st.err[s] = sqrt(st.red[s].x);
        st.maxit[s] = m;
        st.act[s] = 1;
        st.iters[s] = restarts * m;
    }
    __syncthreads();
    seg_dot(sp, b, b, st.red);
    for (int s = tid; s < nseg; s += blockDim.x) st.normb[s] = sqrt(st.red[s].x);
    __syncthreads();

    for (int k = 0; k < restarts; k++) {
        int any = 0;
        for (int s = 0; s < nseg; s++) any |= st.act[s];
        if (!any) break;
        // V0 = r / beta, g0 = beta
        for (int s = tid; s < nseg; s += blockDim.x) {
            st.arn[s] = st.act[s];
            if (st.act[s]) st.g[s * (m + 1)] = mk<T>(st.err[s], T(0));
        }
        for (int e = tid; e < tot; e += blockDim.x) {
            const int s = e / seglen;
            if (st.act[s]) { T inv = T(1) / st.err[s]; V[e] = inv * V[e]; }
        }
        __syncthreads();
        for (int j = 0; j < m; j++) {
            int anyarn = 0;
            for (int s = 0; s < nseg; s++) anyarn |= st.arn[s];
            if (!anyarn) break;
            if (E) eng_count(*E, cnt_level, cnt_what);
            cx<T>* Vj = V + (long long)j * vstride;
            cx<T>* Zj = (Z == V) ? Vj : Z + (long long)j * vstride;
            pre(j, Vj, Zj, st.arn);
            op(Zj, w);
            for (int i = 0; i <= j; i++) {
                const cx<T>* Vi = V + (long long)i * vstride;
                seg_dot(sp, w, Vi, st.red);
                for (int s = tid; s < nseg; s += blockDim.x)
                    if (st.arn[s]) st.H[s * (m + 1) * m + i * m + j] = st.red[s];
                for (int e = tid; e < tot; e += blockDim.x) {
                    const int s = e / seglen;
                    if (st.arn[s]) { cx<T> h = st.red[s]; cx<T> vv = Vi[e]; cx<T> ww = w[e]; cfma(ww, -h, vv); w[e] = ww; }
                }
                __syncthreads();
            }
            seg_dot(sp, w, w, st.red);
            for (int e = tid; e < tot; e += blockDim.x) {
                const int s = e / seglen;
                const T h = sqrt(st.red[s].x);
                if (st.arn[s] && h > T(0)) { T inv = T(1) / h; V[(long long)(j + 1) * vstride + e] = inv * w[e]; }
            }
            __syncthreads();
            // rotation(j) (src/fgmres.cpp:90-104) and the g update, one thread per segment
            for (int s = tid; s < nseg; s += blockDim.x) {
                if (!st.arn[s]) continue;
                cx<T>* H = st.H + s * (m + 1) * m;
                cx<T>* cn = st.cn + s * m;
                cx<T>* sn = st.sn + s * m;
                cx<T>* g = st.g + s * (m + 1);
                H[(j + 1) * m + j] = mk<T>(sqrt(st.red[s].x), T(0));
                for (int i = 0; i < j; i++) {
                    cx<T> hij = H[i * m + j], hi1 = H[(i + 1) * m + j];
                    cx<T> temp = cmulc(cn[i], hij) + cmulc(sn[i], hi1);
                    H[(i + 1) * m + j] = cmul(cn[i], hi1) - cmul(sn[i], hij);
                    H[i * m + j] = temp;
                }
                cx<T> hjj = H[j * m + j], hj1 = H[(j + 1) * m + j];
                const T den = sqrt(cnorm2(hjj) + cnorm2(hj1));
                sn[j] = mk<T>(hj1.x / den, hj1.y / den);
                cn[j] = mk<T>(hjj.x / den, hjj.y / den);
                H[j * m + j] = cmulc(cn[j], hjj) + cmulc(sn[j], hj1);
                H[(j + 1) * m + j] = czero<T>();
                cx<T> gj = g[j];
                g[j + 1] = -cmul(sn[j], gj);
                g[j] = cmulc(cn[j], gj);
                const cx<T> gj1 = g[j + 1];
                if (sqrt(cnorm2(gj1)) < tol * st.normb[s]) {
                    st.maxit[s] = j + 1;
                    st.arn[s] = 0;
                }
            }
            __syncthreads();
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115)
        for (int s = tid; s < nseg; s += blockDim.x) {
            if (!st.act[s]) continue;
            const cx<T>* H = st.H + s * (m + 1) * m;
            const cx<T>* g = st.g + s * (m + 1);
            cx<T>* eta = st.eta + s * m;
            const int n = st.maxit[s];
            for (int i = n - 1; i >= 0; i--) {
                cx<T> o = g[i];
                for (int jj = i + 1; jj < n; jj++) o -= cmul(H[i * m + jj], eta[jj]);
                eta[i] = cdiv(o, H[i * m + i]);
            }
        }
        __syncthreads();
        // x += sum_j eta_j Z_j
        for (int e = tid; e < tot; e += blockDim.x) {
            const int s = e / seglen;
            if (!st.act[s]) continue;
            const cx<T>* eta = st.eta + s * m;
            cx<T> acc = x[e];
            const int n = st.maxit[s];
            for (int jj = 0; jj < n; jj++) {
                const cx<T>* Zj = (Z == V) ? V + (long long)jj * vstride : Z + (long long)jj * vstride;
                cfma(acc, eta[jj], Zj[e]);
            }
            x[e] = acc;
        }
        __syncthreads();
        // true residual into V0
        op(x, w);
        for (int e = tid; e < tot; e += blockDim.x) {
            const int s = e / seglen;
            if (st.act[s]) V[e] = b[e] - w[e];
        }
        __syncthreads();
        seg_dot(sp, V, V, st.red);
        for (int s = tid; s < nseg; s += blockDim.x) {
            if (!st.act[s]) continue;
            st.err[s] = sqrt(st.red[s].x);
            if (st.err[s] < tol * st.normb[s]) {
                st.iters[s] = k * m + st.maxit[s];
                st.act[s] = 0;
            }
        }
        __syncthreads();
    }
}



// SAP_C::SAP (src/sap.cpp:64-174) on coarse level l: nu red/black sweeps of block GMRES,
// every block of a colour solved; returns 1 if ||v - D x|| < sap_tol * ||v||.
template <typename T>
__device__ __noinline__ int eng_sap(const Eng<T>& E, int l, const cx<T>* v, cx<T>* x, int nu) {
    const EngLevel<T>& L = E.L(l);
    const EngParams<T>& p = E.a->p;
    const int nvec = L.n * L.K;
    const int spb = L.sxe * L.ste, seglen = spb * L.K, nseg = L.ncol, segtot = nseg * seglen;
    cx<T>* r = E.work(L.off_sap);
    cx<T>* bseg = r + nvec;
    cx<T>* xseg = bseg + segtot;
    cx<T>* wseg = xseg + segtot;
    cx<T>* Vseg = wseg + segtot;
    GmState<T> st = gm_state_at<T>(E.smem + L.sm_sap, nseg, p.sap_m);
    Seg<T> sp1 = make_seg<T>(1, nvec, E.red);
    Seg<T> sps = make_seg<T>(nseg, seglen, E.red);

    eng_count(E, l, CNT_SAP_CALL);
    seg_dot(sp1, v, v, st.red);
    const T vnorm = sqrt(st.red[0].x);
    dc_apply(E, L, p.m0, x, r);
    v_sub<T>(r, v, r, nvec);
        for (int it = 0; it < nu; it++) {
        for (int colour = 0; colour < 2; colour++) {
            const int* blocks = colour == 0 ? L.red : L.black;
            sap_gather(L, blocks, nseg, r, bseg);
            auto lop = [&](const cx<T>* in, cx<T>* out) { dlocal_apply(E, L, p.m0, blocks, nseg, in, out); };
            auto ident = [](int, const cx<T>*, cx<T>*, const int*) {};
            seg_fgmres(&E, l, CNT_SAP_STEP, sps, lop, ident, bseg, xseg, Vseg, Vseg, wseg, st, p.sap_m, p.sap_restarts,
                       p.sap_gmres_tol);
            sap_scatter_add(L, blocks, nseg, xseg, x);
            dc_apply(E, L, p.m0, x, r);
            v_sub<T>(r, v, r, nvec);
        }
        seg_dot(sp1, r, r, st.red);
        const T err = sqrt(st.red[0].x);
        __syncthreads();
        if (err < p.sap_tol * vnorm) return 1;
    }
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
    GmState<T> st = gm_state_at<T>(E.smem + L.sm_cg, 1, L.gm_m);
    Seg<T> sp = make_seg<T>(1, nvec, E.red);
    auto op = [&](const cx<T>* in, cx<T>* out) { dc_apply(E, L, p.m0, in, out); };
    auto ident = [](int, const cx<T>*, cx<T>*, const int*) {};
    seg_fgmres(&E, l, CNT_GMRES_STEP, sp, op, ident, b, x, V, V, w, st, L.gm_m, L.gm_restarts, L.gm_tol);
    return st.iters[0];
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
        GmState<T> st = gm_state_at<T>(E.smem + L.sm_kfg, 1, p.k_m);
        Seg<T> sp = make_seg<T>(1, nvec, E.red);
        auto op = [&](const cx<T>* in, cx<T>* out) { dc_apply(E, L, p.m0, in, out); };
        auto pre = [&](int, const cx<T>* v, cx<T>* z, const int*) { Cycles<T, D>::kcycle(E, l, v, z); };
        seg_fgmres(&E, l, CNT_KFG_STEP, sp, op, pre, b, x, V, Z, w, st, p.k_m, p.k_restarts, p.k_tol);
        return st.iters[0];
    }
};

}  // namespace amgb
