// Fine-lattice (level 0) kernels: the U(1) Wilson-Dirac stencil, the fused residual,
// restriction / prolongation between level 0 and level 1, the SAP block solver and the
// BLAS-1 kernels of the outer FGMRES.
//
// Layout: psi[rhs][n][spin] complex (double2 or float2), n = x*Nt + t; U[n][mu].
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "kernels.h"
#include "stencil.cuh"
#include "dirac_tma.cuh"
#include "sap_lean.cuh"
#include "sap_f32.cuh"
#include "sap_ca.cuh"
#include "sap_h.cuh"
#include "tc_transfer.cuh"

namespace amgb {

// One thread per site; the sources rhs = blockIdx.y, blockIdx.y + gridDim.y, ... share the
// site's links, which are read from memory once per source group instead of once per
// source.
template <typename T, bool DAG>
__global__ void __launch_bounds__(256) k_dirac(const cx<T>* __restrict__ U, const cx<T>* __restrict__ in,
                                               cx<T>* __restrict__ out, int nx, int nt, T m0, int nrhs) {
    const int N = nx * nt;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const SiteOp<T> L = site_op<T>(U, n, nx, nt);
    for (int rhs = blockIdx.y; rhs < nrhs; rhs += gridDim.y) {
        const long long off = (long long)rhs * N * 2;
        cx<T> o0, o1;
        dirac_site<T, DAG>(L, in + off, n, m0 + T(2), o0, o1);
        out[off + 2 * n] = o0;
        out[off + 2 * n + 1] = o1;
    }
}

// out = D in in FP64 for FP32 spinors in (promoted exactly), with in copied to in_copy: the
// outer FGMRES's w = D z_j and its basis slot Z_j (kept in FP32) in one pass
__global__ void __launch_bounds__(256) k_dirac_promote(const double2* __restrict__ U, const float2* __restrict__ in,
                                                       double2* __restrict__ out, float2* __restrict__ in_copy, int nx,
                                                       int nt, double m0, int nrhs) {
    const int N = nx * nt;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const SiteOp<double> L = site_op<double>(U, n, nx, nt);
    for (int rhs = blockIdx.y; rhs < nrhs; rhs += gridDim.y) {
        const long long off = (long long)rhs * N * 2;
        double2 o0, o1;
        dirac_site<double, false, float>(L, in + off, n, m0 + 2.0, o0, o1);
        out[off + 2 * n] = o0;
        out[off + 2 * n + 1] = o1;
        in_copy[off + 2 * n] = in[off + 2 * n];
        in_copy[off + 2 * n + 1] = in[off + 2 * n + 1];
    }
}

// r = b - D x, and per-CTA partial sums of |r|^2 (deterministic second stage); sources
// grouped per thread as in k_dirac.  Inactive sources (act[rhs] == 0) are skipped.
template <typename T>
__global__ void __launch_bounds__(256) k_residual(const Links<T> U, const cx<T>* __restrict__ b,
                                                  long long bstride, const cx<T>* __restrict__ x,
                                                  cx<T>* __restrict__ r, int nx, int nt, T m0,
                                                  double* __restrict__ partial, const int* __restrict__ act,
                                                  int nrhs) {
    __shared__ double red[8];
    const int N = nx * nt;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    SiteOp<T> L;
    if (n < N) L = site_op<T>(U, n, nx, nt);
    for (int rhs = blockIdx.y; rhs < nrhs; rhs += gridDim.y) {
        if (act && !act[rhs]) continue;
        const long long off = (long long)rhs * N * 2;
        const cx<T>* bb = b + (long long)rhs * bstride;
        double nrm = 0;
        if (n < N) {
            cx<T> o0, o1;
            dirac_site<T, false>(L, x + off, n, m0 + T(2), o0, o1);
            const cx<T> r0 = bb[2 * n] - o0, r1 = bb[2 * n + 1] - o1;
            r[off + 2 * n] = r0;
            r[off + 2 * n + 1] = r1;
            nrm = (double)cnorm2(r0) + (double)cnorm2(r1);
        }
        if (partial) {
            nrm = cta_sum(nrm, red);
            if (threadIdx.x == 0) partial[(long long)rhs * gridDim.x + blockIdx.x] = nrm;
        }
    }
}

// out[rhs] = sum_k partial[rhs][k] in a fixed order
__global__ void k_sum_partials(const double* __restrict__ partial, int nparts, double* __restrict__ out) {
    __shared__ double red[32];
    double s = 0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += partial[(long long)blockIdx.x * nparts + k];
    s = cta_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------------
// Level::Pt_v at level 0 (src/level.cpp:212-237, colors = 1):
//   out[rhs][nc][2cc+s] = sum_{n in block nc} conj(W[cc][n][s]) v[rhs][n][s]
// Grid (chunk, block, rhs); per-chunk partials reduced by k_restrict0_sum in chunk order.
// ---------------------------------------------------------------------------------
// Multi-source form of the level-0 restriction: one CTA per (chunk of an aggregation
// block, block) serves every source, one warp per source at a time, so the chunk's test
// vectors come from DRAM once and from L1 for the other sources; each warp reduces its
// own source's 2*ntest sums with shuffles.
template <typename T, typename TW, int NV>
__global__ void __launch_bounds__(256) k_restrict0m(const TW* __restrict__ W, const cx<T>* __restrict__ v,
                                                    cx<T>* __restrict__ partial, int nx, int nt, int bt, int xe,
                                                    int te, int nchunk, int ntest, int nrhs) {
    const int N = nx * nt;
    const int chunk = blockIdx.x, nc = blockIdx.y;
    const int bxi = nc / bt, bti = nc - bxi * bt;
    const int spb = xe * te;
    const int per = (spb + nchunk - 1) / nchunk;
    const int q0 = chunk * per, q1 = min(spb, q0 + per);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int rhs = wid; rhs < nrhs; rhs += nw) {
        const cx<T>* vv = v + (long long)rhs * N * 2;
        cx<T> acc[NV][2];
#pragma unroll
        for (int k = 0; k < NV; k++) { acc[k][0] = czero<T>(); acc[k][1] = czero<T>(); }
        for (int q = q0 + lane; q < q1; q += 32) {
            const int mx = q / te, mt = q - mx * te;
            const long long n = (long long)(bxi * xe + mx) * nt + (bti * te + mt);
            const cx<T> p0 = vv[2 * n], p1 = vv[2 * n + 1];
#pragma unroll
            for (int k = 0; k < NV; k++) {
                if (k < ntest) {
                    const cx<T> w0 = ccast<T>(load_cx(W + ((long long)k * N + n) * 2));
                    const cx<T> w1 = ccast<T>(load_cx(W + ((long long)k * N + n) * 2 + 1));
                    cfmac(acc[k][0], w0, p0);
                    cfmac(acc[k][1], w1, p1);
                }
            }
        }
        cx<T>* out = partial + (((long long)rhs * gridDim.y + nc) * nchunk + chunk) * (2 * ntest);
#pragma unroll
        for (int k = 0; k < NV; k++) {
            if (k >= ntest) break;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const T xr = warp_sum(acc[k][s].x), xi = warp_sum(acc[k][s].y);
                if (lane == 0) out[2 * k + s] = mk<T>(xr, xi);
            }
        }
    }
}

// Tiled multi-source form: CTA (split, block) walks its share of the aggregation block's
// sites in tiles of kRtTile sites.  A tile's test vectors (converted to T) and sources are
// staged in shared memory with coalesced loads, laid out [site][spin][test vector] and
// [site][spin][source]; each thread then accumulates a 2 x 2 tile of outputs (two test
// vectors x two sources, one spin) over the sites of its site group, reading two adjacent
// pairs per site.  Site groups are summed in shared memory at the end; the partials have
// the layout of k_restrict0m, so k_restrict0_sum finishes both.
constexpr int kRtTile = 64;

__host__ __device__ inline int rt_out_tiles(int ntest, int nrhs) { return ((ntest + 1) / 2) * 2 * ((nrhs + 1) / 2); }

template <typename T>
inline int rt_smem_bytes(int ntest, int nrhs) {
    const int K2 = 2 * ((ntest + 1) / 2), R2 = 2 * ((nrhs + 1) / 2);
    const int tiles = kRtTile * (2 * K2 + 1 + 2 * R2 + 1);
    const int red = rt_out_tiles(ntest, nrhs) * 4 * (256 / rt_out_tiles(ntest, nrhs));
    return (tiles > red ? tiles : red) * (int)sizeof(cx<T>);
}

template <typename T, typename TW>
__global__ void __launch_bounds__(256) k_restrict0t(const TW* __restrict__ W, const cx<T>* __restrict__ v,
                                                    cx<T>* __restrict__ partial, int nx, int nt, int bt, int xe,
                                                    int te, int nsplit, int ntest, int nrhs) {
    extern __shared__ __align__(16) unsigned char smraw_t[];
    const int N = nx * nt;
    const int split = blockIdx.x, nc = blockIdx.y, nblk = gridDim.y;
    const int bxi = nc / bt, bti = nc - bxi * bt;
    const int spb = xe * te;
    // each split takes whole tiles (a split past the end takes none and writes zeros)
    const int per = ((spb + nsplit - 1) / nsplit + kRtTile - 1) / kRtTile * kRtTile;
    const int q0 = split * per, q1 = min(spb, q0 + per);
    const int KP = (ntest + 1) / 2, RP = (nrhs + 1) / 2, K2 = 2 * KP, R2 = 2 * RP;
    const int OT = KP * 2 * RP;
    const int G = blockDim.x / OT;
    cx<T>* Ws = reinterpret_cast<cx<T>*>(smraw_t);   // [kRtTile][2 * K2 + 1]
    // a site's row holds both spins plus one pad element, so the staging stores of
    // consecutive sites (one per thread) fall in different banks
    const int WR = 2 * K2 + 1, VR = 2 * R2 + 1;
    cx<T>* Vs = Ws + kRtTile * WR;                   // [kRtTile][2 * R2 + 1]
    const int tid = threadIdx.x;
    const bool active = tid < OT * G;
    const int ot = tid % OT, grp = tid / OT;
    const int kp = ot % KP, s = (ot / KP) & 1, rp = ot / (2 * KP);
    cx<T> acc[2][2];
#pragma unroll
    for (int a = 0; a < 2; a++) { acc[a][0] = czero<T>(); acc[a][1] = czero<T>(); }

    // tiles of whole kRtTile-site runs inside one x row (te a multiple of the tile, the usual
    // case) stage with shifts and one base index instead of a division per element
    // the tile's products, accumulated over its sites by this thread's site group
    auto compute = [&](int nq) {
        if (active) {
            for (int qq = grp; qq < nq; qq += G) {
                const cx<T>* wp = Ws + qq * WR + s * K2 + 2 * kp;
                const cx<T>* vp = Vs + qq * VR + s * R2 + 2 * rp;
                const cx<T> wa = wp[0], wb = wp[1], va = vp[0], vb = vp[1];
                cfmac(acc[0][0], wa, va);
                cfmac(acc[0][1], wa, vb);
                cfmac(acc[1][0], wb, va);
                cfmac(acc[1][1], wb, vb);
            }
        }
    };
    // Tiles of whole kRtTile-site runs inside one x row (te a multiple of the tile, the usual
    // case) stage with shifts and one base index instead of a division per element, and when a
    // thread's share of a tile fits in registers (kPW test-vector and kPV source elements) the
    // next tile's loads are issued before the current tile is computed, so their latency hides
    // behind the products.
    constexpr int kPW = 4, kPV = 8;
    const bool rows = (te % kRtTile) == 0;
    if (rows && blockDim.x == 256 && K2 * kRtTile <= kPW * 256 && R2 * kRtTile <= kPV * 256) {
        cx<T> pw[kPW][2], pv[kPV][2];
        auto fetch = [&](int qt) {
            const int mx = qt / te, mt = qt - mx * te;
            const long long n0 = (long long)(bxi * xe + mx) * nt + (bti * te + mt);
#pragma unroll
            for (int i = 0; i < kPW; i++) {
                const int idx = tid + 256 * i, k = idx / kRtTile;
                const long long n = n0 + idx % kRtTile;
                pw[i][0] = pw[i][1] = czero<T>();
                if (k < ntest) {
                    pw[i][0] = ccast<T>(load_cx(W + ((long long)k * N + n) * 2));
                    pw[i][1] = ccast<T>(load_cx(W + ((long long)k * N + n) * 2 + 1));
                }
            }
#pragma unroll
            for (int i = 0; i < kPV; i++) {
                const int idx = tid + 256 * i, r = idx / kRtTile;
                const long long n = n0 + idx % kRtTile;
                pv[i][0] = pv[i][1] = czero<T>();
                if (r < nrhs) {
                    pv[i][0] = v[(long long)r * N * 2 + 2 * n];
                    pv[i][1] = v[(long long)r * N * 2 + 2 * n + 1];
                }
            }
        };
        if (q0 < q1) fetch(q0);
        for (int qt = q0; qt < q1; qt += kRtTile) {
            __syncthreads();   // the previous tile's products are done
#pragma unroll
            for (int i = 0; i < kPW; i++) {
                const int idx = tid + 256 * i, k = idx / kRtTile, qq = idx % kRtTile;
                if (idx < kRtTile * K2) {
                    Ws[qq * WR + k] = pw[i][0];
                    Ws[qq * WR + K2 + k] = pw[i][1];
                }
            }
#pragma unroll
            for (int i = 0; i < kPV; i++) {
                const int idx = tid + 256 * i, r = idx / kRtTile, qq = idx % kRtTile;
                if (idx < kRtTile * R2) {
                    Vs[qq * VR + r] = pv[i][0];
                    Vs[qq * VR + R2 + r] = pv[i][1];
                }
            }
            __syncthreads();
            if (qt + kRtTile < q1) fetch(qt + kRtTile);
            compute(kRtTile);
        }
    } else {
        for (int qt = q0; qt < q1; qt += kRtTile) {
            const int nq = min(kRtTile, q1 - qt);
            __syncthreads();
            for (int idx = tid; idx < nq * K2; idx += blockDim.x) {
                const int k = idx / nq, qq = idx - k * nq;
                const int q = qt + qq, mx = q / te, mt = q - mx * te;
                const long long n = (long long)(bxi * xe + mx) * nt + (bti * te + mt);
                cx<T> w0 = czero<T>(), w1 = czero<T>();
                if (k < ntest) {
                    w0 = ccast<T>(load_cx(W + ((long long)k * N + n) * 2));
                    w1 = ccast<T>(load_cx(W + ((long long)k * N + n) * 2 + 1));
                }
                Ws[qq * WR + k] = w0;
                Ws[qq * WR + K2 + k] = w1;
            }
            for (int idx = tid; idx < nq * R2; idx += blockDim.x) {
                const int r = idx / nq, qq = idx - r * nq;
                const int q = qt + qq, mx = q / te, mt = q - mx * te;
                const long long n = (long long)(bxi * xe + mx) * nt + (bti * te + mt);
                cx<T> p0 = czero<T>(), p1 = czero<T>();
                if (r < nrhs) {
                    p0 = v[(long long)r * N * 2 + 2 * n];
                    p1 = v[(long long)r * N * 2 + 2 * n + 1];
                }
                Vs[qq * VR + r] = p0;
                Vs[qq * VR + R2 + r] = p1;
            }
            __syncthreads();
            compute(nq);
        }
    }
    // sum the site groups and write this split's partials
    __syncthreads();
    cx<T>* red = Ws;   // [G][OT][4]
    if (active) {
#pragma unroll
        for (int a = 0; a < 2; a++) {
            red[(grp * OT + ot) * 4 + 2 * a] = acc[a][0];
            red[(grp * OT + ot) * 4 + 2 * a + 1] = acc[a][1];
        }
    }
    __syncthreads();
    for (int o = tid; o < OT * 4; o += blockDim.x) {
        const int t = o >> 2, a = (o >> 1) & 1, b = o & 1;
        cx<T> sum = czero<T>();
        for (int g = 0; g < G; g++) sum += red[(g * OT + t) * 4 + 2 * a + b];
        const int tk = t % KP, ts = (t / KP) & 1, tr = t / (2 * KP);
        const int k = 2 * tk + a, r = 2 * tr + b;
        if (k < ntest && r < nrhs)
            partial[(((long long)r * nblk + nc) * nsplit + split) * (2 * ntest) + 2 * k + ts] = sum;
    }
}

template <typename T>
__global__ void k_restrict0_sum(const cx<T>* __restrict__ partial, cx<T>* __restrict__ out, int nblk, int nchunk,
                                int K1) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int rhs = blockIdx.y;
    if (o >= nblk * K1) return;
    const int nc = o / K1, d = o - nc * K1;
    const cx<T>* p = partial + (((long long)rhs * nblk + nc) * nchunk) * K1 + d;
    cx<T> s = czero<T>();
    for (int c = 0; c < nchunk; c++) s += p[(long long)c * K1];
    out[(long long)rhs * nblk * K1 + o] = s;
}

// Level::P_v at level 0 (src/level.cpp:182-209) added into psi (add = 1) or stored (add = 0):
//   psi[rhs][n][s] (+)= sum_cc W[cc][n][s] vc[rhs][nc(n)][2cc+s]
// Level::P_v at level 0 added into psi (src/level.cpp:182-209): psi[n][s] += sum_k W_k[n][s]
// vc[nc][2k+s].  One thread per site; the site's KT >= ntest test-vector entries are loaded
// once (BF16 -> T) and kept in registers for every source, so W streams from HBM once per
// launch and each source costs one read-modify-write of psi plus broadcast reads of its
// coarse vector (a warp's 32 consecutive t sites share one aggregate).
template <typename T, typename TW, int KT>
__global__ void __launch_bounds__(256) k_prolong0_add(const TW* __restrict__ W, const cx<T>* __restrict__ vc,
                                                      cx<T>* __restrict__ psi, int nx, int nt, int bt, int xe,
                                                      int te, int ntest, int nblk, int nrhs, int add) {
    const int N = nx * nt;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int x = n / nt, t = n - x * nt;
    const int nc = (x / xe) * bt + (t / te);
    cx<T> w0[KT], w1[KT];
#pragma unroll
    for (int k = 0; k < KT; k++) {
        if (k < ntest) {
            w0[k] = ccast<T>(load_cx(W + ((long long)k * N + n) * 2));
            w1[k] = ccast<T>(load_cx(W + ((long long)k * N + n) * 2 + 1));
        }
    }
    // several sources per trip keep several psi loads in flight (one for FP64 with more than
    // 16 test vectors, whose entries already fill the registers)
    constexpr int UR = (sizeof(T) == 8 && KT > 16) ? 1 : 4;
#pragma unroll UR
    for (int rhs = 0; rhs < nrhs; rhs++) {
        const cx<T>* pv = vc + ((long long)rhs * nblk + nc) * 2 * ntest;
        cx<T> a0 = czero<T>(), a1 = czero<T>();
        cx<T>* o = psi + (long long)rhs * N * 2 + 2 * n;
        if constexpr (sizeof(T) == 4) {
            // both spins of a coarse entry and of a site in one 16-byte access
#pragma unroll
            for (int k = 0; k < KT; k++) {
                if (k < ntest) {
                    const float4 q = __ldg(reinterpret_cast<const float4*>(pv + 2 * k));
                    cfma(a0, w0[k], make_float2(q.x, q.y));
                    cfma(a1, w1[k], make_float2(q.z, q.w));
                }
            }
            float4* o4 = reinterpret_cast<float4*>(o);
            float4 q = add ? *o4 : make_float4(0.f, 0.f, 0.f, 0.f);
            q.x += a0.x; q.y += a0.y; q.z += a1.x; q.w += a1.y;
            *o4 = q;
        } else {
#pragma unroll
            for (int k = 0; k < KT; k++) {
                if (k < ntest) {
                    cfma(a0, w0[k], pv[2 * k]);
                    cfma(a1, w1[k], pv[2 * k + 1]);
                }
            }
            if (add) {
                o[0] += a0;
                o[1] += a1;
            } else {
                o[0] = a0;
                o[1] = a1;
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// SAP block solve at level 0 (src/sap.cpp:44-62 with the block operator of
// src/level.cpp:304-368 at colors = 1): one CTA per (block of the colour, source).
// rhs b = r restricted to the block, GMRES(m, restarts, tol) with x0 = b, then
// x[block] += solution.  Vectors live in shared memory when they fit, otherwise in a
// global scratch slab per CTA.
// ---------------------------------------------------------------------------------
template <typename T>
struct FineBlock {
    int nx, nt, sbt, sxe, ste, x0, t0;   // block origin
    T mass;
    const cx<T>* u;                      // block links [S][2] (staged)
};

// out = D_B in on the block (neighbours outside the block dropped, fermionic sign kept)
template <typename T>
__device__ void fine_block_apply(const FineBlock<T>& B, const cx<T>* in, cx<T>* out) {
    const int S = B.sxe * B.ste;
    for (int m = threadIdx.x; m < S; m += blockDim.x) {
        const int mx = m / B.ste, mt = m - mx * B.ste;
        const int t = B.t0 + mt;
        const T sR = (t == B.nt - 1) ? T(-1) : T(1);
        const T sL = (t == 0) ? T(-1) : T(1);
        // neighbour local indices (or -1 when outside the block); periodic wrap stays
        // inside only when the block spans the whole direction
        int mr0 = -1, mr1 = -1, ml0 = -1, ml1 = -1;
        if (mt + 1 < B.ste) mr0 = m + 1; else if (B.ste == B.nt) mr0 = mx * B.ste;
        if (mt > 0) ml0 = m - 1; else if (B.ste == B.nt) ml0 = mx * B.ste + B.ste - 1;
        if (mx + 1 < B.sxe) mr1 = m + B.ste; else if (B.sxe == B.nx) mr1 = mt;
        if (mx > 0) ml1 = m - B.ste; else if (B.sxe == B.nx) ml1 = (B.sxe - 1) * B.ste + mt;
        const cx<T> p0 = in[2 * m], p1 = in[2 * m + 1];
        cx<T> t0 = czero<T>(), t1 = czero<T>(), t2 = czero<T>(), t3 = czero<T>();
        if (mr0 >= 0) t0 = sR * cmul(B.u[2 * m], in[2 * mr0] - in[2 * mr0 + 1]);
        if (mr1 >= 0) t1 = cmul(B.u[2 * m + 1], in[2 * mr1] + cmuli(in[2 * mr1 + 1]));
        if (ml0 >= 0) t2 = sL * cmul(cconj(B.u[2 * ml0]), in[2 * ml0] + in[2 * ml0 + 1]);
        if (ml1 >= 0) t3 = cmul(cconj(B.u[2 * ml1 + 1]), in[2 * ml1] - cmuli(in[2 * ml1 + 1]));
        out[2 * m] = B.mass * p0 - T(0.5) * (t0 + t1 + t2 + t3);
        out[2 * m + 1] = B.mass * p1 - T(0.5) * ((t2 - t0) + cmuli(t3 - t1));
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) k_sap0_blocks(const Links<T> U, const cx<T>* __restrict__ r,
                                                     cx<T>* __restrict__ x, const int* __restrict__ blocks, int ncol,
                                                     int nx, int nt, int sbt, int sxe, int ste, T m0, int m,
                                                     int restarts, T tol, int use_smem, cx<T>* gscratch,
                                                     int* __restrict__ iters_out, const int* __restrict__ act) {
    extern __shared__ __align__(16) unsigned char smraw_s[];
    const int seg = blockIdx.x, rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    const int block = blocks[seg];
    const int S = sxe * ste, len = 2 * S;
    const int N = nx * nt;
    const int bxi = block / sbt, bti = block - bxi * sbt;
    FineBlock<T> B;
    B.nx = nx; B.nt = nt; B.sbt = sbt; B.sxe = sxe; B.ste = ste;
    B.x0 = bxi * sxe; B.t0 = bti * ste; B.mass = m0 + T(2);
    // carve: red | state | u | b | x | w | V[m+1]
    char* p = reinterpret_cast<char*>(smraw_s);
    T* red = reinterpret_cast<T*>(p); p += 2 * 32 * sizeof(T);
    GmState<T> st = gm_state_at<T>(p, 1, m); p += gm_state_bytes(1, m, sizeof(T));
    cx<T>* vec;
    if (use_smem) vec = reinterpret_cast<cx<T>*>(p);
    else vec = gscratch + ((long long)rhs * gridDim.x + seg) * (long long)(m + 5) * len;
    cx<T>* u = vec;
    cx<T>* b = u + len;
    cx<T>* xs = b + len;
    cx<T>* w = xs + len;
    cx<T>* V = w + len;
    const cx<T>* rr = r + (long long)rhs * N * 2;
    for (int q = threadIdx.x; q < S; q += blockDim.x) {
        const int mx = q / ste, mt = q - mx * ste;
        const long long n = (long long)(B.x0 + mx) * nt + (B.t0 + mt);
        u[2 * q] = U[2 * n]; u[2 * q + 1] = U[2 * n + 1];
        b[2 * q] = rr[2 * n]; b[2 * q + 1] = rr[2 * n + 1];
    }
    __syncthreads();
    B.u = u;
    const Team cta = whole_cta();
    auto op = [&](const cx<T>* in, cx<T>* out) {
        __syncthreads();
        fine_block_apply(B, in, out);
    };
    auto ident = [](int, const cx<T>*, cx<T>*) {};
    const int it = team_fgmres<T>(cta, red, (const Eng<T>*)nullptr, 0, 0, op, ident, b, xs, V, V, w, st, len, m,
                                  restarts, tol);
    __syncthreads();
    cx<T>* xx = x + (long long)rhs * N * 2;
    for (int q = threadIdx.x; q < S; q += blockDim.x) {
        const int mx = q / ste, mt = q - mx * ste;
        const long long n = (long long)(B.x0 + mx) * nt + (B.t0 + mt);
        xx[2 * n] += xs[2 * q];
        xx[2 * n + 1] += xs[2 * q + 1];
    }
    if (iters_out && threadIdx.x == 0) iters_out[rhs * gridDim.x + seg] = it;
}

// ---------------------------------------------------------------------------------
// BLAS-1 for the outer FGMRES (FP64).  Vectors are [rhs][len]; V bases [j][rhs][len].
// ---------------------------------------------------------------------------------
__global__ void k_multidot_sum(const double2* __restrict__ partial, int nparts, double2* __restrict__ out) {
    __shared__ double red[64];
    const int o = blockIdx.x;   // (rhs, k) flattened
    double sx = 0, sy = 0;
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) {
        double2 v = partial[(long long)o * nparts + q];
        sx += v.x; sy += v.y;
    }
    sx = cta_sum(sx, red);
    sy = cta_sum(sy, red + 32);
    if (threadIdx.x == 0) out[o] = make_double2(sx, sy);
}

// w[rhs] -= sum_k h[rhs][k] V_k[rhs]   (masked by act[rhs])
__global__ void __launch_bounds__(256) k_multiaxpy(double2* __restrict__ w, const double2* __restrict__ V,
                                                   long long len, long long vstride, int nv,
                                                   const double2* __restrict__ h, int hstride,
                                                   const int* __restrict__ act) {
    const int rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    double2* ww = w + (long long)rhs * len;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x) {
        double2 a = ww[e];
        for (int k = 0; k < nv; k++) {
            const double2 hk = h[(long long)rhs * hstride + k];
            const double2 b = V[(long long)k * vstride + (long long)rhs * len + e];
            a.x -= hk.x * b.x - hk.y * b.y;
            a.y -= hk.x * b.y + hk.y * b.x;
        }
        ww[e] = a;
    }
}

// One pass over w and the basis V_0..V_{nv-1} of every source (FP64):
//   w -= sum_k h[k] V_k            (skipped when h is null; with y given, the result goes to
//                                   y scaled by sc[rhs] and w is left as it was)
//   partial[k] = sum_e w[e] conj(V_k[e]) for k < nd, and |w|^2 at k = nd
// with the accumulators in registers (NV bounds nv and nd at compile time); per-CTA
// partials are reduced by k_multidot_sum in a fixed order.  Sources with act[rhs] = 0 are
// skipped (their partials are not written).
// Up to 8 vectors two CTAs per SM fit; more vectors keep their loaded elements in registers
// at one CTA per SM (the loads of 8 warps x 13 vectors still cover the HBM latency).
template <int NV>
__global__ void __launch_bounds__(256, (NV <= 8 ? 2 : 1)) k_axpy_dots(double2* __restrict__ w, const double2* __restrict__ V,
                                                      long long len, long long vstride, int nv,
                                                      const double2* __restrict__ h, int hstride, int nd,
                                                      const int* __restrict__ act, double2* __restrict__ partial,
                                                      double2* __restrict__ y, const double* __restrict__ sc,
                                                      float2* __restrict__ yf) {
    __shared__ double red[8][2 * (NV + 1)];
    __shared__ double2 hk[NV];   // the axpy coefficients, read as broadcasts (fewer live registers)
    const int rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    double2* ww = w + (long long)rhs * len;
    const double2* vb = V + (long long)rhs * len;
    double ax[NV + 1], ay[NV + 1];
#pragma unroll
    for (int k = 0; k <= NV; k++) { ax[k] = 0; ay[k] = 0; }
    if (threadIdx.x < NV)
        hk[threadIdx.x] = (h && (int)threadIdx.x < nv) ? h[(long long)rhs * hstride + threadIdx.x] : make_double2(0, 0);
    __syncthreads();
    const int nload = (h && nv > nd) ? nv : nd;
    const double f = y ? sc[rhs] : 1.0;
    double2* yy = y ? y + (long long)rhs * len : nullptr;
    float2* yyf = yf ? yf + (long long)rhs * len : nullptr;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x) {
        double2 a = ww[e];
        // every V_k element is loaded once and kept for both the update and the dots
        double2 bk[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) bk[k] = k < nload ? vb[(long long)k * vstride + e] : make_double2(0, 0);
        if (h) {
#pragma unroll
            for (int k = 0; k < NV; k++) {
                if (k < nv) {
                    a.x -= hk[k].x * bk[k].x - hk[k].y * bk[k].y;
                    a.y -= hk[k].x * bk[k].y + hk[k].y * bk[k].x;
                }
            }
            if (yy) {
                const double2 o = make_double2(f * a.x, f * a.y);
                yy[e] = o;
                if (yyf) yyf[e] = make_float2((float)o.x, (float)o.y);
            } else {
                ww[e] = a;
            }
        }
#pragma unroll
        for (int k = 0; k < NV; k++) {
            if (k < nd) {
                ax[k] += a.x * bk[k].x + a.y * bk[k].y;
                ay[k] += a.y * bk[k].x - a.x * bk[k].y;
            }
        }
        ax[NV] += a.x * a.x + a.y * a.y;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k <= NV; k++) {
        if (k < nd || k == NV) {
            const double sx = warp_sum(ax[k]), sy = warp_sum(ay[k]);
            if (lane == 0) { red[wid][2 * k] = sx; red[wid][2 * k + 1] = sy; }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k <= nd; k += blockDim.x) {
        const int kk = (k == nd) ? NV : k;
        double sx = 0, sy = 0;
        for (int q = 0; q < 8; q++) { sx += red[q][2 * kk]; sy += red[q][2 * kk + 1]; }
        partial[((long long)rhs * (nd + 1) + k) * gridDim.x + blockIdx.x] = make_double2(sx, sy);
    }
}

// x[rhs] += sum_k c[rhs][k] Z_k[rhs]  (masked; Z in FP64, or in FP32 promoted exactly: the
// mixed form's basis of preconditioner outputs)
template <typename TZ>
__global__ void __launch_bounds__(256) k_multiaxpy_add(double2* __restrict__ x, const TZ* __restrict__ Z,
                                                       long long len, long long vstride, int nv,
                                                       const double2* __restrict__ c, int cstride,
                                                       const int* __restrict__ nvr, const int* __restrict__ act) {
    const int rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    const int n = nvr ? nvr[rhs] : nv;
    double2* xx = x + (long long)rhs * len;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x) {
        double2 a = xx[e];
        for (int k = 0; k < n; k++) {
            const double2 ck = c[(long long)rhs * cstride + k];
            const double2 b = ccast<double>(Z[(long long)k * vstride + (long long)rhs * len + e]);
            a.x += ck.x * b.x - ck.y * b.y;
            a.y += ck.x * b.y + ck.y * b.x;
        }
        xx[e] = a;
    }
}

// y[rhs] = s[rhs] * x[rhs]  (masked; s real)
// y = s[rhs] x, and yf = (float) y when yf is given (the FP32 copy the mixed-precision
// preconditioner reads)
__global__ void k_scale(double2* __restrict__ y, const double2* __restrict__ x, long long len,
                        const double* __restrict__ s, const int* __restrict__ act, float2* __restrict__ yf) {
    const int rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    const double f = s[rhs];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x) {
        const double2 v = f * x[(long long)rhs * len + e];
        y[(long long)rhs * len + e] = v;
        if (yf) yf[(long long)rhs * len + e] = make_float2((float)v.x, (float)v.y);
    }
}

// precision conversions between the FP64 outer vectors and the FP32 cycle
__global__ void k_d2f(float2* __restrict__ y, const double2* __restrict__ x, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = make_float2((float)x[e].x, (float)x[e].y);
}
__global__ void k_f2d(double2* __restrict__ y, const float2* __restrict__ x, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = make_double2((double)x[e].x, (double)x[e].y);
}
__global__ void k_d2h(__half2* __restrict__ y, const double2* __restrict__ x, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = __floats2half2_rn((float)x[e].x, (float)x[e].y);
}
__global__ void k_d2bf(__nv_bfloat162* __restrict__ y, const double2* __restrict__ x, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        y[e] = __floats2bfloat162_rn((float)x[e].x, (float)x[e].y);
}

// ---------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------
// Source groups of the stencil kernels: enough threads to fill the GPU (about 2^18), and
// otherwise as few groups as possible so that the links stream from memory once per group.
static int source_groups(int nsites, int nrhs) {
    const int want = (262144 + nsites - 1) / nsites;
    return std::max(1, std::min(nrhs, want));
}

// AMG_DIRAC_TMA=0 keeps every D apply on k_dirac (A/B tests)
static int dirac_tma_enabled() {
    static const int on = [] {
        const char* e = getenv("AMG_DIRAC_TMA");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on;
}

// bit 0 of the device error flag: a bulk-copy wait of k_dirac_tma gave up (the flag is read
// and cleared; the read synchronises the stream)
int fine_error_check(cudaStream_t s) {
    int h = 0;
    if (cudaMemcpyFromSymbolAsync(&h, g_fine_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (h) {
        const int z = 0;
        cudaMemcpyToSymbolAsync(g_fine_err, &z, sizeof(int), 0, cudaMemcpyHostToDevice, s);
    }
    return h;
}

// The bounded-wait self-test: k_dirac_tma without any copy issued and 256 polls per wait, so
// the first wait runs out with nothing in flight; returns the device flag afterwards (1 when
// the kernel reported the timeout, 0 if it did not, -1 on a CUDA error or a lattice the
// kernel does not take).
int dirac_tma_wait_test(const double2* U, const double2* in, double2* out, int nx, int nt, int nrhs, cudaStream_t s) {
    if (nrhs < 1 || nt % kTT != 0 || nx % kTX != 0 || in == out ||
        ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) != 0)
        return -1;
    constexpr int bytes = dirac_tma_smem<double>();
    if (cudaFuncSetAttribute(k_dirac_tma<double, false, double, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
        return -1;
    k_dirac_tma<double, false, double, false, true><<<dim3(nt / kTT, nx / kTX), kTT, bytes, s>>>(
        U, in, out, nx, nt, -0.1, nrhs, nullptr, nullptr, 0, nullptr, nullptr);
    if (cudaGetLastError() != cudaSuccess) return -1;
    return fine_error_check(s);
}

template <typename T>
void launch_dirac(const cx<T>* U, const cx<T>* in, cx<T>* out, int nx, int nt, int nrhs, T m0, int dagger,
                  cudaStream_t s) {
    count_launch(1);
    // lattices tiled by kTX x kTT sites with 16-byte aligned, distinct spinors take the
    // bulk-copy kernel
    if (dirac_tma_enabled() && nrhs >= 1 && nt % kTT == 0 && nx % kTX == 0 && nx >= kTX && in != out &&
        ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0) {
        constexpr int bytes = dirac_tma_smem<T>();
        dim3 g(nt / kTT, nx / kTX);
        if (dagger) {
            cudaFuncSetAttribute(k_dirac_tma<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            k_dirac_tma<T, true><<<g, kTT, bytes, s>>>(U, in, out, nx, nt, m0, nrhs, nullptr, nullptr, 0, nullptr,
                                                       nullptr);
        } else {
            cudaFuncSetAttribute(k_dirac_tma<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            k_dirac_tma<T, false><<<g, kTT, bytes, s>>>(U, in, out, nx, nt, m0, nrhs, nullptr, nullptr, 0, nullptr,
                                                        nullptr);
        }
        return;
    }
    dim3 grid((nx * nt + 255) / 256, source_groups(nx * nt, nrhs));
    if (dagger) k_dirac<T, true><<<grid, 256, 0, s>>>(U, in, out, nx, nt, m0, nrhs);
    else k_dirac<T, false><<<grid, 256, 0, s>>>(U, in, out, nx, nt, m0, nrhs);
}

// out = D in (FP64) for FP32 spinors in, and in_copy = in (FP32)
void launch_dirac_promote(const double2* U, const float2* in, double2* out, float2* in_copy, int nx, int nt,
                          int nrhs, double m0, cudaStream_t s) {
    count_launch(1);
    if (dirac_tma_enabled() && nrhs >= 1 && nt % kTT == 0 && nx % kTX == 0 && nx >= kTX &&
        ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out) |
          reinterpret_cast<uintptr_t>(in_copy)) & 15) == 0) {
        constexpr int bytes = dirac_tma_smem<float>();
        cudaFuncSetAttribute(k_dirac_tma<double, false, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
        k_dirac_tma<double, false, float, true><<<dim3(nt / kTT, nx / kTX), kTT, bytes, s>>>(
            U, in, out, nx, nt, m0, nrhs, in_copy, nullptr, 0, nullptr, nullptr);
        return;
    }
    dim3 grid((nx * nt + 255) / 256, source_groups(nx * nt, nrhs));
    k_dirac_promote<<<grid, 256, 0, s>>>(U, in, out, in_copy, nx, nt, m0, nrhs);
}

template <typename T>
void launch_residual(const Links<T> U, const cx<T>* b, long long bstride, const cx<T>* x, cx<T>* r, int nx, int nt,
                     int nrhs, T m0, double* partial, double* norm2_out, const int* act, cudaStream_t s) {
    count_launch(norm2_out ? 2 : 1);
    // lattices the bulk-copy stencil tiles: x staged through shared memory, source after
    // source, the links in registers (the same site arithmetic as k_residual)
    if (dirac_tma_enabled() && nrhs >= 1 && nt % kTT == 0 && nx % kTX == 0 && nx >= kTX && x != r &&
        ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(r)) & 15) == 0) {
        constexpr int bytes = dirac_tma_smem<T>();
        const dim3 g(nt / kTT, nx / kTX);
        if constexpr (sizeof(T) == 8) {   // FP64 links: a plain pointer
            const cx<T>* Up = static_cast<const cx<T>*>(U.p);
            cudaFuncSetAttribute(k_dirac_tma<T, false, T, false, false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            k_dirac_tma<T, false, T, false, false, true><<<g, kTT, bytes, s>>>(
                Up, x, r, nx, nt, m0, nrhs, nullptr, b, bstride, act, norm2_out ? partial : nullptr);
        } else {
            cudaFuncSetAttribute(k_dirac_tma<T, false, T, false, false, true, Links<T>>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            k_dirac_tma<T, false, T, false, false, true, Links<T>><<<g, kTT, bytes, s>>>(
                U, x, r, nx, nt, m0, nrhs, nullptr, b, bstride, act, norm2_out ? partial : nullptr);
        }
        if (norm2_out) k_sum_partials<<<nrhs, 256, 0, s>>>(partial, (int)(g.x * g.y), norm2_out);
        return;
    }
    const int nblk = (nx * nt + 255) / 256;
    dim3 grid(nblk, source_groups(nx * nt, nrhs));
    k_residual<T><<<grid, 256, 0, s>>>(U, b, bstride, x, r, nx, nt, m0, norm2_out ? partial : nullptr, act, nrhs);
    if (norm2_out) k_sum_partials<<<nrhs, 256, 0, s>>>(partial, nblk, norm2_out);
}

// |v[rhs]|^2 for [nrhs][len] vectors, deterministic
template <typename T>
__global__ void __launch_bounds__(256) k_norm2(const cx<T>* __restrict__ v, long long len, long long stride,
                                               double* __restrict__ partial) {
    __shared__ double red[8];
    const cx<T>* vv = v + (long long)blockIdx.y * stride;
    double s = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x)
        s += (double)cnorm2(vv[e]);
    s = cta_sum(s, red);
    if (threadIdx.x == 0) partial[(long long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}
template <typename T>
void launch_norm2(const cx<T>* v, long long len, long long stride, int nrhs, double* partial, double* out,
                  cudaStream_t s) {
    count_launch(2);
    const int np = 296;
    dim3 grid(np, nrhs);
    k_norm2<T><<<grid, 256, 0, s>>>(v, len, stride, partial);
    k_sum_partials<<<nrhs, 256, 0, s>>>(partial, np, out);
}
int residual_partials(int nx, int nt) { return (nx * nt + 255) / 256; }

// AMG_SAP_KERNEL=generic selects the generic SAP kernel for every block shape (A/B tests)
static int g_sap0_warp = -1;
int sap0_warp_enabled() {
    if (g_sap0_warp < 0) {
        const char* e = getenv("AMG_SAP_KERNEL");
        g_sap0_warp = (e && !strcmp(e, "generic")) ? 0 : 1;
    }
    return g_sap0_warp;
}
void set_sap0_warp(int on) { g_sap0_warp = on; }

// Multiprocessors of the current device, looked up once per device.
int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// CTAs of `func` (threads per CTA, dynamic shared memory per CTA) resident on one SM of the
// current device, from its registers and the SM's thread, register and shared-memory limits.
int resident_ctas(const void* func, int threads, int smem_bytes) {
    cudaFuncAttributes fa{};
    int dev = 0, sm_smem = 0, reserve = 0, sm_regs = 0, sm_threads = 0;
    if (cudaFuncGetAttributes(&fa, func) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserve, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_regs, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
        return 1;
    const int regs = ((std::max(fa.numRegs, 1) + 7) / 8) * 8;   // allocated in units of 8 per thread
    const int by_regs = sm_regs / (regs * threads);
    const int by_smem = sm_smem / (smem_bytes + (int)fa.sharedSizeBytes + reserve);
    const int by_threads = sm_threads / threads;
    return std::max(1, std::min(by_regs, std::min(by_smem, by_threads)));
}

// Largest dynamic shared memory one block may opt into on the current device, looked up once
// per device.
int smem_optin_bytes() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 48 * 1024;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0)
            v = 48 * 1024;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// Returns the status of its own attribute call and launches (cudaGetLastError is not read, so
// an error pending from earlier work on this thread is neither reported nor cleared here).
// The mixed form's level-0 transfers on the tensor cores (tc_transfer.cuh) unless
// AMG_TC_TRANSFER=0 (read once per process): then the CUDA-core kernels run.
int tc_transfer_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("AMG_TC_TRANSFER");
        on = (e && !strcmp(e, "0")) ? 0 : 1;
    }
    return on;
}

// Tensor-core restriction for BF16 test vectors and FP32 sources; returns false (nothing
// launched) for shapes it does not take.
template <typename T, typename TW>
bool launch_restrict0_tc(const TW* W, const cx<T>* v, cx<T>* partial, int nx, int nt, int bx, int bt, int ntest,
                         int nrhs, int nchunk, cudaStream_t s, cudaError_t* err, int* used_chunks) {
    if constexpr (!std::is_same<T, float>::value || !std::is_same<TW, __nv_bfloat162>::value) {
        return false;
    } else {
        const int xe = nx / bx, te = nt / bt, nblk = bx * bt;
        if (!tc_transfer_enabled() || te % kRtcSites || ntest < 1 || ntest > 32 || nrhs < 1 || nrhs > 256 ||
            nblk > 65535 || nchunk < 1)
            return false;
        const int N = nx * nt;
        // 32-bit offsets inside the kernel
        if ((long long)std::max(nrhs, ntest) * N * 2 >= (1ll << 31)) return false;
        // NP padded sources: a power of two >= 16; NB = NP sources x kRtcSites sites / kTcThreads
        int NP = 16;
        while (NP < nrhs) NP *= 2;
        const int M = ntest <= 16 ? 64 : 128, NB = NP * kRtcSites / kTcThreads;
        const int nd = rtc_ring(M, NP, smem_optin_bytes());
        if (nd == 0) return false;
        const int bytes = rtc_smem_bytes(M, NP, nd);
        // one wave: as many chunks per block as the resident CTAs allow (at most the caller's
        // chunk count, which sizes the partial-sum buffer)
        auto go = [&](auto kern) {
            *err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (*err != cudaSuccess) return;
            const int per_sm = resident_ctas(reinterpret_cast<const void*>(kern), kTcThreads, bytes);
            *used_chunks = std::max(1, std::min(nchunk, per_sm * sm_count() / nblk));
            dim3 g(*used_chunks, nblk);
            kern<<<g, kTcThreads, bytes, s>>>(W, v, partial, nx, nt, bt, xe, te, *used_chunks, ntest, nrhs, nd);
        };
        if (M == 64) {
            if (NB == 1) go(k_restrict0_tc<64, 1>);
            else if (NB == 2) go(k_restrict0_tc<64, 2>);
            else if (NB == 4) go(k_restrict0_tc<64, 4>);
            else if (NB == 8) go(k_restrict0_tc<64, 8>);
            else go(k_restrict0_tc<64, 16>);
        } else {
            if (NB == 1) go(k_restrict0_tc<128, 1>);
            else if (NB == 2) go(k_restrict0_tc<128, 2>);
            else if (NB == 4) go(k_restrict0_tc<128, 4>);
            else if (NB == 8) go(k_restrict0_tc<128, 8>);
            else go(k_restrict0_tc<128, 16>);
        }
        if (*err != cudaSuccess) return true;
        *err = cudaPeekAtLastError();
        return true;
    }
}

template <typename T, typename TW>
cudaError_t launch_restrict0(const TW* W, const cx<T>* v, cx<T>* out, cx<T>* partial, int nx, int nt, int bx,
                             int bt, int ntest, int nrhs, int nchunk, cudaStream_t s) {
    count_launch(2);
    const int xe = nx / bx, te = nt / bt, nblk = bx * bt;
    dim3 grid(nchunk, nblk);
    dim3 g2((nblk * 2 * ntest + 127) / 128, nrhs);
    cudaError_t tce = cudaSuccess;
    int tc_chunks = nchunk;
    if (launch_restrict0_tc<T, TW>(W, v, partial, nx, nt, bx, bt, ntest, nrhs, nchunk, s, &tce, &tc_chunks)) {
        if (tce != cudaSuccess) return tce;
        k_restrict0_sum<T><<<g2, 128, 0, s>>>(partial, out, nblk, tc_chunks, 2 * ntest);
        return cudaPeekAtLastError();
    }
    // the tiled kernel when its output tiles fit one CTA and its staging fits the device's
    // shared memory (few test vectors with many sources need more than a block may hold)
    const int bytes = rt_smem_bytes<T>(ntest, nrhs);
    if (rt_out_tiles(ntest, nrhs) <= 256 && bytes <= smem_optin_bytes()) {
        if (bytes > 48 * 1024) {
            const cudaError_t e =
                cudaFuncSetAttribute(k_restrict0t<T, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e != cudaSuccess) return e;
        }
        k_restrict0t<T, TW><<<grid, 256, bytes, s>>>(W, v, partial, nx, nt, bt, xe, te, nchunk, ntest, nrhs);
    } else {
        const int thr = nrhs >= 8 ? 256 : 32 * nrhs;
        if (ntest <= 8)
            k_restrict0m<T, TW, 8><<<grid, thr, 0, s>>>(W, v, partial, nx, nt, bt, xe, te, nchunk, ntest, nrhs);
        else if (ntest <= 16)
            k_restrict0m<T, TW, 16><<<grid, thr, 0, s>>>(W, v, partial, nx, nt, bt, xe, te, nchunk, ntest, nrhs);
        else
            k_restrict0m<T, TW, 32><<<grid, thr, 0, s>>>(W, v, partial, nx, nt, bt, xe, te, nchunk, ntest, nrhs);
    }
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return e;
    k_restrict0_sum<T><<<g2, 128, 0, s>>>(partial, out, nblk, nchunk, 2 * ntest);
    return cudaPeekAtLastError();
}

template <typename T, typename TW>
void launch_prolong0_add(const TW* W, const cx<T>* vc, cx<T>* psi, int nx, int nt, int bx, int bt, int ntest,
                         int nrhs, cudaStream_t s, bool add) {
    count_launch(1);
    const int xe = nx / bx, te = nt / bt;
    if constexpr (std::is_same<T, float>::value && std::is_same<TW, __nv_bfloat162>::value) {
        // tensor cores: 32-site tiles along t, several CTAs per aggregation block
        const int nblk = bx * bt, NP = (nrhs + 31) / 32 * 32;   // two halves of 16-column batches
        const int bytes = ptc_smem_bytes(ntest, NP);
        if (tc_transfer_enabled() && te % kPtcSites == 0 && ntest >= 1 && ntest <= 32 && nrhs >= 1 && nrhs <= 128 &&
            nblk <= 65535 && bytes <= smem_optin_bytes() &&
            cudaFuncSetAttribute(k_prolong0_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess) {
            // one wave of CTAs over the aggregation blocks
            const int per_sm = resident_ctas(reinterpret_cast<const void*>(k_prolong0_tc), kTcThreads, bytes);
            const int tiles = xe * (te / kPtcSites);
            const int nsplit = std::max(1, std::min(tiles, per_sm * sm_count() / nblk));
            dim3 grid(nsplit, nblk);
            k_prolong0_tc<<<grid, kTcThreads, bytes, s>>>(W, vc, psi, nx, nt, bt, xe, te, ntest, nblk, nrhs, NP, nsplit,
                                                          add);
            return;
        }
    }
    const int grid = (nx * nt + 255) / 256;
    if (ntest <= 8) k_prolong0_add<T, TW, 8><<<grid, 256, 0, s>>>(W, vc, psi, nx, nt, bt, xe, te, ntest, bx * bt, nrhs, add);
    else if (ntest <= 16) k_prolong0_add<T, TW, 16><<<grid, 256, 0, s>>>(W, vc, psi, nx, nt, bt, xe, te, ntest, bx * bt, nrhs, add);
    else k_prolong0_add<T, TW, 32><<<grid, 256, 0, s>>>(W, vc, psi, nx, nt, bt, xe, te, ntest, bx * bt, nrhs, add);
}

template <typename T>
int sap0_smem_bytes(int S, int m, int use_smem) {
    int b = 2 * 32 * (int)sizeof(T) + gm_state_bytes(1, m, sizeof(T));
    if (use_smem) b += (m + 5) * 2 * S * (int)sizeof(cx<T>);
    return b;
}

template <typename T, int SPT, int NW>
cudaError_t launch_sap0_lean(const Links<T> U, const cx<T>* r, cx<T>* x, const int* blocks, int ncol, int nrhs, int nx,
                             int nt, int sbt, int sxe, int ste, T m0, int restarts, T tol, int* iters, const int* act,
                             cudaStream_t s) {
    const int bytes = sap0_lean_smem<T, 5, SPT, NW>();
    cudaError_t e = cudaFuncSetAttribute(k_sap0_lean<T, 5, SPT, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    dim3 grid(ncol, nrhs);
    k_sap0_lean<T, 5, SPT, NW><<<grid, 32 * NW, bytes, s>>>(U, r, x, blocks, ncol, nx, nt, sbt, sxe, ste, m0, restarts,
                                                            tol, act, iters);
    return cudaGetLastError();
}

// AMG_SAP_KERNEL=lean keeps FP32 solves on the lean kernel (A/B tests); AMG_SAP_SPT=2 puts
// two sites on each thread of the paired-FP32 kernel (twice the threads) instead of four.
// AMG_SAP_KERNEL=ca selects the communication-avoiding FP32 kernel (sap_ca.cuh) instead of
// the paired-FP32 MGS kernel: it executes about a third fewer instructions, but its
// per-step small dense algebra sits on one warp's critical path and the two measure within
// a few percent of each other on B200, so the MGS form (the reference's arithmetic) stays
// the default.  AMG_SAP_KERNEL=cgs selects the paired kernel with classical Gram-Schmidt
// (one reduction per Arnoldi step instead of j + 2, a second projection on cancellation).
// AMG_SAP_KERNEL=half selects the FP16-basis kernel (sap_h.cuh; FP16 fine links only) and
// AMG_SAP_KERNEL=bf16 the same kernel with a BF16 basis.
static int g_sap0_f32 = -1, g_sap0_spt = -1, g_sap0_f32_variant = -1;
static int sap0_f32_enabled() {
    if (g_sap0_f32 < 0) {
        const char* e = getenv("AMG_SAP_KERNEL");
        g_sap0_f32 = (e && (!strcmp(e, "generic") || !strcmp(e, "lean"))) ? 0 : 1;
        g_sap0_f32_variant = !e                  ? 0
                             : !strcmp(e, "ca")   ? SAP_VARIANT_CA
                             : !strcmp(e, "cgs")  ? SAP_VARIANT_CGS
                             : !strcmp(e, "half") ? SAP_VARIANT_HALF
                             : !strcmp(e, "bf16") ? SAP_VARIANT_BF16B
                                                  : 0;
        const char* t = getenv("AMG_SAP_SPT");
        g_sap0_spt = (t && atoi(t) == 2) ? 2 : 4;
    }
    return g_sap0_f32;
}

template <int SPT, int NW>
cudaError_t launch_sap0_ca(const Links<float> U, const float2* r, float2* x, const int* blocks, int ncol, int nrhs, int nx,
                           int nt, int sbt, int sxe, int ste, float m0, int restarts, float tol, int* iters,
                           const int* act, cudaStream_t s) {
    const int bytes = sap0_ca_smem<SPT, NW>();
    cudaError_t e = cudaFuncSetAttribute(k_sap0_ca<SPT, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    dim3 grid(ncol, nrhs);
    k_sap0_ca<SPT, NW><<<grid, 32 * NW, bytes, s>>>(U, r, x, blocks, ncol, nx, nt, sbt, sxe, ste, m0, restarts, tol, act,
                                                    iters);
    return cudaGetLastError();
}

template <int SPT, int NW, bool CGS = false>
cudaError_t launch_sap0_f32(const Links<float> U, float2* r, float2* x, const int* blocks, int ncol, int nrhs, int nx,
                            int nt, int sbt, int sxe, int ste, float m0, int restarts, float tol, int* iters,
                            const int* act, cudaStream_t s, const float2* vsrc, long long vstride) {
    const int bytes = sap0_f32_smem<5, SPT, NW, CGS>();
    cudaError_t e = cudaFuncSetAttribute(k_sap0_f32<5, SPT, NW, CGS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    dim3 grid(ncol, nrhs);
    k_sap0_f32<5, SPT, NW, CGS><<<grid, 32 * NW, bytes, s>>>(U, r, x, blocks, ncol, nx, nt, sbt, sxe, ste, m0, restarts,
                                                             tol, act, iters, vsrc, vstride);
    return cudaGetLastError();
}

// The FP16-basis kernel for blocks of 256, 512 or 1024 sites (NW = sites / 128 warps of four
// sites per thread), three CTAs per SM: the largest shared-memory carveout is requested so
// that three blocks' 73 KB fit.
template <int NW, bool BF>
cudaError_t launch_sap0_h(const __half2* U, float2* r, float2* x, const int* blocks, int ncol, int nrhs, int nx,
                          int nt, int sbt, int sxe, int ste, float m0, int restarts, float tol, int* iters,
                          const int* act, cudaStream_t s) {
    constexpr int bytes = sap0_h_smem<5, 4, NW>();
    cudaError_t e = cudaFuncSetAttribute(k_sap0_h<5, 4, NW, BF>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sap0_h<5, 4, NW, BF>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    dim3 grid(ncol, nrhs);
    k_sap0_h<5, 4, NW, BF><<<grid, 32 * NW, bytes, s>>>(U, r, x, blocks, ncol, nx, nt, sbt, sxe, ste, m0, restarts,
                                                        tol, act, iters);
    return cudaGetLastError();
}
template <int NW, bool BF>
static cudaError_t launch_sap0_h_group_nw(const SapTask* tasks, const int* col_task, const int* col_seg, int ncols,
                                          int max_rhs, cudaStream_t s) {
    constexpr int bytes = sap0_h_smem<5, 4, NW>();
    cudaError_t e = cudaFuncSetAttribute(k_sap0_h_group<5, 4, NW, BF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sap0_h_group<5, 4, NW, BF>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    k_sap0_h_group<5, 4, NW, BF><<<dim3(ncols, max_rhs), 32 * NW, bytes, s>>>(tasks, col_task, col_seg);
    return cudaGetLastError();
}
cudaError_t launch_sap0_h_group(const SapTask* tasks, const int* col_task, const int* col_seg, int ncols, int max_rhs,
                                int S, bool bf, cudaStream_t s) {
    count_launch(1);
    if (ncols < 1 || max_rhs < 1 || max_rhs > 65535) return cudaErrorInvalidValue;
    switch (S) {
        case 256: return bf ? launch_sap0_h_group_nw<2, true>(tasks, col_task, col_seg, ncols, max_rhs, s)
                            : launch_sap0_h_group_nw<2, false>(tasks, col_task, col_seg, ncols, max_rhs, s);
        case 512: return bf ? launch_sap0_h_group_nw<4, true>(tasks, col_task, col_seg, ncols, max_rhs, s)
                            : launch_sap0_h_group_nw<4, false>(tasks, col_task, col_seg, ncols, max_rhs, s);
        case 1024: return bf ? launch_sap0_h_group_nw<8, true>(tasks, col_task, col_seg, ncols, max_rhs, s)
                             : launch_sap0_h_group_nw<8, false>(tasks, col_task, col_seg, ncols, max_rhs, s);
        default: return cudaErrorInvalidValue;
    }
}

template <bool BF>
static cudaError_t launch_sap0_h_shape(const __half2* U, float2* r, float2* x, const int* blocks, int ncol, int nrhs,
                                       int nx, int nt, int sbt, int sxe, int ste, float m0, int restarts, float tol,
                                       int* iters, const int* act, cudaStream_t s, bool* done) {
    *done = true;
    switch (sxe * ste) {
        case 256: return launch_sap0_h<2, BF>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
        case 512: return launch_sap0_h<4, BF>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
        case 1024: return launch_sap0_h<8, BF>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
        default: break;
    }
    *done = false;
    return cudaSuccess;
}

// FP32 solves of 64- to 1024-site blocks take the paired-FP32 kernel.
static cudaError_t launch_sap0_paired(const Links<float> U, float2* r, float2* x, const int* blocks, int ncol,
                                      int nrhs, int nx, int nt, int sbt, int sxe, int ste, float m0, int restarts,
                                      float tol, int* iters, const int* act, cudaStream_t s, bool* done, int v,
                                      const float2* vsrc, long long vstride) {
    *done = true;
    const int S = sxe * ste;
    // the paired kernel gives each thread a run of SPT consecutive t sites (SPT = 2 for 64-site
    // blocks or the MGS form with AMG_SAP_SPT=2, else 4), so the block's t extent must be a
    // multiple of it
    const bool two = v == SAP_VARIANT_PAIRED2 || (v != SAP_VARIANT_CGS && g_sap0_spt == 2);
    const int spt = (S == 64 || two) ? 2 : 4;
    if (v != SAP_VARIANT_CA && ste % spt != 0) {
        *done = false;
        return cudaSuccess;
    }
    if (v == SAP_VARIANT_CGS) {
        switch (S) {
            case 64: return launch_sap0_f32<2, 1, true>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 128: return launch_sap0_f32<4, 1, true>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 256: return launch_sap0_f32<4, 2, true>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 512: return launch_sap0_f32<4, 4, true>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 1024: return launch_sap0_f32<4, 8, true>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            default: break;
        }
    }
    if (v == SAP_VARIANT_CA) {
        switch (S) {
            case 64: return launch_sap0_ca<2, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 128: return launch_sap0_ca<4, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 256: return launch_sap0_ca<4, 2>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 512: return launch_sap0_ca<4, 4>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 1024: return launch_sap0_ca<4, 8>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            default: break;
        }
    }
    if (two) {
        switch (S) {
            case 64: return launch_sap0_f32<2, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 128: return launch_sap0_f32<2, 2>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 256: return launch_sap0_f32<2, 4>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 512: return launch_sap0_f32<2, 8>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 1024: return launch_sap0_f32<2, 16>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            default: break;
        }
    } else {
        switch (S) {
            case 64: return launch_sap0_f32<2, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 128: return launch_sap0_f32<4, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 256: return launch_sap0_f32<4, 2>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 512: return launch_sap0_f32<4, 4>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            case 1024: return launch_sap0_f32<4, 8>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, vsrc, vstride);
            default: break;
        }
    }
    *done = false;
    return cudaSuccess;
}

// Blocks of 64 to 1024 sites with the reference's restart length 5 take the paired-FP32
// kernel (sap_f32.cuh) in FP32 and the lean kernel (sap_lean.cuh) in FP64; any other shape
// or restart length takes the generic kernel above.
template <typename T>
cudaError_t launch_sap0(const Links<T> U, cx<T>* r, cx<T>* x, const int* blocks, int ncol, int nrhs, int nx,
                        int nt, int sbt, int sxe, int ste, T m0, int m, int restarts, T tol, int use_smem,
                        cx<T>* gscratch, int* iters, const int* act, cudaStream_t s, int variant, const cx<T>* vfuse,
                        long long vstride) {
    count_launch(1);
    const int S = sxe * ste;
    // variant: SAP_VARIANT_* (a context's tuned choice) or -1 for the environment's default
    int v = variant;
    if (v < 0) {
        const int f32 = sap0_f32_enabled();
        v = !sap0_warp_enabled() ? SAP_VARIANT_GENERIC : (f32 ? (g_sap0_f32_variant ? g_sap0_f32_variant : SAP_VARIANT_PAIRED)
                                                               : SAP_VARIANT_LEAN);
    }
    if (vfuse) {
        // r = v - D x inside the block solve: the paired kernels (MGS and CGS forms) on shapes
        // they take, when no two blocks of one colour touch (an even number of blocks in both
        // directions, so the red/black colouring is a checkerboard, wrap-around included);
        // otherwise the residual runs as its own launch first
        bool fused = false;
        if constexpr (std::is_same<T, float>::value) {
            const bool two = v == SAP_VARIANT_PAIRED2 || (v != SAP_VARIANT_CGS && g_sap0_spt == 2);
            const int spt = (S == 64 || two) ? 2 : 4;
            fused = m == 5 && (v == SAP_VARIANT_PAIRED || v == SAP_VARIANT_PAIRED2 || v == SAP_VARIANT_CGS) &&
                    S >= 64 && S <= 1024 &&
                    (S & (S - 1)) == 0 && ste % spt == 0 && (nx / sxe) % 2 == 0 && sbt % 2 == 0;
        }
        if (!fused) {
            launch_residual<T>(U, vfuse, vstride, x, r, nx, nt, nrhs, m0, nullptr, nullptr, act, s);
            vfuse = nullptr;
        }
    }
    if constexpr (std::is_same<T, float>::value) {
        if (v == SAP_VARIANT_HALF || v == SAP_VARIANT_BF16B) {
            // 16-bit basis: FP16 links, restart length 5, four sites per thread in one t row
            if (m == 5 && U.fmt == LINK_F16 && ste % 4 == 0) {
                const __half2* Uh = static_cast<const __half2*>(U.p);
                bool done = false;
                const cudaError_t e =
                    v == SAP_VARIANT_BF16B
                        ? launch_sap0_h_shape<true>(Uh, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, &done)
                        : launch_sap0_h_shape<false>(Uh, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s, &done);
                if (done) return e;
            }
            v = SAP_VARIANT_PAIRED;
        }
        if (m == 5 && (v == SAP_VARIANT_PAIRED || v == SAP_VARIANT_PAIRED2 || v == SAP_VARIANT_CA ||
                       v == SAP_VARIANT_CGS)) {
            bool done = false;
            const cudaError_t e = launch_sap0_paired(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts,
                                                     tol, iters, act, s, &done, v, vfuse, vstride);
            if (done) return e;
        }
    }
    if (m == 5 && v != SAP_VARIANT_GENERIC) {
        switch (S) {
            case 64: return launch_sap0_lean<T, 2, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 128: return launch_sap0_lean<T, 4, 1>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 256: return launch_sap0_lean<T, 4, 2>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 512: return launch_sap0_lean<T, 4, 4>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            case 1024: return launch_sap0_lean<T, 4, 8>(U, r, x, blocks, ncol, nrhs, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters, act, s);
            default: break;
        }
    }
    const int bytes = sap0_smem_bytes<T>(sxe * ste, m, use_smem);
    cudaError_t e = cudaFuncSetAttribute(k_sap0_blocks<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    dim3 grid(ncol, nrhs);
    k_sap0_blocks<T><<<grid, 256, bytes, s>>>(U, r, x, blocks, ncol, nx, nt, sbt, sxe, ste, m0, m, restarts, tol,
                                               use_smem, gscratch, iters, act);
    return cudaGetLastError();
}

template <int NV>
static void axpy_dots_nv(double2* w, const double2* V, long long len, long long vstride, int nv, const double2* h,
                         int hstride, int nd, const int* act, int nrhs, double2* partial, int nparts, cudaStream_t s,
                         double2* y = nullptr, const double* sc = nullptr, float2* yf = nullptr) {
    dim3 grid(nparts, nrhs);
    k_axpy_dots<NV><<<grid, 256, 0, s>>>(w, V, len, vstride, nv, h, hstride, nd, act, partial, y, sc, yf);
}

// w -= sum_{k<nv} h[k] V_k (h may be null), then out[rhs][k] = <w, V_k> for k < nd and
// out[rhs][nd] = |w|^2.
void launch_axpy_multidot(double2* w, const double2* V, long long len, long long vstride, int nv, const double2* h,
                          int hstride, int nd, const int* act, int nrhs, double2* partial, int nparts, double2* out,
                          cudaStream_t s) {
    count_launch(2);
    const int n = nv > nd ? nv : nd;
    if (n <= 4) axpy_dots_nv<4>(w, V, len, vstride, nv, h, hstride, nd, act, nrhs, partial, nparts, s);
    else if (n <= 8) axpy_dots_nv<8>(w, V, len, vstride, nv, h, hstride, nd, act, nrhs, partial, nparts, s);
    else if (n <= 12) axpy_dots_nv<12>(w, V, len, vstride, nv, h, hstride, nd, act, nrhs, partial, nparts, s);
    else if (n <= 16) axpy_dots_nv<16>(w, V, len, vstride, nv, h, hstride, nd, act, nrhs, partial, nparts, s);
    else axpy_dots_nv<24>(w, V, len, vstride, nv, h, hstride, nd, act, nrhs, partial, nparts, s);
    k_multidot_sum<<<nrhs * (nd + 1), 256, 0, s>>>(partial, nparts, out);
}

void launch_axpy_scale_to(double2* y, const double2* w, const double2* V, long long len, long long vstride, int nv,
                          const double2* h, int hstride, const double* sc, const int* act, int nrhs, double2* partial,
                          int nparts, cudaStream_t s, float2* yf) {
    count_launch(1);
    double2* ww = const_cast<double2*>(w);   // read only when y is given
    if (nv <= 4) axpy_dots_nv<4>(ww, V, len, vstride, nv, h, hstride, 0, act, nrhs, partial, nparts, s, y, sc, yf);
    else if (nv <= 8) axpy_dots_nv<8>(ww, V, len, vstride, nv, h, hstride, 0, act, nrhs, partial, nparts, s, y, sc, yf);
    else if (nv <= 12) axpy_dots_nv<12>(ww, V, len, vstride, nv, h, hstride, 0, act, nrhs, partial, nparts, s, y, sc, yf);
    else if (nv <= 16) axpy_dots_nv<16>(ww, V, len, vstride, nv, h, hstride, 0, act, nrhs, partial, nparts, s, y, sc, yf);
    else axpy_dots_nv<24>(ww, V, len, vstride, nv, h, hstride, 0, act, nrhs, partial, nparts, s, y, sc, yf);
}

void launch_multidot(const double2* w, const double2* V, long long len, long long vstride, int nv, int nrhs,
                     double2* partial, int nparts, double2* out, const int* act, cudaStream_t s) {
    launch_axpy_multidot(const_cast<double2*>(w), V, len, vstride, 0, nullptr, 0, nv, act, nrhs, partial, nparts, out,
                         s);
}

void launch_multiaxpy(double2* w, const double2* V, long long len, long long vstride, int nv, const double2* h,
                      int hstride, const int* act, int nrhs, cudaStream_t s) {
    count_launch(1);
    dim3 grid(592, nrhs);
    k_multiaxpy<<<grid, 256, 0, s>>>(w, V, len, vstride, nv, h, hstride, act);
}
template <typename TZ>
void launch_multiaxpy_add(double2* x, const TZ* Z, long long len, long long vstride, int nv, const double2* c,
                          int cstride, const int* nvr, const int* act, int nrhs, cudaStream_t s) {
    count_launch(1);
    dim3 grid(592, nrhs);
    k_multiaxpy_add<TZ><<<grid, 256, 0, s>>>(x, Z, len, vstride, nv, c, cstride, nvr, act);
}
template void launch_multiaxpy_add<double2>(double2*, const double2*, long long, long long, int, const double2*, int,
                                            const int*, const int*, int, cudaStream_t);
template void launch_multiaxpy_add<float2>(double2*, const float2*, long long, long long, int, const double2*, int,
                                           const int*, const int*, int, cudaStream_t);
void launch_scale(double2* y, const double2* x, long long len, const double* sc, const int* act, int nrhs,
                  cudaStream_t s, float2* yf) {
    count_launch(1);
    dim3 grid(592, nrhs);
    k_scale<<<grid, 256, 0, s>>>(y, x, len, sc, act, yf);
}
void launch_d2f(float2* y, const double2* x, long long n, cudaStream_t s) {
    count_launch(1); k_d2f<<<592, 256, 0, s>>>(y, x, n); }
void launch_f2d(double2* y, const float2* x, long long n, cudaStream_t s) {
    count_launch(1); k_f2d<<<592, 256, 0, s>>>(y, x, n); }
void launch_d2h(__half2* y, const double2* x, long long n, cudaStream_t s) {
    count_launch(1); k_d2h<<<592, 256, 0, s>>>(y, x, n); }
void launch_d2bf(__nv_bfloat162* y, const double2* x, long long n, cudaStream_t s) {
    count_launch(1); k_d2bf<<<592, 256, 0, s>>>(y, x, n); }

// ---------------------------------------------------------------------------------
// Adjoint support.  gamma5 = diag(1, -1) on the spin index; D^dagger = gamma5 D gamma5
// (the projectors of src/dirac_operator.cpp:3-27 swapped, as D_dagger_phi does, :30-54).
// ---------------------------------------------------------------------------------
__global__ void k_gamma5(double2* __restrict__ y, const double2* __restrict__ x, long long nsites) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsites;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 a = x[2 * i], b = x[2 * i + 1];
        y[2 * i] = a;
        y[2 * i + 1] = make_double2(-b.x, -b.y);
    }
}

// Fermion force F[n][mu] = -sum_r Re(lam_r^dagger (dD/dtheta_mu(n)) x_r) for U = exp(i theta).
// theta_mu(n) enters D through two hops of src/dirac_operator.cpp:11-22: row n, column
// n+mu, -1/2 (1 - sigma_mu) U_mu(n) s; and row n+mu, column n, -1/2 (1 + sigma_mu) conj(U_mu(n)) s,
// with s = -1 on the time hop across t = Nt-1 (the antiperiodic boundary, include/boundary.h:29-40).
// With A = lam(n)^dagger (1 - sigma_mu) x(n+mu) and B = lam(n+mu)^dagger (1 + sigma_mu) x(n):
//   F = s/2 (Im(conj(U) B) - Im(U A)).
// One thread per site; the projector contractions are summed over sources before the link.
__global__ void __launch_bounds__(256) k_force(const double2* __restrict__ U, const double2* __restrict__ lam,
                                               const double2* __restrict__ x, double2* __restrict__ F, int nx,
                                               int nt, int nrhs) {
    const int N = nx * nt;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int xi = n / nt, t = n - xi * nt;
    const int nT = xi * nt + (t + 1 == nt ? 0 : t + 1);
    const int nX = (xi + 1 == nx ? 0 : xi + 1) * nt + t;
    double2 A0 = czero<double>(), B0 = czero<double>(), A1 = czero<double>(), B1 = czero<double>();
    for (int r = 0; r < nrhs; r++) {
        const long long off = (long long)r * N * 2;
        const double2 l0 = lam[off + 2 * n], l1 = lam[off + 2 * n + 1];
        const double2 x0 = x[off + 2 * n], x1 = x[off + 2 * n + 1];
        const double2 xt0 = x[off + 2 * nT], xt1 = x[off + 2 * nT + 1];
        const double2 lt0 = lam[off + 2 * nT], lt1 = lam[off + 2 * nT + 1];
        const double2 xs0 = x[off + 2 * nX], xs1 = x[off + 2 * nX + 1];
        const double2 ls0 = lam[off + 2 * nX], ls1 = lam[off + 2 * nX + 1];
        // time, sigma_0 = [[0,1],[1,0]]: (1 - s0) -> (l0 - l1)^* (x0 - x1), (1 + s0) -> (l0 + l1)^* (x0 + x1)
        cfmac(A0, l0 - l1, xt0 - xt1);
        cfmac(B0, lt0 + lt1, x0 + x1);
        // space, sigma_1 = [[0,-i],[i,0]]: (1 - s1) -> (l0 + i l1)^* (x0 + i x1),
        //                                  (1 + s1) -> (l0 - i l1)^* (x0 - i x1)
        cfmac(A1, l0 + cmuli(l1), xs0 + cmuli(xs1));
        cfmac(B1, ls0 - cmuli(ls1), x0 - cmuli(x1));
    }
    const double2 u0 = U[2 * n], u1 = U[2 * n + 1];
    const double s0 = (t == nt - 1) ? -0.5 : 0.5;
    const double f0 = s0 * ((u0.x * B0.y - u0.y * B0.x) - (u0.x * A0.y + u0.y * A0.x));
    const double f1 = 0.5 * ((u1.x * B1.y - u1.y * B1.x) - (u1.x * A1.y + u1.y * A1.x));
    F[n] = make_double2(f0, f1);
}

void launch_gamma5(double2* y, const double2* x, long long nsites, cudaStream_t s) {
    count_launch(1);
    k_gamma5<<<1184, 256, 0, s>>>(y, x, nsites);
}
void launch_force(const double2* U, const double2* lam, const double2* x, double2* F, int nx, int nt, int nrhs,
                  cudaStream_t s) {
    count_launch(1);
    k_force<<<(nx * nt + 255) / 256, 256, 0, s>>>(U, lam, x, F, nx, nt, nrhs);
}

#define INST(T)                                                                                                 \
    template void launch_dirac<T>(const cx<T>*, const cx<T>*, cx<T>*, int, int, int, T, int, cudaStream_t);     \
    template void launch_residual<T>(const Links<T>, const cx<T>*, long long, const cx<T>*, cx<T>*, int, int, int, T,\
                                     double*, double*, const int*, cudaStream_t);                                \
    template void launch_norm2<T>(const cx<T>*, long long, long long, int, double*, double*, cudaStream_t);      \
    template int sap0_smem_bytes<T>(int, int, int);                                                              \
    template cudaError_t launch_sap0<T>(const Links<T>, cx<T>*, cx<T>*, const int*, int, int, int, int, int, \
                                        int, int, T, int, int, T, int, cx<T>*, int*, const int*, cudaStream_t, int, \
                                        const cx<T>*, long long);
INST(double)
INST(float)
template cudaError_t launch_restrict0<double, double2>(const double2*, const cx<double>*, cx<double>*, cx<double>*, int,
                                                 int, int, int, int, int, int, cudaStream_t);
template cudaError_t launch_restrict0<float, float2>(const float2*, const cx<float>*, cx<float>*, cx<float>*, int, int,
                                               int, int, int, int, int, cudaStream_t);
template cudaError_t launch_restrict0<float, __nv_bfloat162>(const __nv_bfloat162*, const cx<float>*, cx<float>*,
                                                       cx<float>*, int, int, int, int, int, int, int, cudaStream_t);
template void launch_prolong0_add<double, double2>(const double2*, const cx<double>*, cx<double>*, int, int, int,
                                                    int, int, int, cudaStream_t, bool);
template void launch_prolong0_add<float, float2>(const float2*, const cx<float>*, cx<float>*, int, int, int, int,
                                                  int, int, cudaStream_t, bool);
template void launch_prolong0_add<float, __nv_bfloat162>(const __nv_bfloat162*, const cx<float>*, cx<float>*, int,
                                                          int, int, int, int, int, cudaStream_t, bool);

}  // namespace amgb
