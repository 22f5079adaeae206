// SAP block solve with one warp per block (src/sap.cpp:44-62 with the block operator of
// src/level.cpp:304-368 at colors = 1).
//
// Each warp owns one Schwarz block of S = 32*SPL sites and runs the reference's
// GMRES(M, restarts, tol) with x0 = b on it.  The Krylov basis V[0..M] lives in shared
// memory (the only on-chip storage a block needs); the operator output w and the solution x
// are held in registers (SPL sites x 2 spins per lane); the block's source b (the global
// residual) and its links are read through L1.  Reductions are warp shuffles, so no CTA
// barrier appears anywhere and each warp runs its block at its own pace.
#pragma once
#include "common.cuh"

namespace amgb {

template <typename T>
__device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct BlockGeo {
    int nx, nt, sxe, ste, x0, t0;
};

// w = D_B v for the SPL sites of this lane; v is the block vector in shared memory.
template <typename T, int SPL>
__device__ __forceinline__ void warp_block_apply(const BlockGeo& g, const cx<T>* __restrict__ U, T mass,
                                                 const cx<T>* v, cx<T> (&w)[SPL][2], int lane) {
#pragma unroll
    for (int k = 0; k < SPL; k++) {
        const int m = lane + 32 * k;
        const int mx = m / g.ste, mt = m - mx * g.ste;
        const int t = g.t0 + mt;
        const long long n = (long long)(g.x0 + mx) * g.nt + t;
        const T sR = (t == g.nt - 1) ? T(-1) : T(1);
        const T sL = (t == 0) ? T(-1) : T(1);
        int mr0 = -1, mr1 = -1, ml0 = -1, ml1 = -1;
        if (mt + 1 < g.ste) mr0 = m + 1; else if (g.ste == g.nt) mr0 = mx * g.ste;
        if (mt > 0) ml0 = m - 1; else if (g.ste == g.nt) ml0 = mx * g.ste + g.ste - 1;
        if (mx + 1 < g.sxe) mr1 = m + g.ste; else if (g.sxe == g.nx) mr1 = mt;
        if (mx > 0) ml1 = m - g.ste; else if (g.sxe == g.nx) ml1 = (g.sxe - 1) * g.ste + mt;
        const cx<T> p0 = v[2 * m], p1 = v[2 * m + 1];
        cx<T> t0 = czero<T>(), t1 = czero<T>(), t2 = czero<T>(), t3 = czero<T>();
        if (mr0 >= 0) t0 = sR * cmul(__ldg(&U[2 * n]), v[2 * mr0] - v[2 * mr0 + 1]);
        if (mr1 >= 0) t1 = cmul(__ldg(&U[2 * n + 1]), v[2 * mr1] + cmuli(v[2 * mr1 + 1]));
        if (ml0 >= 0) {
            const long long nl = (long long)(g.x0 + ml0 / g.ste) * g.nt + g.t0 + (ml0 - (ml0 / g.ste) * g.ste);
            t2 = sL * cmul(cconj(__ldg(&U[2 * nl])), v[2 * ml0] + v[2 * ml0 + 1]);
        }
        if (ml1 >= 0) {
            const long long nl = (long long)(g.x0 + ml1 / g.ste) * g.nt + g.t0 + (ml1 - (ml1 / g.ste) * g.ste);
            t3 = cmul(cconj(__ldg(&U[2 * nl + 1])), v[2 * ml1] - cmuli(v[2 * ml1 + 1]));
        }
        w[k][0] = mass * p0 - T(0.5) * (t0 + t1 + t2 + t3);
        w[k][1] = mass * p1 - T(0.5) * ((t2 - t0) + cmuli(t3 - t1));
    }
}

// dot of the lane-distributed register vector a with the shared vector v: sum a conj(v)
template <typename T, int SPL>
__device__ __forceinline__ cx<T> warp_dot_rv(const cx<T> (&a)[SPL][2], const cx<T>* v, int lane) {
    T sx = 0, sy = 0;
#pragma unroll
    for (int k = 0; k < SPL; k++) {
        const int m = lane + 32 * k;
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const cx<T> u = a[k][s], b = v[2 * m + s];
            sx += u.x * b.x + u.y * b.y;
            sy += u.y * b.x - u.x * b.y;
        }
    }
    return mk<T>(wsum(sx), wsum(sy));
}

template <typename T, int SPL>
__device__ __forceinline__ T warp_norm2_r(const cx<T> (&a)[SPL][2]) {
    T s = 0;
#pragma unroll
    for (int k = 0; k < SPL; k++) s += cnorm2(a[k][0]) + cnorm2(a[k][1]);
    return wsum(s);
}

// One warp: GMRES on the block, then x_global[block] += solution.  Returns the reference's
// FGMRES return value for the block (k*M + maxIt, or restarts*M).
template <typename T, int M, int SPL>
__device__ int warp_block_gmres(const BlockGeo& g, const cx<T>* __restrict__ U, const cx<T>* __restrict__ r,
                                cx<T>* __restrict__ xg, T mass, int restarts, T tol, cx<T>* V, cx<T>* H, cx<T>* sc,
                                int lane) {
    const int len = 64 * SPL;
    // per-warp scalars in shared memory: g[M+1], cn[M], sn[M]
    cx<T>* gv = sc;
    cx<T>* cn = sc + (M + 1);
    cx<T>* sn = cn + M;
    cx<T> x[SPL][2], w[SPL][2];
    auto gsite = [&](int m) -> long long {
        const int mx = m / g.ste, mt = m - mx * g.ste;
        return (long long)(g.x0 + mx) * g.nt + g.t0 + mt;
    };
#pragma unroll
    for (int k = 0; k < SPL; k++) {
        const int m = lane + 32 * k;
        const long long n = gsite(m);
        x[k][0] = __ldg(&r[2 * n]);
        x[k][1] = __ldg(&r[2 * n + 1]);
        V[2 * m] = x[k][0];
        V[2 * m + 1] = x[k][1];
    }
    __syncwarp();
    // r = b - A x0 with x0 = b, into V0
    warp_block_apply<T, SPL>(g, U, mass, V, w, lane);
    __syncwarp();
    T nb2 = 0;
#pragma unroll
    for (int k = 0; k < SPL; k++) {
        const int m = lane + 32 * k;
        nb2 += cnorm2(x[k][0]) + cnorm2(x[k][1]);
        w[k][0] = x[k][0] - w[k][0];
        w[k][1] = x[k][1] - w[k][1];
        V[2 * m] = w[k][0];
        V[2 * m + 1] = w[k][1];
    }
    T err = sqrt(warp_norm2_r<T, SPL>(w));
    const T normb = sqrt(wsum(nb2));
    int maxit = M;
    int ret = restarts * M;
    for (int kk = 0; kk < restarts; kk++) {
        // V0 = r / beta, g0 = beta
        {
            const T inv = T(1) / err;
#pragma unroll
            for (int k = 0; k < SPL; k++) {
                const int m = lane + 32 * k;
                V[2 * m] = inv * V[2 * m];
                V[2 * m + 1] = inv * V[2 * m + 1];
            }
        }
        if (lane == 0) gv[0] = mk<T>(err, T(0));
        __syncwarp();
#pragma unroll
        for (int j = 0; j < M; j++) {
            const cx<T>* Vj = V + j * len;
            warp_block_apply<T, SPL>(g, U, mass, Vj, w, lane);
            // modified Gram-Schmidt (src/fgmres.cpp:24-32); column j of H kept in registers
            cx<T> col[M + 1];
#pragma unroll
            for (int i = 0; i <= j; i++) {
                const cx<T>* Vi = V + i * len;
                const cx<T> h = warp_dot_rv<T, SPL>(w, Vi, lane);
                col[i] = h;
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    const int m = lane + 32 * k;
                    cfma(w[k][0], -h, Vi[2 * m]);
                    cfma(w[k][1], -h, Vi[2 * m + 1]);
                }
            }
            const T hn = sqrt(warp_norm2_r<T, SPL>(w));
            if (hn > T(0)) {
                const T inv = T(1) / hn;
                cx<T>* Vn = V + (j + 1) * len;
#pragma unroll
                for (int k = 0; k < SPL; k++) {
                    const int m = lane + 32 * k;
                    Vn[2 * m] = inv * w[k][0];
                    Vn[2 * m + 1] = inv * w[k][1];
                }
            }
            // rotation(j) (src/fgmres.cpp:90-104), identical in every lane
            col[j + 1] = mk<T>(hn, T(0));
#pragma unroll
            for (int i = 0; i < j; i++) {
                const cx<T> c = cn[i], s = sn[i];
                const cx<T> temp = cmulc(c, col[i]) + cmulc(s, col[i + 1]);
                col[i + 1] = cmul(c, col[i + 1]) - cmul(s, col[i]);
                col[i] = temp;
            }
            const T den = sqrt(cnorm2(col[j]) + cnorm2(col[j + 1]));
            const cx<T> snj = mk<T>(col[j + 1].x / den, col[j + 1].y / den);
            const cx<T> cnj = mk<T>(col[j].x / den, col[j].y / den);
            col[j] = cmulc(cnj, col[j]) + cmulc(snj, col[j + 1]);
            const cx<T> gj = gv[j];
            const cx<T> gj1 = -cmul(snj, gj);
            __syncwarp();
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i <= j; i++) H[i * M + j] = col[i];
                sn[j] = snj;
                cn[j] = cnj;
                gv[j + 1] = gj1;
                gv[j] = cmulc(cnj, gj);
            }
            __syncwarp();
            if (sqrt(cnorm2(gj1)) < tol * normb) {
                maxit = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115), then x += sum eta_j V_j
        cx<T> eta[M];
#pragma unroll
        for (int i = M - 1; i >= 0; i--) {
            if (i >= maxit) { eta[i] = czero<T>(); continue; }
            cx<T> o = gv[i];
#pragma unroll
            for (int jj = i + 1; jj < M; jj++)
                if (jj < maxit) o = o - cmul(H[i * M + jj], eta[jj]);
            eta[i] = cdiv(o, H[i * M + i]);
        }
#pragma unroll
        for (int jj = 0; jj < M; jj++) {
            if (jj >= maxit) break;
            const cx<T>* Vj = V + jj * len;
#pragma unroll
            for (int k = 0; k < SPL; k++) {
                const int m = lane + 32 * k;
                cfma(x[k][0], eta[jj], Vj[2 * m]);
                cfma(x[k][1], eta[jj], Vj[2 * m + 1]);
            }
        }
        __syncwarp();
        // true residual r = b - A x: x goes through V1 (free at the end of a cycle), r into V0
        cx<T>* X = V + len;
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int m = lane + 32 * k;
            X[2 * m] = x[k][0];
            X[2 * m + 1] = x[k][1];
        }
        __syncwarp();
        warp_block_apply<T, SPL>(g, U, mass, X, w, lane);
#pragma unroll
        for (int k = 0; k < SPL; k++) {
            const int m = lane + 32 * k;
            const long long n = gsite(m);
            w[k][0] = __ldg(&r[2 * n]) - w[k][0];
            w[k][1] = __ldg(&r[2 * n + 1]) - w[k][1];
            V[2 * m] = w[k][0];
            V[2 * m + 1] = w[k][1];
        }
        err = sqrt(warp_norm2_r<T, SPL>(w));
        __syncwarp();
        if (err < tol * normb) {
            ret = kk * M + maxit;
            break;
        }
    }
#pragma unroll
    for (int k = 0; k < SPL; k++) {
        const long long n = gsite(lane + 32 * k);
        xg[2 * n] += x[k][0];
        xg[2 * n + 1] += x[k][1];
    }
    return ret;
}

}  // namespace amgb

namespace amgb {

template <typename T, int M, int SPL, int WPB>
__global__ void __launch_bounds__(32 * WPB) k_sap0_warp(const cx<T>* __restrict__ U, const cx<T>* __restrict__ r,
                                                        cx<T>* __restrict__ x, const int* __restrict__ blocks, int ncol,
                                                        int nx, int nt, int sbt, int sxe, int ste, T m0, int restarts,
                                                        T tol, const int* __restrict__ act, int* __restrict__ iters_out) {
    extern __shared__ __align__(16) unsigned char smraw_w[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int seg = blockIdx.x * WPB + warp, rhs = blockIdx.y;
    if (seg >= ncol) return;
    if (act && !act[rhs]) return;
    constexpr int len = 64 * SPL;
    constexpr int per_warp = (M + 1) * len + M * M + 3 * M + 1;
    cx<T>* V = reinterpret_cast<cx<T>*>(smraw_w) + warp * per_warp;
    cx<T>* H = V + (M + 1) * len;
    cx<T>* sc = H + M * M;
    const int block = blocks[seg];
    const int bxi = block / sbt, bti = block - bxi * sbt;
    BlockGeo g;
    g.nx = nx; g.nt = nt; g.sxe = sxe; g.ste = ste; g.x0 = bxi * sxe; g.t0 = bti * ste;
    const long long off = (long long)rhs * nx * nt * 2;
    const int ret = warp_block_gmres<T, M, SPL>(g, U, r + off, x + off, m0 + T(2), restarts, tol, V, H, sc, lane);
    if (iters_out && lane == 0) iters_out[rhs * ncol + seg] = ret;
}

template <typename T, int M, int SPL>
inline int sap0_warp_smem(int wpb) { return wpb * ((M + 1) * 64 * SPL + M * M + 3 * M + 1) * (int)sizeof(cx<T>); }

}  // namespace amgb
