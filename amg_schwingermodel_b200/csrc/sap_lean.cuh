// SAP block solve on the fine level, one CTA per Schwarz block (src/sap.cpp:44-62 with the
// block operator of src/level.cpp:304-368 at colors = 1).
//
// The CTA has 32*NW threads and each thread owns SPT sites of the block (S = 32*NW*SPT
// sites).  Everything a thread needs for its sites is set up once: the local indices of the
// four neighbours and the four hop links with the fermionic sign and the factor 1/2 folded
// in (zero, with the neighbour index pointing at the site itself, when the neighbour lies
// outside the block), so applying D_B is branch-free.  The Krylov basis V[0..M] is kept in
// shared memory with the two spin components in separate planes (conflict-free accesses);
// the operator output w, the iterate x and the block's source b stay in registers.  Every
// reduction is a warp shuffle plus one CTA barrier on a double-buffered partial array.
//
// The arithmetic follows FGMRES::fgmres (src/fgmres.cpp:5-115) with x0 = b: modified
// Gram-Schmidt, Givens rotations, the Arnoldi exit |g_{j+1}| < tol*||b||, a true residual
// after each cycle, and maxIt carried over restart cycles.
#pragma once
#include "common.cuh"

namespace amgb {

template <typename T, int NW>
struct LeanRed {
    T* part;      // [2][NW][2*NV] double-buffered partials
    int buf;
};

// Sum of (ax, ay) over the CTA; every thread gets the result.
template <typename T, int NW>
__device__ __forceinline__ cx<T> lean_sum2(T ax, T ay, T* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (NW == 1) return mk<T>(ax, ay);
    T* p = part + buf * NW * 2;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { p[2 * wid] = ax; p[2 * wid + 1] = ay; }
    __syncthreads();
    T sx = 0, sy = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) { sx += p[2 * k]; sy += p[2 * k + 1]; }
    buf ^= 1;
    return mk<T>(sx, sy);
}

template <typename T, int NW>
__device__ __forceinline__ void lean_sync() {
    if (NW == 1) __syncwarp(); else __syncthreads();
}

template <typename T, int M, int SPT, int NW>
__global__ void __launch_bounds__(32 * NW, (sizeof(T) == 4 ? 16 : 8) / NW) k_sap0_lean(const Links<T> U, const cx<T>* __restrict__ r,
                                                       cx<T>* __restrict__ xg, const int* __restrict__ blocks,
                                                       int ncol, int nx, int nt, int sbt, int sxe, int ste, T m0,
                                                       int restarts, T tol, const int* __restrict__ act,
                                                       int* __restrict__ iters_out) {
    constexpr int TPB = 32 * NW, S = TPB * SPT;
    extern __shared__ __align__(16) unsigned char smraw_l[];
    const int seg = blockIdx.x, rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    cx<T>* V = reinterpret_cast<cx<T>*>(smraw_l);          // [M+1][2][S]
    cx<T>* H = V + (M + 1) * 2 * S;                          // [M][M]
    cx<T>* gcs = H + M * M;                                  // g[M+1], cn[M], sn[M]
    T* part = reinterpret_cast<T*>(gcs + 3 * M + 1);         // [2][NW][2]
    cx<T>* gv = gcs;
    cx<T>* cn = gcs + (M + 1);
    cx<T>* sn = cn + M;
    int buf = 0;
    const int tid = threadIdx.x;
    const int block = blocks[seg];
    const int bxi = block / sbt, bti = block - bxi * sbt;
    const int x0 = bxi * sxe, t0 = bti * ste;
    const long long off = (long long)rhs * nx * nt * 2;
    const T mass = m0 + T(2);

    // per-site set-up: global site, neighbour local indices, folded hop links
    int nb[SPT][4];
    cx<T> lk[SPT][4];
    long long gs[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int m = tid + TPB * k;
        const int mx = m / ste, mt = m - mx * ste;
        const int t = t0 + mt, x = x0 + mx;
        gs[k] = (long long)x * nt + t;
        const T half = T(0.5);
        const T sR = (t == nt - 1) ? T(-1) : T(1);
        const T sL = (t == 0) ? T(-1) : T(1);
        // forward time
        int q = -1;
        if (mt + 1 < ste) q = m + 1; else if (ste == nt) q = mx * ste;
        nb[k][0] = q < 0 ? m : q;
        lk[k][0] = q < 0 ? czero<T>() : (half * sR) * U[2 * gs[k]];
        // forward space
        q = -1;
        if (mx + 1 < sxe) q = m + ste; else if (sxe == nx) q = mt;
        nb[k][1] = q < 0 ? m : q;
        lk[k][1] = q < 0 ? czero<T>() : half * U[2 * gs[k] + 1];
        // backward time: conj(U_0(n - t))
        q = -1;
        if (mt > 0) q = m - 1; else if (ste == nt) q = mx * ste + ste - 1;
        nb[k][2] = q < 0 ? m : q;
        if (q >= 0) {
            const long long nl = (long long)x * nt + ((t == 0) ? nt - 1 : t - 1);
            lk[k][2] = (half * sL) * cconj(U[2 * nl]);
        } else {
            lk[k][2] = czero<T>();
        }
        // backward space: conj(U_1(n - x))
        q = -1;
        if (mx > 0) q = m - ste; else if (sxe == nx) q = (sxe - 1) * ste + mt;
        nb[k][3] = q < 0 ? m : q;
        if (q >= 0) {
            const long long nl = (long long)((x == 0) ? nx - 1 : x - 1) * nt + t;
            lk[k][3] = half * cconj(U[2 * nl + 1]);
        } else {
            lk[k][3] = czero<T>();
        }
    }
    // out = D_B v for this thread's sites; v is a basis slot [2][S]
    auto apply = [&](const cx<T>* v, cx<T> (&w)[SPT][2]) {
        const cx<T>* v0 = v;
        const cx<T>* v1 = v + S;
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int m = tid + TPB * k;
            const cx<T> ta = cmul(lk[k][0], v0[nb[k][0]] - v1[nb[k][0]]);
            const cx<T> tb = cmul(lk[k][1], v0[nb[k][1]] + cmuli(v1[nb[k][1]]));
            const cx<T> tc = cmul(lk[k][2], v0[nb[k][2]] + v1[nb[k][2]]);
            const cx<T> td = cmul(lk[k][3], v0[nb[k][3]] - cmuli(v1[nb[k][3]]));
            w[k][0] = mass * v0[m] - (ta + tb + tc + td);
            w[k][1] = mass * v1[m] - ((tc - ta) + cmuli(td - tb));
        }
    };
    auto store = [&](cx<T>* v, const cx<T> (&a)[SPT][2]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int m = tid + TPB * k;
            v[m] = a[k][0];
            v[S + m] = a[k][1];
        }
    };
    auto norm2 = [&](const cx<T> (&a)[SPT][2]) -> T {
        T s = 0;
#pragma unroll
        for (int k = 0; k < SPT; k++) s += cnorm2(a[k][0]) + cnorm2(a[k][1]);
        return lean_sum2<T, NW>(s, T(0), part, buf).x;
    };

    // the block's source b is the global residual, read through L1 where it is needed
    const cx<T>* rb = r + off;
    cx<T> x[SPT][2], w[SPT][2];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        x[k][0] = __ldg(&rb[2 * gs[k]]);
        x[k][1] = __ldg(&rb[2 * gs[k] + 1]);
    }
    // r = b - A x0 (x0 = b) into V0
    store(V, x);
    const T normb = sqrt(norm2(x));
    lean_sync<T, NW>();
    apply(V, w);
#pragma unroll
    for (int k = 0; k < SPT; k++) { w[k][0] = x[k][0] - w[k][0]; w[k][1] = x[k][1] - w[k][1]; }
    T err = sqrt(norm2(w));
    int maxit = M;
    int ret = restarts * M;
    for (int kk = 0; kk < restarts; kk++) {
        // V0 = r / beta (r is in w), g0 = beta
        {
            const T inv = T(1) / err;
#pragma unroll
            for (int k = 0; k < SPT; k++) { w[k][0] = inv * w[k][0]; w[k][1] = inv * w[k][1]; }
            store(V, w);
        }
        if (tid == 0) gv[0] = mk<T>(err, T(0));
        lean_sync<T, NW>();
#pragma unroll
        for (int j = 0; j < M; j++) {
            const cx<T>* Vj = V + j * 2 * S;
            apply(Vj, w);
            cx<T> col[M + 1];
            // modified Gram-Schmidt (src/fgmres.cpp:24-32)
#pragma unroll
            for (int i = 0; i <= j; i++) {
                const cx<T>* Vi = V + i * 2 * S;
                T ax = 0, ay = 0;
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const int m = tid + TPB * k;
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        const cx<T> u = w[k][s], vv = Vi[s * S + m];
                        ax += u.x * vv.x + u.y * vv.y;
                        ay += u.y * vv.x - u.x * vv.y;
                    }
                }
                const cx<T> h = lean_sum2<T, NW>(ax, ay, part, buf);
                col[i] = h;
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const int m = tid + TPB * k;
                    cfma(w[k][0], -h, Vi[m]);
                    cfma(w[k][1], -h, Vi[S + m]);
                }
            }
            const T hn = sqrt(norm2(w));
            if (hn > T(0)) {
                const T inv = T(1) / hn;
                cx<T>* Vn = V + (j + 1) * 2 * S;
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const int m = tid + TPB * k;
                    Vn[m] = inv * w[k][0];
                    Vn[S + m] = inv * w[k][1];
                }
            }
            // rotation(j) (src/fgmres.cpp:90-104): warp 0 computes it, lane 0 stores it
            lean_sync<T, NW>();
            if (tid < 32) {
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
                if (tid == 0) {
#pragma unroll
                    for (int i = 0; i <= j; i++) H[i * M + j] = col[i];
                    sn[j] = snj;
                    cn[j] = cnj;
                    gv[j + 1] = -cmul(snj, gj);
                    gv[j] = cmulc(cnj, gj);
                }
            }
            lean_sync<T, NW>();
            if (sqrt(cnorm2(gv[j + 1])) < tol * normb) {
                maxit = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115) and x += sum eta_j V_j
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
            const cx<T>* Vj = V + jj * 2 * S;
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const int m = tid + TPB * k;
                cfma(x[k][0], eta[jj], Vj[m]);
                cfma(x[k][1], eta[jj], Vj[S + m]);
            }
        }
        // true residual r = b - A x (x staged through V1, r into V0).  After the last cycle it
        // only decides the returned iteration count, so it is skipped when nobody reads that.
        if (kk == restarts - 1 && !iters_out) break;
        lean_sync<T, NW>();
        store(V + 2 * S, x);
        lean_sync<T, NW>();
        apply(V + 2 * S, w);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            w[k][0] = __ldg(&rb[2 * gs[k]]) - w[k][0];
            w[k][1] = __ldg(&rb[2 * gs[k] + 1]) - w[k][1];
        }
        err = sqrt(norm2(w));
        if (err < tol * normb) {
            ret = kk * M + maxit;
            break;
        }
        lean_sync<T, NW>();
    }
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        xg[off + 2 * gs[k]] += x[k][0];
        xg[off + 2 * gs[k] + 1] += x[k][1];
    }
    if (iters_out && tid == 0) iters_out[rhs * ncol + seg] = ret;
}

template <typename T, int M, int SPT, int NW>
inline int sap0_lean_smem() {
    constexpr int S = 32 * NW * SPT;
    return ((M + 1) * 2 * S + M * M + 3 * M + 1) * (int)sizeof(cx<T>) + 2 * NW * 2 * (int)sizeof(T) + 16;
}

}  // namespace amgb
