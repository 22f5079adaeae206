// FP32 SAP block solve with a communication-avoiding GMRES(5): the same block solve as the
// reference (src/sap.cpp:44-62, GMRES_D_B include/sap.h:27-47, FGMRES::fgmres
// src/fgmres.cpp:5-115 with x0 = b, restart length 5), restructured so that a restart cycle
// needs one CTA reduction per basis vector instead of one per Gram-Schmidt projection.
//
// Mathematically every restart cycle computes the reference's iterate: the minimiser of
// |r - D_B y| over the Krylov space K_5(D_B, r).  Instead of building an orthonormal basis
// with modified Gram-Schmidt (one CTA reduction per projection), a cycle builds the shifted
// power basis B_0 = r/|r|, B_{j+1} = (D_B - s) B_j with s = m0 + 2 (the block operator's
// diagonal, which keeps the basis well conditioned), and the Gram matrix G = B^H B, whose
// column j+1 is reduced over the CTA in one step together with B_{j+1}.  With G = R^H R
// (Cholesky), Q = B R^{-1} is orthonormal and D_B Q_5 = Q Hb with
//     Hb = s I + R[:, 1:6] W,   W = R[0:5, 0:5]^{-1}
// (upper Hessenberg), so the least-squares problem, its Givens rotations and the Arnoldi
// exit test |g_{j+1}| < tol |b| are the reference's (src/fgmres.cpp:90-115) on Hb, and the
// update is x += B_5 W y.  R, W, Hb and the rotations are built one column per step by every
// thread (the reduced Gram column is the same in all threads); thread 0 keeps the columns
// that later steps read in shared memory.  The true residual after each cycle, maxIt across
// restarts and the returned count follow the reference.
//
// Storage as in the paired kernel (sap_f32.cuh): a basis vector is one float4 per site in
// shared memory, a site is a pair of f32x2 values in registers.
#pragma once
#include "common.cuh"
#include "sap_f32.cuh"

namespace amgb {

// Sum over the CTA of NV complex values per thread; every thread receives the sums.
// part: [2][NW][NV] float2, double-buffered (one barrier per call).
template <int NW, int NV>
__device__ __forceinline__ void psum_vec(float2 (&v)[NV], float2* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            float2 b;
            b.x = __shfl_xor_sync(0xffffffffu, v[q].x, o);
            b.y = __shfl_xor_sync(0xffffffffu, v[q].y, o);
            v[q] = p_add(v[q], b);
        }
    }
    if (NW == 1) {
        // one warp: still a memory fence and a point every lane passes together, so the
        // lane-0 writes before it are seen by every lane after it
        __syncwarp();
        return;
    }
    float2* p = part + buf * NW * 6;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) p[wid * 6 + q] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = p[q];
#pragma unroll
    for (int k = 1; k < NW; k++) {
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] = p_add(v[q], p[k * 6 + q]);
    }
    buf ^= 1;
}

// CTA sum of one real per thread, in the same double-buffered area and buffer sequence as
// psum_vec (a buffer's region never overlaps the other buffer's).
template <int NW>
__device__ __forceinline__ float psum1_ca(float a, float2* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (NW == 1) {
        __syncwarp();
        return a;
    }
    float* p = reinterpret_cast<float*>(part + buf * NW * 6);
    if ((threadIdx.x & 31) == 0) p[threadIdx.x >> 5] = a;
    __syncthreads();
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < NW; k++) sum += p[k];
    buf ^= 1;
    return sum;
}

template <int SPT, int NW>
__global__ void __launch_bounds__(32 * NW, 2) k_sap0_ca(const Links<float> U, const float2* __restrict__ r,
                                                         float2* __restrict__ xg, const int* __restrict__ blocks,
                                                         int ncol, int nx, int nt, int sbt, int sxe, int ste, float m0,
                                                         int restarts, float tol, const int* __restrict__ act,
                                                         int* __restrict__ iters_out) {
    constexpr int M = 5, TPB = 32 * NW, S = TPB * SPT;
    extern __shared__ __align__(16) unsigned char smraw_ca[];
    const int seg = blockIdx.x, rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    float4* P = reinterpret_cast<float4*>(smraw_ca);            // planes: B_0..B_4, staging (5)
    float2* Rs = reinterpret_cast<float2*>(P + (M + 1) * S);     // R[i][c] at i*6 + c  (6 x 6)
    float2* Ws = Rs + 36;                                        // W[i][j] at i*5 + j  (5 x 5)
    float2* Hs = Ws + 25;                                        // rotated Hb[i][j] at i*5 + j
    float2* Cs = Hs + 30;                                        // cn[5], sn[5], g[6]
    float2* part = Cs + 16;                                      // [2][NW][6]
    float2* cvec = part + 2 * NW * 6;                            // x update coefficients c = W y
    // flag[0..1]: Arnoldi exit seen at a step of even / odd index (written by warp 0 after a
    // step's barrier, read by everyone after the next step's barrier, so a step's write never
    // meets a read of the same word); flag[2]: maxit
    int* flag = reinterpret_cast<int*>(cvec + 5);
    int buf = 0;
    const int tid = threadIdx.x;
    const int block = blocks[seg];
    const int bxi = block / sbt, bti = block - bxi * sbt;
    const int x0 = bxi * sxe, t0 = bti * ste;
    const long long off = (long long)rhs * nx * nt * 2;
    const float mass = m0 + 2.0f;
    const float sig = mass;                                      // basis shift

    // neighbour local indices (< 65536) packed two per register: nbp[k][0] = t+ | t-,
    // nbp[k][1] = x+ | x-; the global site of local site m is recomputed where needed
    unsigned nbp[SPT][2];
    float2 lk[SPT][4];
    auto gsite = [&](int k) {
        const int m = tid + TPB * k;
        const int mx = m / ste, mt = m - mx * ste;
        return (x0 + mx) * nt + t0 + mt;
    };
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int m = tid + TPB * k;
        const int mx = m / ste, mt = m - mx * ste;
        const int t = t0 + mt, x = x0 + mx;
        const int gsk = x * nt + t;
        int nb[4];
        const float sR = (t == nt - 1) ? -0.5f : 0.5f;
        const float sL = (t == 0) ? -0.5f : 0.5f;
        int q = -1;
        if (mt + 1 < ste) q = m + 1; else if (ste == nt) q = mx * ste;
        nb[0] = q < 0 ? m : q;
        lk[k][0] = q < 0 ? czero<float>() : sR * U[2 * gsk];
        q = -1;
        if (mx + 1 < sxe) q = m + ste; else if (sxe == nx) q = mt;
        nb[1] = q < 0 ? m : q;
        lk[k][1] = q < 0 ? czero<float>() : 0.5f * U[2 * gsk + 1];
        q = -1;
        if (mt > 0) q = m - 1; else if (ste == nt) q = mx * ste + ste - 1;
        nb[2] = q < 0 ? m : q;
        lk[k][2] = q < 0 ? czero<float>() : sL * cconj(U[2 * (x * nt + ((t == 0) ? nt - 1 : t - 1))]);
        q = -1;
        if (mx > 0) q = m - ste; else if (sxe == nx) q = (sxe - 1) * ste + mt;
        nb[3] = q < 0 ? m : q;
        lk[k][3] = q < 0 ? czero<float>() : 0.5f * cconj(U[2 * (((x == 0) ? nx - 1 : x - 1) * nt + t) + 1]);
        nbp[k][0] = (unsigned)nb[0] | ((unsigned)nb[2] << 16);
        nbp[k][1] = (unsigned)nb[1] | ((unsigned)nb[3] << 16);
    }

    // w = D_B v (- s v_own when shifted) for this thread's sites
    auto apply = [&](const float4* __restrict__ v, SiteP (&w)[SPT], float diag) {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int m = tid + TPB * k;
            const float4 c = v[m], a = v[nbp[k][0] & 0xffffu], b = v[nbp[k][1] & 0xffffu], e = v[nbp[k][0] >> 16],
                         g = v[nbp[k][1] >> 16];
            const float2 ta = cmul(lk[k][0], make_float2(a.x - a.y, a.z - a.w));
            const float2 tb = cmul(lk[k][1], make_float2(b.x - b.w, b.z + b.y));
            const float2 tc = cmul(lk[k][2], make_float2(e.x + e.y, e.z + e.w));
            const float2 td = cmul(lk[k][3], make_float2(g.x + g.w, g.z - g.y));
            w[k].re = make_float2(diag * c.x - (ta.x + tb.x + tc.x + td.x), diag * c.y - tc.x + ta.x + td.y - tb.y);
            w[k].im = make_float2(diag * c.z - (ta.y + tb.y + tc.y + td.y), diag * c.w - tc.y + ta.y - td.x + tb.x);
        }
    };
    auto norm2 = [&](const SiteP (&a)[SPT]) -> float {
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            acc = p_fma(a[k].re, a[k].re, acc);
            acc = p_fma(a[k].im, a[k].im, acc);
        }
        return psum1_ca<NW>(acc.x + acc.y, part, buf);
    };
    auto store = [&](float4* Pd, const SiteP (&a)[SPT]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) site_st(Pd, tid + TPB * k, a[k]);
    };
    // <u, v> summed over this thread's sites and both spins (packed)
    auto dotp = [&](const SiteP& u, const SiteP& v, float2& ar, float2& ai, float2& an) {
        ar = p_fma(v.re, u.re, ar);
        ar = p_fma(v.im, u.im, ar);
        ai = p_fma(v.im, u.re, ai);
        an = p_fma(v.re, u.im, an);
    };

    const float4* rb4 = reinterpret_cast<const float4*>(r + off);
    float4* stg = P + M * S;
    SiteP x[SPT], w[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) x[k] = site_from_global(__ldg(&rb4[gsite(k)]));
    // r = b - A x0 (x0 = b)
    store(stg, x);
    const float normb = sqrtf(norm2(x));
    __syncthreads();
    apply(stg, w, mass);
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        w[k].re = p_sub(x[k].re, w[k].re);
        w[k].im = p_sub(x[k].im, w[k].im);
    }
    if (tid == 0) flag[2] = M;   // maxit, carried over restart cycles as the reference does
    float err = sqrtf(norm2(w));
    int ret = restarts * M;
    int maxit = M;
    for (int kk = 0; kk < restarts; kk++) {
        // B_0 = r / |r|
        {
            const float2 inv = p_bc(1.0f / err);
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                w[k].re = p_mul(inv, w[k].re);
                w[k].im = p_mul(inv, w[k].im);
            }
            store(P, w);
        }
        float2 g_cur = make_float2(0.f, 0.f);   // g[j] of the running rotation (warp 0)
        if (tid == 0) { flag[0] = 0; flag[1] = 0; }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < M; j++) {
            // B_{j+1} = (D_B - s) B_j, stored for the next step (B_5 only enters the Gram matrix)
            apply(P + j * S, w, mass - sig);
            if (j + 1 < M) store(P + (j + 1) * S, w);
            // Gram column j+1: <B_i, B_{j+1}> for i <= j+1 (and <B_0, B_0> with the first)
            constexpr int NV = 6;
            float2 gc[NV];
            {
                // <B_i, B_{j+1}>: re += B_i.re w.re + B_i.im w.im, im += B_i.re w.im - B_i.im w.re
                float2 ar[NV], ai[NV];
#pragma unroll
                for (int q = 0; q < NV; q++) { ar[q] = make_float2(0.f, 0.f); ai[q] = ar[q]; }
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const float2 nwre = p_sub(make_float2(0.f, 0.f), w[k].re);
#pragma unroll
                    for (int i = 0; i <= j; i++) {
                        const SiteP bi = site_ld(P + i * S, tid + TPB * k);
                        ar[i] = p_fma(w[k].re, bi.re, ar[i]);
                        ar[i] = p_fma(w[k].im, bi.im, ar[i]);
                        ai[i] = p_fma(w[k].im, bi.re, ai[i]);
                        ai[i] = p_fma(nwre, bi.im, ai[i]);
                        if (j == 0) {
                            ar[NV - 1] = p_fma(bi.re, bi.re, ar[NV - 1]);
                            ar[NV - 1] = p_fma(bi.im, bi.im, ar[NV - 1]);
                        }
                    }
                    ar[j + 1] = p_fma(w[k].re, w[k].re, ar[j + 1]);
                    ar[j + 1] = p_fma(w[k].im, w[k].im, ar[j + 1]);
                }
#pragma unroll
                for (int q = 0; q < NV; q++) gc[q] = make_float2(ar[q].x + ar[q].y, ai[q].x + ai[q].y);
            }
            psum_vec<NW, NV>(gc, part, buf);
            // warp 0 ran the previous step's algebra before this barrier: stop if the Arnoldi
            // exit test held there (this step's vector was computed ahead and is not used)
            if (j > 0 && flag[(j - 1) & 1]) break;
            if (tid >= 32) continue;
            // ---- warp 0: column j+1 of R, column j of W and Hb, rotation j ----
            // Lane i owns row i.  With W = R^{-1} (upper triangular) every piece is a short
            // triangular product instead of a substitution:
            //   W[0:j, j] = -W[0:j, 0:j] R[0:j, j] / R[j][j],  W[j][j] = 1 / R[j][j]
            //   R[0:c, c] = W[0:c, 0:c]^H G[0:c, c],  R[c][c] = sqrt(G[c][c] - |R[0:c, c]|^2)
            //   Hb[i][j]  = s d_ij + sum_{q <= j} R[i][q+1] W[q][j]
            const int lane = tid;
            const int c = j + 1;
            const float r00 = sqrtf(gc[NV - 1].x);
            const float rjj = (j == 0) ? r00 : Rs[j * 6 + j].x;
            if (j == 0 && lane == 0) Rs[0] = make_float2(r00, 0.f);
            float2 wij = czero<float>();
            if (lane < j) {
                float2 acc = czero<float>();
#pragma unroll
                for (int q = 0; q < M; q++)
                    if (q >= lane && q < j) acc = acc + cmul(Ws[lane * 5 + q], Rs[q * 6 + j]);
                wij = make_float2(-acc.x / rjj, -acc.y / rjj);
            } else if (lane == j) {
                wij = make_float2(1.0f / rjj, 0.f);
            }
            if (lane <= j) Ws[lane * 5 + j] = wij;
            __syncwarp();
            float2 rci = czero<float>();
            if (lane < c) {
#pragma unroll
                for (int q = 0; q < M; q++)
                    if (q <= lane) rci = rci + cmulc(Ws[q * 5 + lane], gc[q]);
            }
            float ss = lane < c ? cnorm2(rci) : 0.f;
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
            if (lane == c) rci = make_float2(sqrtf(fmaxf(gc[c].x - ss, 0.f)), 0.f);
            if (lane <= c) Rs[lane * 6 + c] = rci;
            __syncwarp();
            float2 hi = czero<float>();
            if (lane <= c) {
#pragma unroll
                for (int q = 0; q < M; q++)
                    if (q <= j && q + 1 >= lane) hi = hi + cmul(Rs[lane * 6 + q + 1], Ws[q * 5 + j]);
                if (lane == j) hi = hi + make_float2(sig, 0.f);
            }
            // rotation(j) (src/fgmres.cpp:90-104), every lane on the gathered column
            float2 h[M + 1];
#pragma unroll
            for (int i = 0; i <= M; i++) {
                h[i].x = __shfl_sync(0xffffffffu, hi.x, i);
                h[i].y = __shfl_sync(0xffffffffu, hi.y, i);
            }
            if (j == 0) g_cur = make_float2(err * r00, 0.f);
#pragma unroll
            for (int i = 0; i < j; i++) {
                const float2 cn = Cs[i], sn = Cs[5 + i];
                const float2 temp = cmulc(cn, h[i]) + cmulc(sn, h[i + 1]);
                h[i + 1] = cmul(cn, h[i + 1]) - cmul(sn, h[i]);
                h[i] = temp;
            }
            const float den = sqrtf(cnorm2(h[j]) + cnorm2(h[j + 1]));
            const float2 snj = make_float2(h[j + 1].x / den, h[j + 1].y / den);
            const float2 cnj = make_float2(h[j].x / den, h[j].y / den);
            h[j] = cmulc(cnj, h[j]) + cmulc(snj, h[j + 1]);
            const float2 gnext = -cmul(snj, g_cur);
            g_cur = cmulc(cnj, g_cur);
            if (lane <= j) Hs[lane * 5 + j] = h[lane];
            if (lane == 0) {
                Cs[j] = cnj;
                Cs[5 + j] = snj;
                Cs[10 + j] = g_cur;
                Cs[10 + j + 1] = gnext;
            }
            g_cur = gnext;
            if (sqrtf(cnorm2(gnext)) < tol * normb && lane == 0) {
                flag[j & 1] = 1;
                flag[2] = j + 1;
            }
        }
        // warp 0: solve_upper_triangular (src/fgmres.cpp:107-115) on the rotated Hb, c = W y
        if (tid < 32) {
            __syncwarp();
            const int mi = flag[2];
            float2 y[M];
#pragma unroll
            for (int i = M - 1; i >= 0; i--) {
                if (i >= mi) { y[i] = czero<float>(); continue; }
                float2 o = Cs[10 + i];
#pragma unroll
                for (int jj = i + 1; jj < M; jj++)
                    if (jj < mi) o = o - cmul(Hs[i * 5 + jj], y[jj]);
                y[i] = cdiv(o, Hs[i * 5 + i]);
            }
            if (tid < M) {
                float2 ci = czero<float>();
#pragma unroll
                for (int jj = 0; jj < M; jj++)
                    if (jj >= tid && jj < mi) ci = ci + cmul(Ws[tid * 5 + jj], y[jj]);
                cvec[tid] = ci;
            }
        }
        __syncthreads();
        maxit = flag[2];
#pragma unroll
        for (int i = 0; i < M; i++) {
            if (i >= maxit) break;
            const float2 ci = cvec[i];
            const float2 ex = p_bc(ci.x), ey = p_bc(ci.y), ney = p_bc(-ci.y);
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const SiteP v = site_ld(P + i * S, tid + TPB * k);
                x[k].re = p_fma(ex, v.re, x[k].re);
                x[k].re = p_fma(ney, v.im, x[k].re);
                x[k].im = p_fma(ex, v.im, x[k].im);
                x[k].im = p_fma(ey, v.re, x[k].im);
            }
        }
        // true residual; after the last cycle it only decides the returned count
        if (kk == restarts - 1 && !iters_out) break;
        store(stg, x);
        __syncthreads();
        apply(stg, w, mass);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const SiteP b = site_from_global(__ldg(&rb4[gsite(k)]));
            w[k].re = p_sub(b.re, w[k].re);
            w[k].im = p_sub(b.im, w[k].im);
        }
        err = sqrtf(norm2(w));
        if (err < tol * normb) {
            ret = kk * M + maxit;
            break;
        }
    }
    float4* xo = reinterpret_cast<float4*>(xg + off);
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int gk = gsite(k);
        float4 o = xo[gk];
        o.x += x[k].re.x;
        o.y += x[k].im.x;
        o.z += x[k].re.y;
        o.w += x[k].im.y;
        xo[gk] = o;
    }
    if (iters_out && tid == 0) iters_out[rhs * ncol + seg] = ret;
}

template <int SPT, int NW>
inline int sap0_ca_smem() {
    constexpr int S = 32 * NW * SPT;
    return 6 * S * 16 + (36 + 25 + 30 + 16) * 8 + 2 * NW * 6 * 8 + 5 * 8 + 3 * 4 + 16;
}

}  // namespace amgb
