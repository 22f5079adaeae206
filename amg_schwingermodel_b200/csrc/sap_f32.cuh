// FP32 SAP block solve on the fine level with paired (f32x2) arithmetic: the same solve as
// k_sap0_lean (src/sap.cpp:44-62, GMRES_D_B include/sap.h:27-47, FGMRES::fgmres
// src/fgmres.cpp:5-115 with x0 = b), restructured for sm_100's two-wide FP32 instructions.
//
// A site's two spin components travel together: in shared memory a basis vector is one
// float4 per site (spin0.re, spin1.re, spin0.im, spin1.im), so a site moves with one 16-byte
// access, and in registers a site is a pair of f32x2 values (re = (s0.re, s1.re), im =
// (s0.im, s1.im)).  Every Gram-Schmidt dot, axpy, norm and solution update then works on
// both spins with one paired instruction, and each basis vector is read from shared memory
// once per Gram-Schmidt step (kept in registers across the reduction between the dot and
// the axpy).  The block operator D_B is evaluated per site in scalar FP32 with the four
// neighbour indices and the four hop links (sign and 1/2 folded in, zero outside the block)
// set up once in registers, as in k_sap0_lean.
#pragma once
#include "common.cuh"
#include "sap_lean.cuh"
#include "stencil.cuh"

namespace amgb {

// ---- two-wide FP32 arithmetic (PTX add/sub/mul/fma .rn.f32x2, sm_100 and later) ----------
__device__ __forceinline__ float2 p_add(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 a, b, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; add.rn.f32x2 d, a, b; mov.b64 {%0, %1}, d;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 a, b, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; sub.rn.f32x2 d, a, b; mov.b64 {%0, %1}, d;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) {
    float2 r;
    asm("{.reg .b64 a, b, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; mul.rn.f32x2 d, a, b; mov.b64 {%0, %1}, d;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{.reg .b64 a, b, c, d; mov.b64 a, {%2, %3}; mov.b64 b, {%4, %5}; mov.b64 c, {%6, %7};"
        " fma.rn.f32x2 d, a, b, c; mov.b64 {%0, %1}, d;}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ float2 p_bc(float a) { return make_float2(a, a); }

// one site, both spins
struct SiteP {
    float2 re, im;
};
__device__ __forceinline__ SiteP site_ld(const float4* __restrict__ V, int m) {
    const float4 q = V[m];
    return {make_float2(q.x, q.y), make_float2(q.z, q.w)};
}
__device__ __forceinline__ void site_st(float4* __restrict__ V, int m, const SiteP& a) {
    V[m] = make_float4(a.re.x, a.re.y, a.im.x, a.im.y);
}
// a global [N][2] complex64 site (s0.re, s0.im, s1.re, s1.im) as a SiteP
__device__ __forceinline__ SiteP site_from_global(float4 g) { return {make_float2(g.x, g.z), make_float2(g.y, g.w)}; }

// CTA sums with paired adds: warp shuffles, one barrier, then every thread adds the NW warp
// partials (read two at a time) in warp order.  part holds two buffers of STR float2 each
// (STR >= NW, a multiple of 2) on a 16-byte boundary, so consecutive reductions need one
// barrier each.
template <int NW, int STR = NW>
__device__ __forceinline__ float2 psum2(float2 a, float2* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float2 b;
        b.x = __shfl_xor_sync(0xffffffffu, a.x, o);
        b.y = __shfl_xor_sync(0xffffffffu, a.y, o);
        a = p_add(a, b);
    }
    if (NW == 1) return a;
    float2* p = part + buf * STR;
    if ((threadIdx.x & 31) == 0) p[threadIdx.x >> 5] = a;
    __syncthreads();
    const float4* p4 = reinterpret_cast<const float4*>(p);
    float4 q = p4[0];
    float2 sum = p_add(make_float2(q.x, q.y), make_float2(q.z, q.w));
#pragma unroll
    for (int k = 1; k < NW / 2; k++) {
        q = p4[k];
        sum = p_add(sum, make_float2(q.x, q.y));
        sum = p_add(sum, make_float2(q.z, q.w));
    }
    buf ^= 1;
    return sum;
}
template <int NW, int STR = NW>
__device__ __forceinline__ float psum1(float a, float2* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (NW == 1) return a;
    float* p = reinterpret_cast<float*>(part + buf * STR);
    if ((threadIdx.x & 31) == 0) p[threadIdx.x >> 5] = a;
    __syncthreads();
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < NW; k++) sum += p[k];
    buf ^= 1;
    return sum;
}

// CTA sums of the first n of K complex values per thread (n is a constant once the caller's
// loops are unrolled), every thread receiving the same sums; one barrier for all n.  A buffer
// of part holds the values one after another, each as its NW warp partials ([K][NW] float2,
// read two warps at a time), and the two buffers are STR float2 apart as in psum2.  The xor
// butterfly adds the same pair in both lanes of every exchange, so with one warp every lane
// already holds the same sums.
template <int NW, int STR, int K>
__device__ __forceinline__ void psum_n(float2 (&v)[K], int n, float2* part, int& buf) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < K; q++) {
            if (q < n) {
                float2 b;
                b.x = __shfl_xor_sync(0xffffffffu, v[q].x, o);
                b.y = __shfl_xor_sync(0xffffffffu, v[q].y, o);
                v[q] = p_add(v[q], b);
            }
        }
    }
    if (NW == 1) return;
    float2* p = part + buf * STR;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int q = 0; q < K; q++)
            if (q < n) p[q * NW + (threadIdx.x >> 5)] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; q++) {
        if (q < n) {
            const float4* p4 = reinterpret_cast<const float4*>(p + q * NW);
            float4 t = p4[0];
            float2 sum = p_add(make_float2(t.x, t.y), make_float2(t.z, t.w));
#pragma unroll
            for (int k = 1; k < NW / 2; k++) {
                t = p4[k];
                sum = p_add(sum, make_float2(t.x, t.y));
                sum = p_add(sum, make_float2(t.z, t.w));
            }
            v[q] = sum;
        }
    }
    buf ^= 1;
}

// float2 stride between the two reduction buffers: the batched classical Gram-Schmidt
// reduction holds up to M + 2 values per warp, the modified form 2 (the last projection's dot
// and |w|^2)
template <int M, int NW, bool CGS>
constexpr int sap0_f32_pst() { return CGS ? NW * (M + 2) : NW * 2; }

template <int M, int SPT, int NW, bool CGS = false>
__global__ void __launch_bounds__(32 * NW, 2) k_sap0_f32(const Links<float> U, float2* __restrict__ r,
                                                          float2* __restrict__ xg, const int* __restrict__ blocks,
                                                          int ncol, int nx, int nt, int sbt, int sxe, int ste, float m0,
                                                          int restarts, float tol, const int* __restrict__ act,
                                                          int* __restrict__ iters_out, const float2* __restrict__ vsrc,
                                                          long long vstride) {
    constexpr int TPB = 32 * NW, S = TPB * SPT;
    constexpr int PST = sap0_f32_pst<M, NW, CGS>();
    extern __shared__ __align__(16) unsigned char smraw_f[];
    const int seg = blockIdx.x, rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    float4* V = reinterpret_cast<float4*>(smraw_f);             // [M+1][S]
    float2* H = reinterpret_cast<float2*>(V + (M + 1) * S);     // [M][M]
    float2* part = H + ((M * M + 1) & ~1);                      // [2][PST], 16-byte aligned
    float2* hcor = part + 2 * PST;                               // [M]: second-projection column
    int buf = 0;
    const int tid = threadIdx.x;
    const int block = blocks[seg];
    const int bxi = block / sbt, bti = block - bxi * sbt;
    const int x0 = bxi * sxe, t0 = bti * ste;
    const long long off = (long long)rhs * nx * nt * 2;
    const float mass = m0 + 2.0f;

    // Thread tid owns the SPT consecutive sites m = SPT*tid + k (k = 0..SPT-1) of one t row
    // (the dispatcher guarantees SPT | ste), and site m lives at shared index
    // sidx(m) = (m % SPT)*TPB + m / SPT, so a warp's accesses to "site k of every thread" are
    // contiguous.  A site's t neighbours are then the thread's own registers except at the
    // ends of its run, and only the x neighbours and those two come from shared memory.
    // Per-site set-up: the shared indices of those neighbours and the folded hop links.
    auto sidx = [&](int q) { return (q % SPT) * TPB + q / SPT; };
    int nbt[2];          // t-1 neighbour of site 0, t+1 neighbour of site SPT-1
    int nbx[SPT][2];     // x+1, x-1 neighbours
    float2 lk[SPT][4];
    int gs[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int m = SPT * tid + k;
        const int mx = m / ste, mt = m - mx * ste;
        const int t = t0 + mt, x = x0 + mx;
        gs[k] = x * nt + t;
        const float sR = (t == nt - 1) ? -0.5f : 0.5f;
        const float sL = (t == 0) ? -0.5f : 0.5f;
        int q = -1;
        if (mt + 1 < ste) q = m + 1; else if (ste == nt) q = mx * ste;
        if (k == SPT - 1) nbt[1] = sidx(q < 0 ? m : q);
        lk[k][0] = q < 0 ? czero<float>() : sR * U[2 * gs[k]];
        q = -1;
        if (mx + 1 < sxe) q = m + ste; else if (sxe == nx) q = mt;
        nbx[k][0] = sidx(q < 0 ? m : q);
        lk[k][1] = q < 0 ? czero<float>() : 0.5f * U[2 * gs[k] + 1];
        q = -1;
        if (mt > 0) q = m - 1; else if (ste == nt) q = mx * ste + ste - 1;
        if (k == 0) nbt[0] = sidx(q < 0 ? m : q);
        lk[k][2] = q < 0 ? czero<float>() : sL * cconj(U[2 * (x * nt + ((t == 0) ? nt - 1 : t - 1))]);
        q = -1;
        if (mx > 0) q = m - ste; else if (sxe == nx) q = (sxe - 1) * ste + mt;
        nbx[k][1] = sidx(q < 0 ? m : q);
        lk[k][3] = q < 0 ? czero<float>() : 0.5f * cconj(U[2 * (((x == 0) ? nx - 1 : x - 1) * nt + t) + 1]);
    }

    // w = D_B v for this thread's sites
    // (cw: the thread's own sites of v are also in w, so the t neighbours inside the run come
    // from registers; the sites are done in order and each keeps its old value for the next)
    auto apply = [&](const float4* __restrict__ v, SiteP (&w)[SPT], bool cw) {
        float4 prev = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int mi = tid + TPB * k;
            float4 c, a, e;
            if (cw) {
                c = make_float4(w[k].re.x, w[k].re.y, w[k].im.x, w[k].im.y);
                a = (k < SPT - 1) ? make_float4(w[k + 1].re.x, w[k + 1].re.y, w[k + 1].im.x, w[k + 1].im.y) : v[nbt[1]];
                e = (k > 0) ? prev : v[nbt[0]];
                prev = c;
            } else {
                c = v[mi];
                a = (k < SPT - 1) ? v[mi + TPB] : v[nbt[1]];
                e = (k > 0) ? v[mi - TPB] : v[nbt[0]];
            }
            const float4 b = v[nbx[k][0]], g = v[nbx[k][1]];
            const float2 ta = cmul(lk[k][0], make_float2(a.x - a.y, a.z - a.w));   // (1 - sigma_0) forward t
            const float2 tb = cmul(lk[k][1], make_float2(b.x - b.w, b.z + b.y));   // (1 - sigma_1) forward x
            const float2 tc = cmul(lk[k][2], make_float2(e.x + e.y, e.z + e.w));   // (1 + sigma_0) backward t
            const float2 td = cmul(lk[k][3], make_float2(g.x + g.w, g.z - g.y));   // (1 + sigma_1) backward x
            const float w0r = mass * c.x - (ta.x + tb.x + tc.x + td.x);
            const float w0i = mass * c.z - (ta.y + tb.y + tc.y + td.y);
            const float w1r = mass * c.y - tc.x + ta.x + td.y - tb.y;
            const float w1i = mass * c.w - tc.y + ta.y - td.x + tb.x;
            w[k].re = make_float2(w0r, w1r);
            w[k].im = make_float2(w0i, w1i);
        }
    };
    auto norm2 = [&](const SiteP (&a)[SPT]) -> float {
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            acc = p_fma(a[k].re, a[k].re, acc);
            acc = p_fma(a[k].im, a[k].im, acc);
        }
        return psum1<NW, PST>(acc.x + acc.y, part, buf);
    };
    auto store = [&](float4* Vd, const SiteP (&a)[SPT]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) site_st(Vd, tid + TPB * k, a[k]);
    };
    // this thread's parts of <V_i, w> for i <= j (d[i]) and of |w|^2 (d[j + 1].x)
    auto dots = [&](int j, const SiteP (&w)[SPT], float2 (&d)[M + 2]) {
        float2 nw = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            nw = p_fma(w[k].re, w[k].re, nw);
            nw = p_fma(w[k].im, w[k].im, nw);
        }
#pragma unroll
        for (int i = 0; i <= M; i++) {
            if (i <= j) {
                float2 ar = make_float2(0.f, 0.f), ai = ar, an = ar;
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const SiteP vi = site_ld(V + i * S, tid + TPB * k);
                    ar = p_fma(w[k].re, vi.re, ar);
                    ar = p_fma(w[k].im, vi.im, ar);
                    ai = p_fma(w[k].im, vi.re, ai);
                    an = p_fma(w[k].re, vi.im, an);
                }
                d[i] = make_float2(ar.x + ar.y, (ai.x + ai.y) - (an.x + an.y));
            }
        }
        d[j + 1] = make_float2(nw.x + nw.y, 0.f);
    };
    // w -= sum_{i <= j} h_i V_i
    auto project = [&](int j, const float2 (&h)[M + 2], SiteP (&w)[SPT]) {
#pragma unroll
        for (int i = 0; i <= M; i++) {
            if (i <= j) {
                const float2 nhx = p_bc(-h[i].x), hy = p_bc(h[i].y), nhy = p_bc(-h[i].y);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const SiteP vi = site_ld(V + i * S, tid + TPB * k);
                    w[k].re = p_fma(nhx, vi.re, w[k].re);
                    w[k].re = p_fma(hy, vi.im, w[k].re);
                    w[k].im = p_fma(nhx, vi.im, w[k].im);
                    w[k].im = p_fma(nhy, vi.re, w[k].im);
                }
            }
        }
    };

    float4* rb4 = reinterpret_cast<float4*>(r + off);
    // The iterate x lives in basis slot M, which the Arnoldi process never needs (the update
    // uses V_0..V_{M-1} and each cycle restarts from the true residual), so it holds no
    // registers during the Arnoldi steps and the residual's operator reads it in place.
    float4* X = V + M * S;
    SiteP w[SPT];
    float normb;
    {
        // r = b - A x0 (x0 = b)
        SiteP b[SPT];
        if (vsrc) {
            // fused SAP residual (src/sap.cpp:64-174 recomputes r = v - D x after every colour):
            // b = v - D x on this block's sites, from the global iterate, whose halo belongs to
            // blocks of the other colour that this launch does not write; b is kept in r for
            // the restart residuals
            const float2* xr = xg + off;
            const float2* vr = vsrc + (long long)rhs * vstride;
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                const SiteOp<float> L = site_op<float>(U, gs[k], nx, nt);
                float2 o0, o1;
                dirac_site<float, false>(L, xr, gs[k], mass, o0, o1);
                const float2 v0 = vr[2 * gs[k]], v1 = vr[2 * gs[k] + 1];
                const float4 q = make_float4(v0.x - o0.x, v0.y - o0.y, v1.x - o1.x, v1.y - o1.y);
                rb4[gs[k]] = q;
                b[k] = site_from_global(q);
            }
        } else {
#pragma unroll
            for (int k = 0; k < SPT; k++) b[k] = site_from_global(rb4[gs[k]]);
        }
        store(X, b);
        normb = sqrtf(norm2(b));
        lean_sync<float, NW>();
        apply(X, w, false);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            w[k].re = p_sub(b[k].re, w[k].re);
            w[k].im = p_sub(b[k].im, w[k].im);
        }
    }
    float err2 = norm2(w), rerr = rsqrtf(err2), err = err2 * rerr;
    const float tolb2 = (tol * normb) * (tol * normb);   // the exit test on |g_{j+1}|^2
    int maxit = M;
    int ret = restarts * M;
    for (int kk = 0; kk < restarts; kk++) {
        {
            const float2 inv = p_bc(rerr);
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                w[k].re = p_mul(inv, w[k].re);
                w[k].im = p_mul(inv, w[k].im);
            }
            store(V, w);
        }
        // The Givens rotations run redundantly in every thread (the Hessenberg column is the
        // same in all threads after the reductions), so an Arnoldi step needs one barrier,
        // before the next operator application reads V_{j+1}; only H goes to shared memory.
        float2 g[M + 1], cs[M], sns[M];
        g[0] = make_float2(err, 0.f);
        lean_sync<float, NW>();
#pragma unroll
        for (int j = 0; j < M; j++) {
            apply(V + j * S, w, true);   // w holds V_j
            float2 col[M + 1];
            float hn2;
            if constexpr (CGS) {
                // classical Gram-Schmidt: the j + 1 dots and |w|^2 in one reduction and the
                // norm of the projected w by Pythagoras, so one barrier per step instead of
                // j + 2; the same Hessenberg column as the modified form in exact
                // arithmetic.  When the projection cancels below 1/8 of |w| (the
                // re-orthogonalisation test of Daniel, Gragg, Kaufman and Stewart, Math.
                // Comp. 30 (1976), with eta = 1/8) w is projected once more and its norm
                // taken directly, which keeps the Pythagorean norm accurate to ~64 ulp and
                // bounds the loss of orthogonality per step by 8x.  On 32x32 Wilson blocks
                // the ratio stays near 0.6 (min 0.45), so the second projection is the rare
                // path; it goes one basis vector at a time, which needs fewer registers than
                // a second batched pass.
                float2 d[M + 2];
                dots(j, w, d);
                psum_n<NW, PST>(d, j + 2, part, buf);
                float hs = 0.f;
#pragma unroll
                for (int i = 0; i <= j; i++) {
                    col[i] = d[i];
                    hs += cnorm2(d[i]);
                }
                const float ww = d[j + 1].x;
                hn2 = ww - hs;
                project(j, d, w);
                if (hn2 < ww * (1.0f / 64.0f)) {
                    // second projection, one basis vector at a time in a loop that is not
                    // unrolled (the rare path stays small); thread 0 passes the corrections
                    // to the column through shared memory, ordered by the norm's barrier
#pragma unroll 1
                    for (int i = 0; i <= j; i++) {
                        const float4* Vi = V + i * S;
                        float2 ar = make_float2(0.f, 0.f), ai = ar, an = ar;
#pragma unroll
                        for (int k = 0; k < SPT; k++) {
                            const SiteP vi = site_ld(Vi, tid + TPB * k);
                            ar = p_fma(w[k].re, vi.re, ar);
                            ar = p_fma(w[k].im, vi.im, ar);
                            ai = p_fma(w[k].im, vi.re, ai);
                            an = p_fma(w[k].re, vi.im, an);
                        }
                        const float2 h = psum2<NW, PST>(make_float2(ar.x + ar.y, (ai.x + ai.y) - (an.x + an.y)), part, buf);
                        if (tid == 0) hcor[i] = h;
                        const float2 nhx = p_bc(-h.x), hy = p_bc(h.y), nhy = p_bc(-h.y);
#pragma unroll
                        for (int k = 0; k < SPT; k++) {
                            const SiteP vi = site_ld(Vi, tid + TPB * k);
                            w[k].re = p_fma(nhx, vi.re, w[k].re);
                            w[k].re = p_fma(hy, vi.im, w[k].re);
                            w[k].im = p_fma(nhx, vi.im, w[k].im);
                            w[k].im = p_fma(nhy, vi.re, w[k].im);
                        }
                    }
                    hn2 = norm2(w);
                    if (NW == 1) __syncwarp();
#pragma unroll
                    for (int i = 0; i <= j; i++) col[i] = col[i] + hcor[i];
                }
                hn2 = fmaxf(hn2, 0.f);
            } else {
                // modified Gram-Schmidt (src/fgmres.cpp:24-32), V_i read once per step.  The
                // last projection's reduction also carries |w|^2, and |w - h_j V_j|^2 =
                // |w|^2 - |h_j|^2 (w is already orthogonal to V_0..V_{j-1}) saves the norm's
                // own reduction; when it cancels below 1/8 of |w| the norm is taken directly.
                float ww = 0.f;
#pragma unroll
                for (int i = 0; i <= j; i++) {
                    SiteP vi[SPT];
                    float2 ar = make_float2(0.f, 0.f), ai = ar, an = ar, nw = ar;
#pragma unroll
                    for (int k = 0; k < SPT; k++) {
                        vi[k] = site_ld(V + i * S, tid + TPB * k);
                        ar = p_fma(w[k].re, vi[k].re, ar);
                        ar = p_fma(w[k].im, vi[k].im, ar);
                        ai = p_fma(w[k].im, vi[k].re, ai);
                        an = p_fma(w[k].re, vi[k].im, an);
                        if (i == j) {
                            nw = p_fma(w[k].re, w[k].re, nw);
                            nw = p_fma(w[k].im, w[k].im, nw);
                        }
                    }
                    float2 h;
                    if (i == j) {
                        float2 d[2] = {make_float2(ar.x + ar.y, (ai.x + ai.y) - (an.x + an.y)),
                                       make_float2(nw.x + nw.y, 0.f)};
                        psum_n<NW, PST>(d, 2, part, buf);
                        h = d[0];
                        ww = d[1].x;
                    } else {
                        h = psum2<NW, PST>(make_float2(ar.x + ar.y, (ai.x + ai.y) - (an.x + an.y)), part, buf);
                    }
                    col[i] = h;
                    const float2 nhx = p_bc(-h.x), hy = p_bc(h.y), nhy = p_bc(-h.y);
#pragma unroll
                    for (int k = 0; k < SPT; k++) {
                        w[k].re = p_fma(nhx, vi[k].re, w[k].re);
                        w[k].re = p_fma(hy, vi[k].im, w[k].re);
                        w[k].im = p_fma(nhx, vi[k].im, w[k].im);
                        w[k].im = p_fma(nhy, vi[k].re, w[k].im);
                    }
                }
                hn2 = ww - cnorm2(col[j]);
                if (hn2 < ww * (1.0f / 64.0f)) hn2 = norm2(w);
            }
            // 1/|w| and |w| from one reciprocal square root
            const float rhn = rsqrtf(hn2);
            const float hn = hn2 > 0.f ? hn2 * rhn : 0.f;
            if (j + 1 < M && hn2 > 0.f) {
                const float2 inv = p_bc(rhn);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    w[k].re = p_mul(inv, w[k].re);
                    w[k].im = p_mul(inv, w[k].im);
                }
                store(V + (j + 1) * S, w);
            }
            // rotation(j) (src/fgmres.cpp:90-104)
            col[j + 1] = make_float2(hn, 0.f);
#pragma unroll
            for (int i = 0; i < j; i++) {
                const float2 temp = cmulc(cs[i], col[i]) + cmulc(sns[i], col[i + 1]);
                col[i + 1] = cmul(cs[i], col[i + 1]) - cmul(sns[i], col[i]);
                col[i] = temp;
            }
            const float rden = rsqrtf(cnorm2(col[j]) + cnorm2(col[j + 1]));
            sns[j] = make_float2(col[j + 1].x * rden, col[j + 1].y * rden);
            cs[j] = make_float2(col[j].x * rden, col[j].y * rden);
            col[j] = cmulc(cs[j], col[j]) + cmulc(sns[j], col[j + 1]);
            if (tid == 0) {
#pragma unroll
                for (int i = 0; i <= j; i++) H[i * M + j] = col[i];
            }
            g[j + 1] = -cmul(sns[j], g[j]);
            g[j] = cmulc(cs[j], g[j]);
            lean_sync<float, NW>();
            if (cnorm2(g[j + 1]) < tolb2) {
                maxit = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115) and x += sum eta_j V_j
        float2 eta[M];
#pragma unroll
        for (int i = M - 1; i >= 0; i--) {
            if (i >= maxit) { eta[i] = czero<float>(); continue; }
            float2 o = g[i];
#pragma unroll
            for (int jj = i + 1; jj < M; jj++)
                if (jj < maxit) o = o - cmul(H[i * M + jj], eta[jj]);
            eta[i] = cdiv(o, H[i * M + i]);
        }
        {
            SiteP x[SPT];
#pragma unroll
            for (int k = 0; k < SPT; k++) x[k] = site_ld(X, tid + TPB * k);
#pragma unroll
            for (int jj = 0; jj < M; jj++) {
                if (jj >= maxit) break;
                const float2 ex = p_bc(eta[jj].x), ey = p_bc(eta[jj].y), ney = p_bc(-eta[jj].y);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const SiteP v = site_ld(V + jj * S, tid + TPB * k);
                    x[k].re = p_fma(ex, v.re, x[k].re);
                    x[k].re = p_fma(ney, v.im, x[k].re);
                    x[k].im = p_fma(ex, v.im, x[k].im);
                    x[k].im = p_fma(ey, v.re, x[k].im);
                }
            }
            store(X, x);
        }
        // true residual r = b - A x.  After the last cycle it only decides the returned
        // iteration count, so it is skipped when nobody reads that.
        if (kk == restarts - 1 && !iters_out) break;
        lean_sync<float, NW>();
        apply(X, w, false);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const SiteP b = site_from_global(rb4[gs[k]]);
            w[k].re = p_sub(b.re, w[k].re);
            w[k].im = p_sub(b.im, w[k].im);
        }
        err2 = norm2(w);
        rerr = rsqrtf(err2);
        err = err2 * rerr;
        if (err2 < tolb2) {
            ret = kk * M + maxit;
            break;
        }
        lean_sync<float, NW>();
    }
    float4* xo = reinterpret_cast<float4*>(xg + off);
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const SiteP xk = site_ld(X, tid + TPB * k);
        float4 o = xo[gs[k]];
        o.x += xk.re.x;
        o.y += xk.im.x;
        o.z += xk.re.y;
        o.w += xk.im.y;
        xo[gs[k]] = o;
    }
    if (iters_out && tid == 0) iters_out[rhs * ncol + seg] = ret;
}

template <int M, int SPT, int NW, bool CGS = false>
inline int sap0_f32_smem() {
    constexpr int S = 32 * NW * SPT;
    // V [M+1][S] float4, H [M][M] float2 (even count), part [2][PST] float2, hcor [M] float2
    return (M + 1) * S * 16 + ((M * M + 1) & ~1) * 8 + 2 * sap0_f32_pst<M, NW, CGS>() * 8 + M * 8 + 16;
}

}  // namespace amgb
