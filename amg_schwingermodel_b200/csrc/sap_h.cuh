// FP32 SAP block solve with its Krylov basis stored in 16 bits (FP16, or BF16 with BF = true):
// the solve of k_sap0_f32 (MGS form; src/sap.cpp:44-62, GMRES_D_B include/sap.h:27-47,
// FGMRES::fgmres src/fgmres.cpp:5-115 with x0 = b) laid out for three CTAs per SM instead
// of two.  The block body (sap0_h_solve) serves one launch per lattice (k_sap0_h) and one
// launch over several lattices' blocks (k_sap0_h_group, the many-configuration solve).
//
// What sets the SM's share: the paired kernel holds its basis (M + 1 vectors of 16 bytes per
// site, 98 KB for a 1024-site block) in shared memory and its folded links, neighbour
// indices and Givens rotations in registers (128 per thread), so two CTAs of 8 warps fill an
// SM.  Here
//   * the M basis vectors are 16-bit pairs (8 bytes per site, 40 KB); the iterate stays FP32
//     in its own array (16 KB), and so do every dot, axpy, norm and the solution update;
//   * the folded hop links (sign, 1/2 and the zero outside the block applied; FP16 storage of
//     the fine links) are staged once per CTA in shared memory (16 KB) instead of registers;
//   * a thread's neighbour indices reduce to four offsets (its run of SPT sites lies in one
//     t row), and the Givens rotations, g, the exit decision and the least-squares solution
//     live in shared memory: thread 0 computes them while the other threads wait at the
//     barrier the step takes anyway (the paired kernel repeats them in every thread);
// which fits 80 registers and 73 KB, three CTAs (24 warps) per SM.
//
// Every basis vector is rounded to 16 bits when it is stored and the thread's registers are
// rounded the same way, so the operator, the Gram-Schmidt dots and the projections all see
// the stored vectors; the Arnoldi relation then holds to the rounding of V_{j+1} (relative
// 2^-11 in FP16, 2^-8 in BF16), while the true residual of every restart cycle is formed in
// FP32 from the FP32 iterate.
#pragma once
#include "common.cuh"
#include "sap_f32.cuh"

namespace amgb {

// a 16-bit basis site: (s0.re, s1.re) and (s0.im, s1.im) as two 16-bit pairs in a uint2,
// FP16 (BF = false) or BF16 (BF = true).  FP16 keeps 11 significant bits; its conversions to
// FP32 run on the FMA pipe.  BF16 keeps 8; its conversions are a shift and a mask on the
// integer pipe.
template <bool BF>
__device__ __forceinline__ float2 p16_to_f2(unsigned u) {
    if constexpr (BF) {
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    } else {
        __half2 a;
        memcpy(&a, &u, 4);
        return __half22float2(a);
    }
}
template <bool BF>
__device__ __forceinline__ unsigned f2_to_p16(float2 v) {
    unsigned u;
    if constexpr (BF) {
        const __nv_bfloat162 a = __float22bfloat162_rn(v);
        memcpy(&u, &a, 4);
    } else {
        const __half2 a = __float22half2_rn(v);
        memcpy(&u, &a, 4);
    }
    return u;
}
template <bool BF>
__device__ __forceinline__ SiteP h_unpack(uint2 q) {
    return {p16_to_f2<BF>(q.x), p16_to_f2<BF>(q.y)};
}
template <bool BF>
__device__ __forceinline__ uint2 h_pack(const SiteP& s) {
    return make_uint2(f2_to_p16<BF>(s.re), f2_to_p16<BF>(s.im));
}
__device__ __forceinline__ float2 h2f(unsigned u) {
    __half2 a;
    memcpy(&a, &u, 4);
    return __half22float2(a);
}
__device__ __forceinline__ unsigned f2h(float2 v) {
    const __half2 a = __float22half2_rn(v);
    unsigned u;
    memcpy(&u, &a, 4);
    return u;
}

template <int M, int SPT, int NW>
__host__ __device__ constexpr int sap0_h_smem() {
    // X [S] float4, LK [S] uint4, V [M][S] uint2, H [M][M] float2 (even count), part [2][2 NW]
    // float2, Givens cs [M], sn [M], g [M + 1], eta [M] float2, the exit flag
    return 32 * NW * SPT * (16 + 16 + 8 * M) + ((M * M + 1) & ~1) * 8 + 2 * 2 * NW * 8 + (4 * M + 1) * 8 + 16;
}

// the block solve of block blocks[seg] for source rhs (called by every thread of the CTA)
template <int M, int SPT, int NW, bool BF>
__device__ __forceinline__ void sap0_h_solve(const __half2* __restrict__ U, float2* __restrict__ r,
                                             float2* __restrict__ xg, const int* __restrict__ blocks, int ncol,
                                             int nx, int nt, int sbt, int sxe, int ste, float m0, int restarts,
                                             float tol, int* __restrict__ iters_out, int seg, int rhs) {
    constexpr int TPB = 32 * NW, S = TPB * SPT, PST = 2 * NW;
    extern __shared__ __align__(16) unsigned char smraw_h[];
    float4* X = reinterpret_cast<float4*>(smraw_h);   // [S] iterate (FP32)
    uint4* LK = reinterpret_cast<uint4*>(X + S);      // [S] folded hop links (FP16)
    uint2* V = reinterpret_cast<uint2*>(LK + S);      // [M][S] basis (FP16)
    float2* H = reinterpret_cast<float2*>(V + M * S); // [M][M]
    float2* part = H + ((M * M + 1) & ~1);            // [2][PST], 16-byte aligned
    float2* cs_s = part + 2 * PST;                    // [M]
    float2* sn_s = cs_s + M;                          // [M]
    float2* g_s = sn_s + M;                           // [M + 1]
    float2* eta_s = g_s + M + 1;                      // [M]
    int* exit_s = reinterpret_cast<int*>(eta_s + M);  // the step's exit decision
    int buf = 0;
    const int tid = threadIdx.x;
    const int block = blocks[seg];
    const int bxi = block / sbt, bti = block - bxi * sbt;
    const long long off = (long long)rhs * nx * nt * 2;
    const float mass = m0 + 2.0f;

    // Thread tid owns the SPT consecutive sites m = SPT*tid + k of one t row (SPT | ste), site
    // m at shared index (m % SPT)*TPB + m / SPT = tid + TPB*k, so its x neighbours are at
    // tid + TPB*k + dxp and + dxm for all k, and only the ends of the run have t neighbours
    // outside its registers.  A hop leaving the block points at the site itself with a zero
    // link.
    const int m0s = SPT * tid, mx = m0s / ste, mt0 = m0s - mx * ste;
    const int x = bxi * sxe + mx, t0 = bti * ste + mt0;
    const int gs0 = x * nt + t0;                      // global site of k = 0; site k is gs0 + k
    int dxp = 0, dxm = 0, nbt0, nbt1;
    bool inx_p = true, inx_m = true;
    if (mx + 1 < sxe) dxp = ste / SPT;
    else if (sxe == nx) dxp = -(sxe - 1) * (ste / SPT);
    else inx_p = false;
    if (mx > 0) dxm = -(ste / SPT);
    else if (sxe == nx) dxm = (sxe - 1) * (ste / SPT);
    else inx_m = false;
    bool int_p = true, int_m = true;
    {
        // t+1 of site SPT-1 and t-1 of site 0
        const int mlast = m0s + SPT - 1, mtl = mt0 + SPT - 1;
        int q = -1;
        if (mtl + 1 < ste) q = mlast + 1; else if (ste == nt) q = mx * ste;
        int_p = q >= 0;
        const int qq = q < 0 ? mlast : q;
        nbt1 = (qq % SPT) * TPB + qq / SPT;
        q = -1;
        if (mt0 > 0) q = m0s - 1; else if (ste == nt) q = mx * ste + ste - 1;
        int_m = q >= 0;
        const int qm = q < 0 ? m0s : q;
        nbt0 = (qm % SPT) * TPB + qm / SPT;
    }
    // stage the folded links: hop order t+, x+, t-, x- (as k_sap0_f32)
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const int t = t0 + k, gs = gs0 + k;
        const bool tp = (k < SPT - 1) || int_p, tm = (k > 0) || int_m;
        const float sR = (t == nt - 1) ? -0.5f : 0.5f;
        const float sL = (t == 0) ? -0.5f : 0.5f;
        const float2 z = make_float2(0.f, 0.f);
        const float2 l0 = tp ? sR * __half22float2(U[2 * gs]) : z;
        const float2 l1 = inx_p ? 0.5f * __half22float2(U[2 * gs + 1]) : z;
        const float2 l2 = tm ? sL * cconj(__half22float2(U[2 * (x * nt + ((t == 0) ? nt - 1 : t - 1))])) : z;
        const float2 l3 = inx_m ? 0.5f * cconj(__half22float2(U[2 * (((x == 0) ? nx - 1 : x - 1) * nt + t) + 1])) : z;
        LK[tid + TPB * k] = make_uint4(f2h(l0), f2h(l1), f2h(l2), f2h(l3));
    }

    // one site of D_B: out from its centre c, t neighbours a (t+1) and e (t-1), x neighbours
    // b (x+1) and g (x-1), and the site's folded links
    auto site_op = [&](int mi, const SiteP& c, const SiteP& a, const SiteP& e, const SiteP& b, const SiteP& g) {
        const uint4 lq = LK[mi];
        const float2 ta = cmul(h2f(lq.x), make_float2(a.re.x - a.re.y, a.im.x - a.im.y));   // (1 - sigma_0) forward t
        const float2 tb = cmul(h2f(lq.y), make_float2(b.re.x - b.im.y, b.im.x + b.re.y));   // (1 - sigma_1) forward x
        const float2 tc = cmul(h2f(lq.z), make_float2(e.re.x + e.re.y, e.im.x + e.im.y));   // (1 + sigma_0) backward t
        const float2 td = cmul(h2f(lq.w), make_float2(g.re.x + g.im.y, g.im.x - g.re.y));   // (1 + sigma_1) backward x
        const float w0r = mass * c.re.x - (ta.x + tb.x + tc.x + td.x);
        const float w0i = mass * c.im.x - (ta.y + tb.y + tc.y + td.y);
        const float w1r = mass * c.re.y - tc.x + ta.x + td.y - tb.y;
        const float w1i = mass * c.im.y - tc.y + ta.y - td.x + tb.x;
        return SiteP{make_float2(w0r, w1r), make_float2(w0i, w1i)};
    };
    // w = D_B v for a basis vector v whose own sites are already in w (rounded as stored)
    auto apply_v = [&](const uint2* __restrict__ v, SiteP (&w)[SPT]) {
        SiteP prev = w[0];
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int mi = tid + TPB * k;
            const SiteP c = w[k];
            const SiteP a = (k < SPT - 1) ? w[k + 1] : h_unpack<BF>(v[nbt1]);
            const SiteP e = (k > 0) ? prev : h_unpack<BF>(v[nbt0]);
            prev = c;
            w[k] = site_op(mi, c, a, e, h_unpack<BF>(v[mi + dxp]), h_unpack<BF>(v[mi + dxm]));
        }
    };
    // w = D_B X
    auto apply_x = [&](SiteP (&w)[SPT]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const int mi = tid + TPB * k;
            const SiteP c = site_ld(X, mi);
            const SiteP a = site_ld(X, (k < SPT - 1) ? mi + TPB : nbt1);
            const SiteP e = site_ld(X, (k > 0) ? mi - TPB : nbt0);
            w[k] = site_op(mi, c, a, e, site_ld(X, mi + dxp), site_ld(X, mi + dxm));
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
    // store w as basis vector d and round w to the stored values
    auto store_v = [&](uint2* d, SiteP (&w)[SPT]) {
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const uint2 q = h_pack<BF>(w[k]);
            d[tid + TPB * k] = q;
            w[k] = h_unpack<BF>(q);
        }
    };

    const float4* rb4 = reinterpret_cast<const float4*>(r + off);
    SiteP w[SPT];
    float normb;
    lean_sync<float, NW>();   // LK complete
    {
        // r = b - A x0 (x0 = b)
#pragma unroll
        for (int k = 0; k < SPT; k++) w[k] = site_from_global(rb4[gs0 + k]);
#pragma unroll
        for (int k = 0; k < SPT; k++) site_st(X, tid + TPB * k, w[k]);
        normb = sqrtf(norm2(w));
        lean_sync<float, NW>();
        SiteP d[SPT];
        apply_x(d);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            w[k].re = p_sub(w[k].re, d[k].re);
            w[k].im = p_sub(w[k].im, d[k].im);
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
            store_v(V, w);
        }
        if (tid == 0) g_s[0] = make_float2(err, 0.f);
        lean_sync<float, NW>();
#pragma unroll
        for (int j = 0; j < M; j++) {
            apply_v(V + j * S, w);   // w held V_j
            float2 col[M + 1];
            // modified Gram-Schmidt (src/fgmres.cpp:24-32); the last projection's reduction
            // also carries |w|^2, and |w - h_j V_j|^2 = |w|^2 - |h_j|^2 saves the norm's own
            // reduction unless it cancels below 1/8 of |w|
            float ww = 0.f;
#pragma unroll
            for (int i = 0; i <= M; i++) {
                if (i <= j) {
                    SiteP vi[SPT];
                    float2 ar = make_float2(0.f, 0.f), ai = ar, an = ar, nw = ar;
#pragma unroll
                    for (int k = 0; k < SPT; k++) {
                        vi[k] = h_unpack<BF>(V[i * S + tid + TPB * k]);
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
            }
            float hn2 = ww - cnorm2(col[j]);
            if (hn2 < ww * (1.0f / 64.0f)) hn2 = norm2(w);
            const float rhn = rsqrtf(hn2);
            const float hn = hn2 > 0.f ? hn2 * rhn : 0.f;
            if (j + 1 < M && hn2 > 0.f) {
                const float2 inv = p_bc(rhn);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    w[k].re = p_mul(inv, w[k].re);
                    w[k].im = p_mul(inv, w[k].im);
                }
                store_v(V + (j + 1) * S, w);
            }
            // rotation(j) (src/fgmres.cpp:90-104) and the exit test, by thread 0; the step's
            // barrier publishes them (the column is the same in every thread after the
            // reductions, so thread 0's copy is the one the others would have computed)
            if (tid == 0) {
                col[j + 1] = make_float2(hn, 0.f);
#pragma unroll
                for (int i = 0; i < j; i++) {
                    const float2 ci = cs_s[i], si = sn_s[i];
                    const float2 temp = cmulc(ci, col[i]) + cmulc(si, col[i + 1]);
                    col[i + 1] = cmul(ci, col[i + 1]) - cmul(si, col[i]);
                    col[i] = temp;
                }
                const float rden = rsqrtf(cnorm2(col[j]) + cnorm2(col[j + 1]));
                const float2 snj = make_float2(col[j + 1].x * rden, col[j + 1].y * rden);
                const float2 csj = make_float2(col[j].x * rden, col[j].y * rden);
                col[j] = cmulc(csj, col[j]) + cmulc(snj, col[j + 1]);
                const float2 gj = g_s[j];
                const float2 gj1 = -cmul(snj, gj);
#pragma unroll
                for (int i = 0; i <= j; i++) H[i * M + j] = col[i];
                cs_s[j] = csj;
                sn_s[j] = snj;
                g_s[j] = cmulc(csj, gj);
                g_s[j + 1] = gj1;
                *exit_s = cnorm2(gj1) < tolb2;
            }
            lean_sync<float, NW>();
            if (*exit_s) {
                maxit = j + 1;
                break;
            }
        }
        // solve_upper_triangular (src/fgmres.cpp:107-115) by thread 0, then x += sum eta_j V_j
        if (tid == 0) {
            float2 eta[M];
#pragma unroll
            for (int i = M - 1; i >= 0; i--) {
                if (i >= maxit) { eta[i] = czero<float>(); continue; }
                float2 o = g_s[i];
#pragma unroll
                for (int jj = i + 1; jj < M; jj++)
                    if (jj < maxit) o = o - cmul(H[i * M + jj], eta[jj]);
                eta[i] = cdiv(o, H[i * M + i]);
            }
#pragma unroll
            for (int i = 0; i < M; i++) eta_s[i] = eta[i];
        }
        lean_sync<float, NW>();
        {
            SiteP xs[SPT];
#pragma unroll
            for (int k = 0; k < SPT; k++) xs[k] = site_ld(X, tid + TPB * k);
#pragma unroll
            for (int jj = 0; jj < M; jj++) {
                if (jj >= maxit) break;
                const float2 ej = eta_s[jj];
                const float2 ex = p_bc(ej.x), ey = p_bc(ej.y), ney = p_bc(-ej.y);
#pragma unroll
                for (int k = 0; k < SPT; k++) {
                    const SiteP v = h_unpack<BF>(V[jj * S + tid + TPB * k]);
                    xs[k].re = p_fma(ex, v.re, xs[k].re);
                    xs[k].re = p_fma(ney, v.im, xs[k].re);
                    xs[k].im = p_fma(ex, v.im, xs[k].im);
                    xs[k].im = p_fma(ey, v.re, xs[k].im);
                }
            }
#pragma unroll
            for (int k = 0; k < SPT; k++) site_st(X, tid + TPB * k, xs[k]);
        }
        // true residual r = b - A x; after the last cycle it only decides the returned
        // iteration count, so it is skipped when nobody reads that
        if (kk == restarts - 1 && !iters_out) break;
        lean_sync<float, NW>();
        apply_x(w);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
            const SiteP b = site_from_global(rb4[gs0 + k]);
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
        float4 o = xo[gs0 + k];
        o.x += xk.re.x;
        o.y += xk.im.x;
        o.z += xk.re.y;
        o.w += xk.im.y;
        xo[gs0 + k] = o;
    }
    if (iters_out && tid == 0) iters_out[rhs * ncol + seg] = ret;
}

// one launch per colour and lattice: CTA (seg, rhs)
template <int M, int SPT, int NW, bool BF = false>
__global__ void __launch_bounds__(32 * NW, 3) k_sap0_h(const __half2* __restrict__ U, float2* __restrict__ r,
                                                        float2* __restrict__ xg, const int* __restrict__ blocks,
                                                        int ncol, int nx, int nt, int sbt, int sxe, int ste, float m0,
                                                        int restarts, float tol, const int* __restrict__ act,
                                                        int* __restrict__ iters_out) {
    const int seg = blockIdx.x, rhs = blockIdx.y;
    if (act && !act[rhs]) return;
    sap0_h_solve<M, SPT, NW, BF>(U, r, xg, blocks, ncol, nx, nt, sbt, sxe, ste, m0, restarts, tol, iters_out, seg,
                                 rhs);
}

// one launch per colour over several lattices (the many-configuration solve): column c of
// the grid is block col_seg[c] of task col_task[c]; rows beyond a task's sources and
// inactive sources return at once
template <int M, int SPT, int NW, bool BF = false>
__global__ void __launch_bounds__(32 * NW, 3) k_sap0_h_group(const SapTask* __restrict__ tasks,
                                                              const int* __restrict__ col_task,
                                                              const int* __restrict__ col_seg) {
    const SapTask& k = tasks[col_task[blockIdx.x]];
    const int rhs = blockIdx.y;
    if (rhs >= k.nrhs || (k.act && !k.act[rhs])) return;
    sap0_h_solve<M, SPT, NW, BF>(static_cast<const __half2*>(k.U), k.r, k.x, k.blocks, k.ncol, k.nx, k.nt, k.sbt,
                                 k.sxe, k.ste, k.m0, k.restarts, k.tol, nullptr, col_seg[blockIdx.x], rhs);
}

}  // namespace amgb
