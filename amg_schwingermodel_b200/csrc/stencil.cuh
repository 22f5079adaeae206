// The U(1) Wilson-Dirac stencil of one fine-lattice site, shared by the stencil kernels and
// by the SAP kernel's fused residual.
//
// Layout: psi[n][spin] complex (double2 or float2), n = x*Nt + t; U[n][mu].
#pragma once
#include <type_traits>

#include "common.cuh"

namespace amgb {

// ---------------------------------------------------------------------------------
// D_phi / D_dagger_phi (src/dirac_operator.cpp:3-54) for one site.  With forward
// neighbours (a,b) = psi(n+t), (c,d) = psi(n+x) and backward (e,f) = psi(n-t),
// (g,h) = psi(n-x):
//   D:   t0 = sR U0 (a-b), t1 = U1 (c+id), t2 = sL U0*(n-t) (e+f), t3 = U1*(n-x) (g-ih)
//        out0 = (m0+2) p0 - (t0+t1+t2+t3)/2,  out1 = (m0+2) p1 - (-t0 - i t1 + t2 + i t3)/2
//   D^+: the (1 -/+ sigma) projectors swap between forward and backward hops.
// ---------------------------------------------------------------------------------
// The geometry and links of one site, loaded once and reused for every source.
template <typename T>
struct SiteOp {
    int r0, r1, l0, l1;        // neighbours n+t, n+x, n-t, n-x
    cx<T> u0, u1, ul0, ul1;    // U_0(n), U_1(n), conj(U_0(n-t)), conj(U_1(n-x))
    T sR, sL;                  // antiperiodic signs of the two time hops
};

template <typename T, typename UA>
__device__ __forceinline__ SiteOp<T> site_op(const UA& U, int n, int nx, int nt) {
    SiteOp<T> o;
    const int x = n / nt, t = n - x * nt;
    o.r0 = x * nt + ((t + 1 == nt) ? 0 : t + 1);
    o.r1 = ((x + 1 == nx) ? 0 : x + 1) * nt + t;
    o.l0 = x * nt + ((t == 0) ? nt - 1 : t - 1);
    o.l1 = ((x == 0) ? nx - 1 : x - 1) * nt + t;
    o.u0 = U[2 * n];
    o.u1 = U[2 * n + 1];
    o.ul0 = cconj(U[2 * o.l0]);
    o.ul1 = cconj(U[2 * o.l1 + 1]);
    o.sR = (t == nt - 1) ? T(-1) : T(1);
    o.sL = (t == 0) ? T(-1) : T(1);
    return o;
}

// psi may be stored in a narrower type TP (FP32 spinors into the FP64 operator): its values
// are promoted exactly, so the result equals the T-precision operator on the promoted field.
template <typename T, typename TP>
__device__ __forceinline__ cx<T> promote_cx(const cx<TP>& v) {
    if constexpr (std::is_same<T, TP>::value) return v;
    else return ccast<T>(v);
}
// Both spin components of site n.  TILE: psi is a shared-memory tile read by consecutive lanes
// at consecutive sites.  A FP32 site (16 bytes) is then one 16-byte load.  A FP64 site is two
// 16-byte halves 32 bytes apart from lane to lane, so eight lanes reading the same half would
// hit every bank twice; lanes 4-7 of each eight read the second half first, which puts the
// eight addresses of each load in distinct banks.
template <typename T, typename TP, bool TILE>
__device__ __forceinline__ void site_spins(const cx<TP>* __restrict__ psi, int n, cx<T>& s0, cx<T>& s1) {
    if constexpr (TILE && sizeof(TP) == 4) {
        const float4 q = reinterpret_cast<const float4*>(psi)[n];
        s0 = promote_cx<T, TP>(make_float2(q.x, q.y));
        s1 = promote_cx<T, TP>(make_float2(q.z, q.w));
    } else if constexpr (TILE) {
        const int sw = (threadIdx.x >> 2) & 1;
        const cx<TP> u = psi[2 * n + sw], v = psi[2 * n + 1 - sw];
        s0 = promote_cx<T, TP>(sw ? v : u);
        s1 = promote_cx<T, TP>(sw ? u : v);
    } else {
        s0 = promote_cx<T, TP>(psi[2 * n]);
        s1 = promote_cx<T, TP>(psi[2 * n + 1]);
    }
}

template <typename T, bool DAG, typename TP = T, bool TILE = false>
__device__ __forceinline__ void dirac_site(const SiteOp<T>& L, const cx<TP>* __restrict__ psi, int n, T mass,
                                           cx<T>& o0, cx<T>& o1) {
    cx<T> a, b, c, d, e, f, g, h, p0, p1;
    site_spins<T, TP, TILE>(psi, L.r0, a, b);
    site_spins<T, TP, TILE>(psi, L.r1, c, d);
    site_spins<T, TP, TILE>(psi, L.l0, e, f);
    site_spins<T, TP, TILE>(psi, L.l1, g, h);
    site_spins<T, TP, TILE>(psi, n, p0, p1);
    cx<T> t0, t1, t2, t3;
    if (!DAG) {
        t0 = L.sR * cmul(L.u0, a - b);
        t1 = cmul(L.u1, c + cmuli(d));
        t2 = L.sL * cmul(L.ul0, e + f);
        t3 = cmul(L.ul1, g - cmuli(h));
    } else {
        t0 = L.sL * cmul(L.ul0, e - f);
        t1 = cmul(L.ul1, g + cmuli(h));
        t2 = L.sR * cmul(L.u0, a + b);
        t3 = cmul(L.u1, c - cmuli(d));
    }
    o0 = mass * p0 - T(0.5) * (t0 + t1 + t2 + t3);
    o1 = mass * p1 - T(0.5) * ((t2 - t0) + cmuli(t3 - t1));
}

}  // namespace amgb
