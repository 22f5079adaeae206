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
template <typename T, bool DAG, typename TP = T>
__device__ __forceinline__ void dirac_site(const SiteOp<T>& L, const cx<TP>* __restrict__ psi, int n, T mass,
                                           cx<T>& o0, cx<T>& o1) {
    const cx<T> a = promote_cx<T, TP>(psi[2 * L.r0]), b = promote_cx<T, TP>(psi[2 * L.r0 + 1]);
    const cx<T> c = promote_cx<T, TP>(psi[2 * L.r1]), d = promote_cx<T, TP>(psi[2 * L.r1 + 1]);
    const cx<T> e = promote_cx<T, TP>(psi[2 * L.l0]), f = promote_cx<T, TP>(psi[2 * L.l0 + 1]);
    const cx<T> g = promote_cx<T, TP>(psi[2 * L.l1]), h = promote_cx<T, TP>(psi[2 * L.l1 + 1]);
    const cx<T> p0 = promote_cx<T, TP>(psi[2 * n]), p1 = promote_cx<T, TP>(psi[2 * n + 1]);
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
