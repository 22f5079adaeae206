// Shared device helpers: complex arithmetic on double2 / float2, precision traits,
// deterministic CTA reductions, error handling.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <cstdio>

namespace amgb {

// ---------------------------------------------------------------------------------
// precision traits: T is the real type the arithmetic runs in
// ---------------------------------------------------------------------------------
template <typename T> struct CxT;
template <> struct CxT<double> { using type = double2; };
template <> struct CxT<float> { using type = float2; };
template <typename T> using cx = typename CxT<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T re, T im) { cx<T> r; r.x = re; r.y = im; return r; }
template <typename T> __host__ __device__ __forceinline__ cx<T> czero() { return mk<T>(T(0), T(0)); }

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a) { return make_double2(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2& operator+=(double2& a, double2 b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ __forceinline__ double2& operator-=(double2& a, double2 b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ __forceinline__ float2& operator+=(float2& a, float2 b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ __forceinline__ float2& operator-=(float2& a, float2 b) { a.x -= b.x; a.y -= b.y; return a; }

// a * b
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
// acc += a * b
template <typename C> __host__ __device__ __forceinline__ void cfma(C& acc, C a, C b) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
template <typename C> __host__ __device__ __forceinline__ void cfmac(C& acc, C a, C b) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C> __host__ __device__ __forceinline__ C cmuli(C a) { C r; r.x = -a.y; r.y = a.x; return r; }   // i*a
template <typename C> __host__ __device__ __forceinline__ auto cnorm2(C a) -> decltype(a.x) { return a.x * a.x + a.y * a.y; }
// a / b for complex b
template <typename C> __host__ __device__ __forceinline__ C cdiv(C a, C b) {
    auto d = b.x * b.x + b.y * b.y;
    C r; r.x = (a.x * b.x + a.y * b.y) / d; r.y = (a.y * b.x - a.x * b.y) / d; return r;
}

template <typename To, typename From> __host__ __device__ __forceinline__ cx<To> ccast(From a) { return mk<To>((To)a.x, (To)a.y); }

// storage conversions (bf16 pairs for test vectors / links in the mixed form)
__device__ __forceinline__ float2 load_cx(const __nv_bfloat162* p) { return __bfloat1622float2(*p); }
__device__ __forceinline__ float2 load_cx(const float2* p) { return *p; }
__device__ __forceinline__ double2 load_cx(const double2* p) { return *p; }

// Fine-lattice links U[N][2] as a kernel reads them: cx<T> (the FP64 set, and the FP32 copy of
// the mixed form) or, in the mixed form, BF16 or FP16 pairs; element i converts to cx<T>.
enum { LINK_NATIVE = 0, LINK_BF16 = 1, LINK_F16 = 2 };
template <typename T>
struct Links {
    const void* p;
    int fmt;
    __host__ __device__ Links(const cx<T>* q) : p(q), fmt(LINK_NATIVE) {}
    __host__ __device__ Links(const void* q, int f) : p(q), fmt(f) {}
    __device__ __forceinline__ cx<T> operator[](long long i) const {
        if constexpr (sizeof(T) == 4) {
            if (fmt == LINK_BF16) return __bfloat1622float2(static_cast<const __nv_bfloat162*>(p)[i]);
            if (fmt == LINK_F16) return __half22float2(static_cast<const __half2*>(p)[i]);
        }
        return static_cast<const cx<T>*>(p)[i];
    }
};

// ---------------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic sum over the whole CTA; every thread receives the result.
// `red` is shared scratch of at least blockDim.x/32 + 1 entries of T.
template <typename T> __device__ __forceinline__ T cta_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    T s = T(0);
    for (int i = 0; i < nw; i++) s += red[i];
    return s;
}

}  // namespace amgb

#define AMG_CUDA_TRY(expr)                                                         \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) {                                                    \
            amgb::set_last_error(cudaGetErrorString(_e), __FILE__, __LINE__);       \
            return AMG_ERR_CUDA;                                                    \
        }                                                                           \
    } while (0)
