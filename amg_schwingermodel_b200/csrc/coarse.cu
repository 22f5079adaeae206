// The coarse-level engine kernel: one CTA per source runs a whole multigrid operation
// below the fine level (K-cycle FGMRES, cycles, SAP, coarsest GMRES) without returning
// to the host, so the data-dependent inner iterations cost no launches or host syncs.
#include "kernels.h"

namespace amgb {

template <typename T>
__global__ void __launch_bounds__(kEngineThreads) k_engine(const EngArgs<T>* __restrict__ a, int op, int level,
                                                           int nu, const cx<T>* in, long long in_stride, cx<T>* out,
                                                           long long out_stride) {
    extern __shared__ __align__(16) unsigned char smraw_e[];
    Eng<T> E;
    E.a = a;
    E.slab = a->work + (long long)blockIdx.x * a->slab;
    E.smem = reinterpret_cast<char*>(smraw_e);
    E.red = reinterpret_cast<T*>(smraw_e + a->smem_red);
    const cx<T>* b = in + (long long)blockIdx.x * in_stride;
    cx<T>* x = out + (long long)blockIdx.x * out_stride;
    int ret = 0;
    switch (op) {
        case ENG_KFGMRES: ret = Cycles<T, kMaxLevels>::kfgmres(E, level, b, x); break;
        case ENG_KCYCLE: Cycles<T, kMaxLevels>::kcycle(E, level, b, x); break;
        case ENG_VCYCLE: Cycles<T, kMaxLevels>::vcycle(E, level, b, x); break;
        case ENG_SAP: ret = eng_sap(E, level, b, x, nu); break;
        case ENG_APPLY: dc_apply(E.L(level), a->p.m0, b, x); break;
        case ENG_GMRES: ret = eng_coarse_gmres(E, level, b, x); break;
        case ENG_RESTRICT: restrict_v(E.L(level), b, x); break;
        case ENG_PROLONG: prolong_v(E.L(level), b, x, 0); break;
        default: break;
    }
    if (threadIdx.x == 0 && a->status) a->status[blockIdx.x] = ret;
}

template <typename T>
cudaError_t launch_engine_dev(const EngArgs<T>* dev_args, int op, int level, int nu, const cx<T>* in,
                              long long in_stride, cx<T>* out, long long out_stride, int nsrc, int smem_bytes,
                              cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_engine<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    k_engine<T><<<nsrc, kEngineThreads, smem_bytes, s>>>(dev_args, op, level, nu, in, in_stride, out, out_stride);
    count_launch(1);
    return cudaGetLastError();
}

template cudaError_t launch_engine_dev<double>(const EngArgs<double>*, int, int, int, const cx<double>*, long long,
                                               cx<double>*, long long, int, int, cudaStream_t);
template cudaError_t launch_engine_dev<float>(const EngArgs<float>*, int, int, int, const cx<float>*, long long,
                                              cx<float>*, long long, int, int, cudaStream_t);

}  // namespace amgb
