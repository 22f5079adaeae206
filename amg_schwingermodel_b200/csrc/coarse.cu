// The coarse-level engine kernel: one CTA per source runs a whole multigrid operation
// below the fine level (K-cycle FGMRES, cycles, SAP, coarsest GMRES) without returning
// to the host, so the data-dependent inner iterations cost no launches or host syncs.
#include <cstdlib>
#include <cstring>

#include "kernels.h"

namespace amgb {

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// One source per thread-block cluster of `csize` CTAs (csize = 1: a plain CTA).  Every CTA
// keeps its own copy of all vectors in its slab and runs the same control flow; the level
// operators are split across the cluster.  The entry op reads `in` and (for the in/out ops)
// `out` into slab copies, and cluster rank 0 writes the result back.
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_engine(const EngArgs<T>* __restrict__ a, int op, int level,
                                                           int nu, const cx<T>* in, long long in_stride, cx<T>* out,
                                                           long long out_stride, int csize) {
    extern __shared__ __align__(16) unsigned char smraw_e[];
    Eng<T> E;
    E.a = a;
    E.csize = csize;
    E.crank = csize > 1 ? (int)cluster_rank() : 0;
    E.slab = a->work + (long long)blockIdx.x * a->slab;
    E.smem = reinterpret_cast<char*>(smraw_e);
    E.red = reinterpret_cast<T*>(smraw_e + a->smem_red);
    const int src = blockIdx.x / csize;
    const cx<T>* b = in + (long long)src * in_stride;
    cx<T>* xo = out + (long long)src * out_stride;
    const EngLevel<T>& L = a->lv[level];
    const int nl = L.n * L.K;
    const int nc = (op == ENG_RESTRICT || op == ENG_PROLONG) ? a->lv[level + 1].n * a->lv[level + 1].K : nl;
    const int nin = op == ENG_PROLONG ? nc : nl;
    const int nout = op == ENG_RESTRICT ? nc : nl;
    cx<T>* ib = E.work(a->off_io);
    cx<T>* ob = ib + a->io_len;
    for (int e = threadIdx.x; e < nin; e += blockDim.x) ib[e] = b[e];
    if (op == ENG_KCYCLE || op == ENG_VCYCLE || op == ENG_SAP)
        for (int e = threadIdx.x; e < nout; e += blockDim.x) ob[e] = xo[e];
    __syncthreads();
    int ret = 0;
    switch (op) {
        case ENG_KFGMRES: ret = Cycles<T, kMaxLevels>::kfgmres(E, level, ib, ob); break;
        case ENG_KCYCLE: Cycles<T, kMaxLevels>::kcycle(E, level, ib, ob); break;
        case ENG_VCYCLE: Cycles<T, kMaxLevels>::vcycle(E, level, ib, ob); break;
        case ENG_SAP: ret = eng_sap(E, level, ib, ob, nu); break;
        case ENG_APPLY: dc_apply(E, L, a->p.m0, ib, ob); break;
        case ENG_GMRES: ret = eng_coarse_gmres(E, level, ib, ob); break;
        case ENG_RESTRICT: restrict_v(E, L, ib, ob); break;
        case ENG_PROLONG: prolong_v(E, L, ib, ob, 0); break;
        default: break;
    }
    __syncthreads();
    if (E.crank == 0) {
        for (int e = threadIdx.x; e < nout; e += blockDim.x) xo[e] = ob[e];
        if (threadIdx.x == 0 && a->status) a->status[src] = ret;
    }
}

// Threads per engine CTA: kEngineThreads, or 256 with AMG_ENGINE_THREADS=256 (read once per
// process; fewer threads per CTA leave each thread more registers).
int engine_threads() {
    static int nt = 0;
    if (!nt) {
        const char* e = getenv("AMG_ENGINE_THREADS");
        nt = (e && !strcmp(e, "256")) ? 256 : kEngineThreads;
    }
    return nt;
}

template <typename T, int NT>
cudaError_t launch_engine_nt(const EngArgs<T>* dev_args, int op, int level, int nu, const cx<T>* in,
                             long long in_stride, cx<T>* out, long long out_stride, int nsrc, int smem_bytes,
                             int csize, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_engine<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    if (csize > 8) {
        e = cudaFuncSetAttribute(k_engine<T, NT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nsrc * csize);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_engine<T, NT>, dev_args, op, level, nu, in, in_stride, out, out_stride, csize);
    count_launch(1);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_engine_dev(const EngArgs<T>* dev_args, int op, int level, int nu, const cx<T>* in,
                              long long in_stride, cx<T>* out, long long out_stride, int nsrc, int smem_bytes,
                              int csize, cudaStream_t s) {
    if (engine_threads() == 256)
        return launch_engine_nt<T, 256>(dev_args, op, level, nu, in, in_stride, out, out_stride, nsrc, smem_bytes,
                                        csize, s);
    return launch_engine_nt<T, kEngineThreads>(dev_args, op, level, nu, in, in_stride, out, out_stride, nsrc,
                                               smem_bytes, csize, s);
}

// Active clusters of `csize` engine CTAs the device can hold at once (0 when that size is
// not schedulable).
template <typename T, int NT>
int engine_max_clusters_nt(int csize, int smem_bytes) {
    if (cudaFuncSetAttribute(k_engine<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes) != cudaSuccess)
        return 0;
    if (csize > 8 &&
        cudaFuncSetAttribute(k_engine<T, NT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem_bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_engine<T, NT>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <typename T>
int engine_max_clusters(int csize, int smem_bytes) {
    return engine_threads() == 256 ? engine_max_clusters_nt<T, 256>(csize, smem_bytes)
                                   : engine_max_clusters_nt<T, kEngineThreads>(csize, smem_bytes);
}

template cudaError_t launch_engine_dev<double>(const EngArgs<double>*, int, int, int, const cx<double>*, long long,
                                               cx<double>*, long long, int, int, int, cudaStream_t);
template cudaError_t launch_engine_dev<float>(const EngArgs<float>*, int, int, int, const cx<float>*, long long,
                                              cx<float>*, long long, int, int, int, cudaStream_t);
template int engine_max_clusters<double>(int, int);
template int engine_max_clusters<float>(int, int);

}  // namespace amgb
