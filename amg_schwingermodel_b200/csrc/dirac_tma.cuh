// D_phi / D_dagger_phi (src/dirac_operator.cpp:3-54) for many sources, fed by the bulk-copy
// engine (TMA, cp.async.bulk) through shared memory.
//
// A CTA owns a tile of kTX x-rows by kTT t-sites and walks the sources (two CTAs per SM, so
// one's start overlaps the other's work).  For each source the tile plus its one-site halo
// ((kTX + 2) row segments of kTT + 2 sites, periodic in both directions) is brought into
// shared memory by 1-D bulk copies that complete on an mbarrier; two buffers alternate, so
// the copies of source r + 2 are in flight while source r is computed from the other buffer.
// The links of the tile's sites are read once and kept in registers for every source.  Each thread computes the kTX sites of one t column with the
// same per-site arithmetic as k_dirac (dirac_site), reading the neighbours from shared memory,
// and writes them with coalesced stores.
//
// Every wait on an mbarrier is bounded: after kTmaSpinLimit polls the kernel sets bit 0 of
// the device flag g_fine_err, waits (bounded again) for the copies it still has in flight and
// returns; the host reads the flag after the work (fine_error_check).  dirac_tma_wait_test
// runs the kernel without issuing any copy, so its first wait runs out with nothing in flight,
// and returns the flag (the self-test of that path).
#pragma once
#include "common.cuh"
#include "stencil.cuh"

namespace amgb {

constexpr int kTX = 4;                 // x rows per tile (sites per thread)
constexpr int kTT = 256;               // t sites per tile (threads per CTA)
constexpr int kTmaSpinLimit = 1 << 22;

__device__ int g_fine_err;             // bit 0: a bulk-copy wait gave up

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// true once the phase with this parity has completed, false after `limit` polls
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; i++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(bar)
        : "memory");
}

// shared memory per tile buffer for spinors stored as TIN
template <typename TIN>
__host__ __device__ constexpr int dirac_tma_buf_bytes() {
    return (kTX + 2) * (kTT + 2) * 2 * (int)sizeof(cx<TIN>);
}
// dynamic shared memory: two tile buffers, then two mbarriers
template <typename TIN>
__host__ __device__ constexpr int dirac_tma_smem() { return 2 * dirac_tma_buf_bytes<TIN>() + 16; }

// TIN: the spinors' storage type (T, or float for FP32 spinors into the FP64 operator); COPY:
// also copy the input (as stored, FP32) to in_copy; SELF_TEST: issue no copies at all and poll 256
// times per wait, so the first wait runs out with nothing in flight (the bounded-wait
// self-test); RES: the residual out = b - D in instead (source r's b at bres + r * bstride, the
// same site arithmetic as k_residual), skipping the sources with act[r] == 0 and, when
// partial is given, writing each CTA's sum of |out|^2 to partial[r * gridDim.x * gridDim.y +
// CTA]
// (UA: the links' type, a plain pointer or the storage-format view of the mixed form's links)
template <typename T, bool DAG, typename TIN = T, bool COPY = false, bool SELF_TEST = false, bool RES = false,
          typename UA = const cx<T>* __restrict__>
__global__ void __launch_bounds__(kTT, 2) k_dirac_tma(UA U, const cx<TIN>* __restrict__ in,
                                                      cx<T>* __restrict__ out, int nx, int nt, T m0, int nrhs,
                                                      cx<TIN>* __restrict__ in_copy, const cx<T>* __restrict__ bres,
                                                      long long bstride, const int* __restrict__ act,
                                                      double* __restrict__ partial) {
    constexpr int wait_limit = SELF_TEST ? 256 : kTmaSpinLimit;
    extern __shared__ __align__(128) unsigned char smraw_d[];
    __shared__ double red[kTT / 32 + 1];                // the residual's norm reduction
    constexpr int RS = kTT + 2;                         // sites per staged row segment
    constexpr int SB = 2 * (int)sizeof(cx<TIN>);        // bytes per site (both spins)
    constexpr int BUF = dirac_tma_buf_bytes<TIN>();
    cx<TIN>* buf0 = reinterpret_cast<cx<TIN>*>(smraw_d);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smraw_d + 2 * BUF);
    const unsigned bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const int N = nx * nt;
    const int tid = threadIdx.x;
    const int t0 = blockIdx.x * kTT, x0 = blockIdx.y * kTX;
    const bool interior_t = t0 >= 1 && t0 + kTT + 1 <= nt;

    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // the copies of one source into buffer b: warp 0, lane r < kTX + 2 stages row x0 - 1 + r
    auto issue = [&](int rhs, int b) {
        const unsigned bar = b ? bar1 : bar0;
        const unsigned dst0 = smem_u32(smraw_d + b * BUF);
        const cx<TIN>* src = in + (long long)rhs * N * 2;
        if (tid == 0) mbar_arrive_expect_tx(bar, (unsigned)((kTX + 2) * RS * SB));
        __syncwarp();
        if (tid < kTX + 2) {
            const int xr = (x0 - 1 + tid + nx) % nx;
            const unsigned drow = dst0 + (unsigned)(tid * RS * SB);
            const cx<TIN>* srow = src + (long long)xr * nt * 2;
            if (interior_t) {
                bulk_g2s(drow, srow + 2 * (t0 - 1), (unsigned)(RS * SB), bar);
            } else {
                bulk_g2s(drow, srow + 2 * ((t0 - 1 + nt) % nt), (unsigned)SB, bar);
                bulk_g2s(drow + SB, srow + 2 * t0, (unsigned)(kTT * SB), bar);
                bulk_g2s(drow + (unsigned)((kTT + 1) * SB), srow + 2 * ((t0 + kTT) % nt), (unsigned)SB, bar);
            }
        }
    };

    // links and geometry of this thread's kTX sites, read once for every source; the
    // neighbour indices point into the staged tile (row r + 1 of the buffer holds lattice
    // row x0 + r)
    SiteOp<T> L[kTX];
#pragma unroll
    for (int r = 0; r < kTX; r++) {
        L[r] = site_op<T>(U, (x0 + r) * nt + t0 + tid, nx, nt);
        const int c = (r + 1) * RS + tid + 1;
        L[r].r0 = c + 1;
        L[r].l0 = c - 1;
        L[r].r1 = c + RS;
        L[r].l1 = c - RS;
    }
    if (tid < 32 && !SELF_TEST) {
        issue(0, 0);
        if (nrhs > 1) issue(1, 1);
    }
    int issued = SELF_TEST ? 0 : (nrhs > 1 ? 2 : 1);   // sources whose copies have been issued
    const T mass = m0 + T(2);
    int done = 0;                      // sources whose copies every thread has seen land
    for (int rhs = 0; rhs < nrhs; rhs++) {
        const int b = rhs & 1;
        const bool ok = mbar_wait(b ? bar1 : bar0, (unsigned)((rhs >> 1) & 1), wait_limit);
        // one decision for the whole CTA, so no thread leaves the barriers below
        if (__syncthreads_or(!ok)) break;
        done = rhs + 1;
        const cx<TIN>* tile = buf0 + (size_t)b * (BUF / sizeof(cx<TIN>));
        cx<T>* o = out + (long long)rhs * N * 2;
        if (!RES || !act || act[rhs]) {
            double nrm = 0;
#pragma unroll
            for (int r = 0; r < kTX; r++) {
                const int c = (r + 1) * RS + tid + 1;
                cx<T> o0, o1;
                dirac_site<T, DAG, TIN, true>(L[r], tile, c, mass, o0, o1);
                const long long n = (long long)(x0 + r) * nt + t0 + tid;
                if constexpr (RES) {
                    const cx<T>* bb = bres + (long long)rhs * bstride;
                    o0 = bb[2 * n] - o0;
                    o1 = bb[2 * n + 1] - o1;
                    nrm += (double)cnorm2(o0) + (double)cnorm2(o1);
                }
                o[2 * n] = o0;
                o[2 * n + 1] = o1;
                if constexpr (COPY) {
                    static_assert(sizeof(TIN) == 4, "the copy moves one FP32 site (16 bytes)");
                    reinterpret_cast<float4*>(in_copy + (long long)rhs * N * 2)[n] =
                        reinterpret_cast<const float4*>(tile)[c];
                }
            }
            if (RES && partial) {
                // the whole CTA takes this branch (act is per source)
                nrm = cta_sum(nrm, red);
                if (tid == 0) partial[(long long)rhs * gridDim.x * gridDim.y + blockIdx.y * gridDim.x + blockIdx.x] = nrm;
            }
        }
        __syncthreads();   // every thread is done with buffer b
        if (rhs + 2 < nrhs) {
            if (tid < 32) {
                if (tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                issue(rhs + 2, b);
            }
            issued = rhs + 3;
        }
    }
    if (done < nrhs) {
        if (tid == 0) atomicOr(&g_fine_err, 1);
        // let the copies still in flight land before the CTA's shared memory goes away (the
        // waits are bounded like the others)
        for (int q = done; q < issued; q++)
            (void)mbar_wait((q & 1) ? bar1 : bar0, (unsigned)((q >> 1) & 1), wait_limit);
    }
}

}  // namespace amgb
