// Level-0 transfers of the mixed form on the 5th-generation tensor cores (tcgen05, TF32 inputs,
// FP32 accumulators in tensor memory): the restriction P^dagger v (Level::Pt_v,
// src/level.cpp:212-237) and the prolongation psi += P vc (Level::P_v, src/level.cpp:182-209)
// for a batch of sources, with BF16 test vectors and FP32 sources.
//
// Both are multi-source GEMMs per aggregation block.  A complex product becomes a real one by
// laying the two spins and the real/imaginary parts of a site along the contraction (K) or
// row (M) index; entries that couple different spins are zero.  Operands are K-major in
// shared memory in the tensor cores' no-swizzle canonical layout: 8-row x 16-byte core
// matrices, the two core matrices of one MMA's K = 8 step 128 bytes apart (the descriptor's
// leading-dimension offset) and consecutive 8-row groups `sbo` bytes apart (its
// stride-dimension offset).  Element (row, k) of a tile therefore sits at byte
//     (row / 8) * sbo + (k / 4) * 128 + (row % 8) * 16 + (k % 4) * 4,
// and one 16-byte chunk holds one site's four K values for one row (sbo = K_tile / 4 * 128).
//
// Restriction (k_restrict0_tc): per CTA one chunk of one aggregation block's sites, in
// tiles of kRtcSites consecutive t sites (K = 4 per site: spin 0 re/im, spin 1 re/im).
//   A [M x K]: row m = (2k + s) * 2 + part, k < ntest test vectors, s the spin, part re/im:
//     (s, re) = [Wr, Wi] and (s, im) = [-Wi, Wr] on the spin-s pair of the site, 0 on the other
//     (so D = conj(W) v), built by the threads from BF16 W staged with cp.async;
//   B [N x K]: row r = source, the site's 16 bytes of v exactly as they lie in global memory
//     (cp.async straight into the core-matrix layout);
//   D [M x N] accumulates over the CTA's tiles in TMEM; the epilogue writes the chunk's
//   partial sums in the layout k_restrict0_sum finishes (row m is float m of an output
//   record, so a warp's stores are contiguous).
// The tiles go through a kRtcStages-deep ring: cp.async groups for tile t + kRtcStages - 1
// are in flight while tile t's A is built and its MMAs run; a stage is reused once the
// tcgen05.commit of the MMAs that read it has arrived on its mbarrier.
//
// Prolongation (k_prolong0_tc): per CTA one aggregation block; B [N x K] = the block's coarse
// vector for every source, K = (k, s', part') (4 ntest, padded to a multiple of 8) loaded once;
// per tile of 32 sites A [128 x K] with row m = (site, s, c) and (s, re) = [Wr, -Wi],
// (s, im) = [Wi, Wr] on the spin-s pair of test vector k, so D[m][r] is exactly the float of
// psi[r] that row m adds to (a warp's read-modify-write of psi is contiguous).
//
// M = 64 accumulators (restriction with ntest <= 16) live in TMEM lanes 32 w + i of warp w's
// sub-partition for rows 16 w + i (i < 16); M = 128 rows map to lanes one to one.
//
// Every mbarrier wait is bounded (kTmaSpinLimit polls).  A CTA whose wait gives up sets bit 1
// of g_fine_err, stops issuing work, waits (bounded) for its outstanding copies and MMAs,
// frees its tensor memory and returns; the host reads the flag (fine_error_check).
#pragma once
#include "common.cuh"
#include "dirac_tma.cuh"

namespace amgb {

constexpr int kRtcSites = 8;      // restriction: sites per tile (K = 32, four MMAs of K = 8)
constexpr int kRtcStages = 4;     // restriction: tile ring depth
constexpr int kPtcSites = 32;     // prolongation: sites per tile (M = 128 rows)

// ---- tcgen05 / async-copy primitives ---------------------------------------------------
__device__ __forceinline__ void tc_alloc(unsigned dst_smem, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory (st.shared, cp.async) made visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[adesc] * B[bdesc]^T, TF32 inputs, FP32 accumulators; issued by one thread
__device__ __forceinline__ void tc_mma_tf32(unsigned d_tmem, uint64_t adesc, uint64_t bdesc, unsigned idesc,
                                            unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
// the mbarrier at `bar` receives one arrival once every MMA this thread issued has completed
__device__ __forceinline__ void tc_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// 32 lanes x 32 columns of 32-bit accumulators: this thread's lane, columns col .. col + 31
__device__ __forceinline__ void tc_ld32(unsigned taddr, float (&d)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) d[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void cp_async16(unsigned dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(__cvta_generic_to_global(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle, leading-dimension (K) core-matrix
// offset 128 bytes, stride-dimension (8-row group) offset sbo bytes, version 1.
__device__ __forceinline__ uint64_t tc_sdesc(unsigned saddr, unsigned sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}
// Instruction descriptor of kind::tf32: FP32 accumulators, TF32 A and B, both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr unsigned tc_idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}
__host__ __device__ constexpr int tc_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }

// ---- restriction ------------------------------------------------------------------------
// shared memory: kRtcStages x (A [M][32] f32 | B [NP][32] f32 | Wraw [M/4][kRtcSites][2] bf16x2),
// then kRtcStages + 0 mbarriers, a word for the TMEM address and an abort flag
__host__ __device__ constexpr int rtc_stage_bytes(int M, int NP) {
    return M * 128 + NP * 128 + (M / 4) * kRtcSites * 8;
}
__host__ __device__ constexpr int rtc_smem_bytes(int M, int NP) {
    return kRtcStages * rtc_stage_bytes(M, NP) + kRtcStages * 8 + 16;
}

template <int M>
__global__ void __launch_bounds__(128) k_restrict0_tc(const __nv_bfloat162* __restrict__ W,
                                                      const float2* __restrict__ v, float2* __restrict__ partial,
                                                      int nx, int nt, int bt, int xe, int te, int nchunk, int ntest,
                                                      int nrhs, int NP) {
    extern __shared__ __align__(128) unsigned char smraw_r[];
    constexpr int KS = kRtcSites, NST = kRtcStages, D = NST - 1;
    const int N = nx * nt;
    const int chunk = blockIdx.x, blk = blockIdx.y, nblk = gridDim.y;
    const int bxi = blk / bt, bti = blk - bxi * bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int stage_bytes = rtc_stage_bytes(M, NP);
    const int a_bytes = M * 128, b_bytes = NP * 128;
    unsigned char* bars_p = smraw_r + NST * stage_bytes;
    unsigned* tslot = reinterpret_cast<unsigned*>(bars_p + NST * 8);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const unsigned sbase = smem_u32(smraw_r), bar0 = smem_u32(bars_p);
    const int tiles_row = te / KS, tiles = xe * tiles_row;
    const int per = (tiles + nchunk - 1) / nchunk;
    const int tile0 = min(tiles, chunk * per), T = min(tiles, tile0 + per) - tile0;
    const int rows = 4 * ntest;
    const unsigned ncols = tc_cols(NP);

    // zero every stage once (rows >= 4 ntest of A and rows >= nrhs of B stay zero), set up the
    // mbarriers and the tensor memory
    for (int q = tid; q < NST * stage_bytes / 16; q += 128)
        reinterpret_cast<float4*>(smraw_r)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid == 0) {
        for (int s = 0; s < NST; s++) mbar_init(bar0 + 8 * s, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tc_alloc(smem_u32(tslot), ncols);
        tc_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;

    auto site0 = [&](int tile) -> long long {   // first global site of a tile
        const int mx = tile / tiles_row, mt0 = (tile - mx * tiles_row) * KS;
        return (long long)(bxi * xe + mx) * nt + (bti * te + mt0);
    };
    // cp.async of tile t into stage t % NST: v rows (sources) and the test vectors' bytes
    auto produce = [&](int t) {
        const unsigned st = sbase + (t % NST) * stage_bytes;
        const long long n0 = site0(tile0 + t);
        // B: chunk (r, j) = v[r][n0 + j] (16 bytes) at (r / 8) * 1024 + j * 128 + (r % 8) * 16;
        // a warp's 32 chunks are 8 sources x 4 sites, i.e. four contiguous 128-byte runs
        for (int q = tid; q < ((nrhs + 7) / 8) * 8 * KS; q += 128) {
            const int rl = q & 7, j = (q >> 3) % KS, rg = (q >> 3) / KS;
            const int r = rg * 8 + rl;
            if (r < nrhs)
                cp_async16(st + a_bytes + rg * 1024 + j * 128 + rl * 16, v + ((long long)r * N + n0 + j) * 2);
        }
        // Wraw [k][j][s]: per test vector KS sites x 8 bytes contiguous in W
        for (int q = tid; q < ntest * (KS / 2); q += 128) {
            const int k = q / (KS / 2), c = q - k * (KS / 2);
            cp_async16(st + a_bytes + b_bytes + k * (KS * 8) + c * 16, W + ((long long)k * N + n0) * 2 + 4 * c);
        }
    };

    // ring: at step t the copies of tile t are issued and tile u = t - D (whose copies were
    // issued D steps earlier) is built and multiplied
    bool ok = true;
    int last_issued = -1;
    for (int t = 0; t < T + D; t++) {
        if (t < T) {
            if (t >= NST && !mbar_wait(bar0 + 8 * (t % NST), ((t / NST) - 1) & 1, kTmaSpinLimit)) *abort_flag = 1;
            else produce(t);
        }
        cp_async_commit();
        const int u = t - D;
        if (u < 0) continue;
        cp_async_wait<D>();
        __syncthreads();
        if (*abort_flag) {
            ok = false;
            break;
        }
        // A rows m = (2k + s) * 2 + part from Wraw: chunk (m, j) at (m / 8) * 1024 + j * 128 +
        // (m % 8) * 16; a warp writes 8 rows x 4 sites, four contiguous 128-byte runs
        unsigned char* st = smraw_r + (u % NST) * stage_bytes;
        const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(st + a_bytes + b_bytes);
        for (int q = tid; q < ((rows + 7) / 8) * 8 * KS; q += 128) {
            const int ml = q & 7, j = (q >> 3) % KS, mg = (q >> 3) / KS;
            const int m = mg * 8 + ml;
            if (m < rows) {
                const int part = m & 1, s = (m >> 1) & 1, k = m >> 2;
                const float2 w = __bfloat1622float2(wr[(k * KS + j) * 2 + s]);
                const float a0 = part ? -w.y : w.x, a1 = part ? w.x : w.y;
                const float4 val = s ? make_float4(0.f, 0.f, a0, a1) : make_float4(a0, a1, 0.f, 0.f);
                *reinterpret_cast<float4*>(st + mg * 1024 + j * 128 + ml * 16) = val;
            }
        }
        fence_async_smem();
        __syncthreads();
        if (warp == 0) {
            tc_fence_after();
            if (lane == 0) {
                const unsigned sa = sbase + (u % NST) * stage_bytes;
                const unsigned idesc = tc_idesc_tf32(M, NP);
#pragma unroll
                for (int q = 0; q < KS / 2; q++)
                    tc_mma_tf32(tmem, tc_sdesc(sa + q * 256, 1024), tc_sdesc(sa + a_bytes + q * 256, 1024), idesc,
                                (u > 0 || q > 0) ? 1u : 0u);
                tc_commit(bar0 + 8 * (u % NST));
            }
            __syncwarp();
        }
        last_issued = u;
    }

    // the last commit covers every MMA issued before it
    bool done = true;
    if (last_issued >= 0)
        done = mbar_wait(bar0 + 8 * (last_issued % NST), (last_issued / NST) & 1, kTmaSpinLimit);
    cp_async_wait_all();
    tc_fence_after();
    // one decision for the whole CTA (the TMEM loads below are warp-collective)
    if (!__syncthreads_and(ok && done)) {
        if (tid == 0) atomicOr(&g_fine_err, 2);
    } else {
        // epilogue: row m of D is float m of the (source, block, chunk) record
        const int m = (M == 64) ? (warp * 16 + lane) : (warp * 32 + lane);
        const bool row_ok = (M == 64 ? lane < 16 : true) && m < rows;
        float* pf = reinterpret_cast<float*>(partial);
        for (int c0 = 0; c0 < NP; c0 += 32) {
            float d[32];
            tc_ld32(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, d);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const int r = c0 + i;
                if (row_ok && r < nrhs) {
                    const long long rec = ((long long)r * nblk + blk) * nchunk + chunk;
                    pf[rec * (4 * ntest) + m] = T > 0 ? d[i] : 0.f;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, ncols);
}

// ---- prolongation -------------------------------------------------------------------------
// shared memory: A [128][KP] f32 | B [NP][KP] f32 | Wraw [ntest][kPtcSites][2] bf16x2 | mbarrier,
// TMEM address, abort flag
__host__ __device__ constexpr int ptc_kp(int ntest) { return (4 * ntest + 7) / 8 * 8; }
__host__ __device__ constexpr int ptc_smem_bytes(int ntest, int NP) {
    return 128 * ptc_kp(ntest) * 4 + NP * ptc_kp(ntest) * 4 + ntest * kPtcSites * 8 + 8 + 16;
}

__global__ void __launch_bounds__(128) k_prolong0_tc(const __nv_bfloat162* __restrict__ W,
                                                     const float2* __restrict__ vc, float2* __restrict__ psi, int nx,
                                                     int nt, int bt, int xe, int te, int ntest, int nblk, int nrhs,
                                                     int NP, int nsplit) {
    extern __shared__ __align__(128) unsigned char smraw_p[];
    constexpr int KS = kPtcSites;
    const int N = nx * nt;
    const int split = blockIdx.x, blk = blockIdx.y;
    const int bxi = blk / bt, bti = blk - bxi * bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KP = ptc_kp(ntest), SBO = (KP / 4) * 128;
    const int a_bytes = 128 * KP * 4, b_bytes = NP * KP * 4;
    unsigned char* wraw_p = smraw_p + a_bytes + b_bytes;
    unsigned char* bar_p = wraw_p + ntest * KS * 8;
    unsigned* tslot = reinterpret_cast<unsigned*>(bar_p + 8);
    const unsigned sbase = smem_u32(smraw_p), bar = smem_u32(bar_p);
    const int tiles_row = te / KS, tiles = xe * tiles_row;
    const int per = (tiles + nsplit - 1) / nsplit;
    const int tile0 = min(tiles, split * per), T = min(tiles, tile0 + per) - tile0;
    const unsigned ncols = tc_cols(NP);

    // A zero (the spin-coupling zeros and rows stay zero where no chunk writes), B = the
    // block's coarse vector of every source: row r, K (k, s', part') = vc[r][blk][2k + s'].part'
    for (int q = tid; q < (a_bytes + b_bytes) / 16; q += 128)
        reinterpret_cast<float4*>(smraw_p)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    for (int q = tid; q < nrhs * ntest; q += 128) {
        const int r = q / ntest, k = q - r * ntest;
        const float4 c = *reinterpret_cast<const float4*>(vc + ((long long)r * nblk + blk) * 2 * ntest + 2 * k);
        *reinterpret_cast<float4*>(smraw_p + a_bytes + (r / 8) * SBO + k * 128 + (r % 8) * 16) = c;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tc_alloc(smem_u32(tslot), ncols);
        tc_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;

    auto site0 = [&](int tile) -> long long {
        const int mx = tile / tiles_row, mt0 = (tile - mx * tiles_row) * KS;
        return (long long)(bxi * xe + mx) * nt + (bti * te + mt0);
    };
    auto fetch_w = [&](int t) {   // Wraw [k][j][s] <- W[k][n0 + j][s], 256 bytes per test vector
        const long long n0 = site0(tile0 + t);
        for (int q = tid; q < ntest * (KS / 2); q += 128) {
            const int k = q / (KS / 2), c = q - k * (KS / 2);
            cp_async16(smem_u32(wraw_p) + k * (KS * 8) + c * 16, W + ((long long)k * N + n0) * 2 + 4 * c);
        }
        cp_async_commit();
    };

    const unsigned idesc = tc_idesc_tf32(128, NP);
    const int m = warp * 32 + lane;                 // this thread's D row: site m / 4, spin, part
    const int jm = m >> 2, sm = (m >> 1) & 1, cm = m & 1;
    bool ok = true;
    if (T > 0) fetch_w(0);
    for (int t = 0; t < T; t++) {
        cp_async_wait<0>();
        __syncthreads();
        // A rows m = (site, s, c) from Wraw: chunk (m, k) at (m / 8) * SBO + k * 128 + (m % 8) * 16
        const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(wraw_p);
        for (int q = tid; q < 128 * ntest; q += 128) {
            const int ml = q & 7, k = (q >> 3) % ntest, mg = (q >> 3) / ntest;
            const int mm = mg * 8 + ml;
            const int j = mm >> 2, s = (mm >> 1) & 1, c = mm & 1;
            const float2 w = __bfloat1622float2(wr[(k * KS + j) * 2 + s]);
            const float a0 = c ? w.y : w.x, a1 = c ? w.x : -w.y;
            const float4 val = s ? make_float4(0.f, 0.f, a0, a1) : make_float4(a0, a1, 0.f, 0.f);
            *reinterpret_cast<float4*>(smraw_p + mg * SBO + k * 128 + ml * 16) = val;
        }
        fence_async_smem();
        __syncthreads();
        if (t + 1 < T) fetch_w(t + 1);   // Wraw is free once A is built
        if (warp == 0) {
            tc_fence_after();
            if (lane == 0) {
                for (int q = 0; q < KP / 8; q++)
                    tc_mma_tf32(tmem, tc_sdesc(sbase + q * 256, SBO), tc_sdesc(sbase + a_bytes + q * 256, SBO), idesc,
                                q > 0 ? 1u : 0u);
                tc_commit(bar);
            }
            __syncwarp();
        }
        if (!__syncthreads_and(mbar_wait(bar, t & 1, kTmaSpinLimit))) {
            ok = false;
            break;
        }
        tc_fence_after();
        // epilogue: psi[r] at float (n0 + j) * 4 + s * 2 + c gets D[m][r]
        const long long n = site0(tile0 + t) + jm;
        float* pf = reinterpret_cast<float*>(psi) + n * 4 + sm * 2 + cm;
        for (int c0 = 0; c0 < NP; c0 += 32) {
            float d[32];
            tc_ld32(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0, d);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const int r = c0 + i;
                if (r < nrhs) pf[(long long)r * N * 4] += d[i];
            }
        }
        tc_fence_before();
    }
    cp_async_wait_all();
    if (!ok && tid == 0) atomicOr(&g_fine_err, 2);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, ncols);
}

}  // namespace amgb
