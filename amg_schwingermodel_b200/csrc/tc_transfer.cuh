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
// The copies run several tiles ahead through a ring of data slots, and the A tiles go
// through a ring of their own; a slot is reused once the tcgen05.commit of the MMAs that
// read it has arrived on its mbarrier, two steps after they were issued.
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

constexpr int kTcThreads = 256;   // threads per CTA of both kernels
constexpr int kRtcSites = 16;     // restriction: sites per tile (K = 64, eight MMAs of K = 8)
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
// 32 lanes x 16 columns
__device__ __forceinline__ void tc_ld16(unsigned taddr, float (&d)[16]) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) d[i] = __uint_as_float(r[i]);
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
// cp.async.wait_group takes an immediate: at most n (0 .. 6) groups left in flight
__device__ __forceinline__ void cp_async_wait_dyn(int n) {
    switch (n) {
        case 0: cp_async_wait<0>(); break;
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        case 4: cp_async_wait<4>(); break;
        case 5: cp_async_wait<5>(); break;
        default: cp_async_wait<6>(); break;
    }
}

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
// Two rings in shared memory: nd data slots (B [NP][4 KS] f32 | Wraw [M/4][KS][2] bf16x2, filled
// by cp.async) and kRtcA slots for the A tiles the threads build; then one mbarrier per data
// slot (the MMAs of the tile in a slot commit to its barrier), a word for the TMEM address and
// an abort flag.  Copies run `lead` = nd - 2 tiles ahead of the tile being multiplied, so a data
// slot or an A slot is reused two steps after the MMAs that read it were issued.  With
// KS = kRtcSites sites per tile a row's chunks are 128 bytes apart and its 8-row groups
// KS * 128 bytes apart.
constexpr int kRtcA = 2;
// bytes per test vector in Wraw: KS sites x 8 bytes + 32 bytes, so the two test vectors a warp's
// A build reads at once fall in different banks
constexpr int kRtcWStride = kRtcSites * 8 + 32;
__host__ __device__ constexpr int rtc_data_bytes(int M, int NP) { return NP * kRtcSites * 16 + (M / 4) * kRtcWStride; }
__host__ __device__ constexpr int rtc_smem_bytes(int M, int NP, int nd) {
    return kRtcA * M * kRtcSites * 16 + nd * rtc_data_bytes(M, NP) + nd * 8 + 16;
}
// the deepest data ring (3 .. 6 slots) that fits `limit` bytes of shared memory, 0 if none does
// (4 slots of the 32-source, 16-test-vector shape take 72 KB, three CTAs per SM)
__host__ __device__ constexpr int rtc_ring(int M, int NP, int limit) {
    int nd = NP <= 32 ? 4 : 6;
    while (nd >= 3 && rtc_smem_bytes(M, NP, nd) > limit) nd--;
    return nd >= 3 ? nd : 0;
}

// NB: B chunks (16 bytes) per thread and tile = NP sources x KS sites / kTcThreads.  Every
// thread copies and builds the same chunks of every tile, so their offsets are computed once;
// ring positions and the tile's first site advance by counters.  One thread waits on the
// mbarriers while the others sleep at the CTA barrier that follows.
template <int M, int NB>
__global__ void __launch_bounds__(kTcThreads) k_restrict0_tc(const __nv_bfloat162* __restrict__ W,
                                                      const float2* __restrict__ v, float2* __restrict__ partial,
                                                      int nx, int nt, int bt, int xe, int te, int nchunk, int ntest,
                                                      int nrhs, int nd) {
    extern __shared__ __align__(128) unsigned char smraw_r[];
    constexpr int TPB = kTcThreads, KS = kRtcSites, NP = NB * TPB / KS, NA = M * KS / TPB;
    constexpr int NWC = ((M / 4) * (KS / 2) + TPB - 1) / TPB;
    constexpr int SBO = KS * 128;
    const int lead = nd - 2;
    const int N = nx * nt;
    const int chunk = blockIdx.x, blk = blockIdx.y, nblk = gridDim.y;
    const int bxi = blk / bt, bti = blk - bxi * bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int a_bytes = M * KS * 16, b_bytes = NP * KS * 16, data_bytes = rtc_data_bytes(M, NP);
    unsigned char* data_p = smraw_r + kRtcA * a_bytes;
    unsigned char* bars_p = data_p + nd * data_bytes;
    unsigned* tslot = reinterpret_cast<unsigned*>(bars_p + nd * 8);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const unsigned sbase = smem_u32(smraw_r), dbase = smem_u32(data_p), bar0 = smem_u32(bars_p);
    const int tiles_row = te / KS, tiles = xe * tiles_row;
    const int per = (tiles + nchunk - 1) / nchunk;
    const int tile0 = min(tiles, chunk * per), T = min(tiles, tile0 + per) - tile0;
    const int rows = 4 * ntest;
    const unsigned ncols = tc_cols(NP);

    // zero both rings once (rows >= 4 ntest of A and rows >= nrhs of B stay zero), set up the
    // mbarriers and the tensor memory
    for (int q = tid; q < (kRtcA * a_bytes + nd * data_bytes) / 16; q += TPB)
        reinterpret_cast<float4*>(smraw_r)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid == 0) {
        for (int s = 0; s < nd; s++) mbar_init(bar0 + 8 * s, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tc_alloc(smem_u32(tslot), ncols);
        tc_relinquish();
    }

    // this thread's chunks.  B chunk q = tid + TPB i: source r = (q / 8 / KS) * 8 + q % 8 and
    // site j = (q / 8) % KS, from float2 offset (r N + n0 + j) * 2 to (r / 8) * SBO + j * 128 +
    // (r % 8) * 16 (a warp: 8 sources x 4 sites, four contiguous 128-byte runs).
    int bsrc[NB];
    unsigned bdst[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int q = tid + TPB * i;
        const int rl = q & 7, j = (q >> 3) % KS, rg = (q >> 3) / KS, r = rg * 8 + rl;
        bsrc[i] = r < nrhs ? (r * N + j) * 2 : -1;
        bdst[i] = rg * SBO + j * 128 + rl * 16;
    }
    // W chunk q = tid + TPB i (< ntest KS / 2): test vector k = q / (KS / 2), sites 2c, 2c + 1
    // (c = q % (KS / 2)), from bf16x2 offset k N * 2 + 4 c (+ 2 n0) to Wraw at k kRtcWStride + c 16
    int wsrc[NWC];
    unsigned wdst[NWC];
#pragma unroll
    for (int i = 0; i < NWC; i++) {
        const int q = tid + TPB * i, k = q / (KS / 2), c = q % (KS / 2);
        wsrc[i] = k < ntest ? k * N * 2 + 4 * c : -1;
        wdst[i] = b_bytes + k * kRtcWStride + c * 16;
    }
    // A chunk q = tid + TPB i: row m = (q / 8 / KS) * 8 + q % 8, site j = (q / 8) % KS, at
    // (m / 8) * SBO + j * 128 + (m % 8) * 16, from Wraw word k kRtcWStride / 4 + j * 2 + s
    // (m = (2k + s) * 2 + part; a warp: 8 rows x 4 sites, four contiguous 128-byte runs).  The
    // row's spin and part are the same for all of a thread's chunks (m % 4 = tid % 4).
    unsigned adst[NA], asrc[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) {
        const int q = tid + TPB * i;
        const int ml = q & 7, j = (q >> 3) % KS, mg = (q >> 3) / KS, m = mg * 8 + ml;
        adst[i] = mg * SBO + j * 128 + ml * 16;
        asrc[i] = m < rows ? ((m >> 2) * (kRtcWStride / 4) + j * 2 + ((m >> 1) & 1)) : 0xFFFFFFFFu;
    }
    const bool apart = tid & 1, aspin = (tid >> 1) & 1;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;
    const uint64_t adesc0 = tc_sdesc(sbase, SBO), bdesc0 = tc_sdesc(dbase, SBO);
    constexpr unsigned idesc = tc_idesc_tf32(M, NP);

    // step t: copies of tile t are issued into data slot pslot; tile u = t - lead (copied
    // `lead` steps earlier, in data slot cslot) gets its A tile in slot u % 2 and its MMAs.
    // The MMAs of tile t - nd (issued two steps before) were the last readers of data slot
    // pslot and of A slot u % 2; thread 0 waits for them (phase bits per data slot in ph).
    bool ok = true;
    int last_issued = -1;
    int pslot = 0, cslot = 0;
    unsigned ph = 0;
    int pmx = tile0 / tiles_row, pmt = (tile0 - pmx * tiles_row) * KS;   // tile t's row and t offset
    for (int t = 0; t < T + lead; t++) {
        const int u = t - lead;
        if (tid == 0 && t >= nd) {
            if (!mbar_wait(bar0 + 8 * pslot, (ph >> pslot) & 1, kTmaSpinLimit)) *abort_flag = 1;
            ph ^= 1u << pslot;
        }
        cp_async_wait_dyn(lead - 1);   // tile u's copies have landed
        __syncthreads();
        if (*abort_flag) {
            ok = false;
            break;
        }
        if (t < T) {
            const unsigned st = dbase + pslot * data_bytes;
            const int n0 = (bxi * xe + pmx) * nt + bti * te + pmt;
#pragma unroll
            for (int i = 0; i < NB; i++)
                if (bsrc[i] >= 0) cp_async16(st + bdst[i], v + bsrc[i] + 2 * n0);
#pragma unroll
            for (int i = 0; i < NWC; i++)
                if (wsrc[i] >= 0) cp_async16(st + wdst[i], W + wsrc[i] + 2 * n0);
            pmt += KS;
            if (pmt == te) {
                pmt = 0;
                pmx++;
            }
        }
        cp_async_commit();
        if (++pslot == nd) pslot = 0;
        if (u < 0) continue;
        unsigned char* at = smraw_r + (u & 1) * a_bytes;
        const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(data_p + cslot * data_bytes + b_bytes);
#pragma unroll
        for (int i = 0; i < NA; i++) {
            if (asrc[i] != 0xFFFFFFFFu) {
                const float2 w = __bfloat1622float2(wr[asrc[i]]);
                const float a0 = apart ? -w.y : w.x, a1 = apart ? w.x : w.y;
                *reinterpret_cast<float4*>(at + adst[i]) =
                    aspin ? make_float4(0.f, 0.f, a0, a1) : make_float4(a0, a1, 0.f, 0.f);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint64_t ad = adesc0 + (uint64_t)((u & 1) * (a_bytes >> 4));
            const uint64_t bd = bdesc0 + (uint64_t)(cslot * (data_bytes >> 4));
#pragma unroll
            for (int q = 0; q < KS / 2; q++)
                tc_mma_tf32(tmem, ad + (uint64_t)(q * 16), bd + (uint64_t)(q * 16), idesc, (u > 0 || q > 0) ? 1u : 0u);
            tc_commit(bar0 + 8 * cslot);
        }
        if (++cslot == nd) cslot = 0;
        last_issued = u;
    }

    // the last commit covers every MMA issued before it
    bool done = true;
    if (tid == 0 && last_issued >= 0)
        done = mbar_wait(bar0 + 8 * (last_issued % nd), (last_issued / nd) & 1, kTmaSpinLimit);
    cp_async_wait_all();
    // one decision for the whole CTA (the TMEM loads below are warp-collective)
    if (!__syncthreads_and(ok && done)) {
        if (tid == 0) atomicOr(&g_fine_err, 2);
    } else if (warp < 4) {
        tc_fence_after();
        // epilogue (warps 0-3, one per TMEM sub-partition): row m of D is float m of the
        // (source, block, chunk) record
        const int m = (M == 64) ? (warp * 16 + lane) : (warp * 32 + lane);
        const bool row_ok = (M == 64 ? lane < 16 : true) && m < rows;
        float* pf = reinterpret_cast<float*>(partial);
#pragma unroll
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
// shared memory: A [128][KP] f32 | B [NP][KP] f32 | Wraw [ntest][kPtcSites sites x 8 bytes + 16
// bytes of padding, so the A build's reads of four test vectors fall in different banks] |
// mbarrier | TMEM address.  Two accumulator buffers of NP columns in TMEM: the MMAs of tile t
// run while the threads apply tile t - 1.
constexpr int kPtcWStride = kPtcSites * 8 + 16;
__host__ __device__ constexpr int ptc_kp(int ntest) { return (4 * ntest + 7) / 8 * 8; }
__host__ __device__ constexpr int ptc_smem_bytes(int ntest, int NP) {
    return 128 * ptc_kp(ntest) * 4 + NP * ptc_kp(ntest) * 4 + ntest * kPtcWStride + 8 + 16;
}

__global__ void __launch_bounds__(kTcThreads) k_prolong0_tc(const __nv_bfloat162* __restrict__ W,
                                                     const float2* __restrict__ vc, float2* __restrict__ psi, int nx,
                                                     int nt, int bt, int xe, int te, int ntest, int nblk, int nrhs,
                                                     int NP, int nsplit, int add) {
    extern __shared__ __align__(128) unsigned char smraw_p[];
    constexpr int TPB = kTcThreads, KS = kPtcSites;
    const int N = nx * nt;
    const int split = blockIdx.x, blk = blockIdx.y;
    const int bxi = blk / bt, bti = blk - bxi * bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KP = ptc_kp(ntest), SBO = (KP / 4) * 128;
    const int a_bytes = 128 * KP * 4, b_bytes = NP * KP * 4;
    unsigned char* wraw_p = smraw_p + a_bytes + b_bytes;
    unsigned char* bar_p = wraw_p + ntest * kPtcWStride;
    unsigned* tslot = reinterpret_cast<unsigned*>(bar_p + 8);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const unsigned sbase = smem_u32(smraw_p), bar = smem_u32(bar_p);
    const int tiles_row = te / KS, tiles = xe * tiles_row;
    const int per = (tiles + nsplit - 1) / nsplit;
    const int tile0 = min(tiles, split * per), T = min(tiles, tile0 + per) - tile0;
    const unsigned ncols = tc_cols(2 * NP);

    // A zero (the spin-coupling zeros and rows stay zero where no chunk writes), B = the
    // block's coarse vector of every source: row r, K (k, s', part') = vc[r][blk][2k + s'].part'
    for (int q = tid; q < (a_bytes + b_bytes) / 16; q += TPB)
        reinterpret_cast<float4*>(smraw_p)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    for (int q = tid; q < nrhs * ntest; q += TPB) {
        const int r = q / ntest, k = q - r * ntest;
        const float4 c = *reinterpret_cast<const float4*>(vc + ((long long)r * nblk + blk) * 2 * ntest + 2 * k);
        *reinterpret_cast<float4*>(smraw_p + a_bytes + (r / 8) * SBO + k * 128 + (r % 8) * 16) = c;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tc_alloc(smem_u32(tslot), ncols);
        tc_relinquish();
    }
    fence_async_smem();
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
        for (int q = tid; q < ntest * (KS / 2); q += TPB) {
            const int k = q >> 4, c = q & 15;   // KS / 2 = 16 chunks per test vector
            cp_async16(smem_u32(wraw_p) + k * kPtcWStride + c * 16, W + ((long long)k * N + n0) * 2 + 4 * c);
        }
        cp_async_commit();
    };
    // psi[r] at float (n0 + j) * 4 + s * 2 + c gets D[m][r] for this thread's row m = (j, s, c)
    // (warps w and w + 4 share TMEM sub-partition w: rows 32 w .. 32 w + 31, columns split in
    // halves); every load of a batch of 16 sources before any store: the sources' addresses are
    // distinct, but the compiler cannot know it, and interleaved load/store pairs would wait
    // for DRAM one source at a time
    const int m = (warp & 3) * 32 + lane, half = warp >> 2;
    const int arow = (m >> 2) * 2 + ((m >> 1) & 1);   // Wraw word of row m's site and spin
    const bool acm = m & 1, asm_ = (m >> 1) & 1;
    const long long rs = (long long)N * 4;             // floats between two sources of psi
    auto apply = [&](int t) {
        const int jm = m >> 2, sm = (m >> 1) & 1, cm = m & 1;
        const int c_lo = half * (NP / 2), c_hi = min(nrhs, c_lo + NP / 2);
        float* pf = reinterpret_cast<float*>(psi) + (site0(tile0 + t) + jm) * 4 + sm * 2 + cm + c_lo * rs;
        const unsigned dcol = (t & 1) * NP;
        for (int c0 = c_lo; c0 < c_lo + NP / 2; c0 += 16) {
            float d[16], old[16];
            tc_ld16(tmem + ((unsigned)((warp & 3) * 32) << 16) + dcol + (unsigned)c0, d);
            float* p = pf;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                old[i] = (add && c0 + i < c_hi) ? *p : 0.f;   // add = 0: psi is stored, not read
                p += rs;
            }
            p = pf;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                if (c0 + i < c_hi) *p = old[i] + d[i];
                p += rs;
            }
            pf += 16 * rs;
        }
        tc_fence_before();
    };

    const unsigned idesc = tc_idesc_tf32(128, NP);
    bool ok = true;
    int last_issued = -1;
    if (T > 0) fetch_w(0);
    // step t: build A(t) and issue its MMAs into D[t % 2], then apply tile t - 1 from
    // D[(t - 1) % 2]; the MMAs of tile t - 1 (the last readers of A) are waited for first
    for (int t = 0; t <= T; t++) {
        if (tid == 0 && t >= 1 && !mbar_wait(bar, (t - 1) & 1, kTmaSpinLimit)) *abort_flag = 1;
        cp_async_wait<0>();
        __syncthreads();
        if (*abort_flag) {
            ok = false;
            break;
        }
        tc_fence_after();
        if (t < T) {
            // A row m = (site j, s, c) from Wraw, test vectors k = half, half + 2, ...: chunk
            // (m, k) at (m / 8) * SBO + k * 128 + (m % 8) * 16 (a warp writes four contiguous
            // 128-byte runs per k); Wraw word k * (kPtcWStride / 4) + j * 2 + s
            const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(wraw_p) + arow;
            unsigned char* ap = smraw_p + (m >> 3) * SBO + (m & 7) * 16;
            for (int k = half; k < ntest; k += 2) {
                const float2 w = __bfloat1622float2(wr[k * (kPtcWStride / 4)]);
                const float a0 = acm ? w.y : w.x, a1 = acm ? w.x : -w.y;
                *reinterpret_cast<float4*>(ap + k * 128) = asm_ ? make_float4(0.f, 0.f, a0, a1) : make_float4(a0, a1, 0.f, 0.f);
            }
            fence_async_smem();
            __syncthreads();
            if (t + 1 < T) fetch_w(t + 1);   // Wraw is free once A is built
            if (tid == 0) {
                tc_fence_after();
                for (int q = 0; q < KP / 8; q++)
                    tc_mma_tf32(tmem + (t & 1) * NP, tc_sdesc(sbase + q * 256, SBO),
                                tc_sdesc(sbase + a_bytes + q * 256, SBO), idesc, q > 0 ? 1u : 0u);
                tc_commit(bar);
            }
            last_issued = t;
        }
        if (t >= 1) apply(t - 1);
    }
    // an aborted step may leave the last tile's MMAs in flight: one more bounded wait
    if (!ok && tid == 0) {
        if (last_issued >= 0) mbar_wait(bar, last_issued & 1, kTmaSpinLimit);
        atomicOr(&g_fine_err, 2);
    }
    cp_async_wait_all();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, ncols);
}

}  // namespace amgb
