// Set-up kernels: the fine level's hop matrices, the Galerkin coarse links
// (Level::makeCoarseLinks, src/level.cpp:242-301) and the aggregate-wise
// orthonormalisation of the test vectors (Level::orthonormalize, src/level.cpp:373-417).
#include "kernels.h"

namespace amgb {

// Level::makeDirac (src/level.cpp:87-125) as dense 2x2 hop matrices, stored like the
// coarse links: hops[n][h][j][i] = G_h[n](row i, col j), h = self, R0, R1, L0, L1.
//   R_mu = 1/2 (1 - sigma_mu) U_mu(n),  L_mu = 1/2 (1 + sigma_mu) conj(U_mu(n - mu)),  self = 0
template <typename T>
__global__ void k_fine_hops(const cx<T>* __restrict__ U, cx<T>* __restrict__ hops, int nx, int nt) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nx * nt) return;
    const int x = n / nt, t = n - x * nt;
    const int l0 = x * nt + ((t == 0) ? nt - 1 : t - 1);
    const int l1 = ((x == 0) ? nx - 1 : x - 1) * nt + t;
    const cx<T> u0 = U[2 * n], u1 = U[2 * n + 1];
    const cx<T> c0 = cconj(U[2 * l0]), c1 = cconj(U[2 * l1 + 1]);
    const T h = T(0.5);
    cx<T>* o = hops + (long long)n * 20;
    // index: h*4 + j*2 + i  (column j, row i)
    for (int k = 0; k < 4; k++) o[k] = czero<T>();
    // M0 = [[1,-1],[-1,1]]
    o[4 + 0] = h * u0; o[4 + 1] = -h * u0; o[4 + 2] = -h * u0; o[4 + 3] = h * u0;
    // M1 = [[1, i],[-i, 1]]: (0,0)=1, (1,0)=-i, (0,1)=i, (1,1)=1
    o[8 + 0] = h * u1; o[8 + 1] = -h * cmuli(u1); o[8 + 2] = h * cmuli(u1); o[8 + 3] = h * u1;
    // P0 = [[1,1],[1,1]]
    o[12 + 0] = h * c0; o[12 + 1] = h * c0; o[12 + 2] = h * c0; o[12 + 3] = h * c0;
    // P1 = [[1,-i],[i,1]]: (0,0)=1, (1,0)=i, (0,1)=-i, (1,1)=1
    o[16 + 0] = h * c1; o[16 + 1] = h * cmuli(c1); o[16 + 2] = -h * cmuli(c1); o[16 + 3] = h * c1;
}

// Galerkin links for level l+1 from level l (src/level.cpp:242-301).  For coarse site nc
// and every fine site n of its block and every hop h of n: the contribution
//   C[(2p+alf),(2s+bet)] += sum_{c,b} conj(W_p[n][2c+alf]) G_h[n][(2c+alf),(2b+bet)] W_s[nbr][2b+bet]
// goes to A (self) when nbr lies in the same block, to B_mu / C_mu when it lies in the
// coarse right / left neighbour block, and nowhere otherwise.  No sign is applied.
// Grid: (chunk, nc).  Output partial[nc][chunk][cat][jj][ii].
template <typename T, int EPT>
__global__ void __launch_bounds__(256) k_coarse_links(const cx<T>* __restrict__ W, const cx<T>* __restrict__ hops,
                                                      cx<T>* __restrict__ partial, int nx, int nt, int K, int bx,
                                                      int bt, int ntest, int nchunk, int tile, int entry0) {
    extern __shared__ __align__(16) unsigned char smraw_c[];
    const int nc = blockIdx.y, chunk = blockIdx.x;
    const int xe = nx / bx, te = nt / bt, spb = xe * te;
    const int Kc = 2 * ntest, nout = 5 * Kc * Kc;
    const int cbx = nc / bt, cbt = nc - cbx * bt;
    const int N = nx * nt;
    const int per = (spb + nchunk - 1) / nchunk;
    const int q0 = chunk * per, q1 = min(spb, q0 + per);
    // smem: Y[tile][5][K][ntest][2], cat[tile][5], nsite[tile]
    const int ysz = 5 * K * ntest * 2;
    cx<T>* Y = reinterpret_cast<cx<T>*>(smraw_c);
    int* cat = reinterpret_cast<int*>(Y + (long long)tile * ysz);
    int* nsite = cat + tile * 5;
    cx<T> acc[EPT];
#pragma unroll
    for (int k = 0; k < EPT; k++) acc[k] = czero<T>();
    // coarse neighbours of nc (RightPB_l / LeftPB_l of level l+1)
    const int cr0 = cbx * bt + ((cbt + 1 == bt) ? 0 : cbt + 1);
    const int cr1 = ((cbx + 1 == bx) ? 0 : cbx + 1) * bt + cbt;
    const int cl0 = cbx * bt + ((cbt == 0) ? bt - 1 : cbt - 1);
    const int cl1 = ((cbx == 0) ? bx - 1 : cbx - 1) * bt + cbt;
    for (int qb = q0; qb < q1; qb += tile) {
        const int nts = min(tile, q1 - qb);
        // categories and site indices
        for (int k = threadIdx.x; k < nts * 5; k += blockDim.x) {
            const int ts = k / 5, h = k - ts * 5;
            const int q = qb + ts, mx = q / te, mt = q - mx * te;
            const int x = cbx * xe + mx, t = cbt * te + mt;
            const int n = x * nt + t;
            const int nb = nb_site(x, t, nx, nt, h);
            const int nbx = nb / nt, nbt = nb - nbx * nt;
            const int blk = (nbx / xe) * bt + (nbt / te);
            int c = -1;
            if (h == HOP_SELF) c = 0;
            else if (blk == nc) c = 0;
            else if (h == HOP_R0 && blk == cr0) c = 1;
            else if (h == HOP_R1 && blk == cr1) c = 2;
            else if (h == HOP_L0 && blk == cl0) c = 3;
            else if (h == HOP_L1 && blk == cl1) c = 4;
            cat[k] = c;
            if (h == 0) nsite[ts] = n;
        }
        __syncthreads();
        // Y[ts][h][i][s][bet] = sum_b G_h[n](i, 2b+bet) W_s[nbr][2b+bet]
        const int ytot = nts * ysz;
        for (int e = threadIdx.x; e < ytot; e += blockDim.x) {
            const int ts = e / ysz;
            int r = e - ts * ysz;
            const int h = r / (K * ntest * 2);
            r -= h * (K * ntest * 2);
            const int i = r / (ntest * 2);
            r -= i * (ntest * 2);
            const int s = r >> 1, bet = r & 1;
            cx<T> y = czero<T>();
            if (cat[ts * 5 + h] >= 0) {
                const int n = nsite[ts];
                const int x = n / nt, t = n - x * nt;
                const int nb = nb_site(x, t, nx, nt, h);
                const cx<T>* G = hops + ((long long)n * 5 + h) * K * K;
                const cx<T>* ws = W + ((long long)s * N + nb) * K;
                for (int b = 0; b < K / 2; b++) cfma(y, G[(2 * b + bet) * K + i], ws[2 * b + bet]);
            }
            Y[e] = y;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < EPT; k++) {
            const int o = entry0 + threadIdx.x + k * blockDim.x;
            if (o >= nout) break;
            const int c = o / (Kc * Kc);
            int r = o - c * Kc * Kc;
            const int jj = r / Kc, ii = r - jj * Kc;
            const int s = jj >> 1, bet = jj & 1, p = ii >> 1, alf = ii & 1;
            for (int ts = 0; ts < nts; ts++) {
                const int n = nsite[ts];
                const cx<T>* wp = W + ((long long)p * N + n) * K;
                for (int h = 0; h < 5; h++) {
                    if (cat[ts * 5 + h] != c) continue;
                    const cx<T>* y = Y + (long long)ts * ysz + (long long)h * K * ntest * 2;
                    for (int cc = 0; cc < K / 2; cc++)
                        cfmac(acc[k], wp[2 * cc + alf], y[((2 * cc + alf) * ntest + s) * 2 + bet]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        const int o = entry0 + threadIdx.x + k * blockDim.x;
        if (o >= nout) break;
        partial[((long long)nc * nchunk + chunk) * nout + o] = acc[k];
    }
}

template <typename T>
__global__ void k_sum_chunks(const cx<T>* __restrict__ partial, cx<T>* __restrict__ out, int nout, int nchunk,
                             int nblk) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= (long long)nblk * nout) return;
    const long long nc = o / nout, e = o - nc * nout;
    cx<T> s = czero<T>();
    for (int c = 0; c < nchunk; c++) s += partial[(nc * nchunk + c) * nout + e];
    out[o] = s;
}

// Level::orthonormalize (src/level.cpp:373-417): one CTA per aggregate a = 2*block + spin,
// modified Gram-Schmidt over the Ntest pieces in the reference's order.
template <typename T>
__global__ void __launch_bounds__(256) k_orthonormalize(cx<T>* __restrict__ W, int nx, int nt, int K, int bx, int bt,
                                                        int ntest) {
    __shared__ T red[2 * 8 + 2];
    const int a = blockIdx.x, nc = a >> 1, s = a & 1;
    const int xe = nx / bx, te = nt / bt, col = K / 2, nel = xe * te * col;
    const int cbx = nc / bt, cbt = nc - cbx * bt;
    const long long N = (long long)nx * nt;
    auto idx = [&](int e) -> long long {
        const int q = e / col, c = e - q * col;
        const int mx = q / te, mt = q - mx * te;
        const long long n = (long long)(cbx * xe + mx) * nt + (cbt * te + mt);
        return n * K + 2 * c + s;
    };
    for (int ntv = 0; ntv < ntest; ntv++) {
        cx<T>* wn = W + (long long)ntv * N * K;
        for (int ntt = 0; ntt < ntv; ntt++) {
            const cx<T>* wt = W + (long long)ntt * N * K;
            T px = 0, py = 0;
            for (int e = threadIdx.x; e < nel; e += blockDim.x) {
                const long long i = idx(e);
                const cx<T> u = wn[i], v = wt[i];
                px += u.x * v.x + u.y * v.y;
                py += u.y * v.x - u.x * v.y;
            }
            px = cta_sum(px, red);
            py = cta_sum(py, red + 9);
            const cx<T> proj = mk<T>(px, py);
            for (int e = threadIdx.x; e < nel; e += blockDim.x) {
                const long long i = idx(e);
                cx<T> u = wn[i];
                cfma(u, -proj, wt[i]);
                wn[i] = u;
            }
            __syncthreads();
        }
        T nn = 0;
        for (int e = threadIdx.x; e < nel; e += blockDim.x) nn += cnorm2(wn[idx(e)]);
        nn = cta_sum(nn, red);
        const T inv = T(1) / sqrt(nn);
        for (int e = threadIdx.x; e < nel; e += blockDim.x) {
            const long long i = idx(e);
            wn[i] = inv * wn[i];
        }
        __syncthreads();
    }
}

template <typename T>
void launch_fine_hops(const cx<T>* U, cx<T>* hops, int nx, int nt, cudaStream_t s) {
    count_launch(1);
    k_fine_hops<T><<<(nx * nt + 255) / 256, 256, 0, s>>>(U, hops, nx, nt);
}

template <typename T>
void launch_coarse_links(const cx<T>* W, const cx<T>* hops, cx<T>* out, int nx, int nt, int K, int bx, int bt,
                         int ntest, cx<T>* partial, int nchunk, cudaStream_t s) {
    count_launch(1);
    constexpr int EPT = 20;
    const int Kc = 2 * ntest, nout = 5 * Kc * Kc;
    const int ysz_bytes = 5 * K * ntest * 2 * (int)sizeof(cx<T>);
    int tile = (64 * 1024) / ysz_bytes;
    if (tile < 1) tile = 1;
    if (tile > 16) tile = 16;
    const int smem = tile * ysz_bytes + tile * 6 * 4 + 64;
    cudaFuncSetAttribute(k_coarse_links<T, EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int nblk = bx * bt;
    dim3 grid(nchunk, nblk);
    for (int e0 = 0; e0 < nout; e0 += 256 * EPT)
    {
        k_coarse_links<T, EPT><<<grid, 256, smem, s>>>(W, hops, partial, nx, nt, K, bx, bt, ntest, nchunk, tile, e0);
        count_launch(1);
    }
    const long long tot = (long long)nblk * nout;
    k_sum_chunks<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(partial, out, nout, nchunk, nblk);
}

template <typename T>
void launch_orthonormalize(cx<T>* W, int nx, int nt, int K, int bx, int bt, int ntest, cudaStream_t s) {
    count_launch(1);
    k_orthonormalize<T><<<2 * bx * bt, 256, 0, s>>>(W, nx, nt, K, bx, bt, ntest);
}

template void launch_fine_hops<double>(const cx<double>*, cx<double>*, int, int, cudaStream_t);
template void launch_fine_hops<float>(const cx<float>*, cx<float>*, int, int, cudaStream_t);
template void launch_coarse_links<double>(const cx<double>*, const cx<double>*, cx<double>*, int, int, int, int, int,
                                          int, cx<double>*, int, cudaStream_t);
template void launch_orthonormalize<double>(cx<double>*, int, int, int, int, int, int, cudaStream_t);
template void launch_orthonormalize<float>(cx<float>*, int, int, int, int, int, int, cudaStream_t);

}  // namespace amgb
