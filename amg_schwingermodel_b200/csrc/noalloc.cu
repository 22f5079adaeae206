// amg_restrict_raw_noalloc: the level-0 restriction P^dagger v on caller-owned device memory,
// with its chunk partial sums kept in a fixed scratch array that this library owns instead of
// in memory it allocates.
//
// Who needs it: code that may not call cudaMalloc (or anything that allocates device memory
// behind its back) while it runs -- a host application whose device memory comes from its own
// pool and that forbids any other allocation, or a caller inside a region where an allocation
// would synchronise the device or fail.  Such callers pass the inputs and the output; the only
// extra device memory the restriction needs is the per-chunk partial sums, and here those live
// in g_restrict_scratch, a file-scope __device__ array that exists on every GPU that loads the
// library, from module load until the process exits.
#include <climits>
#include <cstdint>
#include <mutex>
#include <string>

#include "kernels.h"
#include "../../include/schwinger_amg.h"

namespace amgb {

namespace {

// 4 MiB of partial sums: nrhs * blocks * (2 * ntest) complex128 values with one chunk per
// block must fit, so e.g. 16 sources x 64 aggregates x 32 values or 1 source x 4096
// aggregates x 32 values.
constexpr long long kScratchBytes = 4ll << 20;
constexpr long long kScratchElems = kScratchBytes / (long long)sizeof(double2);
constexpr int kMaxDevices = 64;

// Every call on a device reuses this array and finds the previous call's partial sums in it.
// Nothing in it needs to start at zero: the chunk kernel writes every slot the summing kernel
// then reads, in the same call and on the same stream.
static __device__ __align__(256) double2 g_restrict_scratch[kScratchElems];

std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_restrict_scratch on the current device.  In host code the array's name
// refers to a host-side shadow, not to device memory, so the address is looked up once per
// device with that device current and kept for the life of the process.  A cudaDeviceReset
// unloads the module and makes the kept address stale: a process that resets a device must
// not call amg_restrict_raw_noalloc on it afterwards.
int scratch_address(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
        return AMG_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("device ordinal outside the scratch address table", __FILE__, __LINE__);
        return AMG_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_restrict_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "null scratch address", __FILE__, __LINE__);
            return AMG_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return AMG_OK;
}

int invalid(const char* msg) {
    set_last_error(msg, __FILE__, __LINE__);
    return AMG_ERR_INVALID;
}

bool aligned16(const void* p) { return (reinterpret_cast<std::uintptr_t>(p) & 15u) == 0; }

}  // namespace

}  // namespace amgb

using namespace amgb;

extern "C" AMG_API int amg_restrict_raw_noalloc(const void* W_dev, const void* v_dev, void* out_dev, int nx, int nt,
                                                int bx, int bt, int ntest, int nrhs, void* stream) {
    if (!W_dev || !v_dev || !out_dev) return invalid("null device pointer");
    if (!aligned16(W_dev) || !aligned16(v_dev) || !aligned16(out_dev))
        return invalid("device pointers must be 16-byte aligned (complex128 arrays)");
    if (nx < 2 || nt < 2) return invalid("lattice must be at least 2x2");
    if ((long long)nx * nt * 2 > INT_MAX) return invalid("nx * nt * 2 must fit in an int");
    if (bx < 1 || bt < 1 || nx % bx || nt % bt) return invalid("lattice not divisible into bx x bt aggregates");
    if (ntest < 1 || ntest > 32) return invalid("ntest must be in [1, 32]");
    if (nrhs < 1 || nrhs > 65535) return invalid("nrhs must be in [1, 65535]");
    const long long nblk = (long long)bx * bt;
    if (nblk > 65535) return invalid("at most 65535 aggregates");
    // one chunk per aggregate is the least scratch the partial sums can take
    const long long per_chunk = (long long)nrhs * nblk * 2 * ntest;
    if (per_chunk > kScratchElems)
        return invalid("nrhs * bx * bt * 2 * ntest * 16 bytes exceeds the 4 MiB restriction scratch");
    // the same chunking as the context's restriction, reduced until the partials fit
    const long long spb = (long long)(nx / bx) * (nt / bt);
    long long nchunk = std::max(1ll, std::min(std::max(1ll, spb / 128), (1184 + nblk - 1) / nblk));
    nchunk = std::min(nchunk, kScratchElems / per_chunk);

    // An error left pending by the caller's earlier work on this thread would be read back as
    // this call's launch status: report it as such, without clearing it, and launch nothing.
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        set_last_error((std::string("a CUDA error from earlier work is pending on this thread: ") +
                        cudaGetErrorString(e)).c_str(), __FILE__, __LINE__);
        return AMG_ERR_CUDA;
    }
    void* scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != AMG_OK) return rc;
    e = launch_restrict0<double, double2>(static_cast<const double2*>(W_dev), static_cast<const double2*>(v_dev),
                                          static_cast<double2*>(out_dev), static_cast<double2*>(scratch), nx, nt, bx,
                                          bt, ntest, nrhs, (int)nchunk, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();  // this call's own launch error: cleared once reported
        set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
        return AMG_ERR_CUDA;
    }
    return AMG_OK;
}
