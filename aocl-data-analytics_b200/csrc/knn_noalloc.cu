// Brute-force euclidean k nearest neighbours for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not
// wanted -- inside a custom device allocator or memory-pool callback (which
// would recurse), real-time or safety-certified pipelines that forbid
// allocation after start-up, and host code whose device memory is fully
// reserved by another framework.  Such a caller already owns its inputs and
// outputs on the device; what the search needs beyond them is the per-chunk
// candidate lists, and those live here in one fixed array of device memory
// that belongs to the library.
//
// The array is a file-scope __device__ variable: every GPU on which this
// library's device code is loaded holds DA_B200_KNN_NOALLOC_SCRATCH_BYTES of
// it until the process exits.  All calls on a device share it, and each call
// overwrites what the previous one left there (every entry the merge reads is
// written first by the same call), so two calls whose work overlaps on the
// GPU (different streams, or different host threads without ordering) race
// on it and give wrong results.  The first call on each device looks up the
// array's device address (cudaGetSymbolAddress, with that device current);
// make that first call before any stream capture on the device.  The address
// belongs to the device's current context: when that context is replaced
// (cudaDeviceReset, or another primary context made current), the next call
// looks the address up again instead of using the old one.
#include "b200_kernels.hpp"
#include "../../include/aoclda_b200_ext.h"
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>

namespace {

__device__ __align__(256) unsigned char knn_noalloc_scratch[DA_B200_KNN_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
struct ScratchSlot {
    unsigned long long ctx_id; // unique id of the context the address belongs to
    void *addr;
};
ScratchSlot g_scratch[MAX_DEVICES] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

template <typename F> F driver_entry(const char *name) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<F>(p);
}

// Unique id of the calling thread's current context (0 when there is none).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_cur = driver_entry<CtxGetCurrentFn>("cuCtxGetCurrent");
    static CtxGetIdFn get_id = driver_entry<CtxGetIdFn>("cuCtxGetId");
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on the current device, looked up
// once per device and context.
cudaError_t scratch_address(int dev, void **out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    const unsigned long long id = current_context_id();
    if (!g_scratch[dev].addr || id == 0 || g_scratch[dev].ctx_id != id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, knn_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[dev].addr = p;
        // the lookup makes the device's primary context current if none was
        g_scratch[dev].ctx_id = current_context_id();
    }
    *out = g_scratch[dev].addr;
    return cudaSuccess;
}

} // namespace

extern "C" da_status da_b200_knn_euclidean_noalloc_s(const float *X, da_int n, const float *Q,
                                                     da_int nq, da_int d, da_int ld, da_int k,
                                                     float *dist, da_int *ind, void *stream) {
    using namespace b200;
    if (sizeof(da_int) != sizeof(int)) return da_status_not_implemented;
    if (!X || !Q || !dist || !ind) return da_status_invalid_pointer;
    if (n < 1 || nq < 1 || d < 1) return da_status_invalid_array_dimension;
    if (ld < d || ld % 4 != 0) return da_status_invalid_leading_dimension;
    if (((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Q)) & 15) != 0)
        return da_status_invalid_input;
    if (k < 1 || k > n || k > knn_max_k(false)) return da_status_invalid_input;
    // one candidate list (k keys + k indices) per query is the least the
    // search needs; beyond that the rows are split into fewer chunks
    const size_t per_chunk = (size_t)nq * k * (sizeof(float) + sizeof(int)) + 256;
    if (per_chunk > (size_t)DA_B200_KNN_NOALLOC_SCRATCH_BYTES)
        return da_status_invalid_array_dimension;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        cudaGetLastError();
        return da_status_arch_not_supported;
    }
    void *base = nullptr;
    if (scratch_address(dev, &base) != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);

    // chunking of the training rows (same plan as the handle path, capped by
    // the scratch capacity); the neighbours do not depend on it
    const int BN = knn_tile_rows_train(false);
    const int q_tiles = (int)((nq + 63) / 64);
    const int max_chunks = (int)((n + BN - 1) / BN);
    // enough CTAs to fill the GPU, but at most ~16K partial entries per query
    // (the merge ranks every entry against every chunk list)
    int n_chunks = std::max(1, std::min({max_chunks, (nsm * 8 + q_tiles - 1) / q_tiles,
                                         std::max(8, 16384 / (int)k)}));
    const int cap = (int)std::min<size_t>((size_t)DA_B200_KNN_NOALLOC_SCRATCH_BYTES / per_chunk,
                                          (size_t)max_chunks);
    n_chunks = std::max(1, std::min(n_chunks, cap));
    int chunk_rows = (int)((n + n_chunks - 1) / n_chunks);
    chunk_rows = ((chunk_rows + BN - 1) / BN) * BN;
    n_chunks = (int)((n + chunk_rows - 1) / chunk_rows);

    const size_t parts = (size_t)nq * n_chunks * k;
    float *part_key = static_cast<float *>(base);
    int *part_idx = reinterpret_cast<int *>(static_cast<unsigned char *>(base) +
                                            ((parts * sizeof(float) + 255) / 256) * 256);

    // metric "euclidean" of the handle path: direct differences in the
    // reference's accumulation order (256-wide blocks), sqrt on output
    KnnArgs a{ACC_SQEUC, POST_NONE, 256, 2.0, (int)k, chunk_rows, n_chunks};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = launch_knn_chunks<float>(Q, (int)ld, (int)nq, X, (int)ld, (int)n, (int)d,
                                             nullptr, nullptr, a, part_key, part_idx, nullptr, s);
    if (e == cudaSuccess)
        e = launch_knn_merge<float>(part_key, part_idx, (int)nq, n_chunks, (int)k, 1, dist,
                                    reinterpret_cast<int *>(ind), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    return da_status_success;
}
