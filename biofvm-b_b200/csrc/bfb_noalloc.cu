// bfb_noalloc.cu -- per-substrate field sums for callers that cannot allocate
// device memory.
//
// bfb_checksum works through a bfb_env, whose first checksum call allocates a
// small scratch buffer with cudaMalloc. Some callers cannot allow that: code
// that hands us a bare device field from its own memory pool, and host loops
// running other streams concurrently, where cudaMalloc and cudaFree would
// synchronize the whole device. bfb_checksum_noalloc runs the same two
// reduction kernels with their scratch in a fixed array compiled into this
// library instead, so it allocates nothing.
#include <mutex>

#include "bfb_aux.cuh"
#include "bfb_internal.cuh"

namespace {

constexpr int kNoallocBlocks = 296;  // reduction blocks (2 per SM of a B200)

// The scratch: kNoallocBlocks partial sums per substrate, for up to
// BFB_NOALLOC_MAX_SUBSTRATES substrates (296 * 64 * 8 B = 151.5 KB). Every
// GPU that loads the library holds one copy until the process exits. Each
// call first writes every slot it later reads, so nothing needs clearing; the
// array keeps the last call's partial sums. Calls that overlap on the GPU
// (different streams, no ordering between them) share it and race.
static __device__ __align__(256) double g_noalloc_partials[kNoallocBlocks * BFB_NOALLOC_MAX_SUBSTRATES];

// Host code may not take the array's address directly (its host-side name
// is a stand-in, not a device address); it is looked up once per device.
std::mutex g_mu;
double *g_partials_dev[64] = {nullptr};

int partials_for_current_device(double **out) {
    int dev = 0;
    BFB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return bfb::fail(BFB_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_partials_dev[dev]) {
        void *p = nullptr;
        BFB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
        g_partials_dev[dev] = static_cast<double *>(p);
    }
    *out = g_partials_dev[dev];
    return BFB_OK;
}

}  // namespace

extern "C" BFB_API int bfb_checksum_noalloc(const void *field_dev, int precision, long long n_voxels,
                                            int n_substrates, double *out_dev, void *stream) {
    if (!field_dev || !out_dev) return bfb::fail(BFB_ERR_INVALID_ARG, "field_dev and out_dev must not be NULL");
    if (precision != BFB_FP64 && precision != BFB_FP32)
        return bfb::fail(BFB_ERR_INVALID_ARG, "precision must be BFB_FP64 or BFB_FP32");
    if (n_voxels < 0 || n_substrates < 1) return bfb::fail(BFB_ERR_INVALID_ARG, "bad field size");
    if (n_substrates > BFB_NOALLOC_MAX_SUBSTRATES)
        return bfb::fail(BFB_ERR_SIZE, "bfb_checksum_noalloc: at most BFB_NOALLOC_MAX_SUBSTRATES (64) substrates");
    double *partials = nullptr;
    int st = partials_for_current_device(&partials);
    if (st) return st;
    return bfb::launch_checksum_raw(field_dev, precision, n_voxels, n_substrates, partials, kNoallocBlocks, out_dev,
                                    (cudaStream_t)stream);
}
