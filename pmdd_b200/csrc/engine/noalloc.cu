// Allocation-free variant of the standalone Pareto filter (pmdd_pareto_filter).
//
// Some callers cannot allocate device memory at all: host libraries embedded in a
// framework whose caching allocator has already reserved the device's memory (a
// cudaMalloc beside it fails or fragments that pool), and latency-bound services that
// forbid allocation after start-up, because cudaMalloc and cudaFree can synchronise
// the device and stall every stream on it.  They own their input and output buffers
// already; what they cannot do is obtain the filter's scratch space.  This entry
// point takes that scratch from a fixed, file-scope device array instead of the
// engine's arena, and allocates nothing -- no cudaMalloc, no cudaFree, no engine.
//
// Limits and sharing:
//  * at most kNoAllocMaxPoints points of at most 8 objectives per call (larger inputs
//    are rejected with PMDD_ERR_RANGE);
//  * the scratch array (about 9.4 MB) exists on every device that loads this library,
//    for the life of the process;
//  * every call on a device uses the same array, and it keeps the last call's
//    contents: the kernel writes every scratch word it later reads, so nothing needs
//    clearing between calls, but calls that overlap on the GPU (two host threads, or
//    two streams without ordering between them) race on the array and corrupt each
//    other's results -- serialise them;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call before any
//    stream capture begins;
//  * the call copies the result count to the host and synchronises `stream` before it
//    returns.
#include <mutex>

#include "pareto.cuh"
#include "pmdd.h"

namespace {

constexpr int64_t kNoAllocMaxPoints = 1 << 17;
constexpr int kNoAllocMaxObjs = 8;
constexpr int kMaxDevices = 64;

// Scratch of the largest allowed call, plus room for the device-side result count.
constexpr size_t kScratchBytes = (2 * ((kNoAllocMaxPoints * kNoAllocMaxObjs * 4 + 255) / 256 * 256) +
                                  2 * ((kNoAllocMaxPoints * 4 + 255) / 256 * 256));
constexpr size_t kCountOffset = kScratchBytes;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes + 256];

std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

void put_err(char *err, size_t errlen, const char *msg) {
    if (!err || errlen == 0) return;
    size_t i = 0;
    for (; msg[i] && i + 1 < errlen; ++i) err[i] = msg[i];
    err[i] = '\0';
}

}  // namespace

extern "C" int pmdd_pareto_filter_noalloc(const int32_t *d_points, int64_t num_points, int32_t nobjs,
                                          int32_t *d_out, int64_t *out_points, void *stream, char *err,
                                          size_t errlen) {
    if (out_points) *out_points = 0;
    if (nobjs < 1 || nobjs > kNoAllocMaxObjs || num_points < 0 || !out_points ||
        (num_points > 0 && (!d_points || !d_out))) {
        put_err(err, errlen, "invalid arguments (nobjs 1..8, num_points >= 0, non-NULL buffers)");
        return PMDD_ERR_INVALID;
    }
    if (num_points > kNoAllocMaxPoints) {
        put_err(err, errlen, "point set exceeds the allocation-free limit of 131072 points; use pmdd_pareto_filter");
        return PMDD_ERR_RANGE;
    }
    if (num_points == 0) return PMDD_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        put_err(err, errlen, "no usable current CUDA device");
        return PMDD_ERR_NO_DEVICE;
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_ptr[dev]) {
            // one-time set-up on this device: the device address of the static array
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                put_err(err, errlen, "cudaGetSymbolAddress of the allocation-free scratch failed");
                return PMDD_ERR_CUDA;
            }
            g_scratch_ptr[dev] = p;
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t *d_count = reinterpret_cast<int64_t *>(static_cast<unsigned char *>(scratch) + kCountOffset);
    cudaError_t e = pmdd::dev::launch_pareto_filter(nobjs, d_points, num_points, scratch, d_out, d_count, st);
    int64_t n_out = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n_out, d_count, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        put_err(err, errlen, cudaGetErrorString(e));
        return PMDD_ERR_CUDA;
    }
    *out_points = n_out;
    return PMDD_OK;
}
