// fx_noalloc.cu -- an FP64 dot product that allocates no device memory.
//
// fx_dot needs scratch in device memory for its per-block partial sums, and takes it from
// the context, which allocates it with cudaMalloc.  Some callers cannot let a library do
// that: a host application that owns all device memory through its own pool and accounts
// for every byte, or a latency-critical loop that must never reach the allocator.  For them
// fx_dot_f64_noalloc runs the same compensated, deterministic reduction kernel with its
// scratch in a fixed, file-scope __device__ array that is loaded with the library.
//
// Limits and behaviour:
//  - at most kNoAllocMaxN = 8,388,608 elements per call (4096 blocks of 2048 elements; the
//    array holds one partial pair per block, 64 KiB, plus the result and a counter);
//    larger n is rejected with FX_ERR_INVALID_ARGUMENT;
//  - every GPU that loads the library holds the array until the process exits;
//  - all calls share the array: calls whose kernels overlap on the GPU (different streams,
//    or different host threads on one device) race and must be serialised by the caller;
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//    with that device current; make that first call before any stream capture begins;
//  - that address is kept for the life of the process: calls after a reset of the device's
//    primary context (cudaDeviceReset, by this process or a library in it) are not supported.
#include <mutex>

#include "fx_internal.cuh"

namespace {

constexpr int kNoAllocBlocks = 4096;
constexpr size_t kNoAllocTile = 8 * (size_t)fx::kBlock;  // elements per block
constexpr size_t kNoAllocMaxN = kNoAllocBlocks * kNoAllocTile;
// layout of the scratch array: [0, 2*blocks) partial (sum, compensation) pairs,
// [2*blocks] the result, [2*blocks + 1] the last-block ticket counter (as an unsigned)
constexpr int kResultSlot = 2 * kNoAllocBlocks;
constexpr int kCounterSlot = 2 * kNoAllocBlocks + 1;

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocBlocks + 2];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_lock;
double *g_noalloc_addr[kMaxDevices] = {};

struct NaDot {
    const double *x, *y;
    __device__ __forceinline__ void operator()(size_t i, fx::CSum *acc) const {
        fx::csum_add_prod(acc[0], x[i], y[i]);
    }
};

// In host code g_noalloc_scratch names a host-side stand-in, not device memory; the kernel
// gets the device address resolved here, once per device, with that device current.
int scratch_address(double **out) {
    int dev = 0;
    FX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fx::fail(FX_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> g(g_noalloc_lock);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        FX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = (double *)p;
    }
    *out = g_noalloc_addr[dev];
    return FX_OK;
}

}  // namespace

extern "C" int fx_dot_f64_noalloc(const double *x, const double *y, size_t n, double *out, void *stream) {
    if (!out || (n && (!x || !y))) return fx::fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (n > kNoAllocMaxN)
        return fx::fail(FX_ERR_INVALID_ARGUMENT, "fx_dot_f64_noalloc: n = " + std::to_string(n) +
                                                     " exceeds the static scratch limit of " +
                                                     std::to_string(kNoAllocMaxN) + " elements");
    if (n == 0) {
        *out = 0.0;
        return FX_OK;
    }
    double *s = nullptr;
    FX_TRY(scratch_address(&s));
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *counter = reinterpret_cast<unsigned *>(s + kCounterSlot);
    // the ticket counter must start at zero (every completed call leaves it at zero)
    FX_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
    const int blocks = (int)((n + kNoAllocTile - 1) / kNoAllocTile);
    fx::k_flat<1><<<blocks, fx::kBlock, 0, st>>>(n, NaDot{x, y}, fx::StoreFin<1>{s + kResultSlot},
                                                 fx::RedArgs<1>{s, counter}, nullptr);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fx::fail(FX_ERR_BACKEND, std::string("fx_dot_f64_noalloc: ") + cudaGetErrorString(e));
    FX_CUDA(cudaMemcpyAsync(out, s + kResultSlot, sizeof(double), cudaMemcpyDeviceToHost, st));
    FX_CUDA(cudaStreamSynchronize(st));
    return FX_OK;
}
