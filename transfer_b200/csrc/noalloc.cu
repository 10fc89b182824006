// tr_dot_noalloc: the FP64 dot product of tr_dot without a context and
// without allocating device memory.
//
// Who needs it: a caller that may not call cudaMalloc at this point, for
// example a host application whose memory pool owns all device memory (a
// plugin host that hands in preallocated buffers), code running between the
// steps of a loop where cudaMalloc/cudaFree would synchronise the device, or
// a caller that has not created (and so has not allocated) a tr_ctx.  tr_dot
// needs a context, whose creation allocates the operator tables and the
// reduction scratch; this entry point needs neither.
//
// Scratch: the per-block partial sums and the arrival ticket of the
// deterministic grid reduction (reduce.cuh) live in the file-scope array
// g_dot_scratch below, kDotNoAllocMaxBlocks + 32 doubles (about 16 KiB).
// Every GPU that loads this library holds that array until the process
// exits.  The array is shared by every call on a device and keeps the last
// call's contents:
//   - the partial slots need no clearing (each block writes its own slot
//     before it takes a ticket);
//   - the ticket must be zero when a call starts: static device memory is
//     zero when the module loads, and the last block of every call sets it
//     back to zero;
//   - two calls whose kernels overlap on the GPU (other streams, other host
//     threads) race on the array and may return wrong sums: order them.
// In host code g_dot_scratch names a host-side stand-in, not device memory,
// so the host never passes it to a kernel: the first call on each device
// (with that device current) asks cudaGetSymbolAddress for the device
// address and keeps it.  That first call therefore does set-up work and
// should come before any stream capture on that device.
#include <atomic>
#include <mutex>
#include <string>

#include "internal.h"
#include "reduce.cuh"

namespace transfer {

tr_status set_global_error(tr_status st, const std::string &msg);  // capi.cpp

constexpr int kDotNoAllocPerThread = 64;                           // entries per thread
constexpr size_t kDotNoAllocChunk = size_t(kBlock) * kDotNoAllocPerThread;  // entries per block
constexpr int kDotNoAllocMaxBlocks = 2048;
constexpr size_t kDotNoAllocMaxEntries = kDotNoAllocChunk * kDotNoAllocMaxBlocks;  // 33,554,432
constexpr int kMaxDevices = 64;

// [0, kDotNoAllocMaxBlocks): block partials; slot kDotNoAllocMaxBlocks: the
// arrival ticket (an unsigned int in the first 4 bytes); the rest pads to 256 B.
static __device__ __align__(256) double g_dot_scratch[kDotNoAllocMaxBlocks + 32];

// Block b sums the entries [b * chunk, (b + 1) * chunk) with lm < slm; the
// partition depends only on n, so the result is the same bits on any GPU.
__global__ void __launch_bounds__(kBlock) k_dot_noalloc(size_t n, uint32_t aslm, uint32_t slm,
                                                        const double *__restrict__ x, const double *__restrict__ y,
                                                        double *partials, unsigned int *ticket, double *out) {
    const size_t base = blockIdx.x * kDotNoAllocChunk + threadIdx.x;
    double acc = 0.0;
#pragma unroll 8
    for (int k = 0; k < kDotNoAllocPerThread; ++k) {
        const size_t i = base + static_cast<size_t>(k) * kBlock;
        if (i < n && static_cast<uint32_t>(i % aslm) < slm) acc = fma(__ldg(x + i), __ldg(y + i), acc);
    }
    double v[1] = {acc}, tot[1];
    if (grid_reduce<1>(v, partials, ticket, tot) && threadIdx.x == 0) *out = tot[0];
}

static std::mutex g_setup_mutex;
static std::atomic<double *> g_scratch_addr[kMaxDevices];

// Device address of g_dot_scratch on the current device (looked up once).
static tr_status scratch_address(int dev, double **addr) {
    double *p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        p = g_scratch_addr[dev].load(std::memory_order_relaxed);
        if (!p) {
            cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_dot_scratch);
            if (e != cudaSuccess)
                return set_global_error(TR_ERR_CUDA, std::string("tr_dot_noalloc: cudaGetSymbolAddress: ") +
                                                         cudaGetErrorString(e));
            g_scratch_addr[dev].store(p, std::memory_order_release);
        }
    }
    *addr = p;
    return TR_OK;
}

// x, y, out must be device (or managed) memory that the current device reaches
static tr_status check_device_ptr(const void *p, int dev, const char *name) {
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_global_error(TR_ERR_INVALID_ARG, std::string("tr_dot_noalloc: ") + name +
                                                        " is not a CUDA pointer: " + cudaGetErrorString(e));
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
        return set_global_error(TR_ERR_INVALID_ARG,
                                std::string("tr_dot_noalloc: ") + name + " must point to device memory");
    if (at.type == cudaMemoryTypeDevice && at.device != dev)
        return set_global_error(TR_ERR_INVALID_ARG, std::string("tr_dot_noalloc: ") + name +
                                                        " is on device " + std::to_string(at.device) +
                                                        ", the current device is " + std::to_string(dev));
    if (reinterpret_cast<uintptr_t>(p) % alignof(double) != 0)
        return set_global_error(TR_ERR_INVALID_ARG,
                                std::string("tr_dot_noalloc: ") + name + " is not 8-byte aligned");
    return TR_OK;
}

}  // namespace transfer

using namespace transfer;

extern "C" tr_status tr_dot_noalloc(const double *x, const double *y, uint32_t nP, uint32_t aslm, uint32_t slm,
                                    double *out, void *stream) {
    if (!x || !y || !out) return set_global_error(TR_ERR_INVALID_ARG, "tr_dot_noalloc: null pointer");
    if (aslm == 0 || slm == 0 || slm > aslm)
        return set_global_error(TR_ERR_INVALID_ARG, "tr_dot_noalloc: need 0 < slm <= aslm");
    const size_t n = static_cast<size_t>(nP) * aslm;
    if (n > kDotNoAllocMaxEntries)
        return set_global_error(TR_ERR_INVALID_ARG,
                                "tr_dot_noalloc: nP * aslm = " + std::to_string(n) + " exceeds the maximum of " +
                                    std::to_string(kDotNoAllocMaxEntries) +
                                    " entries (its fixed scratch holds 2048 blocks of 16384 entries); use tr_dot");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return set_global_error(TR_ERR_NO_DEVICE, std::string("tr_dot_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return set_global_error(TR_ERR_UNSUPPORTED, "tr_dot_noalloc: device index beyond 63");
    tr_status st = check_device_ptr(x, dev, "x");
    if (st == TR_OK) st = check_device_ptr(y, dev, "y");
    if (st == TR_OK) st = check_device_ptr(out, dev, "out");
    if (st != TR_OK) return st;
    double *scratch = nullptr;
    st = scratch_address(dev, &scratch);
    if (st != TR_OK) return st;
    const int grid = n == 0 ? 1 : static_cast<int>((n + kDotNoAllocChunk - 1) / kDotNoAllocChunk);
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch + kDotNoAllocMaxBlocks);
    k_dot_noalloc<<<grid, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(n, aslm, slm, x, y, scratch, ticket, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_global_error(TR_ERR_CUDA, std::string("tr_dot_noalloc: launch: ") + cudaGetErrorString(e));
    return TR_OK;
}
