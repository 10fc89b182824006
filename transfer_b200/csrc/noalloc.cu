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
// so the host never passes it to a kernel: every call asks
// cudaGetSymbolAddress, with the caller's device current, for the array's
// device address in the current context.  The first call on a device loads
// this library's module there (set-up work), so that first call should come
// before any stream capture on that device.  Because the address is looked
// up again on each call, a cudaDeviceReset, or another CUDA context made
// current on the same device, between two calls leaves no stale address
// behind; the array's contents start at zero again in the new context.
#include <string>

#include "internal.h"
#include "reduce.cuh"

namespace transfer {

tr_status set_global_error(tr_status st, const std::string &msg);  // capi.cpp

constexpr int kDotNoAllocPerThread = 64;                           // entries per thread
constexpr size_t kDotNoAllocChunk = size_t(kBlock) * kDotNoAllocPerThread;  // entries per block
constexpr int kDotNoAllocMaxBlocks = 2048;
constexpr size_t kDotNoAllocMaxEntries = kDotNoAllocChunk * kDotNoAllocMaxBlocks;  // 33,554,432

// [0, kDotNoAllocMaxBlocks): block partials; slot kDotNoAllocMaxBlocks: the
// arrival ticket (an unsigned int in the first 4 bytes); the rest pads to 256 B.
static __device__ __align__(256) double g_dot_scratch[kDotNoAllocMaxBlocks + 32];

// Block b sums the entries [b * chunk, (b + 1) * chunk) with lm < slm; the
// partition depends only on n, so the result is the same bits on any GPU.
// n <= kDotNoAllocMaxEntries < 2^32, so indices are 32-bit; each thread
// finds its column (lm) once and steps it by kBlock modulo aslm.
__global__ void __launch_bounds__(kBlock) k_dot_noalloc(uint32_t n, uint32_t aslm, uint32_t slm,
                                                        const double *__restrict__ x, const double *__restrict__ y,
                                                        double *partials, unsigned int *ticket, double *out) {
    uint32_t i = blockIdx.x * static_cast<uint32_t>(kDotNoAllocChunk) + threadIdx.x;
    uint32_t lm = i % aslm;
    const uint32_t step = kBlock % aslm;
    double acc = 0.0;
#pragma unroll 8
    for (int k = 0; k < kDotNoAllocPerThread; ++k) {
        if (i < n && lm < slm) acc = fma(__ldg(x + i), __ldg(y + i), acc);
        i += kBlock;
        lm += step;
        if (lm >= aslm) lm -= aslm;
    }
    double v[1] = {acc}, tot[1];
    if (grid_reduce<1>(v, partials, ticket, tot) && threadIdx.x == 0) *out = tot[0];
}

// Device address of g_dot_scratch in the current context of the current
// device (looked up on every call: see the header comment).
static tr_status scratch_address(double **addr) {
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_dot_scratch);
    if (e != cudaSuccess || !p)
        return set_global_error(TR_ERR_CUDA, std::string("tr_dot_noalloc: cudaGetSymbolAddress: ") +
                                                 cudaGetErrorString(e));
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
    tr_status st = check_device_ptr(x, dev, "x");
    if (st == TR_OK) st = check_device_ptr(y, dev, "y");
    if (st == TR_OK) st = check_device_ptr(out, dev, "out");
    if (st != TR_OK) return st;
    double *scratch = nullptr;
    st = scratch_address(&scratch);
    if (st != TR_OK) return st;
    const int grid = n == 0 ? 1 : static_cast<int>((n + kDotNoAllocChunk - 1) / kDotNoAllocChunk);
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch + kDotNoAllocMaxBlocks);
    k_dot_noalloc<<<grid, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<uint32_t>(n), aslm, slm, x, y, scratch, ticket, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_global_error(TR_ERR_CUDA, std::string("tr_dot_noalloc: launch: ") + cudaGetErrorString(e));
    return TR_OK;
}
