// MEASUREMENT INFRASTRUCTURE ONLY (never part of the product).
//
// Times the reference's own GPU kernels, built from its kernels.cu for
// sm_100a, through the reference's own `struct CudaContext` (CudaContext.cpp,
// driver API, legacy default stream): the Config, AngularData and MeshData of
// a radiation.cfg are built by the reference's host code (the mesh through
// the meshProcessor stand-in in ref_stub/), then
//   computeLhs(f, Af)   (CudaContext.cpp:99-108: volumePart + surfacePart)
//   dot(x, y)           (CudaContext.cpp:186-198: one-block dotKern + DtoH)
// are launched back to back and timed with CUDA events on stream 0 after a
// warm-up.  Prints one line: lhs_ms=<ms per computeLhs> dot_ms=<ms per dot>
// nP=<> aslm=<>.  kernels.sm_100.cubin must sit in the working directory,
// as for the reference program.
//
//   ref_bench <radiation.cfg> [repetitions]
#include "AngularData.h"
#include "Config.h"
#include "CudaContext.h"
#include "MeshData.h"

#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#define CK(x)                                                                         \
    do {                                                                              \
        CUresult r_ = (x);                                                            \
        if (r_ != CUDA_SUCCESS) {                                                     \
            std::fprintf(stderr, "%s:%d: %s failed (%d)\n", __FILE__, __LINE__, #x, (int)r_); \
            return 2;                                                                 \
        }                                                                             \
    } while (0)

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <config-file> [repetitions]\n", argv[0]);
        return 1;
    }
    const int reps = argc > 2 ? std::atoi(argv[2]) : 50;
    Config cfg(argv[1]);
    AngularData ad(cfg.getMaxK());
    MeshData md(cfg);
    CudaContext *ctx = new CudaContext(cfg.getDevice(), md, ad);
    const idx N = ctx->N();
    REAL *b = ctx->allocVector();
    REAL *Af = ctx->allocVector();
    ctx->computeRhs(b);
    // a right-hand side is a vector with data in the l = 0 slots only; use
    // it as the operand (the kernels' cost does not depend on the values)
    CUevent e0, e1;
    CK(cuEventCreate(&e0, CU_EVENT_DEFAULT));
    CK(cuEventCreate(&e1, CU_EVENT_DEFAULT));
    for (int i = 0; i < 3; ++i) ctx->computeLhs(b, Af);
    CK(cuCtxSynchronize());
    CK(cuEventRecord(e0, 0));
    for (int i = 0; i < reps; ++i) ctx->computeLhs(b, Af);
    CK(cuEventRecord(e1, 0));
    CK(cuEventSynchronize(e1));
    float lhs_ms = 0.f;
    CK(cuEventElapsedTime(&lhs_ms, e0, e1));
    volatile double sink = 0.0;
    sink += ctx->dot(b, Af);
    CK(cuEventRecord(e0, 0));
    for (int i = 0; i < reps; ++i) sink += ctx->dot(b, Af);
    CK(cuEventRecord(e1, 0));
    CK(cuEventSynchronize(e1));
    float dot_ms = 0.f;
    CK(cuEventElapsedTime(&dot_ms, e0, e1));
    std::printf("lhs_ms=%.6f dot_ms=%.6f nP=%u aslm=%u N=%u\n", lhs_ms / reps, dot_ms / reps,
                (unsigned)md.nP, (unsigned)ctx->angdata->aslm, (unsigned)N);
    ctx->deviceFree(b);
    ctx->deviceFree(Af);
    delete ctx;
    return 0;
}
