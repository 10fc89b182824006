// Moments of FP32 psi with TMA-staged tiles (moments_tc.cu): on the tcgen05
// tensor cores, or on paired FP32 FMAs.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace transfer {

// Dynamic shared memory of the kernel for nq ordinates.
size_t moments_tcgen05_smem(uint32_t nq);
// Whether the kernel takes this shape (M = 4 nT rows, nq ordinates).
bool moments_tcgen05_supported(uint32_t M, uint32_t nq);
// mom[n][r] = sum_q W[n][q] psi[q][r] for n < nmom (nmom <= 16), r < M, in
// split TF32 with FP32 accumulation.  psi: FP32 [nq][M] (16-byte aligned);
// W: FP64 [16][nq]; mom: FP64 [nmom][M]; err: one device word, bit 0 set if
// a pipeline wait of the kernel gave up (the caller clears it before).
cudaError_t launch_moments_tcgen05(const float *psi, uint32_t M, uint32_t nq, const double *W, int nmom,
                                   double *mom, unsigned int *err, int num_sms, cudaStream_t stream);
// The same product on paired FP32 FMAs (FFMA2), psi still loaded by TMA; the
// same arguments and error word.
bool moments_tma_ffma2_supported(uint32_t M, uint32_t nq);
cudaError_t launch_moments_tma_ffma2(const float *psi, uint32_t M, uint32_t nq, const double *W, int nmom,
                                     double *mom, unsigned int *err, int num_sms, cudaStream_t stream);

}  // namespace transfer
