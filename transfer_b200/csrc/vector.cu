// Vector kernels: BLAS-1 (scaleKern/addProdKern/mulAddKern/mulAddProdKern,
// kernels.cu:12-50), reductions (normKern/dotKern, kernels.cu:55-115) as
// grid-wide deterministic reductions instead of the reference's single
// 128-thread block, the fused CG update steps, the FP32 <-> FP64 transfers
// of the defect-correction solve, and the moment / flux reductions
// (MeshData::ComputeMoments / ComputeFlux, MeshData.cpp:96-136).
#include <cmath>

#include "internal.h"
#include "reduce.cuh"

namespace transfer {

// x = wx*x + wy*y over all n entries (padding included, as the reference).
__global__ void __launch_bounds__(kBlock) k_blas(size_t n, int op, double *__restrict__ x,
                                                 const double *__restrict__ y, double wx, double wy) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        switch (op) {
        case BLAS_SCALE: x[i] *= wx; break;
        case BLAS_ADD_PROD: x[i] += wy * y[i]; break;
        case BLAS_MUL_ADD: x[i] = wx * x[i] + y[i]; break;
        default: x[i] = wx * x[i] + wy * y[i]; break;
        }
    }
}

// <x, y> over vertices and lm < slm, in double.
template <typename TX, typename TY>
__global__ void __launch_bounds__(kBlock) k_dot(size_t n, uint32_t aslm, uint32_t slm, const TX *__restrict__ x,
                                                const TY *__restrict__ y, double *partials, unsigned int *counter,
                                                double *out) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        if (static_cast<uint32_t>(i % aslm) < slm) acc += static_cast<double>(x[i]) * static_cast<double>(y[i]);
    double v[1] = {acc}, tot[1];
    if (grid_reduce<1>(v, partials, counter, tot) && threadIdx.x == 0) *out = tot[0];
}

// 16-byte vectors of T and component access (indices are compile-time
// constants after unrolling)
template <typename T>
struct VecT;
template <>
struct VecT<double> {
    typedef double2 V;
    static constexpr int W = 2;
    __device__ static double get(const V &v, int k) { return k == 0 ? v.x : v.y; }
    __device__ static void set(V &v, int k, double a) {
        if (k == 0) v.x = a;
        else v.y = a;
    }
};
template <>
struct VecT<float> {
    typedef float4 V;
    static constexpr int W = 4;
    __device__ static float get(const V &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
    __device__ static void set(V &v, int k, float a) {
        if (k == 0) v.x = a;
        else if (k == 1) v.y = a;
        else if (k == 2) v.z = a;
        else v.w = a;
    }
};

// CG update (main.cpp:144-154): f += alpha p; r -= alpha Ap; optional
// Jacobi z = D^-1 r; then, in the last block, the stop test on ||r||, the
// residual history and beta = (r,z)_new / (r,z)_old.  n is in 16-byte
// vectors (aslm is a multiple of the vector width, so a vector never
// straddles two vertices).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_cg_update(size_t nvec, uint32_t aslm, uint32_t slm, T *__restrict__ f,
                                                      T *__restrict__ r, const T *__restrict__ p,
                                                      const T *__restrict__ Ap, T *__restrict__ z,
                                                      const T *__restrict__ dinv, CgScalars *s, double *partials,
                                                      unsigned int *counter, double *hist, int hist_cap,
                                                      int defer_beta) {
    if (s->done) return;
    typedef VecT<T> O;
    typedef typename O::V V;
    const T alpha = static_cast<T>(s->alpha);
    double rr = 0.0, rz = 0.0;
    for (size_t iv = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; iv < nvec;
         iv += static_cast<size_t>(gridDim.x) * blockDim.x) {
        V fv = reinterpret_cast<const V *>(f)[iv], rv = reinterpret_cast<const V *>(r)[iv];
        const V pv = reinterpret_cast<const V *>(p)[iv], av = reinterpret_cast<const V *>(Ap)[iv];
        V dv, zv;
        if (dinv) dv = reinterpret_cast<const V *>(dinv)[iv];
        const uint32_t lm0 = static_cast<uint32_t>((iv * O::W) % aslm);
#pragma unroll
        for (int k = 0; k < O::W; ++k) {
            O::set(fv, k, fma(alpha, O::get(pv, k), O::get(fv, k)));
            const T ri = fma(-alpha, O::get(av, k), O::get(rv, k));
            O::set(rv, k, ri);
            const bool live = lm0 + k < slm;
            if (dinv) {
                const T zi = O::get(dv, k) * ri;
                O::set(zv, k, zi);
                if (live) rz += static_cast<double>(ri) * static_cast<double>(zi);
            }
            if (live) rr += static_cast<double>(ri) * static_cast<double>(ri);
        }
        reinterpret_cast<V *>(f)[iv] = fv;
        reinterpret_cast<V *>(r)[iv] = rv;
        if (dinv) reinterpret_cast<V *>(z)[iv] = zv;
    }
    double v[2] = {rr, rz}, tot[2];
    if (grid_reduce<2>(v, partials, counter, tot) && threadIdx.x == 0) {
        const double nr = sqrt(tot[0]);
        const int k = s->k;
        if (hist && k < hist_cap) hist[k] = nr;
        int done = 0;
        if (!isfinite(nr)) done = 3;
        else if (nr < s->tol) done = 1;
        else if (k + 1 >= s->maxit) done = 2;
        const double rznew = dinv ? tot[1] : tot[0];
        if (!done && !defer_beta) {
            s->beta = rznew / s->nrz;
            s->nrz = rznew;
        }
        s->rr = tot[0];
        s->k = k + 1;
        s->done = done;
    }
}

// p = beta p + z (mulAdd, main.cpp:158)
template <typename T>
__global__ void __launch_bounds__(kBlock) k_cg_direction(size_t n, T *__restrict__ p, const T *__restrict__ z,
                                                         const CgScalars *s) {
    if (s->done) return;
    const T beta = static_cast<T>(s->beta);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        p[i] = fma(beta, p[i], z[i]);
}

// CG start: r = b - A f0 is r = b for f0 = 0; z = D^-1 r or r; nrz = (r, z);
// p = z, or, for the fused-direction iteration, p = 0 with beta = 0 (the
// first operator launch then forms p = z + 0 p).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_cg_start(size_t n, uint32_t aslm, uint32_t slm, const T *__restrict__ b,
                                                     T *__restrict__ f, T *__restrict__ r, T *__restrict__ z,
                                                     T *__restrict__ p, const T *__restrict__ dinv, CgScalars *s,
                                                     double *partials, unsigned int *counter, int zero_p) {
    double rz = 0.0, bb = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const T bi = b[i];
        f[i] = T(0);
        r[i] = bi;
        const T zi = dinv ? dinv[i] * bi : bi;
        if (dinv) z[i] = zi;
        p[i] = zero_p ? T(0) : zi;
        if (static_cast<uint32_t>(i % aslm) < slm) {
            rz += static_cast<double>(bi) * static_cast<double>(zi);
            bb += static_cast<double>(bi) * static_cast<double>(bi);
        }
    }
    double v[2] = {rz, bb}, tot[2];
    if (grid_reduce<2>(v, partials, counter, tot) && threadIdx.x == 0) {
        s->nrz = tot[0];
        s->rr = tot[1];
        s->beta = 0.0;
        s->k = 0;
        s->done = (tot[0] == 0.0) ? 1 : 0;
    }
}

// Reliable update of the FP32 CG of the mixed mode (after x64 += scale d and
// an FP64 residual): r holds the new true residual in its new scale; the
// correction d restarts at 0, z = D^-1 r (or r), and the CG continues with
// its last direction p: beta = (r, z)_new / (r, z)_old * ratio, where ratio
// = new scale / old scale carries p into the new scale (see solve_mixed).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_cg_reliable(size_t n, uint32_t aslm, uint32_t slm, T *__restrict__ f,
                                                        const T *__restrict__ r, T *__restrict__ z,
                                                        const T *__restrict__ dinv, CgScalars *s, double ratio,
                                                        double *partials, unsigned int *counter) {
    double rz = 0.0, rr = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const T ri = r[i];
        f[i] = T(0);
        const T zi = dinv ? dinv[i] * ri : ri;
        if (dinv) z[i] = zi;
        if (static_cast<uint32_t>(i % aslm) < slm) {
            rz += static_cast<double>(ri) * static_cast<double>(zi);
            rr += static_cast<double>(ri) * static_cast<double>(ri);
        }
    }
    double v[2] = {rz, rr}, tot[2];
    if (grid_reduce<2>(v, partials, counter, tot) && threadIdx.x == 0) {
        s->beta = (s->nrz != 0.0) ? tot[0] / s->nrz * ratio : 0.0;
        s->nrz = tot[0];
        s->rr = tot[1];
        s->done = (tot[0] == 0.0) ? 1 : 0;
    }
}

// Defect correction: r = b - Ax in FP64 with ||r||^2 -> s->rr, s->scale.
__global__ void __launch_bounds__(kBlock) k_residual(size_t n, uint32_t aslm, uint32_t slm,
                                                     const double *__restrict__ b, const double *__restrict__ Ax,
                                                     double *__restrict__ r, CgScalars *s, double *partials,
                                                     unsigned int *counter) {
    double rr = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const double ri = b[i] - Ax[i];
        r[i] = ri;
        if (static_cast<uint32_t>(i % aslm) < slm) rr += ri * ri;
    }
    double v[1] = {rr}, tot[1];
    if (grid_reduce<1>(v, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->scale = sqrt(tot[0]);
    }
}

// r32[v][lm] = r64[v][lm] / scale   (aslm -> aslm32 re-padding)
__global__ void __launch_bounds__(kBlock) k_to_f32(uint32_t nP, uint32_t slm, uint32_t aslm, uint32_t aslm32,
                                                   const double *__restrict__ r64, float *__restrict__ r32,
                                                   const CgScalars *s) {
    const double inv = (s->scale > 0.0) ? 1.0 / s->scale : 0.0;
    const size_t n = static_cast<size_t>(nP) * aslm32;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t v = static_cast<uint32_t>(i / aslm32), lm = static_cast<uint32_t>(i % aslm32);
        r32[i] = (lm < slm) ? static_cast<float>(r64[static_cast<size_t>(v) * aslm + lm] * inv) : 0.0f;
    }
}

// x64 += scale * d32
__global__ void __launch_bounds__(kBlock) k_correct(uint32_t nP, uint32_t slm, uint32_t aslm, uint32_t aslm32,
                                                    double *__restrict__ x, const float *__restrict__ d32,
                                                    const CgScalars *s) {
    const double sc = s->scale;
    const size_t n = static_cast<size_t>(nP) * aslm;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t v = static_cast<uint32_t>(i / aslm), lm = static_cast<uint32_t>(i % aslm);
        if (lm < slm) x[i] += sc * static_cast<double>(d32[static_cast<size_t>(v) * aslm32 + lm]);
    }
}

// MeshData::ComputeMoments (MeshData.cpp:96-116) on the device.
__global__ void __launch_bounds__(kBlock) k_moments(uint32_t nP, uint32_t slm, uint32_t aslm,
                                                    const double *__restrict__ f, const double *__restrict__ w,
                                                    const uint32_t *__restrict__ pos, double *__restrict__ U,
                                                    double *__restrict__ T) {
    const double fourpi = 12.5663706143591729538505735331;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nP; k += gridDim.x * blockDim.x) {
        const double *fk = f + static_cast<size_t>(k) * aslm;
        double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        U[k] = fourpi * fk[0];
        for (uint32_t lm = 0; lm < slm; ++lm) {
            const double x = fk[lm];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const uint32_t j = __ldg(pos + i * slm + lm);
                const double fw = fourpi * __ldg(w + i * slm + lm);
                // 9-way select keeps t[] in registers
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    if (q == static_cast<int>(j)) t[3 * i + q] += fw * x;
            }
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) T[static_cast<size_t>(q) * nP + k] = t[q];
    }
}

// MeshData::ComputeFlux (MeshData.cpp:118-136): one thread per tet.
__global__ void __launch_bounds__(kBlock) k_flux(const FluxData d, const double *__restrict__ T,
                                                 double *__restrict__ W) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < d.nT; t += gridDim.x * blockDim.x) {
        const uint4 p = d.tet_p[t];
        const uint32_t pk[4] = {p.x, p.y, p.z, p.w};
        const double *s = d.tet_s + static_cast<size_t>(t) * 12;
        const double kv = d.tet_kv[t];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double w = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int a = 0; a < 3; ++a) w += s[3 * k + a] * T[static_cast<size_t>(3 * a + j) * d.nP + pk[k]];
            W[static_cast<size_t>(j) * d.nT + t] = (1.0 / 3.0) * w / kv;
        }
    }
}

// ------------------------------------------------------------------ launch
cudaError_t launch_blas(const tr_ctx *c, int op, double *x, const double *y, double wx, double wy, cudaStream_t s) {
    k_blas<<<c->grid_vec, kBlock, 0, s>>>(static_cast<size_t>(c->nP) * c->aslm, op, x, y, wx, wy);
    return cudaGetLastError();
}
template <typename TX, typename TY>
cudaError_t launch_dot(const tr_ctx *c, uint32_t aslm, const TX *x, const TY *y, double *out, cudaStream_t s) {
    k_dot<TX, TY><<<c->grid_vec, kBlock, 0, s>>>(static_cast<size_t>(c->nP) * aslm, aslm, c->slm, x, y, c->partials,
                                                 c->counters + 1, out);
    return cudaGetLastError();
}
template cudaError_t launch_dot<double, double>(const tr_ctx *, uint32_t, const double *, const double *, double *,
                                                cudaStream_t);
template cudaError_t launch_dot<float, float>(const tr_ctx *, uint32_t, const float *, const float *, double *,
                                              cudaStream_t);

template <typename T>
cudaError_t launch_cg_start(const tr_ctx *c, uint32_t aslm, const T *b, T *f, T *r, T *z, T *p, const T *dinv,
                            CgScalars *s, int zero_p, cudaStream_t st) {
    k_cg_start<T><<<c->grid_vec, kBlock, 0, st>>>(static_cast<size_t>(c->nP) * aslm, aslm, c->slm, b, f, r, z, p,
                                                  dinv, s, c->partials, c->counters + 2, zero_p);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_cg_update(const tr_ctx *c, uint32_t aslm, T *f, T *r, const T *p, const T *Ap, T *z,
                             const T *dinv, CgScalars *s, double *hist, int hist_cap, int defer_beta,
                             cudaStream_t st) {
    const size_t nvec = static_cast<size_t>(c->nP) * aslm / VecT<T>::W;
    const int grid = sizeof(T) == 8 ? c->grid_vec64 : c->grid_vec32;
    k_cg_update<T><<<grid, kBlock, 0, st>>>(nvec, aslm, c->slm, f, r, p, Ap, z, dinv, s, c->partials,
                                            c->counters + 2, hist, hist_cap, defer_beta);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_cg_direction(const tr_ctx *c, uint32_t aslm, T *p, const T *z, const CgScalars *s,
                                cudaStream_t st) {
    k_cg_direction<T><<<c->grid_vec, kBlock, 0, st>>>(static_cast<size_t>(c->nP) * aslm, p, z, s);
    return cudaGetLastError();
}
template cudaError_t launch_cg_start<double>(const tr_ctx *, uint32_t, const double *, double *, double *, double *,
                                             double *, const double *, CgScalars *, int, cudaStream_t);
template cudaError_t launch_cg_start<float>(const tr_ctx *, uint32_t, const float *, float *, float *, float *,
                                            float *, const float *, CgScalars *, int, cudaStream_t);
template cudaError_t launch_cg_update<double>(const tr_ctx *, uint32_t, double *, double *, const double *,
                                              const double *, double *, const double *, CgScalars *, double *, int,
                                              int, cudaStream_t);
template cudaError_t launch_cg_update<float>(const tr_ctx *, uint32_t, float *, float *, const float *,
                                             const float *, float *, const float *, CgScalars *, double *, int, int,
                                             cudaStream_t);
template cudaError_t launch_cg_direction<double>(const tr_ctx *, uint32_t, double *, const double *,
                                                 const CgScalars *, cudaStream_t);
template cudaError_t launch_cg_direction<float>(const tr_ctx *, uint32_t, float *, const float *, const CgScalars *,
                                                cudaStream_t);

cudaError_t launch_residual(const tr_ctx *c, const double *b, const double *Ax, double *r, CgScalars *s,
                            cudaStream_t st) {
    k_residual<<<c->grid_vec, kBlock, 0, st>>>(static_cast<size_t>(c->nP) * c->aslm, c->aslm, c->slm, b, Ax, r, s,
                                               c->partials, c->counters + 3);
    return cudaGetLastError();
}
cudaError_t launch_to_f32(const tr_ctx *c, const double *r64, float *r32, const CgScalars *s, cudaStream_t st) {
    k_to_f32<<<c->grid_vec, kBlock, 0, st>>>(c->nP, c->slm, c->aslm, c->aslm32, r64, r32, s);
    return cudaGetLastError();
}
cudaError_t launch_cg_reliable(const tr_ctx *c, float *f, const float *r, float *z, const float *dinv, CgScalars *s,
                               double ratio, cudaStream_t st) {
    k_cg_reliable<float><<<c->grid_vec, kBlock, 0, st>>>(static_cast<size_t>(c->nP) * c->aslm32, c->aslm32, c->slm,
                                                         f, r, z, dinv, s, ratio, c->partials, c->counters + 2);
    return cudaGetLastError();
}
cudaError_t launch_correct(const tr_ctx *c, double *x, const float *d32, const CgScalars *s, cudaStream_t st) {
    k_correct<<<c->grid_vec, kBlock, 0, st>>>(c->nP, c->slm, c->aslm, c->aslm32, x, d32, s);
    return cudaGetLastError();
}

cudaError_t launch_moments(const tr_ctx *c, const double *f, double *U, double *T, cudaStream_t s) {
    const int grid = static_cast<int>((c->nP + kBlock - 1) / kBlock);
    k_moments<<<grid, kBlock, 0, s>>>(c->nP, c->slm, c->aslm, f, c->mom_w, c->mom_pos, U, T);
    return cudaGetLastError();
}
cudaError_t launch_flux(const tr_ctx *c, const double *T, double *W, cudaStream_t s) {
    FluxData d;
    d.nP = c->nP;
    d.nT = c->nT;
    d.slm = c->slm;
    d.aslm = c->aslm;
    d.tet_p = c->tet_p;
    d.tet_s = c->tet_s;
    d.tet_kv = c->tet_kv;
    d.mom_w = c->mom_w;
    d.mom_pos = c->mom_pos;
    const int grid = static_cast<int>((c->nT + kBlock - 1) / kBlock);
    k_flux<<<grid, kBlock, 0, s>>>(d, T, W);
    return cudaGetLastError();
}

}  // namespace transfer
