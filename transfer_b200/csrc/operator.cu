// Operator kernels: A f (volumePart + surfacePart, kernels.cu:200-287 and
// 383-438), its angle-diagonal part (volumePartDiag + surfacePartDiag,
// kernels.cu:290-357 and 440-493) and the right-hand side (rightHandSide,
// kernels.cu:135-165), on the assembled vertex-pair layout of internal.h.
//
// Mapping: a group of G lanes (a warp or a part of one) owns one vertex v
// at a time; lane l holds the harmonics lm = l + G*h, h < H.  One pass over
// the neighbours u of v gathers the row f[u][*] (coalesced, G*H*sizeof(T)
// bytes) and accumulates, in registers, the mass term and the nine spatial
// sums S_v[3i+j][lm].  The angular coupling then runs from shared memory:
// lane lm sums omega_i[lms][lm] * S_v[3i+pos][lms] over the nonzero
// (i, lms) of its column (a sparse list built at context creation).
// Boundary vertices add the half-range term the same way from three
// per-axis sums B_n[lms].  One launch computes the whole of A f (the
// reference needs two), and optionally the dot product <f, A f> with a
// deterministic grid reduction for the CG step.
#include <cooperative_groups.h>

#include "internal.h"
#include "reduce.cuh"

namespace cg = cooperative_groups;

namespace transfer {

template <typename T>
struct CoefLoad;
template <>
struct CoefLoad<double> {
    __device__ __forceinline__ static void load(const double *c, double (&K)[9], double &M, double &M0) {
        const double2 *c2 = reinterpret_cast<const double2 *>(c);
        double2 a = __ldg(c2 + 0), b = __ldg(c2 + 1), d = __ldg(c2 + 2), e = __ldg(c2 + 3), g = __ldg(c2 + 4),
                h = __ldg(c2 + 5);
        K[0] = a.x; K[1] = a.y; K[2] = b.x; K[3] = b.y; K[4] = d.x; K[5] = d.y;
        K[6] = e.x; K[7] = e.y; K[8] = g.x; M = g.y; M0 = h.x;
    }
    __device__ __forceinline__ static void load_b(const double *c, double (&E)[3]) {
        const double2 *c2 = reinterpret_cast<const double2 *>(c);
        double2 a = __ldg(c2), b = __ldg(c2 + 1);
        E[0] = a.x; E[1] = a.y; E[2] = b.x;
    }
};
template <>
struct CoefLoad<float> {
    __device__ __forceinline__ static void load(const float *c, float (&K)[9], float &M, float &M0) {
        const float4 *c4 = reinterpret_cast<const float4 *>(c);
        float4 a = __ldg(c4 + 0), b = __ldg(c4 + 1), d = __ldg(c4 + 2);
        K[0] = a.x; K[1] = a.y; K[2] = a.z; K[3] = a.w; K[4] = b.x; K[5] = b.y;
        K[6] = b.z; K[7] = b.w; K[8] = d.x; M = d.y; M0 = d.z;
    }
    __device__ __forceinline__ static void load_b(const float *c, float (&E)[3]) {
        float4 a = __ldg(reinterpret_cast<const float4 *>(c));
        E[0] = a.x; E[1] = a.y; E[2] = a.z;
    }
};

struct FinNone {
    __device__ void operator()(double) const {}
};
struct FinStore {
    double *out;
    __device__ void operator()(double t) const { *out = t; }
};
struct FinAlpha {  // CG step length alpha = (r,z) / (p, A p)
    CgScalars *s;
    __device__ void operator()(double pAp) const { s->alpha = s->nrz / pAp; }
};

template <int G, int H, typename T, bool DOT, class Fin>
__global__ void __launch_bounds__(kBlock) k_lhs(const OpData<T> d, const T *__restrict__ f, T *__restrict__ r,
                                                double *partials, unsigned int *counter, Fin fin,
                                                const int32_t *__restrict__ done) {
    if (done && *done) return;
    constexpr int SA = G * H + 1;  // padded row of the shared S / B tables
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw) + (threadIdx.x / G) * (9 * SA);
    cg::thread_block_tile<G> tile = cg::tiled_partition<G>(cg::this_thread_block());
    const int lane = threadIdx.x % G;
    const uint32_t gpb = kBlock / G;
    const uint32_t ng = gridDim.x * gpb;
    const uint32_t slm = d.slm, aslm = d.aslm;
    double dacc = 0.0;

    for (uint32_t v = blockIdx.x * gpb + threadIdx.x / G; v < d.nP; v += ng) {
        T mass[H], S[9][H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            mass[h] = T(0);
#pragma unroll
            for (int q = 0; q < 9; ++q) S[q][h] = T(0);
        }
        const uint32_t e1 = __ldg(d.row + v + 1);
        for (uint32_t e = __ldg(d.row + v); e < e1; ++e) {
            const uint32_t u = __ldg(d.col + e);
            T K[9], M, M0;
            CoefLoad<T>::load(d.coef + static_cast<size_t>(e) * kCoefStride, K, M, M0);
            const T *fu = f + static_cast<size_t>(u) * aslm;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                const T x = (lm < slm) ? __ldg(fu + lm) : T(0);
                mass[h] = fma(lm == 0 ? M0 : M, x, mass[h]);
#pragma unroll
                for (int q = 0; q < 9; ++q) S[q][h] = fma(K[q], x, S[q][h]);
            }
        }
        // angular coupling through shared memory
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int q = 0; q < 9; ++q) sm[q * SA + lane + G * h] = S[q][h];
        tile.sync();
        T out[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            T acc = T(0);
            if (lm < slm) {
                const uint32_t a1 = __ldg(d.ang_start + lm + 1);
                for (uint32_t a = __ldg(d.ang_start + lm); a < a1; ++a) {
                    const uint32_t src = __ldg(d.ang_src + a);
                    acc = fma(__ldg(d.ang_w + a), sm[(src >> 8) * SA + (src & 255u)], acc);
                }
            }
            out[h] = mass[h] + acc;
        }
        tile.sync();
        // half-range boundary term
        const uint32_t b1 = __ldg(d.brow + v + 1);
        uint32_t b0 = __ldg(d.brow + v);
        if (b1 > b0) {
            T B[3][H];
#pragma unroll
            for (int h = 0; h < H; ++h) B[0][h] = B[1][h] = B[2][h] = T(0);
            for (; b0 < b1; ++b0) {
                const uint32_t u = __ldg(d.bcol + b0);
                T E[3];
                CoefLoad<T>::load_b(d.bcoef + static_cast<size_t>(b0) * kBCoefStride, E);
                const T *fu = f + static_cast<size_t>(u) * aslm;
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    const uint32_t lm = lane + G * h;
                    const T x = (lm < slm) ? __ldg(fu + lm) : T(0);
                    B[0][h] = fma(E[0], x, B[0][h]);
                    B[1][h] = fma(E[1], x, B[1][h]);
                    B[2][h] = fma(E[2], x, B[2][h]);
                }
            }
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int n = 0; n < 3; ++n) sm[n * SA + lane + G * h] = B[n][h];
            tile.sync();
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                if (lm < slm) {
                    T acc = T(0);
                    for (int n = 0; n < 3; ++n) {
                        const T *On = d.O + static_cast<size_t>(n) * slm * slm + lm;
                        const T *Bn = sm + n * SA;
                        for (uint32_t lms = 0; lms < slm; ++lms) acc = fma(__ldg(On + lms * slm), Bn[lms], acc);
                    }
                    out[h] += acc;
                }
            }
            tile.sync();
        }
        T *rv = r + static_cast<size_t>(v) * aslm;
        const T *fv = f + static_cast<size_t>(v) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm < aslm) rv[lm] = (lm < slm) ? out[h] : T(0);
            if (DOT && lm < slm) dacc += static_cast<double>(__ldg(fv + lm)) * static_cast<double>(out[h]);
        }
    }
    if (DOT) {
        double vv[1] = {dacc}, tot[1];
        if (grid_reduce<1>(vv, partials, counter, tot) && threadIdx.x == 0) fin(tot[0]);
    }
}

template <int G, int H, typename T>
__global__ void __launch_bounds__(kBlock) k_lhs_diag(const OpData<T> d, const T *__restrict__ f,
                                                     T *__restrict__ r, const int32_t *__restrict__ done) {
    if (done && *done) return;
    const int lane = threadIdx.x % G;
    const uint32_t gpb = kBlock / G;
    const uint32_t ng = gridDim.x * gpb;
    const uint32_t slm = d.slm, aslm = d.aslm;
    for (uint32_t v = blockIdx.x * gpb + threadIdx.x / G; v < d.nP; v += ng) {
        T mass[H], s0[H], s1[H], s2[H], B[3][H];
#pragma unroll
        for (int h = 0; h < H; ++h) mass[h] = s0[h] = s1[h] = s2[h] = B[0][h] = B[1][h] = B[2][h] = T(0);
        const uint32_t e1 = __ldg(d.row + v + 1);
        for (uint32_t e = __ldg(d.row + v); e < e1; ++e) {
            const uint32_t u = __ldg(d.col + e);
            T K[9], M, M0;
            CoefLoad<T>::load(d.coef + static_cast<size_t>(e) * kCoefStride, K, M, M0);
            const T *fu = f + static_cast<size_t>(u) * aslm;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                const T x = (lm < slm) ? __ldg(fu + lm) : T(0);
                mass[h] = fma(lm == 0 ? M0 : M, x, mass[h]);
                s0[h] = fma(K[0], x, s0[h]);
                s1[h] = fma(K[4], x, s1[h]);
                s2[h] = fma(K[8], x, s2[h]);
            }
        }
        const uint32_t b1 = __ldg(d.brow + v + 1);
        for (uint32_t b = __ldg(d.brow + v); b < b1; ++b) {
            const uint32_t u = __ldg(d.bcol + b);
            T E[3];
            CoefLoad<T>::load_b(d.bcoef + static_cast<size_t>(b) * kBCoefStride, E);
            const T *fu = f + static_cast<size_t>(u) * aslm;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                const T x = (lm < slm) ? __ldg(fu + lm) : T(0);
                B[0][h] = fma(E[0], x, B[0][h]);
                B[1][h] = fma(E[1], x, B[1][h]);
                B[2][h] = fma(E[2], x, B[2][h]);
            }
        }
        T *rv = r + static_cast<size_t>(v) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm >= aslm) continue;
            T out = T(0);
            if (lm < slm) {
                out = mass[h] + __ldg(d.ang_diag + lm) * s0[h] + __ldg(d.ang_diag + slm + lm) * s1[h] +
                      __ldg(d.ang_diag + 2 * slm + lm) * s2[h];
                out += __ldg(d.O_diag + lm) * B[0][h] + __ldg(d.O_diag + slm + lm) * B[1][h] +
                       __ldg(d.O_diag + 2 * slm + lm) * B[2][h];
            }
            rv[lm] = out;
        }
    }
}

// rightHandSide (kernels.cu:135-165): b[v][0] = sum_t kappa_volume I_p / 4 in
// the vertex's tet order; inflow faces add I A/3 <|Omega_n| Y_lm>.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_rhs(const RhsData d, T *__restrict__ b, uint32_t aslm) {
    const size_t n = static_cast<size_t>(d.nP) * aslm;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t v = static_cast<uint32_t>(i / aslm), lm = static_cast<uint32_t>(i % aslm);
        double sum = 0.0;
        if (lm == 0) {
            const uint32_t j1 = d.vt_start[v + 1];
            for (uint32_t j = d.vt_start[v]; j < j1; ++j) sum += d.tet_q[d.vt_tet[j]] * (1.0 / 4.0);
        }
        if (d.inflow && lm < d.slm) {
            const double *in = d.inflow + 3 * static_cast<size_t>(v);
            const size_t ss = static_cast<size_t>(d.slm) * d.slm;
            sum += in[0] * d.O[lm] + in[1] * d.O[ss + lm] + in[2] * d.O[2 * ss + lm];
        }
        b[i] = static_cast<T>(lm < d.slm ? sum : 0.0);
    }
}

// ------------------------------------------------------------------ launch
template <int G, int H, typename T>
static cudaError_t launch_lhs_gh(const tr_ctx *c, const OpData<T> &d, const T *f, T *r, int fin_kind,
                                 double *fin_out, CgScalars *cgs, const int32_t *done, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(kBlock / G) * 9 * (G * H + 1) * sizeof(T);
    const int grid = c->grid_op;
    unsigned int *counter = c->counters;
    switch (fin_kind) {
    case 0:
        k_lhs<G, H, T, false, FinNone><<<grid, kBlock, smem, s>>>(d, f, r, nullptr, nullptr, FinNone(), done);
        break;
    case 1:
        k_lhs<G, H, T, true, FinStore>
            <<<grid, kBlock, smem, s>>>(d, f, r, c->partials, counter, FinStore{fin_out}, done);
        break;
    default:
        k_lhs<G, H, T, true, FinAlpha>
            <<<grid, kBlock, smem, s>>>(d, f, r, c->partials, counter, FinAlpha{cgs}, done);
        break;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, int fin_kind, double *fin_out,
                       CgScalars *cgs, const int32_t *done, cudaStream_t s) {
    const OpData<T> d = op.data(c->nP, c->slm);
    const uint32_t a = op.aslm;
    if (a <= 8) return launch_lhs_gh<8, 1, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
    if (a <= 16) return launch_lhs_gh<16, 1, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
    if (a <= 32) return launch_lhs_gh<32, 1, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
    if (a <= 64) return launch_lhs_gh<32, 2, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
    if (a <= 96) return launch_lhs_gh<32, 3, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
    return launch_lhs_gh<32, 4, T>(c, d, f, r, fin_kind, fin_out, cgs, done, s);
}

template <typename T>
cudaError_t launch_lhs_diag(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, const int32_t *done,
                            cudaStream_t s) {
    const OpData<T> d = op.data(c->nP, c->slm);
    const uint32_t a = op.aslm;
    const int grid = c->grid_op;
    if (a <= 8) k_lhs_diag<8, 1, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    else if (a <= 16) k_lhs_diag<16, 1, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    else if (a <= 32) k_lhs_diag<32, 1, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    else if (a <= 64) k_lhs_diag<32, 2, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    else if (a <= 96) k_lhs_diag<32, 3, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    else k_lhs_diag<32, 4, T><<<grid, kBlock, 0, s>>>(d, f, r, done);
    return cudaGetLastError();
}

static RhsData rhs_data(const tr_ctx *c) {
    RhsData d;
    d.nP = c->nP;
    d.slm = c->slm;
    d.aslm = c->aslm;
    d.vt_start = c->vt_start;
    d.vt_tet = c->vt_tet;
    d.tet_q = c->tet_q;
    d.inflow = c->inflow;
    d.O = c->O64;
    return d;
}
cudaError_t launch_rhs(const tr_ctx *c, double *b, cudaStream_t s) {
    k_rhs<double><<<c->grid_vec, kBlock, 0, s>>>(rhs_data(c), b, c->aslm);
    return cudaGetLastError();
}
cudaError_t launch_rhs_f32(const tr_ctx *c, float *b, cudaStream_t s) {
    k_rhs<float><<<c->grid_vec, kBlock, 0, s>>>(rhs_data(c), b, c->aslm32);
    return cudaGetLastError();
}

// shared-memory opt-in for the largest instantiations (called once per ctx)
template <typename T>
static cudaError_t set_smem_attr() {
    cudaError_t e = cudaSuccess;
    auto one = [&](auto kern, int G, int H) {
        size_t smem = static_cast<size_t>(kBlock / G) * 9 * (G * H + 1) * sizeof(T);
        if (smem > 48 * 1024 && e == cudaSuccess)
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    };
    one(k_lhs<32, 2, T, false, FinNone>, 32, 2);
    one(k_lhs<32, 2, T, true, FinStore>, 32, 2);
    one(k_lhs<32, 2, T, true, FinAlpha>, 32, 2);
    one(k_lhs<32, 3, T, false, FinNone>, 32, 3);
    one(k_lhs<32, 3, T, true, FinStore>, 32, 3);
    one(k_lhs<32, 3, T, true, FinAlpha>, 32, 3);
    one(k_lhs<32, 4, T, false, FinNone>, 32, 4);
    one(k_lhs<32, 4, T, true, FinStore>, 32, 4);
    one(k_lhs<32, 4, T, true, FinAlpha>, 32, 4);
    return e;
}
cudaError_t operator_init_attributes() {
    cudaError_t e = set_smem_attr<double>();
    if (e == cudaSuccess) e = set_smem_attr<float>();
    return e;
}

template cudaError_t launch_lhs<double>(const tr_ctx *, const DeviceOp<double> &, const double *, double *, int,
                                        double *, CgScalars *, const int32_t *, cudaStream_t);
template cudaError_t launch_lhs<float>(const tr_ctx *, const DeviceOp<float> &, const float *, float *, int,
                                       double *, CgScalars *, const int32_t *, cudaStream_t);
template cudaError_t launch_lhs_diag<double>(const tr_ctx *, const DeviceOp<double> &, const double *, double *,
                                             const int32_t *, cudaStream_t);
template cudaError_t launch_lhs_diag<float>(const tr_ctx *, const DeviceOp<float> &, const float *, float *,
                                            const int32_t *, cudaStream_t);

}  // namespace transfer
