// Operator kernels: A f (volumePart + surfacePart, kernels.cu:200-287 and
// 383-438), its angle-diagonal part (volumePartDiag + surfacePartDiag,
// kernels.cu:290-357 and 440-493) and the right-hand side (rightHandSide,
// kernels.cu:135-165), on the assembled vertex-pair layout of internal.h.
//
// Mapping: a group of G lanes (a warp or a part of one) owns one vertex v
// at a time; lane l holds the harmonics lm = l + G*h, h < H.  The edges
// (v, u) of v are taken in chunks of G: every lane loads one neighbour
// index (coalesced) and stages that edge's 12 coefficients in shared
// memory; the group then walks the chunk NB edges at a time, broadcasting
// u by shuffle, so NB independent row gathers f[u][*] are in flight at
// once.  The mass term and the nine spatial sums S_v[3i+j][lm] accumulate
// in registers.  The angular coupling then runs from shared memory: lane
// lm sums omega_i[lms][lm] * S_v[3i+pos][lms] over the nonzero (i, lms) of
// its column (a sparse list staged in shared memory when it fits).
// Boundary vertices add the half-range term from three per-axis sums
// B_n[lms], skipping absent axes.  One launch computes all of A f (the
// reference needs two) and, for CG, fuses <p, A p> with a deterministic
// grid reduction and, optionally, the direction update p = z + beta p_old
// applied to every gathered row (double-buffered p), which removes a
// separate vector kernel per iteration.
#include <cooperative_groups.h>

#include <algorithm>

#include "internal.h"
#include "reduce.cuh"

namespace cg = cooperative_groups;

namespace transfer {

template <typename T>
struct Vec16;  // 16-byte vector of T
template <>
struct Vec16<double> {
    typedef double2 type;
    static constexpr int n = 2;
};
template <>
struct Vec16<float> {
    typedef float4 type;
    static constexpr int n = 4;
};

// 16-byte vectors of T with component access
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

__host__ __device__ constexpr int batch_of(int H) { return H <= 2 ? 4 : 2; }

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

template <typename T>
__host__ __device__ inline size_t ang_smem_bytes(uint32_t nnz) {
    return align16(nnz * sizeof(AngEntry<T>));
}
// per-group shared slab: staged edge coefficients + the S / B table,
// rounded to 16 bytes so every slab (and its vector stores) stays aligned
template <int G, int H, typename T>
__host__ __device__ constexpr size_t group_smem_elems() {
    return (G * kCoefStride + 9 * (G * H + 1) + (16 / sizeof(T)) - 1) / (16 / sizeof(T)) * (16 / sizeof(T));
}

// loads of vectors that other blocks of the same launch may have written
// (persistent kernel) bypass the non-coherent read-only path: L2 only
template <bool COH, typename T>
__device__ __forceinline__ T ldv(const T *p) {
    return COH ? __ldcg(p) : __ldg(p);
}

// x_u = f[u] (plain) or z[u] + beta p_old[u] (fused CG direction)
template <int G, int H, typename T, bool FUSEP, bool COH = false>
__device__ __forceinline__ void gather_row(const T *__restrict__ f, const T *__restrict__ pold, T beta, uint32_t u,
                                           uint32_t aslm, uint32_t slm, int lane, T (&x)[H]) {
    const T *fu = f + u * aslm;
    const T *pu = FUSEP ? pold + u * aslm : nullptr;
#pragma unroll
    for (int h = 0; h < H; ++h) {
        const uint32_t lm = lane + G * h;
        if (lm < slm) {
            x[h] = ldv<COH>(fu + lm);
            if (FUSEP) x[h] = fma(beta, ldv<COH>(pu + lm), x[h]);
        } else {
            x[h] = T(0);
        }
    }
}

// Shared-memory tables staged once per block: the sparse angular lists and,
// when small, the three half-range tables O_n.
template <typename T>
struct Staged {
    const AngEntry<T> *ang;
    const T *O;
    size_t bytes;
};
template <typename T>
__host__ __device__ inline size_t O_smem_bytes(uint32_t slm) {
    return align16(3 * static_cast<size_t>(slm) * slm * sizeof(T));
}

template <typename T>
__device__ __forceinline__ Staged<T> stage_tables(const OpData<T> &d, unsigned char *smem, int flags) {
    Staged<T> st{d.ang, d.O, 0};
    const uint32_t nnz = d.ang_start[d.slm];
    if (flags & 1) {
        AngEntry<T> *se = reinterpret_cast<AngEntry<T> *>(smem);
        for (uint32_t i = threadIdx.x; i < nnz; i += blockDim.x) se[i] = d.ang[i];
        st.ang = se;
        st.bytes = ang_smem_bytes<T>(nnz);
    }
    if (flags & 2) {
        T *so = reinterpret_cast<T *>(smem + st.bytes);
        const uint32_t n = 3 * d.slm * d.slm;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) so[i] = __ldg(d.O + i);
        st.O = so;
        st.bytes += O_smem_bytes<T>(d.slm);
    }
    if (flags) __syncthreads();
    return st;
}

// the 14 coefficients of one staged edge record (vector shared loads)
template <typename T>
__device__ __forceinline__ void load_coef(const T *c, T (&k)[14]);
template <>
__device__ __forceinline__ void load_coef<float>(const float *c, float (&k)[14]) {
    const float4 a = reinterpret_cast<const float4 *>(c)[0], b = reinterpret_cast<const float4 *>(c)[1],
                 e = reinterpret_cast<const float4 *>(c)[2], g = reinterpret_cast<const float4 *>(c)[3];
    k[0] = a.x; k[1] = a.y; k[2] = a.z; k[3] = a.w; k[4] = b.x; k[5] = b.y; k[6] = b.z;
    k[7] = b.w; k[8] = e.x; k[9] = e.y; k[10] = e.z; k[11] = e.w; k[12] = g.x; k[13] = g.y;
}
template <>
__device__ __forceinline__ void load_coef<double>(const double *c, double (&k)[14]) {
    const double2 *v = reinterpret_cast<const double2 *>(c);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const double2 t = v[i];
        k[2 * i] = t.x;
        k[2 * i + 1] = t.y;
    }
}

// A x over the vertices of this block (grid-stride by vertex groups);
// returns this thread's share of <x, A x> (DOT) -- x = f, or, with FUSEP,
// x = f + beta pold, written to pnew.  smem_groups: the block's per-group
// slabs (after the staged tables).
template <int G, int H, typename T, bool DOT, bool FUSEP, bool COH = false>
__device__ __forceinline__ double lhs_vertices(const OpData<T> &d, const Staged<T> &tab, unsigned char *smem_groups,
                                               const T *__restrict__ f, const T *__restrict__ pold,
                                               T *__restrict__ pnew, T *__restrict__ r, const T beta) {
    constexpr int SA = G * H + 1;  // padded row of the shared S / B tables
    constexpr int NB = batch_of(H);
    const uint32_t slm = d.slm, aslm = d.aslm;
    T *scoef = reinterpret_cast<T *>(smem_groups) + (threadIdx.x / G) * group_smem_elems<G, H, T>();
    T *sm = scoef + G * kCoefStride;
    cg::thread_block_tile<G> tile = cg::tiled_partition<G>(cg::this_thread_block());
    const int lane = threadIdx.x % G;
    const uint32_t gpb = kBlock / G;
    const uint32_t ng = gridDim.x * gpb;
    double dacc = 0.0;

    for (uint32_t v = blockIdx.x * gpb + threadIdx.x / G; v < d.nP; v += ng) {
        const uint32_t axes = __ldg(d.bmask + v);
        T mass[H], S[9][H], B[3][H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            mass[h] = B[0][h] = B[1][h] = B[2][h] = T(0);
#pragma unroll
            for (int q = 0; q < 9; ++q) S[q][h] = T(0);
        }
        const uint32_t e0 = __ldg(d.row + v), e1 = __ldg(d.row + v + 1);
        for (uint32_t base = e0; base < e1; base += G) {
            const int cnt = min(static_cast<int>(e1 - base), G);
            uint32_t ul = 0;
            if (lane < cnt) {
                ul = __ldg(d.col + base + lane);
                typedef typename Vec16<T>::type V;
                const V *src = reinterpret_cast<const V *>(d.coef + static_cast<size_t>(base + lane) * kCoefStride);
                V *dst = reinterpret_cast<V *>(scoef + lane * kCoefStride);
#pragma unroll
                for (int q = 0; q < kCoefStride / Vec16<T>::n; ++q) dst[q] = __ldg(src + q);
            }
            tile.sync();
            auto accumulate = [&](const T *cp, const T(&x)[H]) {
                T c[14];
                load_coef<T>(cp, c);
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    const uint32_t lm = lane + G * h;
                    mass[h] = fma(lm == 0 ? c[10] : c[9], x[h], mass[h]);
#pragma unroll
                    for (int q = 0; q < 9; ++q) S[q][h] = fma(c[q], x[h], S[q][h]);
                }
                if (axes) {
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        B[0][h] = fma(c[11], x[h], B[0][h]);
                        B[1][h] = fma(c[12], x[h], B[1][h]);
                        B[2][h] = fma(c[13], x[h], B[2][h]);
                    }
                }
            };
            int jj = 0;
            for (; jj + NB <= cnt; jj += NB) {
                T x[NB][H];
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    gather_row<G, H, T, FUSEP, COH>(f, pold, beta, tile.shfl(ul, jj + b), aslm, slm, lane, x[b]);
#pragma unroll
                for (int b = 0; b < NB; ++b) accumulate(scoef + (jj + b) * kCoefStride, x[b]);
            }
            for (; jj < cnt; ++jj) {
                T x[H];
                gather_row<G, H, T, FUSEP, COH>(f, pold, beta, tile.shfl(ul, jj), aslm, slm, lane, x);
                accumulate(scoef + jj * kCoefStride, x);
            }
            tile.sync();
        }
        // angular coupling through shared memory (two partial sums)
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int q = 0; q < 9; ++q) sm[q * SA + lane + G * h] = S[q][h];
        tile.sync();
        T out[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            T acc0 = T(0), acc1 = T(0);
            if (lm < slm) {
                const uint32_t a1 = __ldg(d.ang_start + lm + 1);
                uint32_t a = __ldg(d.ang_start + lm);
                for (; a + 1 < a1; a += 2) {
                    const AngEntry<T> p0 = tab.ang[a], p1 = tab.ang[a + 1];
                    acc0 = fma(p0.w, sm[p0.off], acc0);
                    acc1 = fma(p1.w, sm[p1.off], acc1);
                }
                if (a < a1) {
                    const AngEntry<T> p0 = tab.ang[a];
                    acc0 = fma(p0.w, sm[p0.off], acc0);
                }
            }
            out[h] = mass[h] + (acc0 + acc1);
        }
        // half-range boundary term from the per-axis sums B_n
        if (axes) {
            tile.sync();
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int n = 0; n < 3; ++n) sm[n * SA + lane + G * h] = B[n][h];
            tile.sync();
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                if (lm < slm) {
                    T acc0 = T(0), acc1 = T(0);
                    for (int n = 0; n < 3; ++n) {
                        if (!(axes & (1u << n))) continue;
                        const T *On = tab.O + static_cast<size_t>(n) * slm * slm + lm;
                        const T *Bn = sm + n * SA;
                        uint32_t lms = 0;
                        for (; lms + 1 < slm; lms += 2) {
                            acc0 = fma(On[lms * slm], Bn[lms], acc0);
                            acc1 = fma(On[(lms + 1) * slm], Bn[lms + 1], acc1);
                        }
                        if (lms < slm) acc0 = fma(On[lms * slm], Bn[lms], acc0);
                    }
                    out[h] += acc0 + acc1;
                }
            }
        }
        tile.sync();
        T *rv = r + static_cast<size_t>(v) * aslm;
        T xv[H];
        if (DOT || FUSEP) gather_row<G, H, T, FUSEP, COH>(f, pold, beta, v, aslm, slm, lane, xv);
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm < aslm) {
                rv[lm] = (lm < slm) ? out[h] : T(0);
                if (FUSEP) pnew[static_cast<size_t>(v) * aslm + lm] = xv[h];
            }
            if (DOT && lm < slm) dacc += static_cast<double>(xv[h]) * static_cast<double>(out[h]);
        }
    }
    return dacc;
}

// register budget: FP64 128 registers (2 resident blocks), FP32 80 (3
// blocks); one block per SM for FP64 with H > 2 harmonics per lane
#define TR_LHS_MINBLOCKS(T, H) (sizeof(T) == 8 ? ((H) > 2 ? 1 : 2) : ((H) > 1 ? 2 : 3))

template <int G, int H, typename T, bool DOT, bool FUSEP, class Fin>
__global__ void __launch_bounds__(kBlock, TR_LHS_MINBLOCKS(T, H)) k_lhs(
    const OpData<T> d, const T *__restrict__ f, const T *__restrict__ pold, T *__restrict__ pnew,
    T *__restrict__ r, double *partials, unsigned int *counter, Fin fin, const int32_t *__restrict__ done,
    const CgScalars *__restrict__ cgs, int stage_flags) {
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Staged<T> tab = stage_tables<T>(d, smem_raw, stage_flags);
    const T beta = FUSEP ? static_cast<T>(cgs->beta) : T(0);
    const double dacc =
        lhs_vertices<G, H, T, DOT, FUSEP>(d, tab, smem_raw + tab.bytes, f, pold, pnew, r, beta);
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
#pragma unroll 2
        for (uint32_t e = __ldg(d.row + v); e < e1; ++e) {
            const uint32_t u = __ldg(d.col + e);
            const T *c = d.coef + static_cast<size_t>(e) * kCoefStride;
            const T K0 = __ldg(c), K4 = __ldg(c + 4), K8 = __ldg(c + 8), M = __ldg(c + 9), M0 = __ldg(c + 10);
            const T E0 = __ldg(c + 11), E1 = __ldg(c + 12), E2 = __ldg(c + 13);
            T x[H];
            gather_row<G, H, T, false>(f, nullptr, T(0), u, aslm, slm, lane, x);
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                mass[h] = fma(lm == 0 ? M0 : M, x[h], mass[h]);
                s0[h] = fma(K0, x[h], s0[h]);
                s1[h] = fma(K4, x[h], s1[h]);
                s2[h] = fma(K8, x[h], s2[h]);
                B[0][h] = fma(E0, x[h], B[0][h]);
                B[1][h] = fma(E1, x[h], B[1][h]);
                B[2][h] = fma(E2, x[h], B[2][h]);
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

// ------------------------------------------------------- persistent CG
// Bounded sense-reversing grid barrier for a co-resident (cooperatively
// launched) grid.  Gives up after kBarrierPolls polls, or as soon as another
// block has given up: sets *err and returns false.
constexpr unsigned int kBarrierPolls = 1u << 24;
__device__ __forceinline__ bool grid_barrier(unsigned int *count, unsigned int *gen, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned int g = atomicAdd(gen, 0u);
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            unsigned int polls = 0;
            while (*reinterpret_cast<volatile unsigned int *>(gen) == g) {
                if (++polls > kBarrierPolls || *reinterpret_cast<volatile int *>(err)) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Totals of per-block partials [NV][gridDim.x], summed by every block in the
// same fixed order (identical results in all blocks).
template <int NV>
__device__ __forceinline__ void sum_partials(const double *partials, double (&tot)[NV]) {
    __shared__ double sh[32];
    __shared__ double res[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double acc = 0.0;
        for (unsigned int i = threadIdx.x; i < gridDim.x; i += blockDim.x) acc += __ldcg(partials + q * gridDim.x + i);
        const double t = block_sum(acc, sh);
        if (threadIdx.x == 0) res[q] = t;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = res[q];
}

// CG (main.cpp:142-160) for up to a.iters iterations in one cooperative
// launch: per iteration, phase A forms p = z + beta p_old inside the
// operator's gather and computes A p and <p, A p>; after a grid barrier
// every block derives alpha, and phase B updates x, r (and z = D^-1 r) with
// ||r||^2 and (r, z); after a second barrier every block takes the stop
// test and beta.  The scalars never leave the device; block 0 mirrors them
// (and the residual history) into CgScalars for the host.
template <int G, int H, typename T, bool JAC>
__global__ void __launch_bounds__(kBlock, TR_LHS_MINBLOCKS(T, H))
    k_cg_persistent(const OpData<T> d, const PcgArgs<T> a, int stage_flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[32];
    const Staged<T> tab = stage_tables<T>(d, smem_raw, stage_flags);
    CgScalars *s = a.s;
    int k = __ldcg(&s->k);
    if (__ldcg(&s->done)) return;
    const int maxit = s->maxit;
    const double tol = s->tol;
    double nrz = __ldcg(&s->nrz), beta = __ldcg(&s->beta);
    typedef VecT<T> O;
    typedef typename O::V V;
    const uint32_t slm = d.slm, aslm = d.aslm;
    for (int it = 0; it < a.iters; ++it) {
        const int parity = k & 1;
        const T *pold = parity ? a.p1 : a.p0;
        T *pnew = parity ? a.p0 : a.p1;
        // phase A: p = z + beta p_old, A p, <p, A p>
        const double dacc = lhs_vertices<G, H, T, true, true, true>(d, tab, smem_raw + tab.bytes, JAC ? a.z : a.r,
                                                                    pold, pnew, a.Ap, static_cast<T>(beta));
        const double bs = block_sum(dacc, sh);
        if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
        if (!grid_barrier(a.bar, a.bar + 1, a.err)) return;
        double t1[1];
        sum_partials<1>(a.partials, t1);
        const double alpha_d = nrz / t1[0];
        const T alpha = static_cast<T>(alpha_d);
        // phase B: x += alpha p; r -= alpha Ap; z = D^-1 r
        double rr = 0.0, rz = 0.0;
        for (uint32_t iv = blockIdx.x * blockDim.x + threadIdx.x; iv < a.nvec; iv += gridDim.x * blockDim.x) {
            V fv = __ldcg(reinterpret_cast<const V *>(a.x) + iv), rv = __ldcg(reinterpret_cast<const V *>(a.r) + iv);
            const V pv = __ldcg(reinterpret_cast<const V *>(pnew) + iv);
            const V av = __ldcg(reinterpret_cast<const V *>(a.Ap) + iv);
            V dv, zv;
            if (JAC) dv = __ldg(reinterpret_cast<const V *>(a.dinv) + iv);
            const uint32_t lm0 = (iv * O::W) % aslm;
#pragma unroll
            for (int q = 0; q < O::W; ++q) {
                O::set(fv, q, fma(alpha, O::get(pv, q), O::get(fv, q)));
                const T ri = fma(-alpha, O::get(av, q), O::get(rv, q));
                O::set(rv, q, ri);
                const bool live = lm0 + q < slm;
                if (JAC) {
                    const T zi = O::get(dv, q) * ri;
                    O::set(zv, q, zi);
                    if (live) rz += static_cast<double>(ri) * static_cast<double>(zi);
                }
                if (live) rr += static_cast<double>(ri) * static_cast<double>(ri);
            }
            reinterpret_cast<V *>(a.x)[iv] = fv;
            reinterpret_cast<V *>(a.r)[iv] = rv;
            if (JAC) reinterpret_cast<V *>(a.z)[iv] = zv;
        }
        const double brr = block_sum(rr, sh);
        const double brz = JAC ? block_sum(rz, sh) : 0.0;
        if (threadIdx.x == 0) {
            a.partials[gridDim.x + blockIdx.x] = brr;
            a.partials[2 * gridDim.x + blockIdx.x] = brz;
        }
        if (!grid_barrier(a.bar, a.bar + 1, a.err)) return;
        double t2[2];
        sum_partials<2>(a.partials + gridDim.x, t2);
        const double nr = sqrt(t2[0]);
        int dn = 0;
        if (!isfinite(nr)) dn = 3;
        else if (nr < tol) dn = 1;
        else if (k + 1 >= maxit) dn = 2;
        const double rznew = JAC ? t2[1] : t2[0];
        if (!dn) {
            beta = rznew / nrz;
            nrz = rznew;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (a.hist && k < a.hist_cap) a.hist[k] = nr;
            s->alpha = alpha_d;
            s->rr = t2[0];
            s->nrz = nrz;
            s->beta = beta;
            s->k = k + 1;
            s->done = dn;
        }
        ++k;
        if (dn) break;
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
constexpr size_t kAngSmemBudget = 64 * 1024;
constexpr size_t kOSmemBudget = 40 * 1024;

template <typename T>
static int stage_flags(uint32_t slm, uint32_t nnz) {
    return (ang_smem_bytes<T>(nnz) <= kAngSmemBudget ? 1 : 0) | (O_smem_bytes<T>(slm) <= kOSmemBudget ? 2 : 0);
}
template <int G, int H, typename T>
static size_t lhs_smem(uint32_t slm, uint32_t nnz) {
    const int fl = stage_flags<T>(slm, nnz);
    return ((fl & 1) ? ang_smem_bytes<T>(nnz) : 0) + ((fl & 2) ? O_smem_bytes<T>(slm) : 0) +
           (kBlock / G) * group_smem_elems<G, H, T>() * sizeof(T);
}

template <int G, int H, typename T, bool DOT, bool FUSEP, class Fin>
static cudaError_t launch_one(const tr_ctx *c, const OpData<T> &d, const LhsArgs<T> &a, Fin fin, cudaStream_t s) {
    const size_t smem = lhs_smem<G, H, T>(d.slm, a.ang_nnz);
    auto kern = k_lhs<G, H, T, DOT, FUSEP, Fin>;
    static size_t opted = 0;  // dynamic shared memory granted so far (per instantiation)
    if (smem > 48 * 1024 && smem > opted) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        opted = smem;
    }
    kern<<<c->grid_op, kBlock, smem, s>>>(d, a.x, a.pold, a.pnew, a.y, c->partials, c->counters, fin, a.done, a.cgs,
                                          stage_flags<T>(d.slm, a.ang_nnz));
    return cudaGetLastError();
}

template <int G, int H, typename T>
static cudaError_t launch_lhs_gh(const tr_ctx *c, const OpData<T> &d, const LhsArgs<T> &a, cudaStream_t s) {
    switch (a.fin_kind) {
    case 0: return launch_one<G, H, T, false, false>(c, d, a, FinNone(), s);
    case 1: return launch_one<G, H, T, true, false>(c, d, a, FinStore{a.fin_out}, s);
    case 2: return launch_one<G, H, T, true, false>(c, d, a, FinAlpha{a.cgs}, s);
    default: return launch_one<G, H, T, true, true>(c, d, a, FinAlpha{a.cgs}, s);
    }
}

template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, LhsArgs<T> a, cudaStream_t s) {
    const OpData<T> d = op.data(c->nP, c->slm);
    a.ang_nnz = op.ang_nnz;
    const uint32_t as = op.aslm;
    if (as <= 8) return launch_lhs_gh<8, 1, T>(c, d, a, s);
    if (as <= 16) return launch_lhs_gh<16, 1, T>(c, d, a, s);
    if (as <= 32) return launch_lhs_gh<32, 1, T>(c, d, a, s);
    if (as <= 64) return launch_lhs_gh<32, 2, T>(c, d, a, s);
    if (as <= 96) return launch_lhs_gh<32, 3, T>(c, d, a, s);
    return launch_lhs_gh<32, 4, T>(c, d, a, s);
}

template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, int fin_kind, double *fin_out,
                       CgScalars *cgs, const int32_t *done, cudaStream_t s) {
    LhsArgs<T> a;
    a.x = f;
    a.y = r;
    a.fin_kind = fin_kind;
    a.fin_out = fin_out;
    a.cgs = cgs;
    a.done = done;
    return launch_lhs<T>(c, op, a, s);
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

template <int G, int H, typename T, bool JAC>
static cudaError_t launch_pcg_gh(const tr_ctx *c, const OpData<T> &d, const PcgArgs<T> &a, uint32_t nnz,
                                 cudaStream_t s, int *grid_out) {
    auto kern = k_cg_persistent<G, H, T, JAC>;
    const size_t smem = lhs_smem<G, H, T>(d.slm, nnz);
    static size_t opted = 0;
    if (smem > 48 * 1024 && smem > opted) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        opted = smem;
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    // enough blocks for the vertices, at most one wave of resident blocks
    const int gpb = kBlock / G;
    const int need = static_cast<int>((d.nP + gpb - 1) / gpb);
    const int grid = std::max(1, std::min(per_sm * c->num_sms, std::min(need, kMaxGrid)));
    *grid_out = grid;
    int flags = stage_flags<T>(d.slm, nnz);
    OpData<T> dd = d;
    PcgArgs<T> aa = a;
    void *args[] = {&dd, &aa, &flags};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), grid, kBlock, args, smem, s);
}

template <typename T>
cudaError_t launch_cg_persistent(const tr_ctx *c, const DeviceOp<T> &op, const PcgArgs<T> &a, cudaStream_t s,
                                 int *grid_out) {
    const OpData<T> d = op.data(c->nP, c->slm);
    const uint32_t as = op.aslm, nnz = op.ang_nnz;
    const bool jac = a.dinv != nullptr;
#define TR_PCG(G, H)                                                                                   \
    return jac ? launch_pcg_gh<G, H, T, true>(c, d, a, nnz, s, grid_out)                              \
               : launch_pcg_gh<G, H, T, false>(c, d, a, nnz, s, grid_out)
    if (as <= 8) TR_PCG(8, 1);
    if (as <= 16) TR_PCG(16, 1);
    if (as <= 32) TR_PCG(32, 1);
    if (as <= 64) TR_PCG(32, 2);
    if (as <= 96) TR_PCG(32, 3);
    TR_PCG(32, 4);
#undef TR_PCG
}
template cudaError_t launch_cg_persistent<double>(const tr_ctx *, const DeviceOp<double> &, const PcgArgs<double> &,
                                                  cudaStream_t, int *);
template cudaError_t launch_cg_persistent<float>(const tr_ctx *, const DeviceOp<float> &, const PcgArgs<float> &,
                                                 cudaStream_t, int *);

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

cudaError_t operator_init_attributes() { return cudaSuccess; }

// largest dynamic shared memory the operator needs for this context
size_t lhs_max_smem(uint32_t aslm, uint32_t slm, uint32_t nnz, bool fp64) {
    auto pick = [&](auto tag) -> size_t {
        typedef decltype(tag) T;
        if (aslm <= 8) return lhs_smem<8, 1, T>(slm, nnz);
        if (aslm <= 16) return lhs_smem<16, 1, T>(slm, nnz);
        if (aslm <= 32) return lhs_smem<32, 1, T>(slm, nnz);
        if (aslm <= 64) return lhs_smem<32, 2, T>(slm, nnz);
        if (aslm <= 96) return lhs_smem<32, 3, T>(slm, nnz);
        return lhs_smem<32, 4, T>(slm, nnz);
    };
    return fp64 ? pick(double()) : pick(float());
}

template cudaError_t launch_lhs<double>(const tr_ctx *, const DeviceOp<double> &, LhsArgs<double>, cudaStream_t);
template cudaError_t launch_lhs<float>(const tr_ctx *, const DeviceOp<float> &, LhsArgs<float>, cudaStream_t);
template cudaError_t launch_lhs<double>(const tr_ctx *, const DeviceOp<double> &, const double *, double *, int,
                                        double *, CgScalars *, const int32_t *, cudaStream_t);
template cudaError_t launch_lhs<float>(const tr_ctx *, const DeviceOp<float> &, const float *, float *, int,
                                       double *, CgScalars *, const int32_t *, cudaStream_t);
template cudaError_t launch_lhs_diag<double>(const tr_ctx *, const DeviceOp<double> &, const double *, double *,
                                             const int32_t *, cudaStream_t);
template cudaError_t launch_lhs_diag<float>(const tr_ctx *, const DeviceOp<float> &, const float *, float *,
                                            const int32_t *, cudaStream_t);

}  // namespace transfer
