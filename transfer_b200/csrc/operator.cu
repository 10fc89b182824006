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
// in registers.  The angular coupling then runs from shared memory:
// out[lm] = sum omega_i[lms][lm] * S_v[3i+pos][lms] over the nonzero
// (i, lms) of column lm, all columns' entries cut into equal runs, one per
// lane (Runs in internal.h; staged in shared memory when they fit).
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

// neighbour rows gathered at once per lane (loads in flight).  With one
// harmonic per lane the persistent CG kernels (one block of 24 warps per SM,
// which wait at grid barriers between iterations) gain from 8 rows in flight
// (the mixed solve on milne_slab_ref 2% faster), the operator launched alone
// (3 blocks of 8 warps per SM) from 4 (6% faster alone).
#ifndef TR_GATHER_BATCH1
#define TR_GATHER_BATCH1 4
#endif
#ifndef TR_GATHER_BATCH1_PERSISTENT
#define TR_GATHER_BATCH1_PERSISTENT 8
#endif
__host__ __device__ constexpr int batch_of(int H, bool persistent = false) {
    return H == 1 ? (persistent ? TR_GATHER_BATCH1_PERSISTENT : TR_GATHER_BATCH1) : H == 2 ? 4 : 2;
}

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// per-group shared slab: staged edge coefficients + the S / B table,
// rounded to 16 bytes so every slab (and its vector stores) stays aligned
template <int G, int H, typename T>
__host__ __device__ constexpr size_t group_smem_elems() {
    // two edge-record buffers [2][G][kCoefStride], two neighbour-index
    // buffers [2][G] (uint32), the S / B table [kSymRows][G*H+1], the chunk
    // sums of the contraction rounds [runs_part_elems(G, H)]
    return (2 * G * kCoefStride + (2 * G * 4 + sizeof(T) - 1) / sizeof(T) + kSymRows * (G * H + 1) +
            runs_part_elems(G, H) + (16 / sizeof(T)) - 1) / (16 / sizeof(T)) * (16 / sizeof(T));
}
// Loads of vectors that other blocks of the same launch may have written
// (persistent kernel) avoid the non-coherent read-only path (ld.global.nc
// requires data that no thread writes during the kernel) and use ordinary
// cached loads (ld.global.ca); they only read data written before the last
// grid barrier, whose fences order those writes before these loads.
template <bool COH, typename T>
__device__ __forceinline__ T ldv(const T *p) {
    return COH ? __ldca(p) : __ldg(p);
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

// Shared-memory tables staged once per block: the contraction rounds of the
// kernel's form and, when small, the three half-range tables O_n.
template <typename T>
struct Staged {
    const unsigned char *run;  // Runs entries
    const uint32_t *rsp;       // chunk span of each harmonic [slm]
    const T *O;
    size_t bytes;
};
template <typename T>
__host__ __device__ inline size_t O_smem_bytes(uint32_t slm, uint32_t cls) {
    return align16(3 * static_cast<size_t>(slm) * cls * sizeof(T));
}

// flags: 1 stage the contraction rounds, 2 stage O, 4 the tensor-core
// rounds (C-table offsets) instead of the SIMT ones
template <typename T>
__device__ __forceinline__ Staged<T> stage_tables(const OpData<T> &d, unsigned char *smem, int flags) {
    const Runs<T> &R = (flags & 4) ? d.rt : d.rs;
    Staged<T> st{R.tab, R.span, d.O, 0};
    if (flags & 1) {
        const size_t eb = runs_entry_bytes(R);  // a multiple of 16: L, R are multiples of 4
        uint32_t *ss = reinterpret_cast<uint32_t *>(smem + align16(eb));
        for (uint32_t i = threadIdx.x; i < eb / 16; i += blockDim.x)
            reinterpret_cast<uint4 *>(smem)[i] = __ldg(reinterpret_cast<const uint4 *>(R.tab) + i);
        for (uint32_t i = threadIdx.x; i < d.slm; i += blockDim.x) ss[i] = __ldg(R.span + i);
        st.run = smem;
        st.rsp = ss;
        st.bytes = runs_smem_bytes<T>(R, d.slm);
    }
    if (flags & 2) {
        T *so = reinterpret_cast<T *>(smem + st.bytes);
        const uint32_t n = 3 * d.slm * d.cls;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) so[i] = __ldg(d.O + i);
        st.O = so;
        st.bytes += O_smem_bytes<T>(d.slm, d.cls);
    }
    if (flags & 3) __syncthreads();
    return st;
}

// entry i of a Runs table of n entries: FP32 one (w, o) pair, FP64 the
// weight block then the offset block
template <typename T>
__device__ __forceinline__ void run_entry(const unsigned char *tab, size_t n, size_t i, T &w, uint32_t &o);
template <>
__device__ __forceinline__ void run_entry<float>(const unsigned char *tab, size_t, size_t i, float &w, uint32_t &o) {
    const uint2 e = reinterpret_cast<const uint2 *>(tab)[i];
    w = __uint_as_float(e.x);
    o = e.y;
}
template <>
__device__ __forceinline__ void run_entry<double>(const unsigned char *tab, size_t n, size_t i, double &w,
                                                  uint32_t &o) {
    w = reinterpret_cast<const double *>(tab)[i];
    o = reinterpret_cast<const uint32_t *>(tab + 8 * n)[i];
}

// The lane's chunks of the contraction rounds (Runs): in round r the lane
// sums chunk r * L + lane over R steps (four accumulators, the loads of four
// steps issued before their FMAs) from the table S and stores the sum to
// part[r * L + lane].
template <typename T, int L>
__device__ __forceinline__ void contract_rounds(const Runs<T> &R, const unsigned char *tab, int lane, const T *S,
                                                T *part) {
    const size_t n = static_cast<size_t>(R.rounds) * R.R * L;
    size_t i = lane;
    for (uint32_t r = 0; r < R.rounds; ++r) {
        T a[4] = {T(0), T(0), T(0), T(0)};
        for (uint32_t j = 0; j < R.R; j += 4, i += 4 * L) {
            T w[4], x[4];
            uint32_t o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) run_entry<T>(tab, n, i + q * L, w[q], o[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) x[q] = S[o[q]];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = fma(w[q], x[q], a[q]);
        }
        part[r * L + lane] = (a[0] + a[2]) + (a[1] + a[3]);
    }
}
// harmonic lm's coupling: acc0 plus its chunk sums, in chunk order
template <typename T>
__device__ __forceinline__ T sum_chunks(const uint32_t *span, const T *part, uint32_t lm, T acc0) {
    const uint32_t sp = span[lm], c1 = sp >> 16;
    for (uint32_t c = sp & 0xFFFFu; c < c1; ++c) acc0 += part[c];
    return acc0;
}

// the 11 used coefficients of one staged edge record (vector shared loads)
template <typename T>
__device__ __forceinline__ void load_coef(const T *c, T (&k)[12]);
template <>
__device__ __forceinline__ void load_coef<float>(const float *c, float (&k)[12]) {
    const float4 a = reinterpret_cast<const float4 *>(c)[0], b = reinterpret_cast<const float4 *>(c)[1],
                 e = reinterpret_cast<const float4 *>(c)[2];
    k[0] = a.x; k[1] = a.y; k[2] = a.z; k[3] = a.w; k[4] = b.x; k[5] = b.y;
    k[6] = b.z; k[7] = b.w; k[8] = e.x; k[9] = e.y; k[10] = e.z; k[11] = e.w;
}
template <>
__device__ __forceinline__ void load_coef<double>(const double *c, double (&k)[12]) {
    const double2 *v = reinterpret_cast<const double2 *>(c);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double2 t = v[i];
        k[2 * i] = t.x;
        k[2 * i + 1] = t.y;
    }
}

// Edge-loop accumulators of one harmonic lm: the six symmetric stiffness
// sums S_q, the mass term and the three boundary sums B_n.
//   FP64: the mass row is chosen per lane (M0 for lm = 0, M otherwise).
//   FP32: the sums are float2 pairs updated by paired FMAs (__ffma2_rn,
//   FFMA2 on sm_100: one instruction, two independent round-to-nearest
//   FMAs), and the mass pair (M, M0) is accumulated for every lane, the
//   lane choosing its half at the end.  Same products, same order, same
//   rounding as scalar FMAs.
template <typename T>
struct EdgeAcc;
template <>
struct EdgeAcc<double> {
    typedef double Coef[12];
    double S_[kSymRows], m_, B_[3];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int q = 0; q < kSymRows; ++q) S_[q] = 0.0;
        m_ = B_[0] = B_[1] = B_[2] = 0.0;
    }
    __device__ static __forceinline__ void load(const double *cp, Coef &c) { load_coef<double>(cp, c); }
    __device__ __forceinline__ void add(const Coef &c, double x, bool l0) {
        m_ = fma(l0 ? c[kRowM0] : c[kRowM], x, m_);
#pragma unroll
        for (int q = 0; q < kSymRows; ++q) S_[q] = fma(c[q], x, S_[q]);
    }
    __device__ __forceinline__ void add_bnd(const Coef &c, double x) {
#pragma unroll
        for (int n = 0; n < 3; ++n) B_[n] = fma(c[kRowE + n], x, B_[n]);
    }
    __device__ __forceinline__ double S(int q) const { return S_[q]; }
    __device__ __forceinline__ double mass(bool) const { return m_; }
    __device__ __forceinline__ double B(int n) const { return B_[n]; }
};
template <>
struct EdgeAcc<float> {
    typedef float4 Coef[3];  // records 0-11: K (6), M, M0, E (3), pad
    float2 s01_, s23_, s45_, mm_, e01_;
    float e2_;
    __device__ __forceinline__ void zero() {
        s01_ = s23_ = s45_ = mm_ = e01_ = make_float2(0.0f, 0.0f);
        e2_ = 0.0f;
    }
    __device__ static __forceinline__ void load(const float *cp, Coef &c) {
        const float4 *v = reinterpret_cast<const float4 *>(cp);
        c[0] = v[0];
        c[1] = v[1];
        c[2] = v[2];
    }
    __device__ __forceinline__ void add(const Coef &c, float x, bool) {
        const float2 xx = make_float2(x, x);
        s01_ = __ffma2_rn(make_float2(c[0].x, c[0].y), xx, s01_);
        s23_ = __ffma2_rn(make_float2(c[0].z, c[0].w), xx, s23_);
        s45_ = __ffma2_rn(make_float2(c[1].x, c[1].y), xx, s45_);
        mm_ = __ffma2_rn(make_float2(c[1].z, c[1].w), xx, mm_);
    }
    __device__ __forceinline__ void add_bnd(const Coef &c, float x) {
        e01_ = __ffma2_rn(make_float2(c[2].x, c[2].y), make_float2(x, x), e01_);
        e2_ = fmaf(c[2].z, x, e2_);
    }
    __device__ __forceinline__ float S(int q) const {
        return q == 0 ? s01_.x : q == 1 ? s01_.y : q == 2 ? s23_.x : q == 3 ? s23_.y : q == 4 ? s45_.x : s45_.y;
    }
    __device__ __forceinline__ float mass(bool l0) const { return l0 ? mm_.y : mm_.x; }
    __device__ __forceinline__ float B(int n) const { return n == 0 ? e01_.x : n == 1 ? e01_.y : e2_; }
};
static_assert(kRowM == 6 && kRowM0 == 7 && kRowE == 8 && kSymRows == 6, "EdgeAcc<float> pairs the record rows");

// Asynchronous global -> shared copies (cp.async, no registers held while
// in flight): a group queues the next vertex's neighbour indices and edge
// records while it still works on the current vertex.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// queue the edges [base, base + cnt) of a vertex into one staging buffer:
// lane l < cnt copies edge base + l (its neighbour index and record rows
// 0-7; rows 8-15 only for a vertex with boundary faces, bnd)
template <typename T>
__device__ __forceinline__ void stage_edges_async(const OpData<T> &d, uint32_t base, int cnt, int lane, T *scoef,
                                                  uint32_t *scol, bool bnd) {
    if (lane < cnt) {
        cp_async4(scol + lane, d.col + base + lane);
        constexpr int kChunks = kCoefHalf * static_cast<int>(sizeof(T)) / 16, kPer = 16 / sizeof(T);
        const T *src = d.coef + static_cast<size_t>(base + lane) * kCoefHalf;
        T *dst = scoef + lane * kCoefStride;
#pragma unroll
        for (int q = 0; q < kChunks; ++q) cp_async16(dst + q * kPer, src + q * kPer);
        if (bnd) {
            const T *srcb = d.coef_bnd + static_cast<size_t>(base + lane) * kCoefHalf;
#pragma unroll
            for (int q = 0; q < kChunks; ++q) cp_async16(dst + kCoefHalf + q * kPer, srcb + q * kPer);
        }
    }
    cp_async_commit();
}

// ---- what the SIMT vertex loop reads and what its owner step writes
// Src::row(u, lane, x): the input row of neighbour u.  Out::load(v, lane)
// fetches what the owner step of vertex v needs (issued early), Out::store
// writes the results of v from its operator row `out` and adds Out::NV
// partial sums.

// plain operator input (x_u = f[u]) or CG's fused direction (z[u] + beta p_old[u])
template <int G, int H, typename T, bool FUSEP, bool COH>
struct SrcDir {
    static constexpr bool kPersistent = COH;  // the persistent kernels read rows written in the same launch
    const T *f, *pold;
    T beta;
    uint32_t aslm, slm;
    __device__ __forceinline__ void row(uint32_t u, int lane, T (&x)[H]) const {
        gather_row<G, H, T, FUSEP, COH>(f, pold, beta, u, aslm, slm, lane, x);
    }
};
// A x stored in r; with FUSEP the direction row is stored in pnew; with DOT
// the partial sum <x, A x>
template <int G, int H, typename T, bool DOT, bool FUSEP, bool COH>
struct OutStd {
    static constexpr int NV = 1;
    const T *f, *pold;
    T *pnew, *r;
    T beta;
    uint32_t aslm, slm;
    struct Pre {
        T xv[H];
    };
    __device__ __forceinline__ Pre load(uint32_t v, int lane) const {
        Pre p;
        if (DOT || FUSEP) gather_row<G, H, T, FUSEP, COH>(f, pold, beta, v, aslm, slm, lane, p.xv);
        return p;
    }
    __device__ __forceinline__ void store(uint32_t v, int lane, const T (&out)[H], const Pre &p,
                                          double (&acc)[NV]) const {
        T *rv = r + static_cast<size_t>(v) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm < aslm) {
                rv[lm] = (lm < slm) ? out[h] : T(0);
                if (FUSEP) pnew[static_cast<size_t>(v) * aslm + lm] = p.xv[h];
            }
            if (DOT && lm < slm) acc[0] += static_cast<double>(p.xv[h]) * static_cast<double>(out[h]);
        }
    }
};

// Single-reduction CG (Chronopoulos & Gear, J. Comput. Appl. Math. 25 (1989))
// with preconditioner M (identity or Jacobi).  Step j reads r_{j-1},
// w_{j-1} = A u_{j-1}, s_{j-2} and the scalars alpha_{j-1}, beta_{j-1}, and
// in one pass over the operator forms
//   s_{j-1} = w_{j-1} + beta s_{j-2},  p_{j-1} = u_{j-1} + beta p_{j-2},
//   x_j = x_{j-1} + alpha p_{j-1},     r_j = r_{j-1} - alpha s_{j-1},
//   u_j = M r_j,  w_j = A u_j,  and (r_j, u_j), (w_j, u_j), (r_j, r_j):
// the neighbours' u_j are formed on the fly from their r, w, s rows, so the
// two reductions of a CG step meet at one grid barrier.  r, w, s are double
// buffered (read j-1, write j); p and x are only touched by their owner.
template <typename T>
struct SrStep {
    const T *r, *w, *s;  // r_{j-1}, w_{j-1}, s_{j-2}
    T *rn, *wn, *sn;     // r_j, w_j, s_{j-1}
    T *p, *x;            // p_{j-2} -> p_{j-1}, x_{j-1} -> x_j
    const T *dinv;       // Jacobi, or null
    T alpha, beta;       // alpha_{j-1}, beta_{j-1}
};
// u_j from the step-(j-1) rows; the owner forms the same value with the same operations
template <typename T, bool JAC>
__device__ __forceinline__ T sr_u(T r, T w, T s, T dv, T alpha, T beta, T &s1, T &r1) {
    s1 = fma(beta, s, w);
    r1 = fma(-alpha, s1, r);
    return JAC ? dv * r1 : r1;
}
template <int G, int H, typename T, bool JAC>
struct SrcSr {
    static constexpr bool kPersistent = true;
    SrStep<T> st;
    uint32_t aslm, slm;
    __device__ __forceinline__ void row(uint32_t u, int lane, T (&x)[H]) const {
        const size_t o = static_cast<size_t>(u) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm < slm) {
                const T dv = JAC ? ldv<false>(st.dinv + o + lm) : T(1);
                T s1, r1;
                x[h] = sr_u<T, JAC>(ldv<true>(st.r + o + lm), ldv<true>(st.w + o + lm), ldv<true>(st.s + o + lm), dv,
                                    st.alpha, st.beta, s1, r1);
            } else {
                x[h] = T(0);
            }
        }
    }
};
template <int G, int H, typename T, bool JAC>
struct OutSr {
    static constexpr int NV = 3;  // (r_j, u_j), (w_j, u_j), (r_j, r_j)
    SrStep<T> st;
    uint32_t aslm, slm;
    struct Pre {
        T r[H], w[H], s[H], p[H], x[H], dv[H];
    };
    __device__ __forceinline__ Pre load(uint32_t v, int lane) const {
        Pre q;
        const size_t o = static_cast<size_t>(v) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            const bool in = lm < aslm;
            q.r[h] = in ? ldv<true>(st.r + o + lm) : T(0);
            q.w[h] = in ? ldv<true>(st.w + o + lm) : T(0);
            q.s[h] = in ? ldv<true>(st.s + o + lm) : T(0);
            q.p[h] = in ? st.p[o + lm] : T(0);
            q.x[h] = in ? st.x[o + lm] : T(0);
            q.dv[h] = (JAC && in) ? ldv<false>(st.dinv + o + lm) : T(1);
        }
        return q;
    }
    __device__ __forceinline__ void store(uint32_t v, int lane, const T (&out)[H], const Pre &q,
                                          double (&acc)[NV]) const {
        const size_t o = static_cast<size_t>(v) * aslm;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            if (lm >= aslm) continue;
            T s1, r1;
            const T uj = sr_u<T, JAC>(q.r[h], q.w[h], q.s[h], q.dv[h], st.alpha, st.beta, s1, r1);
            const T u0 = JAC ? q.dv[h] * q.r[h] : q.r[h];     // u_{j-1}
            const T p1 = fma(st.beta, q.p[h], u0);            // p_{j-1}
            const T wj = (lm < slm) ? out[h] : T(0);
            st.sn[o + lm] = s1;
            st.p[o + lm] = p1;
            st.x[o + lm] = fma(st.alpha, p1, q.x[h]);
            st.rn[o + lm] = r1;
            st.wn[o + lm] = wj;
            if (lm < slm) {
                acc[0] += static_cast<double>(r1) * static_cast<double>(uj);
                acc[1] += static_cast<double>(wj) * static_cast<double>(uj);
                acc[2] += static_cast<double>(r1) * static_cast<double>(r1);
            }
        }
    }
};

template <int G, int H, typename T, class Src, class Out>
__device__ __forceinline__ void simt_vertices(const OpData<T> &d, const Staged<T> &tab, unsigned char *smem_groups,
                                              const Src &src, const Out &fin, double (&dacc)[Out::NV]) {
    constexpr int SA = G * H + 1;  // padded row of the shared S / B tables
    constexpr int NB = batch_of(H, Src::kPersistent);
    constexpr int LS = G * H < 32 ? 32 : G * H;  // lane stride of O (== d.cls, checked at launch)
    const uint32_t slm = d.slm, aslm = d.aslm;
    T *slab = reinterpret_cast<T *>(smem_groups) + (threadIdx.x / G) * group_smem_elems<G, H, T>();
    uint32_t *scolbuf = reinterpret_cast<uint32_t *>(slab + 2 * G * kCoefStride);  // [2][G]
    T *sm = slab + 2 * G * kCoefStride + (2 * G * 4 + sizeof(T) - 1) / sizeof(T);
    cg::thread_block_tile<G> tile = cg::tiled_partition<G>(cg::this_thread_block());
    const int lane = threadIdx.x % G;
    const uint32_t gpb = blockDim.x / G;
#pragma unroll
    for (int q = 0; q < Out::NV; ++q) dacc[q] = 0.0;

    // Each block owns a contiguous range of vertices (neighbouring rows are
    // shared in L1); its groups take the range's vertices one at a time from
    // a shared counter, so a group that drew cheap vertices draws more.
    __shared__ unsigned int s_next;
    const uint32_t per_block = (d.nP + gridDim.x - 1) / gridDim.x;
    const uint32_t vb0 = min(d.nP, blockIdx.x * per_block), vb1 = min(d.nP, vb0 + per_block);
    if (threadIdx.x == 0) s_next = gpb;
    __syncthreads();

    // software pipeline over this group's vertices: the first chunk of edges
    // of its next vertex is queued (cp.async) before the current vertex's
    // angular coupling runs
    uint32_t v = vb0 + threadIdx.x / G;
    uint32_t e0 = 0, e1 = 0, axes = 0;
    int cur = 0;
    if (v < vb1) {
        e0 = __ldg(d.row + v);
        e1 = __ldg(d.row + v + 1);
        axes = __ldg(d.bmask + v);
        stage_edges_async<T>(d, e0, min(static_cast<int>(e1 - e0), G), lane, slab, scolbuf, axes != 0);
    }
    while (v < vb1) {
        uint32_t vn = 0;
        if (lane == 0) vn = vb0 + atomicAdd(&s_next, 1u);
        vn = tile.shfl(vn, 0);
        // loads whose results are used only later in this step are issued
        // first: the next vertex's edge range and boundary axes, and this
        // vertex's own row (for <x, A x> and the stored direction)
        uint32_t e0n = 0, e1n = 0, axesn = 0;
        if (vn < vb1) {
            e0n = __ldg(d.row + vn);
            e1n = __ldg(d.row + vn + 1);
            axesn = __ldg(d.bmask + vn);
        }
        const typename Out::Pre pre = fin.load(v, lane);
        EdgeAcc<T> acc[H];
#pragma unroll
        for (int h = 0; h < H; ++h) acc[h].zero();
        T *scoef = slab + cur * G * kCoefStride;
        uint32_t *scol = scolbuf + cur * G;
        for (uint32_t base = e0; base < e1; base += G) {
            const int cnt = min(static_cast<int>(e1 - base), G);
            if (base != e0) {  // further chunks of a vertex with more than G edges
                tile.sync();
                stage_edges_async<T>(d, base, cnt, lane, scoef, scol, axes != 0);
            }
            cp_async_wait_all();
            tile.sync();
            const uint32_t ul = scol[lane];
            auto accumulate = [&](const T *cp, const T(&x)[H]) {
                typename EdgeAcc<T>::Coef c;
                EdgeAcc<T>::load(cp, c);
#pragma unroll
                for (int h = 0; h < H; ++h) acc[h].add(c, x[h], lane + G * h == 0);
                if (axes) {
#pragma unroll
                    for (int h = 0; h < H; ++h) acc[h].add_bnd(c, x[h]);
                }
            };
            int jj = 0;
            for (; jj + NB <= cnt; jj += NB) {
                T x[NB][H];
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    src.row(tile.shfl(ul, jj + b), lane, x[b]);
#pragma unroll
                for (int b = 0; b < NB; ++b) accumulate(scoef + (jj + b) * kCoefStride, x[b]);
            }
            for (; jj < cnt; ++jj) {
                T x[H];
                src.row(tile.shfl(ul, jj), lane, x);
                accumulate(scoef + jj * kCoefStride, x);
            }
        }
        // queue the next vertex's first chunk into the other buffer; it lands
        // while this vertex's angular coupling runs
        cur ^= 1;
        if (vn < vb1)
            stage_edges_async<T>(d, e0n, min(static_cast<int>(e1n - e0n), G), lane, slab + cur * G * kCoefStride,
                                 scolbuf + cur * G, axesn != 0);
        e0 = e0n;
        e1 = e1n;
        const uint32_t axes_v = axes;
        axes = axesn;
        tile.sync();
        // angular coupling through shared memory
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int q = 0; q < kSymRows; ++q) sm[q * SA + lane + G * h] = acc[h].S(q);
        tile.sync();
        // the contraction rounds: the chunk sums land in `part`, then each
        // harmonic adds its chunks to its mass term
        T *part = sm + kSymRows * SA;
        contract_rounds<T, G>(d.rs, tab.run, lane, sm, part);
        tile.sync();
        T out[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const uint32_t lm = lane + G * h;
            out[h] = acc[h].mass(lm == 0);
            if (lm < slm) out[h] = sum_chunks<T>(tab.rsp, part, lm, out[h]);
        }
        // half-range boundary term from the per-axis sums B_n
        if (axes_v) {
            tile.sync();
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int n = 0; n < 3; ++n) sm[n * SA + lane + G * h] = acc[h].B(n);
            tile.sync();
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const uint32_t lm = lane + G * h;
                if (lm < slm) {
                    T acc0 = T(0), acc1 = T(0), acc2 = T(0), acc3 = T(0);
                    for (int n = 0; n < 3; ++n) {
                        if (!(axes_v & (1u << n))) continue;
                        const T *On = tab.O + static_cast<size_t>(n) * slm * LS + lm;
                        const T *Bn = sm + n * SA;
                        uint32_t lms = 0;
                        for (; lms + 3 < slm; lms += 4, On += 4 * LS) {
                            acc0 = fma(On[0], Bn[lms], acc0);
                            acc1 = fma(On[LS], Bn[lms + 1], acc1);
                            acc2 = fma(On[2 * LS], Bn[lms + 2], acc2);
                            acc3 = fma(On[3 * LS], Bn[lms + 3], acc3);
                        }
                        for (; lms < slm; ++lms, On += LS) acc0 = fma(On[0], Bn[lms], acc0);
                    }
                    out[h] += (acc0 + acc2) + (acc1 + acc3);
                }
            }
        }
        tile.sync();
        fin.store(v, lane, out, pre, dacc);
        v = vn;
    }
}

template <int G, int H, typename T, bool DOT, bool FUSEP, bool COH = false>
__device__ __forceinline__ double lhs_vertices(const OpData<T> &d, const Staged<T> &tab, unsigned char *smem_groups,
                                               const T *__restrict__ f, const T *__restrict__ pold,
                                               T *__restrict__ pnew, T *__restrict__ r, const T beta) {
    const SrcDir<G, H, T, FUSEP, COH> src{f, pold, beta, d.aslm, d.slm};
    const OutStd<G, H, T, DOT, FUSEP, COH> fin{f, pold, pnew, r, beta, d.aslm, d.slm};
    double acc[1];
    simt_vertices<G, H, T>(d, tab, smem_groups, src, fin, acc);
    return acc[0];
}


// ------------------------------------------------------ tensor-core path
// Per vertex v, everything the edge loop accumulates is one small dense
// product: with rows q = K[9], M, M0, E_x, E_y, E_z (the 14 coefficients of
// an edge record, padded to 16) and columns lm,
//   C_v[q][lm] = sum_{edges e of v} coef[e][q] * x[u_e][lm],
// i.e. C_v (16 x 8NT) = A_v (16 x edges) X_v (edges x 8NT), where A_v^T is
// the vertex's run of edge records and X_v its gathered neighbour rows.  One
// warp computes it with mma.sync: FP32 as split-TF32 (3 products per tile,
// a ~ a_hi + a_lo with a_hi, a_lo TF32; the lo*lo term is dropped) on
// m16n8k8 tiles, FP64 exactly on m8n8k4 DMMA tiles.  C goes to shared memory
// and the epilogue (lane = harmonic) takes the mass term from rows 9 / 10,
// the spatial sums S from rows 0-8 for the angular contraction and the
// per-axis boundary sums from rows 11-13.
__device__ __forceinline__ uint32_t tf32_bits(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = tf32_bits(x);
    lo = tf32_bits(x - __uint_as_float(hi));
}
// D = A B + D for one m16n8k8 tile (A row-major, B column-major fragments)
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// D = A B + D for one m8n8k4 FP64 tile
__device__ __forceinline__ void mma_f64(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <int NT>
struct TcShape {
    static constexpr int SA = NT * 8 + 1;  // row stride of the per-warp C table
};

// x_u[lm] for one harmonic (0 outside the valid range)
template <typename T, bool FUSEP, bool COH>
__device__ __forceinline__ T gather_one(const T *__restrict__ f, const T *__restrict__ pold, T beta, uint32_t u,
                                        uint32_t aslm, uint32_t lm, bool ok) {
    if (!ok) return T(0);
    T x = ldv<COH>(f + u * aslm + lm);
    if (FUSEP) x = fma(beta, ldv<COH>(pold + u * aslm + lm), x);
    return x;
}

template <int NT, typename T, bool DOT, bool FUSEP, bool COH = false>
__device__ __forceinline__ double lhs_vertices_tc(const OpData<T> &d, const Staged<T> &tab, unsigned char *smem_warps,
                                                  const T *__restrict__ f, const T *__restrict__ pold,
                                                  T *__restrict__ pnew, T *__restrict__ r, const T beta) {
    constexpr int SA = TcShape<NT>::SA;
    // wide rows are done in column passes of at most 4 n-tiles, so the
    // accumulators and gathered fragments of one pass stay in registers at
    // several resident blocks per SM
    constexpr int kPasses = (NT + 3) / 4;
    constexpr int NTH = (NT + kPasses - 1) / kPasses;
    const uint32_t slm = d.slm, aslm = d.aslm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    T *sm = reinterpret_cast<T *>(smem_warps) + warp * 16 * SA;
    const uint32_t wpb = blockDim.x / 32;
    const uint32_t nw = gridDim.x * wpb;
    double dacc = 0.0;

    for (uint32_t v = blockIdx.x * wpb + warp; v < d.nP; v += nw) {
        const uint32_t axes = __ldg(d.bmask + v);
        const uint32_t e0 = __ldg(d.row + v), e1 = __ldg(d.row + v + 1);
        if constexpr (sizeof(T) == 4) {
          for (int pass = 0; pass < kPasses; ++pass) {
            const int n0 = pass * NTH;  // first n-tile of this column pass
            float acc[NTH][4];
#pragma unroll
            for (int n = 0; n < NTH; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.0f;
            // one k-step of 8 edges: A = coefficient rows, B = gathered rows
            auto kstep = [&](const float (&a)[4], const float (&xa)[NTH], const float (&xb)[NTH]) {
                uint32_t ahi[4], alo[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) split_tf32(a[i], ahi[i], alo[i]);
#pragma unroll
                for (int n = 0; n < NTH; ++n) {
                    if (n0 + n >= NT) break;
                    uint32_t b0h, b0l, b1h, b1l;
                    split_tf32(xa[n], b0h, b0l);
                    split_tf32(xb[n], b1h, b1l);
                    mma_tf32(acc[n], alo, b0h, b1h);
                    mma_tf32(acc[n], ahi, b0l, b1l);
                    mma_tf32(acc[n], ahi, b0h, b1h);
                }
            };
            auto load_step = [&](uint32_t base, float (&a)[4], uint32_t &ua, uint32_t &ub, bool &va, bool &vb) {
                const uint32_t ea = base + t, eb = base + t + 4;
                va = ea < e1;
                vb = eb < e1;
                const size_t oa = static_cast<size_t>(va ? ea : e0) * kCoefHalf;
                const size_t ob = static_cast<size_t>(vb ? eb : e0) * kCoefHalf;
                a[0] = va ? __ldg(d.coef + oa + g) : 0.0f;
                a[1] = (va && axes) ? __ldg(d.coef_bnd + oa + g) : 0.0f;
                a[2] = vb ? __ldg(d.coef + ob + g) : 0.0f;
                a[3] = (vb && axes) ? __ldg(d.coef_bnd + ob + g) : 0.0f;
                ua = va ? __ldg(d.col + ea) : 0u;
                ub = vb ? __ldg(d.col + eb) : 0u;
            };
            // the first 16 edges: all indices and coefficients first, then all
            // row gathers, then the MMAs -- two latency stages per vertex
            {
                float a0[4], a1[4];
                uint32_t ua0, ub0, ua1, ub1;
                bool va0, vb0, va1, vb1;
                load_step(e0, a0, ua0, ub0, va0, vb0);
                load_step(e0 + 8, a1, ua1, ub1, va1, vb1);
                float xa0[NTH], xb0[NTH], xa1[NTH], xb1[NTH];
#pragma unroll
                for (int n = 0; n < NTH; ++n) {
                    const uint32_t lm = (n0 + n) * 8 + g;
                    const bool in = lm < slm;
                    xa0[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ua0, aslm, lm, va0 && in);
                    xb0[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ub0, aslm, lm, vb0 && in);
                    xa1[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ua1, aslm, lm, va1 && in);
                    xb1[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ub1, aslm, lm, vb1 && in);
                }
                kstep(a0, xa0, xb0);
                if (e0 + 8 < e1) kstep(a1, xa1, xb1);
            }
            for (uint32_t base = e0 + 16; base < e1; base += 8) {  // vertices with > 16 edges
                float a[4];
                uint32_t ua, ub;
                bool va, vb;
                load_step(base, a, ua, ub, va, vb);
                float xa[NTH], xb[NTH];
#pragma unroll
                for (int n = 0; n < NTH; ++n) {
                    const uint32_t lm = (n0 + n) * 8 + g;
                    xa[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ua, aslm, lm, va && lm < slm);
                    xb[n] = gather_one<float, FUSEP, COH>(f, pold, beta, ub, aslm, lm, vb && lm < slm);
                }
                kstep(a, xa, xb);
            }
#pragma unroll
            for (int n = 0; n < NTH; ++n) {
                if (n0 + n >= NT) break;
                const int c = (n0 + n) * 8 + 2 * t;
                sm[g * SA + c] = acc[n][0];
                sm[g * SA + c + 1] = acc[n][1];
                sm[(g + 8) * SA + c] = acc[n][2];
                sm[(g + 8) * SA + c + 1] = acc[n][3];
            }
          }
        } else {
          for (int pass = 0; pass < kPasses; ++pass) {
            const int n0 = pass * NTH;  // first n-tile of this column pass
            double acc[2][NTH][2];
#pragma unroll
            for (int n = 0; n < NTH; ++n) acc[0][n][0] = acc[0][n][1] = acc[1][n][0] = acc[1][n][1] = 0.0;
            // edges in k-steps of 4; batches of KB k-steps load everything
            // (indices, coefficients, then rows) before their MMAs
            constexpr int KB = NTH <= 4 ? 4 : 2;
            for (uint32_t base = e0; base < e1; base += 4 * KB) {
                uint32_t ua[KB];
                bool va[KB];
                double alo[KB], ahi[KB];
#pragma unroll
                for (int k = 0; k < KB; ++k) {
                    const uint32_t ea = base + 4 * k + t;
                    va[k] = ea < e1;
                    const size_t oa = static_cast<size_t>(va[k] ? ea : e0) * kCoefHalf;
                    alo[k] = va[k] ? __ldg(d.coef + oa + g) : 0.0;
                    ahi[k] = (va[k] && axes) ? __ldg(d.coef_bnd + oa + g) : 0.0;
                    ua[k] = va[k] ? __ldg(d.col + ea) : 0u;
                }
                double xa[KB][NTH];
#pragma unroll
                for (int k = 0; k < KB; ++k)
#pragma unroll
                    for (int n = 0; n < NTH; ++n) {
                        const uint32_t lm = (n0 + n) * 8 + g;
                        xa[k][n] = gather_one<double, FUSEP, COH>(f, pold, beta, ua[k], aslm, lm, va[k] && lm < slm);
                    }
#pragma unroll
                for (int k = 0; k < KB; ++k)
#pragma unroll
                    for (int n = 0; n < NTH; ++n)
                        if (n0 + n < NT) mma_f64(acc[0][n][0], acc[0][n][1], alo[k], xa[k][n]);
                if (axes)  // rows 8-15: the boundary sums (warp-uniform)
#pragma unroll
                    for (int k = 0; k < KB; ++k)
#pragma unroll
                        for (int n = 0; n < NTH; ++n)
                            if (n0 + n < NT) mma_f64(acc[1][n][0], acc[1][n][1], ahi[k], xa[k][n]);
            }
#pragma unroll
            for (int n = 0; n < NTH; ++n) {
                if (n0 + n >= NT) break;
                const int c = (n0 + n) * 8 + 2 * t;
                sm[g * SA + c] = acc[0][n][0];
                sm[g * SA + c + 1] = acc[0][n][1];
                sm[(g + 8) * SA + c] = acc[1][n][0];
                sm[(g + 8) * SA + c + 1] = acc[1][n][1];
            }
          }
        }
        __syncwarp();
        // epilogue: the contraction rounds over the C table (chunk sums into
        // rows 11-15, which the edge records leave zero), then lane = harmonic
        // adds its chunks, the mass term and the boundary term
        T *part = sm + 11 * SA;
        contract_rounds<T, 32>(d.rt, tab.run, lane, sm, part);
        __syncwarp();
        T *rv = r + static_cast<size_t>(v) * aslm;
        for (uint32_t lm = lane; lm < aslm; lm += 32) {
            T out = T(0);
            if (lm < slm) {
                T acc0 = sum_chunks<T>(tab.rsp, part, lm, sm[(lm == 0 ? kRowM0 : kRowM) * SA + lm]);
                T acc1 = T(0);
                if (axes) {
                    for (int n = 0; n < 3; ++n) {
                        if (!(axes & (1u << n))) continue;
                        const T *On = tab.O + static_cast<size_t>(n) * slm * d.cls + lm;
                        const T *Bn = sm + (kRowE + n) * SA;
                        const uint32_t ls = d.cls;
                        uint32_t lms = 0;
                        for (; lms + 1 < slm; lms += 2) {
                            acc0 = fma(On[lms * ls], Bn[lms], acc0);
                            acc1 = fma(On[(lms + 1) * ls], Bn[lms + 1], acc1);
                        }
                        if (lms < slm) acc0 = fma(On[lms * ls], Bn[lms], acc0);
                    }
                }
                out = acc0 + acc1;
            }
            rv[lm] = out;
            if (DOT || FUSEP) {
                const T xv = gather_one<T, FUSEP, COH>(f, pold, beta, v, aslm, lm, lm < slm);
                if (FUSEP) pnew[static_cast<size_t>(v) * aslm + lm] = xv;
                if (DOT) dacc += static_cast<double>(xv) * static_cast<double>(out);
            }
        }
        __syncwarp();
    }
    return dacc;
}

// ------------------------------------------------------------- policies
// An operator policy supplies the per-block vertex loop and its shared
// memory: SimtOp (groups of G lanes, H harmonics per lane, FMA pipes) or
// TcOp (one warp per vertex, NT n-tiles, tensor pipes).
// resident blocks per SM the FP32 single-harmonic SIMT kernels are compiled
// for (register cap 65536 / (256 * blocks))
#ifndef TR_SIMT_F32_MINBLOCKS
#define TR_SIMT_F32_MINBLOCKS 3
#endif
template <int G, int H, typename T>
struct SimtOp {
    static constexpr int kMinBlocks = sizeof(T) == 8 ? (H > 2 ? 1 : 2) : (H > 1 ? 2 : TR_SIMT_F32_MINBLOCKS);
    static constexpr int kLanes = G;
    static constexpr uint32_t kLS = G * H < 32 ? 32 : G * H;  // lane stride of the O table
    static constexpr bool kTc = false;
    // the persistent CG kernel runs all resident threads of an SM as one block
    static constexpr int kPersistThreads = kBlock * kMinBlocks > 1024 ? 1024 : kBlock * kMinBlocks;
    static size_t slab_bytes(int threads) { return (threads / G) * group_smem_elems<G, H, T>() * sizeof(T); }
    template <bool DOT, bool FUSEP, bool COH>
    __device__ static double run(const OpData<T> &d, const Staged<T> &tab, unsigned char *slabs, const T *f,
                                 const T *pold, T *pnew, T *r, T beta) {
        return lhs_vertices<G, H, T, DOT, FUSEP, COH>(d, tab, slabs, f, pold, pnew, r, beta);
    }
    template <bool JAC>
    __device__ static void run_sr(const OpData<T> &d, const Staged<T> &tab, unsigned char *slabs, const SrStep<T> &st,
                                  double (&dots)[3]) {
        const SrcSr<G, H, T, JAC> src{st, d.aslm, d.slm};
        const OutSr<G, H, T, JAC> fin{st, d.aslm, d.slm};
        simt_vertices<G, H, T>(d, tab, slabs, src, fin, dots);
    }
};
template <int NT, typename T>
struct TcOp {
    static constexpr int kMinBlocks = 2;  // up to 128 registers (column passes of <= 4 n-tiles)
    static constexpr int kLanes = 32;
    static constexpr uint32_t kLS = 0;  // any lane stride
    static constexpr bool kTc = true;
    static constexpr int kPersistThreads = kBlock * kMinBlocks > 1024 ? 1024 : kBlock * kMinBlocks;
    static size_t slab_bytes(int threads) { return align16((threads / 32) * 16 * TcShape<NT>::SA * sizeof(T)); }
    template <bool DOT, bool FUSEP, bool COH>
    __device__ static double run(const OpData<T> &d, const Staged<T> &tab, unsigned char *slabs, const T *f,
                                 const T *pold, T *pnew, T *r, T beta) {
        return lhs_vertices_tc<NT, T, DOT, FUSEP, COH>(d, tab, slabs, f, pold, pnew, r, beta);
    }
};

template <class Op, typename T, bool DOT, bool FUSEP, class Fin>
__global__ void __launch_bounds__(kBlock, Op::kMinBlocks) k_lhs(
    const OpData<T> d, const T *__restrict__ f, const T *__restrict__ pold, T *__restrict__ pnew,
    T *__restrict__ r, double *partials, unsigned int *counter, Fin fin, const int32_t *__restrict__ done,
    const CgScalars *__restrict__ cgs, int stage_flags) {
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Staged<T> tab = stage_tables<T>(d, smem_raw, stage_flags);
    const T beta = FUSEP ? static_cast<T>(cgs->beta) : T(0);
    const double dacc = Op::template run<DOT, FUSEP, false>(d, tab, smem_raw + tab.bytes, f, pold, pnew, r, beta);
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
            const T *c = d.coef + static_cast<size_t>(e) * kCoefHalf;
            const T *cb = d.coef_bnd + static_cast<size_t>(e) * kCoefHalf;
            const T K0 = __ldg(c), K4 = __ldg(c + 1), K8 = __ldg(c + 2), M = __ldg(c + kRowM), M0 = __ldg(c + kRowM0);
            const T E0 = __ldg(cb), E1 = __ldg(cb + 1), E2 = __ldg(cb + 2);
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
// Bounded grid barrier for a co-resident (cooperatively launched) grid.
// *count is a monotone arrival counter that the host zeroes before every
// launch; barrier number n of the launch completes when it reaches
// n * gridDim.x (`target` carries that per block).  After the block barrier
// thread 0 arrives with a release reduction (publishing the block's writes)
// and polls with acquire loads (making the other blocks' writes visible),
// then the block barrier again.  Measured on a B200 (148 blocks of 768
// threads, 20,000 barriers in one launch): 1.37 us per barrier, against
// 1.56 us for a fence + relaxed add and volatile polls with a 32 ns sleep.
// Gives up after max_polls polls, or as soon as another block has given up:
// sets *err and returns false.
constexpr unsigned int kBarrierPolls = 1u << 24;
__device__ __forceinline__ bool grid_barrier(unsigned int *count, int *err, unsigned int &target,
                                             unsigned int max_polls = kBarrierPolls) {
    __shared__ int ok;
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0) {
        ok = 1;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
        unsigned int polls = 0;
        for (;;) {
            unsigned int v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if (v >= target) break;
            if (++polls > max_polls || *reinterpret_cast<volatile int *>(err)) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

// Self-test of the bounded barrier: `rounds` barriers over the grid; block
// `skip` (if >= 0) never arrives, so the others must give up after
// max_polls polls and report through *err instead of waiting forever.
__global__ void k_barrier_selftest(unsigned int *count, int *err, int skip, int rounds, unsigned int max_polls) {
    unsigned int target = 0;
    if (static_cast<int>(blockIdx.x) == skip) return;
    for (int i = 0; i < rounds; ++i)
        if (!grid_barrier(count, err, target, max_polls)) return;
}
cudaError_t launch_barrier_selftest(int blocks, unsigned int *count, int *err, int skip, int rounds,
                                    unsigned int max_polls, cudaStream_t s) {
    void *args[] = {&count, &err, &skip, &rounds, &max_polls};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(k_barrier_selftest), blocks, 128, args, 0, s);
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
// Whether the persistent CG forms the direction inside the operator's
// gather (one grid barrier fewer per iteration, every neighbour row read
// from two vectors) or in its own vector pass before the operator.  The
// SIMT family fuses; the tensor-core family takes the separate pass unless
// built with TR_PERSIST_FUSE_TC=1 (its gathers are what bound it).
#ifndef TR_PERSIST_FUSE_TC
#define TR_PERSIST_FUSE_TC 0
#endif
#ifndef TR_PERSIST_FUSE_SIMT
#define TR_PERSIST_FUSE_SIMT 1
#endif
template <class Op>
constexpr bool kPersistFuseP = Op::kTc ? TR_PERSIST_FUSE_TC : TR_PERSIST_FUSE_SIMT;

template <class Op, typename T, bool JAC>
__global__ void __launch_bounds__(Op::kPersistThreads, 1)
    k_cg_persistent(const OpData<T> d, const PcgArgs<T> a, int stage_flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[32];
    const Staged<T> tab = stage_tables<T>(d, smem_raw, stage_flags);
    CgScalars *s = a.s;
    unsigned int target = 0;  // grid_barrier arrival target
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
        double dacc;
        if constexpr (kPersistFuseP<Op>) {
            // phase A: p = z + beta p_old inside the operator's gather, A p, <p, A p>
            dacc = Op::template run<true, true, true>(d, tab, smem_raw + tab.bytes, JAC ? a.z : a.r, pold, pnew,
                                                      a.Ap, static_cast<T>(beta));
        } else {
            // p = z + beta p_old as its own vector pass, then A p, <p, A p>:
            // the operator gathers each neighbour row once instead of two
            const T bt = static_cast<T>(beta);
            const V *zs = reinterpret_cast<const V *>(JAC ? a.z : a.r);
            for (uint32_t iv = blockIdx.x * blockDim.x + threadIdx.x; iv < a.nvec; iv += gridDim.x * blockDim.x) {
                const V zv = __ldcg(zs + iv), qv = __ldcg(reinterpret_cast<const V *>(pold) + iv);
                V pv;
#pragma unroll
                for (int q = 0; q < O::W; ++q) O::set(pv, q, fma(bt, O::get(qv, q), O::get(zv, q)));
                reinterpret_cast<V *>(pnew)[iv] = pv;
            }
            if (!grid_barrier(a.bar, a.err, target)) return;
            dacc = Op::template run<true, false, true>(d, tab, smem_raw + tab.bytes, pnew, nullptr, nullptr, a.Ap,
                                                       T(0));
        }
        const double bs = block_sum(dacc, sh);
        if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
        if (!grid_barrier(a.bar, a.err, target)) return;
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
        if (!grid_barrier(a.bar, a.err, target)) return;
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

// Single-reduction CG (see SrStep) for up to a.iters steps in one
// cooperative launch: per step one operator pass with the owner updates,
// one grid barrier, then every block derives
//   step 0:  beta_0 = 0, alpha_0 = gamma_0 / delta_0
//   step j:  beta_j = gamma_j / gamma_{j-1},
//            alpha_j = gamma_j / (delta_j - beta_j gamma_j / alpha_{j-1})
// from gamma_j = (r_j, u_j), delta_j = (w_j, u_j) and stops on ||r_j||
// (rho_j = (r_j, r_j)) like the two-reduction kernel.  After step j the
// solve has made j CG iterations and x holds x_j.
template <class Op, typename T, bool JAC>
__global__ void __launch_bounds__(Op::kPersistThreads, 1)
    k_sr_persistent(const OpData<T> d, const SrArgs<T> a, int stage_flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[32];
    const Staged<T> tab = stage_tables<T>(d, smem_raw, stage_flags);
    CgScalars *s = a.s;
    unsigned int target = 0;  // grid_barrier arrival target
    if (__ldcg(&s->done)) return;
    int j = __ldcg(&s->phase);
    const int maxit = s->maxit;
    const double tol = s->tol;
    double gamma_prev = __ldcg(&s->nrz), alpha_prev = __ldcg(&s->alpha), beta_prev = __ldcg(&s->beta);
    for (int it = 0; it < a.iters; ++it) {
        const int par = j & 1;
        SrStep<T> st;
        st.r = a.R[par ^ 1];
        st.w = a.W[par ^ 1];
        st.s = a.S[par];
        st.rn = a.R[par];
        st.wn = a.W[par];
        st.sn = a.S[par ^ 1];
        st.p = a.p;
        st.x = a.x;
        st.dinv = a.dinv;
        st.alpha = static_cast<T>(alpha_prev);
        st.beta = static_cast<T>(beta_prev);
        double dots[3];
        Op::template run_sr<JAC>(d, tab, smem_raw + tab.bytes, st, dots);
        double *part = a.partials + static_cast<size_t>(par) * 3 * gridDim.x;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double bq = block_sum(dots[q], sh);
            if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = bq;
        }
        if (!grid_barrier(a.bar, a.err, target)) return;
        double t[3];
        sum_partials<3>(part, t);
        const double gamma = t[0], delta = t[1], nr = sqrt(t[2]);
        double alpha = alpha_prev, beta = beta_prev;
        int dn = 0;
        if (!isfinite(nr) || !isfinite(gamma) || !isfinite(delta)) dn = 3;
        else if (nr < tol) dn = 1;
        else if (j >= maxit) dn = 2;
        else {
            if (j == 0) {
                beta = 0.0;
                alpha = gamma / delta;
            } else {
                beta = gamma / gamma_prev;
                alpha = gamma / (delta - beta * gamma / alpha_prev);
            }
            if (!isfinite(alpha) || !isfinite(beta)) dn = 3;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (a.hist && j >= 1 && j - 1 < a.hist_cap) a.hist[j - 1] = nr;
            s->alpha = alpha;
            s->beta = beta;
            s->nrz = gamma;
            s->rr = t[2];
            s->k = j;
            s->phase = j + 1;
            s->done = dn;
        }
        gamma_prev = gamma;
        alpha_prev = alpha;
        beta_prev = beta;
        ++j;
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

template <class Op, typename T>
static const Runs<T> &op_runs(const OpData<T> &d) {
    return Op::kTc ? d.rt : d.rs;
}
template <class Op, typename T>
static int stage_flags(const OpData<T> &d) {
    return (runs_smem_bytes<T>(op_runs<Op>(d), d.slm) <= kAngSmemBudget ? 1 : 0) |
           (O_smem_bytes<T>(d.slm, d.cls) <= kOSmemBudget ? 2 : 0) | (Op::kTc ? 4 : 0);
}
template <class Op, typename T>
static size_t lhs_smem(const OpData<T> &d, int threads) {
    const int fl = stage_flags<Op, T>(d);
    return ((fl & 1) ? runs_smem_bytes<T>(op_runs<Op>(d), d.slm) : 0) +
           ((fl & 2) ? O_smem_bytes<T>(d.slm, d.cls) : 0) + Op::slab_bytes(threads);
}
// the runs of the kernel's form were built for its lanes and the O table for
// its lane stride
template <class Op, typename T>
static bool tables_fit(const OpData<T> &d) {
    return op_runs<Op>(d).L == static_cast<uint32_t>(Op::kLanes) && op_runs<Op>(d).rounds > 0 &&
           (!Op::kLS || d.cls == Op::kLS);
}

// preferred shared-memory carveout (percent of the unified L1/shared array)
// of the operator kernels; negative leaves the driver's choice
#ifndef TR_SMEM_CARVEOUT
#define TR_SMEM_CARVEOUT -1
#endif
template <class K>
static cudaError_t opt_in_smem(K kern, size_t smem, size_t &opted) {
    if (TR_SMEM_CARVEOUT >= 0 && opted == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, TR_SMEM_CARVEOUT);
        if (e != cudaSuccess) return e;
        opted = 1;
    }
    if (smem > 48 * 1024 && smem > opted) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        opted = smem;
    }
    return cudaSuccess;
}

// Calls fn(Op()) with the operator policy of this context and precision:
// SIMT groups (G, H) from the vector stride, or tensor-core tiles NT from slm.
template <typename T, class F>
static cudaError_t with_op(const DeviceOp<T> &op, uint32_t slm, F &&fn) {
    if (op.kind == TR_OPERATOR_TENSOR) {
        const uint32_t nt = (slm + 7) / 8;
        if (nt <= 1) return fn(TcOp<1, T>());
        if (nt <= 2) return fn(TcOp<2, T>());
        if (nt <= 4) return fn(TcOp<4, T>());
        if (nt <= 6) return fn(TcOp<6, T>());
        if (nt <= 9) return fn(TcOp<9, T>());
        if (nt <= 12) return fn(TcOp<12, T>());
        return fn(TcOp<15, T>());
    }
    const uint32_t as = op.aslm;
    if (as <= 8) return fn(SimtOp<8, 1, T>());
    if (as <= 16) return fn(SimtOp<16, 1, T>());
    if (as <= 32) return fn(SimtOp<32, 1, T>());
    if (as <= 64) return fn(SimtOp<32, 2, T>());
    if (as <= 96) return fn(SimtOp<32, 3, T>());
    return fn(SimtOp<32, 4, T>());
}

template <class Op, typename T, bool DOT, bool FUSEP, class Fin>
static cudaError_t launch_one(const tr_ctx *c, const OpData<T> &d, const LhsArgs<T> &a, Fin fin, cudaStream_t s) {
    if (!tables_fit<Op>(d)) return cudaErrorInvalidValue;
    const size_t smem = lhs_smem<Op, T>(d, kBlock);
    auto kern = k_lhs<Op, T, DOT, FUSEP, Fin>;
    static size_t opted = 0;  // dynamic shared memory granted so far (per instantiation)
    cudaError_t e = opt_in_smem(kern, smem, opted);
    if (e != cudaSuccess) return e;
    // one wave of resident blocks (a partial second wave would idle most SMs)
    static int per_sm = 0;
    static size_t per_sm_smem = 0;
    if (per_sm == 0 || per_sm_smem != smem) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
        if (e != cudaSuccess) return e;
        per_sm = std::max(per_sm, 1);
        per_sm_smem = smem;
    }
    const int gpb = kBlock / Op::kLanes;
    const int grid = std::max(1, std::min(c->num_sms * per_sm, static_cast<int>((d.nP + gpb - 1) / gpb)));
    kern<<<grid, kBlock, smem, s>>>(d, a.x, a.pold, a.pnew, a.y, c->partials, c->counters, fin, a.done, a.cgs,
                                    stage_flags<Op, T>(d));
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, LhsArgs<T> a, cudaStream_t s) {
    const OpData<T> d = op.data(c->nP, c->slm);
    return with_op<T>(op, c->slm, [&](auto tag) -> cudaError_t {
        typedef decltype(tag) Op;
        switch (a.fin_kind) {
        case 0: return launch_one<Op, T, false, false>(c, d, a, FinNone(), s);
        case 1: return launch_one<Op, T, true, false>(c, d, a, FinStore{a.fin_out}, s);
        case 2: return launch_one<Op, T, true, false>(c, d, a, FinAlpha{a.cgs}, s);
        default: return launch_one<Op, T, true, true>(c, d, a, FinAlpha{a.cgs}, s);
        }
    });
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

template <class Op, typename T, bool JAC>
static cudaError_t launch_pcg(const tr_ctx *c, const OpData<T> &d, const PcgArgs<T> &a, cudaStream_t s,
                              int *grid_out) {
    if (!tables_fit<Op>(d)) return cudaErrorInvalidValue;
    auto kern = k_cg_persistent<Op, T, JAC>;
    constexpr int threads = Op::kPersistThreads;
    const size_t smem = lhs_smem<Op, T>(d, threads);
    static size_t opted = 0;
    cudaError_t e = opt_in_smem(kern, smem, opted);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    // enough blocks for the vertices, at most one wave of resident blocks
    const int gpb = threads / Op::kLanes;
    const int need = static_cast<int>((d.nP + gpb - 1) / gpb);
    const int grid = std::max(1, std::min(per_sm * c->num_sms, std::min(need, kMaxGrid)));
    *grid_out = grid;
    int flags = stage_flags<Op, T>(d);
    OpData<T> dd = d;
    PcgArgs<T> aa = a;
    void *args[] = {&dd, &aa, &flags};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), grid, threads, args, smem, s);
}

template <typename T>
cudaError_t launch_cg_persistent(const tr_ctx *c, const DeviceOp<T> &op, const PcgArgs<T> &a, cudaStream_t s,
                                 int *grid_out) {
    const OpData<T> d = op.data(c->nP, c->slm);
    const bool jac = a.dinv != nullptr;
    return with_op<T>(op, c->slm, [&](auto tag) -> cudaError_t {
        typedef decltype(tag) Op;
        return jac ? launch_pcg<Op, T, true>(c, d, a, s, grid_out) : launch_pcg<Op, T, false>(c, d, a, s, grid_out);
    });
}
template cudaError_t launch_cg_persistent<double>(const tr_ctx *, const DeviceOp<double> &, const PcgArgs<double> &,
                                                  cudaStream_t, int *);
template cudaError_t launch_cg_persistent<float>(const tr_ctx *, const DeviceOp<float> &, const PcgArgs<float> &,
                                                 cudaStream_t, int *);

template <class Op, typename T, bool JAC>
static cudaError_t launch_sr(const tr_ctx *c, const OpData<T> &d, const SrArgs<T> &a, cudaStream_t s) {
    if (!tables_fit<Op>(d)) return cudaErrorInvalidValue;
    constexpr int threads = Op::kPersistThreads;
    auto kern = k_sr_persistent<Op, T, JAC>;
    const size_t smem = lhs_smem<Op, T>(d, threads);
    static size_t opted = 0;
    cudaError_t e = opt_in_smem(kern, smem, opted);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int gpb = threads / Op::kLanes;
    const int need = static_cast<int>((d.nP + gpb - 1) / gpb);
    const int grid = std::max(1, std::min(per_sm * c->num_sms, std::min(need, kMaxGrid / 2)));
    int flags = stage_flags<Op, T>(d);
    OpData<T> dd = d;
    SrArgs<T> aa = a;
    void *args[] = {&dd, &aa, &flags};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), grid, threads, args, smem, s);
}

// the SIMT operator policies only (TR_OPERATOR_SIMT)
template <typename T>
cudaError_t launch_sr_persistent(const tr_ctx *c, const DeviceOp<T> &op, const SrArgs<T> &a, cudaStream_t s) {
    if (op.kind != TR_OPERATOR_SIMT) return cudaErrorNotSupported;
    const OpData<T> d = op.data(c->nP, c->slm);
    const bool jac = a.dinv != nullptr;
    return with_op<T>(op, c->slm, [&](auto tag) -> cudaError_t {
        typedef decltype(tag) Op;
        if constexpr (Op::kTc) {
            return cudaErrorNotSupported;
        } else {
            return jac ? launch_sr<Op, T, true>(c, d, a, s) : launch_sr<Op, T, false>(c, d, a, s);
        }
    });
}
template cudaError_t launch_sr_persistent<float>(const tr_ctx *, const DeviceOp<float> &, const SrArgs<float> &,
                                                 cudaStream_t);

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
