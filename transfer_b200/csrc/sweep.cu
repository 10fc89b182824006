// Discrete-ordinates transport sweep on the reference's tetrahedral problem
// data (no counterpart in the reference, whose solver is the even-parity
// spherical-harmonics operator of kernels.cu).  The sweep reads the same
// `tetrahedron` records (MeshData.cpp:56-76: outward face area normals s,
// kappa_volume = sigma_t V, I_p = B) and boundary `face` records.
//
// Discretisation: linear discontinuous finite elements per tetrahedron and
// ordinate, upwind coupling across faces; per (cell, ordinate) the 4x4
// system
//   L_ij  = a_j/12 + sigma_t V (1+d_ij)/20 + (1+d_ij)/12 sum_{k in, k!=i,j} a_k
//   rhs_i = sigma_s V/20 (J_i + sum_j J_j) + sigma_a V B/4
//           + sum_{k in, k!=i} a_k/12 (T_k + psi_up_{k,i}),
// a_k = -Omega.s_k (> 0 on inflow faces), T_k the sum of the three upwind
// traces on face k, solved by the adjugate formula (solve4; the
// symmetric part of L is positive definite).  J = sum_q w_q psi_q.
//
// Device layout (one GPU; SoA, cell-major):
//   s [nT][12] (face normals; a shared face stores exactly negated normals,
//   so both sides agree on which one is upwind), sigma_t V, sigma_s V,
//   sigma_a V B / 4 [nT], neighbours nbr [nT][4] (>= 0 cell, < 0 boundary
//   face -(f+1)), vertex maps across faces packed 2 bits per (face, vertex).
//   psi [nq][nT][4] (FP32 or FP64), task records [nq][nT] (uint4, below).
//
// Schedule, built once on the device (k_sched_build, one block per
// ordinate): Kahn levels over the upwind graph; when a level comes out
// empty while cells remain, the smallest unscheduled cell forms a level of
// its own and its inflow from unscheduled cells is lagged (read from the
// extra-unknown vector B, which the Krylov solver carries).
//   task[q][p] = { cell | inflow_mask << 28, up[3] } in level order, up[i]
//   the source of the i-th inflow face (ascending local face index): the
//   upstream cell's position p' in this ordinate's order, kLagBit | slot,
//   or for a boundary face kBndBit | kind << 28 | the index of its inflow
//   value (the reflective B entry, or the face for incident inflow).
//
// Sweep (k_sweep, one block per ordinate): positions in chunks (a level, or
// 256 cells of a longer one), a block barrier between chunks; each cell's
// solution goes to psi and to a shared-memory ring indexed by position, from
// which downstream cells of later levels read their upwind traces (global
// psi for older ones).  The inputs of the next chunk are staged in shared
// memory by the threads shifted by half a block while the current chunk is
// computed.  Blocks never wait on one another, so a sweep has no
// inter-block waits.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/transfer_b200.h"
#include "moments_tc.h"
#include "reduce.cuh"

namespace transfer {
tr_status set_global_error(tr_status st, const std::string &msg);
}

namespace transfer {
namespace sweep {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kLagBit = 0x80000000u;
constexpr uint32_t kCellMask = 0x0FFFFFFFu;
constexpr uint32_t kBndBit = 0x40000000u;    // boundary face: kind in bits 28-29, value index below
constexpr uint32_t kBndIndex = 0x0FFFFFFFu;
constexpr int kSchedThreads = 1024;
constexpr int kSweepThreads = 256;
constexpr int kRedGrid = 296;            // 2 x 148 SMs
constexpr int kDotGrid = 1184;           // 8 x 148 SMs: the multi-dot is HBM-bound
constexpr uint32_t kMaxLag = 1u << 22;   // lagged (cycle-breaking) faces over all ordinates
constexpr int kMaxRestart = 64;
constexpr int kMaxMoments = 16;

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
    using type = float4;
};
template <>
struct Vec4<double> {
    using type = double4;
};

template <typename T>
__device__ __forceinline__ T comp(const typename Vec4<T>::type &v, uint32_t i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

template <typename T>
struct Geom {
    const T *s;          // [nT][12]
    const T *stv;        // sigma_t V
    const T *ssv;        // sigma_s V
    const T *ext;        // sigma_a V B / 4
    const T *coef;       // [nT][4]: sigma_t V, sigma_s V, sigma_a V B / 4, 0
    const int32_t *nbr;  // [nT][4]
    const uint32_t *map; // [nT]
    const int32_t *fbc;  // [nF]
    const T *finc;       // [nF]
    const int32_t *rslot;// [nF]
};

struct Sched {
    const uint4 *task;     // [nq][nT]
    const uint32_t *lvl;   // [nq][lstride]
    const uint32_t *nlev;  // [nq]
    uint32_t lstride;
    // cells whose four faces are all inflow (only an inverted element, whose
    // shared-face normals disagree with its own, can have them): the source
    // of face 3, sorted by key q * nT + position
    const unsigned long long *f4_keys;
    const uint32_t *f4_codes;
    uint32_t n_f4;
};

template <typename T>
struct SweepArgs {
    uint32_t nT, nq;
    const T *ox, *oy, *oz;
    const T *J;        // [nT][4] or null (zero)
    const T *Bin;      // extra unknowns or null (zero)
    T *Bout;           // reflective outflow (mirrored), or null
    T *psi;            // [nq][nT][4]
    int with_ext;
    uint64_t lag_base; // offset of the lag slots in B
};

// ---- schedule -------------------------------------------------------------
struct SchedBuild {
    uint32_t nT, nq;
    const double *s;
    const int32_t *nbr;
    const double *ox, *oy, *oz;
    int32_t *indeg;     // [nq][nT]
    uint32_t *order;    // [nq][nT]
    uint32_t *pos;      // [nq][nT]
    uint8_t *mask;      // [nq][nT] inflow faces
    uint8_t *lagm;      // [nq][nT] lagged faces
    uint32_t *lvl;      // [nq][nT + 1]
    uint32_t *nlev;     // [nq]
    uint32_t *nforced;  // [nq]
};

// Omega . s without contraction, in the order ((x + y) + z): the sign
// decisions must be those of the FP64 oracle and antisymmetric across a face.
__device__ __forceinline__ double odot_rn(double ox, double oy, double oz, const double *s) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ox, s[0]), __dmul_rn(oy, s[1])), __dmul_rn(oz, s[2]));
}

__global__ void __launch_bounds__(kSchedThreads) k_sched_build(SchedBuild b) {
    __shared__ uint32_t s_n, s_min;
    const uint32_t q = blockIdx.x, nT = b.nT;
    const double ox = b.ox[q], oy = b.oy[q], oz = b.oz[q];
    int32_t *indeg = b.indeg + (size_t)q * nT;
    uint32_t *order = b.order + (size_t)q * nT, *pos = b.pos + (size_t)q * nT, *lvl = b.lvl + (size_t)q * (nT + 1);
    uint8_t *mask = b.mask + (size_t)q * nT, *lagm = b.lagm + (size_t)q * nT;
    for (uint32_t c = threadIdx.x; c < nT; c += blockDim.x) {
        uint32_t m = 0;
        int d = 0;
        for (int k = 0; k < 4; ++k) {
            double dd = odot_rn(ox, oy, oz, b.s + 12 * (size_t)c + 3 * k);
            if (dd < 0.0) {
                m |= 1u << k;
                if (b.nbr[4 * (size_t)c + k] >= 0) ++d;
            }
        }
        mask[c] = static_cast<uint8_t>(m);
        lagm[c] = 0;
        indeg[c] = d;
        pos[c] = kNone;
    }
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nT; c += blockDim.x)
        if (indeg[c] == 0) {
            uint32_t p = atomicAdd(&s_n, 1u);
            order[p] = c;
            pos[c] = p;
        }
    uint32_t head = 0, minrem = 0, forced = 0;
    for (uint32_t L = 0;; ++L) {
        __syncthreads();
        uint32_t n = s_n;
        __syncthreads();
        if (head == n) {
            if (n == nT) {
                if (threadIdx.x == 0) {
                    lvl[L] = nT;
                    b.nlev[q] = L;
                    b.nforced[q] = forced;
                }
                return;
            }
            // stalled on a cycle: the smallest unscheduled cell forms a level
            if (threadIdx.x == 0) s_min = nT;
            __syncthreads();
            for (uint32_t c = minrem + threadIdx.x; c < nT; c += blockDim.x)
                if (pos[c] == kNone) {
                    atomicMin(&s_min, c);
                    break;
                }
            __syncthreads();
            const uint32_t c = s_min;
            minrem = c;
            ++forced;
            if (threadIdx.x == 0) {
                uint32_t lg = 0;
                for (int k = 0; k < 4; ++k) {
                    int32_t u = b.nbr[4 * (size_t)c + k];
                    if (u >= 0 && (mask[c] >> k & 1u) && pos[u] == kNone) lg |= 1u << k;
                }
                lagm[c] = static_cast<uint8_t>(lg);
                indeg[c] = -(1 << 20);
                order[n] = c;
                pos[c] = n;
                s_n = n + 1;
            }
            __syncthreads();
            n = n + 1;
        }
        if (threadIdx.x == 0) lvl[L] = head;
        for (uint32_t i = head + threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t c = order[i];
            for (int k = 0; k < 4; ++k) {
                const int32_t d = b.nbr[4 * (size_t)c + k];
                if (d < 0) continue;
                if (!(odot_rn(ox, oy, oz, b.s + 12 * (size_t)c + 3 * k) > 0.0)) continue;
                if (atomicSub(&indeg[d], 1) == 1) {
                    uint32_t p = atomicAdd(&s_n, 1u);
                    order[p] = static_cast<uint32_t>(d);
                    pos[d] = p;
                }
            }
        }
        head = n;
    }
}

// lagged faces -> list of keys ((q * nT + c) * 4 + k)
__global__ void k_lag_collect(uint32_t nT, uint32_t nq, const uint8_t *lagm, unsigned long long *keys,
                              unsigned int *count) {
    const uint64_t n = (uint64_t)nT * nq;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t m = lagm[i];
        for (int k = 0; k < 4; ++k)
            if (m >> k & 1u) {
                unsigned int slot = atomicAdd(count, 1u);
                if (slot < kMaxLag) keys[slot] = i * 4 + k;
            }
    }
}

__global__ void k_records(uint32_t nT, uint32_t nq, const uint32_t *order, const uint32_t *pos, const uint8_t *mask,
                          const uint8_t *lagm, const int32_t *nbr, const int32_t *fbc, const int32_t *rslot,
                          const uint32_t *rent, const unsigned long long *lag_keys, uint32_t nlag, uint4 *task,
                          unsigned long long *f4_keys, uint32_t *f4_codes, unsigned int *f4_count) {
    const uint64_t n = (uint64_t)nT * nq;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t q = static_cast<uint32_t>(i / nT);
        const uint32_t c = order[i];
        const uint64_t qc = (uint64_t)q * nT + c;
        const uint32_t m = mask[qc], lg = lagm[qc];
        uint32_t up[3] = {0u, 0u, 0u};
        int t = 0;
        for (int k = 0; k < 4; ++k) {
            if (!(m >> k & 1u)) continue;
            const int32_t nb = nbr[4 * (size_t)c + k];
            uint32_t code;
            if (nb < 0) {  // boundary: kind and the index of its inflow value
                const int32_t f = -nb - 1;
                const uint32_t bc = static_cast<uint32_t>(fbc[f]);
                const uint32_t idx = bc == TR_BC_REFLECTIVE ? rent[static_cast<size_t>(rslot[f]) * nq + q]
                                                            : static_cast<uint32_t>(f);
                code = kBndBit | (bc << 28) | idx;
            } else if (lg >> k & 1u) {
                const unsigned long long key = qc * 4 + k;
                uint32_t lo = 0, hi = nlag;  // lag keys sorted ascending
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (lag_keys[mid] < key) lo = mid + 1;
                    else hi = mid;
                }
                code = kLagBit | lo;
            } else {
                code = pos[(size_t)q * nT + nb];
            }
            if (t < 3) {
                up[t] = code;
            } else {
                const unsigned int slot = atomicAdd(f4_count, 1u);
                if (slot < kMaxLag) {
                    f4_keys[slot] = i;
                    f4_codes[slot] = code;
                }
            }
            ++t;
        }
        task[i] = make_uint4(c | (m << 28), up[0], up[1], up[2]);
    }
}

// ---- the sweep --------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void load_s(const T *s, T (&v)[12]);
template <>
__device__ __forceinline__ void load_s<float>(const float *s, float (&v)[12]) {
    const float4 *p = reinterpret_cast<const float4 *>(s);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float4 t = __ldg(p + i);
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
    }
}
template <>
__device__ __forceinline__ void load_s<double>(const double *s, double (&v)[12]) {
    const double2 *p = reinterpret_cast<const double2 *>(s);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double2 t = __ldg(p + i);
        v[2 * i] = t.x;
        v[2 * i + 1] = t.y;
    }
}

template <typename T>
__device__ __forceinline__ typename Vec4<T>::type load_v4(const T *p);
template <>
__device__ __forceinline__ float4 load_v4<float>(const float *p) {
    return *reinterpret_cast<const float4 *>(p);
}
template <>
__device__ __forceinline__ double4 load_v4<double>(const double *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = q[0], b = q[1];
    return make_double4(a.x, a.y, b.x, b.y);
}

// Staging of the tasks' inputs in shared memory.  Everything a task reads
// that does not depend on this sweep's results -- its record, face normals,
// coefficients and vertex map, scalar-flux source and the inflow values of
// its boundary and lagged faces -- is copied into a slot indexed by the
// task's position.  Positions are processed in chunks of up to 256 (a level,
// or a part of a long one); while one chunk is computed, the slots of the next
// are filled with cp.async by threads shifted by half a block -- on the
// typical level of fewer than 128 cells, threads that compute nothing -- and
// the copies are waited for before the chunk barrier.  The computing threads
// thus only do arithmetic, shared-memory reads and the barrier.
constexpr uint32_t kSlots = 2 * kSweepThreads;  // two chunks of positions in flight
template <typename T>
struct Slots {
    static constexpr int kR = 16 / sizeof(T);          // reals per 16-byte unit
    static constexpr int kRec = 0, kS = 1, kJ = kS + 12 / kR, kBv = kJ + 4 / kR, kCoef = kBv + 12 / kR;
    static constexpr int kUnits = kCoef + 4 / kR;
    unsigned char *base;
    __device__ __forceinline__ unsigned char *unit(uint32_t slot, int u) const {
        return base + (static_cast<size_t>(u) * kSlots + slot) * 16;
    }
    // N reals of consecutive units from u0 into registers (16-byte shared loads)
    template <int N>
    __device__ __forceinline__ void load(uint32_t slot, int u0, T (&out)[N]) const {
#pragma unroll
        for (int i = 0; i < N / kR; ++i) {
            const uint4 v = *reinterpret_cast<const uint4 *>(unit(slot, u0 + i));
            memcpy(&out[i * kR], &v, 16);
        }
    }
};
// Shared-memory shape of a sweep block: the ring of recent psi by position,
// the staging slots and the level pointers of its ordinate (staged when
// there are at most level_cap levels, else read from global memory).  The
// full shape (FP32 154 KB, FP64 187 KB) fits one block per SM; the small
// FP32 shape (16 KiB ring, 1024 staged levels: 94 KB) fits two, for sets of
// more ordinates than SMs.  Measured (FP32, one sweep, before the staging of
// upwind traces older than the ring): Milne slab, 112 ordinates, 1.40 ms
// full / 1.58 ms small; stellar sphere, 308 ordinates, 190 ms full / 142 ms
// small.
template <typename T>
constexpr size_t slots_bytes() { return static_cast<size_t>(Slots<T>::kUnits) * kSlots * 16; }
// Task records are fetched one chunk earlier than the rest of a slot: while
// chunk i is computed, the records of chunk i + 2 are copied (cp.async) into
// a ring of three chunks' positions, and the slots of chunk i + 1 are filled
// from records already in shared memory.  Each chunk's staging is then one
// global-memory round trip (record-dependent loads only), not two (record,
// then what it names).
constexpr uint32_t kRecSlots = 3 * kSweepThreads;
constexpr size_t recs_bytes = static_cast<size_t>(kRecSlots) * 16;
template <typename T, bool SMALL>
struct SweepShape {
    static constexpr int ring_bytes = SMALL ? 16 * 1024 : (sizeof(T) == 4 ? 64 * 1024 : 32 * 1024);
    static constexpr uint32_t level_cap = SMALL ? 1024 : 4096;
    static constexpr size_t smem = ring_bytes + slots_bytes<T>() + recs_bytes + 4ull * (level_cap + 1);
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src));
}
template <int N>
__device__ __forceinline__ void cp_async_small(void *dst, const void *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(N));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

// fills the slot of position p (record, normals, source, coefficients and
// the inflow values of non-interior faces, zeros where there are none).  An
// interior inflow whose upwind position is already done (< done_end) but
// will have left the ring of R positions when p's chunk (ending at e_next)
// runs gets the upwind cell's psi staged too, from global psi (OLD: the
// shapes whose ring is short enough for that to happen often).
template <typename T, bool OLD>
__device__ __forceinline__ void stage_task(const Slots<T> &S, uint32_t p, const uint4 *recs, const Geom<T> &g,
                                           const SweepArgs<T> &a, uint32_t done_end, uint32_t e_next, uint32_t R,
                                           const T *psi) {
    using Sl = Slots<T>;
    const uint32_t sl = p % kSlots;
    const uint4 rec = recs[p % kRecSlots];
    *reinterpret_cast<uint4 *>(S.unit(sl, Sl::kRec)) = rec;
    const uint32_t c = rec.x & kCellMask, mask = rec.x >> 28;
#pragma unroll
    for (int u = 0; u < 12 / Sl::kR; ++u) cp_async16(S.unit(sl, Sl::kS + u), g.s + 12 * (size_t)c + u * Sl::kR);
    if (a.J) {
#pragma unroll
        for (int u = 0; u < 4 / Sl::kR; ++u) cp_async16(S.unit(sl, Sl::kJ + u), a.J + 4 * (size_t)c + u * Sl::kR);
    }
#pragma unroll
    for (int u = 0; u < 4 / Sl::kR; ++u) cp_async16(S.unit(sl, Sl::kCoef + u), g.coef + 4 * (size_t)c + u * Sl::kR);
    int t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!(mask >> k & 1u) || t >= 3) continue;
        const uint32_t code = t == 0 ? rec.y : t == 1 ? rec.z : rec.w;
        const int u0 = Sl::kBv + t * (4 / Sl::kR);
        const T *src = nullptr;
        bool bcast = false;
        if (code & kLagBit) {
            if (a.Bin) src = a.Bin + a.lag_base + 4 * (size_t)(code & ~kLagBit);
        } else if (code & kBndBit) {
            const uint32_t type = (code >> 28) & 3u, idx = code & kBndIndex;
            if (type == TR_BC_REFLECTIVE && a.Bin) {
                src = a.Bin + 4 * (size_t)idx;
            } else if (type == TR_BC_INCIDENT && a.with_ext) {
                src = g.finc + idx;
                bcast = true;
            }
        } else if (OLD && code < done_end && code + R < e_next) {
            src = psi + 4 * (size_t)__ldg(g.nbr + 4 * (size_t)c + k);  // the upwind cell, in its vertex order
        } else {
            ++t;
            continue;
        }
        if (src && !bcast) {
#pragma unroll
            for (int u = 0; u < 4 / Sl::kR; ++u) cp_async16(S.unit(sl, u0 + u), src + u * Sl::kR);
        } else if (src) {
#pragma unroll
            for (int e = 0; e < 4; ++e)
                cp_async_small<sizeof(T)>(S.unit(sl, u0 + e / Sl::kR) + (e % Sl::kR) * sizeof(T), src);
        } else {
#pragma unroll
            for (int u = 0; u < 4 / Sl::kR; ++u) *reinterpret_cast<uint4 *>(S.unit(sl, u0 + u)) = make_uint4(0, 0, 0, 0);
        }
        ++t;
    }
}

// the chunk after [c0, ...) of level L: the rest of the level, or the next
// level; false when none
__device__ __forceinline__ bool next_chunk(uint32_t &L, uint32_t &c0, const uint32_t *lvl, uint32_t nl) {
    if (c0 + kSweepThreads < lvl[L + 1]) {
        c0 += kSweepThreads;
        return true;
    }
    if (L + 1 < nl) {
        ++L;
        c0 = lvl[L];
        return true;
    }
    return false;
}

// stages the chunk [c0, min(c0 + 256, end of level L)) from threads shifted
// by half a block, while positions below done_end are complete
template <typename T, bool OLD>
__device__ __forceinline__ void stage_chunk(const Slots<T> &S, uint32_t L, uint32_t c0, const uint32_t *lvl,
                                            const uint4 *recs, const Geom<T> &g, const SweepArgs<T> &a,
                                            uint32_t done_end, uint32_t R, const T *psi) {
    const uint32_t e = min(c0 + kSweepThreads, lvl[L + 1]);
    const uint32_t p = c0 + ((threadIdx.x + kSweepThreads / 2) % kSweepThreads);
    if (p < e) stage_task<T, OLD>(S, p, recs, g, a, done_end, e, R, psi);
}

// copies the task records of the chunk [c0, min(c0 + 256, end of level L))
// into the record ring (not committed: the caller's commit covers them)
__device__ __forceinline__ void fetch_records(uint4 *recs, uint32_t L, uint32_t c0, const uint32_t *lvl,
                                              const uint4 *task) {
    const uint32_t e = min(c0 + kSweepThreads, lvl[L + 1]);
    const uint32_t p = c0 + ((threadIdx.x + kSweepThreads / 2) % kSweepThreads);
    if (p < e) cp_async16(recs + p % kRecSlots, task + p);
}

// upwind trace of one inflow face from its source code
template <typename T>
__device__ __forceinline__ void inflow_values(uint32_t code, const T *staged, bool staged_ok, const Geom<T> &g,
                                              const SweepArgs<T> &a, const typename Vec4<T>::type *ring,
                                              uint32_t R, uint32_t e0, const T *psi, uint32_t c, int k, uint32_t mp,
                                              T (&up)[4]) {
    if (code & kLagBit) {
        if (a.Bin) {
            const T *bp = staged_ok ? staged : a.Bin + a.lag_base + 4 * (size_t)(code & ~kLagBit);
#pragma unroll
            for (int j = 0; j < 4; ++j) up[j] = bp[j];
        }
    } else if (code & kBndBit) {
        const uint32_t type = (code >> 28) & 3u, idx = code & kBndIndex;
        if (type == TR_BC_REFLECTIVE && a.Bin) {
            const T *bp = staged_ok ? staged : a.Bin + 4 * (size_t)idx;
#pragma unroll
            for (int j = 0; j < 4; ++j) up[j] = bp[j];
        } else if (type == TR_BC_INCIDENT && a.with_ext) {
            const T v = staged_ok ? staged[0] : __ldg(g.finc + idx);
#pragma unroll
            for (int j = 0; j < 4; ++j) up[j] = v;
        }
    } else {
        typename Vec4<T>::type v;
        if (code + R >= e0) {
            v = ring[code % R];
        } else {
            const int32_t nb = __ldg(g.nbr + 4 * (size_t)c + k);
            v = load_v4<T>(psi + 4 * (size_t)nb);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) up[j] = comp<T>(v, (mp >> (2 * (4 * k + j))) & 3u);
    }
}

// x = L^-1 r for one cell by the adjugate (2x2 minors of rows 0-1 and 2-3,
// one division): a short dependency chain with much independent work, where
// Gaussian elimination would chain four pivots and eight divisions.  The
// matrices are well conditioned (positive definite symmetric part).
template <typename T>
__device__ __forceinline__ void solve4(const T (&a)[4][4], const T (&r)[4], T (&x)[4]) {
    const T s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1], s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    const T s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3], s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    const T s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3], s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    const T c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3], c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    const T c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2], c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    const T c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2], c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    const T det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    const T b[4][4] = {
        {a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3, -a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3,
         a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3, -a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3},
        {-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1, a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1,
         -a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1, a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1},
        {a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0, -a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0,
         a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0, -a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0},
        {-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0, a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0,
         -a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0, a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0}};
    const T inv = T(1) / det;
#pragma unroll
    for (int i = 0; i < 4; ++i) x[i] = (b[i][0] * r[0] + b[i][1] * r[1] + b[i][2] * r[2] + b[i][3] * r[3]) * inv;
}

// one ordinate q of one problem: the body of k_sweep and k_sweep_batch
template <typename T, bool SMALL>
__device__ __forceinline__ void sweep_block(const Geom<T> &g, const Sched &sc, const SweepArgs<T> &a,
                                            const uint32_t q) {
    using V = typename Vec4<T>::type;
    using Sl = Slots<T>;
    using Shape = SweepShape<T, SMALL>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr uint32_t R = Shape::ring_bytes / sizeof(V);
    // stage upwind traces older than the ring (FP64 and the small shape: a
    // ring of 1,024 positions; the full FP32 ring of 4,096 rarely misses)
    constexpr bool kOld = sizeof(T) == 8 || SMALL;
    V *ring = reinterpret_cast<V *>(smem_raw);
    const Slots<T> SL{smem_raw + Shape::ring_bytes};
    const uint32_t nT = a.nT;
    const T ox = a.ox[q], oy = a.oy[q], oz = a.oz[q];
    const uint4 *task = sc.task + (size_t)q * nT;
    const uint32_t nl = sc.nlev[q];
    const uint32_t *lvl = sc.lvl + (size_t)q * sc.lstride;
    if (nl <= Shape::level_cap) {
        uint32_t *lv = reinterpret_cast<uint32_t *>(smem_raw + Shape::ring_bytes + slots_bytes<T>() + recs_bytes);
        for (uint32_t L = threadIdx.x; L <= nl; L += blockDim.x) lv[L] = __ldg(lvl + L);
        __syncthreads();
        lvl = lv;
    }
    if (nl == 0) return;
    T *psi = a.psi + (size_t)q * nT * 4;
    const T c12 = T(1) / T(12), c20 = T(1) / T(20);

    uint4 *recs = reinterpret_cast<uint4 *>(smem_raw + Shape::ring_bytes + slots_bytes<T>());
    uint32_t L = 0, c0 = lvl[0];
    uint32_t prev_c0 = 0;  // positions below it were complete when this chunk was staged
    {  // records of the first two chunks, then the first chunk's slots
        fetch_records(recs, L, c0, lvl, task);
        uint32_t L1 = L, c1 = c0;
        if (next_chunk(L1, c1, lvl, nl)) fetch_records(recs, L1, c1, lvl, task);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        stage_chunk<T, kOld>(SL, L, c0, lvl, recs, g, a, prev_c0, R, psi);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
    }
    for (;;) {
        const uint32_t e0 = min(c0 + kSweepThreads, lvl[L + 1]);  // this chunk is [c0, e0)
        uint32_t nL = L, nc0 = c0;
        const bool more = next_chunk(nL, nc0, lvl, nl);
        if (more) {
            uint32_t nnL = nL, nnc0 = nc0;
            if (next_chunk(nnL, nnc0, lvl, nl)) fetch_records(recs, nnL, nnc0, lvl, task);
            stage_chunk<T, kOld>(SL, nL, nc0, lvl, recs, g, a, c0, R, psi);
        }
        cp_async_commit();
        const uint32_t p = c0 + threadIdx.x;
        if (p < e0) {
            const uint32_t sl = p % kSlots;
            const uint4 rec = *reinterpret_cast<const uint4 *>(SL.unit(sl, Sl::kRec));
            const uint32_t c = rec.x & kCellMask, mask = rec.x >> 28;
            T sv[12], cf[4];
            SL.template load<12>(sl, Sl::kS, sv);
            SL.template load<4>(sl, Sl::kCoef, cf);
            T av[4], al[4], Ain = T(0);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                av[k] = -(ox * sv[3 * k] + oy * sv[3 * k + 1] + oz * sv[3 * k + 2]);
                al[k] = (mask >> k & 1u) ? av[k] : T(0);
                Ain += al[k];
            }
            const T stv = cf[0], ssv = cf[1];
            const T ext = a.with_ext ? cf[2] : T(0);
            T Jc[4] = {T(0), T(0), T(0), T(0)};
            if (a.J) SL.template load<4>(sl, Sl::kJ, Jc);
            const T Js = Jc[0] + Jc[1] + Jc[2] + Jc[3];
            T Lm[4][4], r[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const T face = (i == j) ? T(2) * (Ain - al[i]) : (Ain - al[i] - al[j]);
                    Lm[i][j] = av[j] * c12 + stv * (i == j ? T(2) : T(1)) * c20 + face * c12;
                }
                r[i] = ssv * c20 * (Jc[i] + Js) + ext;
            }
            uint32_t mp;
            memcpy(&mp, &cf[3], sizeof(uint32_t));  // the vertex map rides in the fourth coefficient
            const T *ring_s = reinterpret_cast<const T *>(ring);
            int t = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!(mask >> k & 1u)) continue;
                T up[4] = {T(0), T(0), T(0), T(0)};
                if (t < 3) {
                    const uint32_t code = t == 0 ? rec.y : t == 1 ? rec.z : rec.w;
                    if (code & (kLagBit | kBndBit)) {
                        SL.template load<4>(sl, Sl::kBv + t * (4 / Sl::kR), up);
                    } else if (code + R >= e0) {  // upwind trace from the ring
                        const T *src = ring_s + 4 * (size_t)(code % R);
#pragma unroll
                        for (int j = 0; j < 4; ++j) up[j] = src[(mp >> (2 * (4 * k + j))) & 3u];
                    } else if (kOld && code < prev_c0) {  // older than the ring, staged with the slot
                        T upc[4];
                        SL.template load<4>(sl, Sl::kBv + t * (4 / Sl::kR), upc);
                        V v;  // selects below, not a dynamically indexed array
                        v.x = upc[0];
                        v.y = upc[1];
                        v.z = upc[2];
                        v.w = upc[3];
#pragma unroll
                        for (int j = 0; j < 4; ++j) up[j] = comp<T>(v, (mp >> (2 * (4 * k + j))) & 3u);
                    } else {                      // older than the ring: global psi
                        const T *src = psi + 4 * (size_t)__ldg(g.nbr + 4 * (size_t)c + k);
#pragma unroll
                        for (int j = 0; j < 4; ++j) up[j] = src[(mp >> (2 * (4 * k + j))) & 3u];
                    }
                } else {
                    // the fourth inflow face of an inverted element: its source from the side table
                    const unsigned long long key = (unsigned long long)q * nT + p;
                    uint32_t lo = 0, hi = sc.n_f4;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (sc.f4_keys[mid] < key) lo = mid + 1;
                        else hi = mid;
                    }
                    if (lo < sc.n_f4 && sc.f4_keys[lo] == key)
                        inflow_values<T>(sc.f4_codes[lo], nullptr, false, g, a, ring, R, e0, psi, c, k, mp, up);
                }
                ++t;
                up[k] = T(0);
                const T Tk = up[0] + up[1] + up[2] + up[3];
                const T ak = av[k] * c12;
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (i != k) r[i] += ak * (Tk + up[i]);
            }
            T o[4];
            solve4<T>(Lm, r, o);
            V out;
            out.x = o[0];
            out.y = o[1];
            out.z = o[2];
            out.w = o[3];
            if constexpr (sizeof(T) == 4) {
                *reinterpret_cast<float4 *>(psi + 4 * (size_t)c) = out;
            } else {
                double2 *dst = reinterpret_cast<double2 *>(psi + 4 * (size_t)c);
                dst[0] = make_double2(o[0], o[1]);
                dst[1] = make_double2(o[2], o[3]);
            }
            ring[p % R] = out;
        }
        cp_async_wait<0>();
        __syncthreads();
        if (!more) break;
        L = nL;
        prev_c0 = c0;
        c0 = nc0;
    }
}
template <typename T, bool SMALL>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(Geom<T> g, Sched sc, SweepArgs<T> a) {
    sweep_block<T, SMALL>(g, sc, a, blockIdx.x);
}
// several problems in one launch: job j owns blocks [block0, block0 + nq)
template <typename T>
struct SweepJob {
    Geom<T> g;
    Sched sc;
    SweepArgs<T> a;
    uint32_t block0;
};
template <typename T, bool SMALL>
__global__ void __launch_bounds__(kSweepThreads) k_sweep_batch(const SweepJob<T> *__restrict__ jobs, int njobs) {
    int lo = 0, hi = njobs - 1;  // the last job with block0 <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (jobs[mid].block0 <= blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const Geom<T> g = jobs[lo].g;
    const Sched sc = jobs[lo].sc;
    const SweepArgs<T> a = jobs[lo].a;
    sweep_block<T, SMALL>(g, sc, a, blockIdx.x - jobs[lo].block0);
}

// The same tasks taken from a queue: a persistent grid (as many blocks as are
// resident) in which each block draws task indices from an atomic ticket
// until they run out.  Task t is ordinate t - block0 of the job owning it, in
// the jobs' order (largest problems first).  The ticket must be zero at launch
// (the host clears it before each launch); every draw consumes one index, so
// the loop ends after at most ntasks / gridDim.x + 1 draws per block.
template <typename T, bool SMALL>
__global__ void __launch_bounds__(kSweepThreads) k_sweep_queue(const SweepJob<T> *__restrict__ jobs, int njobs,
                                                               uint32_t ntasks, unsigned int *ticket) {
    __shared__ uint32_t drawn;
    for (;;) {
        if (threadIdx.x == 0) drawn = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t t = drawn;
        __syncthreads();  // all have read it before thread 0 draws again
        if (t >= ntasks) break;
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (jobs[mid].block0 <= t) lo = mid;
            else hi = mid - 1;
        }
        const Geom<T> g = jobs[lo].g;
        const Sched sc = jobs[lo].sc;
        const SweepArgs<T> a = jobs[lo].a;
        sweep_block<T, SMALL>(g, sc, a, t - jobs[lo].block0);
        __syncthreads();  // the block's shared memory is free for the next task
    }
}

// B_out of the reflective faces: the inflow of each (face, incoming q)
// entry is the outflow of the mirrored ordinate at the same face (same
// vertex values; the face's opposite vertex left zero)
template <typename T>
__global__ void k_reflect_out(uint32_t nT, uint32_t nent, const uint32_t *ent_cell, const uint32_t *ent_qout,
                              const T *psi, T *Bout) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += gridDim.x * blockDim.x) {
        const uint32_t ck = ent_cell[e], c = ck >> 2, k = ck & 3u;
        typename Vec4<T>::type v = load_v4<T>(psi + ((size_t)ent_qout[e] * nT + c) * 4);
        if (k == 0) v.x = T(0);
        if (k == 1) v.y = T(0);
        if (k == 2) v.z = T(0);
        if (k == 3) v.w = T(0);
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4 *>(Bout + 4 * (size_t)e) = v;
        } else {
            double2 *dst = reinterpret_cast<double2 *>(Bout + 4 * (size_t)e);
            dst[0] = make_double2(v.x, v.y);
            dst[1] = make_double2(v.z, v.w);
        }
    }
}

// B_out lag slots: the upstream trace of this sweep
template <typename T>
__global__ void k_lag_out(uint32_t nT, uint32_t nlag, const unsigned long long *keys, const int32_t *nbr,
                          const uint32_t *map, const T *psi, T *Bout_lag) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nlag; l += gridDim.x * blockDim.x) {
        const unsigned long long key = keys[l];
        const uint32_t k = static_cast<uint32_t>(key & 3u);
        const uint64_t qc = key >> 2;
        const uint32_t q = static_cast<uint32_t>(qc / nT), c = static_cast<uint32_t>(qc % nT);
        const int32_t u = nbr[4 * (size_t)c + k];
        const uint32_t mp = map[c];
        for (int j = 0; j < 4; ++j)
            Bout_lag[4 * (size_t)l + j] =
                (j == (int)k) ? T(0) : psi[((size_t)q * nT + u) * 4 + ((mp >> (2 * (4 * k + j))) & 3u)];
    }
}

// J[c][j] = sum_q w_q psi_q[c][j], FP64 accumulation in ordinate order
template <typename T>
__global__ void k_scalar_flux(uint32_t nT, uint32_t nq, const double *w, const T *psi, double *J) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nT; c += gridDim.x * blockDim.x) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (uint32_t q = 0; q < nq; ++q) {
            const typename Vec4<T>::type v = load_v4<T>(psi + ((size_t)q * nT + c) * 4);
            const double wq = __ldg(w + q);
            a0 += wq * static_cast<double>(v.x);
            a1 += wq * static_cast<double>(v.y);
            a2 += wq * static_cast<double>(v.z);
            a3 += wq * static_cast<double>(v.w);
        }
        double2 *dst = reinterpret_cast<double2 *>(J + 4 * (size_t)c);
        dst[0] = make_double2(a0, a1);
        dst[1] = make_double2(a2, a3);
    }
}

// moments mom[m][c][j] = sum_q W[m][q] psi_q[c][j], W = w_q Y_m(Omega_q)
template <typename T, int NM>
__global__ void k_moments_simt(uint32_t nT, uint32_t nq, const double *W, const T *psi, double *mom) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nT; c += gridDim.x * blockDim.x) {
        double acc[NM][4];
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[m][0] = acc[m][1] = acc[m][2] = acc[m][3] = 0.0;
        for (uint32_t q = 0; q < nq; ++q) {
            const typename Vec4<T>::type v = load_v4<T>(psi + ((size_t)q * nT + c) * 4);
#pragma unroll
            for (int m = 0; m < NM; ++m) {
                const double wq = __ldg(W + (size_t)m * nq + q);
                acc[m][0] += wq * static_cast<double>(v.x);
                acc[m][1] += wq * static_cast<double>(v.y);
                acc[m][2] += wq * static_cast<double>(v.z);
                acc[m][3] += wq * static_cast<double>(v.w);
            }
        }
#pragma unroll
        for (int m = 0; m < NM; ++m)
#pragma unroll
            for (int j = 0; j < 4; ++j) mom[(size_t)m * 4 * nT + 4 * (size_t)c + j] = acc[m][j];
    }
}

// All 16 moments (l <= 3) of FP64 psi, streamed like the scalar flux: each
// thread owns two consecutive vertex values (rows 2 t, 2 t + 1 of the 4 nT;
// a warp reads 512 contiguous bytes of each ordinate row) and keeps their
// 16 moment sums, 32 FP64 registers, so that more warps stay resident than
// with the 64 sums of a whole cell; the weights of 32 ordinates at a time
// sit in shared memory.  Same FP64 sums in the same ordinate order as
// k_moments_simt<double, 16>.
constexpr int kMom64Chunk = 32;
__global__ void __launch_bounds__(256) k_moments_f64_16(uint32_t nT, uint32_t nq, const double *W, const double *psi,
                                                         double *mom) {
    __shared__ __align__(16) double ws[kMom64Chunk][16];
    const uint64_t M2 = 2ull * nT;  // row pairs
    const uint64_t stride = 4ull * nT;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < M2; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r2 = base + threadIdx.x;
        const bool live = r2 < M2;
        double acc[16][2];
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m][0] = acc[m][1] = 0.0;
        for (uint32_t q0 = 0; q0 < nq; q0 += kMom64Chunk) {
            const uint32_t nc = min(static_cast<uint32_t>(kMom64Chunk), nq - q0);
            __syncthreads();  // the previous chunk's weights have been read
            for (uint32_t i = threadIdx.x; i < kMom64Chunk * 16; i += blockDim.x) {
                const uint32_t qq = i >> 4, m = i & 15u;
                ws[qq][m] = qq < nc ? __ldg(W + (size_t)m * nq + q0 + qq) : 0.0;
            }
            __syncthreads();
            if (live) {
                const double2 *pr = reinterpret_cast<const double2 *>(psi + (size_t)q0 * stride) + r2;
                for (uint32_t qq = 0; qq < nc; ++qq) {
                    const double2 v = pr[(size_t)qq * (stride / 2)];
                    const double2 *wq = reinterpret_cast<const double2 *>(ws[qq]);
#pragma unroll
                    for (int h = 0; h < 8; ++h) {
                        const double2 w2 = wq[h];
                        acc[2 * h][0] += w2.x * v.x;
                        acc[2 * h][1] += w2.x * v.y;
                        acc[2 * h + 1][0] += w2.y * v.x;
                        acc[2 * h + 1][1] += w2.y * v.y;
                    }
                }
            }
        }
        if (live) {
#pragma unroll
            for (int m = 0; m < 16; ++m)
                reinterpret_cast<double2 *>(mom + (size_t)m * stride)[r2] = make_double2(acc[m][0], acc[m][1]);
        }
    }
}

// Moments of FP32 psi on the tensor cores in split TF32 (3 products, FP32
// accumulation): D[r][n] = sum_q A[r][q] W[n][q] with A[r][q] = psi[q][r]
// (r = 4c + j over the M = 4 nT vertex values), N = 16 harmonics (l <= 3).
// One warp per 16 rows, mma.sync m16n8k8 tf32; A fragments straight from
// global memory (lanes of equal k read 8 consecutive rows: whole 32-byte
// sectors), W split into TF32 hi/lo parts in shared memory.
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// The block stages psi through shared memory in stages of kMomK ordinates x
// kMomRows rows (cell vertices), copied with 16-byte cp.async so that each
// ordinate's rows are read as whole 1 KB runs, kMomStages stages in
// flight; each warp then builds its MMA fragments (two 16-row tiles sharing
// each B fragment) from the stage
// (row stride padded to kMomRows + 8 words: the fragment reads hit 32
// distinct banks).  Persistent: the block stages the split weights once and
// walks row tiles tile = blockIdx.x, + gridDim.x, ...
constexpr int kMomWarps = 8;
#ifndef TR_MOM_MT
#define TR_MOM_MT 2  // tuning macro: 16-row MMA tiles per warp of k_moments_tf32x3
#endif
constexpr int kMomMT = TR_MOM_MT;                  // 16-row MMA tiles per warp
constexpr int kMomRows = 16 * kMomMT * kMomWarps;  // 256 rows per tile: 1 KB runs per ordinate
constexpr int kMomK = 16;                          // ordinates per stage
constexpr int kMomStride = kMomRows + 8;
constexpr int kMomStages = 4;
constexpr size_t kMomStageWords = static_cast<size_t>(kMomK) * kMomStride;
__device__ __forceinline__ void cp_async16_zfill(void *dst, const void *src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n));
}
__global__ void __launch_bounds__(32 * kMomWarps) k_moments_tf32x3(uint32_t M, uint32_t nq, uint32_t nqp,
                                                                  const double *W, const float *psi, int nmom,
                                                                  double *mom) {
    // split weights in B-fragment order: for k-step ks and lane (g, t) eight
    // words {hi, hi, lo, lo} at ordinates 8 ks + t, + 4 for moment g, then the
    // same for moment 8 + g -- two 16-byte loads per lane and k-step
    extern __shared__ __align__(16) uint32_t wsh[];  // [nqp / 8][32][8]; then the psi stages
    float *stage = reinterpret_cast<float *>(wsh + 32 * nqp);
    for (uint32_t i = threadIdx.x; i < 32 * nqp; i += blockDim.x) {
        const uint32_t ks = i / 256, ln = (i / 8) % 32, j = i % 8;
        const uint32_t n = (j < 4 ? 0u : 8u) + (ln >> 2), kq = 8 * ks + (ln & 3u) + ((j & 1u) ? 4u : 0u);
        const float w = kq < nq ? static_cast<float>(W[static_cast<size_t>(n) * nq + kq]) : 0.0f;
        const uint32_t hi = to_tf32(w);
        wsh[i] = (j & 2u) ? to_tf32(w - __uint_as_float(hi)) : hi;
    }
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    const uint32_t tiles = (M + kMomRows - 1) / kMomRows, nch = (nq + kMomK - 1) / kMomK;
    const uint32_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint64_t total = static_cast<uint64_t>(my_tiles) * nch;  // (tile, chunk) stages of this block
    // stage s -> row tile and ordinate chunk
    auto issue = [&](uint64_t s) {
        if (s < total) {
            const uint64_t r0 = static_cast<uint64_t>(blockIdx.x + (s / nch) * gridDim.x) * kMomRows;
            const uint32_t k0 = static_cast<uint32_t>(s % nch) * kMomK;
            float *dst = stage + (s % kMomStages) * kMomStageWords;
            for (uint32_t j = threadIdx.x; j < kMomK * (kMomRows / 4); j += blockDim.x) {
                const uint32_t k = j / (kMomRows / 4), rq = j % (kMomRows / 4);
                const uint64_t row = r0 + 4 * rq;
                const bool ok = k0 + k < nq && row < M;
                const float *src = ok ? psi + static_cast<uint64_t>(k0 + k) * M + row : psi;
                cp_async16_zfill(dst + k * kMomStride + 4 * rq, src, ok);
            }
        }
        cp_async_commit();  // one group per stage, empty past the end
    };
    for (int s = 0; s < kMomStages - 1; ++s) issue(s);
    float d[kMomMT][2][4];
#pragma unroll
    for (int mt = 0; mt < kMomMT; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) d[mt][nt][0] = d[mt][nt][1] = d[mt][nt][2] = d[mt][nt][3] = 0.f;
    for (uint64_t s = 0; s < total; ++s) {
        cp_async_wait<kMomStages - 2>();
        __syncthreads();  // stage s visible to all; stage s - 1 no longer read (also the weights, s = 0)
        issue(s + kMomStages - 1);
        const float *sm = stage + (s % kMomStages) * kMomStageWords;
        const uint32_t k0 = static_cast<uint32_t>(s % nch) * kMomK, rw = 16 * kMomMT * warp;
#pragma unroll
        for (int ks = 0; ks < kMomK / 8; ++ks) {
            const uint32_t kg = k0 + 8 * ks;
            if (kg >= nq) break;  // block-uniform
            const uint32_t kl = 8 * ks + t;
            const uint4 *wf = reinterpret_cast<const uint4 *>(wsh) + ((kg / 8) * 32 + lane) * 2;
            const uint4 b0 = wf[0], b1 = wf[1];  // hi, hi, lo, lo of moments g and 8 + g
#pragma unroll
            for (int mt = 0; mt < kMomMT; ++mt) {
                const uint32_t rr = rw + 16 * mt + g;
                float av[4];
                av[0] = sm[kl * kMomStride + rr];
                av[1] = sm[kl * kMomStride + rr + 8];
                av[2] = sm[(kl + 4) * kMomStride + rr];
                av[3] = sm[(kl + 4) * kMomStride + rr + 8];
                uint32_t ahi[4], alo[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    ahi[i] = to_tf32(av[i]);
                    alo[i] = to_tf32(av[i] - __uint_as_float(ahi[i]));
                }
                mma_tf32(d[mt][0], alo, b0.x, b0.y);  // small products first
                mma_tf32(d[mt][0], ahi, b0.z, b0.w);
                mma_tf32(d[mt][0], ahi, b0.x, b0.y);
                mma_tf32(d[mt][1], alo, b1.x, b1.y);
                mma_tf32(d[mt][1], ahi, b1.z, b1.w);
                mma_tf32(d[mt][1], ahi, b1.x, b1.y);
            }
        }
        if (s % nch == nch - 1) {  // last chunk of the tile: write its 16 moments, start the next
#pragma unroll
            for (int mt = 0; mt < kMomMT; ++mt) {
                const uint64_t r0 =
                    static_cast<uint64_t>(blockIdx.x + (s / nch) * gridDim.x) * kMomRows + rw + 16 * mt;
                const bool ok0 = r0 + g < M, ok1 = r0 + g + 8 < M;
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    const int n0 = nt * 8 + 2 * static_cast<int>(t);
                    if (ok0) {
                        if (n0 < nmom) mom[static_cast<uint64_t>(n0) * M + r0 + g] = d[mt][nt][0];
                        if (n0 + 1 < nmom) mom[static_cast<uint64_t>(n0 + 1) * M + r0 + g] = d[mt][nt][1];
                    }
                    if (ok1) {
                        if (n0 < nmom) mom[static_cast<uint64_t>(n0) * M + r0 + g + 8] = d[mt][nt][2];
                        if (n0 + 1 < nmom) mom[static_cast<uint64_t>(n0 + 1) * M + r0 + g + 8] = d[mt][nt][3];
                    }
                    d[mt][nt][0] = d[mt][nt][1] = d[mt][nt][2] = d[mt][nt][3] = 0.f;
                }
            }
        }
    }
    cp_async_wait<0>();
}
// shared memory of k_moments_tf32x3 for nqp (multiple of 8) ordinates
inline size_t moments_smem(uint32_t nqp) { return 32ull * nqp * 4 + kMomStages * kMomStageWords * 4; }

// Adjoint gradient of a boundary functional F (outflow through a set of
// faces).  With mu_q the adjoint angular flux (the sweep in the reversed
// ordinate -Omega_q, unit isotropic inflow on the functional's faces, no
// volume source) and Phi = sum_q w_q mu_q its scalar flux, per cell
//   G     = sum_q w_q mu_q^T M psi_q,          M = (1 + d_ij) / 20,
//   dF/dsigma_a = V (B/4) sum_i Phi_i - V G,
//   dF/dsigma_s = V Phi^T M J       - V G     (sigma_t = sigma_a + sigma_s).
template <typename T>
__global__ void k_gradient(uint32_t nT, uint32_t nq, const double *w, const T *psi, const T *mu, const double *J,
                           const double *Phi, const double *vol, const double *Bp, double *dsa, double *dss) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nT; c += gridDim.x * blockDim.x) {
        double G = 0.0;
        for (uint32_t q = 0; q < nq; ++q) {
            const typename Vec4<T>::type p = load_v4<T>(psi + ((size_t)q * nT + c) * 4);
            const typename Vec4<T>::type m = load_v4<T>(mu + ((size_t)q * nT + c) * 4);
            const double pp[4] = {(double)p.x, (double)p.y, (double)p.z, (double)p.w};
            const double mm[4] = {(double)m.x, (double)m.y, (double)m.z, (double)m.w};
            const double dot = mm[0] * pp[0] + mm[1] * pp[1] + mm[2] * pp[2] + mm[3] * pp[3];
            const double sum = (mm[0] + mm[1] + mm[2] + mm[3]) * (pp[0] + pp[1] + pp[2] + pp[3]);
            G += w[q] * (dot + sum) / 20.0;
        }
        const double *jc = J + 4 * (size_t)c, *fc = Phi + 4 * (size_t)c;
        const double pj = (fc[0] * jc[0] + fc[1] * jc[1] + fc[2] * jc[2] + fc[3] * jc[3] +
                           (fc[0] + fc[1] + fc[2] + fc[3]) * (jc[0] + jc[1] + jc[2] + jc[3])) / 20.0;
        const double V = vol[c];
        dsa[c] = V * (Bp[c] / 4.0 * (fc[0] + fc[1] + fc[2] + fc[3]) - G);
        dss[c] = V * (pj - G);
    }
}

// sum_q w_q sum_{masked boundary faces, Omega.s > 0} (Omega.s) mean_face(psi_q)
template <typename T>
__global__ void k_outflow(uint32_t nT, uint32_t nq, uint32_t nbf, const uint32_t *bcell, const uint32_t *bface,
                          const uint8_t *fmask, const double *s, const double *ox, const double *oy, const double *oz,
                          const double *w, const T *psi, double *partials, unsigned int *counter, double *out) {
    double v[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbf; i += gridDim.x * blockDim.x) {
        if (!fmask[bface[i]]) continue;
        const uint32_t c = bcell[i] >> 2, k = bcell[i] & 3u;
        const double *sk = s + 12 * (size_t)c + 3 * k;
        for (uint32_t q = 0; q < nq; ++q) {
            const double d = odot_rn(ox[q], oy[q], oz[q], sk);
            if (!(d > 0.0)) continue;
            const T *pp = psi + ((size_t)q * nT + c) * 4;
            double m = 0.0;
            for (uint32_t j = 0; j < 4; ++j)
                if (j != k) m += static_cast<double>(pp[j]);
            v[0] += w[q] * d * m / 3.0;
        }
    }
    double tot[1];
    if (grid_reduce<1>(v, partials, counter, tot) && threadIdx.x == 0) out[0] = tot[0];
}

// ---- diffusion synthetic acceleration ----------------------------------------
// The diffusion correction of the scalar flux: b_v = sum over the cells c at
// vertex v (local vertex j) of int_c sigma_s y lambda_j = sigma_s V/20 (y_j +
// sum_i y_i), on the even-parity operator's vertex layout [nP][aslm] (l = 0).
__global__ void k_dsa_rhs(uint32_t nP, uint32_t aslm, const uint32_t *vc_start, const uint32_t *vc_cj,
                          const double *ssv, const double *y, double *b) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nP; v += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint32_t i = vc_start[v]; i < vc_start[v + 1]; ++i) {
            const uint32_t cj = vc_cj[i], c = cj >> 2, j = cj & 3u;
            const double *yc = y + 4 * (size_t)c;
            acc += ssv[c] / 20.0 * (yc[j] + yc[0] + yc[1] + yc[2] + yc[3]);
        }
        for (uint32_t l = 0; l < aslm; ++l) b[(size_t)v * aslm + l] = l == 0 ? acc : 0.0;
    }
}
// z = y + the correction f carried to every unknown: J[c][j] += f[vertex(c,
// j)], and each inflow value of B (reflective entry or lagged face, indexed by
// its cell's local vertex j, zero at the face's own index k) += f[vertex(c,
// j)] -- near the diffusion limit the error of the angular flux is isotropic
__global__ void k_dsa_prolong(uint32_t nT, uint32_t nent, uint64_t nB, uint32_t aslm, const uint4 *cell_p,
                              const uint32_t *ent_cell, const unsigned long long *lag_keys, const double *f,
                              const double *y, double *z) {
    const uint64_t n = 4ull * nT + nB;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double v = y[i];
        uint32_t c, j, k = 4;
        if (i < 4ull * nT) {
            c = static_cast<uint32_t>(i >> 2);
            j = static_cast<uint32_t>(i & 3u);
        } else {
            const uint64_t b = i - 4ull * nT, e = b >> 2;
            j = static_cast<uint32_t>(b & 3u);
            if (e < nent) {
                const uint32_t ck = ent_cell[e];
                c = ck >> 2;
                k = ck & 3u;
            } else {
                const unsigned long long key = lag_keys[e - nent];
                c = static_cast<uint32_t>((key >> 2) % nT);
                k = static_cast<uint32_t>(key & 3u);
            }
        }
        if (j != k) {
            const uint4 p = cell_p[c];
            const uint32_t vert = j == 0 ? p.x : j == 1 ? p.y : j == 2 ? p.z : p.w;
            v += f[(size_t)vert * aslm];
        }
        z[i] = v;
    }
}

// Two-level preconditioned CG on the assembled diffusion matrix (ELL, column
// major: val/col[j * n + i] for row i, padded with zeros on the diagonal)
// run by ONE thread-block cluster.  Rows are split evenly over its CTAs
// (CTA k: rows [k per, (k + 1) per)), and each CTA's rows into kDsaAgg
// contiguous aggregates; the preconditioner is additive two-level,
//   z = D^-1 r + P A_c^-1 P^T r,   A_c = P^T K P  (P: aggregate indicator),
// with A_c^-1 precomputed on the host (nr kDsaAgg square, L2-resident).
// Vectors live in global memory (L2-resident at these sizes); each
// iteration synchronises with four hardware cluster barriers, three of
// which carry dot products or aggregate sums through distributed shared
// memory.  Every CTA sums the CTAs' values in rank order, so all of them see
// bit-identical scalars and take the same branch: the loop needs no grid
// barrier and no spin.  Stops at ||r|| <= tol ||b|| or maxit.
namespace cgr = cooperative_groups;
constexpr int kDsaThreads = 1024;
constexpr int kDsaAgg = 16;                        // aggregates per CTA
constexpr int kDsaMaxCluster = 16;
constexpr uint32_t kDsaClusterMaxRows = 1u << 18;  // larger problems use the even-parity context
struct DsaCg {
    uint32_t n, w;
    const uint32_t *col;
    const double *val, *dinv, *b;
    const double *ainv;          // [nc][nc], nc = cluster size * kDsaAgg
    double *x, *r, *p, *q;
    double tol;
    int maxit;
    unsigned long long *stats;   // [0] CG iterations, [1] solves, [2] non-finite stops
};
struct DsaShared {
    double slots[2][2];          // dot products: ring of two, rewritten only two barriers later
    double agg[1 + kDsaAgg];     // ||r||^2 partial and this CTA's aggregate sums of r
    double rc[kDsaMaxCluster * kDsaAgg];  // every aggregate sum, gathered
    double e[kDsaAgg];           // coarse correction of this CTA's aggregates
    double2 wsum[kDsaThreads / 32];
    double2 bcast;
};
__device__ __forceinline__ double dsa_warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;  // lane 0
}
// sum of (v0, v1) over the cluster, identical bits in every CTA
__device__ __forceinline__ double2 dsa_cluster_sum(cgr::cluster_group &cl, double v0, double v1, double *slot,
                                                   DsaShared &sh) {
    v0 = dsa_warp_sum(v0);
    v1 = dsa_warp_sum(v1);
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) sh.wsum[warp] = make_double2(v0, v1);
    __syncthreads();
    if (warp == 0) {
        const double2 t = lane < (blockDim.x >> 5) ? sh.wsum[lane] : make_double2(0.0, 0.0);
        const double a0 = dsa_warp_sum(t.x), a1 = dsa_warp_sum(t.y);
        if (lane == 0) {
            slot[0] = a0;
            slot[1] = a1;
        }
    }
    cl.sync();
    if (warp == 0) {
        double a0 = 0.0, a1 = 0.0;
        if (lane < cl.num_blocks()) {
            const double *rs = cl.map_shared_rank(slot, static_cast<int>(lane));
            a0 = rs[0];
            a1 = rs[1];
        }
        a0 = dsa_warp_sum(a0);
        a1 = dsa_warp_sum(a1);
        if (lane == 0) sh.bcast = make_double2(a0, a1);
    }
    __syncthreads();
    return sh.bcast;
}
// first row of local aggregate g (g = 0..kDsaAgg) of the rows [r0, r1)
__device__ __forceinline__ uint32_t dsa_agg_bound(uint32_t r0, uint32_t r1, int g) {
    return r0 + static_cast<uint32_t>((static_cast<uint64_t>(r1 - r0) * g) / kDsaAgg);
}
// ||r||^2 over the cluster and every aggregate sum of r (into sh.rc); r of
// this CTA's rows was written by this CTA before the call
__device__ double dsa_exchange(cgr::cluster_group &cl, const DsaCg &a, uint32_t r0, uint32_t r1, double rr,
                               DsaShared &sh) {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    rr = dsa_warp_sum(rr);
    if (lane == 0) sh.wsum[warp] = make_double2(rr, 0.0);
    __syncthreads();  // also orders this CTA's writes of r before the sums below
    if (warp < kDsaAgg) {
        const uint32_t g0 = dsa_agg_bound(r0, r1, warp), g1 = dsa_agg_bound(r0, r1, warp + 1);
        double sum = 0.0;
        for (uint32_t i = g0 + lane; i < g1; i += 32) sum += a.r[i];
        sum = dsa_warp_sum(sum);
        if (lane == 0) sh.agg[1 + warp] = sum;
    } else if (warp == kDsaAgg) {
        const double t = dsa_warp_sum(lane < (blockDim.x >> 5) ? sh.wsum[lane].x : 0.0);
        if (lane == 0) sh.agg[0] = t;
    }
    cl.sync();
    const unsigned nr = cl.num_blocks();
    for (unsigned t = threadIdx.x; t < nr * kDsaAgg; t += blockDim.x) {
        const double *rs = cl.map_shared_rank(sh.agg, static_cast<int>(t / kDsaAgg));
        sh.rc[t] = rs[1 + t % kDsaAgg];
    }
    if (warp == 0) {
        double v = 0.0;
        if (lane < nr) v = cl.map_shared_rank(sh.agg, static_cast<int>(lane))[0];
        v = dsa_warp_sum(v);
        if (lane == 0) sh.bcast = make_double2(v, 0.0);
    }
    __syncthreads();
    return sh.bcast.x;
}
// z = D^-1 r + e[aggregate] into q (own rows); returns the local part of r.z
__device__ double dsa_precondition(cgr::cluster_group &cl, const DsaCg &a, uint32_t r0, uint32_t r1,
                                   DsaShared &sh) {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned nc = cl.num_blocks() * kDsaAgg, rank = cl.block_rank();
    if (warp < kDsaAgg) {
        const double *row = a.ainv + (size_t)(rank * kDsaAgg + warp) * nc;
        double v = 0.0;
        for (unsigned b = lane; b < nc; b += 32) v += __ldg(row + b) * sh.rc[b];
        v = dsa_warp_sum(v);
        if (lane == 0) sh.e[warp] = v;
    }
    __syncthreads();
    double rz = 0.0;
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        int g = 0;
        while (g + 1 < kDsaAgg && i >= dsa_agg_bound(r0, r1, g + 1)) ++g;
        const double ri = a.r[i], zi = __ldg(a.dinv + i) * ri + sh.e[g];
        a.q[i] = zi;
        rz += ri * zi;
    }
    return rz;
}
__global__ void __launch_bounds__(kDsaThreads, 1) k_dsa_cg(const __grid_constant__ DsaCg a) {
    cgr::cluster_group cl = cgr::this_cluster();
    __shared__ DsaShared sh;
    const uint32_t nr = cl.num_blocks(), rank = cl.block_rank();
    const uint32_t per = (a.n + nr - 1) / nr;
    const uint32_t r0 = min(a.n, rank * per), r1 = min(a.n, r0 + per);
    int sl = 0;
    double l0 = 0.0;
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const double bi = __ldg(a.b + i);
        a.x[i] = 0.0;
        a.r[i] = bi;
        l0 += bi * bi;
    }
    const double bb = dsa_exchange(cl, a, r0, r1, l0, sh);
    const double tol = a.tol * sqrt(bb);
    int k = 0, bad = 0;
    if (bb > 0.0 && isfinite(bb)) {
        // z_0 into q, p_0 = z_0
        double2 t = dsa_cluster_sum(cl, dsa_precondition(cl, a, r0, r1, sh), 0.0, sh.slots[sl], sh);
        sl ^= 1;
        double rz = t.x;
        for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.p[i] = a.q[i];
        cl.sync();  // p of every CTA visible before the product
        while (k < a.maxit) {
            l0 = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                double acc = 0.0;
                uint32_t j = 0;
                for (; j + 4 <= a.w; j += 4) {
                    const size_t e = (size_t)j * a.n + i, n = a.n;
                    const uint32_t c0 = __ldg(a.col + e), c1 = __ldg(a.col + e + n), c2 = __ldg(a.col + e + 2 * n),
                                   c3 = __ldg(a.col + e + 3 * n);
                    const double v0 = __ldg(a.val + e), v1 = __ldg(a.val + e + n), v2 = __ldg(a.val + e + 2 * n),
                                 v3 = __ldg(a.val + e + 3 * n);
                    acc += v0 * a.p[c0] + v1 * a.p[c1] + v2 * a.p[c2] + v3 * a.p[c3];
                }
                for (; j < a.w; ++j) {
                    const size_t e = (size_t)j * a.n + i;
                    acc += __ldg(a.val + e) * a.p[__ldg(a.col + e)];
                }
                a.q[i] = acc;
                l0 += a.p[i] * acc;
            }
            t = dsa_cluster_sum(cl, l0, 0.0, sh.slots[sl], sh);
            sl ^= 1;
            const double alpha = rz / t.x;
            l0 = 0.0;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                a.x[i] += alpha * a.p[i];
                const double ri = a.r[i] - alpha * a.q[i];
                a.r[i] = ri;
                l0 += ri * ri;
            }
            const double rr = dsa_exchange(cl, a, r0, r1, l0, sh);
            ++k;
            if (!isfinite(rr) || !isfinite(alpha)) {
                bad = 1;
                break;
            }
            if (sqrt(rr) <= tol) break;
            t = dsa_cluster_sum(cl, dsa_precondition(cl, a, r0, r1, sh), 0.0, sh.slots[sl], sh);
            sl ^= 1;
            const double beta = t.x / rz;
            rz = t.x;
            for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.p[i] = a.q[i] + beta * a.p[i];
            cl.sync();  // p of every CTA visible before the next product
        }
    }
    cl.sync();  // no CTA leaves while another may still read its shared memory
    if (rank == 0 && threadIdx.x == 0) {
        atomicAdd(a.stats, static_cast<unsigned long long>(k));
        atomicAdd(a.stats + 1, 1ull);
        if (bad) atomicAdd(a.stats + 2, 1ull);
    }
}

// ---- FP64 vector kernels of the Krylov solver --------------------------------
__global__ void k_to_f32(uint64_t n, const double *x, float *y) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = static_cast<float>(x[i]);
}
__global__ void k_to_f64(uint64_t n, const float *x, double *y) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = static_cast<double>(x[i]);
}
// y = alpha * x + beta * y (x may alias y)
__global__ void k_axpby(uint64_t n, double alpha, const double *x, double beta, double *y) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = alpha * x[i] + beta * y[i];
}
// out[i] = <V_i, w> for i < k; V rows of length n with stride ld.  Each V
// row is read once, one partial per block and row, summed in a fixed order
// by the last block.
__global__ void k_multidot(uint64_t n, int k, const double *V, uint64_t ld, const double *w, double *partials,
                           unsigned int *counter, double *out) {
    // launched with 256 threads (kMultidotWarps warps); k <= kMaxRestart + 2
    constexpr int kMultidotWarps = 8;
    __shared__ double red[kMultidotWarps][kMaxRestart + 2];
    __shared__ bool am_last;
    const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // block b takes the contiguous range [b0, b1) of every vector, so that
    // each V_i streams in long runs and the block's part of w, read again
    // for every i, stays in L1; one warp-shuffle sum per (warp, vector) and
    // a single block barrier for all k (the grid-stride form with eight
    // vectors per pass and a block reduction per vector ran at about half
    // the copy rate)
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t b0 = min(n, static_cast<uint64_t>(blockIdx.x) * chunk), b1 = min(n, b0 + chunk);
    for (int i = 0; i < k; ++i) {
        const double *Vi = V + static_cast<uint64_t>(i) * ld;
        double acc = 0.0;
#pragma unroll 4
        for (uint64_t t = b0 + threadIdx.x; t < b1; t += blockDim.x) acc = fma(Vi[t], __ldg(w + t), acc);
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) red[warp][i] = acc;
    }
    __syncthreads();
    for (int i = static_cast<int>(threadIdx.x); i < k; i += blockDim.x) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < kMultidotWarps; ++q) sum += red[q][i];
        partials[static_cast<uint64_t>(i) * gridDim.x + blockIdx.x] = sum;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // the last block sums the k partial columns, one warp per column (in a
    // fixed order: lanes stride the blocks, then a shuffle tree)
    for (int i = static_cast<int>(warp); i < k; i += kMultidotWarps) {
        double acc = 0.0;
#pragma unroll 4
        for (unsigned int b = lane; b < gridDim.x; b += 32) acc += __ldcg(partials + (uint64_t)i * gridDim.x + b);
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[i] = acc;
    }
    if (threadIdx.x == 0) *counter = 0u;
}
// w -= sum_i h[i] V_i
__global__ void k_gs_update(uint64_t n, int k, const double *V, uint64_t ld, const double *h, double *w) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        double acc = w[t];
        for (int i = 0; i < k; ++i) acc -= h[i] * V[(uint64_t)i * ld + t];
        w[t] = acc;
    }
}
// x += sum_i y[i] V_i
__global__ void k_combine(uint64_t n, int k, const double *V, uint64_t ld, const double *y, double *x) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        double acc = x[t];
        for (int i = 0; i < k; ++i) acc += y[i] * V[(uint64_t)i * ld + t];
        x[t] = acc;
    }
}

// ---- energy balance (FP64, deterministic) ------------------------------------
struct BalanceArgs {
    uint32_t nT, nq, nbf;
    const double *s, *stv, *ssv, *ext, *w, *ox, *oy, *oz, *finc;
    const int32_t *fbc, *rslot;
    const uint32_t *rent;    // [nrefl][nq] B entry of an incoming ordinate
    const uint32_t *bcell;   // [nbf] owner cell*4 + local face
    const uint32_t *bface;   // [nbf] face id
    const double *Jin, *Jout, *Bin;
};
template <typename T>
__global__ void k_balance(BalanceArgs b, const T *psi, double *partials, unsigned int *counter, double *out) {
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (uint32_t c = tid; c < b.nT; c += nth) {
        double ji = 0.0, jo = 0.0;
        for (int j = 0; j < 4; ++j) {
            if (b.Jin) ji += b.Jin[4 * (size_t)c + j];
            jo += b.Jout[4 * (size_t)c + j];
        }
        v[0] += 4.0 * b.ext[c];
        v[1] += 0.25 * (b.stv[c] * jo - b.ssv[c] * ji);
    }
    for (uint32_t i = tid; i < b.nbf; i += nth) {
        const uint32_t ck = b.bcell[i], c = ck >> 2, k = ck & 3u, f = b.bface[i];
        const double *sk = b.s + 12 * (size_t)c + 3 * k;
        const int32_t bc = b.fbc[f];
        for (uint32_t q = 0; q < b.nq; ++q) {
            const double d = odot_rn(b.ox[q], b.oy[q], b.oz[q], sk);
            if (d > 0.0) {
                const T *pp = psi + ((size_t)q * b.nT + c) * 4;
                double m = 0.0;
                for (uint32_t j = 0; j < 4; ++j)
                    if (j != k) m += static_cast<double>(pp[j]);
                m /= 3.0;
                if (bc == TR_BC_REFLECTIVE) v[4] += b.w[q] * d * m;
                else v[2] += b.w[q] * d * m;
            } else if (d < 0.0) {
                if (bc == TR_BC_INCIDENT) {
                    v[3] += b.w[q] * (-d) * b.finc[f];
                } else if (bc == TR_BC_REFLECTIVE && b.Bin) {
                    const double *bp = b.Bin + 4 * (size_t)b.rent[(size_t)b.rslot[f] * b.nq + q];
                    double m = 0.0;
                    for (uint32_t j = 0; j < 4; ++j)
                        if (j != k) m += bp[j];
                    v[4] -= b.w[q] * (-d) * m / 3.0;
                }
            }
        }
    }
    double tot[5];
    if (grid_reduce<5>(v, partials, counter, tot) && threadIdx.x == 0)
        for (int i = 0; i < 5; ++i) out[i] = tot[i];
}

}  // namespace sweep
}  // namespace transfer

using namespace transfer;
using namespace transfer::sweep;

// ============================================================================
// the context
// ============================================================================
struct tr_sweep {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    uint32_t nT = 0, nF = 0, nq = 0, nrefl = 0, nlag = 0, maxlev = 0, forced = 0, lstride = 0, nbf = 0;
    uint64_t nB = 0, nJ = 0, device_bytes = 0;
    int num_sms = 0;
    // geometry and physics
    double *s64 = nullptr, *stv64 = nullptr, *ssv64 = nullptr, *ext64 = nullptr, *finc64 = nullptr;
    double *coef64 = nullptr;  // [nT][4] sigma_t V, sigma_s V, sigma_a V B / 4, 0
    float *coef32 = nullptr;
    float *s32 = nullptr, *stv32 = nullptr, *ssv32 = nullptr, *ext32 = nullptr, *finc32 = nullptr;
    int32_t *nbr = nullptr, *fbc = nullptr, *rslot = nullptr;
    uint32_t *map = nullptr, *bcell = nullptr, *bface = nullptr;
    uint32_t *rent = nullptr;      // [nrefl][nq] B entry of an incoming ordinate, or kNone
    uint32_t *ent_cell = nullptr;  // [nent] owner cell * 4 + local face of a reflective B entry
    uint32_t *ent_qout = nullptr;  // [nent] the mirrored outgoing ordinate
    uint32_t nent = 0;
    double *o64[4] = {nullptr, nullptr, nullptr, nullptr};  // x y z w
    float *o32[3] = {nullptr, nullptr, nullptr};
    double *Wm = nullptr;          // [16][nq] w_q Y_m(Omega_q)
    double *vol64 = nullptr, *B64 = nullptr;  // cell volume, Planck intensity
    std::vector<double> ord_host;  // x, y, z, w of the ordinates
    // schedule
    uint4 *task = nullptr;
    uint32_t *lvl = nullptr, *nlev = nullptr;
    unsigned long long *lag_keys = nullptr;
    unsigned long long *f4_keys = nullptr;
    uint32_t *f4_codes = nullptr;
    uint32_t n_f4 = 0;
    // state
    double *psi64 = nullptr;
    float *psi32 = nullptr;
    int last_prec = 0;             // precision of the last sweep (0: none)
    float *J32 = nullptr, *Bi32 = nullptr, *Bo32 = nullptr;
    double *partials = nullptr, *red = nullptr;
    unsigned int *counter = nullptr;
    // Krylov work space (allocated on first solve)
    double *kv = nullptr;          // [kMaxRestart + 1][n] basis
    double *kb = nullptr, *kx = nullptr, *kt = nullptr, *kh = nullptr;
    int kv_m = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // diffusion synthetic acceleration (tr_sweep_enable_dsa): the even-parity
    // operator with l = 0 only on the same mesh, vertex -> (cell, local vertex)
    // CSR, cell vertices, the diffusion right-hand side and solution
    tr_ctx *dsa = nullptr;
    uint32_t nP = 0, dsa_aslm = 0;
    uint32_t *vc_start = nullptr, *vc_cj = nullptr;
    uint4 *cell_p = nullptr;
    double *dsa_b = nullptr, *dsa_f = nullptr;
    // the assembled diffusion matrix for the one-cluster CG (k_dsa_cg)
    int dsa_cluster = 0;           // CTAs of the cluster (0: the path is unavailable)
    uint32_t ell_w = 0;
    uint32_t *ell_col = nullptr;
    double *ell_val = nullptr, *dsa_dinv = nullptr;
    double *dsa_ainv = nullptr;    // inverse of the aggregated matrix [nc][nc]
    double *dsa_vec = nullptr;     // b, x, r, p, q  [5][nP]
    unsigned long long *dsa_stats = nullptr;
    double *kz = nullptr;          // flexible GMRES: preconditioned basis [kMaxRestart + 1][n]
    int kz_m = 0;
    int64_t dsa_solves = 0, dsa_iterations = 0;
    std::string prec_error;
    std::vector<void *> allocs;
    int64_t sweeps32 = 0, sweeps64 = 0, launches = 0;
    bool mom_attr = false;         // k_moments_tf32x3 shared-memory opt-in done
    int mom_kernel = TR_MOMENTS_TCGEN05;
    unsigned int *mom_err = nullptr;  // pipeline-timeout flag of k_moments_tcgen05
    int shape32 = -1;              // FP32 sweep shape: -1 by rule, 0 full, 1 small (tr_sweep_autotune)
    // frequency groups (tr_sweep_create_group): a group shares its parent's
    // geometry, ordinates, schedule and task records and owns its
    // coefficients and state; the parent counts its live groups
    tr_sweep *parent = nullptr;
    int groups = 0;
    int batch_cfg = -1;            // batched launch form (tr_sweep_autotune_batch): -1 by rule
    unsigned int *qticket = nullptr;  // ticket of the work-queue launch (k_sweep_queue)
};

static tr_status sw_err(tr_sweep *s, tr_status st, const std::string &m) {
    if (s) s->last_error = m;
    return transfer::set_global_error(st, m);
}
static tr_status sw_cuda(tr_sweep *s, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return TR_OK;
    return sw_err(s, TR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
static cudaError_t sw_alloc(tr_sweep *s, T **p, size_t count) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e != cudaSuccess) return e;
    s->allocs.push_back(*p);
    s->device_bytes += bytes;
    return cudaSuccess;
}
template <typename T>
static cudaError_t sw_upload(tr_sweep *s, T **p, const std::vector<T> &h) {
    cudaError_t e = sw_alloc(s, p, h.size());
    if (e != cudaSuccess) return e;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// frees one allocation made by sw_alloc (work space released between uses)
static void sw_release(tr_sweep *s, void *p) {
    if (!p) return;
    auto it = std::find(s->allocs.begin(), s->allocs.end(), p);
    if (it != s->allocs.end()) s->allocs.erase(it);
    cudaFree(p);
}

static void sw_free(tr_sweep *s) {
    if (!s) return;
    if (s->parent) --s->parent->groups;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->dsa) tr_ctx_destroy(s->dsa);
    for (void *p : s->allocs) cudaFree(p);
    for (auto &e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    cudaSetDevice(prev);
    delete s;
}

static inline int grid_for(const tr_sweep *s, uint64_t n, int block = 256) {
    uint64_t g = (n + block - 1) / block;
    uint64_t cap = static_cast<uint64_t>(s->num_sms) * 8;
    return static_cast<int>(std::max<uint64_t>(1, std::min(g, cap)));
}

// ---- host set-up --------------------------------------------------------------
namespace {
struct FaceKey {
    uint32_t v[3];
    uint32_t cell, k;
    bool operator<(const FaceKey &o) const {
        for (int i = 0; i < 3; ++i)
            if (v[i] != o.v[i]) return v[i] < o.v[i];
        if (cell != o.cell) return cell < o.cell;
        return k < o.k;
    }
    bool same(const FaceKey &o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};
void sort3(uint32_t *v) {
    if (v[0] > v[1]) std::swap(v[0], v[1]);
    if (v[1] > v[2]) std::swap(v[1], v[2]);
    if (v[0] > v[1]) std::swap(v[0], v[1]);
}
}  // namespace

template <typename T, bool SMALL>
static cudaError_t queue_setup();  // the work-queue kernels' attributes and occupancy

static tr_status sweep_setup(tr_sweep *S, const tr_mesh_view *m, const tr_physics_view *ph,
                             const tr_ordinates_view *o) {
    const uint32_t nT = m->nT, nF = m->nF, nq = o->nq;
    S->nT = nT;
    S->nF = nF;
    S->nq = nq;
    S->nJ = 4ull * nT;
    std::vector<double> s(12ull * nT), stv(nT), ssv(nT), ext(nT), vol(nT), bpl(nT);
    for (uint32_t c = 0; c < nT; ++c) {
        const tr_tetrahedron &t = m->mesh[c];
        std::memcpy(&s[12ull * c], t.s, sizeof(double) * 12);
        // |det(s_1, s_2, s_3)| = 9 V^2 / 2 for the face area normals of a tetrahedron
        const double *a = t.s[1], *b2 = t.s[2], *c3 = t.s[3];
        const double det = a[0] * (b2[1] * c3[2] - b2[2] * c3[1]) - a[1] * (b2[0] * c3[2] - b2[2] * c3[0]) +
                           a[2] * (b2[0] * c3[1] - b2[1] * c3[0]);
        vol[c] = std::sqrt(std::fabs(det) / 4.5);
        bpl[c] = t.I_p;
        const double sav = (ph && ph->kappa_abs_volume) ? ph->kappa_abs_volume[c] : t.kappa_volume;
        if (!(t.kappa_volume > 0.0) || sav < 0.0 || sav > t.kappa_volume * (1.0 + 1e-12))
            return sw_err(S, TR_ERR_MESH, "sweep: need kappa_volume > 0 and 0 <= sigma_a V <= sigma_t V");
        stv[c] = t.kappa_volume;
        ssv[c] = t.kappa_volume - sav;
        ext[c] = sav * t.I_p / 4.0;
    }
    std::vector<int32_t> fbc(nF + 1, TR_BC_VACUUM);
    std::vector<double> finc(nF + 1, 0.0);
    for (uint32_t f = 0; f < nF; ++f) {
        if (ph && ph->face_bc) fbc[f] = ph->face_bc[f];
        if (ph && ph->face_incident) finc[f] = ph->face_incident[f];
        if (fbc[f] < 0 || fbc[f] > 2) return sw_err(S, TR_ERR_INVALID_ARG, "sweep: face_bc must be 0, 1 or 2");
    }
    // adjacency by sorted vertex triples
    std::vector<FaceKey> keys(4ull * nT);
    for (uint32_t c = 0; c < nT; ++c)
        for (uint32_t k = 0; k < 4; ++k) {
            FaceKey &e = keys[4ull * c + k];
            int n = 0;
            for (int j = 0; j < 4; ++j)
                if (j != (int)k) e.v[n++] = m->mesh[c].p[j];
            sort3(e.v);
            e.cell = c;
            e.k = k;
        }
    std::sort(keys.begin(), keys.end());
    std::vector<FaceKey> bkeys(nF);
    for (uint32_t f = 0; f < nF; ++f) {
        std::memcpy(bkeys[f].v, m->bnd[f].p, sizeof(uint32_t) * 3);
        sort3(bkeys[f].v);
        bkeys[f].cell = f;
        bkeys[f].k = 0;
    }
    std::sort(bkeys.begin(), bkeys.end());
    std::vector<int32_t> nbr(4ull * nT, 0);
    std::vector<uint32_t> map(nT, 0u), bcell, bface;
    for (size_t i = 0; i < keys.size();) {
        if (i + 1 < keys.size() && keys[i].same(keys[i + 1])) {
            if (i + 2 < keys.size() && keys[i].same(keys[i + 2]))
                return sw_err(S, TR_ERR_MESH, "sweep: a face is shared by more than two tetrahedra");
            const uint32_t a = keys[i].cell, ka = keys[i].k, b = keys[i + 1].cell, kb = keys[i + 1].k;
            nbr[4ull * a + ka] = static_cast<int32_t>(b);
            nbr[4ull * b + kb] = static_cast<int32_t>(a);
            for (int d = 0; d < 3; ++d) s[12ull * b + 3 * kb + d] = -s[12ull * a + 3 * ka + d];
            for (uint32_t j = 0; j < 4; ++j) {
                if (j != ka)
                    for (uint32_t jj = 0; jj < 4; ++jj)
                        if (m->mesh[b].p[jj] == m->mesh[a].p[j]) map[a] |= jj << (2 * (4 * ka + j));
                if (j != kb)
                    for (uint32_t jj = 0; jj < 4; ++jj)
                        if (m->mesh[a].p[jj] == m->mesh[b].p[j]) map[b] |= jj << (2 * (4 * kb + j));
            }
            i += 2;
        } else {
            auto it = std::lower_bound(bkeys.begin(), bkeys.end(), keys[i],
                                       [](const FaceKey &x, const FaceKey &y) {
                                           for (int d = 0; d < 3; ++d)
                                               if (x.v[d] != y.v[d]) return x.v[d] < y.v[d];
                                           return false;
                                       });
            if (it == bkeys.end() || !it->same(keys[i]))
                return sw_err(S, TR_ERR_MESH, "sweep: a tetrahedron face is neither shared nor a boundary face");
            nbr[4ull * keys[i].cell + keys[i].k] = -static_cast<int32_t>(it->cell) - 1;
            bcell.push_back(keys[i].cell * 4 + keys[i].k);
            bface.push_back(it->cell);
            i += 1;
        }
    }
    S->nbf = static_cast<uint32_t>(bcell.size());
    // reflective faces: slots, and for each (slot, incoming q_in) the mirrored
    // outgoing ordinate q_out; the B entries are those pairs in (slot, q) order
    std::vector<int32_t> rslot(nF + 1, -1);
    uint32_t nrefl = 0;
    for (uint32_t f = 0; f < nF; ++f)
        if (fbc[f] == TR_BC_REFLECTIVE) rslot[f] = static_cast<int32_t>(nrefl++);
    S->nrefl = nrefl;
    std::vector<uint32_t> rmap(static_cast<size_t>(nrefl) * nq + 1, kNone), rcell(nrefl + 1, 0u);
    for (uint32_t i = 0; i < S->nbf; ++i) {
        const uint32_t c = bcell[i] >> 2, k = bcell[i] & 3u, f = bface[i];
        if (rslot[f] < 0) continue;
        rcell[rslot[f]] = c * 4 + k;
        const double *sk = &s[12ull * c + 3 * k];
        const double a = std::sqrt(sk[0] * sk[0] + sk[1] * sk[1] + sk[2] * sk[2]);
        const double n[3] = {sk[0] / a, sk[1] / a, sk[2] / a};
        for (uint32_t q = 0; q < nq; ++q) {
            if (!(o->x[q] * sk[0] + o->y[q] * sk[1] + o->z[q] * sk[2] < 0.0)) continue;
            const double on = o->x[q] * n[0] + o->y[q] * n[1] + o->z[q] * n[2];
            const double r[3] = {o->x[q] - 2 * on * n[0], o->y[q] - 2 * on * n[1], o->z[q] - 2 * on * n[2]};
            uint32_t best = 0;
            double bd = 1e300;
            for (uint32_t p = 0; p < nq; ++p) {
                const double d = (o->x[p] - r[0]) * (o->x[p] - r[0]) + (o->y[p] - r[1]) * (o->y[p] - r[1]) +
                                 (o->z[p] - r[2]) * (o->z[p] - r[2]);
                if (d < bd) {
                    bd = d;
                    best = p;
                }
            }
            if (bd > 1e-16)
                return sw_err(S, TR_ERR_INVALID_ARG,
                              "sweep: a reflective face mirrors an ordinate onto a direction outside the set");
            rmap[static_cast<size_t>(rslot[f]) * nq + q] = best;
        }
    }
    std::vector<uint32_t> rent(static_cast<size_t>(nrefl) * nq + 1, kNone), ent_cell, ent_qout;
    for (size_t i = 0; i < static_cast<size_t>(nrefl) * nq; ++i)
        if (rmap[i] != kNone) {
            rent[i] = static_cast<uint32_t>(ent_cell.size());
            ent_cell.push_back(rcell[i / nq]);
            ent_qout.push_back(rmap[i]);
        }
    S->nent = static_cast<uint32_t>(ent_cell.size());
    // ordinates, moment weights
    std::vector<double> ox(o->x, o->x + nq), oy(o->y, o->y + nq), oz(o->z, o->z + nq), w(o->w, o->w + nq);
    std::vector<float> ox32(nq), oy32(nq), oz32(nq);
    for (uint32_t q = 0; q < nq; ++q) {
        ox32[q] = static_cast<float>(ox[q]);
        oy32[q] = static_cast<float>(oy[q]);
        oz32[q] = static_cast<float>(oz[q]);
    }
    std::vector<double> Wm(static_cast<size_t>(kMaxMoments) * nq);
    for (int l = 0, mm = 0; l <= 3; ++l)
        for (int mq = -l; mq <= l; ++mq, ++mm)
            for (uint32_t q = 0; q < nq; ++q)
                Wm[static_cast<size_t>(mm) * nq + q] = w[q] * tr_spherical_value(l, mq, ox[q], oy[q], oz[q]);
    auto f32 = [](const std::vector<double> &v) {
        std::vector<float> r(v.size());
        for (size_t i = 0; i < v.size(); ++i) r[i] = static_cast<float>(v[i]);
        return r;
    };
    cudaError_t e = cudaSuccess;
#define UP(ptr, vec)                                         \
    if (e == cudaSuccess) e = sw_upload(S, &S->ptr, vec);
    // per-cell coefficient record: sigma_t V, sigma_s V, sigma_a V B / 4 and the
    // vertex map in the low 32 bits of the fourth value (copied, never computed on)
    std::vector<double> coef(4ull * nT, 0.0);
    std::vector<float> coef_f(4ull * nT, 0.0f);
    for (uint32_t c = 0; c < nT; ++c) {
        coef[4ull * c] = stv[c];
        coef[4ull * c + 1] = ssv[c];
        coef[4ull * c + 2] = ext[c];
        std::memcpy(&coef[4ull * c + 3], &map[c], sizeof(uint32_t));
        coef_f[4ull * c] = static_cast<float>(stv[c]);
        coef_f[4ull * c + 1] = static_cast<float>(ssv[c]);
        coef_f[4ull * c + 2] = static_cast<float>(ext[c]);
        std::memcpy(&coef_f[4ull * c + 3], &map[c], sizeof(uint32_t));
    }
    UP(s64, s) UP(stv64, stv) UP(ssv64, ssv) UP(ext64, ext) UP(finc64, finc) UP(coef64, coef) UP(coef32, coef_f)
    UP(s32, f32(s)) UP(stv32, f32(stv)) UP(ssv32, f32(ssv)) UP(ext32, f32(ext)) UP(finc32, f32(finc))
    UP(nbr, nbr) UP(fbc, fbc) UP(rslot, rslot) UP(map, map) UP(rent, rent) UP(ent_cell, ent_cell) UP(ent_qout, ent_qout) UP(bcell, bcell) UP(bface, bface)
    UP(o64[0], ox) UP(o64[1], oy) UP(o64[2], oz) UP(o64[3], w) UP(o32[0], ox32) UP(o32[1], oy32) UP(o32[2], oz32)
    UP(Wm, Wm) UP(vol64, vol) UP(B64, bpl)
#undef UP
    S->ord_host.assign(o->x, o->x + nq);
    S->ord_host.insert(S->ord_host.end(), o->y, o->y + nq);
    S->ord_host.insert(S->ord_host.end(), o->z, o->z + nq);
    S->ord_host.insert(S->ord_host.end(), o->w, o->w + nq);
    if (e != cudaSuccess) return sw_cuda(S, e, "sweep: upload");
    // ---- schedule on the device
    SchedBuild b;
    b.nT = nT;
    b.nq = nq;
    b.s = S->s64;
    b.nbr = S->nbr;
    b.ox = S->o64[0];
    b.oy = S->o64[1];
    b.oz = S->o64[2];
    int32_t *indeg = nullptr;
    uint32_t *order = nullptr, *pos = nullptr, *lvl_tmp = nullptr, *nforced = nullptr;
    uint8_t *mask = nullptr, *lagm = nullptr;
    unsigned long long *lag_tmp = nullptr;
    unsigned int *lag_count = nullptr;
    const size_t nqT = static_cast<size_t>(nq) * nT;
    auto tmp_alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    tmp_alloc(reinterpret_cast<void **>(&indeg), nqT * 4);
    tmp_alloc(reinterpret_cast<void **>(&order), nqT * 4);
    tmp_alloc(reinterpret_cast<void **>(&pos), nqT * 4);
    tmp_alloc(reinterpret_cast<void **>(&mask), nqT);
    tmp_alloc(reinterpret_cast<void **>(&lagm), nqT);
    tmp_alloc(reinterpret_cast<void **>(&lvl_tmp), static_cast<size_t>(nq) * (nT + 1) * 4);
    tmp_alloc(reinterpret_cast<void **>(&nforced), static_cast<size_t>(nq) * 4);
    tmp_alloc(reinterpret_cast<void **>(&lag_tmp), static_cast<size_t>(kMaxLag) * 8);
    tmp_alloc(reinterpret_cast<void **>(&lag_count), 4);
    if (e == cudaSuccess) e = sw_alloc(S, &S->nlev, nq);
    if (e == cudaSuccess) e = sw_alloc(S, &S->task, nqT);
    tr_status st = TR_OK;
    std::vector<uint32_t> nlev_h(nq), nforced_h(nq);
    uint32_t nlag = 0;
    if (e == cudaSuccess) {
        b.indeg = indeg;
        b.order = order;
        b.pos = pos;
        b.mask = mask;
        b.lagm = lagm;
        b.lvl = lvl_tmp;
        b.nlev = S->nlev;
        b.nforced = nforced;
        k_sched_build<<<nq, kSchedThreads, 0, S->stream>>>(b);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(lag_count, 0, 4, S->stream);
    if (e == cudaSuccess) {
        k_lag_collect<<<grid_for(S, nqT), 256, 0, S->stream>>>(nT, nq, lagm, lag_tmp, lag_count);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nlag, lag_count, 4, cudaMemcpyDeviceToHost, S->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nlev_h.data(), S->nlev, 4ull * nq, cudaMemcpyDeviceToHost, S->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nforced_h.data(), nforced, 4ull * nq, cudaMemcpyDeviceToHost, S->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e == cudaSuccess && nlag > kMaxLag) st = sw_err(S, TR_ERR_UNSUPPORTED, "sweep: too many cyclic dependencies");
    std::vector<unsigned long long> lag_h(nlag);
    if (e == cudaSuccess && st == TR_OK && nlag) {
        e = cudaMemcpy(lag_h.data(), lag_tmp, 8ull * nlag, cudaMemcpyDeviceToHost);
        std::sort(lag_h.begin(), lag_h.end());
    }
    if (e == cudaSuccess && st == TR_OK) e = sw_upload(S, &S->lag_keys, lag_h);
    S->nlag = nlag;
    uint32_t maxlev = 0, forced = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        maxlev = std::max(maxlev, nlev_h[q]);
        forced += nforced_h[q];
    }
    S->maxlev = maxlev;
    S->forced = forced;
    S->lstride = maxlev + 1;
    unsigned long long *f4k_tmp = nullptr;
    uint32_t *f4c_tmp = nullptr;
    unsigned int *f4_count = nullptr;
    tmp_alloc(reinterpret_cast<void **>(&f4k_tmp), static_cast<size_t>(kMaxLag) * 8);
    tmp_alloc(reinterpret_cast<void **>(&f4c_tmp), static_cast<size_t>(kMaxLag) * 4);
    tmp_alloc(reinterpret_cast<void **>(&f4_count), 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(f4_count, 0, 4, S->stream);
    if (e == cudaSuccess && st == TR_OK) {
        k_records<<<grid_for(S, nqT), 256, 0, S->stream>>>(nT, nq, order, pos, mask, lagm, S->nbr, S->fbc, S->rslot,
                                                           S->rent, S->lag_keys, nlag, S->task, f4k_tmp, f4c_tmp,
                                                           f4_count);
        e = cudaGetLastError();
    }
    // cells with four inflow faces: their face-3 sources, sorted by (ordinate, position)
    uint32_t n_f4 = 0;
    // the context stream does not synchronise with the legacy stream of cudaMemcpy
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e == cudaSuccess) e = cudaMemcpy(&n_f4, f4_count, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && n_f4 > kMaxLag && st == TR_OK)
        st = sw_err(S, TR_ERR_UNSUPPORTED, "sweep: too many inverted elements");
    if (e == cudaSuccess && st == TR_OK) {
        std::vector<unsigned long long> fk(n_f4);
        std::vector<uint32_t> fc(n_f4), idx(n_f4);
        if (n_f4) {
            e = cudaMemcpy(fk.data(), f4k_tmp, 8ull * n_f4, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(fc.data(), f4c_tmp, 4ull * n_f4, cudaMemcpyDeviceToHost);
        }
        for (uint32_t i = 0; i < n_f4; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return fk[x] < fk[y]; });
        std::vector<unsigned long long> sk(n_f4);
        std::vector<uint32_t> scodes(n_f4);
        for (uint32_t i = 0; i < n_f4; ++i) {
            sk[i] = fk[idx[i]];
            scodes[i] = fc[idx[i]];
        }
        if (e == cudaSuccess) e = sw_upload(S, &S->f4_keys, sk);
        if (e == cudaSuccess) e = sw_upload(S, &S->f4_codes, scodes);
        S->n_f4 = n_f4;
    }
    for (void *p : {(void *)f4k_tmp, (void *)f4c_tmp, (void *)f4_count})
        if (p) cudaFree(p);
    if (e == cudaSuccess && st == TR_OK) e = sw_alloc(S, &S->lvl, static_cast<size_t>(nq) * S->lstride);
    if (e == cudaSuccess && st == TR_OK) {
        // compact the level pointers to [nq][lstride]; levels past nlev[q] are empty
        std::vector<uint32_t> lv(static_cast<size_t>(nq) * (nT + 1)), lc(static_cast<size_t>(nq) * S->lstride);
        e = cudaMemcpy(lv.data(), lvl_tmp, lv.size() * 4, cudaMemcpyDeviceToHost);
        for (uint32_t q = 0; q < nq && e == cudaSuccess; ++q)
            for (uint32_t L = 0; L < S->lstride; ++L)
                lc[static_cast<size_t>(q) * S->lstride + L] = L <= nlev_h[q] ? lv[static_cast<size_t>(q) * (nT + 1) + L] : nT;
        if (e == cudaSuccess) e = cudaMemcpy(S->lvl, lc.data(), lc.size() * 4, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    for (void *p : {(void *)indeg, (void *)order, (void *)pos, (void *)mask, (void *)lagm, (void *)lvl_tmp,
                    (void *)nforced, (void *)lag_tmp, (void *)lag_count})
        if (p) cudaFree(p);
    if (st != TR_OK) return st;
    if (e != cudaSuccess) return sw_cuda(S, e, "sweep: schedule");
    S->nB = 4ull * S->nent + 4ull * nlag;
    // reductions
    if (e == cudaSuccess) e = sw_alloc(S, &S->partials, (kMaxRestart + 2ull) * kDotGrid);
    if (e == cudaSuccess) e = sw_alloc(S, &S->red, 256);
    if (e == cudaSuccess) e = sw_alloc(S, &S->counter, 4);
    if (e == cudaSuccess) e = cudaMemset(S->counter, 0, 16);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<double, false>::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<float, false>::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<float, true>::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep_batch<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<double, false>::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep_batch<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<float, false>::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep_batch<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(SweepShape<float, true>::smem));
    if (e == cudaSuccess) e = queue_setup<double, false>();
    if (e == cudaSuccess) e = queue_setup<float, false>();
    if (e == cudaSuccess) e = queue_setup<float, true>();
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev[1]);
    if (e != cudaSuccess) return sw_cuda(S, e, "sweep: allocation");
    return TR_OK;
}

// ---- one sweep ------------------------------------------------------------------
static cudaError_t ensure_psi(tr_sweep *S, int prec) {
    const size_t n = 4ull * S->nT * S->nq;
    cudaError_t e = cudaSuccess;
    if (prec == 64 && !S->psi64) e = sw_alloc(S, &S->psi64, n);
    if (prec == 32 && !S->psi32) {
        e = sw_alloc(S, &S->psi32, n);
        if (e == cudaSuccess) e = sw_alloc(S, &S->J32, S->nJ);
        if (e == cudaSuccess) e = sw_alloc(S, &S->Bi32, S->nB);
        if (e == cudaSuccess) e = sw_alloc(S, &S->Bo32, S->nB);
    }
    return e;
}

template <typename T>
static Geom<T> geom_of(const tr_sweep *S) {
    Geom<T> g;
    if constexpr (sizeof(T) == 8) {
        g.s = S->s64;
        g.stv = S->stv64;
        g.coef = S->coef64;
        g.ssv = S->ssv64;
        g.ext = S->ext64;
        g.finc = S->finc64;
    } else {
        g.s = S->s32;
        g.stv = S->stv32;
        g.coef = S->coef32;
        g.ssv = S->ssv32;
        g.ext = S->ext32;
        g.finc = S->finc32;
    }
    g.nbr = S->nbr;
    g.map = S->map;
    g.fbc = S->fbc;
    g.rslot = S->rslot;
    return g;
}

// The launch arguments of one sweep of S from J, Bin (precision T, null = 0) into psi.
template <typename T>
static SweepJob<T> make_job(tr_sweep *S, const T *J, const T *Bin, int with_ext, T *psi) {
    SweepJob<T> j;
    j.g = geom_of<T>(S);
    j.sc = Sched{S->task, S->lvl, S->nlev, S->lstride, S->f4_keys, S->f4_codes, S->n_f4};
    SweepArgs<T> &a = j.a;
    a.nT = S->nT;
    a.nq = S->nq;
    if constexpr (sizeof(T) == 8) {
        a.ox = S->o64[0];
        a.oy = S->o64[1];
        a.oz = S->o64[2];
    } else {
        a.ox = S->o32[0];
        a.oy = S->o32[1];
        a.oz = S->o32[2];
    }
    a.J = J;
    a.Bin = Bin;
    a.Bout = nullptr;
    a.psi = psi;
    a.with_ext = with_ext;
    a.lag_base = 4ull * S->nent;
    j.block0 = 0;
    return j;
}
// reflective and lagged outflow of the sweep in psi into Bout (null = skip), on st
template <typename T>
static void sweep_outflow_b(tr_sweep *S, cudaStream_t st, const T *psi, T *Bout) {
    if (Bout && S->nent) {
        k_reflect_out<T><<<grid_for(S, S->nent), 256, 0, st>>>(S->nT, S->nent, S->ent_cell, S->ent_qout, psi, Bout);
        ++S->launches;
    }
    if (Bout && S->nlag) {
        k_lag_out<T><<<grid_for(S, S->nlag), 256, 0, st>>>(S->nT, S->nlag, S->lag_keys, S->nbr, S->map, psi,
                                                          Bout + 4ull * S->nent);
        ++S->launches;
    }
}
// Queues one sweep: J_in, B_in FP64 (null = 0) -> J_out, B_out FP64 (null = skip).
template <typename T>
static cudaError_t sweep_launch(tr_sweep *S, const T *J, const T *Bin, int with_ext, T *psi, T *Bout) {
    cudaStream_t st = S->stream;
    const SweepJob<T> j = make_job<T>(S, J, Bin, with_ext, psi);
    bool two_per_sm = false;  // FP32 with more ordinates than SMs (or as tuned): the small shape
    if constexpr (sizeof(T) == 4) {
        two_per_sm = S->shape32 >= 0 ? S->shape32 == 1 : S->nq > static_cast<uint32_t>(S->num_sms);
        if (two_per_sm) k_sweep<T, true><<<S->nq, kSweepThreads, SweepShape<T, true>::smem, st>>>(j.g, j.sc, j.a);
    }
    if (!two_per_sm) k_sweep<T, false><<<S->nq, kSweepThreads, SweepShape<T, false>::smem, st>>>(j.g, j.sc, j.a);
    ++S->launches;
    sweep_outflow_b<T>(S, st, psi, Bout);
    return cudaGetLastError();
}

static cudaError_t sweep_enqueue(tr_sweep *S, int prec, const double *J_in, const double *B_in, int with_ext,
                                 double *J_out, double *B_out) {
    cudaError_t e = ensure_psi(S, prec);
    if (e != cudaSuccess) return e;
    cudaStream_t st = S->stream;
    if (!S->nB) B_in = B_out = nullptr;
    if (prec == 64) {
        e = sweep_launch<double>(S, J_in, B_in, with_ext, S->psi64, B_out);
        if (e == cudaSuccess && J_out) {
            k_scalar_flux<double><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi64, J_out);
            ++S->launches;
        }
        ++S->sweeps64;
    } else {
        if (J_in) {
            k_to_f32<<<grid_for(S, S->nJ), 256, 0, st>>>(S->nJ, J_in, S->J32);
            ++S->launches;
        }
        if (B_in) {
            k_to_f32<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, B_in, S->Bi32);
            ++S->launches;
        }
        e = sweep_launch<float>(S, J_in ? S->J32 : nullptr, B_in ? S->Bi32 : nullptr, with_ext, S->psi32,
                                B_out ? S->Bo32 : nullptr);
        if (e == cudaSuccess && B_out) {
            k_to_f64<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, S->Bo32, B_out);
            ++S->launches;
        }
        if (e == cudaSuccess && J_out) {
            k_scalar_flux<float><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi32, J_out);
            ++S->launches;
        }
        ++S->sweeps32;
    }
    S->last_prec = prec;
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// ---- Krylov solver ------------------------------------------------------------
static cudaError_t krylov_alloc(tr_sweep *S, int m) {
    if (S->kv && S->kv_m >= m) return cudaSuccess;
    const uint64_t n = S->nJ + S->nB;
    cudaError_t e = sw_alloc(S, &S->kv, n * (m + 1));
    if (e == cudaSuccess && !S->kb) e = sw_alloc(S, &S->kb, n);
    if (e == cudaSuccess && !S->kx) e = sw_alloc(S, &S->kx, n);
    if (e == cudaSuccess && !S->kt) e = sw_alloc(S, &S->kt, n);
    if (e == cudaSuccess && !S->kh) e = sw_alloc(S, &S->kh, 2 * (kMaxRestart + 2));
    if (e == cudaSuccess) S->kv_m = m;
    return e;
}

// y = (I - T) x with T the sweep of precision prec without external sources
static cudaError_t op_apply(tr_sweep *S, int prec, const double *x, double *y) {
    const uint64_t n = S->nJ + S->nB;
    cudaError_t e = sweep_enqueue(S, prec, x, S->nB ? x + S->nJ : nullptr, 0, y, S->nB ? y + S->nJ : nullptr);
    if (e != cudaSuccess) return e;
    k_axpby<<<grid_for(S, n), 256, 0, S->stream>>>(n, 1.0, x, -1.0, y);
    ++S->launches;
    return cudaGetLastError();
}

static cudaError_t dots(tr_sweep *S, int k, const double *V, uint64_t ld, const double *w, double *dev_out,
                        double *host_out) {
    const uint64_t n = S->nJ + S->nB;
    k_multidot<<<kDotGrid, 256, 0, S->stream>>>(n, k, V, ld, w, S->partials, S->counter, dev_out);
    ++S->launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !host_out) return e;
    e = cudaMemcpyAsync(host_out, dev_out, sizeof(double) * k, cudaMemcpyDeviceToHost, S->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(S->stream);
}
static cudaError_t vnorm(tr_sweep *S, const double *x, double *out) {
    double v = 0.0;
    cudaError_t e = dots(S, 1, x, 0, x, S->red, &v);
    *out = std::sqrt(v);
    return e;
}

// Diffusion correction f = C sigma_s y: C solves the P1 diffusion problem
// (sigma_a mass, 1 / (3 sigma_t) stiffness, Marshak faces) by FP64 Jacobi CG
// to tol relative to the right-hand side.  cluster: the assembled matrix in
// one thread-block cluster (k_dsa_cg, no host synchronisation); otherwise the
// even-parity context with l = 0 (tr_solve), where a zero right-hand side
// gives f = 0 without a solve.  The result: dsa_f_of(S, cluster).
static inline const double *dsa_f_of(const tr_sweep *S, bool cluster) {
    return cluster ? S->dsa_vec + S->nP : S->dsa_f;
}
static cudaError_t dsa_solve(tr_sweep *S, const double *y, double tol, bool cluster, int maxit) {
    cudaStream_t st = S->stream;
    if (cluster) {
        const uint32_t n = S->nP;
        k_dsa_rhs<<<grid_for(S, n), 256, 0, st>>>(n, 1, S->vc_start, S->vc_cj, S->ssv64, y, S->dsa_vec);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(S->dsa_cluster);
        cfg.blockDim = dim3(kDsaThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = S->dsa_cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        DsaCg a;
        a.n = n;
        a.w = S->ell_w;
        a.col = S->ell_col;
        a.val = S->ell_val;
        a.dinv = S->dsa_dinv;
        a.ainv = S->dsa_ainv;
        a.b = S->dsa_vec;
        a.x = S->dsa_vec + n;
        a.r = S->dsa_vec + 2ull * n;
        a.p = S->dsa_vec + 3ull * n;
        a.q = S->dsa_vec + 4ull * n;
        a.tol = tol;
        a.maxit = maxit;
        a.stats = S->dsa_stats;
        S->launches += 2;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return cudaLaunchKernelEx(&cfg, k_dsa_cg, a);
    }
    const uint64_t np = static_cast<uint64_t>(S->nP) * S->dsa_aslm;
    k_dsa_rhs<<<grid_for(S, S->nP), 256, 0, st>>>(S->nP, S->dsa_aslm, S->vc_start, S->vc_cj, S->ssv64, y, S->dsa_b);
    k_multidot<<<kDotGrid, 256, 0, st>>>(np, 1, S->dsa_b, 0, S->dsa_b, S->partials, S->counter, S->red);
    S->launches += 2;
    double bb = 0.0;
    cudaError_t e = cudaMemcpyAsync(&bb, S->red, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (!(bb > 0.0)) return cudaMemsetAsync(S->dsa_f, 0, np * sizeof(double), st);
    tr_solve_opts o;
    tr_solve_opts_default(&o);
    o.mode = TR_MODE_FP64;
    o.precondition = TR_PREC_JACOBI;
    o.relative = 0;
    o.tol = tol * std::sqrt(bb);
    o.max_iter = maxit;
    tr_solve_report rep;
    const tr_status ts = tr_solve(S->dsa, &o, S->dsa_b, S->dsa_f, &rep);
    ++S->dsa_solves;
    S->dsa_iterations += rep.iterations;
    if (ts != TR_OK && ts != TR_ERR_NOT_CONVERGED) {
        S->prec_error = std::string("diffusion solve: ") + tr_last_error(S->dsa);
        return cudaErrorUnknown;
    }
    return cudaSuccess;
}
// z = base + the correction f on every unknown (k_dsa_prolong)
static cudaError_t dsa_prolong(tr_sweep *S, const double *base, double *z, bool cluster) {
    const uint64_t n = S->nJ + S->nB;
    k_dsa_prolong<<<grid_for(S, n), 256, 0, S->stream>>>(S->nT, S->nent, S->nB, cluster ? 1u : S->dsa_aslm,
                                                         S->cell_p, S->ent_cell, S->lag_keys, dsa_f_of(S, cluster),
                                                         base, z);
    ++S->launches;
    return cudaGetLastError();
}
// the diffusion correction of one solve: tolerance, engine and iteration cap
struct DsaPlan {
    double tol = 0.0;  // 0: no preconditioning
    bool cluster = false;
    int maxit = 10000;
};

// GMRES(m) on (I - T_prec) x = b, x updated in place (device vectors).
// Stops at ||b - (I - T) x|| <= rtol * bref (the recursion estimate,
// confirmed by a true residual at the end of a cycle).  With dsa.tol > 0 it
// is right-preconditioned by the diffusion correction P^-1 y = y + C sigma_s y
// in its flexible form (the inexact inner solve varies from step to step, so
// the preconditioned basis Z is kept and x += Z y).
static cudaError_t gmres(tr_sweep *S, int prec, int prec_res, const double *b, double *x, int m, double rtol,
                         double bref, double cycle_tol, int max_it, int *its, double *res_out, int *cycles_out,
                         const DsaPlan &dsa = DsaPlan()) {
    const uint64_t n = S->nJ + S->nB;
    cudaError_t e = krylov_alloc(S, m);
    if (e != cudaSuccess) return e;
    const bool flex = dsa.tol > 0.0;
    if (flex && (!S->kz || S->kz_m < m)) {
        if ((e = sw_alloc(S, &S->kz, n * (m + 1))) != cudaSuccess) return e;
        S->kz_m = m;
    }
    cudaStream_t st = S->stream;
    std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), h(m + 1);
    double res = 1.0, beta = 0.0;
    int it = 0, cycles = 0;
    bool have_r = false;  // V_0 already holds the true residual (from a failed confirmation)
    const int gr = grid_for(S, n);
    while (it < max_it) {
        // r = b - (I - T) x  into V_0, the operator in the residual precision
        ++cycles;
        if (!have_r) {
            e = op_apply(S, prec_res, x, S->kv);
            if (e != cudaSuccess) return e;
            k_axpby<<<gr, 256, 0, st>>>(n, 1.0, b, -1.0, S->kv);
            ++S->launches;
            if ((e = vnorm(S, S->kv, &beta)) != cudaSuccess) return e;
        }
        have_r = false;
        res = beta / bref;
        if (res <= rtol || beta == 0.0) break;
        k_axpby<<<gr, 256, 0, st>>>(n, 0.0, S->kv, 1.0 / beta, S->kv);
        ++S->launches;
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < m && it < max_it; ++j) {
            double *w = S->kv + static_cast<uint64_t>(j + 1) * n;
            const double *vj = S->kv + static_cast<uint64_t>(j) * n;
            if (flex) {
                double *zj = S->kz + static_cast<uint64_t>(j) * n;
                if ((e = dsa_solve(S, vj, dsa.tol, dsa.cluster, dsa.maxit)) != cudaSuccess) return e;
                if ((e = dsa_prolong(S, vj, zj, dsa.cluster)) != cudaSuccess) return e;
                vj = zj;
            }
            if ((e = op_apply(S, prec, vj, w)) != cudaSuccess) return e;
            ++it;
            // classical Gram-Schmidt; the first pass also gives ||w||^2 (w is
            // basis row j + 1), and a second pass runs only when the first
            // cancelled most of w (Daniel-Gragg-Kaufman-Stewart criterion)
            if ((e = dots(S, j + 2, S->kv, n, w, S->kh, h.data())) != cudaSuccess) return e;
            const double w0 = std::sqrt(std::fmax(h[j + 1], 0.0));
            k_gs_update<<<gr, 256, 0, st>>>(n, j + 1, S->kv, n, S->kh, w);
            ++S->launches;
            for (int i = 0; i <= j; ++i) H[static_cast<size_t>(i) * m + j] += h[i];
            double hn = 0.0;
            if ((e = vnorm(S, w, &hn)) != cudaSuccess) return e;
            if (hn < 0.7 * w0) {
                if ((e = dots(S, j + 1, S->kv, n, w, S->kh, h.data())) != cudaSuccess) return e;
                k_gs_update<<<gr, 256, 0, st>>>(n, j + 1, S->kv, n, S->kh, w);
                ++S->launches;
                for (int i = 0; i <= j; ++i) H[static_cast<size_t>(i) * m + j] += h[i];
                if ((e = vnorm(S, w, &hn)) != cudaSuccess) return e;
            }
            H[static_cast<size_t>(j + 1) * m + j] = hn;
            if (hn > 0.0) {
                k_axpby<<<gr, 256, 0, st>>>(n, 0.0, w, 1.0 / hn, w);
                ++S->launches;
            }
            for (int i = 0; i < j; ++i) {
                const double t0 = cs[i] * H[static_cast<size_t>(i) * m + j] + sn[i] * H[static_cast<size_t>(i + 1) * m + j];
                H[static_cast<size_t>(i + 1) * m + j] =
                    -sn[i] * H[static_cast<size_t>(i) * m + j] + cs[i] * H[static_cast<size_t>(i + 1) * m + j];
                H[static_cast<size_t>(i) * m + j] = t0;
            }
            const double h0 = H[static_cast<size_t>(j) * m + j], h1 = H[static_cast<size_t>(j + 1) * m + j];
            const double rr = std::sqrt(h0 * h0 + h1 * h1);
            cs[j] = h0 / rr;
            sn[j] = h1 / rr;
            H[static_cast<size_t>(j) * m + j] = rr;
            H[static_cast<size_t>(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            res = std::fabs(g[j + 1]) / bref;
            if (res <= rtol || (cycle_tol > 0.0 && std::fabs(g[j + 1]) <= cycle_tol * beta)) {
                ++j;
                break;
            }
        }
        for (int i = j - 1; i >= 0; --i) {
            double v = g[i];
            for (int k = i + 1; k < j; ++k) v -= H[static_cast<size_t>(i) * m + k] * y[k];
            y[i] = v / H[static_cast<size_t>(i) * m + i];
        }
        e = cudaMemcpyAsync(S->kh, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
        k_combine<<<gr, 256, 0, st>>>(n, j, flex ? S->kz : S->kv, n, S->kh, x);
        ++S->launches;
        if (res <= rtol || cycle_tol > 0.0) {  // the true residual: confirm, or start the next cycle from it
            if ((e = op_apply(S, prec_res, x, S->kv)) != cudaSuccess) return e;
            k_axpby<<<gr, 256, 0, st>>>(n, 1.0, b, -1.0, S->kv);
            ++S->launches;
            if ((e = vnorm(S, S->kv, &beta)) != cudaSuccess) return e;
            res = beta / bref;
            if (res <= rtol) break;
            have_r = true;
        }
    }
    *its = it;
    *res_out = res;
    if (cycles_out) *cycles_out = cycles;
    return cudaSuccess;
}

// Batched launch forms (tr_sweep_autotune_batch): a static grid of one block
// per (problem, ordinate) task or a persistent grid drawing tasks from a
// queue, each with the full shared-memory shape (4,096-position ring, one
// block per SM) or, for FP32, the small one (1,024 positions, two per SM).
enum BatchForm { kBatchStaticFull = 0, kBatchStaticSmall = 1, kBatchQueueFull = 2, kBatchQueueSmall = 3 };
constexpr int kBatchForms = 4;

// resident blocks per SM of the queue kernels (FP64 full, FP32 full, FP32
// small), found once at sweep set-up -- outside any stream capture
static int g_queue_per_sm[3] = {0, 0, 0};
template <typename T, bool SMALL>
static constexpr int queue_slot() { return sizeof(T) == 8 ? 0 : (SMALL ? 2 : 1); }
template <typename T, bool SMALL>
static cudaError_t queue_setup() {
    cudaError_t e = cudaFuncSetAttribute(k_sweep_queue<T, SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(SweepShape<T, SMALL>::smem));
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_queue<T, SMALL>, kSweepThreads,
                                                          SweepShape<T, SMALL>::smem);
    g_queue_per_sm[queue_slot<T, SMALL>()] = std::max(per_sm, 1);
    return e;
}

template <typename T, bool SMALL>
static cudaError_t launch_queue(const SweepJob<T> *dj, int n, uint32_t tasks, unsigned int *ticket, int num_sms,
                                cudaStream_t st) {
    const int per_sm = std::max(g_queue_per_sm[queue_slot<T, SMALL>()], 1);
    const uint32_t grid = std::min<uint32_t>(tasks, static_cast<uint32_t>(per_sm * num_sms));
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess)
        k_sweep_queue<T, SMALL><<<grid, kSweepThreads, SweepShape<T, SMALL>::smem, st>>>(dj, n, tasks, ticket);
    return e;
}

// One batched sweep launch in the form the first problem carries (-1: the
// rule -- static grid, small shape for FP32 when the tasks outnumber the SMs).
template <typename T>
static void launch_batch(tr_sweep *s0, const SweepJob<T> *dj, int n, uint32_t tasks, cudaStream_t st) {
    int form = s0->batch_cfg;
    if (form < 0) form = (sizeof(T) == 4 && tasks > static_cast<uint32_t>(s0->num_sms)) ? kBatchStaticSmall
                                                                                        : kBatchStaticFull;
    const bool small = sizeof(T) == 4 && (form == kBatchStaticSmall || form == kBatchQueueSmall);
    if (form == kBatchQueueFull || form == kBatchQueueSmall) {
        if (small) launch_queue<T, sizeof(T) == 4>(dj, n, tasks, s0->qticket, s0->num_sms, st);
        else launch_queue<T, false>(dj, n, tasks, s0->qticket, s0->num_sms, st);
    } else if (small) {
        k_sweep_batch<T, sizeof(T) == 4><<<tasks, kSweepThreads, SweepShape<T, sizeof(T) == 4>::smem, st>>>(dj, n);
    } else {
        k_sweep_batch<T, false><<<tasks, kSweepThreads, SweepShape<T, false>::smem, st>>>(dj, n);
    }
}

// Problem order in a batched launch: largest first (cells, then index), so
// that the blocks with the longest walks start in the first wave and the
// last wave holds short ones (blocks start in index order).
static std::vector<int> largest_first(int n, tr_sweep *const *s) {
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [s](int a, int b) { return s[a]->nT > s[b]->nT; });
    return ord;
}

// One launch of k_sweep_batch over every problem's ordinates, each problem's
// conversions and reductions before and after it on the same stream.
template <typename T>
static cudaError_t batch_sweep(int n, tr_sweep *const *s, cudaStream_t st, const double *const *J_in,
                               const double *const *B_in, int with_ext, double *const *J_out,
                               double *const *B_out) {
    std::vector<SweepJob<T>> jobs(n);
    const std::vector<int> ord = largest_first(n, s);
    uint32_t blocks = 0;
    for (int k = 0; k < n; ++k) {
        const int i = ord[k];
        tr_sweep *S = s[i];
        const double *Ji = J_in ? J_in[i] : nullptr;
        const double *Bi = (B_in && S->nB) ? B_in[i] : nullptr;
        if constexpr (sizeof(T) == 8) {
            jobs[k] = make_job<T>(S, Ji, Bi, with_ext, S->psi64);
        } else {
            if (Ji) {
                k_to_f32<<<grid_for(S, S->nJ), 256, 0, st>>>(S->nJ, Ji, S->J32);
                ++S->launches;
            }
            if (Bi) {
                k_to_f32<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, Bi, S->Bi32);
                ++S->launches;
            }
            jobs[k] = make_job<T>(S, Ji ? S->J32 : nullptr, Bi ? S->Bi32 : nullptr, with_ext, S->psi32);
        }
        jobs[k].block0 = blocks;
        blocks += S->nq;
    }
    SweepJob<T> *dj = nullptr;
    cudaError_t e = cudaMalloc(&dj, sizeof(SweepJob<T>) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dj, jobs.data(), sizeof(SweepJob<T>) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !s[0]->qticket) e = sw_alloc(s[0], &s[0]->qticket, 1);
    if (e == cudaSuccess) {
        launch_batch<T>(s[0], dj, n, blocks, st);
        ++s[0]->launches;
        e = cudaGetLastError();
    }
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        tr_sweep *S = s[i];
        double *Jo = J_out ? J_out[i] : nullptr, *Bo = (B_out && S->nB) ? B_out[i] : nullptr;
        if constexpr (sizeof(T) == 8) {
            sweep_outflow_b<T>(S, st, S->psi64, Bo);
            if (Jo) k_scalar_flux<double><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi64, Jo);
            ++S->sweeps64;
        } else {
            sweep_outflow_b<T>(S, st, S->psi32, Bo ? S->Bo32 : nullptr);
            if (Bo) k_to_f64<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, S->Bo32, Bo);
            if (Jo) k_scalar_flux<float><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi32, Jo);
            ++S->sweeps32;
        }
        S->launches += (Jo ? 1 : 0) + (sizeof(T) == 4 && Bo ? 1 : 0);
        S->last_prec = static_cast<int>(8 * sizeof(T));
        e = cudaGetLastError();
    }
    const cudaError_t es = cudaStreamSynchronize(st);
    if (dj) cudaFree(dj);
    return e != cudaSuccess ? e : es;
}

// One source iteration of every problem, x <- S(x) with sources, queued on st
// (captured once into a CUDA graph by tr_sweep_solve_batch): per problem
// x = S->kx [J | B], the new iterate in S->kt, res[2i] = ||S(x) - x||^2 and
// res[2i + 1] = ||S(x)||^2.  s0 is the caller's first sweep, whose launch
// form and work-queue ticket the batched launch uses: s[0] is the largest
// problem still running, which need not own a ticket (a queue-form launch
// once found a null ticket there when the first problem was not the largest).
template <typename T>
static void batch_si_step(tr_sweep *s0, int n, tr_sweep *const *s, cudaStream_t st, const SweepJob<T> *dj,
                          uint32_t blocks, double *res) {
    for (int i = 0; i < n; ++i) {
        tr_sweep *S = s[i];
        if constexpr (sizeof(T) == 4) {
            k_to_f32<<<grid_for(S, S->nJ), 256, 0, st>>>(S->nJ, S->kx, S->J32);
            if (S->nB) k_to_f32<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, S->kx + S->nJ, S->Bi32);
        }
    }
    launch_batch<T>(s0, dj, n, blocks, st);  // the caller's first sweep: launch form and queue ticket
    for (int i = 0; i < n; ++i) {
        tr_sweep *S = s[i];
        const uint64_t nx = S->nJ + S->nB;
        if constexpr (sizeof(T) == 8) {
            sweep_outflow_b<T>(S, st, S->psi64, S->nB ? S->kt + S->nJ : nullptr);
            k_scalar_flux<double><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi64, S->kt);
        } else {
            sweep_outflow_b<T>(S, st, S->psi32, S->nB ? S->Bo32 : nullptr);
            if (S->nB) k_to_f64<<<grid_for(S, S->nB), 256, 0, st>>>(S->nB, S->Bo32, S->kt + S->nJ);
            k_scalar_flux<float><<<grid_for(S, S->nT), 256, 0, st>>>(S->nT, S->nq, S->o64[3], S->psi32, S->kt);
        }
        k_axpby<<<grid_for(S, nx), 256, 0, st>>>(nx, 1.0, S->kt, -1.0, S->kx);  // kx = S(x) - x
        k_multidot<<<kDotGrid, 256, 0, st>>>(nx, 1, S->kx, 0, S->kx, S->partials, S->counter, res + 2 * i);
        k_multidot<<<kDotGrid, 256, 0, st>>>(nx, 1, S->kt, 0, S->kt, S->partials, S->counter, res + 2 * i + 1);
        cudaMemcpyAsync(S->kx, S->kt, nx * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
}
// Source iteration of the problems s[0..n) until each one's relative change
// is below tol: the iteration of the problems still running is captured as a
// CUDA graph and replayed; when one of them converges it leaves the set and
// the graph is captured again for the rest.
template <typename T>
static cudaError_t batch_si(int n, tr_sweep *const *s, cudaStream_t st, double tol, int max_iter,
                            int32_t *iterations, double *residual) {
    SweepJob<T> *dj = nullptr;
    double *res = nullptr;
    cudaError_t e = cudaMalloc(&dj, sizeof(SweepJob<T>) * n);
    if (e == cudaSuccess) e = cudaMalloc(&res, sizeof(double) * 2 * n);
    for (int i = 0; i < n && e == cudaSuccess; ++i)
        e = cudaMemsetAsync(s[i]->kx, 0, (s[i]->nJ + s[i]->nB) * sizeof(double), st);
    for (int i = 0; i < n; ++i) {
        iterations[i] = 0;
        residual[i] = 0.0;
    }
    std::vector<int> act = largest_first(n, s);
    std::vector<tr_sweep *> sub;
    std::vector<SweepJob<T>> jobs;
    std::vector<double> hr(2 * n);
    int it = 0;
    while (e == cudaSuccess && !act.empty() && it < max_iter) {
        const int m = static_cast<int>(act.size());
        sub.assign(m, nullptr);
        jobs.assign(m, SweepJob<T>());
        uint32_t blocks = 0;
        for (int k = 0; k < m; ++k) {
            tr_sweep *S = s[act[k]];
            sub[k] = S;
            const double *Bx = S->nB ? S->kx + S->nJ : nullptr;
            if constexpr (sizeof(T) == 8) jobs[k] = make_job<T>(S, S->kx, Bx, 1, S->psi64);
            else jobs[k] = make_job<T>(S, S->J32, Bx ? S->Bi32 : nullptr, 1, S->psi32);
            jobs[k].block0 = blocks;
            blocks += S->nq;
        }
        e = cudaMemcpyAsync(dj, jobs.data(), sizeof(SweepJob<T>) * m, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess) e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            batch_si_step<T>(s[0], m, sub.data(), st, dj, blocks, res);
            const cudaError_t ec = cudaStreamEndCapture(st, &graph);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = ec;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        bool changed = false;
        while (e == cudaSuccess && !changed && it < max_iter) {
            ++it;
            e = cudaGraphLaunch(exec, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(hr.data(), res, sizeof(double) * 2 * m, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) break;
            for (int k = 0; k < m; ++k) {
                const int i = act[k];
                const double r = hr[2 * k + 1] > 0.0 ? std::sqrt(hr[2 * k] / hr[2 * k + 1]) : 0.0;
                residual[i] = r;
                if (r < tol) {
                    iterations[i] = it;
                    changed = true;
                }
                s[i]->launches += 8;  // per iteration: conversions, sweep share, outflow, flux, reductions, copy
                if (sizeof(T) == 8) ++s[i]->sweeps64;
                else ++s[i]->sweeps32;
                s[i]->last_prec = static_cast<int>(8 * sizeof(T));
            }
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        std::vector<int> keep;
        for (int i : act)
            if (!iterations[i]) keep.push_back(i);
        act.swap(keep);
    }
    cudaStreamSynchronize(st);
    if (dj) cudaFree(dj);
    if (res) cudaFree(res);
    return e;
}

// ============================================================================
// C ABI
// ============================================================================
#define SW_CHECK(s)                                                                      \
    do {                                                                                 \
        if (!(s)) return transfer::set_global_error(TR_ERR_INVALID_ARG, "null sweep");   \
        if (cudaSetDevice((s)->device) != cudaSuccess)                                   \
            return sw_err((s), TR_ERR_CUDA, "cudaSetDevice failed");                     \
    } while (0)

extern "C" {

tr_status tr_ordinates_product(int n_polar, int n_azim, double *x, double *y, double *z, double *w) {
    if (n_polar < 1 || n_azim < 1 || !x || !y || !z || !w)
        return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_ordinates_product: bad arguments");
    std::vector<double> mu(n_polar), wm(n_polar);
    for (int i = 0; i < n_polar; ++i) {  // Gauss-Legendre nodes by Newton on P_n
        double t = std::cos(M_PI * (i + 0.75) / (n_polar + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = t;
            for (int l = 2; l <= n_polar; ++l) {
                const double p2 = ((2.0 * l - 1.0) * t * p1 - (l - 1.0) * p0) / l;
                p0 = p1;
                p1 = p2;
            }
            dp = n_polar * (t * p1 - p0) / (t * t - 1.0);
            const double dt = p1 / dp;
            t -= dt;
            if (std::fabs(dt) < 1e-16) break;
        }
        mu[i] = t;
        wm[i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
    int q = 0;
    for (int i = 0; i < n_polar; ++i) {
        const double st = std::sqrt(1.0 - mu[i] * mu[i]);
        for (int k = 0; k < n_azim; ++k, ++q) {
            const double phi = (k + 0.5) * 2.0 * M_PI / n_azim;
            x[q] = st * std::cos(phi);
            y[q] = st * std::sin(phi);
            z[q] = mu[i];
            w[q] = 0.5 * wm[i] / n_azim;
        }
    }
    return TR_OK;
}

tr_status tr_sweep_create(int device, const tr_mesh_view *mesh, const tr_physics_view *phys,
                          const tr_ordinates_view *ord, tr_sweep **out) {
    if (!mesh || !ord || !out || !mesh->mesh || (mesh->nF && !mesh->bnd) || !ord->x || !ord->y || !ord->z || !ord->w)
        return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_create: null argument");
    *out = nullptr;
    if (mesh->nT == 0 || mesh->nT > kCellMask || ord->nq == 0 || ord->nq > 65535)
        return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_create: need 0 < nT < 2^28, 0 < nq < 65536");
    if (static_cast<uint64_t>(mesh->nT) * ord->nq >= (1ull << 31))
        return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_create: nT * nq must stay below 2^31");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return transfer::set_global_error(TR_ERR_NO_DEVICE, "tr_sweep_create: no CUDA device");
    if (device < 0 || device >= ndev) return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_create: bad device");
    tr_sweep *S = new (std::nothrow) tr_sweep();
    if (!S) return transfer::set_global_error(TR_ERR_OUT_OF_MEMORY, "tr_sweep_create: host allocation");
    S->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete S;
        return transfer::set_global_error(TR_ERR_CUDA, "cudaSetDevice failed");
    }
    cudaDeviceGetAttribute(&S->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete S;
        return transfer::set_global_error(TR_ERR_CUDA, "tr_sweep_create: stream");
    }
    tr_status st = sweep_setup(S, mesh, phys, ord);
    if (st != TR_OK) {
        std::string msg = S->last_error;
        sw_free(S);
        return transfer::set_global_error(st, msg);
    }
    *out = S;
    return TR_OK;
}

tr_status tr_sweep_destroy(tr_sweep *s) {
    if (s && s->groups > 0)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_destroy: the sweep still has live frequency groups");
    sw_free(s);
    return TR_OK;
}

const char *tr_sweep_last_error(const tr_sweep *s) { return s ? s->last_error.c_str() : ""; }

tr_status tr_sweep_info_get(const tr_sweep *s, tr_sweep_info *info) {
    if (!s || !info) return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_info_get: null argument");
    info->nT = s->nT;
    info->nF = s->nF;
    info->nq = s->nq;
    info->n_extra = s->nB;
    info->n_reflective = s->nrefl;
    info->n_lag = s->nlag;
    info->max_levels = s->maxlev;
    info->forced_levels = s->forced;
    info->device_bytes = s->device_bytes;
    info->device = s->device;
    return TR_OK;
}

tr_status tr_sweep_levels(tr_sweep *s, int32_t *level) {
    SW_CHECK(s);
    if (!level) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_levels: null output");
    const size_t nqT = static_cast<size_t>(s->nq) * s->nT;
    std::vector<uint4> task(nqT);
    std::vector<uint32_t> lvl(static_cast<size_t>(s->nq) * s->lstride), nlev(s->nq);
    cudaError_t e = cudaMemcpy(task.data(), s->task, nqT * sizeof(uint4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lvl.data(), s->lvl, lvl.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(nlev.data(), s->nlev, nlev.size() * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_levels");
    for (uint32_t q = 0; q < s->nq; ++q)
        for (uint32_t L = 0; L < nlev[q]; ++L)
            for (uint32_t p = lvl[static_cast<size_t>(q) * s->lstride + L]; p < lvl[static_cast<size_t>(q) * s->lstride + L + 1]; ++p)
                level[static_cast<size_t>(q) * s->nT + (task[static_cast<size_t>(q) * s->nT + p].x & kCellMask)] =
                    static_cast<int32_t>(L);
    return TR_OK;
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

tr_status tr_sweep_apply(tr_sweep *s, int precision, const double *J_in, const double *B_in, int with_ext,
                         double *J_out, double *B_out) {
    SW_CHECK(s);
    if (precision != 32 && precision != 64) return sw_err(s, TR_ERR_INVALID_ARG, "precision must be 32 or 64");
    if (!aligned16(J_in) || !aligned16(B_in) || !aligned16(J_out) || !aligned16(B_out))
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_apply: device vectors must be 16-byte aligned");
    cudaError_t e = sweep_enqueue(s, precision, J_in, s->nB ? B_in : nullptr, with_ext, J_out, s->nB ? B_out : nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return sw_cuda(s, e, "tr_sweep_apply");
}

tr_status tr_sweep_apply_batch(int n, tr_sweep *const *s, int precision, const double *const *J_in,
                               const double *const *B_in, int with_ext, double *const *J_out,
                               double *const *B_out) {
    if (n < 1 || !s) return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_apply_batch: no sweeps");
    for (int i = 0; i < n; ++i) {
        SW_CHECK(s[i]);
        if (s[i]->device != s[0]->device)
            return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_apply_batch: sweeps on different devices");
        if ((J_in && !aligned16(J_in[i])) || (B_in && !aligned16(B_in[i])) || (J_out && !aligned16(J_out[i])) ||
            (B_out && !aligned16(B_out[i])))
            return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_apply_batch: device vectors must be 16-byte aligned");
        for (int k = 0; k < i; ++k)
            if (s[k] == s[i]) return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_apply_batch: a sweep twice");
    }
    if (precision != 32 && precision != 64) return sw_err(s[0], TR_ERR_INVALID_ARG, "precision must be 32 or 64");
    cudaSetDevice(s[0]->device);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaStreamSynchronize(s[i]->stream);  // nothing of a problem's own stream still in flight
        if (e == cudaSuccess) e = ensure_psi(s[i], precision);
    }
    if (e == cudaSuccess)
        e = precision == 64 ? batch_sweep<double>(n, s, s[0]->stream, J_in, B_in, with_ext, J_out, B_out)
                            : batch_sweep<float>(n, s, s[0]->stream, J_in, B_in, with_ext, J_out, B_out);
    return sw_cuda(s[0], e, "tr_sweep_apply_batch");
}

tr_status tr_sweep_solve_batch(int n, tr_sweep *const *s, int precision, double tol, int max_iter, double *const *J,
                               double *const *B, int32_t *iterations, double *residual) {
    if (n < 1 || !s || !J || !iterations || !residual)
        return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_solve_batch: null argument");
    for (int i = 0; i < n; ++i) {
        SW_CHECK(s[i]);
        if (s[i]->device != s[0]->device)
            return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_solve_batch: sweeps on different devices");
        if (!J[i] || !aligned16(J[i]) || (B && !aligned16(B[i])))
            return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_solve_batch: device vectors must be 16-byte aligned");
        for (int k = 0; k < i; ++k)
            if (s[k] == s[i]) return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_solve_batch: a sweep twice");
    }
    if (precision != 32 && precision != 64) return sw_err(s[0], TR_ERR_INVALID_ARG, "precision must be 32 or 64");
    if (!(tol > 0.0) || max_iter < 1) return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_solve_batch: tol / max_iter");
    cudaSetDevice(s[0]->device);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaStreamSynchronize(s[i]->stream);
        if (e == cudaSuccess) e = ensure_psi(s[i], precision);
        if (e == cudaSuccess) e = krylov_alloc(s[i], 1);
    }
    if (e == cudaSuccess && !s[0]->qticket) e = sw_alloc(s[0], &s[0]->qticket, 1);  // before any capture
    cudaStream_t st = s[0]->stream;
    if (e == cudaSuccess)
        e = precision == 64 ? batch_si<double>(n, s, st, tol, max_iter, iterations, residual)
                            : batch_si<float>(n, s, st, tol, max_iter, iterations, residual);
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaMemcpyAsync(J[i], s[i]->kx, s[i]->nJ * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && B && s[i]->nB)
            e = cudaMemcpyAsync(B[i], s[i]->kx + s[i]->nJ, s[i]->nB * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return sw_cuda(s[0], e, "tr_sweep_solve_batch");
    for (int i = 0; i < n; ++i)
        if (!iterations[i]) return sw_err(s[0], TR_ERR_NOT_CONVERGED, "tr_sweep_solve_batch: not converged");
    return TR_OK;
}

tr_status tr_sweep_autotune_batch(int n, tr_sweep *const *s, int precision, int *form, double *ms) {
    if (n < 1 || !s) return transfer::set_global_error(TR_ERR_INVALID_ARG, "tr_sweep_autotune_batch: null argument");
    for (int i = 0; i < n; ++i) {
        SW_CHECK(s[i]);
        if (s[i]->device != s[0]->device)
            return sw_err(s[0], TR_ERR_INVALID_ARG, "tr_sweep_autotune_batch: sweeps on different devices");
    }
    if (precision != 32 && precision != 64) return sw_err(s[0], TR_ERR_INVALID_ARG, "precision must be 32 or 64");
    cudaSetDevice(s[0]->device);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaStreamSynchronize(s[i]->stream);
        if (e == cudaSuccess) e = ensure_psi(s[i], precision);
    }
    cudaStream_t st = s[0]->stream;
    double t[kBatchForms];
    for (int f = 0; f < kBatchForms; ++f) t[f] = -1.0;
    int best = -1;
    for (int f = 0; f < kBatchForms && e == cudaSuccess; ++f) {
        if (precision == 64 && (f == kBatchStaticSmall || f == kBatchQueueSmall)) continue;  // FP32 only
        for (int i = 0; i < n; ++i) s[i]->batch_cfg = f;
        e = precision == 64 ? batch_sweep<double>(n, s, st, nullptr, nullptr, 1, nullptr, nullptr)
                            : batch_sweep<float>(n, s, st, nullptr, nullptr, 1, nullptr, nullptr);  // warm-up
        double tot = 0.0;
        for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
            e = cudaEventRecord(s[0]->ev[0], st);
            if (e == cudaSuccess)
                e = precision == 64 ? batch_sweep<double>(n, s, st, nullptr, nullptr, 1, nullptr, nullptr)
                                    : batch_sweep<float>(n, s, st, nullptr, nullptr, 1, nullptr, nullptr);
            if (e == cudaSuccess) e = cudaEventRecord(s[0]->ev[1], st);
            if (e == cudaSuccess) e = cudaEventSynchronize(s[0]->ev[1]);
            float ms1 = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms1, s[0]->ev[0], s[0]->ev[1]);
            tot += ms1;
        }
        t[f] = tot / 3.0;
        if (e == cudaSuccess && (best < 0 || t[f] < t[best])) best = f;
    }
    for (int i = 0; i < n; ++i) s[i]->batch_cfg = e == cudaSuccess ? best : -1;
    if (e != cudaSuccess) return sw_cuda(s[0], e, "tr_sweep_autotune_batch");
    if (form) *form = best;
    if (ms)
        for (int f = 0; f < kBatchForms; ++f) ms[f] = t[f];
    return TR_OK;
}

tr_status tr_sweep_set_batch_form(tr_sweep *s, int form) {
    SW_CHECK(s);
    if (form < -1 || form >= kBatchForms)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_set_batch_form: form must be -1 .. 3");
    s->batch_cfg = form;
    return TR_OK;
}

tr_status tr_sweep_autotune(tr_sweep *s, int *shape, double *ms) {
    SW_CHECK(s);
    cudaSetDevice(s->device);
    cudaError_t e = ensure_psi(s, 32);
    double t[2] = {0.0, 0.0};
    for (int c = 0; c < 2 && e == cudaSuccess; ++c) {
        s->shape32 = c;
        for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = sweep_enqueue(s, 32, nullptr, nullptr, 1, nullptr, nullptr);
        if (e == cudaSuccess) e = cudaEventRecord(s->ev[0], s->stream);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) e = sweep_enqueue(s, 32, nullptr, nullptr, 1, nullptr, nullptr);
        if (e == cudaSuccess) e = cudaEventRecord(s->ev[1], s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        float f = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&f, s->ev[0], s->ev[1]);
        t[c] = f / 5.0;
    }
    if (e != cudaSuccess) {
        s->shape32 = -1;
        return sw_cuda(s, e, "tr_sweep_autotune");
    }
    s->shape32 = t[1] < t[0] ? 1 : 0;
    if (shape) *shape = s->shape32;
    if (ms) {
        ms[0] = t[0];
        ms[1] = t[1];
    }
    return TR_OK;
}

tr_status tr_sweep_psi(tr_sweep *s, double *psi) {
    SW_CHECK(s);
    if (!psi) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_psi: null output");
    if (!s->last_prec) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_psi: no sweep has run");
    const uint64_t n = 4ull * s->nT * s->nq;
    cudaError_t e;
    if (s->last_prec == 64) {
        e = cudaMemcpyAsync(psi, s->psi64, n * 8, cudaMemcpyDeviceToDevice, s->stream);
    } else {
        k_to_f64<<<grid_for(s, n), 256, 0, s->stream>>>(n, s->psi32, psi);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return sw_cuda(s, e, "tr_sweep_psi");
}

tr_status tr_sweep_moments(tr_sweep *s, int nmom, double *mom) {
    SW_CHECK(s);
    if (!mom || nmom < 1 || nmom > kMaxMoments)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_moments: need 1 <= nmom <= 16 and an output");
    if (!s->last_prec) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_moments: no sweep has run");
    cudaError_t e = cudaSuccess;
    const uint32_t nqp8 = (s->nq + 7) / 8 * 8;
    const bool tc = s->mom_kernel == TR_MOMENTS_TCGEN05 && transfer::moments_tcgen05_supported(4 * s->nT, s->nq);
    const bool ff = s->mom_kernel == TR_MOMENTS_TMA_FFMA2 && transfer::moments_tma_ffma2_supported(4 * s->nT, s->nq);
    if (s->last_prec == 32 && (tc || ff)) {
        if (!s->mom_err) e = sw_alloc(s, &s->mom_err, 1);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->mom_err, 0, sizeof(unsigned int), s->stream);
        if (e == cudaSuccess)
            e = tc ? transfer::launch_moments_tcgen05(s->psi32, 4 * s->nT, s->nq, s->Wm, nmom, mom, s->mom_err,
                                                      s->num_sms, s->stream)
                   : transfer::launch_moments_tma_ffma2(s->psi32, 4 * s->nT, s->nq, s->Wm, nmom, mom, s->mom_err,
                                                        s->num_sms, s->stream);
        ++s->launches;
        unsigned int flag = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, s->mom_err, sizeof(flag), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess && flag)
            return sw_err(s, TR_ERR_CUDA, "tr_sweep_moments: a pipeline wait of the TMA-fed kernel timed out");
    } else if (s->last_prec == 32 && 2ull * 16 * nqp8 * sizeof(uint32_t) <= 48 * 1024) {  // nq <= 384
        const uint32_t M = 4 * s->nT, nqp = nqp8;
        const size_t smem = moments_smem(nqp);
        if (!s->mom_attr) {  // above 48 KB of dynamic shared memory: opt in once
            e = cudaFuncSetAttribute(k_moments_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(moments_smem(384)));
            if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_moments");
            s->mom_attr = true;
        }
        // persistent grid: as many blocks as are resident, at most one per row tile
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_moments_tf32x3, 32 * kMomWarps, smem);
        const uint64_t want = (M + kMomRows - 1) / kMomRows;
        const int blocks = static_cast<int>(
            std::max<uint64_t>(1, std::min<uint64_t>(want, static_cast<uint64_t>(std::max(per_sm, 1)) * s->num_sms)));
        k_moments_tf32x3<<<blocks, 32 * kMomWarps, smem, s->stream>>>(M, s->nq, nqp, s->Wm, s->psi32, nmom, mom);
        e = cudaGetLastError();
        ++s->launches;
    } else {
        // FP64 (and FP32 with more than 384 ordinates): FP64 accumulation over
        // complete l bands (1, 4, 9 or 16 moments); extra bands go to scratch
        const int gr = grid_for(s, s->nT, 128);
        const int nb = nmom <= 1 ? 1 : nmom <= 4 ? 4 : nmom <= 9 ? 9 : 16;
        double *out = mom, *tmp = nullptr;
        if (nb != nmom) {
            e = cudaMalloc(&tmp, sizeof(double) * nb * 4ull * s->nT);
            out = tmp;
        }
        if (e == cudaSuccess && s->last_prec == 64) {
            if (nb == 1) k_moments_simt<double, 1><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi64, out);
            else if (nb == 4) k_moments_simt<double, 4><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi64, out);
            else if (nb == 9) k_moments_simt<double, 9><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi64, out);
            else k_moments_f64_16<<<grid_for(s, 2ull * s->nT, 256), 256, 0, s->stream>>>(s->nT, s->nq, s->Wm,
                                                                                        s->psi64, out);
            e = cudaGetLastError();
            ++s->launches;
        } else if (e == cudaSuccess) {
            if (nb == 1) k_moments_simt<float, 1><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi32, out);
            else if (nb == 4) k_moments_simt<float, 4><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi32, out);
            else if (nb == 9) k_moments_simt<float, 9><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi32, out);
            else k_moments_simt<float, 16><<<gr, 128, 0, s->stream>>>(s->nT, s->nq, s->Wm, s->psi32, out);
            e = cudaGetLastError();
            ++s->launches;
        }
        if (e == cudaSuccess && tmp)
            e = cudaMemcpyAsync(mom, tmp, sizeof(double) * nmom * 4ull * s->nT, cudaMemcpyDeviceToDevice, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (tmp) cudaFree(tmp);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return sw_cuda(s, e, "tr_sweep_moments");
}

tr_status tr_sweep_set_moments_kernel(tr_sweep *s, int kind) {
    SW_CHECK(s);
    if (kind != TR_MOMENTS_TCGEN05 && kind != TR_MOMENTS_MMA_SYNC && kind != TR_MOMENTS_TMA_FFMA2)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_set_moments_kernel: unknown kernel family");
    s->mom_kernel = kind;
    return TR_OK;
}

tr_status tr_sweep_balance(tr_sweep *s, const double *J_in, const double *B_in, const double *J_out,
                           double out[5]) {
    SW_CHECK(s);
    if (!J_out || !out) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_balance: null argument");
    if (!s->last_prec) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_balance: no sweep has run");
    BalanceArgs b;
    b.nT = s->nT;
    b.nq = s->nq;
    b.nbf = s->nbf;
    b.s = s->s64;
    b.stv = s->stv64;
    b.ssv = s->ssv64;
    b.ext = s->ext64;
    b.w = s->o64[3];
    b.ox = s->o64[0];
    b.oy = s->o64[1];
    b.oz = s->o64[2];
    b.finc = s->finc64;
    b.fbc = s->fbc;
    b.rslot = s->rslot;
    b.rent = s->rent;
    b.bcell = s->bcell;
    b.bface = s->bface;
    b.Jin = J_in;
    b.Jout = J_out;
    b.Bin = s->nB ? B_in : nullptr;
    if (s->last_prec == 64)
        k_balance<double><<<kRedGrid, 256, 0, s->stream>>>(b, s->psi64, s->partials, s->counter, s->red);
    else
        k_balance<float><<<kRedGrid, 256, 0, s->stream>>>(b, s->psi32, s->partials, s->counter, s->red);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, s->red, 5 * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return sw_cuda(s, e, "tr_sweep_balance");
}

// The P1 diffusion matrix on the vertices, assembled per row from the
// vertex -> cell and vertex -> face tables:
//   K_uv = sum_c [ sigma_a V (1 + d_uv) / 20 + s_i . s_j / (27 sigma_t V) ]
//        + sum_f A_f (1 + d_uv) / 24       (vacuum / incident faces)
// (i, j the local indices of u, v in c; the Marshak term 1/2 int phi v over
// the face's exact area), stored ELL column-major with its Jacobi inverse;
// then the largest cluster that can be resident (16 CTAs, else 8).
static cudaError_t dsa_assemble(tr_sweep *s, const tr_mesh_view *m, const tr_physics_view *ph) {
    const uint32_t nP = m->nP;
    const int32_t *bc = ph ? ph->face_bc : nullptr;
    std::vector<std::vector<std::pair<uint32_t, double>>> rows(nP);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t vi = 0; vi < static_cast<int64_t>(nP); ++vi) {
        const uint32_t v = static_cast<uint32_t>(vi);
        auto &row = rows[v];
        auto add = [&row](uint32_t u, double a) {
            for (auto &pr : row)
                if (pr.first == u) {
                    pr.second += a;
                    return;
                }
            row.emplace_back(u, a);
        };
        for (tr_idx t = m->tetstart[v]; t < m->tetstart[v + 1]; ++t) {
            const uint32_t c = m->tetidx[t], i = m->tetpos[t];
            const tr_tetrahedron &T = m->mesh[c];
            const double sav = (ph && ph->kappa_abs_volume) ? ph->kappa_abs_volume[c] : T.kappa_volume;
            for (uint32_t j = 0; j < 4; ++j) {
                const double ss = T.s[i][0] * T.s[j][0] + T.s[i][1] * T.s[j][1] + T.s[i][2] * T.s[j][2];
                add(T.p[j], sav * (i == j ? 2.0 : 1.0) / 20.0 + ss / (27.0 * T.kappa_volume));
            }
        }
        for (tr_idx t = m->nF ? m->facestart[v] : 0; m->nF && t < m->facestart[v + 1]; ++t) {
            const tr_idx f = m->faceidx[t];
            if (bc && bc[f] == TR_BC_REFLECTIVE) continue;
            const tr_face &F = m->bnd[f];
            if (F.p[0] >= nP || F.p[1] >= nP || F.p[2] >= nP) continue;  // rejected below
            const double area = std::sqrt(F.s[0] * F.s[0] + F.s[1] * F.s[1] + F.s[2] * F.s[2]);
            const uint32_t i = m->facepos[t];
            for (uint32_t j = 0; j < 3; ++j) add(F.p[j], area * (i == j ? 2.0 : 1.0) / 24.0);
        }
    }
    for (uint32_t f = 0; f < m->nF; ++f)
        if (m->bnd[f].p[0] >= nP || m->bnd[f].p[1] >= nP || m->bnd[f].p[2] >= nP) return cudaErrorInvalidValue;
    size_t w = 1;
    for (const auto &r : rows) w = std::max(w, r.size());
    std::vector<uint32_t> col(w * nP);
    std::vector<double> val(w * nP, 0.0), dinv(nP, 0.0);
    for (uint32_t v = 0; v < nP; ++v) {
        for (size_t j = 0; j < w; ++j) {
            col[j * nP + v] = j < rows[v].size() ? rows[v][j].first : v;
            if (j < rows[v].size()) val[j * nP + v] = rows[v][j].second;
        }
        for (const auto &pr : rows[v])
            if (pr.first == v) dinv[v] = pr.second > 0.0 ? 1.0 / pr.second : 0.0;
    }
    cudaError_t e = sw_upload(s, &s->ell_col, col);
    if (e == cudaSuccess) e = sw_upload(s, &s->ell_val, val);
    if (e == cudaSuccess) e = sw_upload(s, &s->dsa_dinv, dinv);
    if (e == cudaSuccess) e = sw_alloc(s, &s->dsa_vec, 5ull * nP);
    if (e == cudaSuccess) e = sw_alloc(s, &s->dsa_stats, 3);
    if (e != cudaSuccess) return e;
    s->ell_w = static_cast<uint32_t>(w);
    // the largest resident cluster
    int cluster = 0;
    cudaFuncSetAttribute(k_dsa_cg, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int cs : {kDsaMaxCluster, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(kDsaThreads);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, k_dsa_cg, &cfg) == cudaSuccess && nc >= 1) {
            cluster = cs;
            break;
        }
    }
    cudaGetLastError();  // clear the error a refused cluster size may have left
    if (!cluster) return cudaSuccess;
    // aggregates: kDsaAgg contiguous row blocks of each CTA's rows (the
    // kernel's dsa_agg_bound), A_c = P^T K P inverted by Gauss-Jordan
    const uint32_t per = (nP + cluster - 1) / cluster, nc = static_cast<uint32_t>(cluster) * kDsaAgg;
    std::vector<uint32_t> agg(nP, 0);
    std::vector<char> used(nc, 0);
    for (int k = 0; k < cluster; ++k) {
        const uint32_t r0 = std::min<uint32_t>(nP, k * per), r1 = std::min<uint32_t>(nP, r0 + per);
        for (int g = 0; g < kDsaAgg; ++g) {
            const uint32_t g0 = r0 + static_cast<uint32_t>((static_cast<uint64_t>(r1 - r0) * g) / kDsaAgg);
            const uint32_t g1 = r0 + static_cast<uint32_t>((static_cast<uint64_t>(r1 - r0) * (g + 1)) / kDsaAgg);
            for (uint32_t i = g0; i < g1; ++i) agg[i] = k * kDsaAgg + g;
            used[k * kDsaAgg + g] = g1 > g0;
        }
    }
    std::vector<double> A(static_cast<size_t>(nc) * nc, 0.0), X(static_cast<size_t>(nc) * nc, 0.0);
    for (uint32_t v = 0; v < nP; ++v)
        for (const auto &pr : rows[v]) A[static_cast<size_t>(agg[v]) * nc + agg[pr.first]] += pr.second;
    for (uint32_t g = 0; g < nc; ++g) {
        if (!used[g]) A[static_cast<size_t>(g) * nc + g] = 1.0;
        X[static_cast<size_t>(g) * nc + g] = 1.0;
    }
    for (uint32_t c = 0; c < nc; ++c) {
        uint32_t piv = c;
        for (uint32_t r = c + 1; r < nc; ++r)
            if (std::fabs(A[static_cast<size_t>(r) * nc + c]) > std::fabs(A[static_cast<size_t>(piv) * nc + c])) piv = r;
        const double d = A[static_cast<size_t>(piv) * nc + c];
        if (!(std::fabs(d) > 0.0) || !std::isfinite(d)) return cudaSuccess;  // singular: no cluster path
        if (piv != c)
            for (uint32_t j = 0; j < nc; ++j) {
                std::swap(A[static_cast<size_t>(piv) * nc + j], A[static_cast<size_t>(c) * nc + j]);
                std::swap(X[static_cast<size_t>(piv) * nc + j], X[static_cast<size_t>(c) * nc + j]);
            }
        for (uint32_t j = 0; j < nc; ++j) {
            A[static_cast<size_t>(c) * nc + j] /= d;
            X[static_cast<size_t>(c) * nc + j] /= d;
        }
        for (uint32_t r = 0; r < nc; ++r) {
            if (r == c) continue;
            const double f = A[static_cast<size_t>(r) * nc + c];
            if (f == 0.0) continue;
            for (uint32_t j = 0; j < nc; ++j) {
                A[static_cast<size_t>(r) * nc + j] -= f * A[static_cast<size_t>(c) * nc + j];
                X[static_cast<size_t>(r) * nc + j] -= f * X[static_cast<size_t>(c) * nc + j];
            }
        }
    }
    e = sw_upload(s, &s->dsa_ainv, X);
    if (e != cudaSuccess) return e;
    s->dsa_cluster = cluster;
    return cudaSuccess;
}

void tr_sweep_opts_default(tr_sweep_opts *o) {
    if (!o) return;
    o->method = TR_SWEEP_GMRES;
    o->mode = TR_MODE_FP64;
    o->tol = 1e-8;
    o->max_iter = 1000;
    o->restart = 30;
    o->inner_tol = 0.0;
    o->max_outer = 30;
    o->precondition = TR_SWEEP_PREC_NONE;
    o->precond_tol = 1e-2;
    o->precond_engine = TR_SWEEP_DSA_AUTO;
}

tr_status tr_sweep_enable_dsa(tr_sweep *s, const tr_mesh_view *mesh, const tr_physics_view *phys) {
    SW_CHECK(s);
    if (!mesh || !mesh->mesh || !mesh->tetstart || !mesh->tetidx || !mesh->tetpos)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_enable_dsa: incomplete mesh view");
    if (mesh->nT != s->nT || mesh->nF != s->nF)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_enable_dsa: mesh differs from the sweep's");
    if (s->dsa) return TR_OK;
    const uint32_t nP = mesh->nP, nT = mesh->nT;
    if (mesh->nF && (!mesh->bnd || !mesh->facestart || !mesh->faceidx || !mesh->facepos))
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_enable_dsa: incomplete face arrays");
    if (mesh->tetstart[0] != 0 || mesh->tetstart[nP] != 4ull * nT)
        return sw_err(s, TR_ERR_MESH, "tr_sweep_enable_dsa: vertex -> cell table does not cover 4 nT entries");
    std::vector<uint32_t> vstart(mesh->tetstart, mesh->tetstart + nP + 1), vcj(4ull * nT);
    for (uint32_t v = 0; v < nP; ++v) {
        if (vstart[v + 1] < vstart[v]) return sw_err(s, TR_ERR_MESH, "tr_sweep_enable_dsa: tetstart decreases");
        for (uint32_t i = vstart[v]; i < vstart[v + 1]; ++i) {
            const uint32_t c = mesh->tetidx[i], j = mesh->tetpos[i];
            if (c >= nT || j > 3 || mesh->mesh[c].p[j] != v)
                return sw_err(s, TR_ERR_MESH, "tr_sweep_enable_dsa: inconsistent vertex -> cell table");
            vcj[i] = 4 * c + j;
        }
    }
    std::vector<uint4> cp(nT);
    for (uint32_t c = 0; c < nT; ++c) {
        const tr_idx *p = mesh->mesh[c].p;
        if (p[0] >= nP || p[1] >= nP || p[2] >= nP || p[3] >= nP)
            return sw_err(s, TR_ERR_MESH, "tr_sweep_enable_dsa: vertex index out of range");
        cp[c] = make_uint4(p[0], p[1], p[2], p[3]);
    }
    cudaSetDevice(s->device);
    tr_angular *ang = nullptr;
    tr_status st = tr_angular_create(0, &ang);
    if (st != TR_OK) return sw_err(s, st, "tr_sweep_enable_dsa: angular tables");
    tr_angular_view av;
    tr_angular_view_get(ang, &av);
    // Vacuum and incident faces carry the operator's l = 0 surface term, 1/2
    // of its face measure |s_x + s_y + s_z| (the face area on the axis-aligned
    // faces of a box), a Marshak condition for the homogeneous correction.
    // Reflective faces (zero current) carry none: they are left out of the
    // diffusion context's face list.
    const int32_t *bc = phys ? phys->face_bc : nullptr;
    std::vector<tr_face> fkeep;
    std::vector<tr_idx> fnew(mesh->nF, ~0u), fstart(nP + 1, 0), fidx, fpos;
    for (uint32_t f = 0; f < mesh->nF; ++f)
        if (!bc || bc[f] != TR_BC_REFLECTIVE) {
            fnew[f] = static_cast<tr_idx>(fkeep.size());
            fkeep.push_back(mesh->bnd[f]);
        }
    for (uint32_t v = 0; v < nP && mesh->nF; ++v) {
        for (tr_idx i = mesh->facestart[v]; i < mesh->facestart[v + 1]; ++i) {
            const tr_idx f = mesh->faceidx[i];
            if (f >= mesh->nF) {
                tr_angular_destroy(ang);
                return sw_err(s, TR_ERR_MESH, "tr_sweep_enable_dsa: face index out of range");
            }
            if (fnew[f] == ~0u) continue;
            fidx.push_back(fnew[f]);
            fpos.push_back(mesh->facepos[i]);
        }
        fstart[v + 1] = static_cast<tr_idx>(fidx.size());
    }
    tr_mesh_view mv = *mesh;
    mv.nF = static_cast<tr_idx>(fkeep.size());
    mv.bnd = fkeep.data();
    mv.facestart = fstart.data();
    mv.faceidx = fidx.data();
    mv.facepos = fpos.data();
    const tr_physics_view pv = {phys ? phys->kappa_abs_volume : nullptr, nullptr, nullptr, TR_SURFACE_AXIS};
    tr_ctx *ctx = nullptr;
    st = tr_ctx_create_ex(s->device, &mv, &av, &pv, &ctx);
    tr_angular_destroy(ang);
    if (st != TR_OK) return sw_err(s, st, std::string("tr_sweep_enable_dsa: ") + tr_last_error(nullptr));
    tr_ctx_info info;
    tr_ctx_info_get(ctx, &info);
    s->dsa = ctx;
    s->nP = nP;
    s->dsa_aslm = info.aslm;
    cudaError_t e = sw_upload(s, &s->vc_start, vstart);
    if (e == cudaSuccess) e = sw_upload(s, &s->vc_cj, vcj);
    if (e == cudaSuccess) e = sw_upload(s, &s->cell_p, cp);
    if (e == cudaSuccess) e = sw_alloc(s, &s->dsa_b, static_cast<size_t>(nP) * info.aslm);
    if (e == cudaSuccess) e = sw_alloc(s, &s->dsa_f, static_cast<size_t>(nP) * info.aslm);
    if (e != cudaSuccess) {
        tr_ctx_destroy(s->dsa);
        s->dsa = nullptr;
        return sw_cuda(s, e, "tr_sweep_enable_dsa");
    }
    if (nP <= kDsaClusterMaxRows) {
        e = dsa_assemble(s, mesh, phys);
        if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_enable_dsa: diffusion matrix");
    }
    return TR_OK;
}

tr_status tr_sweep_solve(tr_sweep *s, const tr_sweep_opts *opts, double *J, double *B, tr_sweep_report *rep) {
    SW_CHECK(s);
    if (!J) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_solve: null J");
    tr_sweep_opts o;
    tr_sweep_opts_default(&o);
    if (opts) o = *opts;
    if (o.restart < 1 || o.restart > kMaxRestart) return sw_err(s, TR_ERR_INVALID_ARG, "restart must be 1..64");
    if (o.mode != TR_MODE_FP64 && o.mode != TR_MODE_MIXED) return sw_err(s, TR_ERR_INVALID_ARG, "bad mode");
    if (o.method != TR_SWEEP_GMRES && o.method != TR_SWEEP_SOURCE_ITERATION)
        return sw_err(s, TR_ERR_INVALID_ARG, "bad method");
    if (o.precondition != TR_SWEEP_PREC_NONE && o.precondition != TR_SWEEP_PREC_DSA)
        return sw_err(s, TR_ERR_INVALID_ARG, "bad precondition");
    const bool dsa = o.precondition == TR_SWEEP_PREC_DSA;
    if (dsa && !s->dsa) return sw_err(s, TR_ERR_INVALID_ARG, "precondition DSA needs tr_sweep_enable_dsa");
    if (dsa && !(o.precond_tol > 0.0 && o.precond_tol < 1.0))
        return sw_err(s, TR_ERR_INVALID_ARG, "precond_tol must be in (0, 1)");
    DsaPlan plan;
    if (dsa) {
        if (o.precond_engine < TR_SWEEP_DSA_AUTO || o.precond_engine > TR_SWEEP_DSA_EVEN_PARITY)
            return sw_err(s, TR_ERR_INVALID_ARG, "bad precond_engine");
        if (o.precond_engine == TR_SWEEP_DSA_CLUSTER && !s->dsa_cluster)
            return sw_err(s, TR_ERR_UNSUPPORTED, "the one-cluster diffusion CG is not available for this sweep");
        plan.tol = o.precond_tol;
        plan.cluster = s->dsa_cluster > 0 && o.precond_engine != TR_SWEEP_DSA_EVEN_PARITY;
    }
    if (plan.cluster) {
        cudaError_t e0 = cudaMemsetAsync(s->dsa_stats, 0, 3 * sizeof(unsigned long long), s->stream);
        if (e0 != cudaSuccess) return sw_cuda(s, e0, "tr_sweep_solve");
    }
    s->prec_error.clear();
    const uint64_t n = s->nJ + s->nB;
    cudaError_t e = krylov_alloc(s, o.restart);
    if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_solve: allocation");
    cudaStream_t st = s->stream;
    const int64_t s32_0 = s->sweeps32, s64_0 = s->sweeps64, l0 = s->launches;
    const int64_t d0 = s->dsa_solves, di0 = s->dsa_iterations;
    cudaEventRecord(s->ev[0], st);
    // b = S_64(0) with sources; x = 0
    e = sweep_enqueue(s, 64, nullptr, nullptr, 1, s->kb, s->nB ? s->kb + s->nJ : nullptr);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->kx, 0, n * 8, st);
    double bn = 0.0;
    if (e == cudaSuccess) e = vnorm(s, s->kb, &bn);
    int its = 0, outer = 0;
    double res = 0.0;
    bool conv = false;
    const int gr = grid_for(s, n);
    if (e == cudaSuccess && bn == 0.0) conv = true;
    if (e == cudaSuccess && !conv) {
        if (o.method == TR_SWEEP_SOURCE_ITERATION) {
            // x <- S(x) with sources, in the mode's sweep precision; change measured in FP64
            const int prec = o.mode == TR_MODE_MIXED ? 32 : 64;
            e = cudaMemcpyAsync(s->kx, s->kb, n * 8, cudaMemcpyDeviceToDevice, st);
            while (e == cudaSuccess && its < o.max_iter) {
                e = sweep_enqueue(s, prec, s->kx, s->nB ? s->kx + s->nJ : nullptr, 1, s->kt,
                                  s->nB ? s->kt + s->nJ : nullptr);
                ++its;
                if (e != cudaSuccess) break;
                k_axpby<<<gr, 256, 0, st>>>(n, 1.0, s->kt, -1.0, s->kx);  // kx = kt - kx
                ++s->launches;
                double dn = 0.0, tn = 0.0;
                if ((e = vnorm(s, s->kx, &dn)) != cudaSuccess) break;
                if ((e = vnorm(s, s->kt, &tn)) != cudaSuccess) break;
                if (!std::isfinite(dn) || !std::isfinite(tn)) {  // diverged: not converged
                    res = dn;
                    break;
                }
                if (dsa) {
                    // x <- S(x) + C sigma_s (S(x) - x): the diffusion estimate of the error
                    if ((e = dsa_solve(s, s->kx, plan.tol, plan.cluster, plan.maxit)) != cudaSuccess) break;
                    e = dsa_prolong(s, s->kt, s->kx, plan.cluster);
                } else {
                    e = cudaMemcpyAsync(s->kx, s->kt, n * 8, cudaMemcpyDeviceToDevice, st);
                }
                res = tn > 0.0 ? dn / tn : 0.0;
                if (res < o.tol) {
                    conv = true;
                    break;
                }
            }
        } else if (o.mode == TR_MODE_FP64) {
            e = gmres(s, 64, 64, s->kb, s->kx, o.restart, o.tol, bn, 0.0, o.max_iter, &its, &res, nullptr, plan);
            conv = e == cudaSuccess && res <= o.tol;
        } else {
            // FP32 sweeps inside FP64 defect correction: each GMRES cycle starts
            // from the FP64 residual r = b - (I - T_64) x (one FP64 sweep) and
            // builds its Krylov space with FP32 sweeps; the correction is added
            // to x in FP64.  A cycle ends at its restart length, at the target,
            // or (inner_tol > 0) once it has reduced its residual by inner_tol.
            e = gmres(s, 32, 64, s->kb, s->kx, o.restart, o.tol, bn, o.inner_tol, o.max_iter, &its, &res, &outer,
                      plan);
            conv = e == cudaSuccess && res <= o.tol;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(J, s->kx, s->nJ * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && B && s->nB) e = cudaMemcpyAsync(B, s->kx + s->nJ, s->nB * 8, cudaMemcpyDeviceToDevice, st);
    cudaEventRecord(s->ev[1], st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaErrorUnknown && !s->prec_error.empty()) {
        cudaStreamSynchronize(st);
        return sw_err(s, TR_ERR_CUDA, "tr_sweep_solve: " + s->prec_error);
    }
    if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_solve");
    if (plan.cluster) {
        unsigned long long st3[3] = {0, 0, 0};
        e = cudaMemcpy(st3, s->dsa_stats, sizeof(st3), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_solve");
        s->dsa_iterations += static_cast<int64_t>(st3[0]);
        s->dsa_solves += static_cast<int64_t>(st3[1]);
        if (st3[2]) return sw_err(s, TR_ERR_NAN, "tr_sweep_solve: diffusion CG produced a non-finite residual");
    }
    if (rep) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]);
        rep->converged = conv ? 1 : 0;
        rep->iterations = its;
        rep->outer_steps = outer;
        rep->sweeps_f32 = s->sweeps32 - s32_0;
        rep->sweeps_f64 = s->sweeps64 - s64_0;
        rep->residual = res;
        rep->rhs_norm = bn;
        rep->device_ms = ms;
        rep->kernel_launches = s->launches - l0;
        rep->precond_solves = static_cast<int32_t>(s->dsa_solves - d0);
        rep->precond_iterations = static_cast<int32_t>(s->dsa_iterations - di0);
    }
    if (!conv) return sw_err(s, TR_ERR_NOT_CONVERGED, "tr_sweep_solve: not converged");
    return TR_OK;
}

// coefficient records [nT][4]: sigma_t V, sigma_s V, sigma_a V B / 4 (the
// vertex map in the fourth word is kept)
__global__ void k_set_coef(uint32_t nT, const double *stv, const double *ssv, const double *ext, double *coef64,
                           float *coef32) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nT; c += gridDim.x * blockDim.x) {
        coef64[4ull * c] = stv[c];
        coef64[4ull * c + 1] = ssv[c];
        coef64[4ull * c + 2] = ext[c];
        coef32[4ull * c] = static_cast<float>(stv[c]);
        coef32[4ull * c + 1] = static_cast<float>(ssv[c]);
        coef32[4ull * c + 2] = static_cast<float>(ext[c]);
    }
}

tr_status tr_sweep_set_coefficients(tr_sweep *s, const double *kappa_volume, const double *kappa_abs_volume,
                                    const double *I_p) {
    SW_CHECK(s);
    if (!kappa_volume) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_set_coefficients: null kappa_volume");
    const uint32_t nT = s->nT;
    cudaSetDevice(s->device);
    std::vector<double> bpl(nT), stv(nT), ssv(nT), ext(nT);
    cudaError_t e = cudaSuccess;
    if (I_p) std::copy(I_p, I_p + nT, bpl.begin());
    else e = cudaMemcpy(bpl.data(), s->B64, sizeof(double) * nT, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_set_coefficients");
    for (uint32_t c = 0; c < nT; ++c) {
        const double kv = kappa_volume[c], sav = kappa_abs_volume ? kappa_abs_volume[c] : kv;
        if (!(kv > 0.0) || !(sav >= 0.0) || sav > kv * (1.0 + 1e-12))
            return sw_err(s, TR_ERR_INVALID_ARG,
                          "tr_sweep_set_coefficients: need kappa_volume > 0 and 0 <= sigma_a V <= sigma_t V");
        stv[c] = kv;
        ssv[c] = kv - sav;
        ext[c] = sav * bpl[c] / 4.0;
    }
    auto up = [&](auto *dst, const std::vector<double> &v) {
        using D = std::remove_pointer_t<decltype(dst)>;
        if (e != cudaSuccess) return;
        if constexpr (std::is_same_v<D, double>) {
            e = cudaMemcpy(dst, v.data(), sizeof(double) * nT, cudaMemcpyHostToDevice);
        } else {
            std::vector<float> f(v.begin(), v.end());
            e = cudaMemcpy(dst, f.data(), sizeof(float) * nT, cudaMemcpyHostToDevice);
        }
    };
    cudaStreamSynchronize(s->stream);  // nothing in flight reads the old values
    up(s->stv64, stv);
    up(s->ssv64, ssv);
    up(s->ext64, ext);
    up(s->stv32, stv);
    up(s->ssv32, ssv);
    up(s->ext32, ext);
    if (I_p) up(s->B64, bpl);
    if (e == cudaSuccess) {
        k_set_coef<<<grid_for(s, nT), 256, 0, s->stream>>>(nT, s->stv64, s->ssv64, s->ext64, s->coef64, s->coef32);
        ++s->launches;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    s->last_prec = 0;  // psi of the last sweep belongs to the old coefficients
    return sw_cuda(s, e, "tr_sweep_set_coefficients");
}

tr_status tr_sweep_create_group(tr_sweep *parent, const double *kappa_volume, const double *kappa_abs_volume,
                                const double *I_p, tr_sweep **out) {
    SW_CHECK(parent);
    if (!out || !kappa_volume) return sw_err(parent, TR_ERR_INVALID_ARG, "tr_sweep_create_group: null argument");
    *out = nullptr;
    if (parent->parent)
        return sw_err(parent, TR_ERR_INVALID_ARG, "tr_sweep_create_group: the parent is itself a group");
    cudaSetDevice(parent->device);
    tr_sweep *G = new (std::nothrow) tr_sweep();
    if (!G) return sw_err(parent, TR_ERR_OUT_OF_MEMORY, "tr_sweep_create_group: host allocation");
    const tr_sweep &P = *parent;
    // shared: sizes, geometry, boundary tables, ordinates, schedule, records
    G->device = P.device;
    G->num_sms = P.num_sms;
    G->nT = P.nT; G->nF = P.nF; G->nq = P.nq; G->nrefl = P.nrefl; G->nlag = P.nlag; G->maxlev = P.maxlev;
    G->forced = P.forced; G->lstride = P.lstride; G->nbf = P.nbf; G->nB = P.nB; G->nJ = P.nJ;
    G->s64 = P.s64; G->s32 = P.s32; G->finc64 = P.finc64; G->finc32 = P.finc32;
    G->nbr = P.nbr; G->fbc = P.fbc; G->rslot = P.rslot; G->map = P.map; G->bcell = P.bcell; G->bface = P.bface;
    G->rent = P.rent; G->ent_cell = P.ent_cell; G->ent_qout = P.ent_qout; G->nent = P.nent;
    for (int i = 0; i < 4; ++i) G->o64[i] = P.o64[i];
    for (int i = 0; i < 3; ++i) G->o32[i] = P.o32[i];
    G->Wm = P.Wm; G->vol64 = P.vol64; G->ord_host = P.ord_host;
    G->task = P.task; G->lvl = P.lvl; G->nlev = P.nlev; G->lag_keys = P.lag_keys; G->f4_keys = P.f4_keys;
    G->f4_codes = P.f4_codes; G->n_f4 = P.n_f4;
    G->mom_kernel = P.mom_kernel; G->shape32 = P.shape32;
    // owned: coefficients (the fourth value of each packed record carries the
    // shared vertex map, copied from the parent), reductions, events, stream
    const size_t nT = P.nT;
    cudaError_t e = cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking);
    for (double **p : {&G->stv64, &G->ssv64, &G->ext64, &G->B64})
        if (e == cudaSuccess) e = sw_alloc(G, p, nT);
    for (float **p : {&G->stv32, &G->ssv32, &G->ext32})
        if (e == cudaSuccess) e = sw_alloc(G, p, nT);
    if (e == cudaSuccess) e = sw_alloc(G, &G->coef64, 4 * nT);
    if (e == cudaSuccess) e = sw_alloc(G, &G->coef32, 4 * nT);
    if (e == cudaSuccess) e = cudaMemcpy(G->coef64, P.coef64, 32 * nT, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(G->coef32, P.coef32, 16 * nT, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(G->B64, P.B64, 8 * nT, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = sw_alloc(G, &G->partials, (kMaxRestart + 2ull) * kDotGrid);
    if (e == cudaSuccess) e = sw_alloc(G, &G->red, 256);
    if (e == cudaSuccess) e = sw_alloc(G, &G->counter, 4);
    if (e == cudaSuccess) e = cudaMemset(G->counter, 0, 16);
    if (e == cudaSuccess) e = cudaEventCreate(&G->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&G->ev[1]);
    if (e != cudaSuccess) {
        sw_free(G);
        return sw_cuda(parent, e, "tr_sweep_create_group");
    }
    G->parent = parent;
    ++parent->groups;
    const tr_status st = tr_sweep_set_coefficients(G, kappa_volume, kappa_abs_volume, I_p);
    if (st != TR_OK) {
        const std::string msg = G->last_error;
        sw_free(G);
        return sw_err(parent, st, msg);
    }
    *out = G;
    return TR_OK;
}

tr_status tr_sweep_release_work(tr_sweep *s) {
    SW_CHECK(s);
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (void **p : {(void **)&s->psi64, (void **)&s->psi32, (void **)&s->J32, (void **)&s->Bi32, (void **)&s->Bo32,
                     (void **)&s->kv, (void **)&s->kb, (void **)&s->kx, (void **)&s->kt, (void **)&s->kh,
                     (void **)&s->kz}) {
        sw_release(s, *p);
        *p = nullptr;
    }
    s->kv_m = s->kz_m = 0;
    s->last_prec = 0;
    return TR_OK;
}

tr_status tr_sweep_outflow(tr_sweep *s, const int32_t *face_mask, double *F) {
    SW_CHECK(s);
    if (!face_mask || !F) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_outflow: null argument");
    if (!s->last_prec) return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_outflow: no sweep has run");
    std::vector<uint8_t> m(s->nF + 1, 0);
    for (uint32_t f = 0; f < s->nF; ++f) m[f] = face_mask[f] != 0;
    uint8_t *dm = nullptr;
    cudaError_t e = cudaMalloc(&dm, m.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(dm, m.data(), m.size(), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
        if (s->last_prec == 64)
            k_outflow<double><<<kRedGrid, 256, 0, s->stream>>>(s->nT, s->nq, s->nbf, s->bcell, s->bface, dm, s->s64,
                                                               s->o64[0], s->o64[1], s->o64[2], s->o64[3], s->psi64,
                                                               s->partials, s->counter, s->red);
        else
            k_outflow<float><<<kRedGrid, 256, 0, s->stream>>>(s->nT, s->nq, s->nbf, s->bcell, s->bface, dm, s->s64,
                                                              s->o64[0], s->o64[1], s->o64[2], s->o64[3], s->psi32,
                                                              s->partials, s->counter, s->red);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(F, s->red, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (dm) cudaFree(dm);
    return sw_cuda(s, e, "tr_sweep_outflow");
}

tr_status tr_sweep_gradient(tr_sweep *fwd, tr_sweep *adj, int precision, const double *J, const double *B,
                            const double *J_adj, double *dF_dsigma_a, double *dF_dsigma_s) {
    SW_CHECK(fwd);
    if (!adj || !J || !J_adj || !dF_dsigma_a || !dF_dsigma_s)
        return sw_err(fwd, TR_ERR_INVALID_ARG, "tr_sweep_gradient: null argument");
    if (precision != 32 && precision != 64) return sw_err(fwd, TR_ERR_INVALID_ARG, "precision must be 32 or 64");
    if (!aligned16(J) || !aligned16(B) || !aligned16(J_adj))
        return sw_err(fwd, TR_ERR_INVALID_ARG, "tr_sweep_gradient: device vectors must be 16-byte aligned");
    if (adj->device != fwd->device || adj->nT != fwd->nT || adj->nq != fwd->nq)
        return sw_err(fwd, TR_ERR_INVALID_ARG, "tr_sweep_gradient: adjoint sweep of another problem");
    const uint32_t nq = fwd->nq;
    for (uint32_t q = 0; q < nq; ++q)
        for (int d = 0; d < 3; ++d)
            if (adj->ord_host[d * nq + q] != -fwd->ord_host[d * nq + q])
                return sw_err(fwd, TR_ERR_INVALID_ARG, "tr_sweep_gradient: the adjoint ordinates must be -Omega_q");
    if (fwd->nrefl || fwd->nlag || adj->nrefl || adj->nlag)
        return sw_err(fwd, TR_ERR_UNSUPPORTED,
                      "tr_sweep_gradient: reflective faces and cut dependency cycles are not supported");
    // forward angular flux recomputed from the converged (checkpointed) J, B;
    // adjoint angular flux from the adjoint scalar flux
    cudaError_t e = sweep_enqueue(fwd, precision, J, B, 1, nullptr, nullptr);
    if (e == cudaSuccess) e = sweep_enqueue(adj, precision, J_adj, nullptr, 1, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(adj->stream);
    if (e == cudaSuccess) {
        const int gr = grid_for(fwd, fwd->nT);
        if (precision == 64)
            k_gradient<double><<<gr, 256, 0, fwd->stream>>>(fwd->nT, nq, fwd->o64[3], fwd->psi64, adj->psi64, J, J_adj,
                                                            fwd->vol64, fwd->B64, dF_dsigma_a, dF_dsigma_s);
        else
            k_gradient<float><<<gr, 256, 0, fwd->stream>>>(fwd->nT, nq, fwd->o64[3], fwd->psi32, adj->psi32, J, J_adj,
                                                           fwd->vol64, fwd->B64, dF_dsigma_a, dF_dsigma_s);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(fwd->stream);
    return sw_cuda(fwd, e, "tr_sweep_gradient");
}

tr_status tr_sweep_bench(tr_sweep *s, int precision, int iters, double *ms_per_sweep) {
    SW_CHECK(s);
    if ((precision != 32 && precision != 64) || iters < 1 || !ms_per_sweep)
        return sw_err(s, TR_ERR_INVALID_ARG, "tr_sweep_bench: bad arguments");
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = sweep_enqueue(s, precision, nullptr, nullptr, 1, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev[0], s->stream);
    for (int i = 0; i < iters && e == cudaSuccess; ++i)
        e = sweep_enqueue(s, precision, nullptr, nullptr, 1, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev[1], s->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(s->ev[1]);
    if (e != cudaSuccess) return sw_cuda(s, e, "tr_sweep_bench");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]);
    *ms_per_sweep = ms / iters;
    return TR_OK;
}

}  // extern "C"
