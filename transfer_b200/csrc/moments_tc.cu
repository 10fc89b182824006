// Moments of the FP32 angular flux on the 5th-generation tensor cores
// (tcgen05, accumulators in tensor memory), psi streamed by TMA.
//
//   mom[n][r] = sum_q W[n][q] psi[q][r],   r = 4 c + j over the M = 4 nT
//   cell-vertex values, n < 16 real harmonics (l <= 3), W = w_q Y_n(Omega_q)
//
// This is MeshData::ComputeMoments (MeshData.cpp:96-116, U = 4 pi I_00 and
// the l = 1, 2 moments of the even-parity solution) generalised to discrete
// ordinates: a (M x nq) . (nq x 16) product, A = psi^T read once from HBM.
//
// Split TF32 (3xTF32) with FP32 accumulation: psi = a_hi + a_lo and
// W = w_hi + w_lo, where the hi parts keep the 10-bit TF32 mantissa
// (truncation: the tensor core reads the top 19 bits of an FP32 word) and
// the lo parts are the exact FP32 remainders; the three products
// a_hi w_hi + a_hi w_lo + a_lo w_hi are summed, a_lo w_lo (~2^-22) dropped.
//
// Layout and roles (one CTA per SM, persistent over 128-row tiles):
//   A (psi)   TMA tiles of 32 rows x 32 ordinates, four per stage: a stage is
//             128 rows x 32 ordinates, MN-major (rows contiguous), as many
//             stages in flight as shared memory holds beside the weights (up
//             to kMaxStages, 160 KB: HBM latency under full load needs about
//             that much in flight per SM; 6 stages reached 3.5 TB/s).  MN-major TF32 operands take one shared-memory
//             form, the 128-byte swizzle on 32-byte units (atoms of 32 rows x 4
//             ordinates, 512 B; the 32-byte chunk index of each 128-byte
//             ordinate row XORed with the row's index mod 4), which TMA writes
//             in its SWIZZLE_128B_ATOM_32B mode;
//   B (W)     [w_hi | w_lo] as one N = 32 operand, K-major, built in shared
//             memory once per CTA from the FP64 weights;
//   a_lo      written by the split warps into tensor memory (tcgen05.st), the
//             A operand of the third product (A from tensor memory), in
//             kLoSlots slots of its own, each freed when its products finish;
//   D         per tile (double-buffered) kAccGroups 128 x 32 FP32 accumulators
//             of a [w_hi | w_lo], the 8-ordinate steps dealt to them in turn
//             (with two issuers, issuer i's steps to accumulators 2i and
//             2i + 1), and a 128 x 16 accumulator of a_lo w_hi per issuer,
//             in tensor memory.  The
//             tensor core's FP32 accumulation truncates, so each accumulation
//             into a running sum loses about half an ulp the same way; dealing
//             the steps over four accumulators and summing them in FP64 cuts
//             that bias fourfold (80 accumulations into one sum at 308
//             ordinates left moments 5e-6 low).
//   warp 0    TMA producer (and tensor-memory allocation), with warp 3 a
//             second producer of alternate stages;
//   warp 1    MMA issuer: per 8-ordinate step one N = 32 product from shared
//             memory and one N = 16 product with A from tensor memory; with
//             warp 2 a second issuer of alternate stages (its own a_lo w_hi
//             sum, accumulators 2 and 3);
//   warps 4-11 split each stage (a_lo = a - trunc(a)) into tensor memory,
//             two warpgroups of 16 ordinates each;
//   warps 12-15 read each finished tile's accumulators back (tcgen05.ld), sum
//             them in FP64 and store the 16 moments, while the split warps
//             go on with the next tile (the accumulators are double-buffered).
// Every wait is bounded (kWaitNs of the global timer): past it the kernel
// sets bit 0 of *err, every role stops, in-flight copies and products are
// waited for (bounded), tensor memory is freed and the kernel returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "moments_tc.h"

namespace transfer {

namespace {

constexpr int kTileM = 128;        // rows per tile (one MMA M)
constexpr int kStageK = 32;        // ordinates per stage
constexpr int kMaxStages = 10;     // shared-memory stages (the launch picks how many fit)
// tensor-memory slots of a_lo: how many stages the split warps may run ahead
// of the products that free them (each slot returns only after its stage's
// products finish, so the slots bound the stages in flight on that loop)
#ifndef TR_MOM_LO_SLOTS
#define TR_MOM_LO_SLOTS 4
#endif
constexpr uint32_t kLoSlots = TR_MOM_LO_SLOTS;
static_assert(kLoSlots % 2 == 0, "two issuers take alternate a_lo slots");
constexpr int kAtomBytes = 32 * 4 * kStageK;         // 32 rows x 32 ordinates x 4 B = 4 KB
constexpr int kStageBytes = 4 * kAtomBytes;          // 16 KB
constexpr uint32_t kSplitWarps = 8;                  // warps 4-11; warps 12-15 drain the accumulators
constexpr int kThreads = 32 * (4 + kSplitWarps + 4);
constexpr uint32_t kAccGroups = 4;                   // accumulators of a [w_hi | w_lo] per tile
constexpr uint32_t kBufCols = 160;                   // kAccGroups x 32 + 2 x 16 (a_lo w_hi, one per issuer)
// MMA-issuing (and TMA-producing) threads: 1, or 2 taking alternate stages
// where a tile has at least two stages (more than 32 ordinates)
#ifndef TR_MOM_ISSUERS
#define TR_MOM_ISSUERS 2
#endif
constexpr uint32_t kTmemCols = 512;                  // 2 tile buffers + kLoSlots x 32 a_lo
constexpr uint32_t kLoCol0 = 2 * kBufCols;
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per wait

static_assert(kLoCol0 + kLoSlots * kStageK <= kTmemCols, "tensor-memory plan");
constexpr int kSmemHeader = 1024;  // barriers and flags, ahead of the 1024-aligned stages

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false when the CTA has aborted or this wait timed out (then
// the abort flag and bit 0 of *err are set).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          unsigned int *err) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (uint32_t spin = 0;; ++spin) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if ((spin & 63u) == 63u && global_ns() - t0 > kWaitNs) {
            *abort_flag = 1;
            atomicOr(err, 1u);
            return false;
        }
    }
}

// The same wait for a whole warp: lane 0 polls and the outcome is broadcast,
// so every lane takes the same branch before the warp-wide (.sync.aligned)
// tensor-memory instructions that follow.
__device__ __forceinline__ bool mbar_wait_warp(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                               unsigned int *err) {
    int ok = 0;
    if ((threadIdx.x & 31u) == 0) ok = mbar_wait(bar, parity, abort_flag, err) ? 1 : 0;
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// UMMA shared-memory descriptors (version 1).  A: MN-major, 128-byte swizzle
// with a 32-byte base (layout type 1), 32-row atoms 4 KB apart (leading
// offset), 4-ordinate groups 512 B apart (stride offset).  B: K-major, no swizzle, 8 x 16-byte core matrices; the
// next 4 ordinates 512 B on (leading offset), the next 8 harmonics 128 B on
// (stride offset).
__device__ __forceinline__ uint64_t desc_a(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(4096 >> 4) << 16) |
           (static_cast<uint64_t>(512 >> 4) << 32) | (1ull << 46) | (1ull << 61);
}
__device__ __forceinline__ uint64_t desc_b(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(512 >> 4) << 16) |
           (static_cast<uint64_t>(128 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: D FP32, A and B TF32, M = 128, N, A major
__host__ __device__ constexpr uint32_t idesc_tf32(uint32_t n, uint32_t a_mn) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (a_mn << 15) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float tf32_trunc(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

struct Smem {
    uint64_t full[kMaxStages], empty[kMaxStages], lo_ready[kLoSlots], lo_empty[kLoSlots];
    uint64_t acc_full[2], acc_empty[2], drain;
    uint32_t tmem_base;
    int abort_flag;
};

}  // namespace

__global__ void __launch_bounds__(kThreads, 1)
    k_moments_tcgen05(const __grid_constant__ CUtensorMap psi_map, uint32_t M, uint32_t nq, uint32_t nqp,
                      const double *__restrict__ W, int nmom, double *__restrict__ mom, unsigned int *err,
                      uint32_t nstages, uint32_t issuers) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned base (the swizzle pattern repeats every 512 B)
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    static_assert(sizeof(Smem) <= kSmemHeader, "barrier header");
    Smem &sh = *reinterpret_cast<Smem *>(base);
    uint8_t *smA = base + kSmemHeader;                     // nstages x 16 KB (1024-aligned)
    uint8_t *smB = smA + nstages * kStageBytes;            // nqp x 128 B
    volatile int *abort_flag = &sh.abort_flag;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t tiles = (M + kTileM - 1) / kTileM, nks = nqp / kStageK;

    // B = [w_hi | w_lo] (harmonic n < 16: hi, 16 + n: lo) in K-major core matrices
    for (uint32_t i = threadIdx.x; i < nqp * 32; i += blockDim.x) {
        const uint32_t k = i >> 5, n = i & 31u, h = n & 15u;
        const double w = (k < nq && static_cast<int>(h) < nmom) ? W[static_cast<size_t>(h) * nq + k] : 0.0;
        const float hi = tf32_trunc(static_cast<float>(w));
        const float v = n < 16 ? hi : static_cast<float>(w - static_cast<double>(hi));
        const uint32_t off = (((k >> 2) * 4 + (n >> 3)) * 128) + (n & 7u) * 16 + (k & 3u) * 4;
        *reinterpret_cast<float *>(smB + off) = v;
    }
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < nstages; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (uint32_t l = 0; l < kLoSlots; ++l) {
            mbar_init(smem_u32(&sh.lo_ready[l]), kSplitWarps);
            mbar_init(smem_u32(&sh.lo_empty[l]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&sh.acc_full[b]), issuers);
            mbar_init(smem_u32(&sh.acc_empty[b]), 4);
        }
        mbar_init(smem_u32(&sh.drain), issuers);
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the weights were written by ordinary stores; the tensor cores read
    // them through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sh.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;

    if ((warp == 0 || (warp == 3 && issuers == 2)) && lane == 0) {
        // ---- TMA producer(s).  With two, producer i (warps 0 and 3) fills
        // the stages it = i mod 2 (with the two MMA issuers, 4.39 -> 3.21 ms
        // on the 2.78 M-tet sphere with 302 ordinates; issuing each stage's
        // four copies from four lanes changed nothing).
        const uint32_t me = warp == 0 ? 0u : 1u;
        uint32_t it = 0, inflight = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x)
            for (uint32_t ks = 0; ks < nks; ++ks, ++it) {
                if (issuers == 2 && (it & 1u) != me) continue;
                const uint32_t s = it % nstages, ph = (it / nstages) & 1u;
                if (!(ok = mbar_wait(smem_u32(&sh.empty[s]), ph ^ 1u, abort_flag, err))) break;
                const uint32_t fb = smem_u32(&sh.full[s]);
                mbar_expect_tx(fb, kStageBytes);
                const uint32_t dst = smem_u32(smA + s * kStageBytes);
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    tma_load_2d(dst + a * kAtomBytes, &psi_map, static_cast<int>(tile * kTileM + a * 32),
                                static_cast<int>(ks * kStageK), fb);
                inflight = it + 1;
            }
        if (!ok) {  // aborted: wait (bounded, own timer) for the copies this thread issued
            for (uint32_t j = inflight > nstages ? inflight - nstages : 0; j < inflight; ++j) {
                if (issuers == 2 && (j & 1u) != me) continue;
                const uint32_t bar = smem_u32(&sh.full[j % nstages]), ph = (j / nstages) & 1u;
                const unsigned long long t0 = global_ns();
                while (!mbar_try(bar, ph) && global_ns() - t0 < kWaitNs) {
                }
            }
        }
    } else if ((warp == 1 || (warp == 2 && issuers == 2)) && lane == 0) {
        // ---- MMA issuer(s).  With two issuers, issuer i takes the stages
        // it = i mod 2 (nstages and kLoSlots are even then, so every barrier
        // phase an issuer waits for follows one it consumed itself) into
        // accumulators 2i and 2i + 1 and its own a_lo w_hi sum (columns
        // 128 + 16 i); one thread issuing the stage's eight MMAs and two
        // commits took ~1,300 cycles a stage and bound the kernel.
        const uint32_t me = warp - 1;
        constexpr uint32_t id_hi = idesc_tf32(32, 1), id_lo = idesc_tf32(16, 0);
        uint32_t it = 0, tcount = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x, ++tcount) {
            const uint32_t b = tcount & 1u, bph = (tcount >> 1) & 1u;
            if (!(ok = mbar_wait(smem_u32(&sh.acc_empty[b]), bph ^ 1u, abort_flag, err))) break;
            tc_fence_after();
            const uint32_t d = tmem + kBufCols * b;
            bool started = false;  // this issuer's accumulators of the tile hold a sum
            for (uint32_t ks = 0; ks < nks; ++ks, ++it) {
                if (issuers == 2 && (it & 1u) != me) continue;
                const uint32_t s = it % nstages, ph = (it / nstages) & 1u;
                const uint32_t l = it % kLoSlots, lph = (it / kLoSlots) & 1u;
                if (!(ok = mbar_wait(smem_u32(&sh.full[s]), ph, abort_flag, err))) break;
                if (!(ok = mbar_wait(smem_u32(&sh.lo_ready[l]), lph, abort_flag, err))) break;
                tc_fence_after();
                const uint32_t a0 = smem_u32(smA + s * kStageBytes);
                const uint32_t b0 = smem_u32(smB) + ks * 4u * 1024u;
                const uint32_t dlo = d + 32u * kAccGroups + 16u * me;
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk) {
                    // one issuer: 8-ordinate step kk goes to accumulator kk;
                    // two: steps 0-1 to accumulator 2 me, 2-3 to 2 me + 1.
                    // Each starts from zero with the issuer's first stage.
                    const uint64_t bd = desc_b(b0 + kk * 1024u);
                    const uint32_t g = issuers == 2 ? 2u * me + (kk >> 1) : kk;
                    const bool acc_hi = started || (issuers == 2 && (kk & 1u));
                    mma_ss(d + 32u * g, desc_a(a0 + kk * 1024u), bd, id_hi, acc_hi ? 1u : 0u);
                    mma_ts(dlo, tmem + kLoCol0 + kStageK * l + 8u * kk, bd, id_lo, (started || kk) ? 1u : 0u);
                }
                started = true;
                mma_commit(smem_u32(&sh.empty[s]));     // the stage is free once these finish,
                mma_commit(smem_u32(&sh.lo_empty[l]));  // and so is its a_lo slot
            }
            if (!ok) break;
            mma_commit(smem_u32(&sh.acc_full[b]));
        }
        // every product issued has finished before tensor memory is freed
        mma_commit(smem_u32(&sh.drain));
        const unsigned long long t0 = global_ns();
        while (!mbar_try(smem_u32(&sh.drain), 0) && global_ns() - t0 < kWaitNs) {
        }
    } else if (warp >= 4 && warp < 4 + kSplitWarps) {
        // ---- split: a_lo of 16 ordinates of the stage into tensor memory;
        // warp w handles lanes 32 (w % 4) .. + 31 and ordinates 16 h .. + 15
        const uint32_t wq = warp & 3u, h = (warp - 4) >> 2;
        const uint32_t lane_addr = (32u * wq) << 16;
        uint32_t it = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x)
            for (uint32_t ks = 0; ks < nks; ++ks, ++it) {
                const uint32_t s = it % nstages, ph = (it / nstages) & 1u;
                const uint32_t l = it % kLoSlots, lph = (it / kLoSlots) & 1u;
                if (!(ok = mbar_wait_warp(smem_u32(&sh.full[s]), ph, abort_flag, err))) break;
                if (!(ok = mbar_wait_warp(smem_u32(&sh.lo_empty[l]), lph ^ 1u, abort_flag, err))) break;
                tc_fence_after();
                // row 32 wq + lane of the stage: atom wq, word lane of each
                // 128-byte ordinate row (32-byte chunk c stored at c ^ (k % 4))
                const uint8_t *atom = smA + s * kStageBytes + wq * kAtomBytes;
                uint32_t lo[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint32_t k = 16u * h + j;
                    const uint32_t off = k * 128 + (((lane >> 3) ^ (k & 3u)) << 5) + (lane & 7u) * 4;
                    const float a = *reinterpret_cast<const float *>(atom + off);
                    lo[j] = __float_as_uint(a - tf32_trunc(a));
                }
                tmem_st16(tmem + lane_addr + kLoCol0 + kStageK * l + 16u * h, lo);
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&sh.lo_ready[l]));
            }
    } else if (warp >= 4 + kSplitWarps) {
        // ---- epilogue: each finished tile's accumulators, summed in FP64
        const uint32_t wq = warp & 3u;
        const uint32_t lane_addr = (32u * wq) << 16;
        uint32_t tcount = 0;
        for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++tcount) {
            const uint32_t b = tcount & 1u, bph = (tcount >> 1) & 1u;
            if (!mbar_wait_warp(smem_u32(&sh.acc_full[b]), bph, abort_flag, err)) break;
            tc_fence_after();
            double acc[16];
#pragma unroll
            for (int n = 0; n < 16; ++n) acc[n] = 0.0;
            const uint32_t t0 = tmem + lane_addr + kBufCols * b;
#pragma unroll 1
            for (uint32_t g = 0; g <= kAccGroups; ++g) {  // the kAccGroups sums, then a_lo w_hi (16 columns)
                uint32_t v[32];
                tmem_ld32(t0 + 32u * g, v);
                tmem_wait_ld();
#pragma unroll
                for (int n = 0; n < 16; ++n)
                    acc[n] += static_cast<double>(__uint_as_float(v[n])) +
                              ((g < kAccGroups || issuers == 2) ? static_cast<double>(__uint_as_float(v[16 + n]))
                                                                : 0.0);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh.acc_empty[b]));
            const uint64_t row = static_cast<uint64_t>(tile) * kTileM + 32u * wq + lane;
            if (row < M) {
#pragma unroll
                for (int n = 0; n < 16; ++n)
                    if (n < nmom) mom[static_cast<uint64_t>(n) * M + row] = acc[n];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) {
        __syncwarp();  // lane 0 comes from the producer branch: reconverge for the warp-wide dealloc
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

namespace {
constexpr size_t kSmemLimit = 227u * 1024u;
// shared memory of a launch with `stages` stages for nq ordinates: alignment
// slack, the barrier header, the stages and the weight table
size_t smem_bytes(uint32_t nq, uint32_t stages) {
    const uint32_t nqp = (nq + kStageK - 1) / kStageK * kStageK;
    return 1024 + kSmemHeader + static_cast<size_t>(stages) * kStageBytes + static_cast<size_t>(nqp) * 128;
}
// the most stages (<= kMaxStages) that fit beside the weights; 0 if fewer than 3
uint32_t stages_for(uint32_t nq) {
    for (uint32_t st = kMaxStages; st >= 3; --st)
        if (smem_bytes(nq, st) <= kSmemLimit) return st;
    return 0;
}
}  // namespace

size_t moments_tcgen05_smem(uint32_t nq) {
    const uint32_t st = stages_for(nq);
    return st ? smem_bytes(nq, st) : 0;
}

bool moments_tcgen05_supported(uint32_t M, uint32_t nq) {
    return M > 0 && M % 4 == 0 && nq > 0 && stages_for(nq) != 0;
}

namespace {
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}
}  // namespace

cudaError_t launch_moments_tcgen05(const float *psi, uint32_t M, uint32_t nq, const double *W, int nmom,
                                   double *mom, unsigned int *err, int num_sms, cudaStream_t stream) {
    if (!moments_tcgen05_supported(M, nq) || nmom < 1 || nmom > 16) return cudaErrorInvalidValue;
    EncodeTiled enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    // psi as a 2-D tensor: x = row (M, contiguous), y = ordinate (nq, stride 4 M bytes)
    CUtensorMap map;
    const cuuint64_t dims[2] = {M, nq};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(M) * 4};
    const cuuint32_t box[2] = {32, kStageK};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(psi), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const size_t smem = moments_tcgen05_smem(nq);
    static bool attr = false;  // the opt-in is per function, one process-wide setting
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_moments_tcgen05, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             227 * 1024);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const uint32_t tiles = (M + kTileM - 1) / kTileM;
    const int grid = static_cast<int>(tiles < static_cast<uint32_t>(num_sms) ? tiles : num_sms);
    const uint32_t nqp = (nq + kStageK - 1) / kStageK * kStageK;
    const uint32_t issuers = (TR_MOM_ISSUERS == 2 && nqp >= 2 * kStageK) ? 2u : 1u;
    uint32_t stages = stages_for(nq);
    if (issuers == 2) stages &= ~1u;  // even: a stage's barrier phases then alternate with one issuer
    k_moments_tcgen05<<<grid, kThreads, smem, stream>>>(map, M, nq, nqp, W, nmom, mom, err, stages, issuers);
    return cudaGetLastError();
}

// ------------------------------------------------------------ FFMA2 form
// The same contraction on paired FP32 FMAs (FFMA2: two independent
// round-to-nearest FMAs per instruction), psi streamed by TMA as above.  The
// tensor-core form issues eight small MMAs (M 128, N 32 or 16, K 8) per 16 KB
// stage from one thread, about 1,300 cycles a stage; here the 16 FMAs an
// element needs take a fraction of the SM's issue rate.  Measured on the
// 2.78 M-tet sphere with 302 ordinates, both forms take the same time
// (3.76-3.79 ms, 3.9 TB/s): neither the MMA issue nor the FMAs bound the
// contraction; a TMA stream of the same tiles with no work at all tops out
// at 5.1 TB/s.  One TMA box of 128 rows x 32 ordinates per 16 KB stage (rows
// are the contiguous dimension, no swizzle), up to 8 stages in flight, one
// producer thread.  8 consumer warps: warp w takes ordinates w, w + 8,
// w + 16, w + 24 of each stage and lane l rows 4l .. 4l + 3 of the tile (one
// 16-byte shared load per ordinate, the ordinate's 16 FP32 weights as four
// broadcast loads), 64 FP32 accumulators per thread (16 moments x 4 rows,
// paired by rows).  Each accumulator thus sums an eighth of the ordinates;
// at a tile's end the 8 warps' partial sums meet in shared memory and are
// added in FP64, in warp order.
namespace {
constexpr int kFfRows = 128, kFfK = 32, kFfWarps = 8, kFfThreads = 32 * (kFfWarps + 1);
constexpr int kFfStageBytes = kFfRows * kFfK * 4;            // 16 KB
constexpr int kFfMaxStages = 8;
constexpr int kFfRedBytes = kFfWarps * 16 * kFfRows * 4;     // partial sums, 64 KB
struct FfSmem {
    uint64_t full[kFfMaxStages], empty[kFfMaxStages];
    int abort_flag;
};
__device__ __forceinline__ void ff_bar_sync() { asm volatile("bar.sync 1, %0;" ::"r"(32 * kFfWarps) : "memory"); }
}  // namespace

__global__ void __launch_bounds__(kFfThreads, 1)
    k_moments_tma_ffma2(const __grid_constant__ CUtensorMap psi_map, uint32_t M, uint32_t nq, uint32_t nqp,
                        const double *__restrict__ W, int nmom, double *__restrict__ mom, unsigned int *err,
                        uint32_t nstages) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    static_assert(sizeof(FfSmem) <= kSmemHeader, "barrier header");
    FfSmem &sh = *reinterpret_cast<FfSmem *>(base);
    uint8_t *stg = base + kSmemHeader;                                              // nstages x 16 KB
    float *wsm = reinterpret_cast<float *>(stg + nstages * kFfStageBytes);          // [nqp][16]
    float *red = wsm + static_cast<size_t>(nqp) * 16;                                // [warp][moment][row]
    volatile int *abort_flag = &sh.abort_flag;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t tiles = (M + kFfRows - 1) / kFfRows, nks = nqp / kFfK;

    for (uint32_t i = threadIdx.x; i < nqp * 16; i += blockDim.x) {
        const uint32_t k = i >> 4, n = i & 15u;
        wsm[i] = (k < nq && static_cast<int>(n) < nmom) ? static_cast<float>(W[static_cast<size_t>(n) * nq + k]) : 0.0f;
    }
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < nstages; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), kFfWarps);
        }
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == kFfWarps) {
        if (lane != 0) return;
        // ---- TMA producer
        uint32_t it = 0, inflight = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x)
            for (uint32_t ks = 0; ks < nks; ++ks, ++it) {
                const uint32_t s = it % nstages, ph = (it / nstages) & 1u;
                if (!(ok = mbar_wait(smem_u32(&sh.empty[s]), ph ^ 1u, abort_flag, err))) break;
                const uint32_t fb = smem_u32(&sh.full[s]);
                mbar_expect_tx(fb, kFfStageBytes);
                tma_load_2d(smem_u32(stg + s * kFfStageBytes), &psi_map, static_cast<int>(tile * kFfRows),
                            static_cast<int>(ks * kFfK), fb);
                inflight = it + 1;
            }
        if (!ok) {  // aborted: wait (bounded, own timer) for the copies already issued
            for (uint32_t j = inflight > nstages ? inflight - nstages : 0; j < inflight; ++j) {
                const uint32_t bar = smem_u32(&sh.full[j % nstages]), ph = (j / nstages) & 1u;
                const unsigned long long t0 = global_ns();
                while (!mbar_try(bar, ph) && global_ns() - t0 < kWaitNs) {
                }
            }
        }
        return;
    }
    // ---- consumers (warps 0..7).  Every consumer warp takes the same named
    // barriers in every tile, also after an abort, so none is left waiting.
    uint32_t it = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        float2 a01[16], a23[16];
#pragma unroll
        for (int n = 0; n < 16; ++n) a01[n] = a23[n] = make_float2(0.0f, 0.0f);
        for (uint32_t ks = 0; ks < nks; ++ks, ++it) {
            const uint32_t s = it % nstages, ph = (it / nstages) & 1u;
            if (ok) ok = mbar_wait_warp(smem_u32(&sh.full[s]), ph, abort_flag, err);
            if (!ok) continue;
            const uint8_t *st = stg + s * kFfStageBytes;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t k = warp + 8u * j;
                const float4 v = *reinterpret_cast<const float4 *>(st + k * (kFfRows * 4) + lane * 16);
                const float4 *wq = reinterpret_cast<const float4 *>(wsm + (ks * kFfK + k) * 16);
                float wv[16];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float4 t = wq[c];
                    wv[4 * c] = t.x;
                    wv[4 * c + 1] = t.y;
                    wv[4 * c + 2] = t.z;
                    wv[4 * c + 3] = t.w;
                }
                const float2 p01 = make_float2(v.x, v.y), p23 = make_float2(v.z, v.w);
#pragma unroll
                for (int n = 0; n < 16; ++n) {
                    const float2 ww = make_float2(wv[n], wv[n]);
                    a01[n] = __ffma2_rn(ww, p01, a01[n]);
                    a23[n] = __ffma2_rn(ww, p23, a23[n]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh.empty[s]));
        }
        if (ok) {
#pragma unroll
            for (int n = 0; n < 16; ++n)
                *reinterpret_cast<float4 *>(red + (warp * 16 + n) * kFfRows + 4 * lane) =
                    make_float4(a01[n].x, a01[n].y, a23[n].x, a23[n].y);
        }
        ff_bar_sync();
        if (!*abort_flag) {
            // 16 moments x 128 rows over the 256 consumer threads
            const uint32_t row = threadIdx.x & (kFfRows - 1), n0 = threadIdx.x >> 7;
            const uint64_t grow = static_cast<uint64_t>(tile) * kFfRows + row;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t n = n0 + 2u * i;
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < kFfWarps; ++w) sum += static_cast<double>(red[(w * 16 + n) * kFfRows + row]);
                if (grow < M && static_cast<int>(n) < nmom) mom[static_cast<uint64_t>(n) * M + grow] = sum;
            }
        }
        ff_bar_sync();
    }
}

namespace {
// shared memory of the FFMA2 form with `stages` stages for nq ordinates
size_t ff_smem_bytes(uint32_t nq, uint32_t stages) {
    const uint32_t nqp = (nq + kFfK - 1) / kFfK * kFfK;
    return 1024 + kSmemHeader + static_cast<size_t>(stages) * kFfStageBytes + static_cast<size_t>(nqp) * 64 +
           kFfRedBytes;
}
uint32_t ff_stages_for(uint32_t nq) {
    for (uint32_t st = kFfMaxStages; st >= 3; --st)
        if (ff_smem_bytes(nq, st) <= kSmemLimit) return st;
    return 0;
}
}  // namespace

bool moments_tma_ffma2_supported(uint32_t M, uint32_t nq) {
    return M > 0 && M % 4 == 0 && nq > 0 && ff_stages_for(nq) != 0;
}

cudaError_t launch_moments_tma_ffma2(const float *psi, uint32_t M, uint32_t nq, const double *W, int nmom,
                                     double *mom, unsigned int *err, int num_sms, cudaStream_t stream) {
    if (!moments_tma_ffma2_supported(M, nq) || nmom < 1 || nmom > 16) return cudaErrorInvalidValue;
    if (reinterpret_cast<uintptr_t>(psi) % 16) return cudaErrorInvalidValue;
    EncodeTiled enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    // psi as a 2-D tensor: x = row (M, contiguous), y = ordinate (nq, stride 4 M bytes)
    CUtensorMap map;
    const cuuint64_t dims[2] = {M, nq};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(M) * 4};
    const cuuint32_t box[2] = {kFfRows, kFfK};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(psi), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const uint32_t stages = ff_stages_for(nq);
    const size_t smem = ff_smem_bytes(nq, stages);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_moments_tma_ffma2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kSmemLimit));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const uint32_t tiles = (M + kFfRows - 1) / kFfRows;
    const int grid = static_cast<int>(tiles < static_cast<uint32_t>(num_sms) ? tiles : num_sms);
    const uint32_t nqp = (nq + kFfK - 1) / kFfK * kFfK;
    k_moments_tma_ffma2<<<grid, kFfThreads, smem, stream>>>(map, M, nq, nqp, W, nmom, mom, err, stages);
    return cudaGetLastError();
}

}  // namespace transfer
