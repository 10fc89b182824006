// Internal device-side layout of a tr_ctx and the launch helpers shared by
// the .cu translation units.  Not part of the C ABI.
//
// The operator is stored ASSEMBLED over vertex pairs instead of per
// (vertex, tet) as the reference's volumePart gathers it (kernels.cu:236-261):
// for every vertex v and every vertex u sharing a tet with v
//   K_vu[i][j] = sum_{t ∋ v,u} s_t[loc v][i] s_t[loc u][j] / (9 kappa_volume_t)
//   M_vu       = sum_{t ∋ v,u} kappa_volume_t (1 + delta_vu) / 20
//   M0_vu      = the same with the l = 0 (absorption) coefficient
// so that
//   (A f)[v][lm] = sum_u M_vu(lm) f[u][lm]
//                + sum_i sum_lms omega_i[lms][lm] S_v[3i + pos_i(lms,lm)][lms],
//   S_v[3i+j][lms] = sum_u K_vu[i][j] f[u][lms],
// which is the reference's sum re-associated (same operator, rounding-level
// differences).  Boundary couplings E_vu[n] = sum_{faces ∋ v,u, axis n}
// area (1 + delta_vu) / 12 carry the surface term (kernels.cu:383-438); they
// sit in the same edge record (every face edge is a tet edge).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/transfer_b200.h"

namespace transfer {

// Per-edge coefficient record (16 values; 128 bytes in FP64, 64 in FP32):
//   0-5   the symmetric stiffness sums K_xx, K_yy, K_zz, K_xy+K_yx,
//         K_xz+K_zx, K_yz+K_zy  (the angular weights satisfy
//         omega_ij = omega_ji, so only S_ij + S_ji enters the operator)
//   6, 7  M, M0 (mass; M0 for l = 0)
//   8-10  E_x, E_y, E_z (boundary)      11-15 zero
// In device memory the record is kept in two halves of kCoefHalf values,
// coef[nnz][8] (rows 0-7, read for every edge) and coef_bnd[nnz][8] (rows
// 8-15, read only at vertices with boundary faces), so that interior
// vertices move half the record bytes.  Shared-memory staging keeps the
// whole 16-value record.
constexpr int kCoefStride = 16;
constexpr int kCoefHalf = 8;
constexpr int kSymRows = 6, kRowM = 6, kRowM0 = 7, kRowE = 8;
constexpr int kBlock = 256;

// The angular coupling out[lm] = sum_k w_k S[o_k], over the entries k of
// harmonic lm (o = q * SA + lms addresses S_sym[q][lms] in the kernel's S or
// C table), runs in rounds of R steps (R a multiple of 4).  Each harmonic's
// list is cut into chunks of at most R entries; chunk s (chunks numbered
// harmonic after harmonic, in an order of the harmonics the host picks) is
// done by lane s mod L in round s / L, which stores its sum to part[s];
// harmonic lm then adds its chunks span[lm] & 0xFFFF .. (span[lm] >> 16) - 1
// in order.  R and the harmonic order are chosen per table (the fewest
// shared-memory wavefronts, bank conflicts included), so long and short
// lists share the lanes evenly where a list per lane would pad every lane
// to the longest list (about 1.5x the mean).  Table [rounds * R][L], lane-major; unused entries have w = 0,
// o = 0.  Storage, one block: FP32 (w, o) pairs, 8 bytes per entry (one
// vector load per step); FP64 the weights [n] then the offsets [n] (n =
// rounds * R * L), 8 + 4 bytes per entry.  The SIMT kernels use L = G lanes
// and the S table; the tensor-core kernels L = 32 and the C table.
template <typename T>
struct Runs {
    uint32_t rounds = 0, R = 0, L = 0;
    const unsigned char *tab = nullptr;  // the entries
    const uint32_t *span = nullptr;      // [slm] chunks of each harmonic: first | end << 16
};
template <typename T>
__host__ __device__ inline size_t runs_entry_bytes(const Runs<T> &r) {
    return static_cast<size_t>(r.rounds) * r.R * r.L * (sizeof(T) + 4);
}
// chunk sums a SIMT group of G lanes with H harmonics per lane has room for
__host__ __device__ inline constexpr uint32_t runs_part_elems(int G, int H) {
    return static_cast<uint32_t>(2 * G * H + G);
}
// shared-memory bytes of one staged Runs table for slm harmonics
template <typename T>
__host__ __device__ inline size_t runs_smem_bytes(const Runs<T> &r, uint32_t slm) {
    return ((runs_entry_bytes(r) + 15) & ~size_t(15)) + ((4 * size_t(slm) + 15) & ~size_t(15));
}
// lanes per vertex (G) and harmonics per lane (H) for a vector stride
inline constexpr int group_width(uint32_t aslm) { return aslm <= 8 ? 8 : aslm <= 16 ? 16 : 32; }
inline constexpr int harm_per_lane(uint32_t aslm) {
    return aslm <= 32 ? 1 : aslm <= 64 ? 2 : aslm <= 96 ? 3 : 4;
}
inline constexpr uint32_t s_row_stride(uint32_t aslm) {
    return static_cast<uint32_t>(group_width(aslm) * harm_per_lane(aslm) + 1);
}

template <typename T>
struct OpData {
    uint32_t nP, slm, aslm;          // aslm: vector stride of this precision
    const uint32_t *row;             // [nP+1]
    const uint32_t *col;             // [nnz]
    const T *coef;                   // [nnz][8]: record rows 0-7
    const T *coef_bnd;               // [nnz][8]: record rows 8-15 (boundary couplings)
    uint32_t cls;                    // lane stride of O
    Runs<T> rs, rt;                  // contraction runs: SIMT S table, tensor-core C table
    const T *O;                      // [3][slm][cls]: O_n[lms][lm], rows padded to cls
    const T *ang_diag;               // [3][slm]: omega_i[lm][lm]
    const T *O_diag;                 // [3][slm]: O_n[lm][lm]
    const T *mask;                   // [nP][aslm] reflective constraint or null
    const uint8_t *bmask;            // [nP] boundary axes present (bits 0..2)
};

// Arguments of one operator launch.  fin_kind: 0 plain A x; 1 also <x, A x>
// stored to *fin_out; 2 also the CG step alpha = cgs->nrz / <x, A x>;
// 3 as 2 with the direction update fused into the gather: the operator is
// applied to p_new = x + cgs->beta * pold, which is also written to pnew.
template <typename T>
struct LhsArgs {
    const T *x = nullptr;
    const T *pold = nullptr;
    T *pnew = nullptr;
    T *y = nullptr;
    int fin_kind = 0;
    double *fin_out = nullptr;
    struct CgScalars *cgs = nullptr;
    const int32_t *done = nullptr;
};

// Scalars of a device-resident CG, one per concurrent solve.
struct CgScalars {
    double nrz;      // (r, z)
    double alpha;
    double beta;
    double rr;       // ||r||^2 of the last update
    double tol;      // stop when sqrt(rr) < tol
    double scale;    // mixed mode: scale of the current correction
    int32_t k;       // completed iterations
    int32_t done;    // 0 running, 1 converged, 2 iteration cap, 3 non-finite
    int32_t maxit;
    int32_t prec;    // 0 none, 2 jacobi
    int32_t phase;   // single-reduction CG: steps done (step 0 forms w_0 = A u_0)
    uint32_t counter[4];
};

// Arguments of the persistent CG kernel (one cooperative launch runs up to
// `iters` iterations).  p0 / p1 alternate as p_old / p_new by the parity of
// the iteration count; partials holds [3][grid] per-block sums; bar[0] is
// the grid barrier's monotone arrival count (zeroed before every launch),
// err its timeout flag.
template <typename T>
struct PcgArgs {
    T *x, *r, *z, *p0, *p1, *Ap;
    const T *dinv;
    struct CgScalars *s;
    double *hist;
    int hist_cap;
    double *partials;
    unsigned int *bar;
    int *err;
    uint32_t nvec;
    int iters;
};
constexpr int kMaxGrid = 4096;  // partial-sum slots per reduction

// Arguments of the persistent single-reduction CG kernel (operator.cu
// k_sr_persistent): r, w, s double buffered by step parity; partials holds
// [2][3][grid] per-block sums (parity-buffered: one barrier per step).
template <typename T>
struct SrArgs {
    T *x, *p;
    T *R[2], *W[2], *S[2];
    const T *dinv;
    struct CgScalars *s;
    double *hist;
    int hist_cap;
    double *partials;
    unsigned int *bar;
    int *err;
    int iters;
};

struct CachedGraph {
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    bool valid = false;
};
constexpr int kCgChunk = 16;       // CG iterations per captured graph / status read (even)
// CG iterations per persistent-kernel launch: the host reads the status
// (iterations, stop flag) between launches, one launch, copy and stream
// synchronisation each
#ifndef TR_PERSIST_CHUNK
#define TR_PERSIST_CHUNK 1024
#endif
constexpr int kPersistChunk = TR_PERSIST_CHUNK;

template <typename T>
struct DeviceOp {
    uint32_t *row = nullptr, *col = nullptr;
    uint32_t cls = 0;
    Runs<T> rs, rt;                  // contraction runs (SIMT, tensor core)
    T *coef = nullptr, *O = nullptr, *ang_diag = nullptr, *O_diag = nullptr;  // coef: [2][nnz][8]
    size_t nnz = 0;
    T *mask = nullptr;
    T *dinv = nullptr;               // Jacobi: 1 / diag(A), [nP][aslm]
    uint8_t *bmask = nullptr;
    uint32_t aslm = 0;
    int kind = TR_OPERATOR_TENSOR;   // TR_OPERATOR_*
    OpData<T> data(uint32_t nP, uint32_t slm) const {
        OpData<T> d;
        d.nP = nP;
        d.slm = slm;
        d.aslm = aslm;
        d.row = row;
        d.col = col;
        d.coef = coef;
        d.coef_bnd = coef ? coef + nnz * kCoefHalf : nullptr;
        d.cls = cls;
        d.rs = rs;
        d.rt = rt;
        d.O = O;
        d.ang_diag = ang_diag;
        d.O_diag = O_diag;
        d.mask = mask;
        d.bmask = bmask;
        return d;
    }
};

struct RhsData {
    uint32_t nP, slm, aslm;
    const uint32_t *vt_start;        // [nP+1] vertex -> tets (CSR order of the input)
    const uint32_t *vt_tet;
    const double *tet_q;             // kappa_volume * I_p
    const double *inflow;            // [nP][3] sum I A/3 per axis, or null
    const double *O;                 // [3][slm][slm] FP64
};

struct FluxData {
    uint32_t nP, nT, slm, aslm;
    const uint4 *tet_p;
    const double *tet_s;             // [nT][12]
    const double *tet_kv;
    const double *mom_w;             // [3][slm]: omega_i[lm][0] (unpadded host value)
    const uint32_t *mom_pos;         // [3][slm]
};

}  // namespace transfer

struct tr_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string last_error;

    uint32_t nP = 0, nT = 0, nF = 0, slm = 0, aslm = 0, aslm32 = 0;
    uint64_t n_edges = 0, n_bnd_edges = 0, device_bytes = 0;
    int grid_vec = 0;                // grid of vector kernels (multiple of SMs)
    int grid_op = 0;                 // grid of operator kernels
    int num_sms = 0;

    transfer::DeviceOp<double> op64;
    transfer::DeviceOp<float> op32;

    // rhs / moments / flux
    uint32_t *vt_start = nullptr, *vt_tet = nullptr;
    double *tet_q = nullptr, *inflow = nullptr, *O64 = nullptr;
    uint4 *tet_p = nullptr;
    double *tet_s = nullptr, *tet_kv = nullptr;
    double *mom_w = nullptr;
    uint32_t *mom_pos = nullptr;

    // reductions: per-block partials + last-block counters + results
    double *partials = nullptr;      // [4][kMaxGrid]
    unsigned int *bar = nullptr;     // persistent-kernel grid barrier [2]
    int *bar_err = nullptr;          // barrier timeout flag
    unsigned int *counters = nullptr;
    double *red_out = nullptr;       // [8]
    double *host_pinned = nullptr;   // [16] pinned staging for scalars

    // solver work space (allocated on first solve)
    double *w64[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // x r p Ap z b p'
    float *w32[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // d r p Ap z p' s0 s1
    int grid_vec64 = 0, grid_vec32 = 0;  // vectorised vector kernels
    double *inner[3] = {nullptr, nullptr, nullptr};  // invprec inner CG vectors
    double *io[2] = {nullptr, nullptr};              // tr_solve_host device b / f
    transfer::CgScalars *cg = nullptr;   // [4]: fp64 CG, invprec, outer, inner
    transfer::CachedGraph graphs[4];     // fp64, fp64+jacobi, fp32, fp32+jacobi
    double *dhist = nullptr;             // [hist_cap]
    int hist_cap = 0;
    double *stage_in = nullptr, *stage_out = nullptr;  // pinned host staging
    size_t stage_bytes = 0;

    std::vector<void *> allocations;
    int64_t launches = 0;            // kernels launched (for solve reports)
    int last_cg_engine = 0;          // the engine the last CG run used (TR_ENGINE_*)
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // solve [0,1], CG launches [2,3]
    double cg_ms = 0.0;              // device time of the CG-iteration launches of a solve
    int64_t cg_launches = 0;         // those launches (persistent kernels or graph replays)
};

namespace transfer {

// operator launches (operator.cu)
// see LhsArgs for fin_kind
template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, LhsArgs<T> a, cudaStream_t s);
template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, int fin_kind, double *fin_out,
                       CgScalars *cgs, const int32_t *done, cudaStream_t s);
template <typename T>
cudaError_t launch_cg_persistent(const tr_ctx *c, const DeviceOp<T> &op, const PcgArgs<T> &a, cudaStream_t s,
                                 int *grid_out);
template <typename T>
cudaError_t launch_sr_persistent(const tr_ctx *c, const DeviceOp<T> &op, const SrArgs<T> &a, cudaStream_t s);
// bounded grid barrier self-test (operator.cu)
cudaError_t launch_barrier_selftest(int blocks, unsigned int *count, int *err, int skip, int rounds,
                                    unsigned int max_polls, cudaStream_t s);
cudaError_t operator_init_attributes();
template <typename T>
cudaError_t launch_lhs_diag(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, const int32_t *done,
                            cudaStream_t s);
cudaError_t launch_rhs(const tr_ctx *c, double *b, cudaStream_t s);
cudaError_t launch_rhs_f32(const tr_ctx *c, float *b, cudaStream_t s);

// vector kernels (vector.cu)
enum BlasOp { BLAS_SCALE = 0, BLAS_ADD_PROD = 1, BLAS_MUL_ADD = 2, BLAS_MUL_ADD_PROD = 3 };
cudaError_t launch_blas(const tr_ctx *c, int op, double *x, const double *y, double wx, double wy, cudaStream_t s);
template <typename TX, typename TY>
cudaError_t launch_dot(const tr_ctx *c, uint32_t aslm, const TX *x, const TY *y, double *out, cudaStream_t s);
cudaError_t launch_moments(const tr_ctx *c, const double *f, double *U, double *T, cudaStream_t s);
cudaError_t launch_flux(const tr_ctx *c, const double *T, double *W, cudaStream_t s);

}  // namespace transfer
