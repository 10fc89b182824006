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
// area (1 + delta_vu) / 12 carry the surface term (kernels.cu:383-438).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/transfer_b200.h"

namespace transfer {

constexpr int kCoefStride = 12;  // K[9], M, M0, pad
constexpr int kBCoefStride = 4;  // E_x, E_y, E_z, pad
constexpr int kBlock = 256;

template <typename T>
struct OpData {
    uint32_t nP, slm, aslm;          // aslm: vector stride of this precision
    const uint32_t *row;             // [nP+1]
    const uint32_t *col;             // [nnz]
    const T *coef;                   // [nnz][12]
    const uint32_t *brow;            // [nP+1]
    const uint32_t *bcol;            // [nbnz]
    const T *bcoef;                  // [nbnz][4]
    const uint32_t *ang_start;       // [slm+1]  entries per output lm
    const uint16_t *ang_src;         // (3i+pos) << 8 | lms
    const T *ang_w;                  // omega_i[lms][lm]
    const T *O;                      // [3][slm][slm]: O_n[lms][lm]
    const T *ang_diag;               // [3][slm]: omega_i[lm][lm]
    const T *O_diag;                 // [3][slm]: O_n[lm][lm]
    const T *mask;                   // [nP][aslm] reflective constraint or null
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
    uint32_t counter[4];
};

struct CachedGraph {
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    bool valid = false;
};
constexpr int kCgChunk = 16;  // CG iterations per captured graph / status read

template <typename T>
struct DeviceOp {
    uint32_t *row = nullptr, *col = nullptr, *brow = nullptr, *bcol = nullptr, *ang_start = nullptr;
    uint16_t *ang_src = nullptr;
    T *coef = nullptr, *bcoef = nullptr, *ang_w = nullptr, *O = nullptr, *ang_diag = nullptr, *O_diag = nullptr;
    T *mask = nullptr;
    T *dinv = nullptr;               // Jacobi: 1 / diag(A), [nP][aslm]
    uint32_t aslm = 0;
    OpData<T> data(uint32_t nP, uint32_t slm) const {
        OpData<T> d;
        d.nP = nP;
        d.slm = slm;
        d.aslm = aslm;
        d.row = row;
        d.col = col;
        d.coef = coef;
        d.brow = brow;
        d.bcol = bcol;
        d.bcoef = bcoef;
        d.ang_start = ang_start;
        d.ang_src = ang_src;
        d.ang_w = ang_w;
        d.O = O;
        d.ang_diag = ang_diag;
        d.O_diag = O_diag;
        d.mask = mask;
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
    double *partials = nullptr;      // [4][grid max]
    unsigned int *counters = nullptr;
    double *red_out = nullptr;       // [8]
    double *host_pinned = nullptr;   // [16] pinned staging for scalars

    // solver work space (allocated on first solve)
    double *w64[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    float *w32[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
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
};

namespace transfer {

// operator launches (operator.cu)
// fin_kind: 0 plain A f; 1 also <f, A f> stored to *fin_out; 2 also the CG
// step length cgs->alpha = cgs->nrz / <f, A f>.
template <typename T>
cudaError_t launch_lhs(const tr_ctx *c, const DeviceOp<T> &op, const T *f, T *r, int fin_kind, double *fin_out,
                       CgScalars *cgs, const int32_t *done, cudaStream_t s);
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
