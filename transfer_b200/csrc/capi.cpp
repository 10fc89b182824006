// The C ABI (include/transfer_b200.h): argument checking, stream handling
// and status codes around the device code, plus the host-side problem data
// (AngularData, Config, MeshData) and the Lanczos driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/transfer_b200.h"
#include "angular.h"
#include "config.h"
#include "internal.h"
#include "meshdata.h"
#include "solver.h"

namespace transfer {
tr_status ctx_create(int device, const tr_mesh_view *m, const tr_angular_view *a, const tr_physics_view *ph,
                     tr_ctx **out, std::string &err);
void ctx_free(tr_ctx *c);
}  // namespace transfer

using namespace transfer;

static thread_local std::string g_last_error;

static tr_status set_err(tr_ctx *c, tr_status st, const std::string &msg) {
    if (c) c->last_error = msg;
    g_last_error = msg;
    return st;
}
namespace transfer {
// records a failure that belongs to no context (tr_last_error(NULL))
tr_status set_global_error(tr_status st, const std::string &msg) { return set_err(nullptr, st, msg); }
}  // namespace transfer

static cudaStream_t stream_of(const tr_ctx *c) { return c->stream ? c->stream : c->own_stream; }

static tr_status check_cuda(tr_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return TR_OK;
    return set_err(c, TR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
// launch + synchronise the context stream (API calls are synchronous)
static tr_status finish(tr_ctx *c, cudaError_t launch, const char *what) {
    if (launch != cudaSuccess) return check_cuda(c, launch, what);
    return check_cuda(c, cudaStreamSynchronize(stream_of(c)), what);
}
static tr_status activate(tr_ctx *c) {
    if (!c) return set_err(nullptr, TR_ERR_INVALID_ARG, "null context");
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, TR_ERR_CUDA, "cudaSetDevice failed");
    return TR_OK;
}

#define CHECK_CTX(c)                        \
    do {                                    \
        tr_status _s = activate(c);         \
        if (_s != TR_OK) return _s;         \
    } while (0)
#define CHECK_PTR(c, p)                                                         \
    do {                                                                        \
        if (!(p)) return set_err(c, TR_ERR_INVALID_ARG, "null pointer: " #p);   \
    } while (0)

template <typename T>
static tr_status dot_impl(tr_ctx *c, uint32_t aslm, const T *x, const T *y, double *out) {
    CHECK_CTX(c);
    CHECK_PTR(c, x);
    CHECK_PTR(c, y);
    CHECK_PTR(c, out);
    cudaStream_t st = stream_of(c);
    tr_status s = finish(c, launch_dot<T, T>(c, aslm, x, y, c->red_out + 8, st), "dot");
    if (s != TR_OK) return s;
    s = check_cuda(c, cudaMemcpy(out, c->red_out + 8, sizeof(double), cudaMemcpyDeviceToHost), "dot result");
    return s;
}
template <class Q>
static int fill_rule(const Q &q, double *x, double *y, double *z, double *w, int cap) {
    if (x && y && z && w && cap >= q.order)
        for (int i = 0; i < q.order; ++i) {
            x[i] = q.x[i];
            y[i] = q.y[i];
            z[i] = q.z[i];
            w[i] = q.w[i];
        }
    return q.order;
}
extern "C" {

int tr_abi_version(void) { return TR_ABI_VERSION; }

const char *tr_status_string(tr_status st) {
    switch (st) {
    case TR_OK: return "ok";
    case TR_ERR_INVALID_ARG: return "invalid argument";
    case TR_ERR_CUDA: return "CUDA error";
    case TR_ERR_NOT_CONVERGED: return "not converged";
    case TR_ERR_NAN: return "non-finite value";
    case TR_ERR_NO_DEVICE: return "no CUDA device";
    case TR_ERR_MESH: return "invalid mesh";
    case TR_ERR_CONFIG: return "invalid configuration";
    case TR_ERR_OUT_OF_MEMORY: return "out of memory";
    case TR_ERR_UNSUPPORTED: return "unsupported";
    case TR_ERR_IO: return "I/O error";
    }
    return "unknown status";
}

const char *tr_last_error(const tr_ctx *ctx) { return ctx ? ctx->last_error.c_str() : g_last_error.c_str(); }

tr_status tr_ctx_create(int device, const tr_mesh_view *mesh, const tr_angular_view *ang, tr_ctx **out) {
    return tr_ctx_create_ex(device, mesh, ang, nullptr, out);
}

tr_status tr_ctx_create_ex(int device, const tr_mesh_view *mesh, const tr_angular_view *ang,
                           const tr_physics_view *phys, tr_ctx **out) {
    if (!out) return set_err(nullptr, TR_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    std::string err;
    tr_status st;
    try {
        st = ctx_create(device, mesh, ang, phys, out, err);
    } catch (const std::bad_alloc &) {
        return set_err(nullptr, TR_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    if (st != TR_OK) return set_err(nullptr, st, err);
    return TR_OK;
}

tr_status tr_ctx_destroy(tr_ctx *ctx) {
    if (!ctx) return TR_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->own_stream);
    ctx_free(ctx);
    return TR_OK;
}

tr_status tr_ctx_info_get(const tr_ctx *c, tr_ctx_info *info) {
    if (!c || !info) return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    info->nP = c->nP;
    info->nT = c->nT;
    info->nF = c->nF;
    info->slm = c->slm;
    info->aslm = c->aslm;
    info->aslm_f32 = c->aslm32;
    info->n_edges = c->n_edges;
    info->n_bnd_edges = c->n_bnd_edges;
    info->device_bytes = c->device_bytes;
    info->device = c->device;
    return TR_OK;
}

tr_status tr_ctx_set_operator(tr_ctx *c, int kind) {
    CHECK_CTX(c);
    if (kind != TR_OPERATOR_SIMT && kind != TR_OPERATOR_TENSOR)
        return set_err(c, TR_ERR_INVALID_ARG, "operator kind must be TR_OPERATOR_SIMT or TR_OPERATOR_TENSOR");
    c->op64.kind = c->op32.kind = kind;
    for (auto &g : c->graphs) g.valid = false;  // captured launches name the old kernels
    return TR_OK;
}

tr_status tr_ctx_set_stream(tr_ctx *c, void *stream) {
    CHECK_CTX(c);
    c->stream = static_cast<cudaStream_t>(stream);
    return TR_OK;
}

// ------------------------------------------------------------- operator
tr_status tr_compute_lhs(tr_ctx *c, const double *f, double *Af) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    CHECK_PTR(c, Af);
    if (f == Af) return set_err(c, TR_ERR_INVALID_ARG, "f and Af must not alias");
    return finish(c, launch_lhs<double>(c, c->op64, f, Af, 0, nullptr, nullptr, nullptr, stream_of(c)),
                  "computeLhs");
}
tr_status tr_compute_lhs_diag(tr_ctx *c, const double *f, double *Af) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    CHECK_PTR(c, Af);
    if (f == Af) return set_err(c, TR_ERR_INVALID_ARG, "f and Af must not alias");
    return finish(c, launch_lhs_diag<double>(c, c->op64, f, Af, nullptr, stream_of(c)), "computeLhsDiag");
}
tr_status tr_compute_rhs(tr_ctx *c, double *b) {
    CHECK_CTX(c);
    CHECK_PTR(c, b);
    return finish(c, launch_rhs(c, b, stream_of(c)), "computeRhs");
}
tr_status tr_compute_lhs_f32(tr_ctx *c, const float *f, float *Af) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    CHECK_PTR(c, Af);
    if (f == Af) return set_err(c, TR_ERR_INVALID_ARG, "f and Af must not alias");
    return finish(c, launch_lhs<float>(c, c->op32, f, Af, 0, nullptr, nullptr, nullptr, stream_of(c)),
                  "computeLhs (f32)");
}
tr_status tr_compute_lhs_diag_f32(tr_ctx *c, const float *f, float *Af) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    CHECK_PTR(c, Af);
    if (f == Af) return set_err(c, TR_ERR_INVALID_ARG, "f and Af must not alias");
    return finish(c, launch_lhs_diag<float>(c, c->op32, f, Af, nullptr, stream_of(c)), "computeLhsDiag (f32)");
}
tr_status tr_compute_rhs_f32(tr_ctx *c, float *b) {
    CHECK_CTX(c);
    CHECK_PTR(c, b);
    return finish(c, launch_rhs_f32(c, b, stream_of(c)), "computeRhs (f32)");
}

// ------------------------------------------------------------------ BLAS
static tr_status blas(tr_ctx *c, int op, double *x, const double *y, double wx, double wy) {
    CHECK_CTX(c);
    CHECK_PTR(c, x);
    if (op != BLAS_SCALE) CHECK_PTR(c, y);
    return finish(c, launch_blas(c, op, x, y, wx, wy, stream_of(c)), "blas");
}
tr_status tr_scale(tr_ctx *c, double *x, double wx) { return blas(c, BLAS_SCALE, x, nullptr, wx, 0.0); }
tr_status tr_add_prod(tr_ctx *c, double *x, const double *y, double wy) {
    return blas(c, BLAS_ADD_PROD, x, y, 1.0, wy);
}
tr_status tr_mul_add(tr_ctx *c, double *x, double wx, const double *y) { return blas(c, BLAS_MUL_ADD, x, y, wx, 1.0); }
tr_status tr_mul_add_prod(tr_ctx *c, double *x, double wx, const double *y, double wy) {
    return blas(c, BLAS_MUL_ADD_PROD, x, y, wx, wy);
}

tr_status tr_dot(tr_ctx *c, const double *x, const double *y, double *out) { return dot_impl<double>(c, c ? c->aslm : 0, x, y, out); }
tr_status tr_norm(tr_ctx *c, const double *x, double *out) {
    tr_status s = dot_impl<double>(c, c ? c->aslm : 0, x, x, out);
    if (s == TR_OK) *out = std::sqrt(*out);
    return s;
}
tr_status tr_dot_f32(tr_ctx *c, const float *x, const float *y, double *out) {
    return dot_impl<float>(c, c ? c->aslm32 : 0, x, y, out);
}

// ---------------------------------------------------------------- solver
void tr_solve_opts_default(tr_solve_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->mode = TR_MODE_FP64;
    o->precondition = TR_PREC_NONE;
    o->max_iter = 1000;   // main.cpp:142
    o->relative = 0;
    o->tol = 1e-4;        // main.cpp:149
    o->inner_tol = 0.0;
    o->inner_max_iter = 0;
    o->max_outer = 0;
    o->engine = TR_ENGINE_PERSISTENT;
}

static tr_status check_opts(tr_ctx *c, const tr_solve_opts *o) {
    if (!o) return set_err(c, TR_ERR_INVALID_ARG, "null options");
    if (o->mode != TR_MODE_FP64 && o->mode != TR_MODE_MIXED) return set_err(c, TR_ERR_INVALID_ARG, "bad mode");
    if (o->precondition < 0 || o->precondition > 2) return set_err(c, TR_ERR_INVALID_ARG, "bad precondition");
    if (o->engine < 0 || o->engine > 3) return set_err(c, TR_ERR_INVALID_ARG, "bad engine");
    if (o->mode == TR_MODE_MIXED && o->precondition == TR_PREC_REFERENCE)
        return set_err(c, TR_ERR_UNSUPPORTED, "mixed mode supports precondition 0 or 2");
    if (!(o->tol >= 0.0) || o->max_iter < 0 || o->history_len < 0 || (o->history_len > 0 && !o->history))
        return set_err(c, TR_ERR_INVALID_ARG, "bad tolerance / limits / history");
    return TR_OK;
}

tr_status tr_solve(tr_ctx *c, const tr_solve_opts *o, const double *b, double *f, tr_solve_report *rep) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    tr_status s = check_opts(c, o);
    if (s != TR_OK) return s;
    tr_solve_report local;
    if (!rep) rep = &local;
    s = solve(c, o, b, f, rep);
    if (s != TR_OK) g_last_error = c->last_error;
    return s;
}

// true when p is page-locked host memory (cudaMallocHost or registered),
// which copies can reach by DMA without staging
static bool page_locked(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

tr_status tr_solve_host(tr_ctx *c, const tr_solve_opts *o, const double *b_host, double *f_host,
                        tr_solve_report *rep) {
    CHECK_CTX(c);
    CHECK_PTR(c, f_host);
    tr_status s = check_opts(c, o);
    if (s != TR_OK) return s;
    const size_t bytes = sizeof(double) * c->nP * c->aslm;
    // page-locked caller buffers are copied directly; pageable ones go
    // through the context's pinned staging buffers
    const bool b_locked = b_host && page_locked(b_host), f_locked = page_locked(f_host);
    if ((!b_locked || !f_locked) && c->stage_bytes < bytes) {
        if (c->stage_in) cudaFreeHost(c->stage_in);
        if (c->stage_out) cudaFreeHost(c->stage_out);
        c->stage_in = c->stage_out = nullptr;
        c->stage_bytes = 0;
        if (cudaMallocHost(reinterpret_cast<void **>(&c->stage_in), bytes) != cudaSuccess ||
            cudaMallocHost(reinterpret_cast<void **>(&c->stage_out), bytes) != cudaSuccess)
            return set_err(c, TR_ERR_OUT_OF_MEMORY, "pinned staging allocation failed");
        c->stage_bytes = bytes;
    }
    s = ensure_workspace(c, std::max(o->max_iter, 1));
    if (s != TR_OK) return s;
    cudaStream_t st = stream_of(c);
    // device buffers for b and f owned by the context
    double *db = nullptr;
    if (b_host) {
        const void *src = b_host;
        if (!b_locked) {
            std::memcpy(c->stage_in, b_host, bytes);
            src = c->stage_in;
        }
        db = c->io[0];
        s = check_cuda(c, cudaMemcpyAsync(db, src, bytes, cudaMemcpyHostToDevice, st), "H2D b");
        if (s != TR_OK) return s;
    }
    double *df = c->io[1];
    tr_solve_report local;
    if (!rep) rep = &local;
    tr_status ss = solve(c, o, db, df, rep);
    if (ss != TR_OK && ss != TR_ERR_NOT_CONVERGED) return ss;
    s = check_cuda(c, cudaMemcpyAsync(f_locked ? f_host : c->stage_out, df, bytes, cudaMemcpyDeviceToHost, st),
                   "D2H f");
    if (s == TR_OK) s = check_cuda(c, cudaStreamSynchronize(st), "D2H f");
    if (s != TR_OK) return s;
    if (!f_locked) std::memcpy(f_host, c->stage_out, bytes);
    return ss;
}

tr_status tr_bench_lhs(tr_ctx *c, int precision, const void *x, void *y, int iters, double *ms) {
    CHECK_CTX(c);
    CHECK_PTR(c, x);
    CHECK_PTR(c, y);
    CHECK_PTR(c, ms);
    if ((precision != 32 && precision != 64) || iters < 1 || x == y)
        return set_err(c, TR_ERR_INVALID_ARG, "precision must be 32 or 64, iters >= 1, x != y");
    cudaStream_t st = stream_of(c);
    cudaEvent_t e0, e1;
    tr_status s = check_cuda(c, cudaEventCreate(&e0), "event");
    if (s != TR_OK) return s;
    cudaEventCreate(&e1);
    auto launch = [&]() {
        return precision == 64 ? launch_lhs<double>(c, c->op64, static_cast<const double *>(x),
                                                    static_cast<double *>(y), 0, nullptr, nullptr, nullptr, st)
                               : launch_lhs<float>(c, c->op32, static_cast<const float *>(x), static_cast<float *>(y),
                                                   0, nullptr, nullptr, nullptr, st);
    };
    // untimed warm-up: the first launch of a kernel loads its module
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = launch();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaEventRecord(e0, st);
    for (int i = 0; i < iters && e == cudaSuccess; ++i) e = launch();
    cudaEventRecord(e1, st);
    s = check_cuda(c, e, "bench launch");
    if (s == TR_OK) s = check_cuda(c, cudaEventSynchronize(e1), "bench sync");
    float t = 0.0f;
    if (s == TR_OK) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = static_cast<double>(t) / iters;
    return s;
}

// Operator autotuner: per precision, time each kernel family as the solver
// runs it -- `iters` iterations of the persistent CG (FP64 mode for FP64,
// the mixed mode's FP32 CG for FP32) on this context's own right-hand side,
// the device time of the CG launches divided by the iterations, the second
// of two runs -- and keep the faster.  The operator alone is not the
// measure: on the 64^3 cube the FP32 tensor-core operator takes 0.82 ms
// against 1.04 ms for the SIMT one, while its persistent CG iteration,
// which also gathers the previous direction, takes 1.54 ms against 1.38 ms.
tr_status tr_ctx_autotune_operator(tr_ctx *c, int iters, double ms[4]) {
    CHECK_CTX(c);
    CHECK_PTR(c, ms);
    if (iters < 1) return set_err(c, TR_ERR_INVALID_ARG, "tr_ctx_autotune_operator: iters >= 1");
    tr_status s = ensure_workspace(c, iters);
    if (s != TR_OK) return s;
    const int kinds[2] = {TR_OPERATOR_SIMT, TR_OPERATOR_TENSOR};
    const int k64 = c->op64.kind, k32 = c->op32.kind;
    tr_solve_opts o;
    tr_solve_opts_default(&o);
    o.relative = 1;
    o.tol = 1e-300;  // runs the full `iters` iterations
    o.max_iter = iters;
    o.engine = TR_ENGINE_PERSISTENT;
    for (int p = 0; p < 2 && s == TR_OK; ++p) {  // p = 0: FP64, 1: FP32
        o.mode = p == 0 ? TR_MODE_FP64 : TR_MODE_MIXED;
        for (int k = 0; k < 2 && s == TR_OK; ++k) {
            if (p == 0) c->op64.kind = kinds[k];
            else c->op32.kind = kinds[k];
            for (auto &g : c->graphs) g.valid = false;
            for (int rep = 0; rep < 2 && s == TR_OK; ++rep) {
                tr_solve_report r;
                std::memset(&r, 0, sizeof(r));
                s = solve(c, &o, nullptr, c->io[1], &r);
                if (s == TR_ERR_NOT_CONVERGED) s = TR_OK;
                ms[2 * p + k] = r.cg_kernel_ms / std::max(1, r.iterations);
            }
        }
        if (p == 0) c->op64.kind = k64;  // the FP32 timings run the FP64 residuals in the old family
    }
    if (s != TR_OK) {  // leave the families as they were
        c->op64.kind = k64;
        c->op32.kind = k32;
        return s;
    }
    c->op64.kind = ms[1] < ms[0] ? TR_OPERATOR_TENSOR : TR_OPERATOR_SIMT;
    c->op32.kind = ms[3] < ms[2] ? TR_OPERATOR_TENSOR : TR_OPERATOR_SIMT;
    for (auto &g : c->graphs) g.valid = false;  // captured launches name the old kernels
    return TR_OK;
}

tr_status tr_ctx_get_operator(const tr_ctx *c, int kinds[2]) {
    if (!c || !kinds) return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    kinds[0] = c->op64.kind;
    kinds[1] = c->op32.kind;
    return TR_OK;
}

// ------------------------------------------------------------- self-test
tr_status tr_selftest_grid_barrier(int device, int skip_block, int rounds, unsigned int max_polls, int *timed_out) {
    if (!timed_out || rounds < 1 || max_polls < 1 || max_polls > (1u << 24))
        return set_err(nullptr, TR_ERR_INVALID_ARG, "tr_selftest_grid_barrier: bad arguments");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return set_err(nullptr, TR_ERR_NO_DEVICE, "tr_selftest_grid_barrier: no such CUDA device");
    }
    int prev = 0;
    cudaGetDevice(&prev);
    tr_status st = check_cuda(nullptr, cudaSetDevice(device), "cudaSetDevice");
    if (st != TR_OK) return st;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned int *count = nullptr;
    st = check_cuda(nullptr, cudaMalloc(reinterpret_cast<void **>(&count), 256), "cudaMalloc");
    if (st == TR_OK) st = check_cuda(nullptr, cudaMemset(count, 0, 256), "cudaMemset");
    int *err = reinterpret_cast<int *>(count + 32);
    if (st == TR_OK)
        st = check_cuda(nullptr, launch_barrier_selftest(sms, count, err, skip_block, rounds, max_polls, 0),
                        "barrier self-test launch");
    if (st == TR_OK) st = check_cuda(nullptr, cudaDeviceSynchronize(), "barrier self-test");
    int h = 0;
    if (st == TR_OK) st = check_cuda(nullptr, cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost), "copy");
    if (count) cudaFree(count);
    cudaSetDevice(prev);
    *timed_out = h;
    return st;
}

// --------------------------------------------------------------- moments
tr_status tr_compute_moments(tr_ctx *c, const double *f, double *U, double *T) {
    CHECK_CTX(c);
    CHECK_PTR(c, f);
    CHECK_PTR(c, U);
    CHECK_PTR(c, T);
    return finish(c, launch_moments(c, f, U, T, stream_of(c)), "ComputeMoments");
}
tr_status tr_compute_flux(tr_ctx *c, const double *T, double *W) {
    CHECK_CTX(c);
    CHECK_PTR(c, T);
    CHECK_PTR(c, W);
    return finish(c, launch_flux(c, T, W, stream_of(c)), "ComputeFlux");
}

// --------------------------------------------------------------- Lanczos
// trieig (Eigenvalue.cpp:5-51): Newton on the characteristic polynomial of
// the symmetric tridiagonal, from the Gershgorin upper bound.
double tr_trieig(const double *a, const double *b, int n) {
    if (!a || n < 1) return NAN;
    if (n == 1) return a[0];
    if (n == 2) {
        double ap = 0.5 * (a[0] + a[1]), am = 0.5 * (a[0] - a[1]);
        return ap + std::sqrt(am * am + b[0] * b[0]);
    }
    double lmax = a[0] + std::fabs(b[0]);
    for (int i = 1; i < n - 1; ++i) lmax = std::max(lmax, a[i] + std::fabs(b[i]) + std::fabs(b[i - 1]));
    lmax = std::max(lmax, a[n - 1] + std::fabs(b[n - 2]));
    const double th = 100.0 * std::ldexp(1.0, -53);
    double dl = 1.0;
    for (int it = 0; it < 100 && dl > th; ++it) {
        const double x = lmax;
        double Po = 1.0, P = a[0] - x, Qo = 0.0, Q = -1.0;
        for (int j = 1; j < n; ++j) {
            const double b2 = b[j - 1] * b[j - 1];
            const double Qn = -P + (a[j] - x) * Q - b2 * Qo;
            Qo = Q;
            Q = Qn;
            const double Pn = (a[j] - x) * P - b2 * Po;
            Po = P;
            P = Pn;
        }
        dl = P / Q;
        lmax -= dl;
    }
    return lmax;
}

// eigest (Eigenvalue.cpp:53-83): Lanczos with the reference's indexing of
// the off-diagonal (its b[0] = 0 is passed to trieig as the first coupling).
tr_status tr_eig_lanczos(tr_ctx *c, double *v, double *v0, double *w, int max_steps, double *lmax_out,
                         double *extra_out, int *steps_out) {
    CHECK_CTX(c);
    CHECK_PTR(c, v);
    CHECK_PTR(c, v0);
    CHECK_PTR(c, w);
    CHECK_PTR(c, lmax_out);
    const int m = max_steps > 0 ? max_steps : 30;
    std::vector<double> a(m), b(m + 1, 0.0);
    double nv = 0.0;
    tr_status s = tr_norm(c, v, &nv);
    if (s != TR_OK) return s;
    if (!(nv > 0.0)) return set_err(c, TR_ERR_INVALID_ARG, "Lanczos start vector is zero");
    if ((s = tr_scale(c, v, 1.0 / nv)) != TR_OK) return s;
    if ((s = tr_mul_add(c, v0, 0.0, v)) != TR_OK) return s;
    double lmax = 0.0, lold = 0.0, loold = 0.0;
    double *pv = v, *pv0 = v0;
    int j;
    for (j = 0; j < m; ++j) {
        if ((s = tr_compute_lhs(c, pv, w)) != TR_OK) return s;
        if ((s = tr_mul_add(c, pv0, -b[j], w)) != TR_OK) return s;
        std::swap(pv, pv0);
        if ((s = tr_dot(c, pv, pv0, &a[j])) != TR_OK) return s;
        if ((s = tr_add_prod(c, pv, pv0, -a[j])) != TR_OK) return s;
        if ((s = tr_norm(c, pv, &b[j + 1])) != TR_OK) return s;
        if ((s = tr_scale(c, pv, 1.0 / b[j + 1])) != TR_OK) return s;
        loold = lold;
        lold = lmax;
        lmax = tr_trieig(a.data(), b.data(), j + 1);
        if (std::fabs(lmax - lold) < 1e-6 * lmax) {
            ++j;
            break;
        }
    }
    const double q = (lmax - lold) / (lold - loold);
    *lmax_out = lmax;
    if (extra_out) *extra_out = lmax + (lmax - lold) / (1 - q);
    if (steps_out) *steps_out = j;
    if (pv != v) {  // the latest Lanczos vector is left in v
        s = check_cuda(c, cudaMemcpy(v, pv, sizeof(double) * c->nP * c->aslm, cudaMemcpyDeviceToDevice), "copy");
        if (s != TR_OK) return s;
    }
    return TR_OK;
}

// ------------------------------------------------------ host problem data
double tr_spherical_value(int l, int m, double x, double y, double z) {
    if (l < 0 || l > 64 || m < -l || m > l) return NAN;
    Spherical s(l);
    return s.value(l, m, x, y, z);
}
int tr_hemiquad(int mindegree, double *x, double *y, double *z, double *w, int cap) {
    if (mindegree < 0 || mindegree > 37) return -1;
    return fill_rule(HemiQuad(mindegree), x, y, z, w, cap);
}
int tr_lebedev(int mindegree, double *x, double *y, double *z, double *w, int cap) {
    try {
        return fill_rule(LebedevQuad(mindegree), x, y, z, w, cap);
    } catch (const std::exception &) {
        return -1;
    }
}

struct tr_angular {
    AngularData ad;
    explicit tr_angular(int k) : ad(k) {}
};
tr_status tr_angular_create(int maxk, tr_angular **out) {
    if (!out) return set_err(nullptr, TR_ERR_INVALID_ARG, "null output");
    if (maxk < 0 || maxk > TR_MAXK_MAX) return set_err(nullptr, TR_ERR_INVALID_ARG, "maxk must be in 0..7");
    try {
        *out = new tr_angular(maxk);
    } catch (const std::exception &e) {
        return set_err(nullptr, TR_ERR_INVALID_ARG, e.what());
    }
    return TR_OK;
}
tr_status tr_angular_view_get(const tr_angular *a, tr_angular_view *v) {
    if (!a || !v) return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    v->slm = a->ad.slm;
    v->omega = a->ad.omega.data();
    v->omega_pos = a->ad.omega_pos.data();
    v->Ox = a->ad.Ox.data();
    v->Oy = a->ad.Oy.data();
    v->Oz = a->ad.Oz.data();
    return TR_OK;
}
void tr_angular_destroy(tr_angular *a) { delete a; }

struct tr_config {
    Config cfg;
    std::string tmp;
    explicit tr_config(const char *p) : cfg(p) {}
};
tr_status tr_config_load(const char *path, tr_config **out) {
    if (!path || !out) return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    try {
        *out = new tr_config(path);
    } catch (const ConfigError &e) {
        return set_err(nullptr, TR_ERR_CONFIG, e.what());
    }
    return TR_OK;
}
void tr_config_destroy(tr_config *c) { delete c; }
int tr_config_get_int(const tr_config *c, const char *key, int *ok) {
    if (ok) *ok = 0;
    if (!c || !key) return 0;
    std::string k(key);
    int v = 0;
    bool found = true;
    if (k == "angorder") v = c->cfg.getMaxK();
    else if (k == "device") v = c->cfg.getDevice();
    else if (k == "dump") v = c->cfg.doDump();
    else if (k == "precondition") v = c->cfg.usePrec();
    else if (k == "soltype") v = c->cfg.solType();
    else if (k == "numregs") v = c->cfg.numRegions();
    else if (c->cfg.has(k)) {
        try {
            v = c->cfg.get_int(k, 0);
        } catch (const ConfigError &) {
            found = false;
        }
    } else found = false;
    if (ok) *ok = found;
    return v;
}
double tr_config_get_double(const tr_config *c, const char *key, int *ok) {
    if (ok) *ok = 0;
    if (!c || !key || !c->cfg.has(key)) return 0.0;
    try {
        double v = c->cfg.get_double(key, 0.0);
        if (ok) *ok = 1;
        return v;
    } catch (const ConfigError &) {
        return 0.0;
    }
}
const char *tr_config_get_string(const tr_config *c, const char *key) {
    if (!c || !key) return nullptr;
    std::string k(key);
    if (k == "meshfile") return c->cfg.getMeshFilename();
    if (k == "outfile") return c->cfg.getOutFilename();
    if (!c->cfg.has(k)) return nullptr;
    const_cast<tr_config *>(c)->tmp = c->cfg.get_string(k);
    return c->tmp.c_str();
}
int tr_config_num_regions(const tr_config *c) { return c ? c->cfg.numRegions() : -1; }
double tr_config_region_double(const tr_config *c, int region, const char *key, int *ok) {
    if (ok) *ok = 0;
    if (!c || !key || region < 0 || region > c->cfg.numRegions()) return 0.0;
    std::string k(key);
    try {
        if (k == "kappa") {
            if (ok) *ok = 1;
            return c->cfg.getKappa(region);
        }
        if (k == "Ip") {
            if (ok) *ok = 1;
            return c->cfg.getIp(region);
        }
        if (!c->cfg.region_has(region, k)) return 0.0;
        double v = c->cfg.region_double(region, k, 0.0);
        if (ok) *ok = 1;
        return v;
    } catch (const std::exception &) {
        return 0.0;
    }
}

struct tr_meshdata {
    MeshData md;
};
static RegionParams region_params(const tr_region_params *rp) {
    RegionParams r;
    r.kappa.assign(rp->kappa, rp->kappa + rp->nreg + 1);
    r.Ip.assign(rp->Ip, rp->Ip + rp->nreg + 1);
    if (rp->albedo) r.albedo.assign(rp->albedo, rp->albedo + rp->nreg + 1);
    return r;
}
tr_status tr_meshdata_from_tets(tr_idx nP, const double *xyz, tr_idx nT, const tr_idx *tets,
                                const int32_t *region, const tr_region_params *rp, tr_meshdata **out) {
    if (!xyz || !tets || !region || !rp || !rp->kappa || !rp->Ip || !out || rp->nreg < 1)
        return set_err(nullptr, TR_ERR_INVALID_ARG, "null or empty argument");
    try {
        tr_meshdata *m = new tr_meshdata();
        m->md = MeshData::from_tets(nP, xyz, nT, tets, region, region_params(rp));
        *out = m;
    } catch (const std::exception &e) {
        return set_err(nullptr, TR_ERR_MESH, e.what());
    }
    return TR_OK;
}
tr_status tr_meshdata_kuhn(const tr_kuhn_params *kp, const tr_region_params *rp, tr_meshdata **out) {
    if (!kp || !rp || !rp->kappa || !rp->Ip || !out || rp->nreg < 1)
        return set_err(nullptr, TR_ERR_INVALID_ARG, "null or empty argument");
    KuhnParams k;
    for (int i = 0; i < 3; ++i) k.n[i] = kp->n[i];
    for (int i = 0; i < 6; ++i) k.box[i] = kp->box[i];
    k.jitter = kp->jitter;
    k.seed = kp->seed;
    k.region_kind = kp->region_kind;
    for (int i = 0; i < 4; ++i) k.region_arg[i] = kp->region_arg[i];
    k.ball = kp->ball != 0;
    for (int i = 0; i < 3; ++i) k.ball_center[i] = kp->ball_center[i];
    k.ball_radius = kp->ball_radius;
    try {
        tr_meshdata *m = new tr_meshdata();
        m->md = MeshData::kuhn(k, region_params(rp));
        *out = m;
    } catch (const std::exception &e) {
        return set_err(nullptr, TR_ERR_MESH, e.what());
    }
    return TR_OK;
}
tr_status tr_meshdata_view_get(const tr_meshdata *md, tr_mesh_view *view) {
    if (!md || !view) return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    *view = md->md.view();
    return TR_OK;
}
const double *tr_meshdata_coords(const tr_meshdata *md) { return md ? md->md.coords.data() : nullptr; }
const int32_t *tr_meshdata_regions(const tr_meshdata *md) { return md ? md->md.region.data() : nullptr; }
const double *tr_meshdata_kappa_abs_volume(const tr_meshdata *md) {
    return (md && !md->md.kappa_abs_volume.empty()) ? md->md.kappa_abs_volume.data() : nullptr;
}
const int32_t *tr_meshdata_face_side(const tr_meshdata *md) {
    return (md && !md->md.face_side.empty()) ? md->md.face_side.data() : nullptr;
}
void tr_meshdata_destroy(tr_meshdata *md) { delete md; }

tr_status tr_meshdata_read_vol(const char *path, const tr_region_params *rp, tr_meshdata **out) {
    if (!path || !rp || !rp->kappa || !rp->Ip || !out || rp->nreg < 1)
        return set_err(nullptr, TR_ERR_INVALID_ARG, "null or empty argument");
    try {
        tr_meshdata *m = new tr_meshdata();
        try {
            m->md = MeshData::read_vol(path, region_params(rp));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    } catch (const std::exception &e) {
        return set_err(nullptr, TR_ERR_IO, e.what());
    }
    return TR_OK;
}
const int32_t *tr_meshdata_face_bcnr(const tr_meshdata *md) {
    return (md && !md->md.face_bcnr.empty()) ? md->md.face_bcnr.data() : nullptr;
}
tr_status tr_vtk_write(const char *path, const tr_meshdata *md, int real_bytes, int nfields,
                       const tr_vtk_field *fields) {
    if (!path || !md || nfields < 0 || (nfields > 0 && !fields))
        return set_err(nullptr, TR_ERR_INVALID_ARG, "null argument");
    try {
        write_vtk(path, md->md, real_bytes, nfields, fields);
    } catch (const std::exception &e) {
        return set_err(nullptr, TR_ERR_IO, e.what());
    }
    return TR_OK;
}

}  // extern "C"
