// Solvers: the reference's CG (main.cpp:125-160) with its optional inner-CG
// preconditioner invprec (main.cpp:223-248), a Jacobi variant, and the
// FP32-in-FP64 defect-correction solve.
//
// All CG scalars live in device memory (CgScalars): each iteration is two
// launches -- the new direction p = z + beta p_old formed inside the
// operator's gather, A p with <p, A p> and alpha fused; then the x/r update
// with ||r||, the stop test and beta fused -- neither returns to the host.
// The two p buffers swap roles every iteration.  Iterations run in chunks; a chunk is captured once
// as a CUDA graph and replayed, and the host reads one 8-byte status word
// per chunk.  Kernels of a chunk that starts after convergence return
// immediately, so the result is the same as with a per-iteration test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"
#include "solver.h"

namespace transfer {

template <typename T>
cudaError_t launch_cg_start(const tr_ctx *c, uint32_t aslm, const T *b, T *f, T *r, T *z, T *p, const T *dinv,
                            CgScalars *s, int zero_p, cudaStream_t st);
template <typename T>
cudaError_t launch_cg_update(const tr_ctx *c, uint32_t aslm, T *f, T *r, const T *p, const T *Ap, T *z,
                             const T *dinv, CgScalars *s, double *hist, int hist_cap, int defer_beta,
                             cudaStream_t st);
template <typename T>
cudaError_t launch_cg_direction(const tr_ctx *c, uint32_t aslm, T *p, const T *z, const CgScalars *s,
                                cudaStream_t st);
cudaError_t launch_residual(const tr_ctx *c, const double *b, const double *Ax, double *r, CgScalars *s,
                            cudaStream_t st);
cudaError_t launch_to_f32(const tr_ctx *c, const double *r64, float *r32, const CgScalars *s, cudaStream_t st);
cudaError_t launch_correct(const tr_ctx *c, double *x, const float *d32, const CgScalars *s, cudaStream_t st);
cudaError_t launch_cg_reliable(const tr_ctx *c, float *f, const float *r, float *z, const float *dinv, CgScalars *s,
                               double ratio, cudaStream_t st);

// alpha = nrz / *dot (invprec's inner CG, whose operator launch has no fused dot)
__global__ void k_set_alpha(CgScalars *s, const double *dot) {
    if (s->done) return;
    s->alpha = s->nrz / *dot;
}
// nrz = (r, z) at the start of a preconditioned CG (main.cpp:141)
__global__ void k_set_nrz(CgScalars *s, const double *dot) { s->nrz = *dot; }
// beta = (z, r) / nrz ; nrz = (z, r)   (main.cpp:155-157)
__global__ void k_set_beta(CgScalars *s, const double *dot) {
    if (s->done) return;
    s->beta = *dot / s->nrz;
    s->nrz = *dot;
}

#define TRY(...)                                                    \
    do {                                                            \
        cudaError_t _e = (__VA_ARGS__);                             \
        if (_e != cudaSuccess) return fail(c, _e, #__VA_ARGS__);    \
    } while (0)

// a kernel launch of this library: checked and counted
#define LAUNCH(...)          \
    do {                     \
        TRY(__VA_ARGS__);    \
        ++c->launches;       \
    } while (0)

static tr_status fail(tr_ctx *c, cudaError_t e, const char *what) {
    c->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return TR_ERR_CUDA;
}

static cudaStream_t stream_of(const tr_ctx *c) { return c->stream ? c->stream : c->own_stream; }

// smallest relative residual asked of one FP32 inner solve
constexpr double kMixedInnerFloor = 2e-6;
#ifndef TR_RELIABLE_DELTA
#define TR_RELIABLE_DELTA 1e-3
#endif
constexpr double kReliableDelta = TR_RELIABLE_DELTA;

tr_status ensure_workspace(tr_ctx *c, int hist_cap) {
    const size_t n64 = static_cast<size_t>(c->nP) * c->aslm, n32 = static_cast<size_t>(c->nP) * c->aslm32;
    auto alloc = [&](void **p, size_t bytes) -> bool {
        if (*p) return true;
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        cudaMemset(*p, 0, bytes);
        c->allocations.push_back(*p);
        c->device_bytes += bytes;
        return true;
    };
    for (int i = 0; i < 7; ++i)
        if (!alloc(reinterpret_cast<void **>(&c->w64[i]), n64 * sizeof(double))) {
            c->last_error = "out of device memory (solver work vectors)";
            return TR_ERR_OUT_OF_MEMORY;
        }
    for (int i = 0; i < 8; ++i)
        if (!alloc(reinterpret_cast<void **>(&c->w32[i]), n32 * sizeof(float))) {
            c->last_error = "out of device memory (solver work vectors)";
            return TR_ERR_OUT_OF_MEMORY;
        }
    for (int i = 0; i < 2; ++i)
        if (!alloc(reinterpret_cast<void **>(&c->io[i]), n64 * sizeof(double))) {
            c->last_error = "out of device memory (solver work vectors)";
            return TR_ERR_OUT_OF_MEMORY;
        }
    for (int i = 0; i < 3; ++i)
        if (!alloc(reinterpret_cast<void **>(&c->inner[i]), n64 * sizeof(double))) {
            c->last_error = "out of device memory (solver work vectors)";
            return TR_ERR_OUT_OF_MEMORY;
        }
    if (!alloc(reinterpret_cast<void **>(&c->cg), 4 * sizeof(CgScalars))) {
        c->last_error = "out of device memory";
        return TR_ERR_OUT_OF_MEMORY;
    }
    if (hist_cap > c->hist_cap) {
        if (c->dhist) {
            cudaFree(c->dhist);
            c->allocations.erase(std::find(c->allocations.begin(), c->allocations.end(), (void *)c->dhist));
            c->dhist = nullptr;
        }
        int cap = std::max(hist_cap, 1024);
        if (!alloc(reinterpret_cast<void **>(&c->dhist), cap * sizeof(double))) {
            c->last_error = "out of device memory";
            return TR_ERR_OUT_OF_MEMORY;
        }
        c->hist_cap = cap;
        for (auto &g : c->graphs) g.valid = false;  // history pointer changed
    }
    return TR_OK;
}

static tr_status init_scalars(tr_ctx *c, CgScalars *s, double tol, int maxit, cudaStream_t st) {
    CgScalars h;
    std::memset(&h, 0, sizeof(h));
    h.tol = tol;
    h.maxit = maxit;
    TRY(cudaMemcpyAsync(s, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    return TR_OK;
}

// read k and done of a scalar block (one small D2H)
static tr_status read_status(tr_ctx *c, const CgScalars *s, int *k, int *done, cudaStream_t st) {
    int32_t *h = reinterpret_cast<int32_t *>(c->host_pinned);
    TRY(cudaMemcpyAsync(h, &s->k, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    *k = h[0];
    *done = h[1];
    return TR_OK;
}
static tr_status read_double(tr_ctx *c, const double *d, double *out, cudaStream_t st) {
    TRY(cudaMemcpyAsync(c->host_pinned + 2, d, sizeof(double), cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    *out = c->host_pinned[2];
    return TR_OK;
}

// adds the device time between ev[2] and ev[3] (both complete) to cg_ms
static void add_cg_time(tr_ctx *c) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]) == cudaSuccess) c->cg_ms += ms;
    ++c->cg_launches;
}

// One CG iteration of precision T (two launches, all on device state).
// parity selects which p buffer holds p_old.
template <typename T>
static cudaError_t cg_iteration(tr_ctx *c, const DeviceOp<T> &op, uint32_t aslm, T *x, T *r, T *const pbuf[2], T *Ap,
                                T *z, const T *dinv, CgScalars *s, double *hist, int hcap, int parity,
                                cudaStream_t st) {
    LhsArgs<T> a;
    a.x = dinv ? z : r;
    a.pold = pbuf[parity];
    a.pnew = pbuf[parity ^ 1];
    a.y = Ap;
    a.fin_kind = 3;
    a.cgs = s;
    a.done = &s->done;
    cudaError_t e = launch_lhs<T>(c, op, a, st);
    if (e == cudaSuccess) e = launch_cg_update<T>(c, aslm, x, r, a.pnew, Ap, z, dinv, s, hist, hcap, 0, st);
    c->launches += 2;
    return e;
}

// Runs CG iterations from a started state until done (converged, cap or
// non-finite).  TR_ENGINE_PERSISTENT: cooperative launches of the persistent
// kernel, kPersistChunk iterations each; TR_ENGINE_GRAPH: graph slot `slot`
// caches a captured chunk of kCgChunk two-launch iterations; TR_ENGINE_LAUNCH:
// the same launches issued directly.  All three give bitwise equal results.
template <typename T>
static tr_status run_cg(tr_ctx *c, int slot, const DeviceOp<T> &op, uint32_t aslm, T *x, T *r, T *const pbuf[2],
                        T *Ap, T *z, const T *dinv, CgScalars *s, double *hist, int hcap, int engine, int *iters,
                        int *done_out) {
    if (engine == TR_ENGINE_PERSISTENT) {
        cudaStream_t st = stream_of(c);
        PcgArgs<T> a;
        a.x = x;
        a.r = r;
        a.z = z;
        a.p0 = pbuf[0];
        a.p1 = pbuf[1];
        a.Ap = Ap;
        a.dinv = dinv;
        a.s = s;
        a.hist = hist;
        a.hist_cap = hcap;
        a.partials = c->partials;
        a.bar = c->bar;
        a.err = c->bar_err;
        a.nvec = static_cast<uint32_t>(static_cast<size_t>(c->nP) * aslm / (16 / sizeof(T)));
        a.iters = kPersistChunk;
        int k = 0, done = 0;
        for (int guard = 0; guard < (1 << 24); ++guard) {
            int grid = 0;
            TRY(cudaMemsetAsync(c->bar, 0, sizeof(unsigned int), st));  // grid_barrier's arrival count
            TRY(cudaEventRecord(c->ev[2], st));
            cudaError_t e = launch_cg_persistent<T>(c, op, a, st, &grid);
            if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported) {
                cudaGetLastError();  // this device cannot co-schedule the grid: replay graphs instead
                return run_cg<T>(c, slot, op, aslm, x, r, pbuf, Ap, z, dinv, s, hist, hcap, TR_ENGINE_GRAPH,
                                 iters, done_out);
            }
            TRY(e);
            TRY(cudaEventRecord(c->ev[3], st));
            ++c->launches;
            int32_t *h = reinterpret_cast<int32_t *>(c->host_pinned);
            TRY(cudaMemcpyAsync(h, &s->k, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            TRY(cudaMemcpyAsync(h + 2, c->bar_err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            TRY(cudaStreamSynchronize(st));
            k = h[0];
            done = h[1];
            add_cg_time(c);
            if (h[2]) {
                c->last_error = "persistent CG: grid barrier timed out";
                cudaMemsetAsync(c->bar_err, 0, sizeof(int), st);
                cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned int), st);
                return TR_ERR_CUDA;
            }
            if (done) break;
        }
        *iters = k;
        *done_out = done;
        c->last_cg_engine = TR_ENGINE_PERSISTENT;
        return TR_OK;
    }
    c->last_cg_engine = engine;
    const int use_graph = (engine == TR_ENGINE_GRAPH);
    static_assert(kCgChunk % 2 == 0, "the p buffers must be back in place after a chunk");
    cudaStream_t st = stream_of(c);
    const int chunk = kCgChunk;
    CachedGraph &g = c->graphs[slot];
    if (use_graph && (!g.valid || g.stream != st)) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        const int64_t counted = c->launches;  // capturing launches nothing
        TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = cudaSuccess;
        for (int i = 0; i < chunk && ce == cudaSuccess; ++i)
            ce = cg_iteration<T>(c, op, aslm, x, r, pbuf, Ap, z, dinv, s, hist, hcap, i & 1, st);
        cudaError_t ee = cudaStreamEndCapture(st, &graph);
        c->launches = counted;
        if (ce != cudaSuccess) return fail(c, ce, "capture of CG chunk");
        if (ee != cudaSuccess) return fail(c, ee, "cudaStreamEndCapture");
        cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return fail(c, ie, "cudaGraphInstantiate");
        g.valid = true;
        g.stream = st;
    }
    int k = 0, done = 0;
    for (int guard = 0; guard < (1 << 24); ++guard) {
        TRY(cudaEventRecord(c->ev[2], st));
        if (use_graph) {
            TRY(cudaGraphLaunch(g.exec, st));
            c->launches += 2 * chunk;
        } else {
            for (int i = 0; i < chunk; ++i)
                TRY(cg_iteration<T>(c, op, aslm, x, r, pbuf, Ap, z, dinv, s, hist, hcap, i & 1, st));
        }
        TRY(cudaEventRecord(c->ev[3], st));
        tr_status rs = read_status(c, s, &k, &done, st);
        if (rs != TR_OK) return rs;
        add_cg_time(c);
        if (done) break;
    }
    *iters = k;
    *done_out = done;
    return TR_OK;
}

// the engine of the two-reduction CG loops (TR_ENGINE_PERSISTENT_SR only
// changes the FP32 inner solves of the mixed mode)
static int base_engine(int engine) { return engine == TR_ENGINE_PERSISTENT_SR ? TR_ENGINE_PERSISTENT : engine; }

// Single-reduction CG steps (k_sr_persistent) from a started state until
// done; the same launch / status-read loop as the persistent engine.
template <typename T>
static tr_status run_sr(tr_ctx *c, const DeviceOp<T> &op, SrArgs<T> a, int *iters, int *done_out) {
    cudaStream_t st = stream_of(c);
    a.partials = c->partials;
    a.bar = c->bar;
    a.err = c->bar_err;
    a.iters = kPersistChunk;
    int k = 0, done = 0;
    for (int guard = 0; guard < (1 << 24); ++guard) {
        TRY(cudaMemsetAsync(c->bar, 0, sizeof(unsigned int), st));  // grid_barrier's arrival count
        TRY(cudaEventRecord(c->ev[2], st));
        TRY(launch_sr_persistent<T>(c, op, a, st));
        TRY(cudaEventRecord(c->ev[3], st));
        ++c->launches;
        int32_t *h = reinterpret_cast<int32_t *>(c->host_pinned);
        TRY(cudaMemcpyAsync(h, &a.s->k, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        TRY(cudaMemcpyAsync(h + 2, c->bar_err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        k = h[0];
        done = h[1];
        add_cg_time(c);
        if (h[2]) {
            c->last_error = "single-reduction CG: grid barrier timed out";
            cudaMemsetAsync(c->bar_err, 0, sizeof(int), st);
            cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned int), st);
            return TR_ERR_CUDA;
        }
        if (done) break;
    }
    *iters = k;
    *done_out = done;
    return TR_OK;
}

// invprec (main.cpp:223-248): z = approximately D^-1 r by an inner CG on
// computeLhsDiag from z = 0 to ||r_inner|| < inner_tol (absolute).
static tr_status invprec(tr_ctx *c, const double *b, double *z, int inner_max, double inner_tol, int *inner_k,
                         int64_t *diag_apps) {
    cudaStream_t st = stream_of(c);
    double *ip = c->inner[0], *iAp = c->inner[1], *ir = c->inner[2];
    CgScalars *s = c->cg + 1;
    tr_status ts = init_scalars(c, s, inner_tol, inner_max, st);
    if (ts != TR_OK) return ts;
    LAUNCH(launch_cg_start<double>(c, c->aslm, b, z, ir, nullptr, ip, nullptr, s, 0, st));
    int k = 0, done = 0;
    for (int guard = 0; guard < (1 << 24); ++guard) {
        for (int i = 0; i < kCgChunk; ++i) {
            LAUNCH(launch_lhs_diag<double>(c, c->op64, ip, iAp, &s->done, st));
            LAUNCH(launch_dot<double, double>(c, c->aslm, ip, iAp, c->red_out + 4, st));
            k_set_alpha<<<1, 1, 0, st>>>(s, c->red_out + 4); ++c->launches;
            TRY(cudaGetLastError());
            LAUNCH(launch_cg_update<double>(c, c->aslm, z, ir, ip, iAp, nullptr, nullptr, s, nullptr, 0, 0, st));
            LAUNCH(launch_cg_direction<double>(c, c->aslm, ip, ir, s, st));
        }
        ts = read_status(c, s, &k, &done, st);
        if (ts != TR_OK) return ts;
        if (done) break;
    }
    // reference count: the loop index at exit (main.cpp:232-247)
    *inner_k += (done == 1) ? k - 1 : k;
    *diag_apps += k;
    return TR_OK;
}

// ----------------------------------------------------------------- FP64
static tr_status solve_fp64(tr_ctx *c, const tr_solve_opts *o, const double *b, double *x,
                            tr_solve_report *rep) {
    cudaStream_t st = stream_of(c);
    double *r = c->w64[1], *p = c->w64[2], *Ap = c->w64[3], *z = c->w64[4];
    CgScalars *s = c->cg;
    const int maxit = o->max_iter > 0 ? o->max_iter : 1000;
    const double *dinv = (o->precondition == TR_PREC_JACOBI) ? c->op64.dinv : nullptr;

    LAUNCH(launch_dot<double, double>(c, c->aslm, b, b, c->red_out, st));

    double bb = 0.0;
    tr_status ts = read_double(c, c->red_out, &bb, st);
    if (ts != TR_OK) return ts;
    const double bnorm = std::sqrt(bb);
    rep->rhs_norm = bnorm;
    rep->initial_residual = bnorm;
    const double tol = o->relative ? o->tol * bnorm : o->tol;
    ts = init_scalars(c, s, tol, maxit, st);
    if (ts != TR_OK) return ts;

    int k = 0, done = 0;
    if (o->precondition != TR_PREC_REFERENCE) {
        double *const pbuf[2] = {p, c->w64[6]};
        LAUNCH(launch_cg_start<double>(c, c->aslm, b, x, r, z, p, dinv, s, 1, st));
        int slot = dinv ? 1 : 0;
        ts = run_cg<double>(c, slot, c->op64, c->aslm, x, r, pbuf, Ap, z, dinv, s, c->dhist, c->hist_cap,
                            base_engine(o->engine), &k, &done);
        if (ts != TR_OK) return ts;
        rep->lhs_applications_f64 += k;
    } else {
        // host-driven outer loop around the inner CG (main.cpp:131-160)
        const int imax = o->inner_max_iter > 0 ? o->inner_max_iter : 1000;
        const double itol = o->inner_tol > 0 ? o->inner_tol : 1e-8;
        int inner = 0;
        int64_t dapps = 0;
        TRY(cudaMemsetAsync(x, 0, sizeof(double) * c->nP * c->aslm, st));
        TRY(cudaMemcpyAsync(r, b, sizeof(double) * c->nP * c->aslm, cudaMemcpyDeviceToDevice, st));
        ts = invprec(c, r, z, imax, itol, &inner, &dapps);
        if (ts != TR_OK) return ts;
        TRY(cudaMemcpyAsync(p, z, sizeof(double) * c->nP * c->aslm, cudaMemcpyDeviceToDevice, st));
        LAUNCH(launch_dot<double, double>(c, c->aslm, r, z, c->red_out + 1, st));
        k_set_nrz<<<1, 1, 0, st>>>(s, c->red_out + 1); ++c->launches;
        TRY(cudaGetLastError());
        for (int it = 0; it < maxit; ++it) {
            LAUNCH(launch_lhs<double>(c, c->op64, p, Ap, 2, nullptr, s, &s->done, st));
            // x += alpha p, r -= alpha Ap, stop test; beta follows invprec
            LAUNCH(launch_cg_update<double>(c, c->aslm, x, r, p, Ap, nullptr, nullptr, s, c->dhist, c->hist_cap, 1,
                                         st));
            rep->lhs_applications_f64 += 1;
            ts = read_status(c, s, &k, &done, st);
            if (ts != TR_OK) return ts;
            if (done) break;
            ts = invprec(c, r, z, imax, itol, &inner, &dapps);
            if (ts != TR_OK) return ts;
            LAUNCH(launch_dot<double, double>(c, c->aslm, z, r, c->red_out + 1, st));
            k_set_beta<<<1, 1, 0, st>>>(s, c->red_out + 1); ++c->launches;
            TRY(cudaGetLastError());
            LAUNCH(launch_cg_direction<double>(c, c->aslm, p, z, s, st));
        }
        rep->inner_iterations = inner;
        rep->diag_applications = dapps;
    }
    rep->iterations = k;
    rep->converged = (done == 1);
    if (done == 3) {
        c->last_error = "CG produced a non-finite residual";
        return TR_ERR_NAN;
    }
    return TR_OK;
}

// ---------------------------------------------------------------- mixed
static tr_status solve_mixed(tr_ctx *c, const tr_solve_opts *o, const double *b, double *x,
                             tr_solve_report *rep) {
    cudaStream_t st = stream_of(c);
    double *r64 = c->w64[1], *Ax = c->w64[3];
    float *d = c->w32[0], *r = c->w32[1], *p = c->w32[2], *Ap = c->w32[3], *z = c->w32[4];
    CgScalars *so = c->cg + 2, *si = c->cg + 3;
    const double *bb_src = b;
    const float *dinv = (o->precondition == TR_PREC_JACOBI) ? c->op32.dinv : nullptr;
    const int max_outer = o->max_outer > 0 ? o->max_outer : 30;
    // single-reduction inner CG: the SIMT FP32 operator only
    const bool single_reduction = o->engine == TR_ENGINE_PERSISTENT_SR && c->op32.kind == TR_OPERATOR_SIMT;
    const int inner_max = o->inner_max_iter > 0 ? o->inner_max_iter : (o->max_iter > 0 ? o->max_iter : 1000);

    tr_status ts = init_scalars(c, so, 0.0, 0, st);
    if (ts != TR_OK) return ts;
    TRY(cudaMemsetAsync(x, 0, sizeof(double) * c->nP * c->aslm, st));
    TRY(cudaMemsetAsync(Ax, 0, sizeof(double) * c->nP * c->aslm, st));
    LAUNCH(launch_residual(c, bb_src, Ax, r64, so, st));  // r = b, scale = ||b||
    double bnorm = 0.0;
    ts = read_double(c, &so->scale, &bnorm, st);
    if (ts != TR_OK) return ts;
    rep->rhs_norm = bnorm;
    rep->initial_residual = bnorm;
    const double target = o->relative ? o->tol * bnorm : o->tol;
    double rn = bnorm;
    int total = 0, outer = 0, hist_used = 0;
    bool converged = (rn < target);
    // The two-reduction FP32 CG runs with reliable updates: after each
    // defect correction it continues with its last direction instead of
    // restarting, so the Krylov space built so far is kept (the FP32 CG
    // runs in the frame of the normalised residual; frame_scale is that
    // frame's ||r64||).  The single-reduction engine restarts each time.
    bool started = false, restart = true;
    int k_run = 0, leg_k = 0;
    double frame_scale = rn, leg_tol = 0.0;
    while (!converged && outer < max_outer && total < (o->max_iter > 0 ? o->max_iter : 1 << 30)) {
        LAUNCH(launch_to_f32(c, r64, r, so, st));
        // each FP32 solve aims at what is still missing to the target
        // (relative to the normalised residual), floored where FP32 CG
        // stops gaining true accuracy
        // (the continued CG updates reliably every kReliableDelta of residual
        // reduction: longer FP32 legs let the recursive residual drift from
        // the true one, which a continued direction cannot absorb)
        const double inner_tol =
            o->inner_tol > 0 ? o->inner_tol
                             : std::min(0.5, std::max(0.3 * target / rn,
                                                      single_reduction ? kMixedInnerFloor : kReliableDelta));
        int k = 0, done = 0;
        if (single_reduction) {
            ts = init_scalars(c, si, inner_tol, inner_max, st);
            if (ts != TR_OK) return ts;
            // step 0 reads r_{-1} = r (the FP32 residual) and zero w_{-1},
            // s_{-2}, p_{-2}, x_{-1}
            const size_t bytes = sizeof(float) * c->nP * c->aslm32;
            SrArgs<float> a;
            a.x = d;
            a.p = p;
            a.R[0] = z;
            a.R[1] = r;
            a.W[0] = Ap;
            a.W[1] = c->w32[5];
            a.S[0] = c->w32[6];
            a.S[1] = c->w32[7];
            a.dinv = dinv;
            a.s = si;
            a.hist = nullptr;
            a.hist_cap = 0;
            TRY(cudaMemsetAsync(a.x, 0, bytes, st));
            TRY(cudaMemsetAsync(a.p, 0, bytes, st));
            TRY(cudaMemsetAsync(a.W[1], 0, bytes, st));
            TRY(cudaMemsetAsync(a.S[0], 0, bytes, st));
            ts = run_sr<float>(c, c->op32, a, &k, &done);
        } else {
            if (restart) {
                ts = init_scalars(c, si, inner_tol, inner_max, st);
                if (ts != TR_OK) return ts;
                LAUNCH(launch_cg_start<float>(c, c->aslm32, r, d, r, z, p, dinv, si, 1, st));
                started = true;
                k_run = 0;
            } else {
                // new stop rule for this leg, then the reliable update
                CgScalars h;
                h.tol = inner_tol;
                h.maxit = k_run + inner_max;
                TRY(cudaMemcpyAsync(&si->tol, &h.tol, sizeof(double), cudaMemcpyHostToDevice, st));
                TRY(cudaMemcpyAsync(&si->maxit, &h.maxit, sizeof(int32_t), cudaMemcpyHostToDevice, st));
                LAUNCH(launch_cg_reliable(c, d, r, z, dinv, si, rn / frame_scale, st));
                // The persistent kernel reads p_old from buffer k & 1 (k the
                // running iteration count), where its last leg left it.  The
                // graph and launch engines start every leg at chunk position
                // 0, reading buffer 0, and a leg of m iterations leaves its
                // last direction in buffer m & 1.
                if (c->last_cg_engine != TR_ENGINE_PERSISTENT && (leg_k & 1))
                    TRY(cudaMemcpyAsync(p, c->w32[5], sizeof(float) * c->nP * c->aslm32, cudaMemcpyDeviceToDevice,
                                        st));
            }
            frame_scale = rn;
            int slot = dinv ? 3 : 2;
            float *const pbuf[2] = {p, c->w32[5]};
            int kc = 0;
            ts = run_cg<float>(c, slot, c->op32, c->aslm32, d, r, pbuf, Ap, z, dinv, si, nullptr, 0,
                               base_engine(o->engine), &kc, &done);
            k = kc - k_run;  // iterations of this leg
            k_run = kc;
            leg_k = k;
            leg_tol = inner_tol;
        }
        if (ts != TR_OK) return ts;
        total += k;
        rep->lhs_applications_f32 += k;
        LAUNCH(launch_correct(c, x, d, so, st));
        LAUNCH(launch_lhs<double>(c, c->op64, x, Ax, 0, nullptr, nullptr, nullptr, st));
        rep->lhs_applications_f64 += 1;
        LAUNCH(launch_residual(c, bb_src, Ax, r64, so, st));
        ts = read_double(c, &so->scale, &rn, st);
        if (ts != TR_OK) return ts;
        if (o->history && hist_used < o->history_len) o->history[hist_used++] = rn;
        ++outer;
        if (!std::isfinite(rn)) {
            c->last_error = "defect correction produced a non-finite residual";
            return TR_ERR_NAN;
        }
        converged = rn < target;
        // continue the Krylov space only while the FP32 recursion tracks the
        // true residual; if the leg's true residual missed its goal by more
        // than 10x, the next leg restarts from p = 0
        if (started && !single_reduction) restart = !(rn <= 10.0 * leg_tol * frame_scale) || done == 2;
        if (done == 3) {
            c->last_error = "FP32 inner CG produced a non-finite residual";
            return TR_ERR_NAN;
        }
    }
    rep->iterations = total;
    rep->outer_steps = outer;
    rep->converged = converged;
    rep->final_residual = rn;
    return TR_OK;
}

tr_status solve(tr_ctx *c, const tr_solve_opts *o, const double *b_in, double *f, tr_solve_report *rep) {
    cudaStream_t st = stream_of(c);
    std::memset(rep, 0, sizeof(*rep));
    const int64_t launches0 = c->launches;
    tr_status ts = ensure_workspace(c, std::max(o->max_iter, 1));
    if (ts != TR_OK) return ts;
    for (cudaEvent_t &e : c->ev)
        if (!e) TRY(cudaEventCreate(&e));
    c->cg_ms = 0.0;
    c->cg_launches = 0;
    cudaEvent_t e0 = c->ev[0], e1 = c->ev[1];
    TRY(cudaEventRecord(e0, st));
    double *b = c->w64[5];
    if (b_in) TRY(cudaMemcpyAsync(b, b_in, sizeof(double) * c->nP * c->aslm, cudaMemcpyDeviceToDevice, st));
    else LAUNCH(launch_rhs(c, b, st));
    double *x = c->w64[0];
    if (o->mode == TR_MODE_MIXED) ts = solve_mixed(c, o, b, x, rep);
    else ts = solve_fp64(c, o, b, x, rep);
    if (ts != TR_OK && ts != TR_ERR_NAN) return ts;
    tr_status solve_status = ts;
    if (o->mode != TR_MODE_MIXED) {
        // true FP64 residual of the returned solution
        CgScalars *sr = c->cg + 2;
        LAUNCH(launch_lhs<double>(c, c->op64, x, c->w64[3], 0, nullptr, nullptr, nullptr, st));
        LAUNCH(launch_residual(c, b, c->w64[3], c->w64[1], sr, st));
        tr_status rs = read_double(c, &sr->scale, &rep->final_residual, st);
        if (rs != TR_OK) return rs;
        if (o->history && o->history_len > 0) {
            int n = std::min(rep->iterations, std::min(o->history_len, c->hist_cap));
            if (n > 0) TRY(cudaMemcpyAsync(o->history, c->dhist, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
    }
    TRY(cudaMemcpyAsync(f, x, sizeof(double) * c->nP * c->aslm, cudaMemcpyDeviceToDevice, st));
    TRY(cudaEventRecord(e1, st));
    TRY(cudaEventSynchronize(e1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    rep->device_ms = ms;
    rep->kernel_launches = c->launches - launches0;
    rep->cg_kernel_ms = c->cg_ms;
    rep->cg_kernel_launches = c->cg_launches;
    if (solve_status != TR_OK) return solve_status;
    if (!rep->converged) {
        c->last_error = "solver reached its iteration limit before the tolerance";
        return TR_ERR_NOT_CONVERGED;
    }
    return TR_OK;
}

}  // namespace transfer
