/*
 * transfer_b200.h -- C ABI of the B200-native radiative-transfer hot path.
 *
 * The path: the matrix-free even-parity spherical-harmonics Galerkin operator
 * on a P1 tetrahedral mesh (reference kernels.cu: volumePart/surfacePart and
 * their Diag variants, rightHandSide, the BLAS-1 and reduction kernels), the
 * Conjugate Gradient solve that drives it (main.cpp:125-160, invprec at
 * main.cpp:223-248), the Lanczos estimate of lambda_max (Eigenvalue.cpp:5-83)
 * and the reduction of the solution to energy density U, radiation pressure
 * tensor T and flux W (MeshData.cpp:96-136).
 *
 * Every entry point below replaces one member of the reference's
 * `struct CudaContext` (CudaContext.h:9-50) or one host routine it is used
 * with; each declaration cites the reference symbol it stands in for.
 *
 * Conventions
 *  - All functions return a tr_status; TR_OK == 0.  tr_last_error() gives a
 *    human-readable message for the last failure on a context (or globally,
 *    for failures before a context exists).
 *  - Vectors are DEVICE pointers laid out like the reference's:
 *    f[vertex][lm] at f[vertex*aslm + lm], aslm = slm rounded up to 8 doubles
 *    (64 bytes; common.cuh:5-6 with REAL=double) for the FP64 entry points and
 *    to 16 floats for the *_f32 ones.  Padding entries are written as zero.
 *  - Every call runs on the context's stream (tr_ctx_set_stream) and has
 *    completed when the call returns (as the reference's synchronous
 *    driver-API calls had), unless the name ends in _async.
 *  - No entry point falls back to a CPU implementation: without a usable
 *    CUDA device tr_ctx_create returns TR_ERR_NO_DEVICE.
 */
#ifndef TRANSFER_B200_H
#define TRANSFER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TR_ABI_VERSION 2

/* Vertex / element index type (util.h:6 `typedef uint32_t idx`). */
typedef uint32_t tr_idx;

/* Maximum padded angular size (common.cuh:7 ASLM_MAX = 128, so maxk <= 7). */
#define TR_ASLM_MAX 128
#define TR_MAXK_MAX 7

/* Element record, byte-compatible with the reference's `tetrahedron`
 * built with REAL=double (tetrahedron.h:7-20, 128 bytes):
 *   p[4]          vertex indices
 *   kappa_volume  kappa(region) * volume            (MeshData.cpp:63)
 *   I_p           Planck intensity of the region      (MeshData.cpp:64)
 *   s[j][0..2]    area-weighted normal of the face opposite local vertex j;
 *                 sum_j s[j] = 0 (MeshData.cpp:65-76). */
typedef struct tr_tetrahedron {
    tr_idx p[4];
    double kappa_volume;
    double I_p;
    double s[4][3];
} tr_tetrahedron;

/* Boundary face record, byte-compatible with the reference's `face`
 * with REAL=double (face.h:8-18, 64 bytes).  p[3] is padding. */
typedef struct tr_face {
    tr_idx p[4];
    double s[3];
    double _pad[3];
} tr_face;

/* Host view of the reference's MeshData (MeshData.h:13-32).  All arrays are
 * HOST pointers owned by the caller; tr_ctx_create copies them. */
typedef struct tr_mesh_view {
    tr_idx nP, nF, nT;
    const tr_idx *tetstart;          /* [nP+1]  vertex -> incident tets (CSR) */
    const tr_idx *tetidx;            /* [tetstart[nP]] */
    const tr_idx *tetpos;            /* [tetstart[nP]] local vertex 0..3 */
    const tr_tetrahedron *mesh;      /* [nT] */
    const tr_idx *facestart;         /* [nP+1]  vertex -> boundary faces */
    const tr_idx *faceidx;           /* [facestart[nP]] */
    const tr_idx *facepos;           /* [facestart[nP]] local vertex 0..2 */
    const tr_face *bnd;              /* [nF] */
} tr_mesh_view;

/* Host view of the reference's AngularData (AngularData.h:8-18): UNPADDED
 * tables with stride slm, omega[i][lm1][lm2] at omega[i*slm*slm+lm1*slm+lm2],
 * omega_pos likewise (0..2), O_x/O_y/O_z [slm][slm]. */
typedef struct tr_angular_view {
    tr_idx slm;
    const double *omega;
    const tr_idx *omega_pos;
    const double *Ox, *Oy, *Oz;
} tr_angular_view;

/* Physics beyond the reference (all optional; a NULL view or NULL member
 * reproduces the reference exactly: absorption + emission, vacuum).
 *  kappa_abs_volume[nT]  coefficient of the l=0 mass term (sigma_a * V) for
 *                        isotropic scattering; NULL -> kappa_volume.
 *  face_bc[nF]           TR_BC_VACUUM (reference), TR_BC_REFLECTIVE or
 *                        TR_BC_INCIDENT (vacuum + isotropic inflow).
 *  face_incident[nF]     isotropic incoming intensity for TR_BC_INCIDENT.
 *  surface_mode          TR_SURFACE_AXIS (reference: dominant-axis |Omega.n|,
 *                        kernels.cu:419-425) or TR_SURFACE_EXACT. */
enum { TR_BC_VACUUM = 0, TR_BC_REFLECTIVE = 1, TR_BC_INCIDENT = 2 };
enum { TR_SURFACE_AXIS = 0, TR_SURFACE_EXACT = 1 };
typedef struct tr_physics_view {
    const double *kappa_abs_volume;
    const int32_t *face_bc;
    const double *face_incident;
    int32_t surface_mode;
} tr_physics_view;

typedef enum tr_status {
    TR_OK = 0,
    TR_ERR_INVALID_ARG = 1,
    TR_ERR_CUDA = 2,
    TR_ERR_NOT_CONVERGED = 3,
    TR_ERR_NAN = 4,
    TR_ERR_NO_DEVICE = 5,
    TR_ERR_MESH = 6,
    TR_ERR_CONFIG = 7,
    TR_ERR_OUT_OF_MEMORY = 8,
    TR_ERR_UNSUPPORTED = 9,
    TR_ERR_IO = 10
} tr_status;

typedef struct tr_ctx tr_ctx;

typedef struct tr_ctx_info {
    tr_idx nP, nT, nF;
    tr_idx slm;
    tr_idx aslm;          /* FP64 vector padding (8 doubles)  */
    tr_idx aslm_f32;      /* FP32 vector padding (16 floats)  */
    uint64_t n_edges;     /* assembled vertex-vertex couplings */
    uint64_t n_bnd_edges; /* boundary couplings                */
    uint64_t device_bytes;/* device memory held by the context */
    int device;
} tr_ctx_info;

/* ---- context (CudaContext::CudaContext / ~CudaContext, CudaContext.cpp:24-58) */
tr_status tr_ctx_create(int device, const tr_mesh_view *mesh,
                        const tr_angular_view *ang, tr_ctx **out);
tr_status tr_ctx_create_ex(int device, const tr_mesh_view *mesh,
                           const tr_angular_view *ang,
                           const tr_physics_view *phys, tr_ctx **out);
tr_status tr_ctx_destroy(tr_ctx *ctx);
tr_status tr_ctx_info_get(const tr_ctx *ctx, tr_ctx_info *info);
/* Operator kernel family (no reference counterpart; results agree to
 * rounding): TR_OPERATOR_TENSOR computes each vertex's edge sums as a small
 * dense product on the tensor cores (FP32: split-TF32, FP64: DMMA);
 * TR_OPERATOR_SIMT accumulates them with FMA instructions.  A new context
 * uses TENSOR for FP64 and SIMT for FP32; this call sets both precisions. */
enum { TR_OPERATOR_SIMT = 0, TR_OPERATOR_TENSOR = 1 };
tr_status tr_ctx_set_operator(tr_ctx *ctx, int kind);
/* Operator autotuner (no reference counterpart): for each precision, times
 * both kernel families as the solver runs them -- `iters` iterations of the
 * persistent CG on this context's right-hand side (FP64 mode for FP64, the
 * mixed mode's FP32 CG for FP32), device time of the CG launches per
 * iteration, the second of two runs -- and keeps the faster for that
 * precision.  ms receives the milliseconds per CG iteration: {FP64 SIMT,
 * FP64 tensor, FP32 SIMT, FP32 tensor}.  Allocates the solver work space if
 * no solve has done so yet. */
tr_status tr_ctx_autotune_operator(tr_ctx *ctx, int iters, double ms[4]);
/* The kernel family in use: kinds[0] for FP64, kinds[1] for FP32. */
tr_status tr_ctx_get_operator(const tr_ctx *ctx, int kinds[2]);
/* cudaStream_t passed as void*; NULL selects the context's own stream. */
tr_status tr_ctx_set_stream(tr_ctx *ctx, void *stream);
const char *tr_last_error(const tr_ctx *ctx);
const char *tr_status_string(tr_status st);
int tr_abi_version(void);

/* ---- operator (CudaContext::computeLhs/computeLhsDiag/computeRhs,
 *      CudaContext.cpp:99-130; kernels.cu:135-493) ------------------------ */
/* Af = A f : volumePart (kernels.cu:200-287) + surfacePart (:383-438). */
tr_status tr_compute_lhs(tr_ctx *ctx, const double *f, double *Af);
/* Af = D f : volumePartDiag (:290-357) + surfacePartDiag (:440-493). */
tr_status tr_compute_lhs_diag(tr_ctx *ctx, const double *f, double *Af);
/* b = (e_i, kappa I_p) : rightHandSide (:135-165), plus inflow terms. */
tr_status tr_compute_rhs(tr_ctx *ctx, double *b);

/* ---- BLAS-1 over all nP*aslm entries (kernels.cu:12-50,
 *      CudaContext.cpp:137-173) ------------------------------------------ */
tr_status tr_scale(tr_ctx *ctx, double *x, double wx);                  /* x *= wx */
tr_status tr_add_prod(tr_ctx *ctx, double *x, const double *y, double wy); /* x += wy*y */
tr_status tr_mul_add(tr_ctx *ctx, double *x, double wx, const double *y);  /* x = wx*x+y */
tr_status tr_mul_add_prod(tr_ctx *ctx, double *x, double wx,
                          const double *y, double wy);                  /* x = wx*x+wy*y */
/* Reductions over vertices and lm < slm (normKern/dotKern, kernels.cu:55-115;
 * CudaContext::norm/dot, CudaContext.cpp:175-198).  Deterministic order. */
tr_status tr_norm(tr_ctx *ctx, const double *x, double *out);
tr_status tr_dot(tr_ctx *ctx, const double *x, const double *y, double *out);

/* tr_dot without a context and without allocating (no counterpart in the
 * reference).  For callers that may not call cudaMalloc here: a host whose
 * memory pool owns all device memory, a loop where cudaMalloc/cudaFree would
 * synchronise the device, or a caller without a tr_ctx (creating one
 * allocates).  x, y: FP64 device vectors [nP][aslm] on the current device;
 * the sum runs over lm < slm.  out: ONE double of device memory, written by
 * a kernel queued on `stream` (cudaStream_t as void*, NULL = legacy default
 * stream); the call returns without waiting for it.  Limit: nP * aslm <=
 * 33,554,432 entries, else TR_ERR_INVALID_ARG (message in
 * tr_last_error(NULL)).  Its scratch is one static device array of about
 * 16 KiB per GPU, shared by all calls: calls that overlap on the GPU race
 * and must be ordered by the caller.  Each call looks up that array's
 * device address in the current context, so a cudaDeviceReset (or another
 * context made current) between calls is safe; the first call on a device
 * also loads the library's module there (set-up work), so make it before
 * any stream capture on that device.  nP = 0 writes 0.0 to *out.
 * Summation order depends only on nP * aslm, so the
 * bits do not depend on the GPU; they may differ from tr_dot's in the last
 * places. */
tr_status tr_dot_noalloc(const double *x, const double *y, uint32_t nP,
                         uint32_t aslm, uint32_t slm, double *out,
                         void *stream);

/* FP32 variants (the reference's default REAL=float build): vectors with
 * aslm_f32 padding, operator tables rounded to float once at creation. */
tr_status tr_compute_lhs_f32(tr_ctx *ctx, const float *f, float *Af);
tr_status tr_compute_lhs_diag_f32(tr_ctx *ctx, const float *f, float *Af);
tr_status tr_compute_rhs_f32(tr_ctx *ctx, float *b);
tr_status tr_dot_f32(tr_ctx *ctx, const float *x, const float *y, double *out);

/* ---- solver (main.cpp:125-160 CG; main.cpp:223-248 invprec) ------------ */
enum {
    TR_PREC_NONE = 0,        /* z = r                                       */
    TR_PREC_REFERENCE = 1,   /* invprec: inner CG on computeLhsDiag to 1e-8 */
    TR_PREC_JACOBI = 2       /* z = diag(A)^-1 r                            */
};
enum {
    TR_MODE_FP64 = 0,        /* plain FP64 CG (the drop-in)                 */
    TR_MODE_MIXED = 1        /* FP32 CG inside FP64 defect correction       */
};
enum {
    TR_ENGINE_PERSISTENT = 0,/* one cooperative kernel runs many iterations */
    TR_ENGINE_GRAPH = 1,     /* CUDA-graph replay of 2-launch iterations    */
    TR_ENGINE_LAUNCH = 2,    /* the same launches issued one by one         */
    TR_ENGINE_PERSISTENT_SR = 3 /* mixed mode: the FP32 inner solves run
                                single-reduction CG (Chronopoulos-Gear: one
                                grid barrier per iteration) in one
                                cooperative kernel; same iterates in exact
                                arithmetic, different rounding.  FP64 mode
                                and the tensor-core FP32 operator run
                                TR_ENGINE_PERSISTENT.  No reference
                                counterpart.                                */
};
typedef struct tr_solve_opts {
    int32_t mode;            /* TR_MODE_*                                   */
    int32_t precondition;    /* TR_PREC_*                                   */
    int32_t max_iter;        /* outer CG iterations (reference: 1000)       */
    int32_t relative;        /* 0: stop when ||r|| < tol (reference),
                                1: stop when ||r||/||b|| < tol              */
    double  tol;             /* reference: 1e-4 absolute                    */
    double  inner_tol;       /* invprec tolerance (reference 1e-8, absolute);
                                mixed mode: relative reduction per inner
                                FP32 solve (0 -> adaptive: 0.3 x what is
                                still missing to tol, at least 2e-6)        */
    int32_t inner_max_iter;  /* invprec / FP32 inner cap (0 -> 1000)       */
    int32_t max_outer;       /* mixed mode: defect-correction steps (0->30) */
    int32_t engine;          /* TR_ENGINE_* (0-2 give identical results)    */
    int32_t history_len;     /* capacity of history[] (may be 0)            */
    double *history;         /* host array: ||r|| after each CG iteration   */
} tr_solve_opts;

typedef struct tr_solve_report {
    int32_t converged;
    int32_t iterations;          /* outer CG iterations (FP64 mode) or total
                                    FP32 CG iterations (mixed mode)         */
    int32_t inner_iterations;    /* invprec iterations summed (main.cpp:247) */
    int32_t outer_steps;         /* mixed mode defect-correction steps       */
    int64_t lhs_applications_f64;/* operator applications, FP64              */
    int64_t lhs_applications_f32;/* operator applications, FP32              */
    int64_t diag_applications;   /* preconditioner operator applications     */
    double  initial_residual;    /* ||b - A f0||_2, FP64                      */
    double  final_residual;      /* ||b - A f||_2 recomputed in FP64          */
    double  rhs_norm;            /* ||b||_2                                   */
    double  device_ms;           /* device time of the solve (CUDA events)    */
    int64_t kernel_launches;     /* kernels of this library launched (graph
                                    nodes counted one by one)               */
    double  cg_kernel_ms;        /* device time of the CG-iteration launches
                                    (persistent kernels or graph replays),
                                    CUDA events around each                 */
    int64_t cg_kernel_launches;  /* those launches                           */
} tr_solve_report;

void tr_solve_opts_default(tr_solve_opts *opts);   /* reference settings */

/* Solve A f = b from f = 0.  b: device vector, or NULL to use computeRhs.
 * f: device vector (output). */
tr_status tr_solve(tr_ctx *ctx, const tr_solve_opts *opts, const double *b,
                   double *f, tr_solve_report *report);
/* Same with HOST buffers: copies b in and f out.  Page-locked buffers
 * (cudaMallocHost, cudaHostRegister, torch pin_memory) are copied by DMA
 * directly; pageable ones through the context's pinned staging buffers. */
tr_status tr_solve_host(tr_ctx *ctx, const tr_solve_opts *opts,
                        const double *b_host, double *f_host,
                        tr_solve_report *report);

/* Measurement helper (no reference counterpart): launches the operator
 * (precision 64: tr_compute_lhs, 32: tr_compute_lhs_f32) `iters` times back
 * to back on the context stream from x into y (device vectors of that
 * precision), after 3 untimed launches, and returns the mean device time
 * per launch from CUDA events. */
tr_status tr_bench_lhs(tr_ctx *ctx, int precision, const void *x, void *y,
                       int iters, double *ms_per_launch);

/* Self-test of the bounded grid barrier of the persistent CG kernels (no
 * reference counterpart): a cooperative grid of one block per SM on `device`
 * runs `rounds` barriers; if skip_block >= 0 that block never arrives, and
 * the others must give up after max_polls (<= 2^24) polls each.
 * *timed_out = 1 when the barrier gave up (the device stays usable). */
tr_status tr_selftest_grid_barrier(int device, int skip_block, int rounds,
                                   unsigned int max_polls, int *timed_out);

/* ---- post-processing (MeshData::ComputeMoments / ComputeFlux,
 *      MeshData.cpp:96-136), on the device ----------------------------- */
/* U[nP] = 4 pi I_00 ; T[3][3][nP] = 4 pi sum_lm omega_i[lm][0] I_lm. */
tr_status tr_compute_moments(tr_ctx *ctx, const double *f, double *U, double *T);
/* W[3][nT] = (1/3) sum_k sum_a s_k,a T_aj(p_k) / kappa_volume. */
tr_status tr_compute_flux(tr_ctx *ctx, const double *T, double *W);

/* ---- Lanczos lambda_max estimate (eigest/trieig, Eigenvalue.cpp:5-83) -- */
/* v: device vector, overwritten; w, v0: device work vectors.  Up to
 * max_steps (reference: 30) steps, stop when |dl| < 1e-6 lmax. */
tr_status tr_eig_lanczos(tr_ctx *ctx, double *v, double *v0, double *w,
                         int max_steps, double *lmax, double *extrapolated,
                         int *steps);
/* Largest eigenvalue of the symmetric tridiagonal (a[0..n-1], b[1..n-1] as
 * b[0..n-2]) by Newton on the characteristic polynomial (trieig). */
double tr_trieig(const double *a, const double *b, int n);

/* ---- discrete-ordinates sweep (no counterpart in the reference) --------
 *
 * The reference solves only the even-parity spherical-harmonics system
 * above.  This is the upwind transport sweep over the SAME problem data: the
 * `tetrahedron` records (outward face area normals s, kappa_volume = sigma_t
 * V, I_p = Planck intensity B) and boundary `face` records of tr_mesh_view,
 * with tr_physics_view's kappa_abs_volume (sigma_a V; sigma_s = sigma_t -
 * sigma_a scatters isotropically), face_bc and face_incident.  Angles are an
 * ordinate set (directions + weights summing to 1).
 *
 * Discretisation: linear discontinuous finite elements on each tetrahedron
 * (values at its 4 vertices), upwind between cells.  The unknowns of the
 * outer iteration are the scalar flux J[nT][4] (mean intensity at each
 * cell's vertices, J = sum_q w_q psi_q) and the extra vector B[n_extra]:
 * the inflow through reflective faces (4 values for each pair of a
 * reflective face and an ordinate entering through it, in (face, ordinate)
 * order) and through faces where a dependency cycle was cut ([n_lag][4]).
 * All vectors are FP64 DEVICE pointers, 16-byte aligned (TR_ERR_INVALID_ARG
 * otherwise). */
typedef struct tr_sweep tr_sweep;
typedef struct tr_ordinates_view {
    uint32_t nq;
    const double *x, *y, *z;   /* unit directions       */
    const double *w;           /* weights, sum 1         */
} tr_ordinates_view;
typedef struct tr_sweep_info {
    uint32_t nT, nF, nq;
    uint64_t n_extra;          /* length of B                              */
    uint32_t n_reflective;     /* reflective boundary faces                */
    uint32_t n_lag;            /* faces lagged to break dependency cycles  */
    uint32_t max_levels;       /* longest per-ordinate dependency chain    */
    uint32_t forced_levels;    /* levels started by cutting a cycle        */
    uint64_t device_bytes;
    int device;
} tr_sweep_info;
enum { TR_SWEEP_GMRES = 0, TR_SWEEP_SOURCE_ITERATION = 1 };
/* Diffusion synthetic acceleration (TR_SWEEP_PREC_DSA, after
 * tr_sweep_enable_dsa): GMRES becomes flexible GMRES right-preconditioned by
 * P^-1 y = y + C sigma_s y, and source iteration adds C sigma_s (S(x) - x)
 * to each iterate, where C solves the P1 diffusion problem -div(1 / (3
 * sigma_t)) grad f + sigma_a f = g with Marshak faces (vacuum and incident)
 * and zero current (reflective) -- the even-parity operator with l = 0 only,
 * continuous linear elements on the vertices, by FP64 Jacobi CG. */
enum { TR_SWEEP_PREC_NONE = 0, TR_SWEEP_PREC_DSA = 1 };
/* Where the diffusion CG runs.  CLUSTER: the assembled matrix (ELL) in one
 * thread-block cluster of 16 (or 8) CTAs with hardware cluster barriers, no
 * host round trip per solve, preconditioned by Jacobi plus an aggregation
 * coarse space (16 row blocks per CTA); meshes up to 2^18 vertices.  EVEN_PARITY: the
 * even-parity operator with l = 0 (tr_solve on its own context; its face
 * term uses the operator's face measure |s_x + s_y + s_z|, equal to the area
 * on axis-aligned faces).  AUTO: CLUSTER where available. */
enum { TR_SWEEP_DSA_AUTO = 0, TR_SWEEP_DSA_CLUSTER = 1, TR_SWEEP_DSA_EVEN_PARITY = 2 };
typedef struct tr_sweep_opts {
    int32_t method;            /* TR_SWEEP_*                                */
    int32_t mode;              /* TR_MODE_FP64, or TR_MODE_MIXED: FP32
                                  sweeps inside FP64 defect correction
                                  (each GMRES cycle starts from the FP64
                                  residual, its Krylov steps sweep in FP32) */
    double  tol;               /* GMRES: ||b - (I - T) x|| / ||b||, FP64;
                                  source iteration: relative change        */
    int32_t max_iter;          /* sweeps of the iteration (Krylov steps)   */
    int32_t restart;           /* GMRES restart length, 1..64              */
    double  inner_tol;         /* GMRES: end a cycle early once it reduced
                                  its residual by this factor, then restart
                                  from the true residual (0: never)        */
    int32_t max_outer;         /* unused; kept for layout                   */
    int32_t precondition;      /* TR_SWEEP_PREC_*                           */
    double  precond_tol;       /* DSA: relative tolerance of each diffusion
                                  solve (FP64 Jacobi CG), in (0, 1)        */
    int32_t precond_engine;    /* TR_SWEEP_DSA_*                            */
} tr_sweep_opts;
typedef struct tr_sweep_report {
    int32_t converged;
    int32_t iterations;        /* Krylov steps (or source iterations)      */
    int32_t outer_steps;       /* mixed mode: GMRES cycles (each from an
                                  FP64 residual)                           */
    int64_t sweeps_f32, sweeps_f64;
    double  residual;          /* final relative residual, FP64            */
    double  rhs_norm;
    double  device_ms;
    int64_t kernel_launches;   /* sweep kernels; the diffusion solves' own
                                  launches are not counted here            */
    int32_t precond_solves;    /* diffusion solves (DSA)                   */
    int32_t precond_iterations;/* their CG iterations summed               */
} tr_sweep_report;

/* Gauss-Legendre (n_polar in cos theta) x uniform azimuth (n_azim, at
 * (k + 1/2) 2 pi / n_azim) ordinates, n_polar * n_azim points, weights
 * summing to 1; mirror-symmetric in x, y, z for even n_azim. */
tr_status tr_ordinates_product(int n_polar, int n_azim, double *x, double *y, double *z, double *w);
/* Builds the device geometry (face adjacency, consistent face normals) and
 * the per-ordinate dependency levels (on the device). */
tr_status tr_sweep_create(int device, const tr_mesh_view *mesh, const tr_physics_view *phys,
                          const tr_ordinates_view *ord, tr_sweep **out);
/* Fails (TR_ERR_INVALID_ARG) while the sweep has live frequency groups. */
tr_status tr_sweep_destroy(tr_sweep *s);
/* A frequency group of `parent` (no reference counterpart: the reference
 * solves one grey problem): a sweep over the same mesh, boundary kinds,
 * ordinates and dependency schedule -- shared with the parent, not copied --
 * with its own per-cell sigma_t V (kappa_volume), sigma_a V (NULL: no
 * scattering) and Planck intensity I_p (NULL: the parent's), and its own
 * angular flux and solver state.  Groups are independent problems (no group
 * coupling); the batched calls run any mix of parents and groups in one
 * launch.  The parent must outlive its groups; a group cannot have groups. */
tr_status tr_sweep_create_group(tr_sweep *parent, const double *kappa_volume, const double *kappa_abs_volume,
                                const double *I_p, tr_sweep **out);
/* Frees the angular flux and Krylov work space of a sweep (allocated again
 * by the next sweep or solve): lets a caller solve many problems in FP64
 * one after another without holding every problem's work space. */
tr_status tr_sweep_release_work(tr_sweep *s);
const char *tr_sweep_last_error(const tr_sweep *s);
tr_status tr_sweep_info_get(const tr_sweep *s, tr_sweep_info *info);
/* level[q * nT + c]: dependency level of cell c in ordinate q (host array). */
tr_status tr_sweep_levels(tr_sweep *s, int32_t *level);
/* One sweep of all ordinates in FP32 (precision 32) or FP64 (64) from the
 * scattering source of J_in and the inflow B_in (NULL = 0); with_ext adds
 * emission and the incident boundary inflow.  J_out: scalar flux of the
 * result; B_out: the resulting reflective / lagged inflow (either NULL). */
tr_status tr_sweep_apply(tr_sweep *s, int precision, const double *J_in, const double *B_in, int with_ext,
                         double *J_out, double *B_out);
/* tr_sweep_apply for n independent problems (distinct sweeps on one device,
 * of any sizes and ordinate sets) in ONE launch of the sweep kernel, one
 * block per (problem, ordinate); per-problem arrays of device pointers (an
 * array pointer NULL = none for all).  Results equal n separate
 * tr_sweep_apply calls. */
tr_status tr_sweep_apply_batch(int n, tr_sweep *const *s, int precision, const double *const *J_in,
                               const double *const *B_in, int with_ext, double *const *J_out,
                               double *const *B_out);
/* Source iteration x <- S(x) (with sources, from x = 0) of n independent
 * problems at once: each iteration is one batched sweep launch plus every
 * problem's reductions, captured as a CUDA graph and replayed; a problem
 * whose relative change ||S(x) - x|| / ||S(x)|| falls below tol leaves the
 * running set (the graph is captured again for the rest), until all have
 * (or max_iter iterations).  Sweeps in precision 32 or 64 (FP64 iterates and stopping
 * test).  J[i] (and B[i] if B, for problems with n_extra > 0): device
 * outputs; iterations[i] (first iteration below tol, 0 if none) and
 * residual[i] (last relative change): host arrays [n]. */
tr_status tr_sweep_solve_batch(int n, tr_sweep *const *s, int precision, double tol, int max_iter, double *const *J,
                               double *const *B, int32_t *iterations, double *residual);
/* Form of the batched sweep launch (no reference counterpart; results do
 * not depend on it): a static grid of one block per (problem, ordinate)
 * task, or a persistent grid whose blocks draw tasks from an atomic queue
 * (largest problems first); each with the full shared-memory shape (a ring
 * of 4,096 upwind positions, one block per SM) or, for FP32, the small one
 * (1,024 positions, two blocks per SM).  TR_BATCH_RULE (-1): static grid,
 * small shape for FP32 when the tasks outnumber the SMs. */
enum { TR_BATCH_RULE = -1, TR_BATCH_STATIC_FULL = 0, TR_BATCH_STATIC_SMALL = 1, TR_BATCH_QUEUE_FULL = 2,
       TR_BATCH_QUEUE_SMALL = 3 };
tr_status tr_sweep_set_batch_form(tr_sweep *s, int form);
/* Autotuner of the batched launch: times one batched sweep of these n
 * problems (precision 32 or 64) in every form, sets the fastest on all n
 * (the batched calls use the form of their first sweep) and returns it in
 * *form; ms[4] (may be NULL): mean time of one batched sweep per form, -1
 * for a form that does not apply (the small shape in FP64). */
tr_status tr_sweep_autotune_batch(int n, tr_sweep *const *s, int precision, int *form, double *ms);
/* Times the FP32 sweep kernel in both shared-memory shapes on this problem
 * (full: one block per SM; small: two per SM, shorter ring) and keeps the
 * faster for its later FP32 sweeps (without it: small when there are more
 * ordinates than SMs).  shape: 0 full / 1 small; ms[2]: mean time of one
 * sweep in each (either may be NULL).  Results do not depend on the shape. */
tr_status tr_sweep_autotune(tr_sweep *s, int *shape, double *ms);
/* psi of the last sweep as FP64, device [nq][nT][4]. */
tr_status tr_sweep_psi(tr_sweep *s, double *psi);
/* Angular moments of the last sweep's psi: mom[m][nT][4] = sum_q w_q
 * Y_m(Omega_q) psi_q for m < nmom <= 16 (l <= 3, m index l^2 + l + mm,
 * real harmonics of tr_spherical_value, Y_00 = 1).  Generalises
 * MeshData::ComputeMoments (MeshData.cpp:96-116) to discrete ordinates.
 * After an FP32 sweep the product runs on the tensor cores in split TF32
 * with FP32 accumulation; after an FP64 sweep it accumulates in FP64. */
tr_status tr_sweep_moments(tr_sweep *s, int nmom, double *mom);
/* Kernel family of tr_sweep_moments after an FP32 sweep (no reference
 * counterpart; results agree to FP32 rounding):
 * TR_MOMENTS_TCGEN05 (default): tcgen05 MMAs with tensor-memory
 * accumulators, psi tiles loaded by TMA (up to 1,024 ordinates);
 * TR_MOMENTS_MMA_SYNC: warp-level mma.sync with cp.async staging (up to 384
 * ordinates);
 * TR_MOMENTS_TMA_FFMA2: psi tiles loaded by TMA, paired FP32 FMAs, each
 * accumulator over an eighth of the ordinates and the eight partial sums
 * added in FP64 (up to 1,024 ordinates).
 * Larger ordinate sets, and FP64 sweeps, use FP64 FMAs. */
enum { TR_MOMENTS_TCGEN05 = 0, TR_MOMENTS_MMA_SYNC = 1, TR_MOMENTS_TMA_FFMA2 = 2 };
tr_status tr_sweep_set_moments_kernel(tr_sweep *s, int kind);
/* FP64 energy balance of the last sweep given its inputs J_in, B_in and its
 * scalar flux J_out:  out = {emitted, absorbed, escaped, incoming,
 * reflective_net} with emitted + incoming = absorbed + escaped +
 * reflective_net (absorbed = sigma_t V mean J_out - sigma_s V mean J_in; at
 * convergence sigma_a V mean J).  Units: mean intensity x area. */
tr_status tr_sweep_balance(tr_sweep *s, const double *J_in, const double *B_in, const double *J_out,
                           double out[5]);
void tr_sweep_opts_default(tr_sweep_opts *opts);
/* Solves J = S(J, B) (scattering source iteration fixed point) by GMRES on
 * (I - T) x = S(0) or by source iteration; J [nT][4], B [n_extra] device
 * outputs (B may be NULL). */
tr_status tr_sweep_solve(tr_sweep *s, const tr_sweep_opts *opts, double *J, double *B, tr_sweep_report *rep);
/* Prepares the diffusion operator for TR_SWEEP_PREC_DSA from the mesh and
 * physics the sweep was created with (the vertex -> cell and vertex -> face
 * tables of the mesh view are used): an even-parity context with l = 0 on
 * the same device, with the reflective faces left out of its face list. */
tr_status tr_sweep_enable_dsa(tr_sweep *s, const tr_mesh_view *mesh, const tr_physics_view *phys);
/* Replaces the per-cell coefficients (HOST arrays [nT]: sigma_t V, sigma_a V
 * (NULL: sigma_a = sigma_t), Planck intensity B (NULL: kept)) without
 * rebuilding geometry or schedule, which depend on neither -- for parameter
 * studies and gradient steps.  The diffusion operator of
 * tr_sweep_enable_dsa keeps the coefficients it was built with (it only
 * preconditions; solves stay exact). */
tr_status tr_sweep_set_coefficients(tr_sweep *s, const double *kappa_volume, const double *kappa_abs_volume,
                                    const double *I_p);
/* Outflow of the last sweep through the boundary faces with face_mask[f]
 * != 0 (HOST array [nF]): F = sum_q w_q sum_f max(Omega_q.s_f, 0) mean_f psi_q
 * (mean intensity x area), FP64. */
tr_status tr_sweep_outflow(tr_sweep *s, const int32_t *face_mask, double *F);
/* Adjoint gradient of F (the outflow through a face set) with respect to
 * each cell's absorption and scattering coefficients sigma_a, sigma_s
 * (sigma_t = sigma_a + sigma_s, volumes fixed).  `adj` is the adjoint
 * problem: a sweep over the same mesh and coefficients with the ordinates
 * reversed (-Omega_q, same order and weights), no emission (I_p = 0),
 * unit isotropic inflow (TR_BC_INCIDENT, 1) on F's faces and vacuum
 * elsewhere -- the transpose of the upwind sweep is the sweep in the
 * reversed direction.  J, B: the converged forward solution; J_adj: the
 * converged adjoint scalar flux (tr_sweep_solve on adj).  Only the scalar
 * fluxes are kept between the solves: both angular fluxes are recomputed
 * here by one sweep each (precision 32 or 64).  Outputs: device [nT].
 * Faces must be vacuum or incident (no reflective faces, no cut cycles). */
tr_status tr_sweep_gradient(tr_sweep *fwd, tr_sweep *adj, int precision, const double *J, const double *B,
                            const double *J_adj, double *dF_dsigma_a, double *dF_dsigma_s);
/* Measurement helper: mean device time of one sweep with sources (3
 * untimed sweeps first). */
tr_status tr_sweep_bench(tr_sweep *s, int precision, int iters, double *ms_per_sweep);

/* ---- host problem data (C++ host code behind the C ABI) ---------------- */
/* AngularData(maxk) (AngularData.cpp:9-67): tables for the even harmonics
 * l = 0,2,..,2maxk; slm = (1+maxk)(1+2maxk). */
typedef struct tr_angular tr_angular;
tr_status tr_angular_create(int maxk, tr_angular **out);
tr_status tr_angular_view_get(const tr_angular *a, tr_angular_view *view);
void      tr_angular_destroy(tr_angular *a);

/* Spherical::value(l, m, x, y, z) (Spherical.cpp:62-82): real harmonic,
 * orthonormal on average over the sphere, no Condon-Shortley phase. */
double tr_spherical_value(int l, int m, double x, double y, double z);
/* HemiQuad(mindegree) (HemiQuad.cpp:265-286) / LebedevQuad(mindegree)
 * (LebedevQuad.cpp:6269-6277): returns the rule's number of points and, if
 * cap >= that number, fills x, y, z, w (weights sum to 1).  Returns -1 for
 * an unsupported degree.  The Lebedev rules are generated from their
 * defining equations instead of stored tables, up to 350 points (precision
 * 31; the first call for a rule solves it on the host's threads, at most a
 * few seconds; later calls use the cached rule); the points may come in
 * another order than the reference's tables. */
int tr_hemiquad(int mindegree, double *x, double *y, double *z, double *w, int cap);
int tr_lebedev(int mindegree, double *x, double *y, double *z, double *w, int cap);

/* Config(const char*) (Config.cpp:8-131): the radiation.cfg grammar. */
typedef struct tr_config tr_config;
tr_status tr_config_load(const char *path, tr_config **out);
void      tr_config_destroy(tr_config *c);
int       tr_config_get_int(const tr_config *c, const char *key, int *ok);
double    tr_config_get_double(const tr_config *c, const char *key, int *ok);
const char *tr_config_get_string(const tr_config *c, const char *key);
int       tr_config_num_regions(const tr_config *c);
double    tr_config_region_double(const tr_config *c, int region,
                                  const char *key, int *ok);

/* MeshData (MeshData.cpp:9-94) built from a tetrahedral mesh given by
 * vertex coordinates and connectivity, or generated (Kuhn-split box). */
typedef struct tr_meshdata tr_meshdata;
typedef struct tr_region_params {
    int32_t nreg;              /* regions are numbered 1..nreg            */
    const double *kappa;       /* [nreg+1], index 0 unused (Config.cpp)    */
    const double *Ip;          /* [nreg+1]                                 */
    const double *albedo;      /* [nreg+1] or NULL (no scattering)         */
} tr_region_params;
tr_status tr_meshdata_from_tets(tr_idx nP, const double *xyz, tr_idx nT,
                                const tr_idx *tets, const int32_t *region,
                                const tr_region_params *rp, tr_meshdata **out);
/* Kuhn box: n[3] cells, box = {x0,x1,y0,y1,z0,z1}, interior vertices jittered
 * uniformly by +-jitter*h (splitmix64 seeded); region_kind selects the
 * region map: 0 all region 1; 1 sphere (centre cx,cy,cz radius r -> region 1,
 * else 2); 2 half space x < x_split -> region 1, else 2. */
typedef struct tr_kuhn_params {
    int32_t n[3];
    double box[6];
    double jitter;
    uint64_t seed;
    int32_t region_kind;
    double region_arg[4];
    int32_t ball;              /* 1: keep only tets with centroid |c-c0|<=R */
    double ball_center[3];
    double ball_radius;
} tr_kuhn_params;
tr_status tr_meshdata_kuhn(const tr_kuhn_params *kp, const tr_region_params *rp,
                           tr_meshdata **out);
tr_status tr_meshdata_view_get(const tr_meshdata *md, tr_mesh_view *view);
/* Vertex coordinates [nP][3] and region id per tet [nT]. */
const double  *tr_meshdata_coords(const tr_meshdata *md);
const int32_t *tr_meshdata_regions(const tr_meshdata *md);
/* Per-tet sigma_a*V (NULL when no region scatters) and per-face box side
 * (0..5 for x0,x1,y0,y1,z0,z1; -1 otherwise). */
const double  *tr_meshdata_kappa_abs_volume(const tr_meshdata *md);
const int32_t *tr_meshdata_face_side(const tr_meshdata *md);
void tr_meshdata_destroy(tr_meshdata *md);

/* Mesh I/O in place of the reference's meshProcessor library (MeshData.cpp:10
 * reads the meshfile of radiation.cfg, main.cpp:209-216 saves the solution
 * with saveVtk).  tr_meshdata_read_vol reads a Netgen ".vol" mesh: points,
 * volumeelements (region = matnr; the first four vertices of each element)
 * and surfaceelements / surfaceelementsgi, whose bcnr is kept per boundary
 * face (tr_meshdata_face_bcnr, -1 where a face has no surface element; NULL
 * for meshes not read from .vol). */
tr_status tr_meshdata_read_vol(const char *path, const tr_region_params *rp, tr_meshdata **out);
const int32_t *tr_meshdata_face_bcnr(const tr_meshdata *md);
/* Legacy VTK unstructured grid (binary, big-endian reals of real_bytes 4 or
 * 8) with the mesh and the given fields, as saveVtk writes "W%v" cell vectors
 * and "U%sT%t..." point scalars / symmetric tensors.  Field data are
 * component-major: data[c * n + i] for component c of point / cell i; a
 * TR_VTK_TENSOR gives the 6 components xx xy xz yy yz zz. */
enum { TR_VTK_POINT = 0, TR_VTK_CELL = 1 };
enum { TR_VTK_SCALAR = 0, TR_VTK_VECTOR = 1, TR_VTK_TENSOR = 2 };
typedef struct tr_vtk_field {
    const char *name;
    int32_t location;          /* TR_VTK_POINT or TR_VTK_CELL */
    int32_t kind;              /* TR_VTK_SCALAR (1), VECTOR (3), TENSOR (6)  */
    const double *data;        /* host, component-major                     */
} tr_vtk_field;
tr_status tr_vtk_write(const char *path, const tr_meshdata *md, int real_bytes, int nfields,
                       const tr_vtk_field *fields);

#ifdef __cplusplus
}
#endif
#endif /* TRANSFER_B200_H */
