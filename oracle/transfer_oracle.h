/*
 * transfer_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the reference's radiative-transfer hot path, used
 * as the parity checker for the CUDA product (tests, smoke check, and the
 * timed CPU baseline of the benchmark).  Nothing in the product links or
 * calls this code.
 *
 * Each function cites the reference file:line it restates.  The kernels are
 * restated per vertex in the reference's own summation order (tets in CSR
 * order, then the lms loop, rows i = 0,1,2), with OpenMP over vertices.
 *
 * Data are the reference's device-side layouts: vectors f[vertex*aslm + lm],
 * angular tables padded to aslm exactly as DeviceAngularData.cpp:10-67 pads
 * them (omega[i][lms][lm] at omega[i*aslm*aslm + lms*aslm + lm]).
 */
#ifndef TRANSFER_ORACLE_H
#define TRANSFER_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_tet {            /* tetrahedron.h:7-20, REAL=double */
    uint32_t p[4];
    double kappa_volume, I_p;
    double s[4][3];
} or_tet;

typedef struct or_face {           /* face.h:8-18, REAL=double */
    uint32_t p[4];
    double s[3];
    double pad[3];
} or_face;

typedef struct or_mesh {           /* DeviceMeshDataRaw, MeshData.h:34-47 */
    uint32_t nP, nT, nF;
    const uint32_t *tetstart, *tetidx, *tetpos;
    const or_tet *mesh;
    const uint32_t *facestart, *faceidx, *facepos;
    const or_face *bnd;
    /* extensions (NULL = reference behaviour) */
    const double *kappa_abs_volume;   /* [nT] l=0 mass coefficient        */
    const int32_t *face_bc;           /* [nF] 0 vacuum 1 reflective 2 inflow */
    const double *face_incident;      /* [nF] isotropic inflow intensity   */
} or_mesh;

typedef struct or_ang {            /* DeviceAngularDataRaw, AngularData.h:20-28 */
    uint32_t slm, aslm;
    const double *omega;           /* [3][aslm][aslm] */
    const uint32_t *omega_pos;     /* [3][aslm][aslm] */
    const double *Ox, *Oy, *Oz;    /* [aslm][aslm]    */
} or_ang;

/* --- angular tables (independent restatement; AngularData.cpp:9-67) ---- */
int  oracle_slm(int maxk);
/* unpadded tables, stride slm (as the host AngularData stores them) */
void oracle_angular(int maxk, double *omega, uint32_t *omega_pos,
                    double *Ox, double *Oy, double *Oz);
/* pad unpadded tables to aslm (DeviceAngularData.cpp:10-67) */
void oracle_align_angular(uint32_t slm, uint32_t aslm,
                          const double *omega, const uint32_t *omega_pos,
                          const double *Ox, const double *Oy, const double *Oz,
                          double *aomega, uint32_t *aomega_pos,
                          double *aOx, double *aOy, double *aOz);
/* real spherical harmonic, orthonormal on average (Spherical.cpp:62-82) */
double oracle_ylm(int l, int m, double x, double y, double z);

/* --- kernels (kernels.cu) --------------------------------------------- */
void oracle_volume_part(const or_mesh *m, const or_ang *a, const double *f, double *r);       /* :200-287 */
void oracle_surface_part(const or_mesh *m, const or_ang *a, const double *f, double *r);      /* :383-438 */
void oracle_volume_part_diag(const or_mesh *m, const or_ang *a, const double *f, double *r);  /* :290-357 */
void oracle_surface_part_diag(const or_mesh *m, const or_ang *a, const double *f, double *r); /* :440-493 */
void oracle_rhs(const or_mesh *m, const or_ang *a, double *b);                                /* :135-165 */
/* CudaContext::computeLhs / computeLhsDiag (CudaContext.cpp:108-130) */
void oracle_compute_lhs(const or_mesh *m, const or_ang *a, const double *f, double *r);
void oracle_compute_lhs_diag(const or_mesh *m, const or_ang *a, const double *f, double *r);

/* BLAS-1 over n = nP*aslm entries (kernels.cu:12-50) */
void oracle_scale(uint64_t n, double *x, double wx);
void oracle_add_prod(uint64_t n, double *x, const double *y, double wy);
void oracle_mul_add(uint64_t n, double *x, double wx, const double *y);
void oracle_mul_add_prod(uint64_t n, double *x, double wx, const double *y, double wy);
/* reductions over lm < slm (kernels.cu:55-115) */
double oracle_norm(uint32_t nP, uint32_t aslm, uint32_t slm, const double *x);
double oracle_dot(uint32_t nP, uint32_t aslm, uint32_t slm, const double *x, const double *y);

/* --- solver (main.cpp:125-160, invprec main.cpp:223-248) --------------- */
typedef struct or_cg_opts {
    int precondition;      /* 0 none, 1 invprec (reference), 2 jacobi */
    int max_iter;          /* reference 1000 */
    int relative;          /* 0 absolute (reference) */
    double tol;            /* reference 1e-4 */
    double inner_tol;      /* invprec 1e-8 */
    int inner_max_iter;    /* invprec 1000 */
    int history_len;
    double *history;       /* ||r|| per iteration */
} or_cg_opts;
typedef struct or_cg_result {
    int iterations, inner_iterations, converged;
    double final_residual, rhs_norm;
} or_cg_result;
/* b: rhs (NULL -> oracle_rhs); f: output. Returns 0 on success. */
int oracle_cg(const or_mesh *m, const or_ang *a, const or_cg_opts *o,
              const double *b, double *f, or_cg_result *res);

/* --- moments / flux (MeshData.cpp:96-136) ------------------------------ */
/* omega/omega_pos UNPADDED (host AngularData); f padded [nP][aslm] */
void oracle_compute_moments(uint32_t nP, uint32_t slm, uint32_t aslm,
                            const double *omega, const uint32_t *omega_pos,
                            const double *f, double *U, double *T);
void oracle_compute_flux(const or_mesh *m, const double *T, double *W);

/* --- Lanczos (Eigenvalue.cpp:5-83) ------------------------------------- */
double oracle_trieig(const double *a, const double *b, uint32_t N);
/* v overwritten; returns lmax, *extra the extrapolated estimate */
double oracle_eigest(const or_mesh *m, const or_ang *a, double *v,
                     int max_steps, double *extra, int *steps);

/* --- exponential integrals (independent of E1.cpp, which mis-scales
 *     xE1 for x > 1) ------------------------------------------------------ */
double oracle_expint_en(int n, double x);   /* E_n(x), x > 0 */

int oracle_num_threads(void);
void oracle_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
