/*
 * sweep_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the discrete-ordinates transport sweep that the
 * CUDA product implements (transfer_b200/csrc/sweep.cu), used by tests/ as
 * its parity checker and by the benchmark as its timed CPU leg.  Nothing in
 * the product links or calls this code.
 *
 * The reference (uranix/Transfer) has no sweep: its solver is the
 * even-parity spherical-harmonics operator of kernels.cu.  The sweep works on
 * the reference's own problem data -- the `tetrahedron` records of
 * MeshData.cpp:56-76 (outward face area normals s[4][3], kappa_volume =
 * sigma_t V, I_p = B) and the boundary `face` records -- so its parity is
 * "unpinned" (no reference output exists); it is pinned instead by the
 * analytic E_2 solution of a purely absorbing slab and by the discrete
 * energy balance (tests/test_sweep_oracle.py).
 *
 * Discretisation (stated once; the CUDA kernels follow it step for step):
 * per tetrahedron K and ordinate Omega, psi is linear (values psi_j at the 4
 * vertices, discontinuous between cells) and satisfies for every test
 * function lambda_i
 *   int_K (Omega.grad psi) lambda_i + sigma_t int_K psi lambda_i
 *     + sum_{inflow faces f} |Omega.n_f| int_f (psi - psi_up) lambda_i
 *     = int_K Q lambda_i,            Q = sigma_s J + sigma_a B,
 * i.e. with a_k = -Omega.s_k (> 0 on inflow faces k) the 4x4 system
 *   L_ij = -(Omega.s_j)/12 + sigma_t V (1+d_ij)/20
 *          + (1+d_ij)/12 * sum_{k inflow, k != i, k != j} a_k
 *   rhs_i = (sigma_s V/20) (J_i + sum_j J_j) + sigma_a V B / 4
 *          + sum_{k inflow, k != i} a_k/12 (T_k + psi_up_{k,i}),
 *   T_k = sum_{j != k} psi_up_{k,j},
 * solved by Gaussian elimination without pivoting (the symmetric part of L
 * is positive definite).  J = sum_q w_q psi_q with sum_q w_q = 1.
 *
 * Schedule per ordinate: Kahn levels over the upwind graph (a cell is ready
 * when all its interior inflow neighbours are done); if a level comes out
 * empty while cells remain, the smallest-index remaining cell forms the next
 * level alone and its inflow from unfinished cells is "lagged" (read from
 * the extra-unknown vector B).  Lag slots are numbered in (q, cell, face)
 * order.  B = [reflective inflow: one entry of 4 values per (reflective
 * face, incoming ordinate), in (face, ordinate) order][lag: n_lag x 4].
 */
#ifndef SWEEP_ORACLE_H
#define SWEEP_ORACLE_H
#include <stdint.h>

#include "transfer_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_sweep_mesh {
    uint32_t nT, nF;
    const or_tet *mesh;               /* [nT] */
    const or_face *bnd;               /* [nF] */
    const double *kappa_abs_volume;   /* [nT] sigma_a V, NULL: sigma_a = sigma_t */
    const int32_t *face_bc;           /* [nF] 0 vacuum 1 reflective 2 incident, NULL: vacuum */
    const double *face_incident;      /* [nF] isotropic inflow intensity */
} or_sweep_mesh;

typedef struct or_sweep or_sweep;

/* Returns NULL (and sets *err to a message) on an unmatched boundary face
 * or a reflective face whose mirrored ordinates are not in the set. */
or_sweep *oracle_sweep_create(const or_sweep_mesh *m, uint32_t nq, const double *ox, const double *oy,
                              const double *oz, const double *w, const char **err);
void oracle_sweep_destroy(or_sweep *s);
/* info[0] length of B, [1] reflective faces, [2] lag slots, [3] max levels,
 * [4] forced (cycle-breaking) levels, [5] interior faces */
void oracle_sweep_info(const or_sweep *s, int64_t info[6]);
/* level[q * nT + c] */
void oracle_sweep_levels(const or_sweep *s, int32_t *level);
/* One sweep of all ordinates: J_in [nT][4] and B_in (NULL = 0); with_ext
 * adds emission and incident inflow.  Outputs (any may be NULL): J_out
 * [nT][4], B_out [len B], psi [nq][nT][4]. */
void oracle_sweep_apply(const or_sweep *s, const double *J_in, const double *B_in, int with_ext,
                        double *J_out, double *B_out, double *psi);
/* method 0: source iteration x <- S(x); 1: GMRES(restart) on (I - T) x = S(0).
 * Stops when the relative change (0) or relative residual (1) < tol.
 * J [nT][4], B [len B] outputs.  Returns 0 when converged. */
int oracle_sweep_solve(const or_sweep *s, int method, double tol, int max_iter, int restart, double *J,
                       double *B, int *iterations, double *residual);
/* Energy balance of one sweep (with_ext = 1) given its inputs J_in, B_in
 * (NULL = 0) and its output psi; for ANY such sweep
 *   emitted + incoming = absorbed + escaped + reflective_net
 * holds to rounding, and at convergence absorbed = sum sigma_a V mean(J).
 * out[0] emitted        sum sigma_a V B
 * out[1] absorbed       sum (sigma_t V mean(J_out) - sigma_s V mean(J_in))
 * out[2] escaped        sum over vacuum/incident faces of w (Omega.s) mean_f psi
 * out[3] incoming       sum over incident faces of w |Omega.s| I_inc
 * out[4] reflective_net outflow minus inflow (B_in) through reflective faces
 * (mean over the sphere, i.e. in units of the mean intensity x area). */
void oracle_sweep_balance(const or_sweep *s, const double *J_in, const double *B_in, const double *psi,
                          double out[5]);
/* moments m < nmom (nmom <= 16: l <= 3, order l^2 + l + m):
 * mom[m][nT*4] = sum_q w_q Y_m(Omega_q) psi_q, Y orthonormal on average
 * (Y_00 = 1). */
void oracle_sweep_moments(const or_sweep *s, const double *psi, int nmom, double *mom);

/* Outflow through the boundary faces with face_mask[f] != 0:
 * sum_q w_q sum_f max(Omega_q.s_f, 0) mean_f psi_q. */
double oracle_sweep_outflow(const or_sweep *s, const double *psi, const int32_t *face_mask);

/* Product ordinate set: Gauss-Legendre in mu (n_polar) x uniform azimuth
 * (n_azim, phi_k = (k + 1/2) 2 pi / n_azim), weights summing to 1. */
void oracle_ordinates_product(int n_polar, int n_azim, double *x, double *y, double *z, double *w);

#ifdef __cplusplus
}
#endif
#endif
