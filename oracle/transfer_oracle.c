/*
 * transfer_oracle.c -- TEST INFRASTRUCTURE ONLY (see transfer_oracle.h).
 *
 * FP64 CPU restatement of the reference path, used by tests/, the smoke
 * check and the benchmark's CPU baseline.  Never linked into the product.
 * OpenMP over vertices; every per-vertex sum runs in the reference order,
 * so results do not depend on the thread count.
 */
#include "transfer_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_ASLM_MAX 128

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void oracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ======================================================================
 * Angular tables.  Independent restatement of AngularData.cpp:9-67: the
 * same averages, evaluated with theta/phi associated Legendre functions
 * and product rules (Gauss in cos(theta) x trapezoid in phi) chosen with
 * a margin above exactness, instead of Lebedev/HemiQuad points.
 * ==================================================================== */
int oracle_slm(int maxk) { return (1 + maxk) * (1 + 2 * maxk); }

/* Associated Legendre P_l^m(x) without Condon-Shortley phase, standard
 * upward recurrence in l (Spherical.cpp builds the same function from
 * derivative polynomials). */
static double assoc_legendre(int l, int m, double x) {
    double somx2 = sqrt((1.0 - x) * (1.0 + x));
    double pmm = 1.0, fact = 1.0;
    for (int i = 1; i <= m; i++) {
        pmm *= fact * somx2;
        fact += 2.0;
    }
    if (l == m) return pmm;
    double pmmp1 = x * (2.0 * m + 1.0) * pmm;
    if (l == m + 1) return pmmp1;
    double pll = 0.0;
    for (int ll = m + 2; ll <= l; ll++) {
        pll = (x * (2.0 * ll - 1.0) * pmmp1 - (ll + m - 1.0) * pmm) / (ll - m);
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}

double oracle_ylm(int l, int m, double x, double y, double z) {
    /* Spherical::value(l,m,x,y,z) = value(l,m,acos z, atan2(y,x)) */
    double theta = acos(z > 1.0 ? 1.0 : (z < -1.0 ? -1.0 : z));
    double phi = atan2(y, x);
    int am = m < 0 ? -m : m;
    double c = (2.0 * l + 1.0) * (am == 0 ? 1.0 : 2.0);
    for (int k = l - am + 1; k <= l + am; k++) c /= k;
    c = sqrt(c);
    double trig = (m < 0) ? sin(am * phi) : cos(am * phi);
    return c * trig * assoc_legendre(l, am, cos(theta));
}

static void gauss01_rule(int n, double *x, double *w) {
    /* Gauss-Legendre on [-1,1] by Newton, mapped later by callers */
    for (int i = 0; i < n; i++) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 1.0;
        for (int it = 0; it < 200; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-16) break;
        }
        double p1 = 1.0, p2 = 0.0;
        for (int j = 1; j <= n; j++) {
            double p3 = p2;
            p2 = p1;
            p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1.0);
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

void oracle_angular(int maxk, double *omega, uint32_t *omega_pos,
                    double *Ox, double *Oy, double *Oz) {
    int n = oracle_slm(maxk), L = 2 * maxk;
    int *ls = malloc(sizeof(int) * n), *ms = malloc(sizeof(int) * n);
    for (int l = 0, k = 0; l <= L; l += 2)
        for (int m = -l; m <= l; m++, k++) {
            ls[k] = l;
            ms[k] = m;
        }
    /* full sphere: degree 4maxk+2 integrands; use a margin */
    int nz = 2 * maxk + 4, nphi = 4 * maxk + 8, np = nz * nphi;
    double *gx = malloc(sizeof(double) * nz), *gw = malloc(sizeof(double) * nz);
    gauss01_rule(nz, gx, gw);
    double *P = malloc(sizeof(double) * np * 4);
    double *Y = malloc(sizeof(double) * (size_t)n * np);
    for (int a = 0; a < nz; a++)
        for (int b = 0; b < nphi; b++) {
            int p = a * nphi + b;
            double phi = 2.0 * M_PI * (b + 0.5) / nphi, z = gx[a], r = sqrt(1.0 - z * z);
            P[4 * p + 0] = r * cos(phi);
            P[4 * p + 1] = r * sin(phi);
            P[4 * p + 2] = z;
            P[4 * p + 3] = 0.5 * gw[a] / nphi;
        }
    for (int k = 0; k < n; k++)
        for (int p = 0; p < np; p++)
            Y[(size_t)k * np + p] = oracle_ylm(ls[k], ms[k], P[4 * p], P[4 * p + 1], P[4 * p + 2]);
    for (int i = 0; i < 3; i++)
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) {
                for (int j = 0; j < 3; j++) {
                    double s = 0.0;
                    for (int p = 0; p < np; p++)
                        s += P[4 * p + 3] * Y[(size_t)a * np + p] * Y[(size_t)b * np + p] *
                             P[4 * p + i] * P[4 * p + j];
                    if (fabs(s) > 1e-10 || j == 2) {
                        omega[(i * n + a) * n + b] = s;
                        omega_pos[(i * n + a) * n + b] = (uint32_t)j;
                        break;
                    }
                }
            }
    /* half range: <|Omega_n| Y Y> = int_0^1 dmu <mu Y Y>_phi  (even integrand) */
    int hz = 2 * maxk + 4, hphi = 4 * maxk + 8, hp = hz * hphi;
    double *hx = malloc(sizeof(double) * hz), *hw = malloc(sizeof(double) * hz);
    gauss01_rule(hz, hx, hw);
    double *H = malloc(sizeof(double) * hp * 4);
    for (int a = 0; a < hz; a++)
        for (int b = 0; b < hphi; b++) {
            int p = a * hphi + b;
            double mu = 0.5 * (hx[a] + 1.0), r = sqrt(1.0 - mu * mu);
            double phi = 2.0 * M_PI * (b + 0.25) / hphi;
            H[4 * p + 0] = mu;
            H[4 * p + 1] = r * cos(phi);
            H[4 * p + 2] = r * sin(phi);
            H[4 * p + 3] = 0.5 * hw[a] / hphi * mu;
        }
    double *YH = malloc(sizeof(double) * (size_t)n * hp * 3);
    for (int k = 0; k < n; k++)
        for (int p = 0; p < hp; p++) {
            double mu = H[4 * p], u = H[4 * p + 1], v = H[4 * p + 2];
            YH[((size_t)k * hp + p) * 3 + 0] = oracle_ylm(ls[k], ms[k], mu, u, v); /* axis x */
            YH[((size_t)k * hp + p) * 3 + 1] = oracle_ylm(ls[k], ms[k], v, mu, u); /* axis y */
            YH[((size_t)k * hp + p) * 3 + 2] = oracle_ylm(ls[k], ms[k], u, v, mu); /* axis z */
        }
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++) {
            double s[3] = {0, 0, 0};
            for (int p = 0; p < hp; p++)
                for (int c = 0; c < 3; c++)
                    s[c] += H[4 * p + 3] * YH[((size_t)a * hp + p) * 3 + c] * YH[((size_t)b * hp + p) * 3 + c];
            Ox[a * n + b] = s[0];
            Oy[a * n + b] = s[1];
            Oz[a * n + b] = s[2];
        }
    free(ls); free(ms); free(gx); free(gw); free(P); free(Y);
    free(hx); free(hw); free(H); free(YH);
}

void oracle_align_angular(uint32_t slm, uint32_t aslm, const double *omega,
                          const uint32_t *omega_pos, const double *Ox,
                          const double *Oy, const double *Oz, double *aomega,
                          uint32_t *aomega_pos, double *aOx, double *aOy, double *aOz) {
    /* DeviceAngularData.cpp:25-56 */
    for (uint32_t i = 0; i < aslm; i++)
        for (uint32_t j = 0; j < aslm; j++) {
            int in = (i < slm && j < slm);
            for (int c = 0; c < 3; c++) {
                aomega[c * aslm * aslm + i * aslm + j] = in ? omega[c * slm * slm + i * slm + j] : 0.0;
                aomega_pos[c * aslm * aslm + i * aslm + j] = in ? omega_pos[c * slm * slm + i * slm + j] : 0u;
            }
            aOx[i * aslm + j] = in ? Ox[i * slm + j] : 0.0;
            aOy[i * aslm + j] = in ? Oy[i * slm + j] : 0.0;
            aOz[i * aslm + j] = in ? Oz[i * slm + j] : 0.0;
        }
}

/* ======================================================================
 * Kernels (kernels.cu).  One vertex per iteration of the parallel loop,
 * all harmonics lm < aslm of that vertex in the inner loops.
 * ==================================================================== */
static inline double mass_coef(const or_mesh *m, uint32_t t, uint32_t lm) {
    if (lm == 0 && m->kappa_abs_volume) return m->kappa_abs_volume[t];
    return m->mesh[t].kappa_volume;
}

/* kernels.cu:200-287 */
void oracle_volume_part(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    const uint32_t aslm = a->aslm, slm = a->slm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        double sums[9 * OR_ASLM_MAX];
        double sum[OR_ASLM_MAX];
        for (uint32_t lm = 0; lm < aslm; lm++) {
            sum[lm] = 0.0;
            for (int q = 0; q < 9; q++) sums[q * aslm + lm] = 0.0;
        }
        for (uint32_t j = m->tetstart[v]; j < m->tetstart[v + 1]; j++) {
            uint32_t t = m->tetidx[j], local = m->tetpos[j];
            const or_tet *tet = &m->mesh[t];
            for (uint32_t lm = 0; lm < aslm; lm++) {
                double fl[4], fsum = 0.0, sum_i[3];
                for (int s = 0; s < 4; s++) {
                    double tmp = f[(size_t)aslm * tet->p[s] + lm];
                    fl[s] = tmp;
                    fsum += tmp;
                }
                sum[lm] += mass_coef(m, t, lm) * (fl[local] + fsum) * (1.0 / 20.0);
                for (int si = 0; si < 3; si++)
                    sum_i[si] = tet->s[local][si] / tet->kappa_volume * (1.0 / 9.0);
                for (int si = 0; si < 3; si++)
                    for (int sj = 0; sj < 3; sj++)
                        for (int k = 0; k < 4; k++)
                            sums[(3 * si + sj) * aslm + lm] += sum_i[si] * fl[k] * tet->s[k][sj];
            }
        }
        for (uint32_t lm = 0; lm < aslm; lm++) {
            double rowsum = 0.0;
            for (int i = 0; i < 3; i++)
                for (uint32_t lms = 0; lms < slm; lms++) {
                    size_t q = (size_t)i * aslm * aslm + (size_t)lms * aslm + lm;
                    rowsum += a->omega[q] * sums[(3 * i + a->omega_pos[q]) * aslm + lms];
                }
            r[(size_t)aslm * v + lm] = sum[lm] + rowsum;
        }
    }
}

/* kernels.cu:290-357 */
void oracle_volume_part_diag(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    const uint32_t aslm = a->aslm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        for (uint32_t lm = 0; lm < aslm; lm++) {
            double sum = 0.0, sd[3] = {0, 0, 0};
            for (uint32_t j = m->tetstart[v]; j < m->tetstart[v + 1]; j++) {
                uint32_t t = m->tetidx[j], local = m->tetpos[j];
                const or_tet *tet = &m->mesh[t];
                double fl[4], fsum = 0.0, sum_i[3];
                for (int s = 0; s < 4; s++) {
                    double tmp = f[(size_t)aslm * tet->p[s] + lm];
                    fl[s] = tmp;
                    fsum += tmp;
                }
                sum += mass_coef(m, t, lm) * (fl[local] + fsum) * (1.0 / 20.0);
                for (int si = 0; si < 3; si++)
                    sum_i[si] = tet->s[local][si] / tet->kappa_volume * (1.0 / 9.0);
                for (int si = 0; si < 3; si++)
                    for (int k = 0; k < 4; k++) sd[si] += sum_i[si] * fl[k] * tet->s[k][si];
            }
            double rowsum = 0.0;
            size_t q = (size_t)lm + (size_t)lm * aslm;
            rowsum += a->omega[q] * sd[0];
            q += (size_t)aslm * aslm;
            rowsum += a->omega[q] * sd[1];
            q += (size_t)aslm * aslm;
            rowsum += a->omega[q] * sd[2];
            r[(size_t)aslm * v + lm] = sum + rowsum;
        }
    }
}

/* dominant-axis choice of the half-range table (kernels.cu:419-425) */
static inline const double *face_table(const or_ang *a, const or_face *tr, double *surf) {
    double s = fabs(tr->s[0] + tr->s[1] + tr->s[2]);
    *surf = s;
    if (2 * fabs(tr->s[0]) > s) return a->Ox;
    if (2 * fabs(tr->s[1]) > s) return a->Oy;
    return a->Oz;
}

/* kernels.cu:383-438 (accumulates into r) */
void oracle_surface_part(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    const uint32_t aslm = a->aslm, slm = a->slm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        double sum[OR_ASLM_MAX];
        double fv[4 * OR_ASLM_MAX];
        for (uint32_t lm = 0; lm < aslm; lm++) sum[lm] = 0.0;
        for (uint32_t j = m->facestart[v]; j < m->facestart[v + 1]; j++) {
            uint32_t fi = m->faceidx[j], local = m->facepos[j];
            if (m->face_bc && m->face_bc[fi] == 1) continue; /* reflective */
            const or_face *tr = &m->bnd[fi];
            double surf;
            const double *On = face_table(a, tr, &surf);
            for (uint32_t lm = 0; lm < aslm; lm++) {
                fv[3 * aslm + lm] = 0.0;
                for (int s = 0; s < 3; s++) {
                    double tmp = f[(size_t)aslm * tr->p[s] + lm];
                    fv[s * aslm + lm] = tmp;
                    fv[3 * aslm + lm] += tmp;
                }
            }
            for (uint32_t lm = 0; lm < aslm; lm++)
                for (uint32_t lms = 0; lms < slm; lms++)
                    sum[lm] += surf * On[aslm * lms + lm] * (fv[local * aslm + lms] + fv[3 * aslm + lms]) *
                               (1.0 / 12.0);
        }
        for (uint32_t lm = 0; lm < aslm; lm++) r[(size_t)aslm * v + lm] += sum[lm];
    }
}

/* kernels.cu:440-493 (accumulates into r) */
void oracle_surface_part_diag(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    const uint32_t aslm = a->aslm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        for (uint32_t lm = 0; lm < aslm; lm++) {
            double sum = 0.0;
            for (uint32_t j = m->facestart[v]; j < m->facestart[v + 1]; j++) {
                uint32_t fi = m->faceidx[j], local = m->facepos[j];
                if (m->face_bc && m->face_bc[fi] == 1) continue;
                const or_face *tr = &m->bnd[fi];
                double surf, fv[4];
                const double *On = face_table(a, tr, &surf);
                fv[3] = 0.0;
                for (int s = 0; s < 3; s++) {
                    double tmp = f[(size_t)aslm * tr->p[s] + lm];
                    fv[s] = tmp;
                    fv[3] += tmp;
                }
                sum += surf * On[aslm * lm + lm] * (fv[local] + fv[3]) * (1.0 / 12.0);
            }
            r[(size_t)aslm * v + lm] += sum;
        }
    }
}

/* kernels.cu:135-165; inflow faces add I (A/3) <|Omega_n| Y_lm>. */
void oracle_rhs(const or_mesh *m, const or_ang *a, double *b) {
    const uint32_t aslm = a->aslm, slm = a->slm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        double sum = 0.0;
        for (uint32_t j = m->tetstart[v]; j < m->tetstart[v + 1]; j++) {
            const or_tet *tet = &m->mesh[m->tetidx[j]];
            sum += tet->kappa_volume * tet->I_p * (1.0 / 4.0);
        }
        for (uint32_t lm = 0; lm < aslm; lm++) b[(size_t)aslm * v + lm] = (lm == 0) ? sum : 0.0;
        if (m->face_bc && m->face_incident) {
            for (uint32_t j = m->facestart[v]; j < m->facestart[v + 1]; j++) {
                uint32_t fi = m->faceidx[j];
                if (m->face_bc[fi] != 2) continue;
                double surf;
                const double *On = face_table(a, &m->bnd[fi], &surf);
                for (uint32_t lm = 0; lm < slm; lm++)
                    b[(size_t)aslm * v + lm] += m->face_incident[fi] * surf * (1.0 / 3.0) * On[lm];
            }
        }
    }
}

/* CudaContext::computeLhs (CudaContext.cpp:108-120): volumePart then
 * surfacePart accumulating into the same vector. */
void oracle_compute_lhs(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    oracle_volume_part(m, a, f, r);
    oracle_surface_part(m, a, f, r);
}
void oracle_compute_lhs_diag(const or_mesh *m, const or_ang *a, const double *f, double *r) {
    oracle_volume_part_diag(m, a, f, r);
    oracle_surface_part_diag(m, a, f, r);
}

/* ---------------------------------------------------- BLAS (kernels.cu:12-50) */
void oracle_scale(uint64_t n, double *x, double wx) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) x[i] *= wx;
}
void oracle_add_prod(uint64_t n, double *x, const double *y, double wy) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) x[i] += wy * y[i];
}
void oracle_mul_add(uint64_t n, double *x, double wx, const double *y) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) x[i] = wx * x[i] + y[i];
}
void oracle_mul_add_prod(uint64_t n, double *x, double wx, const double *y, double wy) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) x[i] = wx * x[i] + wy * y[i];
}

/* kernels.cu:55-115: per-lm serial sums over vertices, then a fixed
 * 128-wide tree. */
static double tree128(double *red) {
    for (int s = 64; s >= 1; s >>= 1)
        for (int lm = 0; lm < s; lm++) red[lm] += red[lm + s];
    return red[0];
}
double oracle_norm(uint32_t nP, uint32_t aslm, uint32_t slm, const double *x) {
    double red[OR_ASLM_MAX];
    for (int i = 0; i < OR_ASLM_MAX; i++) red[i] = 0.0;
#pragma omp parallel for schedule(static)
    for (int lm = 0; lm < (int)slm; lm++) {
        double acc = 0.0;
        for (uint64_t i = (uint64_t)lm; i < (uint64_t)nP * aslm; i += aslm) acc += x[i] * x[i];
        red[lm] = acc;
    }
    return sqrt(tree128(red));
}
double oracle_dot(uint32_t nP, uint32_t aslm, uint32_t slm, const double *x, const double *y) {
    double red[OR_ASLM_MAX];
    for (int i = 0; i < OR_ASLM_MAX; i++) red[i] = 0.0;
#pragma omp parallel for schedule(static)
    for (int lm = 0; lm < (int)slm; lm++) {
        double acc = 0.0;
        for (uint64_t i = (uint64_t)lm; i < (uint64_t)nP * aslm; i += aslm) acc += x[i] * y[i];
        red[lm] = acc;
    }
    return tree128(red);
}

/* ================================================================ solver */
/* diagonal of A, for the Jacobi extension */
static void oracle_diagonal(const or_mesh *m, const or_ang *a, double *d) {
    const uint32_t aslm = a->aslm, slm = a->slm;
#pragma omp parallel for schedule(static)
    for (long vv = 0; vv < (long)m->nP; vv++) {
        uint32_t v = (uint32_t)vv;
        for (uint32_t lm = 0; lm < aslm; lm++) {
            double acc = 0.0;
            if (lm < slm) {
                for (uint32_t j = m->tetstart[v]; j < m->tetstart[v + 1]; j++) {
                    uint32_t t = m->tetidx[j], loc = m->tetpos[j];
                    const or_tet *tet = &m->mesh[t];
                    acc += mass_coef(m, t, lm) * 2.0 / 20.0;
                    for (int i = 0; i < 3; i++) {
                        size_t q = (size_t)i * aslm * aslm + (size_t)lm * aslm + lm;
                        uint32_t jj = a->omega_pos[q];
                        acc += a->omega[q] * tet->s[loc][i] / tet->kappa_volume / 9.0 * tet->s[loc][jj];
                    }
                }
                for (uint32_t j = m->facestart[v]; j < m->facestart[v + 1]; j++) {
                    uint32_t fi = m->faceidx[j];
                    if (m->face_bc && m->face_bc[fi] == 1) continue;
                    double surf;
                    const double *On = face_table(a, &m->bnd[fi], &surf);
                    acc += surf * On[aslm * lm + lm] * 2.0 / 12.0;
                }
            }
            d[(size_t)aslm * v + lm] = (lm < slm && acc != 0.0) ? 1.0 / acc : 0.0;
        }
    }
}

/* main.cpp:223-248 */
static int oracle_invprec(const or_mesh *m, const or_ang *a, const or_cg_opts *o,
                          double *f, const double *b, double *Ap, double *p, double *r) {
    uint64_t N = (uint64_t)m->nP * a->aslm;
    double itol = o->inner_tol > 0 ? o->inner_tol : 1e-8;
    int imax = o->inner_max_iter > 0 ? o->inner_max_iter : 1000;
    oracle_mul_add_prod(N, f, 0.0, b, 0.0);
    oracle_compute_lhs_diag(m, a, f, Ap);
    oracle_mul_add(N, r, 0.0, b);
    oracle_add_prod(N, r, Ap, -1.0);
    oracle_mul_add(N, p, 0.0, r);
    int k = 0;
    double nrz = oracle_norm(m->nP, a->aslm, a->slm, r);
    nrz *= nrz;
    while (k < imax) {
        oracle_compute_lhs_diag(m, a, p, Ap);
        double alpha = nrz / oracle_dot(m->nP, a->aslm, a->slm, p, Ap);
        oracle_add_prod(N, f, p, alpha);
        oracle_add_prod(N, r, Ap, -alpha);
        double nr = oracle_norm(m->nP, a->aslm, a->slm, r);
        if (nr < itol) break;
        double nrz2 = nr * nr;
        double beta = nrz2 / nrz;
        nrz = nrz2;
        oracle_mul_add(N, p, beta, r);
        k++;
    }
    return k;
}

/* main.cpp:125-160 */
int oracle_cg(const or_mesh *m, const or_ang *a, const or_cg_opts *o,
              const double *bin, double *f, or_cg_result *res) {
    uint64_t N = (uint64_t)m->nP * a->aslm;
    double *b = calloc(N, sizeof(double)), *p = calloc(N, sizeof(double));
    double *Ap = calloc(N, sizeof(double)), *z = calloc(N, sizeof(double));
    double *r = calloc(N, sizeof(double)), *pp = calloc(N, sizeof(double));
    double *pAp = calloc(N, sizeof(double)), *pr = calloc(N, sizeof(double));
    double *dinv = NULL;
    if (!b || !p || !Ap || !z || !r || !pp || !pAp || !pr) return -1;
    if (o->precondition == 2) {
        dinv = calloc(N, sizeof(double));
        oracle_diagonal(m, a, dinv);
    }
    memset(f, 0, N * sizeof(double));
    if (bin) memcpy(b, bin, N * sizeof(double));
    else oracle_rhs(m, a, b);
    double bnorm = oracle_norm(m->nP, a->aslm, a->slm, b);
    double tol = o->relative ? o->tol * bnorm : o->tol;
    int maxit = o->max_iter > 0 ? o->max_iter : 1000;
    int inner = 0;
    oracle_compute_lhs(m, a, f, Ap);
    oracle_mul_add(N, r, 0.0, b);
    oracle_add_prod(N, r, Ap, -1.0);
    if (o->precondition == 1) inner += oracle_invprec(m, a, o, z, r, pAp, pp, pr);
    else if (o->precondition == 2) for (uint64_t i = 0; i < N; i++) z[i] = dinv[i] * r[i];
    else oracle_mul_add(N, z, 0.0, r);
    oracle_mul_add(N, p, 0.0, z);
    int k = 0, conv = 0;
    double nrz = oracle_dot(m->nP, a->aslm, a->slm, r, z), nr = 0.0;
    while (k < maxit) {
        oracle_compute_lhs(m, a, p, Ap);
        double alpha = nrz / oracle_dot(m->nP, a->aslm, a->slm, p, Ap);
        oracle_add_prod(N, f, p, alpha);
        oracle_add_prod(N, r, Ap, -alpha);
        nr = oracle_norm(m->nP, a->aslm, a->slm, r);
        if (o->history && k < o->history_len) o->history[k] = nr;
        if (nr < tol) {
            conv = 1;
            break;
        }
        if (o->precondition == 1) inner += oracle_invprec(m, a, o, z, r, pAp, pp, pr);
        else if (o->precondition == 2) for (uint64_t i = 0; i < N; i++) z[i] = dinv[i] * r[i];
        else oracle_mul_add(N, z, 0.0, r);
        double nrz2 = oracle_dot(m->nP, a->aslm, a->slm, z, r);
        double beta = nrz2 / nrz;
        nrz = nrz2;
        oracle_mul_add(N, p, beta, z);
        k++;
    }
    if (res) {
        res->iterations = conv ? k + 1 : k;
        res->inner_iterations = inner;
        res->converged = conv;
        res->final_residual = nr;
        res->rhs_norm = bnorm;
    }
    free(b); free(p); free(Ap); free(z); free(r); free(pp); free(pAp); free(pr); free(dinv);
    return 0;
}

/* ====================================================== moments / flux */
/* MeshData.cpp:96-116, with I[lm][k] = f[k*aslm + lm] (main.cpp:166-172) */
void oracle_compute_moments(uint32_t nP, uint32_t slm, uint32_t aslm, const double *omega,
                            const uint32_t *omega_pos, const double *f, double *U, double *T) {
    const double fourpi = 12.5663706143591729538505735331;
#pragma omp parallel for schedule(static)
    for (long kk = 0; kk < (long)nP; kk++) {
        size_t k = (size_t)kk;
        U[k] = fourpi * f[k * aslm + 0];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) T[(size_t)(3 * i + j) * nP + k] = 0.0;
        for (uint32_t lm = 0; lm < slm; lm++)
            for (int i = 0; i < 3; i++) {
                uint32_t j = omega_pos[(size_t)i * slm * slm + (size_t)lm * slm];
                double v = omega[(size_t)i * slm * slm + (size_t)lm * slm];
                T[(size_t)(3 * i + j) * nP + k] += fourpi * v * f[k * aslm + lm];
            }
    }
}

/* MeshData.cpp:118-136 */
void oracle_compute_flux(const or_mesh *m, const double *T, double *W) {
    const size_t nP = m->nP;
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < (long)m->nT; ii++) {
        const or_tet *t = &m->mesh[ii];
        for (int j = 0; j < 3; j++) {
            double w = 0.0;
            for (int k = 0; k < 4; k++)
                for (int a = 0; a < 3; a++) w += t->s[k][a] * T[(size_t)(3 * a + j) * nP + t->p[k]];
            W[(size_t)j * m->nT + ii] = (1.0 / 3.0) * w / t->kappa_volume;
        }
    }
}

/* ============================================================ Lanczos */
/* Eigenvalue.cpp:5-51 (uround() of double: 2^-53 -> threshold 100 u) */
double oracle_trieig(const double *a, const double *b, uint32_t N) {
    if (N == 1) return a[0];
    if (N == 2) {
        double ap = 0.5 * (a[0] + a[1]), am = 0.5 * (a[0] - a[1]);
        return ap + sqrt(am * am + b[0] * b[0]);
    }
    double q, lmax = a[0] + fabs(b[0]);
    for (uint32_t i = 1; i < N - 1; i++) {
        q = a[i] + fabs(b[i]) + fabs(b[i - 1]);
        if (q > lmax) lmax = q;
    }
    q = a[N - 1] + fabs(b[N - 2]);
    if (q > lmax) lmax = q;
    int iters = 0;
    double dl = 1.0, u = 1.0;
    while (1.0 + u > 1.0) u *= 0.5;
    double th = 100.0 * u;
    while (iters < 100 && dl > th) {
        double x = lmax, Po = 1.0, P = a[0] - x, Qo = 0.0, Q = -1.0;
        for (uint32_t j = 1; j < N; j++) {
            double Qs = Q;
            Q = -P + (a[j] - x) * Q - b[j - 1] * b[j - 1] * Qo;
            Qo = Qs;
            double Ps = P;
            P = (a[j] - x) * P - b[j - 1] * b[j - 1] * Po;
            Po = Ps;
        }
        dl = P / Q;
        lmax -= dl;
        iters++;
    }
    return lmax;
}

/* Eigenvalue.cpp:53-83, including its indexing of the off-diagonal
 * (b[0] = 0 is passed as the first coupling). */
double oracle_eigest(const or_mesh *m, const or_ang *a, double *v, int max_steps,
                     double *extra, int *steps) {
    uint64_t N = (uint64_t)m->nP * a->aslm;
    int mm = max_steps > 0 ? max_steps : 30;
    double *aa = calloc(mm, sizeof(double)), *bb = calloc(mm + 1, sizeof(double));
    double *v0 = calloc(N, sizeof(double)), *w = calloc(N, sizeof(double));
    double *vv = v, *s;
    oracle_scale(N, vv, 1.0 / oracle_norm(m->nP, a->aslm, a->slm, vv));
    oracle_mul_add(N, v0, 0.0, vv);
    bb[0] = 0.0;
    double lmax = 0.0, lold = 0.0, loold = 0.0;
    int j;
    for (j = 0; j < mm; j++) {
        oracle_compute_lhs(m, a, vv, w);
        oracle_mul_add(N, v0, -bb[j], w);
        s = v0;
        v0 = vv;
        vv = s;
        aa[j] = oracle_dot(m->nP, a->aslm, a->slm, vv, v0);
        oracle_add_prod(N, vv, v0, -aa[j]);
        bb[j + 1] = oracle_norm(m->nP, a->aslm, a->slm, vv);
        oracle_scale(N, vv, 1.0 / bb[j + 1]);
        loold = lold;
        lold = lmax;
        lmax = oracle_trieig(aa, bb, (uint32_t)(j + 1));
        if (fabs(lmax - lold) < 1e-6 * lmax) {
            j++;
            break;
        }
    }
    double q = (lmax - lold) / (lold - loold);
    if (extra) *extra = lmax + (lmax - lold) / (1 - q);
    if (steps) *steps = j;
    /* v0 / vv may have been swapped; keep the caller's buffer valid */
    if (vv != v) memcpy(v, vv, N * sizeof(double));
    free(aa);
    free(bb);
    free(vv == v ? v0 : vv);
    free(w);
    return lmax;
}

/* ==================================================== E_n(x), x > 0
 * Series for x <= 1 and a modified-Lentz continued fraction otherwise
 * (the classical expansions of Abramowitz & Stegun 5.1.11 and 5.1.22). */
double oracle_expint_en(int n, double x) {
    const double euler = 0.57721566490153286061;
    if (n < 0 || x < 0.0) return NAN;
    if (n == 0) return exp(-x) / x;
    if (x == 0.0) return n > 1 ? 1.0 / (n - 1) : INFINITY;
    if (x > 1.0) {
        double b = x + n, c = 1.0 / 1e-300, d = 1.0 / b, h = d;
        for (int i = 1; i < 1000; i++) {
            double an = -(double)i * (n - 1 + i);
            b += 2.0;
            d = 1.0 / (an * d + b);
            c = b + an / c;
            double del = c * d;
            h *= del;
            if (fabs(del - 1.0) < 1e-16) break;
        }
        return h * exp(-x);
    }
    double ans = (n - 1) != 0 ? 1.0 / (n - 1) : -log(x) - euler, fact = 1.0;
    for (int i = 1; i < 1000; i++) {
        fact *= -x / i;
        double del;
        if (i != n - 1) del = -fact / (i - n + 1);
        else {
            double psi = -euler;
            for (int ii = 1; ii <= n - 1; ii++) psi += 1.0 / ii;
            del = fact * (-log(x) + psi);
        }
        ans += del;
        if (fabs(del) < fabs(ans) * 1e-17) break;
    }
    return ans;
}
