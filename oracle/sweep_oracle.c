/*
 * sweep_oracle.c -- TEST INFRASTRUCTURE ONLY (see sweep_oracle.h).
 *
 * FP64 CPU restatement of the linear-discontinuous discrete-ordinates sweep,
 * its Kahn-level schedule, source iteration / GMRES, energy balance and
 * angular moments.  OpenMP over ordinates; every sum over ordinates runs in
 * ordinate order, so results do not depend on the thread count.
 */
#include "sweep_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NONE 0xFFFFFFFFu

struct or_sweep {
    uint32_t nT, nF, nq;
    double *s;          /* [nT][4][3] consistent outward area normals */
    double *stv, *sav;  /* sigma_t V, sigma_a V */
    double *B;          /* emission intensity */
    int64_t *nbr;       /* [nT][4] >= 0 cell, < 0: -(face+1) */
    uint8_t *map;       /* [nT][4][4] local index in the neighbour of vertex j across face k */
    int32_t *bc;        /* [nF] */
    double *inc;        /* [nF] */
    int64_t *rslot;     /* [nF] reflective slot or -1 */
    uint32_t nrefl;
    uint32_t *rmap;     /* [nrefl][nq] mirrored ordinate of an incoming q (NONE if outgoing) */
    uint32_t *rent;     /* [nrefl][nq] B entry of an incoming q (NONE if outgoing) */
    uint32_t nent;      /* reflective B entries: (slot, incoming q) in that order */
    double *ox, *oy, *oz, *w;
    /* schedule */
    uint32_t *order;    /* [nq][nT] */
    int32_t *level;     /* [nq][nT] */
    uint32_t *lagbase;  /* [nq][nT][4] lag slot of (q,c,k) or NONE */
    uint32_t nlag;
    uint32_t *lag_qck;  /* [nlag][3] */
    int64_t maxlev, forced, ninterior;
};

/* ---- helpers ------------------------------------------------------------ */
typedef struct {
    uint32_t v[3];
    uint32_t cell, k;
} facekey;

static int cmp_facekey(const void *a, const void *b) {
    const facekey *x = (const facekey *)a, *y = (const facekey *)b;
    for (int i = 0; i < 3; i++)
        if (x->v[i] != y->v[i]) return x->v[i] < y->v[i] ? -1 : 1;
    if (x->cell != y->cell) return x->cell < y->cell ? -1 : 1;
    return (int)x->k - (int)y->k;
}

static void sort3(uint32_t *v) {
    uint32_t t;
    if (v[0] > v[1]) { t = v[0]; v[0] = v[1]; v[1] = t; }
    if (v[1] > v[2]) { t = v[1]; v[1] = v[2]; v[2] = t; }
    if (v[0] > v[1]) { t = v[0]; v[0] = v[1]; v[1] = t; }
}

void oracle_ordinates_product(int n_polar, int n_azim, double *x, double *y, double *z, double *w) {
    double *mu = (double *)malloc(sizeof(double) * n_polar), *wm = (double *)malloc(sizeof(double) * n_polar);
    for (int i = 0; i < n_polar; i++) { /* Gauss-Legendre by Newton */
        double t = cos(M_PI * (i + 0.75) / (n_polar + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = t;
            for (int l = 2; l <= n_polar; l++) {
                double p2 = ((2.0 * l - 1.0) * t * p1 - (l - 1.0) * p0) / l;
                p0 = p1;
                p1 = p2;
            }
            if (n_polar == 1) { p1 = t; p0 = 1.0; }
            dp = n_polar * (t * p1 - p0) / (t * t - 1.0);
            double dt = p1 / dp;
            t -= dt;
            if (fabs(dt) < 1e-16) break;
        }
        mu[i] = t;
        wm[i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
    int q = 0;
    for (int i = 0; i < n_polar; i++) {
        double st = sqrt(1.0 - mu[i] * mu[i]);
        for (int k = 0; k < n_azim; k++, q++) {
            double phi = (k + 0.5) * 2.0 * M_PI / n_azim;
            x[q] = st * cos(phi);
            y[q] = st * sin(phi);
            z[q] = mu[i];
            w[q] = 0.5 * wm[i] / n_azim;
        }
    }
    free(mu);
    free(wm);
}

static double det3(const double *a, const double *b, const double *c) {
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
           a[2] * (b[0] * c[1] - b[1] * c[0]);
}

/* ---- set-up --------------------------------------------------------------- */
static void build_schedule(or_sweep *S);

or_sweep *oracle_sweep_create(const or_sweep_mesh *m, uint32_t nq, const double *ox, const double *oy,
                              const double *oz, const double *w, const char **err) {
    static const char *e_bnd = "a tetrahedron face is neither shared nor a listed boundary face";
    static const char *e_refl = "a reflective face mirrors an ordinate onto a direction outside the set";
    static const char *e_vol = "degenerate tetrahedron (zero volume)";
    uint32_t nT = m->nT, nF = m->nF;
    or_sweep *S = (or_sweep *)calloc(1, sizeof(or_sweep));
    S->nT = nT;
    S->nF = nF;
    S->nq = nq;
    S->s = (double *)malloc(sizeof(double) * 12 * nT);
    S->stv = (double *)malloc(sizeof(double) * nT);
    S->sav = (double *)malloc(sizeof(double) * nT);
    S->B = (double *)malloc(sizeof(double) * nT);
    S->nbr = (int64_t *)malloc(sizeof(int64_t) * 4 * nT);
    S->map = (uint8_t *)calloc(16 * (size_t)nT, 1);
    S->bc = (int32_t *)calloc(nF + 1, sizeof(int32_t));
    S->inc = (double *)calloc(nF + 1, sizeof(double));
    S->rslot = (int64_t *)malloc(sizeof(int64_t) * (nF + 1));
    S->ox = (double *)malloc(sizeof(double) * nq);
    S->oy = (double *)malloc(sizeof(double) * nq);
    S->oz = (double *)malloc(sizeof(double) * nq);
    S->w = (double *)malloc(sizeof(double) * nq);
    memcpy(S->ox, ox, sizeof(double) * nq);
    memcpy(S->oy, oy, sizeof(double) * nq);
    memcpy(S->oz, oz, sizeof(double) * nq);
    memcpy(S->w, w, sizeof(double) * nq);
    for (uint32_t c = 0; c < nT; c++) {
        const or_tet *t = &m->mesh[c];
        memcpy(&S->s[12 * c], t->s, sizeof(double) * 12);
        S->stv[c] = t->kappa_volume;
        S->sav[c] = m->kappa_abs_volume ? m->kappa_abs_volume[c] : t->kappa_volume;
        S->B[c] = t->I_p;
        if (det3(t->s[1], t->s[2], t->s[3]) == 0.0) {
            *err = e_vol;
            oracle_sweep_destroy(S);
            return NULL;
        }
    }
    for (uint32_t f = 0; f < nF; f++) {
        S->bc[f] = m->face_bc ? m->face_bc[f] : 0;
        S->inc[f] = m->face_incident ? m->face_incident[f] : 0.0;
    }
    /* adjacency by sorted vertex triples; boundary faces matched likewise */
    size_t nk = 4 * (size_t)nT;
    facekey *keys = (facekey *)malloc(sizeof(facekey) * nk);
    for (uint32_t c = 0; c < nT; c++)
        for (uint32_t k = 0; k < 4; k++) {
            facekey *e = &keys[4 * c + k];
            int n = 0;
            for (int j = 0; j < 4; j++)
                if (j != (int)k) e->v[n++] = m->mesh[c].p[j];
            sort3(e->v);
            e->cell = c;
            e->k = k;
        }
    qsort(keys, nk, sizeof(facekey), cmp_facekey);
    facekey *bkeys = (facekey *)malloc(sizeof(facekey) * (nF + 1));
    for (uint32_t f = 0; f < nF; f++) {
        memcpy(bkeys[f].v, m->bnd[f].p, sizeof(uint32_t) * 3);
        sort3(bkeys[f].v);
        bkeys[f].cell = f;
        bkeys[f].k = 0;
    }
    qsort(bkeys, nF, sizeof(facekey), cmp_facekey);
    S->ninterior = 0;
    for (size_t i = 0; i < nk;) {
        if (i + 1 < nk && memcmp(keys[i].v, keys[i + 1].v, sizeof(uint32_t) * 3) == 0) {
            uint32_t a = keys[i].cell, ka = keys[i].k, b = keys[i + 1].cell, kb = keys[i + 1].k;
            S->nbr[4 * a + ka] = b;
            S->nbr[4 * b + kb] = a;
            /* the lower-index cell owns the face normal; the other uses its negation */
            for (int d = 0; d < 3; d++) S->s[12 * b + 3 * kb + d] = -S->s[12 * a + 3 * ka + d];
            for (int j = 0; j < 4; j++) {
                if (j == (int)ka) continue;
                for (int jj = 0; jj < 4; jj++)
                    if (m->mesh[b].p[jj] == m->mesh[a].p[j]) S->map[16 * a + 4 * ka + j] = (uint8_t)jj;
            }
            for (int j = 0; j < 4; j++) {
                if (j == (int)kb) continue;
                for (int jj = 0; jj < 4; jj++)
                    if (m->mesh[a].p[jj] == m->mesh[b].p[j]) S->map[16 * b + 4 * kb + j] = (uint8_t)jj;
            }
            S->ninterior++;
            i += 2;
        } else {
            /* binary search by vertices only */
            facekey *hit = NULL;
            size_t lo = 0, hi = nF;
            while (lo < hi) {
                size_t mid = (lo + hi) / 2;
                int cmp = 0;
                for (int d = 0; d < 3 && !cmp; d++)
                    cmp = bkeys[mid].v[d] < keys[i].v[d] ? -1 : (bkeys[mid].v[d] > keys[i].v[d] ? 1 : 0);
                if (cmp < 0) lo = mid + 1;
                else hi = mid;
            }
            if (lo < nF && bkeys[lo].v[0] == keys[i].v[0] && bkeys[lo].v[1] == keys[i].v[1] &&
                bkeys[lo].v[2] == keys[i].v[2])
                hit = &bkeys[lo];
            if (!hit) {
                free(keys);
                free(bkeys);
                *err = e_bnd;
                oracle_sweep_destroy(S);
                return NULL;
            }
            S->nbr[4 * keys[i].cell + keys[i].k] = -(int64_t)hit->cell - 1;
            i += 1;
        }
    }
    free(keys);
    free(bkeys);
    /* reflective faces: slots and mirrored ordinates */
    S->nrefl = 0;
    for (uint32_t f = 0; f < nF; f++) S->rslot[f] = (S->bc[f] == 1) ? (int64_t)S->nrefl++ : -1;
    S->rmap = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)S->nrefl * nq + 1));
    for (size_t i = 0; i < (size_t)S->nrefl * nq; i++) S->rmap[i] = NONE;
    for (uint32_t c = 0; c < nT; c++)
        for (int k = 0; k < 4; k++) {
            int64_t nb = S->nbr[4 * c + k];
            if (nb >= 0) continue;
            uint32_t f = (uint32_t)(-nb - 1);
            if (S->rslot[f] < 0) continue;
            const double *sk = &S->s[12 * c + 3 * k];
            double a = sqrt(sk[0] * sk[0] + sk[1] * sk[1] + sk[2] * sk[2]);
            double n[3] = {sk[0] / a, sk[1] / a, sk[2] / a};
            for (uint32_t q = 0; q < nq; q++) {
                double on = ox[q] * n[0] + oy[q] * n[1] + oz[q] * n[2];
                if (!(ox[q] * sk[0] + oy[q] * sk[1] + oz[q] * sk[2] < 0.0)) continue;
                double r[3] = {ox[q] - 2 * on * n[0], oy[q] - 2 * on * n[1], oz[q] - 2 * on * n[2]};
                uint32_t best = 0;
                double bd = 1e300;
                for (uint32_t p = 0; p < nq; p++) {
                    double d = (ox[p] - r[0]) * (ox[p] - r[0]) + (oy[p] - r[1]) * (oy[p] - r[1]) +
                               (oz[p] - r[2]) * (oz[p] - r[2]);
                    if (d < bd) { bd = d; best = p; }
                }
                if (bd > 1e-16) {
                    *err = e_refl;
                    oracle_sweep_destroy(S);
                    return NULL;
                }
                S->rmap[(size_t)S->rslot[f] * nq + q] = best;
            }
        }
    S->rent = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)S->nrefl * nq + 1));
    S->nent = 0;
    for (size_t i = 0; i < (size_t)S->nrefl * nq; i++) S->rent[i] = S->rmap[i] == NONE ? NONE : S->nent++;
    build_schedule(S);
    return S;
}

void oracle_sweep_destroy(or_sweep *S) {
    if (!S) return;
    free(S->s); free(S->stv); free(S->sav); free(S->B); free(S->nbr); free(S->map);
    free(S->bc); free(S->inc); free(S->rslot); free(S->rmap); free(S->rent);
    free(S->ox); free(S->oy); free(S->oz); free(S->w);
    free(S->order); free(S->level); free(S->lagbase); free(S->lag_qck);
    free(S);
}

static inline double odots(const or_sweep *S, uint32_t q, uint32_t c, int k) {
    const double *sk = &S->s[12 * c + 3 * k];
    return S->ox[q] * sk[0] + S->oy[q] * sk[1] + S->oz[q] * sk[2];
}

/* Kahn levels per ordinate (header comment). */
static void build_schedule(or_sweep *S) {
    uint32_t nT = S->nT, nq = S->nq;
    S->order = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nq * nT);
    S->level = (int32_t *)malloc(sizeof(int32_t) * (size_t)nq * nT);
    S->lagbase = (uint32_t *)malloc(sizeof(uint32_t) * 4 * (size_t)nq * nT);
    int64_t *maxlev = (int64_t *)calloc(nq, sizeof(int64_t)), *forced = (int64_t *)calloc(nq, sizeof(int64_t));
    uint8_t *lagged = (uint8_t *)calloc((size_t)nq * nT, 1); /* bit k: face k lagged */
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t q = 0; q < nq; q++) {
        int32_t *indeg = (int32_t *)malloc(sizeof(int32_t) * nT);
        int32_t *lev = &S->level[(size_t)q * nT];
        uint32_t *ord = &S->order[(size_t)q * nT];
        for (uint32_t c = 0; c < nT; c++) {
            int d = 0;
            for (int k = 0; k < 4; k++)
                if (S->nbr[4 * c + k] >= 0 && odots(S, q, c, k) < 0.0) d++;
            indeg[c] = d;
            lev[c] = -1;
        }
        uint32_t n = 0, head = 0, minrem = 0;
        for (uint32_t c = 0; c < nT; c++)
            if (indeg[c] == 0) ord[n++] = c;
        int32_t L = 0;
        while (n > head || n < nT) {
            if (head == n) { /* stalled: the smallest cell not yet scheduled forms a level */
                while (lev[minrem] >= 0) minrem++;
                uint32_t c = minrem;
                for (int k = 0; k < 4; k++) {
                    int64_t u = S->nbr[4 * c + k];
                    if (u >= 0 && odots(S, q, c, k) < 0.0 && lev[u] < 0) lagged[(size_t)q * nT + c] |= 1u << k;
                }
                indeg[c] = -(1 << 20); /* never reaches 0 again */
                ord[n++] = c;
                forced[q]++;
            }
            uint32_t end = n;
            for (uint32_t i = head; i < end; i++) lev[ord[i]] = L;
            for (uint32_t i = head; i < end; i++) {
                uint32_t c = ord[i];
                for (int k = 0; k < 4; k++) {
                    int64_t d = S->nbr[4 * c + k];
                    if (d < 0 || !(odots(S, q, c, k) > 0.0)) continue;
                    if (--indeg[d] == 0) ord[n++] = (uint32_t)d;
                }
            }
            for (uint32_t i = end + 1; i < n; i++) { /* next level by ascending index */
                uint32_t v = ord[i], j = i;
                while (j > end && ord[j - 1] > v) {
                    ord[j] = ord[j - 1];
                    j--;
                }
                ord[j] = v;
            }
            head = end;
            L++;
        }
        maxlev[q] = L;
        free(indeg);
    }
    /* lag slots in (q, c, k) order */
    uint32_t nlag = 0;
    for (size_t i = 0; i < (size_t)nq * nT; i++)
        for (int k = 0; k < 4; k++) {
            S->lagbase[4 * i + k] = (lagged[i] >> k & 1) ? nlag++ : NONE;
        }
    S->nlag = nlag;
    S->lag_qck = (uint32_t *)malloc(sizeof(uint32_t) * 3 * (nlag + 1));
    for (size_t i = 0; i < (size_t)nq * nT; i++)
        for (int k = 0; k < 4; k++)
            if (S->lagbase[4 * i + k] != NONE) {
                uint32_t sl = S->lagbase[4 * i + k];
                S->lag_qck[3 * sl] = (uint32_t)(i / nT);
                S->lag_qck[3 * sl + 1] = (uint32_t)(i % nT);
                S->lag_qck[3 * sl + 2] = (uint32_t)k;
            }
    S->maxlev = 0;
    S->forced = 0;
    for (uint32_t q = 0; q < nq; q++) {
        if (maxlev[q] > S->maxlev) S->maxlev = maxlev[q];
        S->forced += forced[q];
    }
    free(maxlev);
    free(forced);
    free(lagged);
}

static inline uint64_t lagbase(const or_sweep *S) { return 4 * (uint64_t)S->nent; }
static inline uint64_t blen(const or_sweep *S) { return lagbase(S) + (uint64_t)S->nlag * 4; }

void oracle_sweep_info(const or_sweep *S, int64_t info[6]) {
    info[0] = (int64_t)blen(S);
    info[1] = S->nrefl;
    info[2] = S->nlag;
    info[3] = S->maxlev;
    info[4] = S->forced;
    info[5] = S->ninterior;
}

void oracle_sweep_levels(const or_sweep *S, int32_t *level) {
    memcpy(level, S->level, sizeof(int32_t) * (size_t)S->nq * S->nT);
}

/* ---- one sweep ----------------------------------------------------------- */
static void solve_cell(const or_sweep *S, uint32_t q, uint32_t c, const double *J_in, const double *B_in,
                       int with_ext, const double *psi_q, double *out) {
    double a[4], al[4], L[4][4], r[4];
    double Ain = 0.0;
    int inflow[4];
    for (int k = 0; k < 4; k++) {
        double d = odots(S, q, c, k);
        a[k] = -d;
        inflow[k] = d < 0.0;
        al[k] = inflow[k] ? a[k] : 0.0;
        Ain += al[k];
    }
    double stv = S->stv[c], ssv = S->stv[c] - S->sav[c];
    double Jc[4] = {0, 0, 0, 0}, Js = 0.0;
    if (J_in)
        for (int j = 0; j < 4; j++) {
            Jc[j] = J_in[4 * c + j];
            Js += Jc[j];
        }
    double ext = with_ext ? S->sav[c] * S->B[c] / 4.0 : 0.0;
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            double face = (i == j) ? 2.0 * (Ain - al[i]) : (Ain - al[i] - al[j]);
            L[i][j] = a[j] / 12.0 + stv * (i == j ? 2.0 : 1.0) / 20.0 + face / 12.0;
        }
        r[i] = ssv / 20.0 * (Jc[i] + Js) + ext;
    }
    for (int k = 0; k < 4; k++) {
        if (!inflow[k]) continue;
        double up[4] = {0, 0, 0, 0};
        int64_t nb = S->nbr[4 * c + k];
        uint32_t lag = S->lagbase[4 * ((size_t)q * S->nT + c) + k];
        if (lag != NONE) {
            uint64_t base = lagbase(S) + 4 * (uint64_t)lag;
            for (int j = 0; j < 4; j++)
                if (j != k) up[j] = B_in ? B_in[base + j] : 0.0;
        } else if (nb >= 0) {
            for (int j = 0; j < 4; j++)
                if (j != k) up[j] = psi_q[4 * nb + S->map[16 * c + 4 * k + j]];
        } else {
            uint32_t f = (uint32_t)(-nb - 1);
            if (S->bc[f] == 1) {
                uint64_t base = 4 * (uint64_t)S->rent[(size_t)S->rslot[f] * S->nq + q];
                for (int j = 0; j < 4; j++)
                    if (j != k) up[j] = B_in ? B_in[base + j] : 0.0;
            } else if (S->bc[f] == 2 && with_ext) {
                for (int j = 0; j < 4; j++)
                    if (j != k) up[j] = S->inc[f];
            }
        }
        double T = up[0] + up[1] + up[2] + up[3];
        for (int i = 0; i < 4; i++)
            if (i != k) r[i] += a[k] / 12.0 * (T + up[i]);
    }
    /* Gaussian elimination without pivoting */
    for (int k = 0; k < 4; k++) {
        double inv = 1.0 / L[k][k];
        for (int i = k + 1; i < 4; i++) {
            double f = L[i][k] * inv;
            for (int j = k + 1; j < 4; j++) L[i][j] -= f * L[k][j];
            r[i] -= f * r[k];
        }
    }
    for (int i = 3; i >= 0; i--) {
        double v = r[i];
        for (int j = i + 1; j < 4; j++) v -= L[i][j] * out[j];
        out[i] = v / L[i][i];
    }
}

void oracle_sweep_apply(const or_sweep *S, const double *J_in, const double *B_in, int with_ext, double *J_out,
                        double *B_out, double *psi_out) {
    uint32_t nT = S->nT, nq = S->nq;
    double *psi = psi_out ? psi_out : (double *)malloc(sizeof(double) * 4 * (size_t)nq * nT);
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t q = 0; q < nq; q++) {
        double *pq = &psi[4 * (size_t)q * nT];
        const uint32_t *ord = &S->order[(size_t)q * nT];
        for (uint32_t i = 0; i < nT; i++) {
            uint32_t c = ord[i];
            solve_cell(S, q, c, J_in, B_in, with_ext, pq, &pq[4 * c]);
        }
    }
    if (J_out) {
#pragma omp parallel for
        for (uint32_t c = 0; c < nT; c++)
            for (int j = 0; j < 4; j++) {
                double acc = 0.0;
                for (uint32_t q = 0; q < nq; q++) acc += S->w[q] * psi[4 * ((size_t)q * nT + c) + j];
                J_out[4 * c + j] = acc;
            }
    }
    if (B_out) {
        memset(B_out, 0, sizeof(double) * blen(S));
        for (uint32_t c = 0; c < nT; c++)
            for (int k = 0; k < 4; k++) {
                int64_t nb = S->nbr[4 * c + k];
                if (nb >= 0) continue;
                uint32_t f = (uint32_t)(-nb - 1);
                if (S->rslot[f] < 0) continue;
                for (uint32_t q = 0; q < nq; q++) {
                    uint32_t p = S->rmap[(size_t)S->rslot[f] * nq + q];
                    if (p == NONE) continue;
                    for (int j = 0; j < 4; j++)
                        if (j != k)
                            B_out[4 * (uint64_t)S->rent[(size_t)S->rslot[f] * nq + q] + j] =
                                psi[4 * ((size_t)p * nT + c) + j];
                }
            }
        uint64_t base = lagbase(S);
        for (uint32_t l = 0; l < S->nlag; l++) {
            uint32_t q = S->lag_qck[3 * l], c = S->lag_qck[3 * l + 1], k = S->lag_qck[3 * l + 2];
            int64_t u = S->nbr[4 * c + k];
            for (int j = 0; j < 4; j++)
                if (j != (int)k) B_out[base + 4 * l + j] = psi[4 * ((size_t)q * nT + u) + S->map[16 * c + 4 * k + j]];
        }
    }
    if (!psi_out) free(psi);
}

/* ---- solvers ------------------------------------------------------------- */
static double vnorm(uint64_t n, const double *x) {
    double s = 0.0;
    for (uint64_t i = 0; i < n; i++) s += x[i] * x[i];
    return sqrt(s);
}
static double vdot(uint64_t n, const double *x, const double *y) {
    double s = 0.0;
    for (uint64_t i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

/* y = (I - T) x, T x = S(x) without external sources */
static void apply_op(const or_sweep *S, const double *x, double *y) {
    uint64_t nJ = 4 * (uint64_t)S->nT, n = nJ + blen(S);
    oracle_sweep_apply(S, x, x + nJ, 0, y, y + nJ, NULL);
    for (uint64_t i = 0; i < n; i++) y[i] = x[i] - y[i];
}

int oracle_sweep_solve(const or_sweep *S, int method, double tol, int max_iter, int restart, double *J,
                       double *B, int *iterations, double *residual) {
    uint64_t nJ = 4 * (uint64_t)S->nT, nB = blen(S), n = nJ + nB;
    double *x = (double *)calloc(n, sizeof(double)), *b = (double *)malloc(sizeof(double) * n);
    oracle_sweep_apply(S, NULL, NULL, 1, b, b + nJ, NULL);
    int it = 0, conv = 0;
    double res = 0.0;
    if (method == 0) {
        double *y = (double *)malloc(sizeof(double) * n);
        memcpy(x, b, sizeof(double) * n);
        for (it = 1; it <= max_iter; it++) {
            oracle_sweep_apply(S, x, x + nJ, 1, y, y + nJ, NULL);
            double dn = 0.0;
            for (uint64_t i = 0; i < n; i++) dn += (y[i] - x[i]) * (y[i] - x[i]);
            res = sqrt(dn) / fmax(vnorm(n, y), 1e-300);
            memcpy(x, y, sizeof(double) * n);
            if (res < tol) { conv = 1; break; }
        }
        free(y);
    } else {
        int m = restart > 0 ? restart : 30;
        double *V = (double *)malloc(sizeof(double) * n * (m + 1));
        double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
        double *cs = (double *)malloc(sizeof(double) * m), *sn = (double *)malloc(sizeof(double) * m);
        double *g = (double *)malloc(sizeof(double) * (m + 1)), *yv = (double *)malloc(sizeof(double) * m);
        double bn = vnorm(n, b);
        if (bn == 0.0) conv = 1;
        while (!conv && it < max_iter) {
            apply_op(S, x, V);
            for (uint64_t i = 0; i < n; i++) V[i] = b[i] - V[i];
            double beta = vnorm(n, V);
            res = beta / bn;
            if (res < tol) { conv = 1; break; }
            for (uint64_t i = 0; i < n; i++) V[i] /= beta;
            memset(g, 0, sizeof(double) * (m + 1));
            g[0] = beta;
            int j;
            for (j = 0; j < m && it < max_iter; j++) {
                double *w = V + (uint64_t)(j + 1) * n;
                apply_op(S, V + (uint64_t)j * n, w);
                it++;
                for (int pass = 0; pass < 2; pass++) /* classical Gram-Schmidt, twice */
                    for (int i = 0; i <= j; i++) {
                        double h = vdot(n, V + (uint64_t)i * n, w);
                        H[i * m + j] += h;
                        for (uint64_t t = 0; t < n; t++) w[t] -= h * V[(uint64_t)i * n + t];
                    }
                double hn = vnorm(n, w);
                H[(j + 1) * m + j] = hn;
                if (hn > 0.0)
                    for (uint64_t t = 0; t < n; t++) w[t] /= hn;
                for (int i = 0; i < j; i++) {
                    double t0 = cs[i] * H[i * m + j] + sn[i] * H[(i + 1) * m + j];
                    H[(i + 1) * m + j] = -sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
                    H[i * m + j] = t0;
                }
                double h0 = H[j * m + j], h1 = H[(j + 1) * m + j], rr = sqrt(h0 * h0 + h1 * h1);
                cs[j] = h0 / rr;
                sn[j] = h1 / rr;
                H[j * m + j] = rr;
                H[(j + 1) * m + j] = 0.0;
                g[j + 1] = -sn[j] * g[j];
                g[j] = cs[j] * g[j];
                res = fabs(g[j + 1]) / bn;
                if (res < tol) { j++; break; }
            }
            for (int i = j - 1; i >= 0; i--) {
                double v = g[i];
                for (int k = i + 1; k < j; k++) v -= H[i * m + k] * yv[k];
                yv[i] = v / H[i * m + i];
            }
            for (int i = 0; i < j; i++)
                for (uint64_t t = 0; t < n; t++) x[t] += yv[i] * V[(uint64_t)i * n + t];
            memset(H, 0, sizeof(double) * (m + 1) * m);
            if (res < tol) { /* confirm with the true residual */
                apply_op(S, x, V);
                for (uint64_t i = 0; i < n; i++) V[i] = b[i] - V[i];
                res = vnorm(n, V) / bn;
                if (res < tol) conv = 1;
            }
        }
        free(V); free(H); free(cs); free(sn); free(g); free(yv);
    }
    memcpy(J, x, sizeof(double) * nJ);
    if (B) memcpy(B, x + nJ, sizeof(double) * nB);
    free(x);
    free(b);
    if (iterations) *iterations = it;
    if (residual) *residual = res;
    return conv ? 0 : 1;
}

/* ---- balance and moments ------------------------------------------------ */
void oracle_sweep_balance(const or_sweep *S, const double *J_in, const double *B_in, const double *psi,
                          double out[5]) {
    uint32_t nT = S->nT, nq = S->nq;
    double em = 0, ab = 0, esc = 0, in = 0, refl = 0;
    for (uint32_t c = 0; c < nT; c++) {
        double Ji = 0.0, Jo = 0.0;
        for (int j = 0; j < 4; j++) {
            Ji += J_in ? J_in[4 * c + j] : 0.0;
            for (uint32_t q = 0; q < nq; q++) Jo += S->w[q] * psi[4 * ((size_t)q * nT + c) + j];
        }
        em += S->sav[c] * S->B[c];
        ab += 0.25 * (S->stv[c] * Jo - (S->stv[c] - S->sav[c]) * Ji);
        for (int k = 0; k < 4; k++) {
            int64_t nb = S->nbr[4 * c + k];
            if (nb >= 0) continue;
            uint32_t f = (uint32_t)(-nb - 1);
            for (uint32_t q = 0; q < nq; q++) {
                double d = odots(S, q, c, k), m = 0.0;
                if (d > 0.0) {
                    for (int j = 0; j < 4; j++)
                        if (j != k) m += psi[4 * ((size_t)q * nT + c) + j];
                    m /= 3.0;
                    if (S->bc[f] == 1) refl += S->w[q] * d * m;
                    else esc += S->w[q] * d * m;
                } else if (d < 0.0) {
                    if (S->bc[f] == 2) {
                        in += S->w[q] * (-d) * S->inc[f];
                    } else if (S->bc[f] == 1 && B_in) {
                        uint64_t base = 4 * (uint64_t)S->rent[(size_t)S->rslot[f] * nq + q];
                        for (int j = 0; j < 4; j++)
                            if (j != k) m += B_in[base + j];
                        refl -= S->w[q] * (-d) * m / 3.0;
                    }
                }
            }
        }
    }
    out[0] = em;
    out[1] = ab;
    out[2] = esc;
    out[3] = in;
    out[4] = refl;
}

void oracle_sweep_moments(const or_sweep *S, const double *psi, int nmom, double *mom) {
    uint32_t nT = S->nT, nq = S->nq;
    double *Y = (double *)malloc(sizeof(double) * 16 * nq);
    for (uint32_t q = 0; q < nq; q++)
        for (int l = 0, m0 = 0; l <= 3; l++)
            for (int m = -l; m <= l; m++, m0++) Y[m0 * nq + q] = oracle_ylm(l, m, S->ox[q], S->oy[q], S->oz[q]);
#pragma omp parallel for
    for (uint32_t c = 0; c < nT; c++)
        for (int mm = 0; mm < nmom; mm++)
            for (int j = 0; j < 4; j++) {
                double acc = 0.0;
                for (uint32_t q = 0; q < nq; q++) acc += S->w[q] * Y[mm * nq + q] * psi[4 * ((size_t)q * nT + c) + j];
                mom[(size_t)mm * 4 * nT + 4 * c + j] = acc;
            }
    free(Y);
}

double oracle_sweep_outflow(const or_sweep *S, const double *psi, const int32_t *face_mask) {
    uint32_t nT = S->nT, nq = S->nq;
    double F = 0.0;
    for (uint32_t c = 0; c < nT; c++)
        for (int k = 0; k < 4; k++) {
            int64_t nb = S->nbr[4 * c + k];
            if (nb >= 0 || !face_mask[-nb - 1]) continue;
            for (uint32_t q = 0; q < nq; q++) {
                double d = odots(S, q, c, k), m = 0.0;
                if (!(d > 0.0)) continue;
                for (int j = 0; j < 4; j++)
                    if (j != k) m += psi[4 * ((size_t)q * nT + c) + j];
                F += S->w[q] * d * m / 3.0;
            }
        }
    return F;
}
