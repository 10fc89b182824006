// LebedevQuad (see angular.h): Lebedev rules generated from their defining
// equations instead of stored tables.
//
// A rule with the symmetry of the octahedral group (with inversion)
// integrates every polynomial of degree <= L exactly on the sphere iff it
// integrates the octahedrally invariant ones; on the unit sphere those of
// even degree are spanned by p4^a p6^b (4a + 6b <= L - 1), p4 = x^4 + y^4 +
// z^4, p6 = x^2 y^2 z^2.  An invariant polynomial takes a single value on an
// orbit of the group, so the rule's sum is sum_orbits w_o |o| P(base_o).
// Orbits: a1 (6 points, the axes), a2 (12, (0,1,1)/sqrt 2), a3 (8,
// (1,1,1)/sqrt 3), b(l) (24, (l,l,m)), c(p) (24, (p,q,0)), d(r,s) (48,
// (r,s,t)).  For each rule the published orbit structure (Lebedev & Laikov,
// Doklady Math. 59 (1999) 477) makes the equations a square system in the
// orbit weights and parameters.  It is solved from seeded random orbit
// parameters by variable projection (the weights, which enter linearly, by
// least squares; Levenberg-Marquardt on the parameters) and a final Newton
// polish of weights and parameters together, until a solution with positive
// weights and distinct, admissible orbits is found.  Rules up to 194 points
// (precision 23) are generated this way (194 takes a few seconds, once per
// process); larger ones are not.  Each generated rule is checked against the
// exact sphere averages before it is returned and cached.
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "angular.h"

namespace transfer {

// Orders and algebraic precisions of the Lebedev-Laikov family
// (order_by_precision, LebedevQuad.cpp:8-30).
static const int kOrders[] = {6,    14,   26,   38,   50,   74,   86,   110,  146,  170,  194,  230,  266,
                              302,  350,  386,  434,  482,  530,  590,  650,  698,  770,  830,  890,  974,
                              1046, 1118, 1202, 1274, 1358, 1454, 1538, 1622, 1730, 1814, 1910, 2030, 2126,
                              2222, 2354, 2450, 2558, 2702, 2810, 2930, 3074, 3182, 3314, 3470, 3590, 3722,
                              3890, 4010, 4154, 4334, 4466, 4610, 4802, 4934, 5090, 5294, 5438, 5606, 5810};

int lebedev_order_by_precision(int prec) {
    for (int i = 0; i < 65; ++i)
        if (3 + 2 * i >= prec) return kOrders[i];
    return -1;
}

namespace {

// orbit structure of the rules generated here: counts of a1, a2, a3 and of
// the b, c, d families
struct OrbitSpec {
    int order, precision, a1, a2, a3, nb, nc, nd;
};
const OrbitSpec kSpecs[] = {
    {6, 3, 1, 0, 0, 0, 0, 0},     {14, 5, 1, 0, 1, 0, 0, 0},    {26, 7, 1, 1, 1, 0, 0, 0},
    {38, 9, 1, 0, 1, 0, 1, 0},    {50, 11, 1, 1, 1, 1, 0, 0},   {74, 13, 1, 1, 1, 1, 1, 0},
    {86, 15, 1, 0, 1, 2, 1, 0},   {110, 17, 1, 0, 1, 3, 1, 0},  {146, 19, 1, 1, 1, 3, 0, 1},
    {170, 21, 1, 1, 1, 3, 1, 1},  {194, 23, 1, 1, 1, 4, 1, 1},
};  // larger rules (230 points and up) are not found reliably from random starts

double dfact(int n) {  // n!! for odd n >= -1
    double r = 1.0;
    for (; n > 1; n -= 2) r *= n;
    return r;
}
// average of x^(2i) y^(2j) z^(2k) over the unit sphere
double sphere_avg(int i, int j, int k) {
    return dfact(2 * i - 1) * dfact(2 * j - 1) * dfact(2 * k - 1) / dfact(2 * (i + j + k) + 1);
}
double factorial(int n) {
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}
// sphere average of p4^A p6^B (multinomial expansion of p4^A)
double invariant_avg(int A, int B) {
    double s = 0.0;
    for (int a = 0; a <= A; ++a)
        for (int b = 0; a + b <= A; ++b) {
            const int c = A - a - b;
            s += factorial(A) / (factorial(a) * factorial(b) * factorial(c)) *
                 sphere_avg(2 * a + B, 2 * b + B, 2 * c + B);
        }
    return s;
}

struct Problem {
    OrbitSpec sp;
    std::vector<std::pair<int, int>> inv;  // (A, B)
    std::vector<double> target;
    int no = 0, nv = 0;                     // orbits, unknowns
};

// base point of an orbit and its derivatives with respect to the orbit's
// parameters (kind: 0 a1, 1 a2, 2 a3, 3 b, 4 c, 5 d)
void base_point(int kind, const double *prm, double p[3], double dp[2][3]) {
    const double r2 = std::sqrt(0.5), r3 = std::sqrt(1.0 / 3.0);
    for (int i = 0; i < 2; ++i) dp[i][0] = dp[i][1] = dp[i][2] = 0.0;
    switch (kind) {
        case 0: p[0] = 1; p[1] = 0; p[2] = 0; break;
        case 1: p[0] = 0; p[1] = r2; p[2] = r2; break;
        case 2: p[0] = p[1] = p[2] = r3; break;
        case 3: {
            const double l = prm[0], m = std::sqrt(std::fmax(1.0 - 2.0 * l * l, 1e-300));
            p[0] = l; p[1] = l; p[2] = m;
            dp[0][0] = 1; dp[0][1] = 1; dp[0][2] = -2.0 * l / m;
            break;
        }
        case 4: {
            const double a = prm[0], q = std::sqrt(std::fmax(1.0 - a * a, 1e-300));
            p[0] = a; p[1] = q; p[2] = 0;
            dp[0][0] = 1; dp[0][1] = -a / q;
            break;
        }
        default: {
            const double r = prm[0], s = prm[1], t = std::sqrt(std::fmax(1.0 - r * r - s * s, 1e-300));
            p[0] = r; p[1] = s; p[2] = t;
            dp[0][0] = 1; dp[0][2] = -r / t;
            dp[1][1] = 1; dp[1][2] = -s / t;
        }
    }
}
// P = p4^A p6^B at p and its gradient
double invariant(int A, int B, const double p[3], double g[3]) {
    const double x2 = p[0] * p[0], y2 = p[1] * p[1], z2 = p[2] * p[2];
    const double p4 = x2 * x2 + y2 * y2 + z2 * z2, p6 = x2 * y2 * z2;
    const double P4 = std::pow(p4, A), P6 = std::pow(p6, B);
    const double dP4 = A ? A * std::pow(p4, A - 1) : 0.0, dP6 = B ? B * std::pow(p6, B - 1) : 0.0;
    const double d4[3] = {4 * p[0] * x2, 4 * p[1] * y2, 4 * p[2] * z2};
    const double d6[3] = {2 * p[0] * y2 * z2, 2 * p[1] * x2 * z2, 2 * p[2] * x2 * y2};
    for (int i = 0; i < 3; ++i) g[i] = dP4 * d4[i] * P6 + P4 * dP6 * d6[i];
    return P4 * P6;
}

const int kSize[6] = {6, 12, 8, 24, 24, 48};
const int kParams[6] = {0, 0, 0, 1, 1, 2};

std::vector<int> orbit_kinds(const OrbitSpec &s) {
    std::vector<int> k;
    for (int i = 0; i < s.a1; ++i) k.push_back(0);
    for (int i = 0; i < s.a2; ++i) k.push_back(1);
    for (int i = 0; i < s.a3; ++i) k.push_back(2);
    for (int i = 0; i < s.nb; ++i) k.push_back(3);
    for (int i = 0; i < s.nc; ++i) k.push_back(4);
    for (int i = 0; i < s.nd; ++i) k.push_back(5);
    return k;
}

// residuals F and Jacobian J (row-major nv x nv) at unknowns v
void eval(const Problem &pr, const std::vector<int> &kinds, const std::vector<double> &v, std::vector<double> &F,
          std::vector<double> *J) {
    const int ne = static_cast<int>(pr.inv.size()), nv = pr.nv, no = pr.no;
    F.assign(ne, 0.0);
    if (J) J->assign(static_cast<size_t>(ne) * nv, 0.0);
    int pi = no;
    for (int o = 0; o < no; ++o) {
        const int kind = kinds[o], np = kParams[kind];
        double p[3], dp[2][3];
        base_point(kind, &v[pi], p, dp);
        for (int e = 0; e < ne; ++e) {
            double g[3];
            const double P = invariant(pr.inv[e].first, pr.inv[e].second, p, g);
            F[e] += v[o] * kSize[kind] * P;
            if (J) {
                (*J)[static_cast<size_t>(e) * nv + o] = kSize[kind] * P;
                for (int k = 0; k < np; ++k)
                    (*J)[static_cast<size_t>(e) * nv + pi + k] =
                        v[o] * kSize[kind] * (g[0] * dp[k][0] + g[1] * dp[k][1] + g[2] * dp[k][2]);
            }
        }
        pi += np;
    }
    // rows scaled by 1 / target, so that every equation counts to relative precision
    for (int e = 0; e < ne; ++e) {
        F[e] = F[e] / pr.target[e] - 1.0;
        if (J)
            for (int k = 0; k < nv; ++k) (*J)[static_cast<size_t>(e) * nv + k] /= pr.target[e];
    }
}

// solves (A) x = b, A n x n (copied), partial pivoting; false if singular
bool solve_dense(std::vector<double> A, std::vector<double> b, int n, std::vector<double> &x) {
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(A[static_cast<size_t>(i) * n + k]) > std::fabs(A[static_cast<size_t>(piv) * n + k])) piv = i;
        if (A[static_cast<size_t>(piv) * n + k] == 0.0) return false;
        if (piv != k) {
            for (int j = 0; j < n; ++j) std::swap(A[static_cast<size_t>(k) * n + j], A[static_cast<size_t>(piv) * n + j]);
            std::swap(b[k], b[piv]);
        }
        for (int i = k + 1; i < n; ++i) {
            const double f = A[static_cast<size_t>(i) * n + k] / A[static_cast<size_t>(k) * n + k];
            for (int j = k; j < n; ++j) A[static_cast<size_t>(i) * n + j] -= f * A[static_cast<size_t>(k) * n + j];
            b[i] -= f * b[k];
        }
    }
    x.assign(n, 0.0);
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= A[static_cast<size_t>(i) * n + j] * x[j];
        x[i] = s / A[static_cast<size_t>(i) * n + i];
    }
    return true;
}

double norm2(const std::vector<double> &F) {
    double s = 0.0;
    for (double f : F) s += f * f;
    return s;
}

// Levenberg-Marquardt from v; true when the residual vanishes to rounding
bool levenberg_marquardt(const Problem &pr, const std::vector<int> &kinds, std::vector<double> &v) {
    const int n = pr.nv;
    std::vector<double> F, J, Ft, vt, JtJ(static_cast<size_t>(n) * n), JtF(n), d;
    eval(pr, kinds, v, F, &J);
    double f = norm2(F), mu = 1e-3;
    for (int it = 0; it < 400; ++it) {
        if (f < 1e-30) return true;
        for (int i = 0; i < n; ++i) {
            JtF[i] = 0.0;
            for (int e = 0; e < n; ++e) JtF[i] -= J[static_cast<size_t>(e) * n + i] * F[e];
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int e = 0; e < n; ++e) s += J[static_cast<size_t>(e) * n + i] * J[static_cast<size_t>(e) * n + j];
                JtJ[static_cast<size_t>(i) * n + j] = s;
            }
        }
        bool moved = false;
        for (int tries = 0; tries < 20 && !moved; ++tries) {
            std::vector<double> A = JtJ;
            for (int i = 0; i < n; ++i) A[static_cast<size_t>(i) * n + i] *= 1.0 + mu;
            if (!solve_dense(A, JtF, n, d)) {
                mu *= 10.0;
                continue;
            }
            vt = v;
            for (int i = 0; i < n; ++i) vt[i] += d[i];
            eval(pr, kinds, vt, Ft, nullptr);
            const double ft = norm2(Ft);
            if (std::isfinite(ft) && ft < f) {
                v = vt;
                f = ft;
                mu = std::fmax(mu * 0.1, 1e-15);
                moved = true;
            } else {
                mu *= 10.0;
            }
        }
        if (!moved) return f < 1e-30;
        eval(pr, kinds, v, F, &J);
    }
    return f < 1e-30;
}

// canonical orbit parameters; false if the solution is not an admissible
// rule (non-positive weight, degenerate or repeated orbit)
// negative_ok: the rule may carry a negative orbit weight (the 74-point rule
// does: its 8-point (1,1,1)/sqrt(3) orbit weighs -0.0296)
bool admissible(const std::vector<int> &kinds, std::vector<double> &v, int no, bool negative_ok) {
    const double r2 = std::sqrt(0.5), r3 = std::sqrt(1.0 / 3.0), eps = 1e-6;
    std::vector<std::vector<double>> seen(6);
    int pi = no;
    for (int o = 0; o < no; ++o) {
        if (!(v[o] > 0.0) && !(negative_ok && v[o] < 0.0)) return false;
        const int kind = kinds[o];
        if (kind == 3) {
            double l = std::fabs(v[pi]);
            if (!(l > eps && l < r2 - eps) || std::fabs(l - r3) < eps) return false;
            v[pi] = l;
            for (double s : seen[3])
                if (std::fabs(s - l) < eps) return false;
            seen[3].push_back(l);
        } else if (kind == 4) {
            double a = std::fabs(v[pi]);
            if (!(a < 1.0 - eps) || a < eps) return false;
            a = std::fmin(a, std::sqrt(1.0 - a * a));  // (p, q, 0) and (q, p, 0) are one orbit
            if (std::fabs(a - r2) < eps) return false;
            v[pi] = a;
            for (double s : seen[4])
                if (std::fabs(s - a) < eps) return false;
            seen[4].push_back(a);
        } else if (kind == 5) {
            double r = std::fabs(v[pi]), s = std::fabs(v[pi + 1]);
            const double t2 = 1.0 - r * r - s * s;
            if (!(t2 > eps)) return false;
            double c[3] = {r, s, std::sqrt(t2)};
            // sort so that the orbit has one representation
            for (int i = 0; i < 3; ++i)
                for (int j = i + 1; j < 3; ++j)
                    if (c[j] < c[i]) std::swap(c[i], c[j]);
            if (c[0] < eps || c[1] - c[0] < eps || c[2] - c[1] < eps) return false;
            v[pi] = c[0];
            v[pi + 1] = c[1];
            for (size_t k = 0; k < seen[5].size(); k += 2)
                if (std::fabs(seen[5][k] - c[0]) < eps && std::fabs(seen[5][k + 1] - c[1]) < eps) return false;
            seen[5].push_back(c[0]);
            seen[5].push_back(c[1]);
        }
        pi += kParams[kind];
    }
    return true;
}

// splitmix64 for the seeded starts
struct Rng {
    uint64_t s;
    double uniform() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    }
};

void expand_orbit(int kind, const double *prm, double w, LebedevQuad &q) {
    double p[3], dp[2][3];
    base_point(kind, prm, p, dp);
    // all sign changes and permutations, duplicates removed
    std::vector<std::array<double, 3>> pts;
    const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (auto &pm : perm)
        for (int sg = 0; sg < 8; ++sg) {
            std::array<double, 3> a = {p[pm[0]] * ((sg & 1) ? -1 : 1), p[pm[1]] * ((sg & 2) ? -1 : 1),
                                       p[pm[2]] * ((sg & 4) ? -1 : 1)};
            bool dup = false;
            for (auto &b : pts)
                if (std::fabs(a[0] - b[0]) + std::fabs(a[1] - b[1]) + std::fabs(a[2] - b[2]) < 1e-12) dup = true;
            if (!dup) pts.push_back(a);
        }
    for (auto &a : pts) {
        q.x.push_back(a[0] == 0.0 ? 0.0 : a[0]);
        q.y.push_back(a[1] == 0.0 ? 0.0 : a[1]);
        q.z.push_back(a[2] == 0.0 ? 0.0 : a[2]);
        q.w.push_back(w);
    }
}

// Variable projection: the equations are linear in the weights, so for
// given orbit parameters theta the weights are the least-squares solution and
// only theta is iterated (rows scaled by 1 / target).  Returns the scaled
// residual vector; w receives the weights.
std::vector<double> projected_residual(const Problem &pr, const std::vector<int> &kinds, const std::vector<double> &theta,
                                       std::vector<double> &w) {
    const int ne = static_cast<int>(pr.inv.size()), no = pr.no;
    std::vector<double> M(static_cast<size_t>(ne) * no), t(ne);
    int pi = 0;
    for (int o = 0; o < no; ++o) {
        double p[3], dp[2][3], g[3];
        base_point(kinds[o], &theta[pi], p, dp);
        for (int e = 0; e < ne; ++e)
            M[static_cast<size_t>(e) * no + o] =
                kSize[kinds[o]] * invariant(pr.inv[e].first, pr.inv[e].second, p, g) / pr.target[e];
        pi += kParams[kinds[o]];
    }
    for (int e = 0; e < ne; ++e) t[e] = 1.0;
    // least squares by modified Gram-Schmidt QR of M (ne x no)
    std::vector<double> Q = M, R(static_cast<size_t>(no) * no, 0.0);
    for (int j = 0; j < no; ++j) {
        for (int i = 0; i < j; ++i) {
            double d = 0.0;
            for (int e = 0; e < ne; ++e) d += Q[static_cast<size_t>(e) * no + i] * Q[static_cast<size_t>(e) * no + j];
            R[static_cast<size_t>(i) * no + j] = d;
            for (int e = 0; e < ne; ++e) Q[static_cast<size_t>(e) * no + j] -= d * Q[static_cast<size_t>(e) * no + i];
        }
        double nn = 0.0;
        for (int e = 0; e < ne; ++e) nn += Q[static_cast<size_t>(e) * no + j] * Q[static_cast<size_t>(e) * no + j];
        nn = std::sqrt(nn);
        R[static_cast<size_t>(j) * no + j] = nn;
        if (nn > 0.0)
            for (int e = 0; e < ne; ++e) Q[static_cast<size_t>(e) * no + j] /= nn;
    }
    std::vector<double> qt(no, 0.0);
    for (int j = 0; j < no; ++j)
        for (int e = 0; e < ne; ++e) qt[j] += Q[static_cast<size_t>(e) * no + j] * t[e];
    w.assign(no, 0.0);
    for (int j = no - 1; j >= 0; --j) {
        double v = qt[j];
        for (int k = j + 1; k < no; ++k) v -= R[static_cast<size_t>(j) * no + k] * w[k];
        const double d = R[static_cast<size_t>(j) * no + j];
        w[j] = d != 0.0 ? v / d : 0.0;
    }
    std::vector<double> r(ne);
    for (int e = 0; e < ne; ++e) {
        double v = -t[e];
        for (int o = 0; o < no; ++o) v += M[static_cast<size_t>(e) * no + o] * w[o];
        r[e] = v;
    }
    return r;
}

// Levenberg-Marquardt on theta for the projected residual (finite-difference
// Jacobian); true when the residual falls below 1e-12
bool lm_projected(const Problem &pr, const std::vector<int> &kinds, std::vector<double> &theta) {
    const int n = static_cast<int>(theta.size());
    std::vector<double> w;
    std::vector<double> r = projected_residual(pr, kinds, theta, w);
    const int ne = static_cast<int>(r.size());
    double f = norm2(r), mu = 1e-3;
    std::vector<double> J(static_cast<size_t>(ne) * n), JtJ(static_cast<size_t>(n) * n), Jtr(n), d;
    for (int it = 0; it < 300; ++it) {
        if (f < 1e-24) return true;
        for (int k = 0; k < n; ++k) {
            const double h = 1e-7;
            std::vector<double> tp = theta, tm = theta, w2;
            tp[k] += h;
            tm[k] -= h;
            const std::vector<double> rp = projected_residual(pr, kinds, tp, w2), rm = projected_residual(pr, kinds, tm, w2);
            for (int e = 0; e < ne; ++e) J[static_cast<size_t>(e) * n + k] = (rp[e] - rm[e]) / (2 * h);
        }
        for (int i = 0; i < n; ++i) {
            Jtr[i] = 0.0;
            for (int e = 0; e < ne; ++e) Jtr[i] -= J[static_cast<size_t>(e) * n + i] * r[e];
            for (int j = 0; j < n; ++j) {
                double s2 = 0.0;
                for (int e = 0; e < ne; ++e) s2 += J[static_cast<size_t>(e) * n + i] * J[static_cast<size_t>(e) * n + j];
                JtJ[static_cast<size_t>(i) * n + j] = s2;
            }
        }
        bool moved = false;
        for (int tries = 0; tries < 20 && !moved; ++tries) {
            std::vector<double> A = JtJ;
            for (int i = 0; i < n; ++i) A[static_cast<size_t>(i) * n + i] = A[static_cast<size_t>(i) * n + i] * (1.0 + mu) + 1e-30;
            if (!solve_dense(A, Jtr, n, d)) {
                mu *= 10.0;
                continue;
            }
            std::vector<double> tt = theta;
            for (int i = 0; i < n; ++i) tt[i] += d[i];
            std::vector<double> w2;
            const std::vector<double> rt = projected_residual(pr, kinds, tt, w2);
            const double ft = norm2(rt);
            if (std::isfinite(ft) && ft < f) {
                theta = tt;
                r = rt;
                f = ft;
                mu = std::fmax(mu * 0.2, 1e-12);
                moved = true;
            } else {
                mu *= 10.0;
            }
        }
        if (!moved) break;
    }
    return f < 1e-24;
}

bool generate(const OrbitSpec &sp, LebedevQuad &q) {
    Problem pr;
    pr.sp = sp;
    for (int A = 0; 4 * A <= sp.precision - 1; ++A)
        for (int B = 0; 4 * A + 6 * B <= sp.precision - 1; ++B) pr.inv.push_back({A, B});
    for (auto &ab : pr.inv) pr.target.push_back(invariant_avg(ab.first, ab.second));
    const std::vector<int> kinds = orbit_kinds(sp);
    pr.no = static_cast<int>(kinds.size());
    pr.nv = pr.no;
    for (int k : kinds) pr.nv += kParams[k];
    if (pr.nv != static_cast<int>(pr.inv.size())) return false;  // not a square system
    Rng rng{0x5EED0000ULL + static_cast<uint64_t>(sp.order)};
    const double r2 = std::sqrt(0.5);
    for (int trial = 0; trial < 4000; ++trial) {
        // random orbit parameters; weights by least squares; then a Newton
        // polish of weights and parameters together
        std::vector<double> theta(pr.nv - pr.no);
        int ti = 0;
        for (int k : kinds) {
            if (k == 3) theta[ti] = 0.02 + (r2 - 0.04) * rng.uniform();
            if (k == 4) theta[ti] = 0.02 + (r2 - 0.04) * rng.uniform();
            if (k == 5) {
                const double a = 0.05 + 0.9 * rng.uniform(), b = 0.05 + 0.9 * rng.uniform();
                const double sc = std::sqrt(a * a + b * b + 0.3);
                theta[ti] = a / sc;
                theta[ti + 1] = b / sc;
            }
            ti += kParams[k];
        }
        if (!lm_projected(pr, kinds, theta)) continue;
        std::vector<double> wts;
        projected_residual(pr, kinds, theta, wts);
        std::vector<double> v(pr.nv);
        for (int o = 0; o < pr.no; ++o) v[o] = wts[o];
        for (size_t i = 0; i < theta.size(); ++i) v[pr.no + i] = theta[i];
        int pi = pr.no;
        if (!levenberg_marquardt(pr, kinds, v)) continue;
        if (!admissible(kinds, v, pr.no, sp.order == 74 || getenv("LEB_NEG") != nullptr)) continue;
        std::vector<double> F;
        eval(pr, kinds, v, F, nullptr);
        double worst = 0.0;
        for (size_t e = 0; e < F.size(); ++e) worst = std::fmax(worst, std::fabs(F[e]));
        if (worst > 1e-14) continue;
        q.x.clear();
        q.y.clear();
        q.z.clear();
        q.w.clear();
        pi = pr.no;
        for (int o = 0; o < pr.no; ++o) {
            expand_orbit(kinds[o], &v[pi], v[o], q);
            pi += kParams[kinds[o]];
        }
        if (static_cast<int>(q.w.size()) != sp.order) continue;
        return true;
    }
    return false;
}

std::mutex g_cache_mutex;
std::map<int, LebedevQuad> g_cache;

}  // namespace

LebedevQuad::LebedevQuad(int mindegree) {
    order = lebedev_order_by_precision(mindegree);
    const OrbitSpec *spec = nullptr;
    for (const OrbitSpec &s : kSpecs)
        if (s.order == order) spec = &s;
    if (!spec) throw std::runtime_error("LebedevQuad: rules above 194 points (precision 23) are not generated");
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    auto it = g_cache.find(order);
    if (it == g_cache.end()) {
        LebedevQuad q;
        q.order = order;
        if (!generate(*spec, q)) throw std::runtime_error("LebedevQuad: the rule's equations were not solved");
        it = g_cache.emplace(order, q).first;
    }
    x = it->second.x;
    y = it->second.y;
    z = it->second.z;
    w = it->second.w;
}

}  // namespace transfer
