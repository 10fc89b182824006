// Angular substrate (see angular.h).
#include "angular.h"

#include <cmath>
#include <stdexcept>

namespace transfer {

// ---------------------------------------------------------------- Spherical
Spherical::Spherical(int topow) : d_(topow), c_((topow + 1) * (topow + 1), 0.0) {
    for (int l = 0; l <= d_; ++l)
        for (int m = 0; m <= l; ++m) {
            // (2l+1)(2-delta) (l-m)!/(l+m)!  built as a running quotient
            double q = (2.0 * l + 1.0) * (m == 0 ? 1.0 : 2.0);
            for (int k = l - m + 1; k <= l + m; ++k) q /= k;
            c_[l * (d_ + 1) + m] = std::sqrt(q);
        }
}

// m-th derivative of the Legendre polynomial P_l at z:
//   D_m^m = (2m-1)!!, D_{m+1}^m = (2m+1) z D_m^m,
//   (l-m) D_l^m = (2l-1) z D_{l-1}^m - (l+m-1) D_{l-2}^m.
static double legendre_derivative(int l, int m, double z) {
    if (m > l) return 0.0;
    double dmm = 1.0;
    for (int k = 1; k <= m; ++k) dmm *= (2.0 * k - 1.0);
    if (l == m) return dmm;
    double prev = dmm, cur = (2.0 * m + 1.0) * z * dmm;
    for (int k = m + 2; k <= l; ++k) {
        double next = ((2.0 * k - 1.0) * z * cur - (k + m - 1.0) * prev) / (k - m);
        prev = cur;
        cur = next;
    }
    return cur;
}

double Spherical::value(int l, int m, double x, double y, double z) const {
    if (l < 0 || l > d_ || m < -l || m > l)
        throw std::out_of_range("Spherical::value: (l,m) out of range");
    int am = m < 0 ? -m : m;
    // (x + i y)^am
    double re = 1.0, im = 0.0;
    for (int k = 0; k < am; ++k) {
        double nre = re * x - im * y;
        im = re * y + im * x;
        re = nre;
    }
    double trig = (m >= 0) ? re : im;
    return c_[l * (d_ + 1) + am] * trig * legendre_derivative(l, am, z);
}

double Spherical::value(int l, int m, double theta, double phi) const {
    double st = std::sin(theta);
    return value(l, m, st * std::cos(phi), st * std::sin(phi), std::cos(theta));
}

// ----------------------------------------------------------- Gauss-Legendre
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        // Newton on P_n from the Chebyshev-like initial guess; node i is the
        // (i+1)-th largest root.
        double r = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = r;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * r * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double pn = (n == 1) ? r : p1;
            double pnm1 = (n == 1) ? 1.0 : p0;
            dp = n * (r * pn - pnm1) / (r * r - 1.0);
            double dr = pn / dp;
            r -= dr;
            if (std::fabs(dr) < 1e-17) break;
        }
        // recompute the derivative at the converged node
        double p0 = 1.0, p1 = r;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2.0 * k - 1.0) * r * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        double pn = (n == 1) ? r : p1, pnm1 = (n == 1) ? 1.0 : p0;
        dp = n * (r * pn - pnm1) / (r * r - 1.0);
        x[i] = r;
        w[i] = 2.0 / ((1.0 - r * r) * dp * dp);
    }
}

// ----------------------------------------------------------------- HemiQuad
HemiQuad::HemiQuad(int mindegree) {
    if (mindegree < 0) throw std::invalid_argument("HemiQuad: negative degree");
    int go = (mindegree + 1) / 2 + 1;
    int naz = mindegree + 1;
    order = go * naz;
    std::vector<double> gx, gw;
    gauss_legendre(go, gx, gw);
    x.resize(order);
    y.resize(order);
    z.resize(order);
    w.resize(order);
    for (int i = 0; i < naz; ++i) {
        double ang = 2.0 * M_PI * i / static_cast<double>(naz);
        double ca = std::cos(ang), sa = std::sin(ang);
        for (int j = 0; j < go; ++j) {
            double zz = 0.5 * (gx[j] + 1.0);  // [-1,1] -> [0,1], descending
            double r = std::sqrt(1.0 - zz * zz);
            x[i * go + j] = r * ca;
            y[i * go + j] = r * sa;
            z[i * go + j] = zz;
            w[i * go + j] = 0.5 * gw[j] / naz;
        }
    }
}

// -------------------------------------------------------------- AngularData
// Index of harmonic (l, m), l even.
static inline int lm_index(int l, int m) {
    // sum_{l' even < l} (2l'+1) = l(l-1)/2 ; then m + l
    return l * (l - 1) / 2 + (m + l);
}

AngularData::AngularData(int maxk_) : maxk(maxk_) {
    if (maxk < 0 || maxk > 7)
        throw std::invalid_argument("AngularData: maxk must be in 0..7");
    slm = static_cast<idx>((1 + maxk) * (1 + 2 * maxk));
    const int n = static_cast<int>(slm);
    const int L = 2 * maxk;
    Spherical sph(L);

    // list of (l,m) in storage order
    std::vector<int> ls(n), ms(n);
    for (int l = 0; l <= L; l += 2)
        for (int m = -l; m <= l; ++m) {
            int k = lm_index(l, m);
            ls[k] = l;
            ms[k] = m;
        }

    // ---- full-sphere product rule, exact for degree <= 4maxk+3
    int nz = 2 * maxk + 2;
    int nphi = 4 * maxk + 4;
    std::vector<double> gx, gw;
    gauss_legendre(nz, gx, gw);
    const int np = nz * nphi;
    std::vector<double> px(np), py(np), pz(np), pw(np);
    for (int a = 0; a < nz; ++a)
        for (int b = 0; b < nphi; ++b) {
            double phi = 2.0 * M_PI * b / nphi;
            double zz = gx[a], r = std::sqrt(1.0 - zz * zz);
            int p = a * nphi + b;
            px[p] = r * std::cos(phi);
            py[p] = r * std::sin(phi);
            pz[p] = zz;
            pw[p] = 0.5 * gw[a] / nphi;
        }
    std::vector<double> Y(static_cast<size_t>(n) * np);
    for (int k = 0; k < n; ++k)
        for (int p = 0; p < np; ++p)
            Y[static_cast<size_t>(k) * np + p] = sph.value(ls[k], ms[k], px[p], py[p], pz[p]);

    omega.assign(3 * n * n, 0.0);
    omega_pos.assign(3 * n * n, 0);
    const double *dir[3] = {px.data(), py.data(), pz.data()};
    std::vector<double> prod(np);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            for (int p = 0; p < np; ++p)
                prod[p] = pw[p] * Y[static_cast<size_t>(a) * np + p] * Y[static_cast<size_t>(b) * np + p];
            for (int i = 0; i < 3; ++i) {
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int p = 0; p < np; ++p) s += prod[p] * dir[i][p] * dir[j][p];
                    if (std::fabs(s) > 1e-10 || j == 2) {
                        omega[(i * n + a) * n + b] = s;
                        omega_pos[(i * n + a) * n + b] = static_cast<idx>(j);
                        break;
                    }
                }
            }
        }

    // ---- half-range tables <|Omega_n| Y Y>: hemisphere Omega_n > 0 with a
    // Gauss (z in [0,1]) x uniform-azimuth rule exact for the polynomial
    // Omega_n Y Y of degree 4maxk+1; the even integrand makes the hemisphere
    // average equal to the sphere average.
    HemiQuad h(4 * maxk + 1);
    Ox.assign(n * n, 0.0);
    Oy.assign(n * n, 0.0);
    Oz.assign(n * n, 0.0);
    std::vector<double> Yx(static_cast<size_t>(n) * h.order), Yy(Yx.size()), Yz(Yx.size());
    for (int k = 0; k < n; ++k)
        for (int p = 0; p < h.order; ++p) {
            size_t q = static_cast<size_t>(k) * h.order + p;
            // Omega = (hz, hx, hy): Omega_x = hz >= 0
            Yx[q] = sph.value(ls[k], ms[k], h.z[p], h.x[p], h.y[p]);
            // Omega = (hy, hz, hx): Omega_y = hz
            Yy[q] = sph.value(ls[k], ms[k], h.y[p], h.z[p], h.x[p]);
            // Omega = (hx, hy, hz)
            Yz[q] = sph.value(ls[k], ms[k], h.x[p], h.y[p], h.z[p]);
        }
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            double sx = 0, sy = 0, sz = 0;
            for (int p = 0; p < h.order; ++p) {
                double wz = h.w[p] * h.z[p];
                size_t qa = static_cast<size_t>(a) * h.order + p, qb = static_cast<size_t>(b) * h.order + p;
                sx += wz * Yx[qa] * Yx[qb];
                sy += wz * Yy[qa] * Yy[qb];
                sz += wz * Yz[qa] * Yz[qb];
            }
            Ox[a * n + b] = sx;
            Oy[a * n + b] = sy;
            Oz[a * n + b] = sz;
        }
}

}  // namespace transfer
