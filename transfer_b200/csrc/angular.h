// Angular substrate: real spherical harmonics, sphere / hemisphere quadrature
// and the angular coupling tables of the even-parity P_N operator.
//
// Interfaces kept from the reference (same names, argument meaning and
// storage): Spherical (Spherical.h:4-13), HemiQuad (HemiQuad.h:4-12),
// LebedevQuad (LebedevQuad.h:4-12), AngularData (AngularData.h:8-18).
#pragma once
#include <cstdint>
#include <vector>

namespace transfer {

typedef uint32_t idx;

// Real spherical harmonics, orthonormal on AVERAGE over the sphere
// (<Y_lm Y_l'm'> = delta), without Condon-Shortley phase:
//   Y_lm = c_lm * cos(m phi) sin^m(theta) P_l^(m)(cos theta)    m >= 0
//   Y_lm = c_lm * sin(|m| phi) sin^|m|(theta) P_l^(|m|)(cos theta) m < 0
//   c_lm = sqrt((2l+1) (2 - delta_m0) (l-m)!/(l+m)!)
// (Spherical.cpp:39-47, 62-82).  Evaluated here in Cartesian form:
// sin^m(theta) cos(m phi) = Re (x+iy)^m, sin^m(theta) sin(m phi) = Im (x+iy)^m,
// with P_l^(m) (the m-th derivative of the Legendre polynomial) from the
// three-term recurrence in l.
class Spherical {
public:
    explicit Spherical(int topow);      // harmonics up to degree topow
    double value(int l, int m, double x, double y, double z) const;
    double value(int l, int m, double theta, double phi) const;
    int maxdeg() const { return d_; }
private:
    int d_;
    std::vector<double> c_;   // c_[l*(d_+1)+m]
};

// Gauss-Legendre rule on [-1,1] (nodes descending, Newton on P_n).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);

// Half-range rule (HemiQuad.cpp:265-286): Gauss in z on [0,1] with
// go = (mindegree+1)/2+1 nodes (descending, weights summing to 1) times
// mindegree+1 uniform azimuths; total weight 1.
struct HemiQuad {
    int order;
    std::vector<double> x, y, z, w;
    explicit HemiQuad(int mindegree);
};

// Lebedev rule of algebraic precision >= mindegree (LebedevQuad.cpp:6269-6277):
// the smallest of the tabulated octahedral rules whose precision reaches
// mindegree; weights sum to 1.  The rules (up to 350 points) are generated
// from their defining equations (lebedev.cpp); throws for larger ones.
struct LebedevQuad {
    int order = 0;
    std::vector<double> x, y, z, w;
    LebedevQuad() {}
    explicit LebedevQuad(int mindegree);
};
// Number of points of the Lebedev rule with precision >= prec, or -1
// (order_by_precision, LebedevQuad.cpp:8-30).
int lebedev_order_by_precision(int prec);

// Angular coupling tables of the even-parity P_N operator for the
// harmonics l = 0,2,..,2maxk, m = -l..l (lm in that order),
// slm = (1+maxk)(1+2maxk) (AngularData.cpp:9-67):
//   omega[i][lm1][lm2] = <Y_lm1 Y_lm2 Omega_i Omega_j>, j = omega_pos[..]:
//       the first j in 0,1,2 whose average exceeds 1e-10 in magnitude,
//       else j = 2;
//   O_n[lm1][lm2]      = <|Omega_n| Y_lm1 Y_lm2>   (n = x, y, z).
// Averages over the unit sphere (weights sum to 1).  They are integrals of
// polynomials of degree <= 4maxk+2 and are evaluated here with exact
// Gauss x trapezoid product rules.
struct AngularData {
    int maxk;
    idx slm;
    std::vector<double> omega;   // [3][slm][slm]
    std::vector<idx> omega_pos;  // [3][slm][slm]
    std::vector<double> Ox, Oy, Oz;  // [slm][slm]
    explicit AngularData(int maxk);
};

}  // namespace transfer
