// Spectral-difference points and Lagrange bases shared by the host set-up
// library and the drop-in's host code.
//   solution points: Chebyshev-Gauss points on [0,1]
//   flux points: the two end points plus the Legendre-Gauss points
// (setsandpoints, initsetup.f90:171-259; hhval, initsetup.f90:322-344).
#pragma once

#include <cmath>

namespace sddc {

constexpr double kPi = 3.141592653589793;  // atan(1.d0)*4.d0, setup2d.f90:66

inline void sd_points(int np, double *Xs, double *Xf)
{
    for (int i = 1; i <= np; i++)
        Xs[i - 1] = 0.5 * (1.0 - std::cos((double)(2 * i - 1) * kPi / (2.0 * (double)np)));
    double *X = Xf - 1;
    switch (np) {
    case 1: X[1] = 0.0; X[2] = 1.0; break;
    case 2: X[1] = 0.0; X[2] = 0.5; X[3] = 1.0; break;
    case 3:
        X[1] = 0.0;
        X[2] = (1.0 - std::sqrt(3.0) / 3.0) / 2.0;
        X[3] = (1.0 + std::sqrt(3.0) / 3.0) / 2.0;
        X[4] = 1.0;
        break;
    case 4:
        X[1] = 0.0;
        X[2] = (1.0 - std::sqrt(15.0) / 5.0) / 2.0;
        X[3] = 0.5;
        X[4] = (1.0 + std::sqrt(15.0) / 5.0) / 2.0;
        X[5] = 1.0;
        break;
    case 5: {
        double a = std::sqrt(525.0 + 70.0 * std::sqrt(30.0)) / 35.0;
        double b = std::sqrt(525.0 - 70.0 * std::sqrt(30.0)) / 35.0;
        X[1] = 0.0; X[2] = (1.0 - a) / 2.0; X[3] = (1.0 - b) / 2.0;
        X[4] = (1.0 + b) / 2.0; X[5] = (1.0 + a) / 2.0; X[6] = 1.0;
        break;
    }
    case 6: {
        double a = std::sqrt(245.0 + 14.0 * std::sqrt(70.0)) / 21.0;
        double b = std::sqrt(245.0 - 14.0 * std::sqrt(70.0)) / 21.0;
        X[1] = 0.0; X[2] = (1.0 - a) / 2.0; X[3] = (1.0 - b) / 2.0; X[4] = 0.5;
        X[5] = (1.0 + b) / 2.0; X[6] = (1.0 + a) / 2.0; X[7] = 1.0;
        break;
    }
    default:
        for (int i = 1; i <= np + 1; i++) X[i] = NAN;
    }
}

// Lagrange basis polynomial i (1-based) on the points X[0..np-1], at x
inline double lagrange(const double *X, int np, int i, double x)
{
    double n = 1.0, d = 1.0;
    for (int s = 1; s <= np; s++)
        if (s != i) {
            n = n * (x - X[s - 1]);
            d = d * (X[i - 1] - X[s - 1]);
        }
    return n / d;
}

}  // namespace sddc
