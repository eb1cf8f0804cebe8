// Forward-mode dual numbers for checking the hand-written adjoint point
// functions (test infrastructure).
//
// Dual<K> carries a value and K directional derivatives.  The point physics
// is templated on its arithmetic type, so instantiating its exact form with
// Dual<K> gives the flux and its directional derivatives from the same source
// as the forward residual.  Comparisons look at the value only, which fixes
// the branch of |x| and of max() at the evaluation point.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace sddc {

#define DUAL_HD __host__ __device__ __forceinline__

template <int K> struct Dual {
    double v;
    double d[K];
    DUAL_HD Dual() {}
    DUAL_HD Dual(double x) : v(x)
    {
        for (int i = 0; i < K; i++) d[i] = 0.0;
    }
    DUAL_HD explicit Dual(int x) : Dual((double)x) {}
};

template <int K> DUAL_HD Dual<K> operator+(const Dual<K> &a, const Dual<K> &b)
{
    Dual<K> r;
    r.v = a.v + b.v;
    for (int i = 0; i < K; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int K> DUAL_HD Dual<K> operator-(const Dual<K> &a, const Dual<K> &b)
{
    Dual<K> r;
    r.v = a.v - b.v;
    for (int i = 0; i < K; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int K> DUAL_HD Dual<K> operator-(const Dual<K> &a)
{
    Dual<K> r;
    r.v = -a.v;
    for (int i = 0; i < K; i++) r.d[i] = -a.d[i];
    return r;
}
template <int K> DUAL_HD Dual<K> operator*(const Dual<K> &a, const Dual<K> &b)
{
    Dual<K> r;
    r.v = a.v * b.v;
    for (int i = 0; i < K; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int K> DUAL_HD Dual<K> operator/(const Dual<K> &a, const Dual<K> &b)
{
    Dual<K> r;
    r.v = a.v / b.v;
    for (int i = 0; i < K; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
template <int K> DUAL_HD bool operator>(const Dual<K> &a, const Dual<K> &b) { return a.v > b.v; }
template <int K> DUAL_HD bool operator<(const Dual<K> &a, const Dual<K> &b) { return a.v < b.v; }
template <int K> DUAL_HD bool operator==(const Dual<K> &a, const Dual<K> &b) { return a.v == b.v; }

template <int K> DUAL_HD Dual<K> Sqrt(const Dual<K> &a)
{
    Dual<K> r;
    r.v = std::sqrt(a.v);
    for (int i = 0; i < K; i++) r.d[i] = a.d[i] * 0.5 / r.v;
    return r;
}
template <int K> DUAL_HD Dual<K> Abs(const Dual<K> &a) { return a.v < 0.0 ? -a : a; }

}  // namespace sddc
