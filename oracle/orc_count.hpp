/*
 * orc_count.hpp -- a double that counts the arithmetic done on it.
 *
 * TEST INFRASTRUCTURE ONLY.  libsddc_oracle_count.so is the oracle's own
 * source compiled as C++ with -DORC_COUNT, so that every state-dependent
 * quantity (the type orc_real) is an orc_count: each +, -, *, / and square
 * root on one adds to a global tally.  One residual evaluation or RK stage of
 * that build then gives the exact operation count of the path per
 * degree of freedom.  Operations on quantities that do not depend on the
 * state (operators, metrics, the AV sensor's double arithmetic) and sign
 * changes, |x| and max() are not counted.  The build is single-threaded (the
 * tally is one set of counters).
 */
#ifndef ORC_COUNT_HPP
#define ORC_COUNT_HPP

#include <cmath>

struct orc_tally_t {
    unsigned long long add, mul, div, sqrt;
};
extern orc_tally_t orc_tally;

struct orc_count {
    double v;
    orc_count() = default;
    orc_count(double x) : v(x) {}
    orc_count &operator+=(orc_count b) { orc_tally.add++; v += b.v; return *this; }
    orc_count &operator-=(orc_count b) { orc_tally.add++; v -= b.v; return *this; }
    orc_count &operator*=(orc_count b) { orc_tally.mul++; v *= b.v; return *this; }
    orc_count &operator/=(orc_count b) { orc_tally.div++; v /= b.v; return *this; }
};

inline orc_count operator+(orc_count a, orc_count b) { orc_tally.add++; return orc_count(a.v + b.v); }
inline orc_count operator-(orc_count a, orc_count b) { orc_tally.add++; return orc_count(a.v - b.v); }
inline orc_count operator*(orc_count a, orc_count b) { orc_tally.mul++; return orc_count(a.v * b.v); }
inline orc_count operator/(orc_count a, orc_count b) { orc_tally.div++; return orc_count(a.v / b.v); }
inline orc_count operator+(orc_count a, double b) { return a + orc_count(b); }
inline orc_count operator-(orc_count a, double b) { return a - orc_count(b); }
inline orc_count operator*(orc_count a, double b) { return a * orc_count(b); }
inline orc_count operator/(orc_count a, double b) { return a / orc_count(b); }
inline orc_count operator+(double a, orc_count b) { return orc_count(a) + b; }
inline orc_count operator-(double a, orc_count b) { return orc_count(a) - b; }
inline orc_count operator*(double a, orc_count b) { return orc_count(a) * b; }
inline orc_count operator/(double a, orc_count b) { return orc_count(a) / b; }
inline orc_count operator-(orc_count a) { return orc_count(-a.v); }
inline orc_count operator+(orc_count a) { return a; }
inline orc_count orc_count_sqrt(orc_count a)
{
    orc_tally.sqrt++;
    return orc_count(std::sqrt(a.v));
}

#endif
