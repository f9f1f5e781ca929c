// Test infrastructure only: forward-mode dual numbers for the oracle's
// templated routines. Running mdt_mvs over Dual<N> propagates N tangent
// directions through exactly the statements the oracle restates (the
// variational equations of the kick and the Kepler drift as the code computes
// them, iterations included); with massless test particles every particle can
// share the same N seeds, since none of them acts on another body.
#pragma once
#include <cmath>

#include "oracle_scalar.hpp"

namespace oracle {

template <int N> struct Dual {
    double v;
    double d[N];
    Dual() : v(0.0) { for (int k = 0; k < N; ++k) d[k] = 0.0; }
    Dual(double x) : v(x) { for (int k = 0; k < N; ++k) d[k] = 0.0; }
};

template <int N> inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v + b.v);
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v - b.v);
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r(-a.v);
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v * b.v);
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v / b.v);
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
template <int N> inline bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> inline bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> inline bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> inline bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N> inline bool operator==(const Dual<N>& a, const Dual<N>& b) { return a.v == b.v; }
template <int N> inline bool operator!=(const Dual<N>& a, const Dual<N>& b) { return a.v != b.v; }

template <int N> inline double val(const Dual<N>& x) { return x.v; }

// f(a) with f'(a) given: the chain rule on every tangent.
template <int N> inline Dual<N> chain(const Dual<N>& a, double fv, double dfv) {
    Dual<N> r(fv);
    for (int k = 0; k < N; ++k) r.d[k] = dfv * a.d[k];
    return r;
}
template <int N> inline Dual<N> Sqrt(const Dual<N>& a) {
    const double s = std::sqrt(a.v);
    return chain(a, s, 0.5 / s);
}
template <int N> inline Dual<N> Cos(const Dual<N>& a) { return chain(a, std::cos(a.v), -std::sin(a.v)); }
template <int N> inline Dual<N> Sin(const Dual<N>& a) { return chain(a, std::sin(a.v), std::cos(a.v)); }
template <int N> inline Dual<N> Sinh(const Dual<N>& a) { return chain(a, std::sinh(a.v), std::cosh(a.v)); }
template <int N> inline Dual<N> Acos(const Dual<N>& a) {
    return chain(a, std::acos(a.v), -1.0 / std::sqrt(1.0 - a.v * a.v));
}
template <int N> inline Dual<N> Acosh(const Dual<N>& a) {
    return chain(a, std::acosh(a.v), 1.0 / std::sqrt(a.v * a.v - 1.0));
}
template <int N> inline Dual<N> Fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
template <int N> inline Dual<N> Fmod(const Dual<N>& a, const Dual<N>& b) {
    const double q = std::trunc(a.v / b.v);
    Dual<N> r(std::fmod(a.v, b.v));
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - q * b.d[k];
    return r;
}
template <int N> inline Dual<N> Pow(const Dual<N>& a, const Dual<N>& b) {
    const double p = std::pow(a.v, b.v);
    Dual<N> r(p);
    const double da = b.v * std::pow(a.v, b.v - 1.0);
    const double db = a.v > 0.0 ? p * std::log(a.v) : 0.0;
    for (int k = 0; k < N; ++k) r.d[k] = da * a.d[k] + db * b.d[k];
    return r;
}
// Fortran SIGN(a, b): |a| with the sign of b.
template <int N> inline Dual<N> Sign(const Dual<N>& a, const Dual<N>& b) {
    const bool flip = std::signbit(a.v) != std::signbit(b.v);
    return flip ? -a : a;
}
template <int N> inline Dual<N> Max(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v ? a : b; }
template <int N> inline Dual<N> Min(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v ? a : b; }

}  // namespace oracle
