// Test infrastructure only: forward-mode dual numbers for the oracle's
// templated routines. Running mdt_mvs over Dual<N> propagates N tangent
// directions through exactly the statements the oracle restates (the
// variational equations of the kick and the Kepler drift as the code computes
// them; the universal-variable solve takes its root's tangent, kepu_tangent
// below); with massless test particles every particle can share the same N
// seeds, since none of them acts on another body.
#pragma once
#include <cmath>

#include "oracle_scalar.hpp"
#include "oracle_mvs.hpp"

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

// kepu_tangent for dual numbers (see oracle_mvs.hpp): at the anomaly sk the
// solver stopped at, the tangent of sk becomes that of the root,
// d sk - dF / F_s with F the universal Kepler residual and F_s = fp, and the
// Stumpff terms and fp are evaluated again with it (same values).
template <int N>
inline void kepu_tangent(Dual<N>& sk, const Dual<N>& dt, const Dual<N>& r0, const Dual<N>& mu, const Dual<N>& alpha,
                         const Dual<N>& u, Dual<N>& fp, Dual<N>& c1, Dual<N>& c2, Dual<N>& c3) {
    auto terms = [&](Dual<N>& c0) {
        const Dual<N> s2 = sk * sk;
        Dual<N> x = s2 * alpha;
        drift_kepu_stumpff(x, c0, c1, c2, c3);
        c1 = c1 * sk;
        c2 = c2 * s2;
        c3 = c3 * sk * s2;
        fp = r0 * c0 + u * c1 + mu * c2;
    };
    Dual<N> c0;
    terms(c0);
    const Dual<N> f = r0 * c1 + u * c2 + mu * c3 - dt;
    for (int k = 0; k < N; ++k) sk.d[k] = sk.d[k] - f.d[k] / fp.v;
    terms(c0);
}

}  // namespace oracle
