// Test infrastructure only: the oracle's scalar type layer.
//
// Every oracle routine is a template over its scalar type R. With R=double it is
// the plain CPU restatement used as the parity checker; with R=Counted the same
// statements run while tallying each IEEE operation, which is how the algorithmic
// FP64 operation count per particle-step is obtained (each +, -, *, /, sqrt counts
// one; libm calls and comparisons are tallied separately).
//
// The oracle is compiled with -O2 -ffp-contract=off -fno-fast-math so that every
// expression rounds exactly as gfortran evaluates the Fortran source it restates
// (reference Makefile:5 uses -ffp-contract=off for the same reason).
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

struct Tally {
    uint64_t add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0, libm = 0;
};
extern thread_local Tally tally;

struct Counted {
    double v;
    Counted() : v(0.0) {}
    Counted(double x) : v(x) {}
};
inline Counted operator+(Counted a, Counted b) { tally.add++; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { tally.add++; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { tally.mul++; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { tally.div++; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline bool operator<(Counted a, Counted b) { tally.cmp++; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { tally.cmp++; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { tally.cmp++; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { tally.cmp++; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { tally.cmp++; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { tally.cmp++; return a.v != b.v; }

inline double val(double x) { return x; }
inline double val(Counted x) { return x.v; }

inline double Sqrt(double x) { return std::sqrt(x); }
inline Counted Sqrt(Counted x) { tally.sqrt++; return Counted(std::sqrt(x.v)); }
inline double Cos(double x) { return std::cos(x); }
inline Counted Cos(Counted x) { tally.libm++; return Counted(std::cos(x.v)); }
inline double Sin(double x) { return std::sin(x); }
inline Counted Sin(Counted x) { tally.libm++; return Counted(std::sin(x.v)); }
inline double Sinh(double x) { return std::sinh(x); }
inline Counted Sinh(Counted x) { tally.libm++; return Counted(std::sinh(x.v)); }
inline double Acos(double x) { return std::acos(x); }
inline Counted Acos(Counted x) { tally.libm++; return Counted(std::acos(x.v)); }
inline double Acosh(double x) { return std::acosh(x); }
inline Counted Acosh(Counted x) { tally.libm++; return Counted(std::acosh(x.v)); }
inline double Fmod(double x, double y) { return std::fmod(x, y); }
inline Counted Fmod(Counted x, Counted y) { tally.libm++; return Counted(std::fmod(x.v, y.v)); }
inline double Pow(double x, double y) { return std::pow(x, y); }
inline Counted Pow(Counted x, Counted y) { tally.libm++; return Counted(std::pow(x.v, y.v)); }
inline double Fabs(double x) { return std::fabs(x); }
inline Counted Fabs(Counted x) { return Counted(std::fabs(x.v)); }
// Fortran SIGN(a,b): |a| carrying the sign bit of b (gfortran honours -0).
inline double Sign(double a, double b) { return std::copysign(std::fabs(a), b); }
inline Counted Sign(Counted a, Counted b) { return Counted(std::copysign(std::fabs(a.v), b.v)); }
inline double Max(double a, double b) { return a > b ? a : b; }
inline Counted Max(Counted a, Counted b) { tally.cmp++; return a.v > b.v ? a : b; }
inline double Min(double a, double b) { return a < b ? a : b; }
inline Counted Min(Counted a, Counted b) { tally.cmp++; return a.v < b.v ? a : b; }

}  // namespace oracle
