// ORACLE — test infrastructure only.  Operation-counting scalar used to take
// the FP64 flop census of the semi-analytic path: the oracle source is
// compiled once more with ORACLE_REAL = oracle_count::CD.
//
// Counting convention: +, -, *, / and sqrt count 1 flop each; every
// transcendental (sin, cos, log, exp, acos, asin, atan2, pow) counts 1 flop
// and is also tallied separately; comparisons, fabs and copies count 0.
#pragma once
#include <cmath>

namespace oracle_count {

struct Tally { long long add, mul, div, sqrt, trans; };
extern thread_local Tally tally;

struct CD {
    double v;
    CD() : v(0) {}
    CD(double x) : v(x) {}
    CD(int x) : v(x) {}
    explicit operator double() const { return v; }
};

inline CD operator+(CD a, CD b) { tally.add++; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { tally.add++; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { tally.mul++; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { tally.div++; return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
inline CD& operator+=(CD& a, CD b) { a = a + b; return a; }
inline CD& operator-=(CD& a, CD b) { a = a - b; return a; }
inline CD& operator*=(CD& a, CD b) { a = a * b; return a; }
inline CD& operator/=(CD& a, CD b) { a = a / b; return a; }
inline bool operator<(CD a, CD b) { return a.v < b.v; }
inline bool operator>(CD a, CD b) { return a.v > b.v; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { return a.v >= b.v; }
inline bool operator==(CD a, CD b) { return a.v == b.v; }
inline bool operator!=(CD a, CD b) { return a.v != b.v; }
inline CD sqrt(CD a) { tally.sqrt++; return CD(std::sqrt(a.v)); }
inline CD fabs(CD a) { return CD(std::fabs(a.v)); }
inline CD sin(CD a) { tally.trans++; return CD(std::sin(a.v)); }
inline CD cos(CD a) { tally.trans++; return CD(std::cos(a.v)); }
inline CD log(CD a) { tally.trans++; return CD(std::log(a.v)); }
inline CD acos(CD a) { tally.trans++; return CD(std::acos(a.v)); }
inline CD asin(CD a) { tally.trans++; return CD(std::asin(a.v)); }
inline CD atan2(CD a, CD b) { tally.trans++; return CD(std::atan2(a.v, b.v)); }

}  // namespace oracle_count
