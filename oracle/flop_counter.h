/*
 * flop_counter.h - an FP64 scalar that counts its arithmetic -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * oracle_flops.cpp compiles the oracle (mfcfd_oracle.cpp) with `double`
 * replaced by CountedDouble, so one run of the restated reference counts the
 * FP64 operations of each phase of fpi_solver exactly as the reference
 * performs them.  With the solver's own exp/log/erf (mfmath.h, plain
 * arithmetic) the transcendentals are counted through their arithmetic too;
 * with the C library's they count as calls.
 *
 * Counting rules: add, subtract, multiply, divide and square root are one
 * operation each, a fused multiply-add is two; comparisons, negation, fabs,
 * rint and bit moves are free.  The value itself is an IEEE double, so the
 * counted run computes the same bits as the plain oracle.
 */
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

struct FlopTally {
    int64_t add = 0, mul = 0, div = 0, sqrt = 0, fma = 0;
    int64_t exp_calls = 0, log_calls = 0, erf_calls = 0, pow_calls = 0;
};

// One tally per phase of fpi_solver; g_flop_phase selects the current one.
constexpr int FLOP_PHASES = 8;
extern FlopTally g_flops[FLOP_PHASES];
extern int g_flop_phase;

struct CountedDouble {
    double v;
    CountedDouble() = default;
    CountedDouble(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
    explicit operator float() const { return (float)v; }
    explicit operator int64_t() const { return (int64_t)v; }
    CountedDouble &operator+=(CountedDouble o) { ++g_flops[g_flop_phase].add; v += o.v; return *this; }
    CountedDouble &operator-=(CountedDouble o) { ++g_flops[g_flop_phase].add; v -= o.v; return *this; }
    CountedDouble &operator*=(CountedDouble o) { ++g_flops[g_flop_phase].mul; v *= o.v; return *this; }
    CountedDouble &operator/=(CountedDouble o) { ++g_flops[g_flop_phase].div; v /= o.v; return *this; }
    CountedDouble operator-() const { return CountedDouble(-v); }
    CountedDouble operator+() const { return *this; }
};
static_assert(sizeof(CountedDouble) == sizeof(double), "CountedDouble must be layout-compatible with double");

inline CountedDouble operator+(CountedDouble a, CountedDouble b) { ++g_flops[g_flop_phase].add; return a.v + b.v; }
inline CountedDouble operator-(CountedDouble a, CountedDouble b) { ++g_flops[g_flop_phase].add; return a.v - b.v; }
inline CountedDouble operator*(CountedDouble a, CountedDouble b) { ++g_flops[g_flop_phase].mul; return a.v * b.v; }
inline CountedDouble operator/(CountedDouble a, CountedDouble b) { ++g_flops[g_flop_phase].div; return a.v / b.v; }
inline bool operator<(CountedDouble a, CountedDouble b) { return a.v < b.v; }
inline bool operator>(CountedDouble a, CountedDouble b) { return a.v > b.v; }
inline bool operator<=(CountedDouble a, CountedDouble b) { return a.v <= b.v; }
inline bool operator>=(CountedDouble a, CountedDouble b) { return a.v >= b.v; }
inline bool operator==(CountedDouble a, CountedDouble b) { return a.v == b.v; }
inline bool operator!=(CountedDouble a, CountedDouble b) { return a.v != b.v; }

// math functions the oracle and mfmath.h call (unqualified and std::)
inline CountedDouble fma(CountedDouble a, CountedDouble b, CountedDouble c) {
    ++g_flops[g_flop_phase].fma;
    return std::fma(a.v, b.v, c.v);
}
inline CountedDouble rint(CountedDouble a) { return std::rint(a.v); }
inline CountedDouble fabs(CountedDouble a) { return std::fabs(a.v); }
inline CountedDouble sqrt(CountedDouble a) { ++g_flops[g_flop_phase].sqrt; return std::sqrt(a.v); }
namespace std {
inline CountedDouble fabs(CountedDouble a) { return std::fabs(a.v); }
inline CountedDouble abs(CountedDouble a) { return std::fabs(a.v); }
inline CountedDouble sqrt(CountedDouble a) { ++g_flops[g_flop_phase].sqrt; return std::sqrt(a.v); }
inline CountedDouble exp(CountedDouble a) { ++g_flops[g_flop_phase].exp_calls; return std::exp(a.v); }
inline CountedDouble log(CountedDouble a) { ++g_flops[g_flop_phase].log_calls; return std::log(a.v); }
inline CountedDouble erf(CountedDouble a) { ++g_flops[g_flop_phase].erf_calls; return std::erf(a.v); }
inline CountedDouble log10(CountedDouble a) { return std::log10(a.v); }
inline CountedDouble pow(CountedDouble a, CountedDouble b) { ++g_flops[g_flop_phase].pow_calls; return std::pow(a.v, b.v); }
inline bool isfinite(CountedDouble a) { return std::isfinite(a.v); }
inline bool isnan(CountedDouble a) { return std::isnan(a.v); }
}  // namespace std
