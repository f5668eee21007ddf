// flopcount.h -- a counting scalar for the flop-count build of the CPU
// oracle (oracle/gdf_oracle_count.cpp). TEST AND MEASUREMENT INFRASTRUCTURE
// ONLY: nothing in the product uses it.
//
// fcnt holds one double and behaves as one (same size and layout, so the
// oracle's C ABI still takes double arrays), rounding every operation
// exactly as double arithmetic does; each + - * / and square root also
// increments a tally. The tally is the algorithmic FP64 work of the
// reference's loops: a division or a square root counts once (the GPU
// executes each as a sequence of several instructions), comparisons,
// absolute values, sign transfers and negations count nothing.
#pragma once

#include <cmath>
#include <cstdint>

struct FlopTally {
  uint64_t add = 0, mul = 0, div = 0, sqrt = 0, pow = 0;
};
extern FlopTally g_flops;

struct fcnt {
  double v;
  fcnt() = default;
  fcnt(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  explicit operator long long() const { return (long long)v; }
  explicit operator bool() const { return v != 0.0; }
  fcnt operator-() const { return fcnt(-v); }
  fcnt operator+() const { return *this; }
  fcnt& operator+=(fcnt o) { ++g_flops.add; v += o.v; return *this; }
  fcnt& operator-=(fcnt o) { ++g_flops.add; v -= o.v; return *this; }
  fcnt& operator*=(fcnt o) { ++g_flops.mul; v *= o.v; return *this; }
  fcnt& operator/=(fcnt o) { ++g_flops.div; v /= o.v; return *this; }
};

#define FCNT_BINOP(OP, FIELD)                                                          \
  inline fcnt operator OP(fcnt a, fcnt b) { ++g_flops.FIELD; return fcnt(a.v OP b.v); } \
  inline fcnt operator OP(fcnt a, double b) { ++g_flops.FIELD; return fcnt(a.v OP b); } \
  inline fcnt operator OP(double a, fcnt b) { ++g_flops.FIELD; return fcnt(a OP b.v); }
FCNT_BINOP(+, add)
FCNT_BINOP(-, add)
FCNT_BINOP(*, mul)
FCNT_BINOP(/, div)
#undef FCNT_BINOP

#define FCNT_CMP(OP)                                                       \
  inline bool operator OP(fcnt a, fcnt b) { return a.v OP b.v; }           \
  inline bool operator OP(fcnt a, double b) { return a.v OP b; }           \
  inline bool operator OP(double a, fcnt b) { return a OP b.v; }
FCNT_CMP(<)
FCNT_CMP(>)
FCNT_CMP(<=)
FCNT_CMP(>=)
FCNT_CMP(==)
FCNT_CMP(!=)
#undef FCNT_CMP

namespace std {
inline fcnt sqrt(fcnt x) { ++g_flops.sqrt; return fcnt(::sqrt(x.v)); }
inline fcnt fabs(fcnt x) { return fcnt(::fabs(x.v)); }
inline fcnt abs(fcnt x) { return fcnt(::fabs(x.v)); }
inline bool isnan(fcnt x) { return ::std::isnan(x.v); }
inline bool isfinite(fcnt x) { return ::std::isfinite(x.v); }
inline fcnt copysign(fcnt a, fcnt b) { return fcnt(::copysign(a.v, b.v)); }
inline fcnt copysign(double a, fcnt b) { return fcnt(::copysign(a, b.v)); }
inline fcnt copysign(fcnt a, double b) { return fcnt(::copysign(a.v, b)); }
inline fcnt pow(fcnt a, double b) { ++g_flops.pow; return fcnt(::pow(a.v, b)); }
inline fcnt pow(fcnt a, fcnt b) { ++g_flops.pow; return fcnt(::pow(a.v, b.v)); }
inline fcnt exp(fcnt x) { ++g_flops.pow; return fcnt(::exp(x.v)); }
inline fcnt sin(fcnt x) { ++g_flops.pow; return fcnt(::sin(x.v)); }
inline fcnt cos(fcnt x) { ++g_flops.pow; return fcnt(::cos(x.v)); }
inline fcnt atan(fcnt x) { ++g_flops.pow; return fcnt(::atan(x.v)); }
}  // namespace std
inline fcnt sqrt(fcnt x) { return std::sqrt(x); }
inline fcnt fabs(fcnt x) { return std::fabs(x); }
inline fcnt copysign(fcnt a, fcnt b) { return std::copysign(a, b); }
inline fcnt copysign(double a, fcnt b) { return std::copysign(a, b); }
