// flop_counter.hpp -- instrumented FP64 scalar for counting the operations of
// the oracle (TEST INFRASTRUCTURE ONLY).
//
// CD behaves like double and counts: + and - (n_add), * (n_mul), / (n_div),
// sqrt (n_sqrt), exp / log / pow / cos / tanh (n_trans) and comparisons
// (n_cmp).  Negation, abs, min and max are not counted.  The counts of one
// column step give the algorithmic operation count the roofline uses; the
// flop-equivalent convention (transcendental = 20) is applied by the caller.
#pragma once
#include <cmath>
#include <cstdint>

namespace gvo {

struct CD {
  double v = 0.0;
  static inline thread_local uint64_t n_add = 0, n_mul = 0, n_div = 0, n_sqrt = 0,
                                      n_trans = 0, n_cmp = 0;
  static void reset() { n_add = n_mul = n_div = n_sqrt = n_trans = n_cmp = 0; }
  CD() = default;
  CD(double x) : v(x) {}
  CD operator-() const { return CD(-v); }
};

inline CD operator+(CD a, CD b) { ++CD::n_add; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++CD::n_add; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++CD::n_mul; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++CD::n_div; return CD(a.v / b.v); }
inline CD operator+(CD a, double b) { return a + CD(b); }
inline CD operator-(CD a, double b) { return a - CD(b); }
inline CD operator*(CD a, double b) { return a * CD(b); }
inline CD operator/(CD a, double b) { return a / CD(b); }
inline CD operator+(double a, CD b) { return CD(a) + b; }
inline CD operator-(double a, CD b) { return CD(a) - b; }
inline CD operator*(double a, CD b) { return CD(a) * b; }
inline CD operator/(double a, CD b) { return CD(a) / b; }
inline CD operator+(CD a, int b) { return a + CD(double(b)); }
inline CD operator-(int a, CD b) { return CD(double(a)) - b; }
inline CD operator*(int a, CD b) { return CD(double(a)) * b; }

#define GVO_CMP(op)                                                         \
  inline bool operator op(CD a, CD b) { ++CD::n_cmp; return a.v op b.v; } \
  inline bool operator op(CD a, double b) { return a op CD(b); }            \
  inline bool operator op(double a, CD b) { return CD(a) op b; }
GVO_CMP(<)
GVO_CMP(>)
GVO_CMP(<=)
GVO_CMP(>=)
GVO_CMP(==)
GVO_CMP(!=)
#undef GVO_CMP

inline CD xexp(CD x) { ++CD::n_trans; return CD(std::exp(x.v)); }
inline CD xlog(CD x) { ++CD::n_trans; return CD(std::log(x.v)); }
inline CD xpow(CD x, double y) { ++CD::n_trans; return CD(std::pow(x.v, y)); }
inline CD xpow(CD x, CD y) { ++CD::n_trans; return CD(std::pow(x.v, y.v)); }
inline CD xcos(CD x) { ++CD::n_trans; return CD(std::cos(x.v)); }
inline CD xtanh(CD x) { ++CD::n_trans; return CD(std::tanh(x.v)); }
inline CD xsqrt(CD x) { ++CD::n_sqrt; return CD(std::sqrt(x.v)); }
inline CD xabs(CD x) { return CD(std::fabs(x.v)); }
inline double val(CD x) { return x.v; }

}  // namespace gvo
