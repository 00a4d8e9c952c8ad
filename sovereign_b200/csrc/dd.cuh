// dd.cuh -- double-double arithmetic (an unevaluated sum hi + lo of two FP64 numbers, about 106
// significand bits), host and device.
//
// Built from the error-free transformations: Knuth's TwoSum (the exact rounding error of a + b),
// Dekker's FastTwoSum for |a| >= |b|, and the product error a*b - fl(a*b) from one fused
// multiply-add. Addition and multiplication follow the accurate double-double algorithms of
// Hida, Li & Bailey ("Algorithms for quad-double precision floating point arithmetic", ARITH-15,
// 2001); division is long division with three FP64 quotient digits. Every step uses only IEEE
// FP64 +, -, * and fma with round-to-nearest, so the results are the same on every device.
#pragma once

#include <cmath>

#ifndef SOV_HD
#define SOV_HD __host__ __device__ __forceinline__
#endif

namespace sov {

struct dd {
  double hi, lo;
};

SOV_HD dd dd_from(double a) { return dd{a, 0.0}; }

// s + e = a + b exactly (any magnitudes)
SOV_HD dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}

// s + e = a + b exactly, assuming |a| >= |b| (or a == 0)
SOV_HD dd fast_two_sum(double a, double b) {
  const double s = a + b;
  return dd{s, b - (s - a)};
}

// p + e = a * b exactly
SOV_HD dd two_prod(double a, double b) {
  const double p = a * b;
  return dd{p, fma(a, b, -p)};
}

SOV_HD dd dd_add(dd x, dd y) {
  dd s = two_sum(x.hi, y.hi);
  const dd t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}

SOV_HD dd dd_neg(dd x) { return dd{-x.hi, -x.lo}; }
SOV_HD dd dd_sub(dd x, dd y) { return dd_add(x, dd_neg(y)); }

SOV_HD dd dd_add_d(dd x, double b) {
  dd s = two_sum(x.hi, b);
  s.lo += x.lo;
  return fast_two_sum(s.hi, s.lo);
}

SOV_HD dd dd_mul(dd x, dd y) {
  dd p = two_prod(x.hi, y.hi);
  p.lo = fma(x.hi, y.lo, fma(x.lo, y.hi, p.lo));
  return fast_two_sum(p.hi, p.lo);
}

SOV_HD dd dd_mul_d(dd x, double b) {
  dd p = two_prod(x.hi, b);
  p.lo = fma(x.lo, b, p.lo);
  return fast_two_sum(p.hi, p.lo);
}

// x / y: three quotient digits q1 + q2 + q3, each the FP64 quotient of the running remainder
SOV_HD dd dd_div(dd x, dd y) {
  const double q1 = x.hi / y.hi;
  dd r = dd_sub(x, dd_mul_d(y, q1));
  const double q2 = r.hi / y.hi;
  r = dd_sub(r, dd_mul_d(y, q2));
  const double q3 = r.hi / y.hi;
  return dd_add_d(fast_two_sum(q1, q2), q3);
}

SOV_HD dd dd_recip(dd y) { return dd_div(dd_from(1.0), y); }

}  // namespace sov
