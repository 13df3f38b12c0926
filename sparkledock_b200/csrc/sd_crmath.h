// Correctly rounded (outside hard cases) double-precision sin and acos for the
// GSO slerp, usable from host C++ and CUDA device code.
//
// The reference slerp (source/dock/src/prepare_gso_tasks.cc:1410-1415) calls
// glibc acos/sin.  GPU libm results are not guaranteed to equal glibc bit for
// bit, so both sides of the parity check instead use functions whose result is
// the double nearest the exact value: the value is evaluated in double-double
// arithmetic (Dekker/Knuth error-free transforms, about 2^-100 relative error)
// and rounded once.  The domain that the slerp reaches is small:
//   acos: q_dot in [0, 0.9995]   (the branch at prepare_gso_tasks.cc:1397)
//   sin : omega*{1, 1-step, step} in (0, pi/2]
// sd_sin_cr is valid for |x| <= 2 (Taylor series truncated at x^35/35!);
// sd_acos_cr for x in [-1, 1] with one double-double Newton step on cos(y)=x
// from the platform acos as the initial guess (any guess within a few ulp
// converges; the platform value never reaches the output directly).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SD_HD __host__ __device__ __forceinline__
#else
#define SD_HD static inline
#endif

namespace sdcr {

struct dd { double hi, lo; };

SD_HD double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
// Knuth two-sum: s + e == a + b exactly.
SD_HD dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
// Dekker fast two-sum, requires |a| >= |b|.
SD_HD dd fast_two_sum(double a, double b) {
  double s = a + b;
  double e = b - (s - a);
  return {s, e};
}
// exact product via FMA
SD_HD dd two_prod(double a, double b) {
  double p = a * b;
  double e = fma_(a, b, -p);
  return {p, e};
}
SD_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
SD_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = fma_(a.hi, b.lo, p.lo);
  p.lo = fma_(a.lo, b.hi, p.lo);
  return fast_two_sum(p.hi, p.lo);
}
// a / d for an exactly representable double d
SD_HD dd dd_div_d(dd a, double d) {
  double q1 = a.hi / d;
  dd p = two_prod(q1, d);
  double r = ((a.hi - p.hi) - p.lo) + a.lo;
  double q2 = r / d;
  return fast_two_sum(q1, q2);
}
// 1 - a
SD_HD dd one_minus(dd a) {
  dd s = two_sum(1.0, -a.hi);
  s.lo -= a.lo;
  return fast_two_sum(s.hi, s.lo);
}

// sin(x) as double-double, |x| <= 2: x * (1 - x^2/(2*3) (1 - x^2/(4*5) (...)))
SD_HD dd sin_dd(dd x) {
  dd x2 = dd_mul(x, x);
  dd p = {1.0, 0.0};
  for (int k = 17; k >= 1; --k) {
    double den = (double)(2 * k) * (double)(2 * k + 1);
    p = one_minus(dd_div_d(dd_mul(x2, p), den));
  }
  return dd_mul(x, p);
}
// cos(x) as double-double, |x| <= 2: 1 - x^2/(1*2) (1 - x^2/(3*4) (...))
SD_HD dd cos_dd(dd x) {
  dd x2 = dd_mul(x, x);
  dd p = {1.0, 0.0};
  for (int k = 17; k >= 1; --k) {
    double den = (double)(2 * k - 1) * (double)(2 * k);
    p = one_minus(dd_div_d(dd_mul(x2, p), den));
  }
  return p;
}

}  // namespace sdcr

// sin(x) rounded to nearest, |x| <= 2
SD_HD double sd_sin_cr(double x) {
  sdcr::dd r = sdcr::sin_dd({x, 0.0});
  return r.hi + r.lo;
}

// acos(x) rounded to nearest for x in [-1, 1]; NaN in, NaN out.
SD_HD double sd_acos_cr(double x) {
  double y0 = acos(x);
  if (!(x > -1.0 && x < 1.0)) return y0;  // endpoints exact (0, pi rounded), NaN passes through
  // acos(x) for x < 0 is pi - acos(-x); keep the Newton iteration on [0, pi/2]
  bool neg = x < 0.0;
  double ax = neg ? -x : x;
  double y = neg ? acos(ax) : y0;
  if (y < 1e-8) {
    // not reached by the slerp (q_dot <= 0.9995); a direct value is exact enough
    return neg ? 3.141592653589793 - y : y;
  }
  sdcr::dd yy = {y, 0.0};
  sdcr::dd c = sdcr::cos_dd(yy);
  sdcr::dd s = sdcr::sin_dd(yy);
  // Newton on f(y) = cos(y) - ax: y1 = y + (cos(y) - ax) / sin(y)
  double num = (c.hi - ax) + c.lo;
  double delta = num / s.hi;
  sdcr::dd y1 = sdcr::two_sum(y, delta);
  if (!neg) return y1.hi + y1.lo;
  // pi - y1 in double-double; pi as a double-double constant
  const sdcr::dd pi = {3.141592653589793116e+00, 1.224646799147353207e-16};
  sdcr::dd r = sdcr::dd_add(pi, {-y1.hi, -y1.lo});
  return r.hi + r.lo;
}
