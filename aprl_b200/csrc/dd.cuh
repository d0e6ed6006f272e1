// dd.cuh -- double-double (compensated binary64) arithmetic shared by the
// device reductions: Knuth's TwoSum, Dekker's exact product through a fused
// multiply-add, and the QD library's renormalisation, division and square
// root (Hida, Li and Bailey).  Host and device compile the same code.
#pragma once

#include <cmath>

namespace aprl_gpu {

struct DD {
  double hi, lo;
};

// s + e == a + b exactly.
__host__ __device__ __forceinline__ DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return DD{s, e};
}

// Requires |a| >= |b| (or a == 0).
__host__ __device__ __forceinline__ DD quick_two_sum(double a, double b) {
  const double s = a + b;
  return DD{s, b - (s - a)};
}

__host__ __device__ __forceinline__ DD two_prod(double a, double b) {
  const double p = a * b;
  return DD{p, fma(a, b, -p)};
}

__host__ __device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}

__host__ __device__ __forceinline__ DD dd_neg(DD a) { return DD{-a.hi, -a.lo}; }

__host__ __device__ __forceinline__ DD dd_mul(DD a, double b) {
  DD p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}

// Division of a double-double by a double.
__host__ __device__ __forceinline__ DD dd_div(DD a, double b) {
  const double q1 = a.hi / b;
  const DD p = two_prod(q1, b);
  const DD s = two_sum(a.hi, -p.hi);
  double e = s.lo - p.lo;
  e += a.lo;
  const double q2 = (s.hi + e) / b;
  return quick_two_sum(q1, q2);
}

// Division of two double-doubles (three quotient terms).
__host__ __device__ __forceinline__ DD dd_div_dd(DD a, DD b) {
  const double q1 = a.hi / b.hi;
  DD r = dd_add(a, dd_neg(dd_mul(b, q1)));
  const double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul(b, q2)));
  const double q3 = r.hi / b.hi;
  return dd_add(quick_two_sum(q1, q2), DD{q3, 0.});
}

// Square root of a non-negative double-double, one Newton correction.
__host__ __device__ __forceinline__ DD dd_sqrt(DD a) {
  if (!(a.hi > 0.)) return DD{0., 0.};
  const double s = sqrt(a.hi);
  const DD e = dd_add(a, dd_neg(two_prod(s, s)));
  return quick_two_sum(s, e.hi / (2.0 * s));
}

__host__ __device__ __forceinline__ double dd_value(DD a) { return a.hi + a.lo; }

}  // namespace aprl_gpu
