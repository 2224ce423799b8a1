// Exact ball integral of a compact bump source (the EXACT source mode).
//
// For the walk's ball B_r(y) and f(x) = A (1 - |x-c|^2/R^2)_+^2, the step's
// source integral is  int_{B_r} G_r(y, z) f(z) dz = N(|y-c|) - mean over the
// sphere |z-y| = r of N(|z-c|), where N is the bump's Newton potential
// (-Delta N = f).  This is the closed form of exact_bump_green,
// benchmarks/submission_study/study.cpp:53-77:
//
//   N(d)   = A R^3 (8/105) / d                                    d >= R
//          = A R^2 (1/6 - t^2/6 + t^4/10 - t^6/42),  t = d/R      d <  R
//   P(x)   = int_0^x s N(s) ds
//          = A R^4 (t^2/12 - t^4/24 + t^6/60 - t^8/336), t = min(x/R, 1)
//            + A R^3 (8/105) (x - R)  when x > R
//   mean   = A R^3 (8/105) / r          when the support lies inside the sphere
//          = N(r)                        when d < 1e-12 R (centred)
//          = (P(d + r) - P(|d - r|)) / (2 d r)   otherwise
//
// The reference evaluates in long double to tame the cancellations in
// P(d + r) - P(|d - r|) (small d r) and N - mean (small r).  Here the same
// formulas run in double-double arithmetic (a value as an unevaluated sum
// hi + lo of two doubles, ~106-bit significand; the error-free sum and
// product steps of Dekker 1971 and Knuth TAOCP vol. 2, 4.2.2, with the
// product's low part from one fused multiply-add), so the only rounding
// that matters is the final one to double.
#pragma once

namespace twos {

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD dd(double a) { return {a, 0.0}; }

// s + e = a + b exactly.
__device__ __forceinline__ DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
// s + e = a + b exactly, given |a| >= |b|.
__device__ __forceinline__ DD fast_two_sum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}
// p + e = a * b exactly.
__device__ __forceinline__ DD two_prod(double a, double b) {
  const double p = a * b;
  return {p, __fma_rn(a, b, -p)};
}

__device__ __forceinline__ DD operator+(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DD operator-(DD a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ DD operator-(DD a, DD b) { return a + (-b); }
__device__ __forceinline__ DD operator*(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return fast_two_sum(p.hi, p.lo);
}
// Long division: three quotient digits.
__device__ __forceinline__ DD operator/(DD a, DD b) {
  const double q1 = a.hi / b.hi;
  DD r = a - b * dd(q1);
  const double q2 = r.hi / b.hi;
  r = r - b * dd(q2);
  const double q3 = r.hi / b.hi;
  return fast_two_sum(q1, q2) + dd(q3);
}
__device__ __forceinline__ bool operator<(DD a, DD b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
__device__ __forceinline__ DD ddmin(DD a, DD b) { return b < a ? b : a; }
__device__ __forceinline__ DD ddabs(DD a) { return a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0) ? -a : a; }
__device__ __forceinline__ DD frac(double p, double q) { return dd(p) / dd(q); }

// Newton potential N(d) of the bump.
__device__ __forceinline__ DD bump_potential(DD d, DD R, DD A) {
  if (!(d < R)) return A * R * R * R * frac(8.0, 105.0) / d;
  const DD t = d / R, s = t * t;
  // 1/6 - s/6 + s^2/10 - s^3/42, Horner in s.
  const DD poly = ((s * (-frac(1.0, 42.0)) + frac(1.0, 10.0)) * s - frac(1.0, 6.0)) * s + frac(1.0, 6.0);
  return A * R * R * poly;
}

// P(x) = int_0^x s N(s) ds.
__device__ __forceinline__ DD potential_primitive(DD x, DD R, DD A) {
  const DD t = ddmin(x / R, dd(1.0)), s = t * t;
  // s/12 - s^2/24 + s^3/60 - s^4/336, Horner in s.
  const DD poly = (((s * (-frac(1.0, 336.0)) + frac(1.0, 60.0)) * s - frac(1.0, 24.0)) * s + frac(1.0, 12.0)) * s;
  DD v = A * R * R * R * R * poly;
  if (R < x) v = v + A * R * R * R * frac(8.0, 105.0) * (x - R);
  return v;
}

// The exact ball integral for a bump at distance d from the ball centre;
// sets `negative` when the difference is below -1e-11 max(1, |N(d)|)
// (study.cpp:74, which throws there).
__device__ double exact_bump_green(double d_, double r_, double R_, double A_, bool &negative) {
  if (d_ >= r_ + R_) return 0.0;
  const DD d = dd(d_), r = dd(r_), R = dd(R_), A = dd(A_);
  const DD at_center = bump_potential(d, R, A);
  DD mean;
  if (!(r < d + R))
    mean = A * R * R * R * frac(8.0, 105.0) / r;
  else if (d < R * dd(1e-12))
    mean = bump_potential(r, R, A);
  else
    mean = (potential_primitive(two_sum(d_, r_), R, A) - potential_primitive(ddabs(two_sum(d_, -r_)), R, A)) /
           (dd(2.0) * d * r);
  const DD value = at_center - mean;
  if (value.hi < -1e-11 * fmax(1.0, fabs(at_center.hi))) negative = true;
  return fmax(0.0, value.hi + value.lo);
}

}  // namespace twos
