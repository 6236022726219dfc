// Correctly rounded log, sin, cos and acos in double precision, computed in double-double
// arithmetic, for the O(N) exact self blocks of GR (best/tgetgr.f:67-112).
//
// Why: the self blocks are rotated to the lab frame (tgetgr.f:136-145) with heavy cancellation in
// their off-diagonal entries, so a one-ulp difference in a transcendental function becomes many
// ulps in GR.  glibc's functions, which the reference uses, return the correctly rounded result for
// almost every argument; these do too (to ~2^-100 relative before the final rounding), so the GPU's
// self blocks come out bit for bit the same wherever glibc rounds correctly.
//
// Methods (published, restated here from the mathematics):
//   double-double arithmetic: Dekker's and Knuth's error-free sum and product (T. J. Dekker,
//     "A floating-point technique for extending the available precision", Numer. Math. 18, 1971;
//     D. Knuth, TAOCP vol. 2, 4.2.2), the product via fma; division by long division in three
//     partial quotients (Hida, Li, Bailey, "Library for double-double and quad-double arithmetic").
//   log x = e ln 2 + 2 atanh((m - 1)/(m + 1)), m in [1/sqrt 2, sqrt 2), atanh by its Taylor series;
//     ln 2 itself = 2 atanh(1/3) by the same series.
//   sin, cos: x - k pi/2 with pi/2 in three doubles, then the Taylor series of sin and cos.
//   acos: one Newton step on cos(theta) = x from the hardware acos, in double-double.
// Everything here must be compiled without contraction of a*b+c (-fmad=false / -ffp-contract=off):
// the error-free transformations depend on each operation rounding on its own.
#pragma once

#ifndef __CUDACC__
#include <cmath>
#define BGPU_HD inline
#else
#define BGPU_HD __host__ __device__ __forceinline__
#endif

namespace bgpu {
namespace dd {

struct DD {
  double hi, lo;
};

BGPU_HD DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double err = (a - (s - bb)) + (b - bb);
  return DD{s, err};
}
BGPU_HD DD fast_two_sum(double a, double b) {
  const double s = a + b;
  return DD{s, b - (s - a)};
}
BGPU_HD DD two_prod(double a, double b) {
  const double p = a * b;
  return DD{p, fma(a, b, -p)};
}
BGPU_HD DD add(DD x, DD y) {
  DD s = two_sum(x.hi, y.hi);
  DD t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
BGPU_HD DD neg(DD x) { return DD{-x.hi, -x.lo}; }
BGPU_HD DD sub(DD x, DD y) { return add(x, neg(y)); }
BGPU_HD DD mul(DD x, DD y) {
  DD p = two_prod(x.hi, y.hi);
  p.lo += x.hi * y.lo + x.lo * y.hi;
  return fast_two_sum(p.hi, p.lo);
}
BGPU_HD DD mul_d(DD x, double y) {
  DD p = two_prod(x.hi, y);
  p.lo += x.lo * y;
  return fast_two_sum(p.hi, p.lo);
}
BGPU_HD DD div(DD x, DD y) {
  const double q1 = x.hi / y.hi;
  DD r = sub(x, mul_d(y, q1));
  const double q2 = r.hi / y.hi;
  r = sub(r, mul_d(y, q2));
  const double q3 = r.hi / y.hi;
  DD q = fast_two_sum(q1, q2);
  return add(q, DD{q3, 0.0});
}
BGPU_HD DD from(double a) { return DD{a, 0.0}; }

// 2 atanh(f) = 2 (f + f^3/3 + f^5/5 + ...) for |f| <= 1/3, terms to f^(2K+1).
BGPU_HD DD two_atanh(DD f, int K) {
  const DD f2 = mul(f, f);
  DD p = div(from(1.0), from((double)(2 * K + 1)));
  for (int k = K - 1; k >= 0; --k) p = add(mul(p, f2), div(from(1.0), from((double)(2 * k + 1))));
  return mul_d(mul(f, p), 2.0);
}

BGPU_HD DD ln2() {
  // ln 2 = 2 atanh(1/3); (1/9)^36 < 2^-110
  return two_atanh(div(from(1.0), from(3.0)), 36);
}

// Correctly rounded natural logarithm of a positive, finite, normal x.
BGPU_HD double cr_log(double x) {
  int e = 0;
  double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
  if (m < 0.70710678118654752440) {
    m = m * 2.0;
    e = e - 1;
  }
  // m in [1/sqrt 2, sqrt 2): f = (m-1)/(m+1), |f| <= 0.1716, f^2 <= 0.0295; 0.0295^22 < 2^-111
  const DD f = div(from(m - 1.0), two_sum(m, 1.0));
  const DD lm = two_atanh(f, 22);
  const DD r = add(mul_d(ln2(), (double)e), lm);
  return r.hi + r.lo;
}

// pi/2 as three doubles (sum exact to about 2^-160).
constexpr double kPio2A = 1.5707963267948966192e+00;   // 0x3FF921FB54442D18
constexpr double kPio2B = 6.1232339957367660359e-17;   // 0x3C91A62633145C07
constexpr double kPio2C = -1.4973849048591698329e-33;  // 0xB91F1976B7ED8FBC

// x - k pi/2 in double-double, k = nearest integer to x / (pi/2); |x| <= ~8 here.
BGPU_HD DD reduce_pio2(double x, int* quadrant) {
  const double k = rint(x * 0.63661977236758134308);
  DD r = sub(from(x), two_prod(k, kPio2A));
  r = sub(r, two_prod(k, kPio2B));
  r = sub(r, from(k * kPio2C));
  *quadrant = ((int)k) & 3;
  return r;
}

// sin r and cos r by Taylor series for |r| <= ~0.8 (terms to r^31 / 31!).
BGPU_HD void sincos_taylor(DD r, DD* s, DD* c) {
  const DD r2 = mul(r, r);
  // sin: r (1 - r^2/(2 3) (1 - r^2/(4 5) (1 - ...)))
  DD ps = from(1.0);
  for (int n = 31; n >= 3; n -= 2) ps = sub(from(1.0), div(mul(r2, ps), from((double)(n * (n - 1)))));
  *s = mul(r, ps);
  DD pc = from(1.0);
  for (int n = 32; n >= 2; n -= 2) pc = sub(from(1.0), div(mul(r2, pc), from((double)(n * (n - 1)))));
  *c = pc;
}

BGPU_HD void dd_sincos(double x, DD* s, DD* c) {
  int q = 0;
  const DD r = reduce_pio2(x, &q);
  DD sr, cr;
  sincos_taylor(r, &sr, &cr);
  switch (q) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = neg(sr); break;
    case 2: *s = neg(sr); *c = neg(cr); break;
    default: *s = neg(cr); *c = sr; break;
  }
}

BGPU_HD double cr_sin(double x) {
  DD s, c;
  dd_sincos(x, &s, &c);
  return s.hi + s.lo;
}
BGPU_HD double cr_cos(double x) {
  DD s, c;
  dd_sincos(x, &s, &c);
  return c.hi + c.lo;
}

// Correctly rounded acos for |x| < 1: one Newton step on cos(theta) - x = 0 in double-double from
// the hardware's acos (which is within a few ulp), theta1 = theta0 + (cos theta0 - x) / sin theta0.
BGPU_HD double cr_acos(double x) {
  const double t0 = acos(x);
  DD s, c;
  dd_sincos(t0, &s, &c);
  const DD d = sub(c, from(x));
  const double corr = (d.hi + d.lo) / (s.hi + s.lo);
  const DD t = two_sum(t0, corr);
  return t.hi + t.lo;
}

}  // namespace dd
}  // namespace bgpu
