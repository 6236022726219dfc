// Correctly rounded log, sin, cos and acos in double precision, computed in double-double
// arithmetic, for the exact entries of GR (best/tgetgr.f:67-112 self blocks, best/triangleint.f:198-206
// pair integrals).
//
// Why: the self blocks are rotated to the lab frame (tgetgr.f:136-145) with heavy cancellation in
// their off-diagonal entries, so a one-ulp difference in a transcendental function becomes many
// ulps in GR; and each pair entry sums 21 logs.  These functions return the correctly rounded
// result (to ~2^-100 relative before the final rounding), so the GPU's entries are a fixed function
// of the input, equal bit for bit to TGETGR's arithmetic evaluated with correctly rounded functions.
// glibc's functions, which the reference uses, are not correctly rounded everywhere (its log is off
// by one ulp on about 0.15 % of arguments); entries differ from the reference's exactly where that
// happens.
//
// Methods (published, restated here from the mathematics):
//   double-double arithmetic: Dekker's and Knuth's error-free sum and product (T. J. Dekker,
//     "A floating-point technique for extending the available precision", Numer. Math. 18, 1971;
//     D. Knuth, TAOCP vol. 2, 4.2.2), the product via fma; division by long division in three
//     partial quotients (Hida, Li, Bailey, "Library for double-double and quad-double arithmetic").
//   log x = e ln 2 + 2 atanh((m - 1)/(m + 1)), m in [1/sqrt 2, sqrt 2), atanh by its Taylor series
//     (cr_log: the accurate phase).
//   cr_log_tab: Ziv's two-phase strategy (A. Ziv, "Fast evaluation of elementary mathematical
//     functions with correctly rounded last bit", ACM TOMS 17, 1991).  The fast phase is Tang's
//     table-driven reduction (logtab.h, gen_logtab.py) with a short series for log1p of the exact
//     reduced argument, evaluated to a relative error below 2^-74; when the result lies within
//     2^-72 of a rounding boundary, cr_log decides.
//   sin, cos: x - k pi/2 with pi/2 in three doubles, then the Taylor series of sin and cos.
//   acos: one Newton step on cos(theta) = x from the hardware acos, in double-double.
// Everything here must be compiled without contraction of a*b+c (-fmad=false / -ffp-contract=off):
// the error-free transformations depend on each operation rounding on its own.
#pragma once

#include <cmath>
#include <cstring>
#ifndef __CUDACC__
#define BGPU_HD inline
#define BGPU_HD_NOINLINE static inline
#define BGPU_LOGTAB_STORAGE static const
#else
#define BGPU_HD __host__ __device__ __forceinline__
#define BGPU_HD_NOINLINE static __host__ __device__ __noinline__
#define BGPU_LOGTAB_STORAGE static __device__ const
#endif

#include "logtab.h"

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

// ln 2 in two doubles (to 2^-107; gen_logtab.py computes it exactly; ln 2 = 2 atanh(1/3) by the
// series above agrees, tests/test_ddmath.py)
BGPU_HD DD ln2() { return DD{kLn2DDHi, kLn2DDLo}; }

// log x in double-double, to about 2^-100 relative, for a positive, finite, normal x.
BGPU_HD DD log_dd(double x) {
  int e = 0;
  double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
  if (m < 0.70710678118654752440) {
    m = m * 2.0;
    e = e - 1;
  }
  // m in [1/sqrt 2, sqrt 2): f = (m-1)/(m+1), |f| <= 0.1716, f^2 <= 0.0295; 0.0295^22 < 2^-111
  const DD f = div(from(m - 1.0), two_sum(m, 1.0));
  const DD lm = two_atanh(f, 22);
  return add(mul_d(ln2(), (double)e), lm);
}

// Correctly rounded natural logarithm of a positive, finite, normal x.
BGPU_HD double cr_log(double x) {
  const DD r = log_dd(x);
  return r.hi + r.lo;
}

// The accurate phase, kept out of line: the fast phase below needs it about once in 2^18 calls.
BGPU_HD_NOINLINE double cr_log_slow(double x) { return cr_log(x); }

BGPU_LOGTAB_STORAGE double kLogTab[3 * kLogTabN] = {BGPU_LOGTAB_ROWS};

BGPU_HD unsigned long long dbits(double x) {
#ifdef __CUDA_ARCH__
  return (unsigned long long)__double_as_longlong(x);
#else
  unsigned long long u;
  std::memcpy(&u, &x, 8);
  return u;
#endif
}
BGPU_HD double dfrom(unsigned long long u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x;
  std::memcpy(&x, &u, 8);
  return x;
#endif
}

// The fast phase: log x as hi + lo with |hi + lo - log x| < 2^-74 |log x| (the bound is derived
// term by term below; tests/test_ddmath.py measures it against cr_log).  tab: kLogTab, or a copy of
// it in shared memory.  x positive, finite (subnormals scaled first).
BGPU_HD DD log_fast_dd(double x, const double* tab) {
  unsigned long long u = dbits(x);
  long long kadj = 0;
  if (u < 0x0010000000000000ull) {  // subnormal: scale by 2^54 (exact)
    u = dbits(x * 18014398509481984.0);
    kadj = -54;
  }
  const unsigned long long t = u - kLogOff;
  const int i = (int)((t >> (52 - kLogTabBits)) & (kLogTabN - 1));
  const double kd = (double)(((long long)t >> 52) + kadj);
  const double z = dfrom(u - (t & 0xFFF0000000000000ull));  // x = 2^k z, z in [0.6865, 1.373)
  const double invc = tab[3 * i], lch = tab[3 * i + 1], lcl = tab[3 * i + 2];
  // r = z invc - 1 is exact (gen_logtab.py: |r| < 2^-7.95 and the integer-multiple argument)
  const double r = fma(z, invc, -1.0);
  // log1p r = r - r^2/2 + r^3/3 + r^4 Q(r): r^2 exactly, r^3/3 to ~2^-104, r^4 Q(r) in double
  // (relative error < 6 2^-53 of |r^4/4| < 2^-33.8, i.e. < 2^-84.2 absolute)
  const DD s = two_prod(r, r);
  DD c3 = two_prod(r, s.hi);
  c3.lo = c3.lo + r * s.lo;
  DD t3 = two_prod(c3.hi, kThirdHi);
  t3.lo = t3.lo + (c3.hi * kThirdLo + c3.lo * kThirdHi);
  const double r4 = s.hi * s.hi;
  const double q =
      r4 * (-0.25 + r * (0.2 + r * (-1.0 / 6.0 + r * (1.0 / 7.0 + r * (-0.125 + r * (1.0 / 9.0 + r * -0.1))))));
  // k ln2_hi is exact (42-bit ln2_hi, |k| < 2^11); the large terms are summed error-free, the small
  // ones (each below 2^-50 of the sum, or q) in one double; |log x| >= 2^-10 outside the subinterval
  // of 1 (where logc = 0 and log x ~ r), so the absolute errors above stay below 2^-74 relative
  const DD A = two_sum(kd * kLn2Hi42, lch);
  const DD B = two_sum(A.hi, r);
  const DD C = two_sum(B.hi, -0.5 * s.hi);
  const DD D = two_sum(C.hi, t3.hi);
  double lo = A.lo + B.lo + C.lo + D.lo + (kd * kLn2Lo + lcl - 0.5 * s.lo + t3.lo);
  lo = lo + q;
  return fast_two_sum(D.hi, lo);
}

// Correctly rounded natural logarithm (Ziv): the fast phase, and the accurate phase cr_log when the
// fast result lies within 2^-72 relative of a rounding boundary.  Zero, negative, infinite and NaN
// arguments return the IEEE special values of the platform's log (the same on every IEEE libm).
BGPU_HD double cr_log_tab(double x, const double* tab) {
  if (!(x > 0.0) || dbits(x) >= 0x7FF0000000000000ull) return log(x);
  const DD y = log_fast_dd(x, tab);
  const double e = fabs(y.hi) * 0x1p-72;
  const double a = y.hi + (y.lo + e), b = y.hi + (y.lo - e);
  if (a == b) return a;
  return cr_log_slow(x);
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
