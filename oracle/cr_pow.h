/*
 * cr_pow.h -- pow(x, y) for x > 0 in double-double arithmetic, for the oracle build.
 *
 * TEST INFRASTRUCTURE ONLY (included by pow_cr.c and nuc3d_oracle.c).
 *
 * The reference resets the energy of a cell whose internal energy went negative with
 * pow(rho, gamma) (src/physicsModel.cpp:329).  glibc's pow is accurate to about 0.52
 * ulp but not correctly rounded, and CUDA's pow is a different algorithm again, so
 * the oracle build and the GPU both evaluate this pow with the method below: the same
 * sequence of IEEE-754 basic operations (+, -, *, /, fma, each correctly rounded), so
 * any IEEE machine returns the same bits.  Its result is the correctly rounded x^y
 * unless x^y lies within about 2^-100 (relative) of a rounding midpoint.
 *
 * Method (double-double arithmetic: Dekker 1971, Knuth's TwoSum, and the add,
 * multiply and divide of Hida, Li & Bailey's QD library, 2001):
 *   log x = e ln2 + log m, x = m 2^e with m in [sqrt(1/2), sqrt(2)),
 *   log m = 2 atanh(s) = 2 s (1 + z/3 + z^2/5 + ...), s = (m-1)/(m+1), z = s^2
 *           (22 terms: z <= 0.0295, the remainder is below 2^-110);
 *   P = y log x;  exp P = 2^k exp r, k = rint(P / ln2), r = P - k ln2, |r| <= 0.347,
 *   exp r = 1 + r(1 + r/2(1 + r/3(... (1 + r/24)))), the Taylor sum to r^24/24!
 *           (the remainder is below 2^-115).
 * ln2 enters as the double-double (0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56).
 * Every constant 1/(2k+3) and every r/n is formed by the same double-double division.
 */
#ifndef NUC3D_CR_POW_H
#define NUC3D_CR_POW_H
#include <math.h>

typedef struct {
  double hi, lo;
} crp_dd;

static crp_dd crp_two_sum(double a, double b) {
  crp_dd r;
  double s = a + b;
  double bb = s - a;
  r.hi = s;
  r.lo = (a - (s - bb)) + (b - bb);
  return r;
}
static crp_dd crp_fast_two_sum(double a, double b) {
  crp_dd r;
  double s = a + b;
  r.hi = s;
  r.lo = b - (s - a);
  return r;
}
static crp_dd crp_two_prod(double a, double b) {
  crp_dd r;
  double p = a * b;
  r.hi = p;
  r.lo = fma(a, b, -p);
  return r;
}
static crp_dd crp_add(crp_dd x, crp_dd y) {
  crp_dd s = crp_two_sum(x.hi, y.hi);
  crp_dd t = crp_two_sum(x.lo, y.lo);
  double e = s.lo + t.hi;
  s = crp_fast_two_sum(s.hi, e);
  e = s.lo + t.lo;
  return crp_fast_two_sum(s.hi, e);
}
static crp_dd crp_neg(crp_dd x) {
  x.hi = -x.hi;
  x.lo = -x.lo;
  return x;
}
static crp_dd crp_mul(crp_dd x, crp_dd y) {
  crp_dd p = crp_two_prod(x.hi, y.hi);
  double c = x.hi * y.lo;
  double d = x.lo * y.hi;
  double e = p.lo + (c + d);
  return crp_fast_two_sum(p.hi, e);
}
static crp_dd crp_mul_d(crp_dd x, double b) {
  crp_dd p = crp_two_prod(x.hi, b);
  double c = x.lo * b;
  double e = p.lo + c;
  return crp_fast_two_sum(p.hi, e);
}
static crp_dd crp_div_d(crp_dd x, double b) {
  double q1 = x.hi / b;
  crp_dd p = crp_two_prod(q1, b);
  double r = ((x.hi - p.hi) - p.lo) + x.lo;
  double q2 = r / b;
  return crp_fast_two_sum(q1, q2);
}
static crp_dd crp_div(crp_dd x, crp_dd y) {
  double q1 = x.hi / y.hi;
  crp_dd r = crp_add(x, crp_neg(crp_mul_d(y, q1)));
  double q2 = r.hi / y.hi;
  r = crp_add(r, crp_neg(crp_mul_d(y, q2)));
  double q3 = r.hi / y.hi;
  crp_dd q = crp_fast_two_sum(q1, q2);
  crp_dd t;
  t.hi = q3;
  t.lo = 0.0;
  return crp_add(q, t);
}
static crp_dd crp_d(double a) {
  crp_dd r;
  r.hi = a;
  r.lo = 0.0;
  return r;
}

/* log x for finite x > 0 (normal) */
static crp_dd crp_log(double x) {
  const crp_dd ln2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
  int e;
  double m = frexp(x, &e); /* x = m 2^e, m in [0.5, 1) */
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = m * 2.0;
    e = e - 1;
  }
  crp_dd num = crp_d(m - 1.0); /* exact (Sterbenz) */
  crp_dd den = crp_two_sum(m, 1.0);
  crp_dd s = crp_div(num, den);
  crp_dd z = crp_mul(s, s);
  crp_dd t = crp_div_d(crp_d(1.0), 45.0);
  for (int k = 20; k >= 0; --k) t = crp_add(crp_div_d(crp_d(1.0), 2.0 * k + 3.0), crp_mul(z, t));
  crp_dd lm = crp_mul_d(crp_mul(s, crp_add(crp_d(1.0), crp_mul(z, t))), 2.0);
  return crp_add(crp_mul_d(ln2, (double)e), lm);
}

/* exp P for |P| well inside the double range */
static double crp_exp_round(crp_dd P) {
  const crp_dd ln2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
  double k = rint(P.hi / ln2.hi);
  crp_dd r = crp_add(P, crp_neg(crp_mul_d(ln2, k)));
  crp_dd sum = crp_d(1.0);
  for (int n = 24; n >= 1; --n) sum = crp_add(crp_d(1.0), crp_mul(crp_div_d(r, (double)n), sum));
  return ldexp(sum.hi, (int)k);
}

/* x^y for finite x > 0 and finite y with x^y a normal double; NaN otherwise */
static double nuc3d_cr_pow(double x, double y) {
  if (!(x > 0x1p-1000 && x < 0x1p1000) || !(fabs(y) < 0x1p20)) return NAN;
  if (x == 1.0 || y == 0.0) return 1.0;
  crp_dd P = crp_mul_d(crp_log(x), y);
  if (!(fabs(P.hi) < 700.0)) return NAN;
  return crp_exp_round(P);
}

#endif /* NUC3D_CR_POW_H */
