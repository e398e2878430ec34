// physics.cuh -- ideal-gas EoS, conservative->primitive, flux splitting, BC point fluxes.
//
// Every expression keeps the reference's operand order and grouping, so that the
// build compiled without FMA contraction (kernels_exact.cu) returns the same bits
// as the reference compiled for x86-64 SSE2.  Citations are to juncas/NUC3d src/.
#pragma once
#include "common.h"

namespace nuc3d {
namespace NUC3D_NS {

__device__ __forceinline__ double sq(double x) { return x * x; }

// a / b.  The reference-order build divides with IEEE division.  The throughput build
// uses a branch-free quotient for finite, normal b: the PTX reciprocal approximation
// x0 ~ 1/b (relative error e0), one Newton-Raphson step x1 = x0 + x0 (1 - b x0)
// (error e0^2), q = a x1, then Markstein's residual correction q + (a - b q) x1, whose
// relative error is of order e0^4 plus the final rounding (P. Markstein, IBM J. Res.
// Dev. 34(1), 1990).  Zero, infinite or NaN b gives a non-finite result, which the
// state checks report as they do for IEEE division.
__device__ __forceinline__ double qdiv(double a, double b) {
#if NUC3D_FAST
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(b));
  x = fma(x, fma(-b, x, 1.0), x);
  const double q = a * x;
  return fma(fma(-b, q, a), x, q);
#else
  return a / b;
#endif
}

// pow(x, 1.5), correctly rounded in all but astronomically rare cases:
// s = sqrt(x); the FMA residual r = x - s*s is exact; sqrt(x) ~= s + r/(2s);
// x*s is split exactly (TwoProduct with FMA) and the small terms are added last.
// The oracle evaluates Sutherland's pow(T, 1.5) (src/physicsModel.cpp:226) with
// the same sequence of IEEE operations (oracle/pow_cr.c).
__device__ __forceinline__ double pow15(double x) {
  if (!(x > 1.0e-300 && x < 1.0e300)) return pow(x, 1.5);
  double s = sqrt(x);
  double r = fma(-s, s, x);
  double e = r / (2.0 * s);
  double hi = x * s;
  double lo = fma(x, s, -hi);
  double t = x * e;
  return hi + (lo + t);
}

// ---- pow(x, y) for the energy reset's pow(rho, gamma) (src/physicsModel.cpp:329) ----
// Double-double arithmetic (Dekker 1971; Knuth's TwoSum; the add, multiply and divide of
// Hida, Li & Bailey's QD library, 2001), every operation an explicit IEEE intrinsic so that
// neither build contracts or reorders it:
//   log x = e ln2 + log m, x = m 2^e, m in [sqrt(1/2), sqrt(2)),
//   log m = 2 s (1 + z/3 + z^2/5 + ... + z^21/45), s = (m-1)/(m+1), z = s^2,
//   exp P = 2^k exp r, k = rint(P/ln2), r = P - k ln2, |r| <= 0.347, with
//   exp r = 1 + r(1 + r/2(1 + r/3(... (1 + r/24)))) (the Taylor sum to r^24/24!),
// with ln2 as the double-double (0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56).  The
// result is the correctly rounded x^y unless x^y lies within about 2^-100 of a rounding
// midpoint; the oracle evaluates the same operation sequence in C, so both return the same
// bits.  Out of line: it runs only in the rare reset branch.
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  return {s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb))};
}
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ DD dd_add(DD x, DD y) {
  DD s = dd_two_sum(x.hi, y.hi);
  const DD t = dd_two_sum(x.lo, y.lo);
  double e = __dadd_rn(s.lo, t.hi);
  s = dd_fast_two_sum(s.hi, e);
  e = __dadd_rn(s.lo, t.lo);
  return dd_fast_two_sum(s.hi, e);
}
__device__ __forceinline__ DD dd_neg(DD x) { return {-x.hi, -x.lo}; }
__device__ __forceinline__ DD dd_mul(DD x, DD y) {
  const DD p = dd_two_prod(x.hi, y.hi);
  const double c = __dmul_rn(x.hi, y.lo), d = __dmul_rn(x.lo, y.hi);
  return dd_fast_two_sum(p.hi, __dadd_rn(p.lo, __dadd_rn(c, d)));
}
__device__ __forceinline__ DD dd_mul_d(DD x, double b) {
  const DD p = dd_two_prod(x.hi, b);
  return dd_fast_two_sum(p.hi, __dadd_rn(p.lo, __dmul_rn(x.lo, b)));
}
__device__ __forceinline__ DD dd_div_d(DD x, double b) {
  const double q1 = __ddiv_rn(x.hi, b);
  const DD p = dd_two_prod(q1, b);
  const double r = __dadd_rn(__dsub_rn(__dsub_rn(x.hi, p.hi), p.lo), x.lo);
  return dd_fast_two_sum(q1, __ddiv_rn(r, b));
}
__device__ __forceinline__ DD dd_div(DD x, DD y) {
  const double q1 = __ddiv_rn(x.hi, y.hi);
  DD r = dd_add(x, dd_neg(dd_mul_d(y, q1)));
  const double q2 = __ddiv_rn(r.hi, y.hi);
  r = dd_add(r, dd_neg(dd_mul_d(y, q2)));
  const double q3 = __ddiv_rn(r.hi, y.hi);
  return dd_add(dd_fast_two_sum(q1, q2), DD{q3, 0.0});
}

__device__ __noinline__ double cr_pow(double x, double y) {
  if (!(x > 0x1p-1000 && x < 0x1p1000) || !(fabs(y) < 0x1p20)) return pow(x, y);
  if (x == 1.0 || y == 0.0) return 1.0;
  const DD ln2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
  int e;
  double m = frexp(x, &e);
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = __dmul_rn(m, 2.0);
    e = e - 1;
  }
  const DD s = dd_div(DD{__dsub_rn(m, 1.0), 0.0}, dd_two_sum(m, 1.0));
  const DD z = dd_mul(s, s);
  DD t = dd_div_d(DD{1.0, 0.0}, 45.0);
#pragma unroll 1
  for (int k = 20; k >= 0; --k)
    t = dd_add(dd_div_d(DD{1.0, 0.0}, __dadd_rn(__dmul_rn(2.0, (double)k), 3.0)), dd_mul(z, t));
  const DD lm = dd_mul_d(dd_mul(s, dd_add(DD{1.0, 0.0}, dd_mul(z, t))), 2.0);
  const DD P = dd_mul_d(dd_add(dd_mul_d(ln2, (double)e), lm), y);
  if (!(fabs(P.hi) < 700.0)) return pow(x, y);
  const double k = rint(__ddiv_rn(P.hi, ln2.hi));
  const DD r = dd_add(P, dd_neg(dd_mul_d(ln2, k)));
  DD sum = {1.0, 0.0};
#pragma unroll 1
  for (int n = 24; n >= 1; --n) sum = dd_add(DD{1.0, 0.0}, dd_mul(dd_div_d(r, (double)n), sum));
  return ldexp(sum.hi, (int)k);
}

struct CellPrim {
  double rho, u, v, w, E, p, alpha;
  double q4;   // energy component of Q actually used (after the reset of :324-332)
  bool reset;  // the reset fired for this cell
};

// physicsModel::con2prim (src/physicsModel.cpp:307-356) with EoSIdealGasFWD (:981-1054).
__device__ __forceinline__ void con2prim(const double q[5], double jac, double gamma, double mach,
                                         CellPrim &s, unsigned &st) {
  double rho = q[0] * jac;
#if NUC3D_FAST
  // one reciprocal instead of three divisions; alpha from the same reciprocal below
  const double rinv = qdiv(1.0, rho);
  const double fj = rinv * jac;
  double u = q[1] * fj;
  double v = q[2] * fj;
  double w = q[3] * fj;
#else
  double u = q[1] / rho * jac;
  double v = q[2] / rho * jac;
  double w = q[3] / rho * jac;
#endif
  double E = q[4] * jac;
  double e0 = E - 0.5 * rho * (u * u + v * v + w * w);
  s.q4 = q[4];
  s.reset = e0 < 0.0;
  if (e0 < 0.0) {
    // the reference-order build takes the oracle's bits (cr_pow); the throughput build,
    // which agrees with the reference to round-off only, CUDA's pow (a call of a few
    // dozen instructions instead of the double-double's thousands, in a branch that some
    // 2% of the cells of a strong blast take every stage)
#if NUC3D_FAST
    const double pg = pow(rho, gamma);
#else
    const double pg = cr_pow(rho, gamma);
#endif
    E = (pg / ((gamma * mach * mach) * (gamma - 1.0)) + 0.5 * rho * (u * u + v * v + w * w));
    s.q4 = E / jac;
    st |= ST_ENERGY_RESET;
  }
  double p = (E - 0.5 * rho * (u * u + v * v + w * w)) * (gamma - 1.0);
  if (p < 0.0) st |= ST_NEG_PRESSURE;
  s.rho = rho;
  s.u = u;
  s.v = v;
  s.w = w;
  s.E = E;
  s.p = p;
#if NUC3D_FAST
  s.alpha = sqrt(fabs(gamma * p * rinv));
#else
  s.alpha = sqrt(fabs(gamma * p / rho));
#endif
}

// EoSIdealGasgetTemp (src/physicsModel.cpp:1020-1030)
__device__ __forceinline__ double temperature(double rho, double p, double gamma, double mach) {
  return gamma * mach * mach * p / rho;
}

// getMachL/R (src/physicsModel.cpp:803-828); identical for AUSMp (:891-916)
__device__ __forceinline__ double mach_l(double m) {
  return fabs(m) < 1.0 ? 0.25 * sq(m + 1.0) + 0.125 * sq(m * m - 1) : 0.50 * (m + fabs(m));
}
__device__ __forceinline__ double mach_r(double m) {
  return fabs(m) < 1.0 ? -0.25 * sq(m - 1.0) - 0.125 * sq(m * m - 1) : 0.50 * (m - fabs(m));
}
// getPressureL/R (:830-850)
__device__ __forceinline__ double pres_l(double m, double p) {
  return fabs(m) < 1.0 ? p * (m + 1.0) / 2.0 : 0.50 * p * (m + fabs(m)) / m;
}
__device__ __forceinline__ double pres_r(double m, double p) {
  return fabs(m) < 1.0 ? -p * (m - 1.0) / 2.0 : 0.5 * p * (m - fabs(m)) / m;
}
// getPressureLp/Rp (:918-938)
__device__ __forceinline__ double pres_lp(double m, double p) {
  return fabs(m) < 1.0 ? p * (0.25 * sq(m + 1.0) * (2.0 - m) + 0.1875 * m * sq(m * m - 1.0))
                       : 0.50 * p * (m + fabs(m)) / m;
}
__device__ __forceinline__ double pres_rp(double m, double p) {
  return fabs(m) < 1.0 ? p * (0.25 * sq(m - 1.0) * (2.0 + m) - 0.1875 * m * sq(m * m - 1.0))
                       : 0.5 * p * (m - fabs(m)) / m;
}

// Cell flux splitting along one computational direction with metric (xx, xy, xz):
// physicsModel::RiemannSolver's per-cell body (src/physicsModel.cpp:557-597) calling
// RiemannLF (:940-979), RiemannAUSM (:762-801) or RiemannAUSMp (:852-889).
// Q holds U/J (energy after the reset); fp/fn are F+/F- of (F/J).
__device__ __forceinline__ void split_cell(int riemann, const double Q[5], const CellPrim &s,
                                           double xx, double xy, double xz, double jac,
                                           double fp[5], double fn[5]) {
  double theta = sqrt(xx * xx + xy * xy + xz * xz);
  double U0 = (xx * s.u + xy * s.v + xz * s.w);
  double a0 = s.alpha * theta;
  double p = s.p;
#if NUC3D_FAST
  // p/J once: every pressure term of the split divides by the same Jacobian
  const double pj = qdiv(p, jac);
#endif
  if (riemann == RIE_LF) {
    double M = fabs(U0) + a0;
    double f0 = U0 * Q[0];
#if NUC3D_FAST
    double f1 = U0 * Q[1] + xx * pj;
    double f2 = U0 * Q[2] + xy * pj;
    double f3 = U0 * Q[3] + xz * pj;
    double f4 = U0 * (Q[4] + pj);
#else
    double f1 = U0 * Q[1] + xx * p / jac;
    double f2 = U0 * Q[2] + xy * p / jac;
    double f3 = U0 * Q[3] + xz * p / jac;
    double f4 = U0 * (Q[4] + p / jac);
#endif
    fp[0] = 0.5 * (f0 + M * Q[0]);
    fp[1] = 0.5 * (f1 + M * Q[1]);
    fp[2] = 0.5 * (f2 + M * Q[2]);
    fp[3] = 0.5 * (f3 + M * Q[3]);
    fp[4] = 0.5 * (f4 + M * Q[4]);
    fn[0] = 0.5 * (f0 - M * Q[0]);
    fn[1] = 0.5 * (f1 - M * Q[1]);
    fn[2] = 0.5 * (f2 - M * Q[2]);
    fn[3] = 0.5 * (f3 - M * Q[3]);
    fn[4] = 0.5 * (f4 - M * Q[4]);
    return;
  }
  double m = qdiv(U0, a0);
  double mp = mach_l(m), mn = mach_r(m);
  double pp, pn;
#if NUC3D_FAST
  // split pressures as fractions of p/J: pp/J = p/J * (pp/p); supersonic (pp/p) is 1 or 0
  if (riemann == RIE_AUSM) {
    pp = fabs(m) < 1.0 ? pj * (m + 1.0) * 0.5 : (m > 0.0 ? pj : 0.0);
    pn = fabs(m) < 1.0 ? -pj * (m - 1.0) * 0.5 : (m < 0.0 ? pj : 0.0);
  } else {
    pp = fabs(m) < 1.0 ? pj * (0.25 * sq(m + 1.0) * (2.0 - m) + 0.1875 * m * sq(m * m - 1.0))
                       : (m > 0.0 ? pj : 0.0);
    pn = fabs(m) < 1.0 ? pj * (0.25 * sq(m - 1.0) * (2.0 + m) - 0.1875 * m * sq(m * m - 1.0))
                       : (m < 0.0 ? pj : 0.0);
  }
  const double ma = mp * a0, na = mn * a0;
  fp[0] = ma * Q[0];
  fp[1] = ma * Q[1] + xx * pp;
  fp[2] = ma * Q[2] + xy * pp;
  fp[3] = ma * Q[3] + xz * pp;
  fp[4] = ma * Q[4] + ma * pj;
  fn[0] = na * Q[0];
  fn[1] = na * Q[1] + xx * pn;
  fn[2] = na * Q[2] + xy * pn;
  fn[3] = na * Q[3] + xz * pn;
  fn[4] = na * Q[4] + na * pj;
  return;
#endif
  if (riemann == RIE_AUSM) {
    pp = pres_l(m, p);
    pn = pres_r(m, p);
  } else {
    pp = pres_lp(m, p);
    pn = pres_rp(m, p);
  }
  fp[0] = mp * a0 * Q[0];
  fp[1] = mp * a0 * Q[1] + xx * pp / jac;
  fp[2] = mp * a0 * Q[2] + xy * pp / jac;
  fp[3] = mp * a0 * Q[3] + xz * pp / jac;
  fp[4] = mp * a0 * Q[4] + mp * a0 * p / jac;
  fn[0] = mn * a0 * Q[0];
  fn[1] = mn * a0 * Q[1] + xx * pn / jac;
  fn[2] = mn * a0 * Q[2] + xy * pn / jac;
  fn[3] = mn * a0 * Q[3] + xz * pn / jac;
  fn[4] = mn * a0 * Q[4] + mn * a0 * p / jac;
}

// |U| + c|grad xi| of one cell along one direction (src/physicsModel.cpp:557-597).
__device__ __forceinline__ double eigen_cell(const CellPrim &s, double xx, double xy, double xz) {
  double theta = sqrt(xx * xx + xy * xy + xz * xz);
  double U0 = (xx * s.u + xy * s.v + xz * s.w);
  return fabs(U0) + s.alpha * theta;
}

// physicsModel::solveRiemannPoint{LF,AUSM,AUSMp} (src/physicsModel.cpp:1159-1398):
// split flux of a primitive state q = (rho,u,v,w,p) at a cell's metric.  side 0
// returns the left split (fluxl), side 1 the right split (fluxr).
__device__ __forceinline__ void split_point(int riemann, const double q[5], double jac, double xx,
                                            double xy, double xz, double gamma, int side,
                                            double out[5], unsigned &st) {
  const double rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  double _rho = rho;
  double _rhou = rho * u;
  double _rhov = rho * v;
  double _rhow = rho * w;
  double _E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
  double _p = (_E - 0.5 * rho * (u * u + v * v + w * w)) * (gamma - 1.0);
  if (_p < 0.0) st |= ST_NEG_PRESSURE;
  double _alpha = sqrt(fabs(gamma * _p / rho));
  double theta = sqrt(xx * xx + xy * xy + xz * xz);
  double alpha = _alpha * theta;
  double U0 = (xx * u + xy * v + xz * w);
  double mach = U0 / alpha;
  if (riemann == RIE_LF) {
    double M = fabs(U0) + alpha;
    double f0 = U0 * _rho / jac;
    double f1 = U0 * _rhou / jac + xx * p / jac;
    double f2 = U0 * _rhov / jac + xy * p / jac;
    double f3 = U0 * _rhow / jac + xz * p / jac;
    double f4 = U0 * (_E / jac + p / jac);
    if (side == 0) {
      out[0] = 0.5 * (f0 + M * _rho / jac);
      out[1] = 0.5 * (f1 + M * _rhou / jac);
      out[2] = 0.5 * (f2 + M * _rhov / jac);
      out[3] = 0.5 * (f3 + M * _rhow / jac);
      out[4] = 0.5 * (f4 + M * _E / jac);
    } else {
      out[0] = 0.5 * (f0 - M * _rho / jac);
      out[1] = 0.5 * (f1 - M * _rhou / jac);
      out[2] = 0.5 * (f2 - M * _rhov / jac);
      out[3] = 0.5 * (f3 - M * _rhow / jac);
      out[4] = 0.5 * (f4 - M * _E / jac);
    }
    return;
  }
  double mm, pm;
  if (side == 0) {
    mm = mach_l(mach);
    pm = riemann == RIE_AUSM ? pres_l(mach, p) : pres_lp(mach, p);
  } else {
    mm = mach_r(mach);
    pm = riemann == RIE_AUSM ? pres_r(mach, p) : pres_rp(mach, p);
  }
  out[0] = mm * alpha * _rho / jac;
  out[1] = mm * alpha * _rhou / jac + xx * pm / jac;
  out[2] = mm * alpha * _rhov / jac + xy * pm / jac;
  out[3] = mm * alpha * _rhow / jac + xz * pm / jac;
  out[4] = mm * alpha * _E / jac + mm * alpha * p / jac;
}

}  // namespace NUC3D_NS
}  // namespace nuc3d
