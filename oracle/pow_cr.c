/*
 * pow_cr.c -- correctly rounded pow for the oracle build.
 *
 * TEST INFRASTRUCTURE ONLY.  The NUC3d reference evaluates squares through
 * std::pow with a run-time exponent p = 2.0 (src/weno5js.cpp:7-8,97-99,
 * src/weno5z.cpp:98-100, src/crweno5.cpp:113-115) and Sutherland's law through
 * pow(T, 1.5) (src/physicsModel.cpp:226).  glibc's pow is accurate to about
 * 0.52 ulp but is not correctly rounded: pow(x, 2.0) differs from the correctly
 * rounded x*x in roughly 0.1% of inputs.  Linking this file into the reference
 * binary interposes `pow` so that
 *   pow(x, 2.0) == x*x                (the correctly rounded square), and
 *   pow(x, 1.5) == cr_pow15(x) below  (x*sqrt(x) with an exact-residual fix),
 *   pow(x, y) == nuc3d_cr_pow(x, y)   (cr_pow.h) for every other exponent and
 *                                      x > 0, which serves the energy reset's
 *                                      pow(rho, gamma) (src/physicsModel.cpp:329);
 * arguments outside cr_pow.h's domain still go to libm.  The GPU kernels evaluate
 * the same formulas, so the reference, the C restatement and the CUDA path can
 * be compared bit for bit.  The stock-libm reference build is kept beside this
 * one and the tests bound the difference between the two to round-off.
 *
 * cr_pow15 method: s = sqrt(x) (IEEE correctly rounded); r = fma(-s, s, x) is
 * the exact residual x - s^2; sqrt(x) = s + r/(2s) + O(r^2); the product
 * x*s is split exactly as hi + lo with an FMA (Dekker/Ogita-Rump-Oishi
 * TwoProduct), and the small terms are added to hi last.  Only IEEE basic
 * operations are used, so any IEEE-754 machine with FMA returns the same bits.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "cr_pow.h"

static double (*libm_pow)(double, double) = 0;

double nuc3d_cr_pow15(double x) {
  double s = sqrt(x);
  double r = fma(-s, s, x);
  double e = r / (2.0 * s);
  double hi = x * s;
  double lo = fma(x, s, -hi);
  double t = x * e;
  return hi + (lo + t);
}

double pow(double x, double y) {
  if (y == 2.0) return x * x;
  if (y == 1.5 && x > 0.0 && x < 1.0e300 && x > 1.0e-300) return nuc3d_cr_pow15(x);
  if (x > 0.0) {
    const double r = nuc3d_cr_pow(x, y);
    if (r == r) return r;
  }
  if (!libm_pow) {
    libm_pow = (double (*)(double, double))dlsym(RTLD_NEXT, "pow");
    if (!libm_pow) {
      fprintf(stderr, "pow_cr: cannot resolve libm pow\n");
      abort();
    }
  }
  return libm_pow(x, y);
}
