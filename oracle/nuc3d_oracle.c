/*
 * nuc3d_oracle.c -- CPU restatement of NUC3d's per-block right-hand side and
 * TVD-RK3 update (the GPU path's correctness oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  It is loaded by the tests (ctypes) and by nothing
 * in the GPU product.  Parity is pinned: the tests require it to reproduce the
 * golden fixtures produced by the reference itself (tests/golden/) bit for bit.
 *
 * Structure follows the reference's passes, not the GPU's fused sweeps:
 *   con2prim over all cells            src/physicsModel.cpp:258-357 (+ EoS :981-1054)
 *   split fluxes per direction         src/physicsModel.cpp:420-760 (LF :940, AUSM :762, AUSMp :852)
 *   ghost slabs per face               neighbour: src/bufferData.cpp:103-239 +
 *                                      src/MPICommunicator.cpp:36-115; physical:
 *                                      src/boundaryConditions.cpp:95-1086 (+ point solvers
 *                                      src/physicsModel.cpp:1145-1398)
 *   line reconstruction                src/weno5js.cpp, src/weno5z.cpp, src/weno7js.cpp,
 *                                      src/reconstructionBoundaryScheme.cpp:52-463
 *   combine + difference               src/euler3d.cpp:23-54,143-241
 *   NS gradients, viscous fluxes, cd6  src/NaiverStokes3d.cpp:63-398,
 *                                      src/centraldifference6th.cpp, src/boundaryScheme.cpp
 *   RHS sum, dt                        src/euler3d.cpp:368-435, src/NaiverStokes3d.cpp:401-513
 *   TVD-RK3                            src/PDEData3d.cpp:152-170, src/TVD-RK3.cpp:16-137
 * Arithmetic is written in the reference's operand order; build with
 * -ffp-contract=off (oracle/Makefile).  pow(x, 2) is x*x, pow(T, 1.5) uses
 * the correctly rounded sequence of oracle/pow_cr.c, and the energy reset's
 * pow(rho, gamma) the double-double pow of oracle/cr_pow.h.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cr_pow.h"

enum { S_WENO5JS = 0, S_WENO5Z = 1, S_WENO7JS = 2, S_CRWENO5 = 3, S_HCCS = 4, S_WENO3JS = 5, S_UPWIND1 = 6,
       S_HCCS77 = 7 };
enum { V_CD6 = 0, V_CD2 = 1, V_CD8 = 2 };
enum { R_LF = 0, R_AUSM = 1, R_AUSMP = 2 };

typedef struct {
  int scheme[3];
  int riemann;
  int model; /* 0 Euler3d, 1 NavierStokes3d */
  int compat;
  int vis[3]; /* V_CD6 / V_CD2 / V_CD8 per direction (scheme_x/y/z_vis) */
  double gamma, mach, reynolds, prandtl, t_ref, t_inf, t_wall, cfl;
} oc_config;

/* bufferSize of a reconstruction scheme (src/fieldOperator.cpp:127-175) */
static int tilesize(int sch) {
  return (sch == S_WENO7JS || sch == S_HCCS || sch == S_HCCS77) ? 4
         : sch == S_WENO3JS ? 2 : sch == S_UPWIND1 ? 1 : 3;
}
/* bfsize = max of the three (src/block.cpp:506-507) */
static int ghost_width(const oc_config *c) {
  int m = 0;
  for (int d = 0; d < 3; ++d)
    if (tilesize(c->scheme[d]) > m) m = tilesize(c->scheme[d]);
  return m;
}

typedef struct {
  int n[3];
  int bc_type[6], bc_id[6];
  double bcv[6][5];
  const double *jac, *xi, *eta, *zeta, *dxyz; /* N, 3N, 3N, 3N, 9N (dxyz may be NULL) */
  double *q;                                  /* 5N: Q = U/J */
  double *rhs;                                /* 5N, may be NULL */
} oc_block;

/* ------------------------------------------------------------------ scalar kernels */
static double sq(double x) { return x * x; }

static double cr_pow15(double x) {
  if (!(x > 1.0e-300 && x < 1.0e300)) return pow(x, 1.5);
  double s = sqrt(x), r = fma(-s, s, x), e = r / (2.0 * s);
  double hi = x * s, lo = fma(x, s, -hi), t = x * e;
  return hi + (lo + t);
}

/* pow for the energy reset (src/physicsModel.cpp:329): cr_pow.h, libm outside its domain */
static double oc_pow(double x, double y) {
  const double r = nuc3d_cr_pow(x, y);
  return r == r ? r : pow(x, y);
}
/* exported for the tests: the oracle's pow(x, y) */
double oc_cr_pow(double x, double y) { return oc_pow(x, y); }

static const double A5[3][3] = {{1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0},
                                {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                                {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0}};
static const double A7[4][4] = {{-3.0 / 12.0, 13.0 / 12.0, -23.0 / 12.0, 25.0 / 12.0},
                                {1.0 / 12.0, -5.0 / 12.0, 13.0 / 12.0, 3.0 / 12.0},
                                {-1.0 / 12.0, 7.0 / 12.0, 7.0 / 12.0, -1.0 / 12.0},
                                {3.0 / 12.0, 13.0 / 12.0, -5.0 / 12.0, 1.0 / 12.0}};
static const double C5[3] = {0.1, 0.6, 0.3};
static const double C7[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
static const double G0 = 13.0 / 12.0, G1 = 1.0 / 4.0;
static const double CD6[3] = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
static const double CD4[2] = {2.0 / 3.0, -1.0 / 12.0};

/* WENO5 on the stencil f[0..4] (already oriented), src/weno5js.cpp:75-108 and
   src/weno5z.cpp:74-109; bug selects the interior is2 of src/weno5z.cpp:80. */
static double weno5(const double *f, int z, int bug) {
  double is0 = G0 * sq(f[0] - 2.0 * f[1] + f[2]) + G1 * sq(f[0] - 4.0 * f[1] + 3.0 * f[2]);
  double is1 = G0 * sq(f[1] - 2.0 * f[2] + f[3]) + G1 * sq(f[1] - f[3]);
  double is2 = G0 * sq(f[2] - 2.0 * f[3] + (bug ? f[3] : f[4])) + G1 * sq(3.0 * f[2] - 4.0 * f[3] + f[4]);
  double q0 = A5[0][0] * f[0] + A5[0][1] * f[1] + A5[0][2] * f[2];
  double q1 = A5[1][0] * f[1] + A5[1][1] * f[2] + A5[1][2] * f[3];
  double q2 = A5[2][0] * f[2] + A5[2][1] * f[3] + A5[2][2] * f[4];
  double a0, a1, a2;
  if (z) {
    double tau = fabs(is2 - is0);
    a0 = C5[0] * (1.0 + sq(tau / (is0 + 1.0e-6)));
    a1 = C5[1] * (1.0 + sq(tau / (is1 + 1.0e-6)));
    a2 = C5[2] * (1.0 + sq(tau / (is2 + 1.0e-6)));
  } else {
    a0 = C5[0] / sq(1.0e-6 + is0);
    a1 = C5[1] / sq(1.0e-6 + is1);
    a2 = C5[2] / sq(1.0e-6 + is2);
  }
  double s = a0 + a1 + a2;
  return a0 / s * q0 + a1 / s * q1 + a2 / s * q2;
}

/* WENO7-JS on f[0..6], src/weno7js.cpp:84-136; z: the WENO7-Z weights of hccs
   (tau7 = |is0 - is3|, src/hccs.cpp:125-137) */
static double weno7zs(const double *f, int z);
static double weno7(const double *f) { return weno7zs(f, 0); }
static double weno7zs(const double *f, int z) {
  double is[4];
  is[0] = f[0] * (547.0 * f[0] - 3882.0 * f[1] + 4642.0 * f[2] - 1854.0 * f[3]) +
          f[1] * (7043.0 * f[1] - 17246.0 * f[2] + 7042.0 * f[3]) +
          f[2] * (11003.0 * f[2] - 9402.0 * f[3]) + 2107.0 * f[3] * f[3];
  is[1] = f[1] * (267.0 * f[1] - 1642.0 * f[2] + 1602.0 * f[3] - 494.0 * f[4]) +
          f[2] * (2843.0 * f[2] - 5966.0 * f[3] + 1922.0 * f[4]) +
          f[3] * (3443.0 * f[3] - 2522.0 * f[4]) + 547.0 * f[4] * f[4];
  is[2] = f[2] * (547.0 * f[2] - 2522.0 * f[3] + 1922.0 * f[4] - 494.0 * f[5]) +
          f[3] * (3443.0 * f[3] - 5966.0 * f[4] + 1602.0 * f[5]) +
          f[4] * (2843.0 * f[4] - 1642.0 * f[5]) + 267.0 * f[5] * f[5];
  is[3] = f[3] * (2107.0 * f[3] - 9402.0 * f[4] + 7042.0 * f[5] - 1854.0 * f[6]) +
          f[4] * (11003.0 * f[4] - 17246.0 * f[5] + 4642.0 * f[6]) +
          f[5] * (7043.0 * f[5] - 3882.0 * f[6]) + 547.0 * f[6] * f[6];
  double q[4], a[4];
  double tau7 = fabs(is[0] - is[3]);
  for (int k = 0; k < 4; ++k) {
    q[k] = A7[k][0] * f[k] + A7[k][1] * f[k + 1] + A7[k][2] * f[k + 2] + A7[k][3] * f[k + 3];
    a[k] = z ? C7[k] * (1.0 + sq(tau7 / (1.0e-40 + is[k]))) : C7[k] / sq(1.0e-40 + is[k]);
  }
  double s = a[0] + a[1] + a[2] + a[3];
  return a[0] / s * q[0] + a[1] / s * q[1] + a[2] / s * q[2] + a[3] / s * q[3];
}

/* Interior tridiagonal row on an oriented stencil f[0..4]: lo multiplies the upwind
   neighbour, up the downwind one.  crweno5: src/crweno5.cpp:130-161 (JS weights
   0.2/0.5/0.3, eps 1e-6); hccs: src/hccs.cpp:145-188 (Z weights eps 1e-40, blended with
   the compact central row 2/7 4/7 1/7 | q7 by theta). */
static const double CR5[3] = {0.2, 0.5, 0.3};
static void compact_row(int hccs, const double *f, double *lo, double *di, double *up, double *rhs) {
  double is0 = G0 * sq(f[0] - 2.0 * f[1] + f[2]) + G1 * sq(f[0] - 4.0 * f[1] + 3.0 * f[2]);
  double is1 = G0 * sq(f[1] - 2.0 * f[2] + f[3]) + G1 * sq(f[1] - f[3]);
  double is2 = G0 * sq(f[2] - 2.0 * f[3] + f[4]) + G1 * sq(3.0 * f[2] - 4.0 * f[3] + f[4]);
  double a0, a1, a2;
  if (hccs) {
    double tau = fabs(is2 - is0);
    a0 = CR5[0] * (1.0 + sq(tau / (is0 + 1.0e-40)));
    a1 = CR5[1] * (1.0 + sq(tau / (is1 + 1.0e-40)));
    a2 = CR5[2] * (1.0 + sq(tau / (is2 + 1.0e-40)));
  } else {
    a0 = CR5[0] / sq(1.0e-6 + is0);
    a1 = CR5[1] / sq(1.0e-6 + is1);
    a2 = CR5[2] / sq(1.0e-6 + is2);
  }
  double sum = a0 + a1 + a2;
  double w0 = a0 / sum, w1 = a1 / sum, w2 = a2 / sum;
  double l = 2.0 / 3.0 * w0 + 1.0 / 3.0 * w1;
  double dd = 1.0 / 3.0 * w0 + 2.0 / 3.0 * (w1 + w2);
  double u = 1.0 / 3.0 * w2;
  double r = 1.0 / 6.0 * w0 * f[1] + (5.0 * (w0 + w1) + w2) * f[2] / 6.0 + (w1 + 5.0 * w2) * f[3] / 6.0;
  if (hccs) {
    double q7 = (-f[0] + 19.0 * f[1] + 239.0 * f[2] + 159.0 * f[3] + 4.0 * f[4]) / 420.0;
    double th = 1.0 / (1.0 + sq(sum - 1.0));
    l = (2.0 / 3.0 * w0 + 1.0 / 3.0 * w1) * (1.0 - th) + 2.0 / 7.0 * th;
    dd = (1.0 / 3.0 * w0 + 2.0 / 3.0 * (w1 + w2)) * (1.0 - th) + 4.0 / 7.0 * th;
    u = (1.0 / 3.0 * w2) * (1.0 - th) + 1.0 / 7.0 * th;
    r = (1.0 / 6.0 * w0 * f[1] + (5.0 * (w0 + w1) + w2) * f[2] / 6.0 + (w1 + 5.0 * w2) * f[3] / 6.0) *
            (1.0 - th) + q7 * th;
  }
  *lo = l; *di = dd; *up = u; *rhs = r;
}

/* ReconstructionboundaryScheme point schemes, src/reconstructionBoundaryScheme.cpp:315-463 */
static double rb2(double f0, double f1) { return 0.5 * (f0 + f1); }
static double rb3(double f0, double f1, double f2) {
  double is0 = sq(f0 - f1), is1 = sq(f1 - f2);
  double q20 = -0.5 * f0 + 1.5 * f1, q21 = 0.5 * f1 + 0.5 * f2;
  double aa0 = 1.0 / 3.0 / sq(1.0e-6 + is0), aa1 = 2.0 / 3.0 / sq(1.0e-6 + is1);
  double w0 = aa0 / (aa0 + aa1), w1 = aa1 / (aa0 + aa1);
  return w0 * q20 + w1 * q21;
}

/* ------------------------------------------------------------------ physics */
typedef struct {
  double rho, u, v, w, p, T, alpha;
} prim_t;

/* physicsModel::con2prim for one cell; may rewrite q[4] (the reset of :324-332) */
static void con2prim(const oc_config *c, double *q4, double q0, double q1, double q2, double q3,
                     double jac, prim_t *s) {
  double g = c->gamma, m = c->mach;
  double rho = q0 * jac;
  double u = q1 / rho * jac, v = q2 / rho * jac, w = q3 / rho * jac;
  double E = *q4 * jac;
  double e0 = E - 0.5 * rho * (u * u + v * v + w * w);
  if (e0 < 0.0) {
    E = (oc_pow(rho, g) / ((g * m * m) * (g - 1.0)) + 0.5 * rho * (u * u + v * v + w * w));
    *q4 = E / jac;
  }
  double p = (E - 0.5 * rho * (u * u + v * v + w * w)) * (g - 1.0);
  s->rho = rho;
  s->u = u;
  s->v = v;
  s->w = w;
  s->p = p;
  s->T = g * m * m * p / rho;
  s->alpha = sqrt(fabs(g * p / rho));
}

static double machL(double m) { return fabs(m) < 1.0 ? 0.25 * sq(m + 1.0) + 0.125 * sq(m * m - 1) : 0.50 * (m + fabs(m)); }
static double machR(double m) { return fabs(m) < 1.0 ? -0.25 * sq(m - 1.0) - 0.125 * sq(m * m - 1) : 0.50 * (m - fabs(m)); }
static double presL(int r, double m, double p) {
  if (fabs(m) >= 1.0) return 0.50 * p * (m + fabs(m)) / m;
  return r == R_AUSM ? p * (m + 1.0) / 2.0 : p * (0.25 * sq(m + 1.0) * (2.0 - m) + 0.1875 * m * sq(m * m - 1.0));
}
static double presR(int r, double m, double p) {
  if (fabs(m) >= 1.0) return 0.5 * p * (m - fabs(m)) / m;
  return r == R_AUSM ? -p * (m - 1.0) / 2.0 : p * (0.25 * sq(m - 1.0) * (2.0 + m) - 0.1875 * m * sq(m * m - 1.0));
}

/* cell splitting along a metric (xx,xy,xz): RiemannSolver body + LF/AUSM/AUSMp */
static void split_cell(int r, const double Q[5], const prim_t *s, double xx, double xy, double xz,
                       double jac, double fp[5], double fn[5], double *eig) {
  double theta = sqrt(xx * xx + xy * xy + xz * xz);
  double U0 = (xx * s->u + xy * s->v + xz * s->w);
  double a0 = s->alpha * theta, p = s->p;
  *eig = fabs(U0) + a0;
  if (r == R_LF) {
    double M = fabs(U0) + a0;
    double f[5] = {U0 * Q[0], U0 * Q[1] + xx * p / jac, U0 * Q[2] + xy * p / jac,
                   U0 * Q[3] + xz * p / jac, U0 * (Q[4] + p / jac)};
    for (int k = 0; k < 5; ++k) {
      fp[k] = 0.5 * (f[k] + M * Q[k]);
      fn[k] = 0.5 * (f[k] - M * Q[k]);
    }
    return;
  }
  double m = U0 / a0, mp = machL(m), mn = machR(m), pp = presL(r, m, p), pn = presR(r, m, p);
  double xs[3] = {xx, xy, xz};
  fp[0] = mp * a0 * Q[0];
  fn[0] = mn * a0 * Q[0];
  for (int k = 1; k < 4; ++k) {
    fp[k] = mp * a0 * Q[k] + xs[k - 1] * pp / jac;
    fn[k] = mn * a0 * Q[k] + xs[k - 1] * pn / jac;
  }
  fp[4] = mp * a0 * Q[4] + mp * a0 * p / jac;
  fn[4] = mn * a0 * Q[4] + mn * a0 * p / jac;
}

/* solveRiemannPoint{LF,AUSM,AUSMp}: split flux of primitive state q at a metric */
static void split_point(const oc_config *c, const double q[5], double jac, double xx, double xy,
                        double xz, double fl[5], double fr[5]) {
  double g = c->gamma, rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  double c5[5] = {rho, rho * u, rho * v, rho * w, p / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w)};
  double _p = (c5[4] - 0.5 * rho * (u * u + v * v + w * w)) * (g - 1.0);
  double _alpha = sqrt(fabs(g * _p / rho));
  double theta = sqrt(xx * xx + xy * xy + xz * xz);
  double alpha = _alpha * theta;
  double U0 = (xx * u + xy * v + xz * w);
  double mach = U0 / alpha;
  double xs[3] = {xx, xy, xz};
  if (c->riemann == R_LF) {
    double M = fabs(U0) + alpha;
    double f[5];
    f[0] = U0 * c5[0] / jac;
    for (int k = 1; k < 4; ++k) f[k] = U0 * c5[k] / jac + xs[k - 1] * p / jac;
    f[4] = U0 * (c5[4] / jac + p / jac);
    for (int k = 0; k < 5; ++k) {
      fl[k] = 0.5 * (f[k] + M * c5[k] / jac);
      fr[k] = 0.5 * (f[k] - M * c5[k] / jac);
    }
    return;
  }
  double mp = machL(mach), mn = machR(mach);
  double pp = presL(c->riemann, mach, p), pn = presR(c->riemann, mach, p);
  fl[0] = mp * alpha * c5[0] / jac;
  fr[0] = mn * alpha * c5[0] / jac;
  for (int k = 1; k < 4; ++k) {
    fl[k] = mp * alpha * c5[k] / jac + xs[k - 1] * pp / jac;
    fr[k] = mn * alpha * c5[k] / jac + xs[k - 1] * pn / jac;
  }
  fl[4] = mp * alpha * c5[4] / jac + mp * alpha * p / jac;
  fr[4] = mn * alpha * c5[4] / jac + mn * alpha * p / jac;
}

/* ------------------------------------------------------------------ block geometry */
typedef struct {
  oc_block *b;
  long N;
  prim_t *w;        /* per cell primitives */
  double *flux[3];  /* per direction: 10N (F+ vars 0..4, F- vars 5..9), k-j-i layout */
  double eig[3];
  double *grad;     /* NS: [var u,v,w,T][dir] 12N */
  double *vis;      /* NS: [dir][var 1..4] 12N */
  double *dinv;     /* 5N inviscid: the running sum df+dg+dh */
  double *dvis[3];  /* NS: 5N per direction (vars 1..4 used) */
} work_t;

static long cell(const oc_block *b, int i, int j, int k) { return ((long)k * b->n[1] + j) * b->n[0] + i; }

/* position pos along d, transverse slab coordinates (a, bb): to (i, j, k) */
static void unslab(int d, int pos, int a, int bb, int *i, int *j, int *k) {
  if (d == 0) { *i = pos; *j = a; *k = bb; }
  else if (d == 1) { *i = bb; *j = pos; *k = a; }
  else { *i = a; *j = bb; *k = pos; }
}
static int slabA(const oc_block *b, int d) { return d == 0 ? b->n[1] : (d == 1 ? b->n[2] : b->n[0]); }
static int slabB(const oc_block *b, int d) { return d == 0 ? b->n[2] : (d == 1 ? b->n[0] : b->n[1]); }

/* The neighbour cell that fills ghost slot `slot` (0..bfs-1) of face f of block b at
   slab coordinates (a, bb): the raw slab copy of the reference (send slab of the
   neighbour's face, received into BufferRecv with the receiver's layout). */
static long ghost_neighbour(work_t *W, int bfs, int bi, int f, int slot, int a, int bb, int *nb) {
  oc_block *b = W[bi].b;
  int d = f >> 1, nf = b->bc_id[f], d2 = nf >> 1, s2 = nf & 1;
  *nb = b->bc_type[f];
  oc_block *o = W[*nb].b;
  long rem = a + (long)slabA(b, d) * bb;
  int A2 = slabA(o, d2);
  int a2 = (int)(rem % A2), b2 = (int)(rem / A2);
  int pos2 = s2 == 0 ? slot : o->n[d2] - bfs + slot;
  int i, j, k;
  unslab(d2, pos2, a2, b2, &i, &j, &k);
  return cell(o, i, j, k);
}

/* ------------------------------------------------------------------ passes */
static void pass_con2prim(const oc_config *c, work_t *w) {
  oc_block *b = w->b;
  long N = w->N;
  for (long x = 0; x < N; ++x)
    con2prim(c, &b->q[4 * N + x], b->q[x], b->q[N + x], b->q[2 * N + x], b->q[3 * N + x], b->jac[x],
             &w->w[x]);
}

static const double *metric(const oc_block *b, int d) { return d == 0 ? b->xi : (d == 1 ? b->eta : b->zeta); }

static void pass_split(const oc_config *c, work_t *w) {
  oc_block *b = w->b;
  long N = w->N;
  for (int d = 0; d < 3; ++d) {
    const double *m = metric(b, d);
    double emax = 0.0;
    for (long x = 0; x < N; ++x) {
      double Q[5] = {b->q[x], b->q[N + x], b->q[2 * N + x], b->q[3 * N + x], b->q[4 * N + x]};
      double fp[5], fn[5], e;
      split_cell(c->riemann, Q, &w->w[x], m[x], m[N + x], m[2 * N + x], b->jac[x], fp, fn, &e);
      for (int v = 0; v < 5; ++v) {
        w->flux[d][v * N + x] = fp[v];
        w->flux[d][(5 + v) * N + x] = fn[v];
      }
      emax = e < emax ? emax : e; /* std::max(e, emax) */
    }
    w->eig[d] = emax;
  }
}

/* point-split ghost flux of a physical face at mirror cell index mc of block b */
static void bc_point(const oc_config *c, const oc_block *b, const prim_t *wc, int f, long mc,
                     double fl[5], double fr[5]) {
  int d = f >> 1, id = b->bc_id[f];
  long N = (long)b->n[0] * b->n[1] * b->n[2];
  const double *m = metric(b, d);
  double q[5];
  if (id == 0) {
    for (int v = 0; v < 5; ++v) q[v] = b->bcv[f][v];
  } else {
    const prim_t *s = &wc[mc];
    q[0] = s->rho; q[1] = s->u; q[2] = s->v; q[3] = s->w; q[4] = s->p;
    if (id == 2) {
      q[0] = q[4] * c->gamma * c->mach * c->mach / c->t_wall;
      q[1] = 0.0; q[2] = 0.0; q[3] = 0.0;
    } else if (id == 3) {
      double U = b->xi[mc] * q[1] + b->xi[N + mc] * q[2] + b->xi[2 * N + mc] * q[3];
      double V = b->eta[mc] * q[1] + b->eta[N + mc] * q[2] + b->eta[2 * N + mc] * q[3];
      double Wc = b->zeta[mc] * q[1] + b->zeta[N + mc] * q[2] + b->zeta[2 * N + mc] * q[3];
      const double *X = b->dxyz;
      double t[9];
      for (int k = 0; k < 9; ++k) t[k] = X[k * N + mc];
      double sg[3] = {d == 0 ? -1.0 : 1.0, d == 1 ? -1.0 : 1.0, d == 2 ? -1.0 : 1.0};
      for (int r = 0; r < 3; ++r) {
        /* e.g. xi face: -x_xi*U + x_eta*V + x_zeta*W (src/boundaryConditions.cpp:886-888) */
        double tU = t[3 * r] * U, tV = t[3 * r + 1] * V, tW = t[3 * r + 2] * Wc;
        double acc = (sg[0] < 0 ? -t[3 * r] * U : tU);
        acc = sg[1] < 0 ? acc - tV : acc + tV;
        acc = sg[2] < 0 ? acc - tW : acc + tW;
        q[1 + r] = acc;
      }
    }
  }
  split_point(c, q, b->jac[mc], m[mc], m[N + mc], m[2 * N + mc], fl, fr);
}

/* Extended line of F+ (side 0) and F- (side 1) values of variable v along direction d:
   ext[g + bfs] for g in [-bfs, L+bfs).  Physical faces fill every ghost slot like the
   BC setters do (mirror cells for wall/symmetry, the edge cell otherwise). */
static void line_ext(const oc_config *c, work_t *W, int bfs, int bi, int d, int a, int bb, int v,
                     double *extP, double *extN) {
  oc_block *b = W[bi].b;
  int L = b->n[d];
  for (int pos = 0; pos < L; ++pos) {
    int i, j, k;
    unslab(d, pos, a, bb, &i, &j, &k);
    long x = cell(b, i, j, k);
    extP[pos + bfs] = W[bi].flux[d][v * W[bi].N + x];
    extN[pos + bfs] = W[bi].flux[d][(5 + v) * W[bi].N + x];
  }
  for (int side = 0; side < 2; ++side) {
    int f = 2 * d + side;
    for (int slot = 0; slot < bfs; ++slot) {
      int g = side == 0 ? slot - bfs : L + slot;
      double P, Nv;
      if (b->bc_type[f] >= 0) {
        int nb;
        long x = ghost_neighbour(W, bfs, bi, f, slot, a, bb, &nb);
        P = W[nb].flux[d][v * W[nb].N + x];
        Nv = W[nb].flux[d][(5 + v) * W[nb].N + x];
      } else {
        /* mirror cell of this slot (src/boundaryConditions.cpp:525-526); inlet/outlet
           use the edge cell for every slot */
        int dist = side == 0 ? bfs - 1 - slot : slot;
        int id = b->bc_id[f];
        int mpos = (id == 2 || id == 3) ? (side == 0 ? dist : L - 1 - dist) : (side == 0 ? 0 : L - 1);
        int i, j, k;
        unslab(d, mpos, a, bb, &i, &j, &k);
        double fl[5], fr[5];
        bc_point(c, b, W[bi].w, f, cell(b, i, j, k), fl, fr);
        P = fl[v];  /* BufferSend */
        Nv = fr[v]; /* BufferRecv */
      }
      extP[g + bfs] = P;
      extN[g + bfs] = Nv;
    }
  }
}

/* explicit face value of one split at face f: BL/BR or inner stencil of the scheme
   (compact schemes use WENO5-JS / WENO7-Z there), or the exterior point schemes */
static double face_explicit(const oc_config *c, int d, int side, int f, int L, int ts, int physL,
                            int physR, int bfs, const double *e) {
#define P(cc) e[(cc) + bfs]
  int sch = c->scheme[d] == S_HCCS77 ? S_HCCS : c->scheme[d]; /* end rows: WENO7-Z */
  int exL = physL && f < ts, exR = physR && f > L - ts;
  if (side == 0) {
    if (exR) {
      int m = L - f;
      if (m == 0) return P(L - 1);
      if (m == 1) return rb2(P(L - 2), P(L - 1));
      if (m == 2) return rb3(P(L - 4), P(L - 3), P(L - 2));
      double s[5] = {P(L - 6), P(L - 5), P(L - 4), P(L - 3), P(L - 2)};
      return weno5(s, 0, 0);
    }
    if (exL) {
      if (f == 0) return e[bfs - 1];
      if (f == 1) return rb2(P(0), P(1));
      if (f == 2) return rb3(P(0), P(1), P(2));
      double s[5] = {P(0), P(1), P(2), P(3), P(4)};
      return weno5(s, 0, 0);
    }
    if (sch == S_WENO3JS) return rb3(P(f - 2), P(f - 1), P(f)); /* src/weno3js.cpp:59-86 */
    if (sch == S_UPWIND1) return P(f - 1);                     /* src/upwind1st.cpp:57-75 */
    if (sch == S_WENO7JS || sch == S_HCCS) {
      double s[7];
      for (int k = 0; k < 7; ++k) s[k] = P(f - 4 + k);
      return weno7zs(s, sch == S_HCCS);
    }
    double s[5];
    for (int k = 0; k < 5; ++k) s[k] = P(f - 3 + k);
    int z = sch == S_WENO5Z;
    return weno5(s, z, z && c->compat && f >= ts && f <= L - ts);
  }
  if (exR) {
    int m = L - f;
    if (m == 0) return e[L + bfs];
    if (m == 1) return rb2(P(L - 1), P(L - 2));
    if (m == 2) return rb3(P(L - 1), P(L - 2), P(L - 3));
    double s[5] = {P(L - 1), P(L - 2), P(L - 3), P(L - 4), P(L - 5)};
    return weno5(s, 0, 0);
  }
  if (exL) {
    if (f == 0) return P(0);
    if (f == 1) return rb2(P(1), P(0));
    if (f == 2) return rb3(P(3), P(2), P(1));
    double s[5] = {P(5), P(4), P(3), P(2), P(1)};
    return weno5(s, 0, 0);
  }
  if (sch == S_WENO3JS) return rb3(P(f + 1), P(f), P(f - 1)); /* src/weno3js.cpp:88-115 */
  if (sch == S_UPWIND1) return P(f);                         /* src/upwind1st.cpp:96-114 */
  if (sch == S_WENO7JS || sch == S_HCCS) {
    double s[7];
    for (int k = 0; k < 7; ++k) s[k] = P(f + 3 - k);
    return weno7zs(s, sch == S_HCCS);
  }
  double s[5];
  for (int k = 0; k < 5; ++k) s[k] = P(f + 2 - k);
  return weno5(s, sch == S_WENO5Z, 0);
#undef P
}

/* face values of one line: positive and negative reconstruction (upwind +1 / -1) */
static void line_faces(const oc_config *c, const oc_block *b, int d, int bfs, const double *eP,
                       const double *eN, double *face) {
  int L = b->n[d], sch = c->scheme[d];
  int ts = tilesize(sch);
  int physL = b->bc_type[2 * d] < 0, physR = b->bc_type[2 * d + 1] < 0;
  int compact = sch == S_CRWENO5 || sch == S_HCCS || sch == S_HCCS77;
  /* hccs77: one system over faces 0 .. L, WENO7-Z rows at 0 and L from the ghost cells,
     hccs rows elsewhere (src/hccs77.cpp:45-195, :218-568, :592-943, solve :945-978);
     defined for neighbour faces only */
  int f0 = sch == S_HCCS77 ? 0 : ts;
  static double hs[2][4096], ra[4096], rb[4096], rc[4096], rd[4096];
  for (int side = 0; side < 2; ++side) {
    const double *e = side ? eN : eP;
    for (int f = 0; f <= L; ++f)
      if (!compact || f < f0 || f > L - f0) hs[side][f] = face_explicit(c, d, side, f, L, ts, physL, physR, bfs, e);
    if (!compact) continue;
    /* tridiagonal system over faces f0 .. L-f0 (src/crweno5.cpp:82-218) */
    int m = L - 2 * f0 + 1;
    for (int r = 0; r < m; ++r) {
      int f = f0 + r;
      if (r == 0 || r == m - 1) {
        ra[r] = 0.0; rb[r] = 1.0; rc[r] = 0.0;
        rd[r] = face_explicit(c, d, side, f, L, ts, 0, 0, bfs, e);
      } else {
        double s5[5], lo, di, up;
        for (int k = 0; k < 5; ++k) s5[k] = side ? e[f + 2 - k + bfs] : e[f - 3 + k + bfs];
        compact_row(sch != S_CRWENO5, s5, &lo, &di, &up, &rd[r]);
        rb[r] = di;
        if (side) { ra[r] = up; rc[r] = lo; } else { ra[r] = lo; rc[r] = up; }
      }
    }
    for (int i = 1; i < m; ++i) {
      rc[i] = rc[i] / (rb[i] - rc[i - 1] * ra[i]);
      rd[i] = (rd[i] - rd[i - 1] * ra[i]) / (rb[i] - rc[i - 1] * ra[i]);
    }
    hs[side][f0 + m - 1] = rd[m - 1];
    for (int i = m - 2; i >= 0; --i) hs[side][f0 + i] = rd[i] - rc[i] * hs[side][f0 + i + 1];
  }
  for (int f = 0; f <= L; ++f) face[f] = hs[0][f] + hs[1][f];
}

/* derivative of an extended line (ghosts at [-bfs, 0) and [L, L+bfs)) at position pos */
static const double CD8[4] = {4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0};
static double line_diff(const double *e, int bfs, int pos, int L, int ts, int physL, int physR,
                        int vis) {
#define V(cc) e[(cc) + bfs]
  if (physR && pos >= L - ts) {
    int m = L - 1 - pos;
    if (m == 0) return V(pos) - V(pos - 1);
    if (m == 1) return 0.5 * (V(pos + 1) - V(pos - 1));
    if (m == 2) return CD4[1] * (V(pos + 2) - V(pos - 2)) + CD4[0] * (V(pos + 1) - V(pos - 1));
    return CD6[2] * (V(pos + 3) - V(pos - 3)) + CD6[1] * (V(pos + 2) - V(pos - 2)) + CD4[0] * (V(pos + 1) - V(pos - 1));
  }
  if (physL && pos < ts) {
    if (pos == 0) return V(pos + 1) - V(pos);
    if (pos == 1) return 0.5 * (V(pos + 1) - V(pos - 1));
    if (pos == 2) return CD4[1] * (V(pos + 2) - V(pos - 2)) + CD4[0] * (V(pos + 1) - V(pos - 1));
    return CD6[2] * (V(pos + 3) - V(pos - 3)) + CD6[1] * (V(pos + 2) - V(pos - 2)) + CD4[0] * (V(pos + 1) - V(pos - 1));
  }
  /* inside the block and at block edges with neighbour ghosts: the scheme_vis operator
     (src/centraldifference2nd.cpp:16-37, 6th :16-183, 8th :16-52) */
  if (vis == V_CD2) return 0.5 * (V(pos + 1) - V(pos - 1));
  if (vis == V_CD8)
    return CD8[3] * (V(pos + 4) - V(pos - 4)) + CD8[2] * (V(pos + 3) - V(pos - 3)) +
           CD8[1] * (V(pos + 2) - V(pos - 2)) + CD8[0] * (V(pos + 1) - V(pos - 1));
  return CD6[2] * (V(pos + 3) - V(pos - 3)) + CD6[1] * (V(pos + 2) - V(pos - 2)) + CD6[0] * (V(pos + 1) - V(pos - 1));
#undef V
}

/* extended line of a cell field F (N values per block, component comp) along d */

static void field_line(work_t *W, int bfs, int bi, int d, int a, int bb, int which, int comp,
                       double *ext) {
  /* which 0: primitive u,v,w,T (comp 0..3); which 1: viscous flux vis[d][comp] */
  oc_block *b = W[bi].b;
  int L = b->n[d];
  for (int g = -bfs; g < L + bfs; ++g) {
    int bk = bi;
    long x = -1;
    if (g >= 0 && g < L) {
      int i, j, k;
      unslab(d, g, a, bb, &i, &j, &k);
      x = cell(b, i, j, k);
    } else {
      int f = 2 * d + (g < 0 ? 0 : 1);
      if (b->bc_type[f] >= 0) x = ghost_neighbour(W, bfs, bi, f, g < 0 ? g + bfs : g - L, a, bb, &bk);
    }
    double val = 0.0;
    if (x >= 0) {
      if (which == 0) {
        const prim_t *s = &W[bk].w[x];
        val = comp == 0 ? s->u : comp == 1 ? s->v : comp == 2 ? s->w : s->T;
      } else {
        val = W[bk].vis[(d * 4 + comp) * W[bk].N + x];
      }
    }
    ext[g + bfs] = val;
  }
}

static void pass_inviscid(const oc_config *c, work_t *W, int nb, int bfs, double *ext1, double *ext2,
                          double *face) {
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    for (int d = 0; d < 3; ++d) {
      int L = b->n[d], A = slabA(b, d), B = slabB(b, d);
      for (int bb = 0; bb < B; ++bb)
        for (int a = 0; a < A; ++a)
          for (int v = 0; v < 5; ++v) {
            line_ext(c, W, bfs, bi, d, a, bb, v, ext1, ext2);
            line_faces(c, b, d, bfs, ext1, ext2, face);
            for (int pos = 0; pos < L; ++pos) {
              int i, j, k;
              unslab(d, pos, a, bb, &i, &j, &k);
              long x = cell(b, i, j, k);
              double df = face[pos + 1] - face[pos];
              /* rhs = df; rhs += dg; rhs += dh (src/euler3d.cpp:383-422) */
              W[bi].dinv[v * N + x] = d == 0 ? df : W[bi].dinv[v * N + x] + df;
            }
          }
    }
  }
}

static void pass_viscous(const oc_config *c, work_t *W, int nb, int bfs, double *ext) {
  int ts[3];
  for (int d = 0; d < 3; ++d) ts[d] = tilesize(c->scheme[d]);
  /* gradients of u, v, w, T along xi, eta, zeta (src/NaiverStokes3d.cpp:63-168) */
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    for (int d = 0; d < 3; ++d) {
      int L = b->n[d], A = slabA(b, d), B = slabB(b, d);
      int pl = b->bc_type[2 * d] < 0, pr = b->bc_type[2 * d + 1] < 0;
      for (int bb = 0; bb < B; ++bb)
        for (int a = 0; a < A; ++a)
          for (int comp = 0; comp < 4; ++comp) {
            field_line(W, bfs, bi, d, a, bb, 0, comp, ext);
            for (int pos = 0; pos < L; ++pos) {
              int i, j, k;
              unslab(d, pos, a, bb, &i, &j, &k);
              W[bi].grad[(comp * 3 + d) * N + cell(b, i, j, k)] = line_diff(ext, bfs, pos, L, ts[d], pl, pr, c->vis[d]);
            }
          }
    }
  }
  /* viscous fluxes (src/NaiverStokes3d.cpp:170-326, sutherland src/physicsModel.cpp:199-234) */
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    for (long x = 0; x < N; ++x) {
      const double *g = W[bi].grad;
      double xi_x = b->xi[x], xi_y = b->xi[N + x], xi_z = b->xi[2 * N + x];
      double eta_x = b->eta[x], eta_y = b->eta[N + x], eta_z = b->eta[2 * N + x];
      double zeta_x = b->zeta[x], zeta_y = b->zeta[N + x], zeta_z = b->zeta[2 * N + x];
#define GR(cmp, dd) g[((cmp) * 3 + (dd)) * N + x]
      double ux = GR(0, 0) * xi_x + GR(0, 1) * eta_x + GR(0, 2) * zeta_x;
      double uy = GR(0, 0) * xi_y + GR(0, 1) * eta_y + GR(0, 2) * zeta_y;
      double uz = GR(0, 0) * xi_z + GR(0, 1) * eta_z + GR(0, 2) * zeta_z;
      double vx = GR(1, 0) * xi_x + GR(1, 1) * eta_x + GR(1, 2) * zeta_x;
      double vy = GR(1, 0) * xi_y + GR(1, 1) * eta_y + GR(1, 2) * zeta_y;
      double vz = GR(1, 0) * xi_z + GR(1, 1) * eta_z + GR(1, 2) * zeta_z;
      double wx = GR(2, 0) * xi_x + GR(2, 1) * eta_x + GR(2, 2) * zeta_x;
      double wy = GR(2, 0) * xi_y + GR(2, 1) * eta_y + GR(2, 2) * zeta_y;
      double wz = GR(2, 0) * xi_z + GR(2, 1) * eta_z + GR(2, 2) * zeta_z;
      double tx = GR(3, 0) * xi_x + GR(3, 1) * eta_x + GR(3, 2) * zeta_x;
      double ty = GR(3, 0) * xi_y + GR(3, 1) * eta_y + GR(3, 2) * zeta_y;
      double tz = GR(3, 0) * xi_z + GR(3, 1) * eta_z + GR(3, 2) * zeta_z;
#undef GR
      const prim_t *s = &W[bi].w[x];
      double T = s->T, nd = c->t_ref / c->t_inf;
      double miu0 = (1.0 + nd) / (T + nd) * cr_pow15(T) / c->reynolds;
      double coeff0 = miu0 / ((c->gamma - 1.0) * c->mach * c->mach * c->prandtl);
      double grad = ux + vy + wz;
      double txx = miu0 * (2.0 * ux - 2.0 / 3.0 * grad), txy = miu0 * (uy + vx - 2.0 / 3.0 * grad);
      double txz = miu0 * (uz + wx - 2.0 / 3.0 * grad), tyy = miu0 * (2.0 * vy - 2.0 / 3.0 * grad);
      double tyz = miu0 * (vz + wy - 2.0 / 3.0 * grad), tzz = miu0 * (2.0 * wz - 2.0 / 3.0 * grad);
      double u = s->u, v = s->v, w = s->w;
      double fv[4] = {txx, txy, txz, u * txx + v * txy + w * txz + coeff0 * tx};
      double gv[4] = {txy, tyy, tyz, u * txy + v * tyy + w * tyz + coeff0 * ty};
      double hv[4] = {txz, tyz, tzz, u * txz + v * tyz + w * tzz + coeff0 * tz};
      double jac = b->jac[x];
      for (int k = 0; k < 4; ++k) {
        W[bi].vis[(0 * 4 + k) * N + x] = (xi_x * fv[k] + xi_y * gv[k] + xi_z * hv[k]) / jac;
        W[bi].vis[(1 * 4 + k) * N + x] = (eta_x * fv[k] + eta_y * gv[k] + eta_z * hv[k]) / jac;
        W[bi].vis[(2 * 4 + k) * N + x] = (zeta_x * fv[k] + zeta_y * gv[k] + zeta_z * hv[k]) / jac;
      }
    }
  }
  /* derivatives of the viscous fluxes (src/NaiverStokes3d.cpp:328-398) */
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    for (int d = 0; d < 3; ++d) {
      int L = b->n[d], A = slabA(b, d), B = slabB(b, d);
      int pl = b->bc_type[2 * d] < 0, pr = b->bc_type[2 * d + 1] < 0;
      for (int bb = 0; bb < B; ++bb)
        for (int a = 0; a < A; ++a)
          for (int comp = 0; comp < 4; ++comp) {
            field_line(W, bfs, bi, d, a, bb, 1, comp, ext);
            for (int pos = 0; pos < L; ++pos) {
              int i, j, k;
              unslab(d, pos, a, bb, &i, &j, &k);
              W[bi].dvis[d][(comp + 1) * N + cell(b, i, j, k)] = line_diff(ext, bfs, pos, L, ts[d], pl, pr, c->vis[d]);
            }
          }
    }
  }
}

/* One right-hand side of every block at its current q.  Returns dt_local
   (min over blocks and directions of 1/maxEigen). */
static int eval_rhs(const oc_config *c, int nb, oc_block *blocks, work_t *W, double *dt_local) {
  int bfs = ghost_width(c);
  int maxL = 0;
  for (int bi = 0; bi < nb; ++bi)
    for (int d = 0; d < 3; ++d)
      if (blocks[bi].n[d] > maxL) maxL = blocks[bi].n[d];
  double *ext1 = malloc(sizeof(double) * (maxL + 2 * bfs + 2));
  double *ext2 = malloc(sizeof(double) * (maxL + 2 * bfs + 2));
  double *face = malloc(sizeof(double) * (maxL + 2));
  for (int bi = 0; bi < nb; ++bi) pass_con2prim(c, &W[bi]);
  for (int bi = 0; bi < nb; ++bi) pass_split(c, &W[bi]);
  pass_inviscid(c, W, nb, bfs, ext1, ext2, face);
  if (c->model == 1) pass_viscous(c, W, nb, bfs, ext1);
  double dtl = 1e300;
  for (int bi = 0; bi < nb; ++bi) {
    long N = W[bi].N;
    oc_block *b = &blocks[bi];
    for (int v = 0; v < 5; ++v)
      for (long x = 0; x < N; ++x) {
        double r = W[bi].dinv[v * N + x];
        if (c->model == 1 && v > 0) {
          r -= W[bi].dvis[0][v * N + x];
          r -= W[bi].dvis[1][v * N + x];
          r -= W[bi].dvis[2][v * N + x];
        }
        if (b->rhs) b->rhs[v * N + x] = r;
        W[bi].dinv[v * N + x] = r;
      }
    /* EulerData3D::getDt (src/euler3d.cpp:429-435) */
    double a = 1.0 / W[bi].eig[0], bb = 1.0 / W[bi].eig[1], cc = 1.0 / W[bi].eig[2];
    double m = a < bb ? a : bb;
    m = m < cc ? m : cc;
    dtl = m < dtl ? m : dtl;
  }
  free(ext1);
  free(ext2);
  free(face);
  *dt_local = dtl;
  return 0;
}

static work_t *alloc_work(const oc_config *c, int nb, oc_block *blocks) {
  work_t *W = calloc(nb, sizeof(work_t));
  for (int bi = 0; bi < nb; ++bi) {
    long N = (long)blocks[bi].n[0] * blocks[bi].n[1] * blocks[bi].n[2];
    W[bi].b = &blocks[bi];
    W[bi].N = N;
    W[bi].w = malloc(sizeof(prim_t) * N);
    for (int d = 0; d < 3; ++d) W[bi].flux[d] = malloc(sizeof(double) * 10 * N);
    W[bi].dinv = malloc(sizeof(double) * 5 * N);
    if (c->model == 1) {
      W[bi].grad = malloc(sizeof(double) * 12 * N);
      W[bi].vis = malloc(sizeof(double) * 12 * N);
      for (int d = 0; d < 3; ++d) W[bi].dvis[d] = calloc(5 * N, sizeof(double));
    }
  }
  return W;
}

static void free_work(int nb, work_t *W) {
  for (int bi = 0; bi < nb; ++bi) {
    free(W[bi].w);
    for (int d = 0; d < 3; ++d) free(W[bi].flux[d]);
    free(W[bi].dinv);
    free(W[bi].grad);
    free(W[bi].vis);
    for (int d = 0; d < 3; ++d) free(W[bi].dvis[d]);
  }
  free(W);
}

/* ------------------------------------------------------------------ entry points */
int oc_rhs(const oc_config *c, int nb, oc_block *blocks, double *dt_local) {
  work_t *W = alloc_work(c, nb, blocks);
  int r = eval_rhs(c, nb, blocks, W, dt_local);
  free_work(nb, W);
  return r;
}

/* nsteps TVD-RK3 steps (block::solve); dt[s] and the accumulated *time are returned */
/* nsteps TVD-RK3 steps; dt[s], *time, and res[s] (may be NULL): the residual of step s,
   PDEData3d::setRES (src/PDEData3d.cpp:90-122) per block in its loop order, the maximum
   over blocks; res_last is per block (a function-static per rank in the reference), from
   0 at the first step of this call. */
int oc_step(const oc_config *c, int nb, oc_block *blocks, int nsteps, double *dt, double *time,
            double *res) {
  work_t *W = alloc_work(c, nb, blocks);
  double **qn = malloc(sizeof(double *) * nb);
  double *res_last = calloc(nb, sizeof(double));
  for (int bi = 0; bi < nb; ++bi) qn[bi] = malloc(sizeof(double) * 5 * W[bi].N);
  for (int s = 0; s < nsteps; ++s) {
    double dtg = 0.0;
    for (int stage = 0; stage < 3; ++stage) {
      double dtl;
      eval_rhs(c, nb, blocks, W, &dtl);
      if (stage == 0) {
        for (int bi = 0; bi < nb; ++bi) memcpy(qn[bi], blocks[bi].q, sizeof(double) * 5 * W[bi].N);
        dtg = dtl * c->cfl; /* Allreduce MIN then *= cfl (src/PDEData3d.cpp:156-162) */
      }
      for (int bi = 0; bi < nb; ++bi) {
        long n5 = 5 * W[bi].N;
        double *u = blocks[bi].q;
        for (long x = 0; x < n5; ++x) {
          double rhs = -W[bi].dinv[x];
          if (stage == 0) u[x] = 1.0 * u[x] + 1.0 * rhs * dtg;
          else if (stage == 1) u[x] = 3.0 / 4.0 * qn[bi][x] + 1.0 / 4.0 * (rhs * dtg + u[x]);
          else u[x] = 1.0 / 3.0 * qn[bi][x] + 2.0 / 3.0 * (rhs * dtg + u[x]);
        }
      }
    }
    if (dt) dt[s] = dtg;
    if (time) *time = *time + dtg;
    double rmax = 0.0;
    for (int bi = 0; bi < nb; ++bi) {
      long n5 = 5 * W[bi].N;
      double sum = 0.0;
      for (long x = 0; x < n5; ++x) {
        double d = blocks[bi].q[x] - qn[bi][x];
        sum += sq(d);
      }
      double r = sqrt(sum / (double)((unsigned long)n5));
      double rl = fabs(r - res_last[bi]) / (dtg * dtg);
      res_last[bi] = r;
      if (rl > rmax) rmax = rl;
    }
    if (res) res[s] = rmax;
  }
  for (int bi = 0; bi < nb; ++bi) free(qn[bi]);
  free(res_last);
  free(qn);
  free_work(nb, W);
  return 0;
}

/* ------------------------------------------------------------------ diagnostics
 * postproc::solveQ (src/postproc.cpp:743-848) after block::Post's getPrim
 * (src/block.cpp:601-618): velocity gradients by the block's difference operator
 * (solveGrad, :1797-1820: halo exchange, cd6 inside, boundaryScheme at physical faces),
 * the chain rule of solveGrad_x/y/z, vorticity, Q, and the totals
 * enstrophy = sum 0.5|w|^2 and kinetic = sum 0.5 rho |u|^2, summed cell by cell in
 * k-j-i order per block and then over the blocks in order (MPI_Allreduce in rank order).
 * fields: per block NULL or 5N (w_x, w_y, w_z, 0.5|w|^2, Q). */
int oc_diag(const oc_config *c, int nb, oc_block *blocks, double *enstrophy, double *kinetic,
            double **fields) {
  int bfs = ghost_width(c), ts[3];
  for (int d = 0; d < 3; ++d) ts[d] = tilesize(c->scheme[d]);
  int maxL = 0;
  for (int bi = 0; bi < nb; ++bi)
    for (int d = 0; d < 3; ++d)
      if (blocks[bi].n[d] > maxL) maxL = blocks[bi].n[d];
  double *ext = malloc(sizeof(double) * (maxL + 2 * bfs + 2));
  work_t *W = calloc(nb, sizeof(work_t));
  for (int bi = 0; bi < nb; ++bi) {
    long N = (long)blocks[bi].n[0] * blocks[bi].n[1] * blocks[bi].n[2];
    W[bi].b = &blocks[bi];
    W[bi].N = N;
    W[bi].w = malloc(sizeof(prim_t) * N);
    W[bi].grad = malloc(sizeof(double) * 12 * N);
    pass_con2prim(c, &W[bi]);
  }
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    for (int d = 0; d < 3; ++d) {
      int L = b->n[d], A = slabA(b, d), B = slabB(b, d);
      int pl = b->bc_type[2 * d] < 0, pr = b->bc_type[2 * d + 1] < 0;
      for (int bb = 0; bb < B; ++bb)
        for (int a = 0; a < A; ++a)
          for (int comp = 0; comp < 3; ++comp) {
            field_line(W, bfs, bi, d, a, bb, 0, comp, ext);
            for (int pos = 0; pos < L; ++pos) {
              int i, j, k;
              unslab(d, pos, a, bb, &i, &j, &k);
              W[bi].grad[(comp * 3 + d) * N + cell(b, i, j, k)] = line_diff(ext, bfs, pos, L, ts[d], pl, pr, c->vis[d]);
            }
          }
    }
  }
  double ens_glb = 0.0, kin_glb = 0.0;
  for (int bi = 0; bi < nb; ++bi) {
    oc_block *b = W[bi].b;
    long N = W[bi].N;
    const double *g = W[bi].grad;
    double ens = 0.0, kin = 0.0;
    for (long x = 0; x < N; ++x) {
#define GR(cmp, dd) g[((cmp) * 3 + (dd)) * N + x]
      double xi_x = b->xi[x], xi_y = b->xi[N + x], xi_z = b->xi[2 * N + x];
      double eta_x = b->eta[x], eta_y = b->eta[N + x], eta_z = b->eta[2 * N + x];
      double zeta_x = b->zeta[x], zeta_y = b->zeta[N + x], zeta_z = b->zeta[2 * N + x];
      double ux = GR(0, 0) * xi_x + GR(0, 1) * eta_x + GR(0, 2) * zeta_x;
      double uy = GR(0, 0) * xi_y + GR(0, 1) * eta_y + GR(0, 2) * zeta_y;
      double uz = GR(0, 0) * xi_z + GR(0, 1) * eta_z + GR(0, 2) * zeta_z;
      double vx = GR(1, 0) * xi_x + GR(1, 1) * eta_x + GR(1, 2) * zeta_x;
      double vy = GR(1, 0) * xi_y + GR(1, 1) * eta_y + GR(1, 2) * zeta_y;
      double vz = GR(1, 0) * xi_z + GR(1, 1) * eta_z + GR(1, 2) * zeta_z;
      double wx = GR(2, 0) * xi_x + GR(2, 1) * eta_x + GR(2, 2) * zeta_x;
      double wy = GR(2, 0) * xi_y + GR(2, 1) * eta_y + GR(2, 2) * zeta_y;
      double wz = GR(2, 0) * xi_z + GR(2, 1) * eta_z + GR(2, 2) * zeta_z;
#undef GR
      double w0 = wy - vz, w1 = uz - wx, w2 = vx - uy;
      double q0 = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
      if (fields && fields[bi]) {
        fields[bi][x] = w0;
        fields[bi][N + x] = w1;
        fields[bi][2 * N + x] = w2;
        fields[bi][3 * N + x] = (w0 * w0 + w1 * w1 + w2 * w2) * 0.5;
        fields[bi][4 * N + x] = q0;
      }
      const prim_t *s = &W[bi].w[x];
      ens += 0.5 * (w0 * w0 + w1 * w1 + w2 * w2);
      kin += 0.5 * s->rho * (s->u * s->u + s->v * s->v + s->w * s->w);
    }
    ens_glb = bi == 0 ? ens : ens_glb + ens;
    kin_glb = bi == 0 ? kin : kin_glb + kin;
  }
  for (int bi = 0; bi < nb; ++bi) {
    free(W[bi].w);
    free(W[bi].grad);
  }
  free(W);
  free(ext);
  *enstrophy = ens_glb;
  *kinetic = kin_glb;
  return 0;
}

/* ------------------------------------------------------------------ metrics
 * block::getJacobians (src/block.cpp:237-325) with the 4x4x4-cell tile Lagrange
 * reconstruction of src/block.cpp:147-235 (centres) and :327-477 (derivatives),
 * coefficients src/block.h:36-48.  x, y, z: node coordinates (nz+1)(ny+1)(nx+1),
 * i fastest; cells per axis must be multiples of 4.  Outputs: jac N, xi/eta/zeta
 * 3N each, dxyz 9N (x_xi x_eta x_zeta y_xi y_eta y_zeta z_xi z_eta z_zeta). */
static const double LAG[4][5] = {
    {35.0 / 128.0, 35.0 / 32.0, -35.0 / 64.0, 7.0 / 32.0, -5.0 / 128.0},
    {-5.0 / 128.0, 15.0 / 32.0, 45.0 / 64.0, -5.0 / 32.0, 3.0 / 128.0},
    {3.0 / 128.0, -5.0 / 32.0, 45.0 / 64.0, 15.0 / 32.0, -5.0 / 128.0},
    {-5.0 / 128.0, 7.0 / 32.0, -35.0 / 64.0, 35.0 / 32.0, 35.0 / 128.0}};
static const double DLAG[4][5] = {
    {-11.0 / 12.0, 17.0 / 24.0, 3.0 / 8.0, -5.0 / 24.0, 1.0 / 24.0},
    {1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0, 0.0},
    {0.0, 1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0},
    {-1.0 / 24.0, 5.0 / 24.0, -3.0 / 8.0, -17.0 / 24.0, 11.0 / 12.0}};

static double tile_value(const double *f, int nx0, int ny0, int i, int j, int k, int dir) {
  int ib = (i / 4) * 4, jb = (j / 4) * 4, kb = (k / 4) * 4;
  const double(*cx)[5] = dir == 0 ? DLAG : LAG;
  const double(*cy)[5] = dir == 1 ? DLAG : LAG;
  const double(*cz)[5] = dir == 2 ? DLAG : LAG;
  double vz = 0.0;
  for (int kk = 0; kk <= 4; ++kk) {
    double vy = 0.0;
    for (int jj = 0; jj <= 4; ++jj) {
      double vx = 0.0;
      for (int ii = 0; ii <= 4; ++ii)
        vx += cx[i - ib][ii] * f[((long)(kb + kk) * ny0 + (jb + jj)) * nx0 + (ib + ii)];
      vy += cy[j - jb][jj] * vx;
    }
    vz += cz[k - kb][kk] * vy;
  }
  return vz;
}

int oc_metrics(int nx, int ny, int nz, const double *x, const double *y, const double *z,
               double *jac, double *xi, double *eta, double *zeta, double *dxyz) {
  if (nx % 4 || ny % 4 || nz % 4) return 1;
  int nx0 = nx + 1, ny0 = ny + 1;
  long N = (long)nx * ny * nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        long c = ((long)k * ny + j) * nx + i;
        double d[3][3]; /* d[coord x,y,z][dir] */
        const double *xyz[3] = {x, y, z};
        for (int a = 0; a < 3; ++a)
          for (int dir = 0; dir < 3; ++dir) d[a][dir] = tile_value(xyz[a], nx0, ny0, i, j, k, dir);
        double x_xi = d[0][0], x_eta = d[0][1], x_zeta = d[0][2];
        double y_xi = d[1][0], y_eta = d[1][1], y_zeta = d[1][2];
        double z_xi = d[2][0], z_eta = d[2][1], z_zeta = d[2][2];
        double jacob = 1.0 / (x_xi * (y_eta * z_zeta - y_zeta * z_eta) + x_eta * (y_zeta * z_xi - y_xi * z_zeta) +
                              x_zeta * (y_xi * z_eta - y_eta * z_xi));
        xi[c] = (y_eta * z_zeta - y_zeta * z_eta) * jacob;
        xi[N + c] = (x_zeta * z_eta - x_eta * z_zeta) * jacob;
        xi[2 * N + c] = (x_eta * y_zeta - x_zeta * y_eta) * jacob;
        eta[c] = (y_zeta * z_xi - y_xi * z_zeta) * jacob;
        eta[N + c] = (x_xi * z_zeta - x_zeta * z_xi) * jacob;
        eta[2 * N + c] = (x_zeta * y_xi - x_xi * y_zeta) * jacob;
        zeta[c] = (y_xi * z_eta - y_eta * z_xi) * jacob;
        zeta[N + c] = (x_eta * z_xi - x_xi * z_eta) * jacob;
        zeta[2 * N + c] = (x_xi * y_eta - x_eta * y_xi) * jacob;
        jac[c] = jacob;
        for (int a = 0; a < 3; ++a)
          for (int dir = 0; dir < 3; ++dir) dxyz[(3 * a + dir) * N + c] = d[a][dir];
      }
  return 0;
}
