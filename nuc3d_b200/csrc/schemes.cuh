// schemes.cuh -- WENO-family face reconstruction and central differences.
//
// Each function evaluates one face (or one cell derivative) from values handed
// in stencil order, with the reference's operand order (see physics.cuh).
// Orientation: for the positive split F+ of face f (between cells f-1 and f) the
// 5-point stencil is (f-3, f-2, f-1, f, f+1); for F- it is the mirror
// (f+2, f+1, f, f-1, f-2).  The 7-point WENO7 stencils extend this by one cell.
// This is exactly the indexing of the reference's inner loops and its ghost-aware
// BL/BR variants (src/weno5js.cpp:59-108,136-185,252-268,470-486), which are one
// uniform stencil over the line extended by the neighbour's ghost cells.
#pragma once
#include "physics.cuh"

namespace nuc3d {
namespace NUC3D_NS {

// src/schemes.hpp:17-44
__device__ constexpr double kA5[3][3] = {{1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0},
                                         {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                                         {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0}};
__device__ constexpr double kA7[4][4] = {{-3.0 / 12.0, 13.0 / 12.0, -23.0 / 12.0, 25.0 / 12.0},
                                         {1.0 / 12.0, -5.0 / 12.0, 13.0 / 12.0, 3.0 / 12.0},
                                         {-1.0 / 12.0, 7.0 / 12.0, 7.0 / 12.0, -1.0 / 12.0},
                                         {3.0 / 12.0, 13.0 / 12.0, -5.0 / 12.0, 1.0 / 12.0}};
__device__ constexpr double kC5[3] = {0.1, 0.6, 0.3};
__device__ constexpr double kC7[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
__device__ constexpr double kG0 = 13.0 / 12.0;
__device__ constexpr double kG1 = 1.0 / 4.0;
__device__ constexpr double kCD6[3] = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
__device__ constexpr double kCD4[2] = {2.0 / 3.0, -1.0 / 12.0};
__device__ constexpr double kCD8[4] = {4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0};
__device__ constexpr double kCD2 = 0.5;

// WENO5 candidate values and smoothness indicators (src/weno5js.cpp:75-95).
struct W5 {
  double is0, is1, is2, q0, q1, q2;
};
__device__ __forceinline__ W5 w5_parts(double f0, double f1, double f2, double f3, double f4,
                                       bool is2_compat) {
  W5 r;
  r.is0 = kG0 * sq(f0 - 2.0 * f1 + f2) + kG1 * sq(f0 - 4.0 * f1 + 3.0 * f2);
  r.is1 = kG0 * sq(f1 - 2.0 * f2 + f3) + kG1 * sq(f1 - f3);
  // src/weno5z.cpp:80 reads f3 where f4 belongs in the first term of is2 on the
  // interior positive faces; is2_compat reproduces that stencil.
  r.is2 = kG0 * sq(f2 - 2.0 * f3 + (is2_compat ? f3 : f4)) + kG1 * sq(3.0 * f2 - 4.0 * f3 + f4);
  r.q0 = kA5[0][0] * f0 + kA5[0][1] * f1 + kA5[0][2] * f2;
  r.q1 = kA5[1][0] * f1 + kA5[1][1] * f2 + kA5[1][2] * f3;
  r.q2 = kA5[2][0] * f2 + kA5[2][1] * f3 + kA5[2][2] * f4;
  return r;
}

// WENO5-JS, eps 1e-6, p 2 (src/weno5js.cpp:7-8,97-108)
__device__ __forceinline__ double weno5js(double f0, double f1, double f2, double f3, double f4) {
  W5 r = w5_parts(f0, f1, f2, f3, f4, false);
  const double ss = 1.0e-6;
#if NUC3D_FAST
  // one division: omega_k = c_k P_k / sum_j c_j P_j with P_k = prod_{j!=k} (ss+is_j)^2
  double b0 = sq(ss + r.is0), b1 = sq(ss + r.is1), b2 = sq(ss + r.is2);
  double a0 = kC5[0] * (b1 * b2), a1 = kC5[1] * (b0 * b2), a2 = kC5[2] * (b0 * b1);
  return qdiv(a0 * r.q0 + a1 * r.q1 + a2 * r.q2, a0 + a1 + a2);
#else
  double a0 = kC5[0] / sq(ss + r.is0);
  double a1 = kC5[1] / sq(ss + r.is1);
  double a2 = kC5[2] / sq(ss + r.is2);
  double s = a0 + a1 + a2;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
  return w0 * r.q0 + w1 * r.q1 + w2 * r.q2;
#endif
}

// WENO5-Z, eps 1e-6, tau = |is2 - is0| (src/weno5z.cpp:96-109)
__device__ __forceinline__ double weno5z(double f0, double f1, double f2, double f3, double f4,
                                         bool is2_compat) {
  W5 r = w5_parts(f0, f1, f2, f3, f4, is2_compat);
  const double ss = 1.0e-6;
  double tau = fabs(r.is2 - r.is0);
#if NUC3D_FAST
  // alpha_k = c_k (1 + tau^2/d_k^2) = c_k (d_k^2 + tau^2) / d_k^2, d_k = is_k + ss
  double t2 = tau * tau;
  double d0 = sq(r.is0 + ss), d1 = sq(r.is1 + ss), d2 = sq(r.is2 + ss);
  double n0 = kC5[0] * (d0 + t2), n1 = kC5[1] * (d1 + t2), n2 = kC5[2] * (d2 + t2);
  double a0 = n0 * (d1 * d2), a1 = n1 * (d0 * d2), a2 = n2 * (d0 * d1);
  return qdiv(a0 * r.q0 + a1 * r.q1 + a2 * r.q2, a0 + a1 + a2);
#else
  double a0 = kC5[0] * (1.0 + sq(tau / (r.is0 + ss)));
  double a1 = kC5[1] * (1.0 + sq(tau / (r.is1 + ss)));
  double a2 = kC5[2] * (1.0 + sq(tau / (r.is2 + ss)));
  double s = a0 + a1 + a2;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
  return w0 * r.q0 + w1 * r.q1 + w2 * r.q2;
#endif
}

// WENO7-JS, eps 1e-40 (src/weno7js.cpp:13-16,84-136)
__device__ __forceinline__ double weno7js(const double f[7]) {
  double is0 = f[0] * (547.0 * f[0] - 3882.0 * f[1] + 4642.0 * f[2] - 1854.0 * f[3]) +
               f[1] * (7043.0 * f[1] - 17246.0 * f[2] + 7042.0 * f[3]) +
               f[2] * (11003.0 * f[2] - 9402.0 * f[3]) + 2107.0 * f[3] * f[3];
  double is1 = f[1] * (267.0 * f[1] - 1642.0 * f[2] + 1602.0 * f[3] - 494.0 * f[4]) +
               f[2] * (2843.0 * f[2] - 5966.0 * f[3] + 1922.0 * f[4]) +
               f[3] * (3443.0 * f[3] - 2522.0 * f[4]) + 547.0 * f[4] * f[4];
  double is2 = f[2] * (547.0 * f[2] - 2522.0 * f[3] + 1922.0 * f[4] - 494.0 * f[5]) +
               f[3] * (3443.0 * f[3] - 5966.0 * f[4] + 1602.0 * f[5]) +
               f[4] * (2843.0 * f[4] - 1642.0 * f[5]) + 267.0 * f[5] * f[5];
  double is3 = f[3] * (2107.0 * f[3] - 9402.0 * f[4] + 7042.0 * f[5] - 1854.0 * f[6]) +
               f[4] * (11003.0 * f[4] - 17246.0 * f[5] + 4642.0 * f[6]) +
               f[5] * (7043.0 * f[5] - 3882.0 * f[6]) + 547.0 * f[6] * f[6];
  double q0 = kA7[0][0] * f[0] + kA7[0][1] * f[1] + kA7[0][2] * f[2] + kA7[0][3] * f[3];
  double q1 = kA7[1][0] * f[1] + kA7[1][1] * f[2] + kA7[1][2] * f[3] + kA7[1][3] * f[4];
  double q2 = kA7[2][0] * f[2] + kA7[2][1] * f[3] + kA7[2][2] * f[4] + kA7[2][3] * f[5];
  double q3 = kA7[3][0] * f[3] + kA7[3][1] * f[4] + kA7[3][2] * f[5] + kA7[3][3] * f[6];
  const double ss = 1.0e-40;
#if NUC3D_FAST
  double b0 = sq(ss + is0), b1 = sq(ss + is1), b2 = sq(ss + is2), b3 = sq(ss + is3);
  double b01 = b0 * b1, b23 = b2 * b3;
  double a0 = kC7[0] * (b1 * b23), a1 = kC7[1] * (b0 * b23), a2 = kC7[2] * (b01 * b3),
         a3 = kC7[3] * (b01 * b2);
  return qdiv(a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3, a0 + a1 + a2 + a3);
#else
  double a0 = kC7[0] / sq(ss + is0);
  double a1 = kC7[1] / sq(ss + is1);
  double a2 = kC7[2] / sq(ss + is2);
  double a3 = kC7[3] / sq(ss + is3);
  double s = a0 + a1 + a2 + a3;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s, w3 = a3 / s;
  return w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
#endif
}

// WENO7-Z: the 7th-order stencils of weno7js with Z weights, tau7 = |is0 - is3|,
// eps 1e-40 -- hccs's block-edge faces and explicit end rows (src/hccs.cpp:92-142,516-990).
__device__ __forceinline__ double weno7z(const double f[7]) {
  double is0 = f[0] * (547.0 * f[0] - 3882.0 * f[1] + 4642.0 * f[2] - 1854.0 * f[3]) +
               f[1] * (7043.0 * f[1] - 17246.0 * f[2] + 7042.0 * f[3]) +
               f[2] * (11003.0 * f[2] - 9402.0 * f[3]) + 2107.0 * f[3] * f[3];
  double is1 = f[1] * (267.0 * f[1] - 1642.0 * f[2] + 1602.0 * f[3] - 494.0 * f[4]) +
               f[2] * (2843.0 * f[2] - 5966.0 * f[3] + 1922.0 * f[4]) +
               f[3] * (3443.0 * f[3] - 2522.0 * f[4]) + 547.0 * f[4] * f[4];
  double is2 = f[2] * (547.0 * f[2] - 2522.0 * f[3] + 1922.0 * f[4] - 494.0 * f[5]) +
               f[3] * (3443.0 * f[3] - 5966.0 * f[4] + 1602.0 * f[5]) +
               f[4] * (2843.0 * f[4] - 1642.0 * f[5]) + 267.0 * f[5] * f[5];
  double is3 = f[3] * (2107.0 * f[3] - 9402.0 * f[4] + 7042.0 * f[5] - 1854.0 * f[6]) +
               f[4] * (11003.0 * f[4] - 17246.0 * f[5] + 4642.0 * f[6]) +
               f[5] * (7043.0 * f[5] - 3882.0 * f[6]) + 547.0 * f[6] * f[6];
  double q0 = kA7[0][0] * f[0] + kA7[0][1] * f[1] + kA7[0][2] * f[2] + kA7[0][3] * f[3];
  double q1 = kA7[1][0] * f[1] + kA7[1][1] * f[2] + kA7[1][2] * f[3] + kA7[1][3] * f[4];
  double q2 = kA7[2][0] * f[2] + kA7[2][1] * f[3] + kA7[2][2] * f[4] + kA7[2][3] * f[5];
  double q3 = kA7[3][0] * f[3] + kA7[3][1] * f[4] + kA7[3][2] * f[5] + kA7[3][3] * f[6];
  const double ss = 1.0e-40;
  double tau7 = fabs(is0 - is3);
  double a0 = kC7[0] * (1.0 + sq(tau7 / (ss + is0)));
  double a1 = kC7[1] * (1.0 + sq(tau7 / (ss + is1)));
  double a2 = kC7[2] * (1.0 + sq(tau7 / (ss + is2)));
  double a3 = kC7[3] * (1.0 + sq(tau7 / (ss + is3)));
  double s = a0 + a1 + a2 + a3;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s, w3 = a3 / s;
  return w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3;
}

// Interior row of the CRWENO5 tridiagonal system on an oriented 5-cell stencil f[0..4]
// (src/crweno5.cpp:130-161 for F+, :310-340 for F-): JS indicators, weights
// 0.2/0.5/0.3, eps 1e-6.  lo multiplies the unknown on the upwind side (a of F+, c of
// F-), up the one on the downwind side.
__device__ constexpr double kCR5[3] = {0.2, 0.5, 0.3};
__device__ __forceinline__ void crweno5_row(const double f[5], double &lo, double &di, double &up,
                                            double &rhs) {
  W5 r = w5_parts(f[0], f[1], f[2], f[3], f[4], false);
  const double ss = 1.0e-6;
#if NUC3D_FAST
  // The row scaled by sum_k alpha_k * prod_k (ss+is_k)^2 (its solution is unchanged): the
  // weights become n_k = c_k prod_{j!=k} (ss+is_j)^2, with no division at all.
  {
    const double d0 = sq(ss + r.is0), d1 = sq(ss + r.is1), d2 = sq(ss + r.is2);
    const double n0 = kCR5[0] * (d1 * d2), n1 = kCR5[1] * (d0 * d2), n2 = kCR5[2] * (d0 * d1);
    lo = 2.0 / 3.0 * n0 + 1.0 / 3.0 * n1;
    di = 1.0 / 3.0 * n0 + 2.0 / 3.0 * (n1 + n2);
    up = 1.0 / 3.0 * n2;
    rhs = 1.0 / 6.0 * n0 * f[1] + (5.0 * (n0 + n1) + n2) * (1.0 / 6.0) * f[2] + (n1 + 5.0 * n2) * (1.0 / 6.0) * f[3];
    return;
  }
#endif
  double a0 = kCR5[0] / sq(ss + r.is0);
  double a1 = kCR5[1] / sq(ss + r.is1);
  double a2 = kCR5[2] / sq(ss + r.is2);
  double s = a0 + a1 + a2;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
  lo = 2.0 / 3.0 * w0 + 1.0 / 3.0 * w1;
  di = 1.0 / 3.0 * w0 + 2.0 / 3.0 * (w1 + w2);
  up = 1.0 / 3.0 * w2;
  rhs = 1.0 / 6.0 * w0 * f[1] + (5.0 * (w0 + w1) + w2) * f[2] / 6.0 + (w1 + 5.0 * w2) * f[3] / 6.0;
}

// Interior row of the hybrid compact scheme (src/hccs.cpp:145-188 for F+, :371-414
// for F-): CRWENO5-Z weights (eps 1e-40), blended with the 7th-order compact central row
// (2/7, 4/7, 1/7 | q7) by theta = 1/(1 + (sum alpha - 1)^2).
__device__ __forceinline__ void hccs_row(const double f[5], double &lo, double &di, double &up,
                                         double &rhs) {
  W5 r = w5_parts(f[0], f[1], f[2], f[3], f[4], false);
  const double ss = 1.0e-40;
#if NUC3D_FAST
  // alpha_k = c_k (e_k + tau^2) / e_k, e_k = (is_k + ss)^2: with den = e0 e1 e2 the
  // numerators m_k = c_k (e_k + tau^2) prod_{j!=k} e_j sum to S = den * sum alpha, so theta
  // takes one division (sum alpha = S / den) and its reciprocal a second; the WENO part of
  // the row is scaled by S and the central part by S as well (the solution is unchanged).
  {
    const double tau = fabs(r.is2 - r.is0), t2 = tau * tau;
    const double e0 = sq(r.is0 + ss), e1 = sq(r.is1 + ss), e2 = sq(r.is2 + ss);
    const double m0 = kCR5[0] * (e0 + t2) * (e1 * e2), m1 = kCR5[1] * (e1 + t2) * (e0 * e2),
                 m2 = kCR5[2] * (e2 + t2) * (e0 * e1);
    const double S = m0 + m1 + m2;
    const double sa = qdiv(S, e0 * (e1 * e2));
    const double theta = qdiv(1.0, 1.0 + sq(sa - 1.0)), omt = 1.0 - theta, ts = theta * S;
    const double q7 = (-f[0] + 19.0 * f[1] + 239.0 * f[2] + 159.0 * f[3] + 4.0 * f[4]) * (1.0 / 420.0);
    lo = (2.0 / 3.0 * m0 + 1.0 / 3.0 * m1) * omt + 2.0 / 7.0 * ts;
    di = (1.0 / 3.0 * m0 + 2.0 / 3.0 * (m1 + m2)) * omt + 4.0 / 7.0 * ts;
    up = (1.0 / 3.0 * m2) * omt + 1.0 / 7.0 * ts;
    rhs = (1.0 / 6.0 * m0 * f[1] + (5.0 * (m0 + m1) + m2) * (1.0 / 6.0) * f[2] +
           (m1 + 5.0 * m2) * (1.0 / 6.0) * f[3]) * omt + q7 * ts;
    return;
  }
#endif
  double q7 = (-f[0] + 19.0 * f[1] + 239.0 * f[2] + 159.0 * f[3] + 4.0 * f[4]) / 420.0;
  double tau = fabs(r.is2 - r.is0);
  double a0 = kCR5[0] * (1.0 + sq(tau / (r.is0 + ss)));
  double a1 = kCR5[1] * (1.0 + sq(tau / (r.is1 + ss)));
  double a2 = kCR5[2] * (1.0 + sq(tau / (r.is2 + ss)));
  double s = a0 + a1 + a2;
  double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
  double theta = 1.0 / (1.0 + sq(s - 1.0));
  lo = (2.0 / 3.0 * w0 + 1.0 / 3.0 * w1) * (1.0 - theta) + 2.0 / 7.0 * theta;
  di = (1.0 / 3.0 * w0 + 2.0 / 3.0 * (w1 + w2)) * (1.0 - theta) + 4.0 / 7.0 * theta;
  up = (1.0 / 3.0 * w2) * (1.0 - theta) + 1.0 / 7.0 * theta;
  rhs = (1.0 / 6.0 * w0 * f[1] + (5.0 * (w0 + w1) + w2) * f[2] / 6.0 + (w1 + 5.0 * w2) * f[3] / 6.0) *
            (1.0 - theta) +
        q7 * theta;
}

// Reduced-order schemes on faces next to a physical boundary
// (ReconstructionboundaryScheme, src/reconstructionBoundaryScheme.cpp:315-463).
__device__ __forceinline__ double rb_second(double f0, double f1) { return 0.5 * (f0 + f1); }
__device__ __forceinline__ double rb_third(double f0, double f1, double f2) {
  double is0 = sq(f0 - f1);
  double is1 = sq(f1 - f2);
  double q20 = -0.5 * f0 + 1.5 * f1;
  double q21 = 0.5 * f1 + 0.5 * f2;
#if NUC3D_FAST
  // one division: w0 : w1 = (1/3)/e0^2 : (2/3)/e1^2 = e1^2 : 2 e0^2, e_k = 1e-6 + is_k
  const double b0 = sq(1.0e-6 + is0), b1 = sq(1.0e-6 + is1);
  return qdiv(b1 * q20 + 2.0 * b0 * q21, b1 + 2.0 * b0);
#endif
  double aa0 = 1.0 / 3.0 / sq(1.0e-6 + is0);
  double aa1 = 2.0 / 3.0 / sq(1.0e-6 + is1);
  double w0 = aa0 / (aa0 + aa1);
  double w1 = aa1 / (aa0 + aa1);
  return w0 * q20 + w1 * q21;
}

// d/dxi at one cell.  cd6 (src/centraldifference6th.cpp:75-77) and the exterior
// one-sided family boundaryScheme (src/boundaryScheme.cpp:380-406).  sixthOrder
// there pairs the cd6 outer terms with the 4th-order inner coefficient
// (src/boundaryScheme.cpp:405); kept as is.
__device__ __forceinline__ double cd6(double m3, double m2, double m1, double p1, double p2,
                                      double p3) {
  return kCD6[2] * (p3 - m3) + kCD6[1] * (p2 - m2) + kCD6[0] * (p1 - m1);
}
// centraldifference8th (src/centraldifference8th.cpp:16-52)
__device__ __forceinline__ double cd8(double m4, double m3, double m2, double m1, double p1,
                                      double p2, double p3, double p4) {
  return kCD8[3] * (p4 - m4) + kCD8[2] * (p3 - m3) + kCD8[1] * (p2 - m2) + kCD8[0] * (p1 - m1);
}
// centraldifference2nd (src/centraldifference2nd.cpp:16-37)
__device__ __forceinline__ double cd2(double m1, double p1) { return 0.5 * (p1 - m1); }
__device__ __forceinline__ double bnd_second(double m1, double p1) { return kCD2 * (p1 - m1); }
__device__ __forceinline__ double bnd_fourth(double m2, double m1, double p1, double p2) {
  return kCD4[1] * (p2 - m2) + kCD4[0] * (p1 - m1);
}
__device__ __forceinline__ double bnd_sixth(double m3, double m2, double m1, double p1, double p2,
                                            double p3) {
  return kCD6[2] * (p3 - m3) + kCD6[1] * (p2 - m2) + kCD4[0] * (p1 - m1);
}

}  // namespace NUC3D_NS
}  // namespace nuc3d
