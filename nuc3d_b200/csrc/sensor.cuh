// sensor.cuh -- the learned smoothness sensor of the hybrid WENO-Z path: face features,
// training labels, and the kernel that records them from a plain WENO-Z sweep.
//
// Per interior face f of a line (cells f-1 | f), 19 features:
//   x[3v+k], v = 0..4, k = 0..2   beta_k / (beta_0 + beta_1 + beta_2 + 1e-6): the WENO5
//                                 smoothness indicators of the positive split flux of
//                                 variable v on cells f-3 .. f+1 (src/weno5js.cpp:75-86),
//                                 normalised with the scheme's epsilon
//   x[15], x[16]                  |rho_f - rho_(f-1)| / (rho_f + rho_(f-1)), same for p
//   x[17], x[18]                  the largest such jump of rho, of p, over the cell pairs
//                                 of the stencil f-3 .. f+2
// Label: 1 when, for any variable and either split, a WENO-Z weight deviates from its
// linear weight (0.1, 0.6, 0.3) by more than kSensorDeviation: the face needs the
// nonlinear weights.  Included by kernels.cuh inside the build's namespace.
#pragma once

constexpr int kSensorIn = 19, kSensorHidden = 32;
constexpr double kSensorDeviation = 0.05;

// Row accessor convention: P(c) = F+ of variable v at line position face + c.
template <class Acc>
__device__ __forceinline__ void sensor_betas(Acc P, double b[3]) {
  const double f0 = P(-3), f1 = P(-2), f2 = P(-1), f3 = P(0), f4 = P(1);
  b[0] = kG0 * sq(f0 - 2.0 * f1 + f2) + kG1 * sq(f0 - 4.0 * f1 + 3.0 * f2);
  b[1] = kG0 * sq(f1 - 2.0 * f2 + f3) + kG1 * sq(f1 - f3);
  b[2] = kG0 * sq(f2 - 2.0 * f3 + f4) + kG1 * sq(3.0 * f2 - 4.0 * f3 + f4);
}

__device__ __forceinline__ float rel_jump(double a, double b) {
  return (float)(fabs(b - a) / (fabs(a) + fabs(b) + 1e-300));
}

// rho(c), pr(c): density and pressure at line position face + c
template <class AccR, class AccPr>
__device__ __forceinline__ void sensor_jumps(AccR rho, AccPr pr, float x[4]) {
  x[0] = rel_jump(rho(-1), rho(0));
  x[1] = rel_jump(pr(-1), pr(0));
  float mr = 0.0f, mp = 0.0f;
#pragma unroll
  for (int c = -3; c < 2; ++c) {
    mr = fmaxf(mr, rel_jump(rho(c), rho(c + 1)));
    mp = fmaxf(mp, rel_jump(pr(c), pr(c + 1)));
  }
  x[2] = mr;
  x[3] = mp;
}

// Largest |omega_k - d_k| of a WENO-Z reconstruction (src/weno5z.cpp:96-109).
__device__ __forceinline__ double weno5z_deviation(double f0, double f1, double f2, double f3,
                                                   double f4, bool compat) {
  W5 r = w5_parts(f0, f1, f2, f3, f4, compat);
  const double tau = fabs(r.is2 - r.is0);
  const double a0 = kC5[0] * (1.0 + sq(tau / (r.is0 + 1.0e-6)));
  const double a1 = kC5[1] * (1.0 + sq(tau / (r.is1 + 1.0e-6)));
  const double a2 = kC5[2] * (1.0 + sq(tau / (r.is2 + 1.0e-6)));
  const double s = a0 + a1 + a2;
  return fmax(fabs(a0 / s - kC5[0]), fmax(fabs(a1 / s - kC5[1]), fabs(a2 / s - kC5[2])));
}

// Features and label of every interior face of a WENO-Z sweep tile: phase 1 of the
// sweep, then one thread per face.  Faces are appended at *count (order unspecified);
// at most cap are written.  where (may be null) gets each face's index in the block's
// face grid of direction DIR: faces along DIR have extent n[DIR] + 1, i fastest.
template <int DIR, int SHP>
__global__ void __launch_bounds__(kThreads, NUC3D_SWEEP_MINB)
sensor_data_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
                   int stage, float *__restrict__ feat, unsigned char *__restrict__ label,
                   long long *__restrict__ where, unsigned long long *count,
                   unsigned long long cap) {
  using M = TileSmem<DIR, SCH_WENO5Z, SHP>;
  constexpr int R = M::R, TW = M::TW, TL = M::TL, SP = M::SP;
  extern __shared__ double smem[];
  double *sF = smem;                 // [10][TW][SP]
  double *sRP = sF + 10 * TW * SP;   // [2][TW][SP]: rho, p
  const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P);
  unsigned st = 0;
  double emax = 0.0;
  phase_split<DIR, SCH_WENO5Z, true, SHP>(blocks, T, P, stage, false, sF, nullptr, st, emax, sRP);
  __syncthreads();
  const bool compat = P.weno5z_compat != 0;
  for (int e = threadIdx.x; e < TW * (TL + 1); e += kThreads) {
    const int fl = e % (TL + 1), w = e / (TL + 1);
    if (w >= T.nw || fl > T.cl) continue;
    const int f = T.c0 + fl;
    if ((T.physR && f > T.G.L - T.ts) || (T.physL && f < T.ts)) continue;  // boundary schemes
    float x[kSensorIn];
    double dev = 0.0;
    const bool cz = compat && f >= T.ts && f <= T.G.L - T.ts;
#pragma unroll 1
    for (int v = 0; v < 5; ++v) {
      const double *rowP = sF + (v * TW + w) * SP + (R + fl);
      const double *rowN = sF + ((5 + v) * TW + w) * SP + (R + fl);
      auto Pacc = [rowP](int c) { return rowP[c]; };
      double b[3];
      sensor_betas(Pacc, b);
      const double den = b[0] + b[1] + b[2] + 1.0e-6;
#pragma unroll
      for (int k = 0; k < 3; ++k) x[3 * v + k] = (float)(b[k] / den);
      dev = fmax(dev, weno5z_deviation(rowP[-3], rowP[-2], rowP[-1], rowP[0], rowP[1], cz));
      dev = fmax(dev, weno5z_deviation(rowN[2], rowN[1], rowN[0], rowN[-1], rowN[-2], false));
    }
    const double *rr = sRP + w * SP + (R + fl), *pp = sRP + (TW + w) * SP + (R + fl);
    sensor_jumps([rr](int c) { return rr[c]; }, [pp](int c) { return pp[c]; }, x + 15);
    const unsigned long long slot = atomicAdd(count, 1ull);
    if (slot < cap) {
#pragma unroll
      for (int i = 0; i < kSensorIn; ++i) feat[slot * kSensorIn + i] = x[i];
      label[slot] = dev > kSensorDeviation ? 1 : 0;
      if (where) {
        int c[3];  // (i, j, k) of the face in the face grid
        const int wl = T.w0 + w;
        if (DIR == 0) { c[0] = f; c[1] = wl; c[2] = T.o; }
        else if (DIR == 1) { c[0] = wl; c[1] = f; c[2] = T.o; }
        else { c[0] = wl; c[1] = T.o; c[2] = f; }
        const long long ex = T.n[0] + (DIR == 0), ey = T.n[1] + (DIR == 1);
        where[slot] = ((long long)c[2] * ey + c[1]) * ex + c[0];
      }
    }
  }
  if (st) atomicOr(&S->status, st);
}

// ---------------------------------------------------------------------------------
// Inference in the sweep (throughput build).  One warp evaluates the 32 faces of its
// lanes at once on the tensor cores: mma.sync m16n8k16, BF16 operands, FP32 accumulators.
// Layer 1 (19 -> 32) takes its A fragments from the face owners' packed features by
// shuffles; its accumulators, ReLU'd and rounded to BF16, are layer 2's A fragments as
// they lie in the registers; layer 3 (32 -> 1) is a per-lane partial dot product plus a
// reduction over the four lanes of a quad.  The same BF16 roundings as the training.
// Every lane of the warp must call it (lanes without a face pass zero features).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Pair p (features 2p, 2p+1) of lane src's packed features, for this lane's column pair q.
__device__ __forceinline__ uint32_t gather_pair(const uint32_t xr[10], int base, int q, int src) {
  uint32_t v = 0;
#pragma unroll
  for (int qq = 0; qq < 4; ++qq) {
    const int pidx = base + qq;
    if (pidx < 10) {
      const uint32_t t = __shfl_sync(0xffffffffu, xr[pidx], src);
      if (q == qq) v = t;
    }
  }
  return v;
}

// The logit of this lane's face by the network.  xr: the lane's 19 features as BF16 pairs
// (pair 9 holds feature 18 and a zero).  S may point to global or shared memory: generic
// loads only (no __ldg, whose non-coherent global path cannot read shared memory).  The
// two m-tiles run unrolled: their independent chains overlap (the unrolled form measured
// 25% off the hybrid step at 256^3).
__device__ __forceinline__ float sensor_logit_net(const SensorDev *S, const uint32_t xr[10]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  float mine = 0.0f;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = mt * 16 + g, r8 = r0 + 8;  // owner lanes of fragment rows g, g+8
    float c[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const float b0 = S->b1[nt * 8 + 2 * q], b1 = S->b1[nt * 8 + 2 * q + 1];
      c[nt][0] = b0; c[nt][1] = b1; c[nt][2] = b0; c[nt][3] = b1;
    }
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      const uint32_t a0 = gather_pair(xr, ks * 8, q, r0), a1 = gather_pair(xr, ks * 8, q, r8);
      const uint32_t a2 = gather_pair(xr, ks * 8 + 4, q, r0), a3 = gather_pair(xr, ks * 8 + 4, q, r8);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const uint2 bw = *reinterpret_cast<const uint2 *>(S->w1[ks][nt][lane]);
        mma_bf16(c[nt], a0, a1, a2, a3, bw.x, bw.y);
      }
    }
    uint32_t h[2][4];  // layer-2 A fragments: ReLU, BF16
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      const float *lo = c[2 * ks], *hi = c[2 * ks + 1];
      h[ks][0] = bf16_pair(fmaxf(lo[0], 0.0f), fmaxf(lo[1], 0.0f));
      h[ks][1] = bf16_pair(fmaxf(lo[2], 0.0f), fmaxf(lo[3], 0.0f));
      h[ks][2] = bf16_pair(fmaxf(hi[0], 0.0f), fmaxf(hi[1], 0.0f));
      h[ks][3] = bf16_pair(fmaxf(hi[2], 0.0f), fmaxf(hi[3], 0.0f));
    }
    float pg = 0.0f, pg8 = 0.0f;  // partial logits of rows g and g+8
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int n0 = nt * 8 + 2 * q;
      float d[4] = {S->b2[n0], S->b2[n0 + 1], S->b2[n0], S->b2[n0 + 1]};
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint2 bw = *reinterpret_cast<const uint2 *>(S->w2[ks][nt][lane]);
        mma_bf16(d, h[ks][0], h[ks][1], h[ks][2], h[ks][3], bw.x, bw.y);
      }
      pg += bf16_round(fmaxf(d[0], 0.0f)) * S->w3[n0] + bf16_round(fmaxf(d[1], 0.0f)) * S->w3[n0 + 1];
      pg8 += bf16_round(fmaxf(d[2], 0.0f)) * S->w3[n0] + bf16_round(fmaxf(d[3], 0.0f)) * S->w3[n0 + 1];
    }
    pg += __shfl_xor_sync(0xffffffffu, pg, 1);
    pg += __shfl_xor_sync(0xffffffffu, pg, 2);
    pg8 += __shfl_xor_sync(0xffffffffu, pg8, 1);
    pg8 += __shfl_xor_sync(0xffffffffu, pg8, 2);
    // the owner of row rho (lane 16 mt + rho) takes it from quad 4 (rho mod 8)
    const float lg = __shfl_sync(0xffffffffu, pg, 4 * (lane & 7));
    const float lg8 = __shfl_sync(0xffffffffu, pg8, 4 * (lane & 7));
    if ((lane >> 4) == mt) mine = S->b3 + ((lane & 15) < 8 ? lg : lg8);
  }
  return mine;
}

// The logit of this lane's face.  A warp whose 32 faces all have zero features (inside a
// uniform region) takes the network's precomputed output for zero input: each output
// row of the mma depends on its own row of features only, so this is the value the
// network would return for them.
__device__ __forceinline__ float sensor_logit(const SensorDev *S, const uint32_t xr[10]) {
  uint32_t any = 0u;
#pragma unroll
  for (int i = 0; i < 10; ++i) any |= xr[i];
  if (__all_sync(0xffffffffu, any == 0u)) return S->zero_logit;
  return sensor_logit_net(S, xr);
}

__global__ void sensor_zero_kernel(SensorDev *S) {
  uint32_t xr[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) xr[i] = 0u;
  const float z = sensor_logit_net(S, xr);
  if (threadIdx.x == 0) S->zero_logit = z;
}

cudaError_t run_sensor_zero(SensorDev *S, cudaStream_t st) {
  sensor_zero_kernel<<<1, 32, 0, st>>>(S);
  return cudaGetLastError();
}

// The sweep's features are built from per-gap values that neighbouring faces share.
// Gap p of a line joins tile positions p and p+1; sG holds, per gap, the first
// differences of the 5 variables' F+ (FP64 subtraction, then FP32) and the relative
// density and pressure jumps: sG[k][w][p], k = 0..4 differences, 5 density, 6 pressure.
constexpr int kSensorGapVals = 7;

__device__ __forceinline__ float rel_jump_f(float a, float b) {
  return fabsf(b - a) * __frcp_rn(fabsf(a) + fabsf(b) + 1e-30f);
}

// Gap p of line w: rowF[v] = F+ of variable v at position 0 of the line, rr/pp = density
// and pressure likewise; out[k] is sG[k][w] (stride gs floats between k).  Returns whether
// all seven values are zero (a gap inside a uniform region).
__device__ __forceinline__ bool sensor_gap(const double *const rowF[5], const double *rr,
                                           const double *pp, int p, float *out, int gs) {
  // A difference at the round-off level of the split fluxes counts as none: metrics
  // computed from a mesh (block::getJacobians) carry relative noise near 1e-14 even on a
  // uniform grid, so a uniform region's fluxes differ in their last bits, and a component
  // whose exact value is zero (a transverse metric term) is noise alone.  The scale is the
  // pair's largest flux component: below 2^-32 of it a difference moves the features by
  // far less than BF16 resolves, and counting it as zero keeps such regions on the
  // zero-input decision (and its shortcuts).
  double scale = 0.0;
#pragma unroll
  for (int v = 0; v < 5; ++v) scale = fmax(scale, fmax(fabs(rowF[v][p]), fabs(rowF[v][p + 1])));
  const double tiny = 0x1p-32 * scale;
  bool zero = true;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const double dd = rowF[v][p + 1] - rowF[v][p];
    const float d = fabs(dd) <= tiny ? 0.0f : (float)dd;
    out[v * gs] = d;
    zero = zero && d == 0.0f;
  }
  const float jr = rel_jump_f((float)rr[p], (float)rr[p + 1]);
  const float jp = rel_jump_f((float)pp[p], (float)pp[p + 1]);
  out[5 * gs] = jr;
  out[6 * gs] = jp;
  return zero && jr == 0.0f && jp == 0.0f;
}

// The 19 features of one face from the gaps g = first gap of its stencil (cells f-3, f-2)
// .. g+4, packed as BF16 pairs: the WENO5 smoothness indicators of F+ rewritten on first
// differences D0..D3 of the stencil f-3..f+1 (d = second difference, e = the indicator's
// first-derivative term), normalised by their sum + 1e-6, then the jumps across the face
// and their maxima over the stencil, as in sensor_data_kernel.
__device__ __forceinline__ void sensor_features_gaps(const float *g, int gs, uint32_t xr[10]) {
  float x[kSensorIn];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const float D0 = g[v * gs], D1 = g[v * gs + 1], D2 = g[v * gs + 2], D3 = g[v * gs + 3];
    const float d0 = D1 - D0, e0 = 3.0f * D1 - D0;
    const float d1 = D2 - D1, e1 = D1 + D2;
    const float d2 = D3 - D2, e2 = D3 - 3.0f * D2;
    const float b0 = (13.0f / 12.0f) * d0 * d0 + 0.25f * e0 * e0;
    const float b1 = (13.0f / 12.0f) * d1 * d1 + 0.25f * e1 * e1;
    const float b2 = (13.0f / 12.0f) * d2 * d2 + 0.25f * e2 * e2;
    const float inv = __frcp_rn(b0 + b1 + b2 + 1.0e-6f);
    x[3 * v] = b0 * inv;
    x[3 * v + 1] = b1 * inv;
    x[3 * v + 2] = b2 * inv;
  }
  const float *jr = g + 5 * gs, *jp = g + 6 * gs;
  x[15] = jr[2];
  x[16] = jp[2];
  float mr = jr[0], mp = jp[0];
#pragma unroll
  for (int c = 1; c < 5; ++c) {
    mr = fmaxf(mr, jr[c]);
    mp = fmaxf(mp, jp[c]);
  }
  x[17] = mr;
  x[18] = mp;
#pragma unroll
  for (int i = 0; i < 9; ++i) xr[i] = bf16_pair(x[2 * i], x[2 * i + 1]);
  xr[9] = bf16_pair(x[18], 0.0f);
}

// WENO5 with the linear weights (0.1, 0.6, 0.3): the fifth-order upwind face value.
__device__ __forceinline__ double weno5_linear(double f0, double f1, double f2, double f3, double f4) {
  const W5 r = w5_parts(f0, f1, f2, f3, f4, false);
  return kC5[0] * r.q0 + kC5[1] * r.q1 + kC5[2] * r.q2;
}
