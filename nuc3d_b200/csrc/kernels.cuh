// kernels.cuh -- the per-stage kernels of the block RHS + TVD-RK3 update.
//
// Included twice: kernels_exact.cu (NUC3D_NS = exact, built with -fmad=false, the
// reference's operation order, bit-comparable with the CPU oracle) and
// kernels_fast.cu (NUC3D_NS = fast, FMA contraction and one-division WENO weights).
//
// One RK stage s (state Q_s = q[s]; stage 0 also fixes dt):
//   [NS]  prim_kernel   u, v, w, T of every cell              (src/physicsModel.cpp:258-357)
//   [NS]  grad_kernel   12 cd6 gradients, Sutherland, stress,   (src/NaiverStokes3d.cpp:63-326)
//                       contravariant viscous fluxes
//   sweep<0>  xi:   split F+/F- (src/physicsModel.cpp:420-760), ghost fill from the neighbour
//                   block or the BC (src/boundaryConditions.cpp:95-1086), WENO faces
//                   (src/euler3d.cpp:305-366), dF = F[i+1/2]-F[i-1/2] (:143-174),
//                   RHS = dF; stage 0 also reduces max(|U|+c|grad xi|) over 3 directions
//   sweep<1>  eta:  RHS += dG
//   sweep<2>  zeta: RHS += dH, [NS] RHS -= dFv + dGv + dHv (src/NaiverStokes3d.cpp:401-513),
//                   then the TVD-RK3 stage update (src/TVD-RK3.cpp:16-137) into q[s+1 mod 3]
// Ghost cells across block faces are read directly from the neighbour block's
// arrays in HBM; this replaces the MPI halo exchange (src/MPICommunicator.cpp:36-115).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "schemes.cuh"

namespace nuc3d {
namespace NUC3D_NS {

// Tile of one sweep CTA: TW lines side by side, TL cells along each line, TW*TL = 256
// in every shape (tile_w / tile_l).  xi lines are contiguous in memory; eta/zeta tiles
// put TW consecutive i in a row (shape 0: one 32-byte sector).  kThreads = 256 + 32 makes
// every phase of shape 0 a single round: TW*(TL+2R) <= 288 split fluxes, TW*(TL+1)
// faces, TW*TL cells, so no warp idles at a barrier waiting for a one-lane tail.
#ifndef NUC3D_SWEEP_MINB
#define NUC3D_SWEEP_MINB 4  // resident sweep CTAs per SM the register budget is cut for (measured best)
#endif
#ifndef NUC3D_SWEEP_MINB_Z
#define NUC3D_SWEEP_MINB_Z NUC3D_SWEEP_MINB  // the same for the zeta sweep (RK epilogue)
#endif
#ifndef NUC3D_RHS_PREFETCH_Z
#define NUC3D_RHS_PREFETCH_Z 0
#endif
constexpr int kThreads = 256 + 32;
template <int SHP> struct Tile {
  static constexpr int TW = tile_w(SHP), TL = tile_l(SHP);
  static_assert(TW * TL == 256 || SHP >= kLineShape, "every sweep tile shape holds 256 cells");
};

template <int SCH> struct Halo {
  static constexpr int R = (SCH == SCH_WENO7JS || SCH == SCH_HCCS) ? 4
                           : SCH == SCH_WENO3JS ? 2 : SCH == SCH_UPWIND1 ? 1 : 3;
};
// Halo of the viscous tiles: the widest viscous stencil (cd8) reaches 4 cells.
constexpr int kVisHalo = 4;

// Row strides of the shared-memory tiles, padded so that the TW rows of one warp
// access fall in different bank halves (stride = 8 mod 16 doubles).
__host__ __device__ constexpr int pad_row(int n) { return ((n + 7) / 16) * 16 + 8; }

struct Geo {
  int L, nW, nO;
  long long sL, sW, sO;
};

__host__ __device__ inline Geo make_geo(int dir, const int n[3]) {
  Geo g;
  long long nxy = (long long)n[0] * n[1];
  if (dir == 0) {
    g.L = n[0]; g.nW = n[1]; g.nO = n[2]; g.sL = 1; g.sW = n[0]; g.sO = nxy;
  } else if (dir == 1) {
    g.L = n[1]; g.nW = n[0]; g.nO = n[2]; g.sL = n[0]; g.sW = 1; g.sO = nxy;
  } else {
    g.L = n[2]; g.nW = n[0]; g.nO = n[1]; g.sL = nxy; g.sW = 1; g.sO = n[0];
  }
  return g;
}

__host__ __device__ inline int sweep_tiles(int dir, const int n[3], int shape) {
  Geo g = make_geo(dir, n);
  const int TL = tile_l(shape), TW = tile_w(shape);
  return ((g.L + TL - 1) / TL) * ((g.nW + TW - 1) / TW) * g.nO;
}

template <int DIR, int SCH, int SHP = 0>
__host__ __device__ constexpr size_t sweep_smem_bytes(bool ns) {
  constexpr int R = Halo<SCH>::R, TW = Tile<SHP>::TW, TL = Tile<SHP>::TL;
  size_t n = (size_t)10 * TW * pad_row(TL + 2 * R) + (size_t)5 * TW * pad_row(TL + 1);
  if (ns) n += (size_t)4 * TW * pad_row(TL + 2 * kVisHalo);
  if (DIR == 2) n += (size_t)5 * TW * pad_row(TL);
  return n * sizeof(double);
}

// The eta sweep accumulates into the right-hand side the xi sweep wrote.  The tile's RHS
// values are copied into shared memory ([5][TL][TW]) by cp.async when the kernel starts,
// so their latency hides behind the split and face phases: 7% off the eta sweep at 256^3.
// Euler only: the Navier-Stokes tiles have no shared memory to spare at 4 CTAs per SM.
// The zeta sweep measured 8% slower with it (its tile already holds the stage state, and
// the extra 10 KB leaves the SM's L1 a few KB).
#ifndef NUC3D_RHS_PREFETCH
#define NUC3D_RHS_PREFETCH 1
#endif
#ifndef NUC3D_HYB_PREFETCH
#define NUC3D_HYB_PREFETCH 0  // the same staging in the hybrid eta sweep (measured 2% slower)
#endif
#ifndef NUC3D_RHS_PREFETCH_NS
#define NUC3D_RHS_PREFETCH_NS 0  // the same staging in the Navier-Stokes eta sweep (measured
#endif                           // 2% slower on the 24-block grid: 3 CTAs per SM with 8x32)
template <int DIR>
__host__ __device__ constexpr bool rhs_prefetch(bool ns) {
  return NUC3D_RHS_PREFETCH && (DIR == 1 || (DIR == 2 && NUC3D_RHS_PREFETCH_Z)) &&
         (!ns || NUC3D_RHS_PREFETCH_NS);
}
template <int DIR>
__host__ __device__ constexpr size_t rhs_stage_bytes(bool ns) {
  return rhs_prefetch<DIR>(ns) ? (size_t)5 * 256 * sizeof(double) : 0;
}

// Shared memory of the hybrid sweep: its copy of the sensor weights, then one decision
// byte per face item of the tile (16-byte multiples).
constexpr size_t kSensorSmem = ((sizeof(SensorDev) + 15) / 16) * 16;
constexpr int kMaxFaceItems = 8 * (32 + 1);  // TW * (TL + 1), largest over the shapes
static_assert(kMaxFaceItems >= 4 * (64 + 1) && kMaxFaceItems >= 2 * (128 + 1), "face items");
constexpr size_t kHybSmem = kSensorSmem + ((size_t)kMaxFaceItems + 15) / 16 * 16;

__device__ __forceinline__ void cp_async8(double *dst_smem, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  const size_t g = __cvta_generic_to_global(src);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

__device__ __forceinline__ int find_block(const TileMap &tm, int t) {
  int lo = 0, hi = tm.nblocks - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (tm.tile_start[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Cell across face 2*d+side seen from line position g (g < 0 or g >= n[d]) of the
// line whose slab coordinates are (a, b).  The reference copies a raw slab of
// bfsize cells (bufferData::setBufferSend, src/bufferData.cpp:103-239) and indexes
// it g+bfsize on the left, g-n on the right (src/weno5js.cpp:257-262,475-480);
// slab coordinates are (j,k) for xi faces, (k,i) for eta, (i,j) for zeta.
// Returns the neighbour block (or -1 for a physical face) and its cell index.
__device__ __forceinline__ int ghost_cell(const BlockDev *__restrict__ blocks, const BlockDev &B,
                                          int d, int g, int a, int b, int bfs, long long &nidx) {
  const int L = B.n[d];
  const int side = g < 0 ? 0 : 1;
  const FaceDev &F = B.face[2 * d + side];
  if (F.type < 0) return -1;
  const int slot = side == 0 ? g + bfs : g - L;
  const int A = d == 0 ? B.n[1] : (d == 1 ? B.n[2] : B.n[0]);
  const long long rem = a + (long long)A * b;
  const BlockDev &NB = blocks[F.type];
  const int d2 = F.id >> 1, s2 = F.id & 1;
  const int A2 = d2 == 0 ? NB.n[1] : (d2 == 1 ? NB.n[2] : NB.n[0]);
  const int a2 = (int)(rem % A2), b2 = (int)(rem / A2);
  const int pos2 = s2 == 0 ? slot : NB.n[d2] - bfs + slot;
  int i, j, k;
  if (d2 == 0) { i = pos2; j = a2; k = b2; }
  else if (d2 == 1) { i = b2; j = pos2; k = a2; }
  else { i = a2; j = b2; k = pos2; }
  nidx = ((long long)k * NB.n[1] + j) * NB.n[0] + i;
  return F.type;
}

__device__ __forceinline__ void load_q(const double *__restrict__ Qs, long long N, long long idx,
                                       double q[5]) {
#pragma unroll
  for (int v = 0; v < 5; ++v) q[v] = __ldg(Qs + v * N + idx);
}

// Split flux of a cell of block B along direction d (own cell or a neighbour's ghost).
__device__ __forceinline__ void cell_split(const BlockDev &B, int stage, long long idx, int d,
                                           const SolverParams &P, double fp[5], double fn[5],
                                           CellPrim &s, double q[5], unsigned &st) {
  const long long N = B.N;
  load_q(B.q[stage], N, idx, q);
  const double jac = __ldg(B.jac + idx);
  con2prim(q, jac, P.gamma, P.mach, s, st);
  q[4] = s.q4;
  const double *m = B.met[d];
  split_cell(P.riemann, q, s, __ldg(m + idx), __ldg(m + N + idx), __ldg(m + 2 * N + idx), jac, fp, fn);
}

// Ghost split flux at a physical face (src/boundaryConditions.cpp:140-1086): the
// point solver evaluated at the edge cell's metric with the BC state.  Only the
// ghost next to the face enters the reconstruction (face 0 takes the last ghost
// slot for F+, face n the first slot for F-: src/reconstructionBoundaryScheme.cpp:88-106,289-308),
// and for the mirrored wall/symmetry ghosts that slot mirrors the edge cell itself
// (iblock = 0 or n-1, src/boundaryConditions.cpp:525-526).
__device__ __forceinline__ void bc_ghost_flux(const BlockDev &B, int stage, int d, int side,
                                              long long eidx, const SolverParams &P, double out[5],
                                              unsigned &st) {
  const FaceDev &F = B.face[2 * d + side];
  const long long N = B.N;
  const double jac = __ldg(B.jac + eidx);
  const double *m = B.met[d];
  const double xx = __ldg(m + eidx), xy = __ldg(m + N + eidx), xz = __ldg(m + 2 * N + eidx);
  double qb[5];
  if (F.id == BC_INLET) {
#pragma unroll
    for (int v = 0; v < 5; ++v) qb[v] = F.bcv[v];
  } else {
    double q[5];
    CellPrim s;
    load_q(B.q[stage], N, eidx, q);
    con2prim(q, jac, P.gamma, P.mach, s, st);
    qb[0] = s.rho; qb[1] = s.u; qb[2] = s.v; qb[3] = s.w; qb[4] = s.p;
    if (F.id == BC_WALL) {
      // src/boundaryConditions.cpp:564-567
      qb[0] = qb[4] * P.gamma * P.mach * P.mach / P.t_wall;
      qb[1] = 0.0; qb[2] = 0.0; qb[3] = 0.0;
    } else if (F.id == BC_SYMM) {
      // contravariant velocities and the mirror of the face-normal one
      // (src/boundaryConditions.cpp:882-888, 971-977, 1061-1067)
      const double *m0 = B.met[0], *m1 = B.met[1], *m2 = B.met[2];
      const double u = qb[1], v = qb[2], w = qb[3];
      double U = __ldg(m0 + eidx) * u + __ldg(m0 + N + eidx) * v + __ldg(m0 + 2 * N + eidx) * w;
      double V = __ldg(m1 + eidx) * u + __ldg(m1 + N + eidx) * v + __ldg(m1 + 2 * N + eidx) * w;
      double W = __ldg(m2 + eidx) * u + __ldg(m2 + N + eidx) * v + __ldg(m2 + 2 * N + eidx) * w;
      const double *X = B.dxyz;
      double t[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) t[c] = __ldg(X + c * N + eidx);
      // t = x_xi x_eta x_zeta y_xi y_eta y_zeta z_xi z_eta z_zeta
      if (d == 0) {
        qb[1] = -t[0] * U + t[1] * V + t[2] * W;
        qb[2] = -t[3] * U + t[4] * V + t[5] * W;
        qb[3] = -t[6] * U + t[7] * V + t[8] * W;
      } else if (d == 1) {
        qb[1] = t[0] * U - t[1] * V + t[2] * W;
        qb[2] = t[3] * U - t[4] * V + t[5] * W;
        qb[3] = t[6] * U - t[7] * V + t[8] * W;
      } else {
        qb[1] = t[0] * U + t[1] * V - t[2] * W;
        qb[2] = t[3] * U + t[4] * V - t[5] * W;
        qb[3] = t[6] * U + t[7] * V - t[8] * W;
      }
    }
  }
  split_point(P.riemann, qb, jac, xx, xy, xz, P.gamma, side, out, st);
}

// Interior reconstructions (no physical face within the scheme's reach): the uniform
// stencil of the line extended by ghost cells.  compat selects the weno5z stencil of
// src/weno5z.cpp:80 (interior positive faces only).
template <int SCH, class Acc>
__device__ __forceinline__ double recon_pos_in(int f, bool compat, Acc P) {
  if (SCH == SCH_WENO3JS) return rb_third(P(f - 2), P(f - 1), P(f));  // src/weno3js.cpp:59-86
  if (SCH == SCH_UPWIND1) return P(f - 1);                            // src/upwind1st.cpp:57-75
  if (SCH == SCH_WENO7JS || SCH == SCH_HCCS) {
    double s[7] = {P(f - 4), P(f - 3), P(f - 2), P(f - 1), P(f), P(f + 1), P(f + 2)};
    return SCH == SCH_HCCS ? weno7z(s) : weno7js(s);
  } else if (SCH == SCH_WENO5Z) {
    return weno5z(P(f - 3), P(f - 2), P(f - 1), P(f), P(f + 1), compat);
  } else {
    return weno5js(P(f - 3), P(f - 2), P(f - 1), P(f), P(f + 1));
  }
}

template <int SCH, class Acc>
__device__ __forceinline__ double recon_neg_in(int f, Acc Nf) {
  if (SCH == SCH_WENO3JS) return rb_third(Nf(f + 1), Nf(f), Nf(f - 1));  // src/weno3js.cpp:88-115
  if (SCH == SCH_UPWIND1) return Nf(f);                                  // src/upwind1st.cpp:96-114
  if (SCH == SCH_WENO7JS || SCH == SCH_HCCS) {
    double s[7] = {Nf(f + 3), Nf(f + 2), Nf(f + 1), Nf(f), Nf(f - 1), Nf(f - 2), Nf(f - 3)};
    return SCH == SCH_HCCS ? weno7z(s) : weno7js(s);
  } else if (SCH == SCH_WENO5Z) {
    return weno5z(Nf(f + 2), Nf(f + 1), Nf(f), Nf(f - 1), Nf(f - 2), false);
  } else {
    return weno5js(Nf(f + 2), Nf(f + 1), Nf(f), Nf(f - 1), Nf(f - 2));
  }
}

// Reconstructed F+ at face f from the split fluxes P(c) of cells c (line coordinates).
// Faces next to a physical face use ReconstructionboundaryScheme
// (src/reconstructionBoundaryScheme.cpp:52-313); the right side is tested first
// because the reference applies BR after BL.
template <int SCH, class Acc>
__device__ __forceinline__ double recon_pos(int f, int L, int ts, bool physL, bool physR,
                                            bool compat, Acc P) {
  if (physR && f > L - ts) {
    switch (L - f) {
      case 0: return P(L - 1);
      case 1: return rb_second(P(L - 2), P(L - 1));
      case 2: return rb_third(P(L - 4), P(L - 3), P(L - 2));
      default: return weno5js(P(L - 6), P(L - 5), P(L - 4), P(L - 3), P(L - 2));
    }
  }
  if (physL && f < ts) {
    switch (f) {
      case 0: return P(-1);
      case 1: return rb_second(P(0), P(1));
      case 2: return rb_third(P(0), P(1), P(2));
      default: return weno5js(P(0), P(1), P(2), P(3), P(4));
    }
  }
  return recon_pos_in<SCH>(f, compat && f >= ts && f <= L - ts, P);
}

template <int SCH, class Acc>
__device__ __forceinline__ double recon_neg(int f, int L, int ts, bool physL, bool physR, Acc Nf) {
  if (physR && f > L - ts) {
    switch (L - f) {
      case 0: return Nf(L);
      case 1: return rb_second(Nf(L - 1), Nf(L - 2));
      case 2: return rb_third(Nf(L - 1), Nf(L - 2), Nf(L - 3));
      default: return weno5js(Nf(L - 1), Nf(L - 2), Nf(L - 3), Nf(L - 4), Nf(L - 5));
    }
  }
  if (physL && f < ts) {
    switch (f) {
      case 0: return Nf(0);
      case 1: return rb_second(Nf(1), Nf(0));
      case 2: return rb_third(Nf(3), Nf(2), Nf(1));
      default: return weno5js(Nf(5), Nf(4), Nf(3), Nf(2), Nf(1));
    }
  }
  return recon_neg_in<SCH>(f, Nf);
}

// F+ + F- of a face within ts of a physical face (recon_pos + recon_neg of such a face),
// without branching on the face: the boundary stencils sit at fixed offsets from the
// line end, so every candidate of the reference's switch is evaluated with its own
// expression on values loaded at those offsets and the one for distance k = face to
// physical face is selected.  Lanes of one warp holding different k then run one path.
// The right end is tested first, as the reference applies BR after BL.  Positions are
// clamped to the tile's shared-memory row [first, last] (a one-cell tile at the right end
// holds fewer cells than the stencils reach; values read there belong only to candidates
// that k does not select), so every load stays inside the row whichever end it serves.
template <int SCH, class AccP, class AccN>
__device__ __forceinline__ double edge_face(int f, int L, int ts, bool physR, int first, int last,
                                            AccP P, AccN Nf) {
  constexpr int NJ = (SCH == SCH_WENO7JS || SCH == SCH_HCCS) ? 6 : 4;
  const bool right = physR && f > L - ts;
  const int k = right ? L - f : f;
  auto at = [first, last](int c) { return min(max(c, first), last); };
  // a[j]: F+ at cells L-1-j (right) or j-1 (left); b[j]: F- at cells L-j (right) or j (left)
  double a[NJ], b[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    a[j] = P(at(right ? L - 1 - j : j - 1));
    b[j] = Nf(at(right ? L - j : j));
  }
  // recon_pos cases: P(L-1) | rb_second(P(L-2),P(L-1)) | rb_third(P(L-4),P(L-3),P(L-2)) |
  // weno5js(P(L-6..L-2)) on the right; P(-1) | rb_second(P(0),P(1)) | rb_third(P(0),P(1),P(2)) |
  // weno5js(P(0..4)) on the left
  const double hp1 = right ? rb_second(a[1], a[0]) : rb_second(a[1], a[2]);
  const double hp2 = right ? rb_third(a[3], a[2], a[1]) : rb_third(a[1], a[2], a[3]);
  // recon_neg cases: Nf(L) | rb_second(Nf(L-1),Nf(L-2)) | rb_third(Nf(L-1),Nf(L-2),Nf(L-3)) |
  // weno5js(Nf(L-1..L-5)) on the right; Nf(0) | rb_second(Nf(1),Nf(0)) |
  // rb_third(Nf(3),Nf(2),Nf(1)) | weno5js(Nf(5..1)) on the left
  const double hn1 = rb_second(b[1], right ? b[2] : b[0]);
  const double hn2 = right ? rb_third(b[1], b[2], b[3]) : rb_third(b[3], b[2], b[1]);
  double hp = k == 0 ? a[0] : (k == 1 ? hp1 : hp2);
  double hn = k == 0 ? b[0] : (k == 1 ? hn1 : hn2);
  if (NJ == 6 && k == 3) {
    const int i1 = 1, i5 = NJ - 1;
    hp = right ? weno5js(a[i5], a[4], a[3], a[2], a[i1]) : weno5js(a[i1], a[2], a[3], a[4], a[i5]);
    hn = right ? weno5js(b[i1], b[2], b[3], b[4], b[i5]) : weno5js(b[i5], b[4], b[3], b[2], b[i1]);
  }
  return hp + hn;
}

// d/dxi of a cell-centred field at line position c: boundaryScheme within ts cells
// of a physical face (src/fieldOperator.cpp:523-624, src/boundaryScheme.cpp:311-406),
// the direction's scheme_vis operator (cd6, cd2 or cd8) elsewhere (ghost values come from
// the neighbour across the face).
template <class Acc>
__device__ __forceinline__ double diff_at(int c, int L, int ts, bool physL, bool physR, int vis,
                                          Acc V) {
  if (physR && c >= L - ts) {
    switch (L - 1 - c) {
      case 0: return V(c) - V(c - 1);
      case 1: return bnd_second(V(c - 1), V(c + 1));
      case 2: return bnd_fourth(V(c - 2), V(c - 1), V(c + 1), V(c + 2));
      default: return bnd_sixth(V(c - 3), V(c - 2), V(c - 1), V(c + 1), V(c + 2), V(c + 3));
    }
  }
  if (physL && c < ts) {
    switch (c) {
      case 0: return V(c + 1) - V(c);
      case 1: return bnd_second(V(c - 1), V(c + 1));
      case 2: return bnd_fourth(V(c - 2), V(c - 1), V(c + 1), V(c + 2));
      default: return bnd_sixth(V(c - 3), V(c - 2), V(c - 1), V(c + 1), V(c + 2), V(c + 3));
    }
  }
  if (vis == VIS_CD2) return cd2(V(c - 1), V(c + 1));
  if (vis == VIS_CD8)
    return cd8(V(c - 4), V(c - 3), V(c - 2), V(c - 1), V(c + 1), V(c + 2), V(c + 3), V(c + 4));
  return cd6(V(c - 3), V(c - 2), V(c - 1), V(c + 1), V(c + 2), V(c + 3));
}

enum SweepFlags : int { SW_EIG = 1, SW_RK = 2, SW_NS = 4, SW_STORE_DVIS = 8, SW_RES = 16 };

// The residual's share of one value of the last RK stage (PDEData3d::setRES,
// src/PDEData3d.cpp:90-122): the reference-order build keeps d = u - u_n per value for the
// residual kernel's sum in the reference's order; the throughput build adds d^2 to the
// thread's sum, which the CTA reduces per tile.
__device__ __forceinline__ void res_value(const BlockDev &B, int v, long long idx, double x,
                                          double un, double &acc) {
  const double d = x - un;
#if NUC3D_FAST
  (void)B; (void)v; (void)idx;
  acc = fma(d, d, acc);
#else
  (void)acc;
  B.dres[v * B.N + idx] = d;
#endif
}

// Sum of acc over the CTA's first nthreads threads (warp shuffles, then the warp sums in
// order): thread 0 writes it to *out.  Every one of those threads calls it; sync is their
// barrier.
template <class Sync>
__device__ __forceinline__ void cta_sum_to(double acc, double *sRed, int nthreads, double *out,
                                           Sync sync) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sRed[threadIdx.x >> 5] = acc;
  sync();
  if (threadIdx.x == 0) {
    double t = sRed[0];
    for (int i = 1; i < nthreads / 32; ++i) t += sRed[i];
    *out = t;
  }
  sync();
}

// TVD-RK3 stage update of one value (src/TVD-RK3.cpp:57-136, coefficients src/TVD-RK3.h:9-12):
// u_i is the stage state, u_n the state saved at stage 0, R the right-hand side.
__device__ __forceinline__ double rk3_update(int stage, double R, double u_i, double u_n, double dt) {
  double rhs = -R;
  if (stage == 0) return 1.0 * u_i + 1.0 * rhs * dt;
  if (stage == 1) return 3.0 / 4.0 * u_n + 1.0 / 4.0 * (rhs * dt + u_i);
  return 1.0 / 3.0 * u_n + 2.0 / 3.0 * (rhs * dt + u_i);
}

// Geometry of one sweep tile (a CTA's share of one block's lines).
struct TileCtx {
  int t, b;
  const BlockDev *B;
  Geo G;
  int n[3];
  int c0, cl, w0, nw, o;  // first cell and cell count along the lines, first lane, lanes, outer index
  long long N;
  int ts;
  bool physL, physR;
};

template <int DIR, int SHP = 0>
__device__ __forceinline__ TileCtx decode_tile(const BlockDev *__restrict__ blocks, const TileMap &tm,
                                               const SolverParams &P, int t) {
  constexpr int TW = Tile<SHP>::TW, TL = Tile<SHP>::TL;
  TileCtx T;
  T.t = t;
  T.b = find_block(tm, T.t);
  T.B = &blocks[T.b];
  for (int d = 0; d < 3; ++d) T.n[d] = T.B->n[d];
  T.G = make_geo(DIR, T.n);
  // xi, eta: tile = (chunk along the line) + nch * ((line group) + nwg * (outer index)).
  // zeta: tile = (line group) + nwg * ((outer index) + nO * (chunk)): the CTAs resident at
  // one time then share one chunk of z-planes (3% faster at 256^3 than chunk-fastest,
  // whose CTAs spread over every plane at 512 KB strides).
  const unsigned lt = (unsigned)(T.t - tm.tile_start[T.b]);
  const unsigned nch = (unsigned)(T.G.L + TL - 1) / TL;
  const unsigned nwg = (unsigned)(T.G.nW + TW - 1) / TW;
  const unsigned q1 = (unsigned)((lt * T.B->tdiv[DIR][0]) >> 40);
  const unsigned q2 = (unsigned)((q1 * T.B->tdiv[DIR][1]) >> 40);
  int ch, wg;
  if (DIR == 2) {
    wg = (int)(lt - q1 * nwg);
    T.o = (int)(q1 - q2 * (unsigned)T.G.nO);
    ch = (int)q2;
  } else {
    ch = (int)(lt - q1 * nch);
    wg = (int)(q1 - q2 * nwg);
    T.o = (int)q2;
  }
  T.c0 = ch * TL;
  T.cl = min(TL, T.G.L - T.c0);
  T.w0 = wg * TW;
  T.nw = min(TW, T.G.nW - T.w0);
  T.N = T.B->N;
  T.ts = P.ts[DIR];
  T.physL = T.B->face[2 * DIR].type < 0;
  T.physR = T.B->face[2 * DIR + 1].type < 0;
  return T;
}
// The tile of this CTA (one tile per CTA, counted from the map's base).
template <int DIR, int SHP = 0>
__device__ __forceinline__ TileCtx decode_tile(const BlockDev *__restrict__ blocks, const TileMap &tm,
                                               const SolverParams &P) {
  return decode_tile<DIR, SHP>(blocks, tm, P, tm.base + (int)blockIdx.x);
}
// Tiles a launch over the map covers.
__host__ __device__ inline int tile_range(const TileMap &tm) {
  return (tm.end > 0 ? tm.end : tm.tile_start[tm.nblocks]) - tm.base;
}

// Shared-memory row strides of a sweep tile.
template <int DIR, int SCH, int SHP = 0> struct TileSmem {
  static constexpr int R = Halo<SCH>::R, TW = Tile<SHP>::TW, TL = Tile<SHP>::TL;
  static constexpr int NP = TL + 2 * R, SP = pad_row(NP);
  static constexpr int NV = TL + 2 * kVisHalo, SV = pad_row(NV);
  static constexpr int SH = pad_row(TL + 1), SQ = pad_row(TL);
};

// Phase 1: split fluxes F+/F- of the tile's line positions c0-R .. c0+cl+R-1 into sF
// ([10][TW][SP]); own cells of the zeta tile also leave their state in sQ; eig reduces
// max(|U|+c|grad xi|) over the three directions; nres (xi sweeps) counts the own cells
// whose energy con2prim reset.
template <int DIR, int SCH, bool RHOP = false, int SHP = 0>
__device__ __forceinline__ void phase_split(const BlockDev *__restrict__ blocks, const TileCtx &T,
                                            const SolverParams &P, int stage, bool eig, double *sF,
                                            double *sQ, unsigned &st, double &emax,
                                            double *sRP = nullptr, unsigned *nres = nullptr) {
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int R = M::R, TW = M::TW, NP = M::NP, SP = M::SP, SQ = M::SQ;
  const BlockDev &B = *T.B;
  const Geo &G = T.G;
  for (int e = threadIdx.x; e < TW * NP; e += kThreads) {
    int p, w;
    if (DIR == 0) { p = e % NP; w = e / NP; } else { w = e % TW; p = e / TW; }
    double fp[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, fn[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int g = T.c0 + p - R;
    if (w < T.nw && p < T.cl + 2 * R) {
      const int wl = T.w0 + w;
      const int sa = (DIR == 1) ? T.o : wl, sb = (DIR == 1) ? wl : T.o;
      // the cell at line position g: this block's, or the neighbour's across the face;
      // one split call serves both, so a neighbour halo adds no divergent copy of it
      const bool own = g >= 0 && g < G.L;
      const BlockDev *CB = &B;
      long long idx = g * G.sL + wl * G.sW + T.o * G.sO;
      if (!own) {
        const int nb = ghost_cell(blocks, B, DIR, g, sa, sb, P.bfs, idx);
        CB = nb >= 0 ? &blocks[nb] : nullptr;
      }
      if (CB) {
        double q[5];
        CellPrim s;
        cell_split(*CB, stage, idx, DIR, P, fp, fn, s, q, st);
        if (RHOP) {  // density and pressure of the position, for the face sensor
          sRP[w * SP + p] = s.rho;
          sRP[(TW + w) * SP + p] = s.p;
        }
        if (DIR == 0 && nres && own && s.reset && g >= T.c0 && g < T.c0 + T.cl) ++*nres;
        if (own && eig && g >= T.c0 && g < T.c0 + T.cl) {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double *m = B.met[d];
            double ev = eigen_cell(s, __ldg(m + idx), __ldg(m + T.N + idx), __ldg(m + 2 * T.N + idx));
            emax = ev > emax ? ev : emax;
          }
        }
        if (DIR == 2 && sQ && own && g >= T.c0 && g < T.c0 + T.cl) {
#pragma unroll
          for (int v = 0; v < 5; ++v) sQ[(v * TW + w) * SQ + (g - T.c0)] = q[v];
        }
      } else {
        if (g == -1 || g == G.L) {
          // ghost next to a physical face, filled by bc_ghost_kernel this stage
          const int f = 2 * DIR + (g < 0 ? 0 : 1);
          const int A = DIR == 0 ? T.n[1] : (DIR == 1 ? T.n[2] : T.n[0]);
          const long long area = (long long)A * (DIR == 0 ? T.n[2] : (DIR == 1 ? T.n[0] : T.n[1]));
          const double *gh = B.ghost + B.goff[f] + (sa + (long long)A * sb);
          if (g < 0) {
#pragma unroll
            for (int v = 0; v < 5; ++v) fp[v] = __ldg(gh + v * area);
          } else {
#pragma unroll
            for (int v = 0; v < 5; ++v) fn[v] = __ldg(gh + v * area);
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      sF[(v * TW + w) * SP + p] = fp[v];
      sF[((5 + v) * TW + w) * SP + p] = fn[v];
    }
  }
}

// Viscous fluxes of the tile's line positions c0-4 .. c0+cl+3 into sV ([4][TW][SV]).
template <int DIR, int SCH, int SHP = 0>
__device__ __forceinline__ void phase_vis(const BlockDev *__restrict__ blocks, const TileCtx &T,
                                          const SolverParams &P, double *sV) {
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int TW = M::TW, NV = M::NV, SV = M::SV;
  const BlockDev &B = *T.B;
  const Geo &G = T.G;
  for (int e = threadIdx.x; e < TW * NV; e += kThreads) {
    int p, w;
    if (DIR == 0) { p = e % NV; w = e / NV; } else { w = e % TW; p = e / TW; }
    double fv[4] = {0.0, 0.0, 0.0, 0.0};
    const int g = T.c0 + p - kVisHalo;
    // ghosts exist up to bfsize cells out; the viscous stencil of a direction never
    // reaches further (nuc3d_create checks reach <= tilesize <= bfsize)
    if (w < T.nw && p < T.cl + 2 * kVisHalo && g >= -P.bfs && g < G.L + P.bfs) {
      const int wl = T.w0 + w;
      const int sa = (DIR == 1) ? T.o : wl, sb = (DIR == 1) ? wl : T.o;
      const double *vis = nullptr;
      long long idx = -1, NN = T.N;
      if (g >= 0 && g < G.L) {
        idx = g * G.sL + wl * G.sW + T.o * G.sO;
        vis = B.vis;
      } else {
        long long nidx;
        const int nb = ghost_cell(blocks, B, DIR, g, sa, sb, P.bfs, nidx);
        if (nb >= 0) {
          idx = nidx;
          vis = blocks[nb].vis;
          NN = blocks[nb].N;
        }
      }
      if (vis) {
#pragma unroll
        for (int v = 0; v < 4; ++v) fv[v] = __ldg(vis + (DIR * 4 + v) * NN + idx);
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) sV[(v * TW + w) * SV + p] = fv[v];
  }
}

// Phase 3: per cell, dF from the face fluxes in sH, RHS accumulation (src/euler3d.cpp:368-427,
// src/NaiverStokes3d.cpp:401-513), and on the zeta sweep the TVD-RK3 stage.
// sR: the tile's RHS staged at the start of the sweep ([5][TL][TW]), or null.
template <int DIR, int SCH, int SHP = 0>
__device__ __forceinline__ void phase_cells(const TileCtx &T, const SolverParams &P, StepState *S,
                                            int stage, int flags, const double *sH, const double *sV,
                                            const double *sQ, unsigned &st, double *sRed,
                                            const double *sR = nullptr) {
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int TW = M::TW, TL = M::TL, SV = M::SV, SH = M::SH, SQ = M::SQ;
  const BlockDev &B = *T.B;
  const Geo &G = T.G;
  const long long N = T.N;
  const bool ns = (flags & SW_NS) != 0;
  double *__restrict__ rhs = B.rhs;
  double dt = 0.0;
  if (flags & SW_RK) {
    if (stage == 0) {
      double me = __longlong_as_double((long long)S->max_eig_bits);
      double dt_local = 1.0 / me;
      dt = dt_local * P.cfl;
      if (T.t == 0 && threadIdx.x == 0) S->dt = dt;
    } else {
      dt = S->dt;
    }
    if (stage == 2 && T.t == 0 && threadIdx.x == 0) S->time = S->time + dt;
  }
  double racc = 0.0;  // the residual's sum of (u - u_n)^2 (SW_RES)
  for (int e = threadIdx.x; e < TW * TL; e += kThreads) {
    int c, w;
    if (DIR == 0) { c = e % TL; w = e / TL; } else { w = e % TW; c = e / TW; }
    if (w >= T.nw || c >= T.cl) continue;
    const int g = T.c0 + c;
    const long long idx = g * G.sL + (T.w0 + w) * G.sW + T.o * G.sO;
    double d[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double *h = sH + (v * TW + w) * SH;
      d[v] = h[c + 1] - h[c];
    }
    double dv[4] = {0.0, 0.0, 0.0, 0.0};
    if (ns) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double *row = sV + (v * TW + w) * SV + (kVisHalo - T.c0);
        auto Vacc = [row](int cc) { return row[cc]; };
        dv[v] = diff_at(g, G.L, T.ts, T.physL, T.physR, P.vis[DIR], Vacc);
      }
    }
    if (DIR == 0) {
#pragma unroll
      for (int v = 0; v < 5; ++v) rhs[v * N + idx] = d[v];
      if (ns) {
#pragma unroll
        for (int v = 0; v < 4; ++v) B.dvis[v * N + idx] = dv[v];
      }
    } else if (DIR == 1) {
#pragma unroll
      for (int v = 0; v < 5; ++v)
        rhs[v * N + idx] = (sR ? sR[(v * TL + c) * TW + w] : rhs[v * N + idx]) + d[v];
      if (ns) {
#pragma unroll
        for (int v = 0; v < 4; ++v) B.dvis[(4 + v) * N + idx] = dv[v];
      }
    } else {
      double r[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) r[v] = (sR ? sR[(v * TL + c) * TW + w] : rhs[v * N + idx]) + d[v];
      if (ns) {
#pragma unroll
        for (int v = 1; v < 5; ++v) {
          r[v] = r[v] - B.dvis[(v - 1) * N + idx];
          r[v] = r[v] - B.dvis[(4 + v - 1) * N + idx];
          r[v] = r[v] - dv[v - 1];
        }
      }
      if (flags & SW_RK) {
        double *__restrict__ qo = B.q[(stage + 1) % 3];
        const double *__restrict__ qn = B.q[0];
        // u_n: the state stage 0 started from, with con2prim's energy reset applied, as
        // the reference's Q_Euler = Q_work copy takes it after stage 0's right-hand side
        // wrote the reset into Q_work (src/physicsModel.cpp:324-332, src/PDEData3d.cpp:74-76)
        double un[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (stage != 0) {
#pragma unroll
          for (int v = 0; v < 5; ++v) un[v] = qn[v * N + idx];
          CellPrim sn;
          unsigned stn = 0;
          con2prim(un, __ldg(B.jac + idx), P.gamma, P.mach, sn, stn);
          un[4] = sn.q4;
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const double ui = sQ[(v * TW + w) * SQ + c];
          const double x = rk3_update(stage, r[v], ui, un[v], dt);
          if (!isfinite(x)) st |= ST_NONFINITE;
          qo[v * N + idx] = x;
          if (flags & SW_RES) res_value(B, v, idx, x, un[v], racc);
        }
      } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) rhs[v * N + idx] = r[v];
      }
    }
  }
#if NUC3D_FAST
  if (flags & SW_RES) cta_sum_to(racc, sRed, kThreads, P.res_part + T.t, [] { __syncthreads(); });
#else
  (void)sRed;
#endif
}

__device__ __forceinline__ void reduce_eig(double emax, double *sRed, StepState *S) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double x = __shfl_xor_sync(0xffffffffu, emax, off);
    emax = x > emax ? x : emax;
  }
  if ((threadIdx.x & 31) == 0) sRed[threadIdx.x >> 5] = emax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sRed[0];
    for (int i = 1; i < kThreads / 32; ++i) m = sRed[i] > m ? sRed[i] : m;
    atomicMax(&S->max_eig_bits, (unsigned long long)__double_as_longlong(m));
  }
}

#include "sensor.cuh"
#include "sweep_pipe.cuh"

// hccs's smoothness switch theta = 1 / (1 + (sum alpha - 1)^2), alpha_k the CRWENO5-Z
// weights' numerators with eps 1e-40 (src/hccs.cpp:154-181), of one 5-point stencil.
__device__ __forceinline__ double theta_stencil(double f0, double f1, double f2, double f3, double f4) {
  const W5 r = w5_parts(f0, f1, f2, f3, f4, false);
  const double ss = 1.0e-40, tau = fabs(r.is2 - r.is0);
  const double s = kCR5[0] * (1.0 + sq(tau / (r.is0 + ss))) + kCR5[1] * (1.0 + sq(tau / (r.is1 + ss))) +
                   kCR5[2] * (1.0 + sq(tau / (r.is2 + ss)));
  return 1.0 / (1.0 + sq(s - 1.0));
}
// The theta switch as a face decision of the hybrid sweep: the smallest theta of the
// face's density and pressure over its positive (f-3 .. f+1) and negative (f+2 .. f-2)
// stencils; rho, p point at the face's position (the cell after it).
__device__ __forceinline__ double theta_face(const double *rho, const double *p) {
  const double a = theta_stencil(rho[-3], rho[-2], rho[-1], rho[0], rho[1]);
  const double b = theta_stencil(rho[2], rho[1], rho[0], rho[-1], rho[-2]);
  const double c = theta_stencil(p[-3], p[-2], p[-1], p[0], p[1]);
  const double d = theta_stencil(p[2], p[1], p[0], p[-1], p[-2]);
  return fmin(fmin(a, b), fmin(c, d));
}

// Explicit-scheme sweep: phases split -> faces -> cells in one CTA.  HYB: the hybrid
// WENO-Z face loop of the throughput build (P.sensor set).
template <int DIR, int SCH, bool HYB = false, int SHP = 0>
__global__ void __launch_bounds__(kThreads, DIR == 2 ? NUC3D_SWEEP_MINB_Z : NUC3D_SWEEP_MINB)
sweep_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
             int stage, int flags) {
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int R = M::R, TW = M::TW, SP = M::SP, SV = M::SV, SH = M::SH;
  extern __shared__ double smem[];
  double *sF = smem;                        // [10][TW][SP]: F+ vars 0..4, F- vars 5..9
  double *sH = sF + 10 * TW * SP;           // [5][TW][SH]: face fluxes
  const bool ns = (flags & SW_NS) != 0;
  double *sV = sH + 5 * TW * SH;            // [4][TW][SV]: viscous fluxes (NS)
  double *sQ = sV + (ns ? 4 * TW * SV : 0); // [5][TW][SQ]: stage state (zeta sweep)
  double *sRP = sQ + (DIR == 2 ? 5 * TW * M::SQ : 0);  // hybrid: [2][TW][SP] rho, p
  // hybrid: the sensor's weights; plain: the staged RHS
  SensorDev *sS = reinterpret_cast<SensorDev *>(sRP + (HYB ? 2 * TW * SP : 0));
  unsigned char *sLin = reinterpret_cast<unsigned char *>(sS) + kSensorSmem;  // hybrid: [TW*(TL+1)]
  double *sRst = reinterpret_cast<double *>(reinterpret_cast<char *>(sS) + (HYB ? kHybSmem : 0));
  __shared__ double sRed[kThreads / 32];

  const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P);
  const bool eig = (flags & SW_EIG) != 0;
  unsigned st = 0;
  double emax = 0.0;
  // (the hybrid sweep measured slower with the staged RHS: its tile is larger already)
  double *sR = ((!HYB || NUC3D_HYB_PREFETCH) && rhs_prefetch<DIR>(ns)) ? sRst : nullptr;
  if constexpr (HYB) {
    // the network's weights, read by every warp's inference: shared memory
    static_assert(sizeof(SensorDev) % 4 == 0, "word copy");
    const uint32_t *src = reinterpret_cast<const uint32_t *>(P.sensor);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sS);
    for (int i = threadIdx.x; i < (int)(sizeof(SensorDev) / 4); i += kThreads) dst[i] = src[i];
  }
  if (sR) {
    // each thread stages the RHS of the cells it finishes in phase_cells (same mapping),
    // so its own wait_all orders them; no barrier needed
    constexpr int TL = M::TL;
    for (int e = threadIdx.x; e < TW * TL; e += kThreads) {
      const int w = e % TW, c = e / TW;
      if (w >= T.nw || c >= T.cl) continue;
      const long long idx = (T.c0 + c) * T.G.sL + (T.w0 + w) * T.G.sW + T.o * T.G.sO;
#pragma unroll
      for (int v = 0; v < 5; ++v) cp_async8(sR + (v * TL + c) * TW + w, T.B->rhs + v * T.N + idx);
    }
  }
  unsigned nres = 0;
  phase_split<DIR, SCH, HYB, SHP>(blocks, T, P, stage, eig, sF, DIR == 2 ? sQ : nullptr, st, emax, sRP,
                                  DIR == 0 ? &nres : nullptr);
  if (ns) phase_vis<DIR, SCH, SHP>(blocks, T, P, sV);
  __syncthreads();

  // ---- faces c0 .. c0+cl: the ten reconstructions of each face ----
  // Faces within ts of a physical face take the boundary schemes: at most ts faces per
  // line end.  Items are ordered interior faces of all lines first, then, from the next
  // warp boundary on, the edge faces, so that one warp at most diverges into them.
  const bool compat = P.weno5z_compat != 0;
  const int nf = T.cl + 1;
  const int lo = T.physL ? min(max(T.ts - T.c0, 0), nf) : 0;                // edge: fl < lo
  const int hi = T.physR ? min(max(T.G.L - T.ts + 1 - T.c0, 0), nf) : nf;   // edge: fl >= hi
  const int ni = hi > lo ? hi - lo : 0;       // interior faces per line
  const int nl = ni > 0 ? lo : nf;            // left edge faces (all faces when ni == 0)
  const int ne = nf - ni;                     // edge faces per line
  const int ei = TW * ni, e0 = (ei + 31) & ~31;
  const float rni = ni > 0 ? 1.0f / (float)ni : 0.0f, rne = ne > 0 ? 1.0f / (float)ne : 0.0f;
  bool hyb_any = true, hyb_lin0 = false;  // hybrid: some gap of the tile nonzero; decision at zero
  if constexpr (HYB) {
    // hybrid WENO-Z, pass 1: the face sensor's decision for every interior face item
    // (linear weights or WENO-Z), into sLin.  Rounds are the same in every thread: the
    // inference is warp-collective.  Pass 2 is the face loop below; keeping the network
    // out of it keeps its registers out of the reconstructions'.
    // 1a: per-gap values (F+ differences, jumps) into sG, in sH's place (sH is written
    // only in pass 2)
    float *sG = reinterpret_cast<float *>(sH);
    unsigned char *sZ = reinterpret_cast<unsigned char *>(sG + kSensorGapVals * TW * SP);
    constexpr int NG = M::NP - 1;
    static_assert(kSensorGapVals * TW * SP * sizeof(float) + TW * SP <= 5 * TW * SH * sizeof(double),
                  "gap values and zero flags fit in the face-flux tile");
    int nonzero = 0;
    for (int e = threadIdx.x; e < TW * NG; e += kThreads) {
      const int w = e / NG, p = e - w * NG;
      if (w >= T.nw) continue;
      const double *rowF[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) rowF[v] = sF + (v * TW + w) * SP;
      const bool zero =
          sensor_gap(rowF, sRP + w * SP, sRP + (TW + w) * SP, p, sG + w * SP + p, TW * SP);
      sZ[w * SP + p] = zero ? 1 : 0;
      nonzero |= zero ? 0 : 1;
    }
    // A tile whose every gap is zero (inside a uniform region) has all-zero features on
    // every face: each face's decision is the network's zero-input one (the theta switch's:
    // theta = 1 on a uniform stencil), and 1b is skipped.
    hyb_any = __syncthreads_or(nonzero) != 0;
    hyb_lin0 = P.sensor_theta ? 1.0f >= P.sensor_threshold : sS->zero_logit < P.sensor_threshold;
    // 1b: features, network, decision; or hccs's theta switch on density and pressure
    if (hyb_any && P.sensor_theta) {
      for (int e = threadIdx.x; e < ei; e += kThreads) {
        const int w = __float2int_rz(((float)e + 0.5f) * rni), fl = lo + (e - w * ni);
        if (w < T.nw)
          sLin[e] = theta_face(sRP + w * SP + (R + fl), sRP + (TW + w) * SP + (R + fl)) >=
                            (double)P.sensor_threshold ? 1 : 0;
      }
    } else if (hyb_any)
    for (int base = 0; base < ei; base += kThreads) {
      const int e = base + threadIdx.x;
      int w = 0, fl = 0;
      if (e < ei) {
        w = __float2int_rz(((float)e + 0.5f) * rni);
        fl = lo + (e - w * ni);
      }
      const bool valid = e < ei && w < T.nw;
      uint32_t xr[10];
#pragma unroll
      for (int i = 0; i < 10; ++i) xr[i] = 0u;
      if (valid) {
        // a face whose five stencil gaps are all zero has all-zero features: skip them
        const unsigned char *z = sZ + w * SP + (R + fl - 3);
        if (!(z[0] & z[1] & z[2] & z[3] & z[4]))
          sensor_features_gaps(sG + w * SP + (R + fl - 3), TW * SP, xr);
      }
      const float logit = sensor_logit(sS, xr);
      if (valid) sLin[e] = logit < P.sensor_threshold ? 1 : 0;
    }
    if (hyb_any) __syncthreads();
  }
  for (int e = threadIdx.x; e < e0 + TW * ne; e += kThreads) {
    // w = e / ni by a float reciprocal: exact, since (e + 1/2) / ni stays at least
    // 1/(2 ni) away from an integer and e < 2^9.
    int w, fl;
    bool edge;
    if (e < ei) {
      w = __float2int_rz(((float)e + 0.5f) * rni);
      fl = lo + (e - w * ni);
      edge = false;
    } else if (e >= e0) {
      const int j = e - e0;
      w = __float2int_rz(((float)j + 0.5f) * rne);
      const int k = j - w * ne;
      fl = k < nl ? k : hi + (k - nl);
      edge = true;
    } else {
      continue;
    }
    if (w >= T.nw) continue;
    const int f = T.c0 + fl;
    if (HYB && !edge && (hyb_any ? sLin[e] != 0 : hyb_lin0)) {
      // hybrid: a face the sensor calls smooth takes the linear weights (0.1, 0.6, 0.3)
#pragma unroll 1
      for (int v = 0; v < 5; ++v) {
        const double *rowP = sF + (v * TW + w) * SP + (R + fl);
        const double *rowN = sF + ((5 + v) * TW + w) * SP + (R + fl);
        sH[(v * TW + w) * SH + fl] = weno5_linear(rowP[-3], rowP[-2], rowP[-1], rowP[0], rowP[1]) +
                                     weno5_linear(rowN[2], rowN[1], rowN[0], rowN[-1], rowN[-2]);
      }
    } else if (!edge) {
      const bool cz = compat && f >= T.ts && f <= T.G.L - T.ts;
#pragma unroll 2  // two variables per iteration: measured 3% faster than none, and than five
      for (int v = 0; v < 5; ++v) {
        const double *rowP = sF + (v * TW + w) * SP + (R + fl);
        const double *rowN = sF + ((5 + v) * TW + w) * SP + (R + fl);
        auto Pacc = [rowP](int c) { return rowP[c]; };
        auto Nacc = [rowN](int c) { return rowN[c]; };
        sH[(v * TW + w) * SH + fl] = recon_pos_in<SCH>(0, cz, Pacc) + recon_neg_in<SCH>(0, Nacc);
      }
    } else {
#pragma unroll 1
      for (int v = 0; v < 5; ++v) {
        const double *rowP = sF + (v * TW + w) * SP + (R - T.c0);
        const double *rowN = sF + ((5 + v) * TW + w) * SP + (R - T.c0);
        auto Pacc = [rowP](int c) { return rowP[c]; };
        auto Nacc = [rowN](int c) { return rowN[c]; };
#if NUC3D_FAST
        sH[(v * TW + w) * SH + fl] =
            edge_face<SCH>(f, T.G.L, T.ts, T.physR, T.c0 - R, T.c0 - R + M::NP - 1, Pacc, Nacc);
#else
        // reference-order build: the reference's switch (IEEE divisions make evaluating
        // every candidate dearer than the divergence)
        const double hp = recon_pos<SCH>(f, T.G.L, T.ts, T.physL, T.physR, compat, Pacc);
        const double hn = recon_neg<SCH>(f, T.G.L, T.ts, T.physL, T.physR, Nacc);
        sH[(v * TW + w) * SH + fl] = hp + hn;
#endif
      }
    }
  }
  __syncthreads();
  if (sR) cp_async_wait_all();
  phase_cells<DIR, SCH, SHP>(T, P, S, stage, flags, sH, sV, sQ, st, sRed, sR);
  if (eig) reduce_eig(emax, sRed, S);
  if (st) atomicOr(&S->status, st);
  if (nres) atomicAdd(&S->reset_cells, (unsigned long long)nres);
}

// ---------------------------------------------------------------------------------
// Compact schemes (crweno5, hccs): the reference solves, per line, variable and split,
// a tridiagonal system over faces ts .. n-ts (src/crweno5.cpp:44-401, src/hccs.cpp:45-493)
// with explicit end rows and explicit block-edge faces.  hccs77 (WHOLE) solves one system
// over all faces 0 .. n: WENO7-Z end rows at faces 0 and n from the neighbour's ghost
// cells and hccs rows everywhere else, the rows next to the block edges included
// (src/hccs77.cpp:45-195 inner, :218-568 left, :592-943 right, :945-978 the solve).
// Three kernels per direction:
//   compact_rows_kernel   split fluxes (phase 1 of the sweep), then per face either the
//                         explicit value (into fh) or the tridiagonal row (a, b, c, d)
//   compact_thomas_kernel one thread per system: the reference's Thomas elimination and
//                         back substitution (src/crweno5.cpp:207-218), into fh
//   compact_finish_kernel faces from fh, then phase 3 (difference, RHS, RK)
// Layouts per block and direction (nl lines = nW*nO, system s = sys*nl + line, sys =
// 2*variable + split): fh[(sys*nl + line)*(L+1) + face]; rows[(r*4 + k)*(10*nl) + s].
// ---------------------------------------------------------------------------------
template <int SCH>
__device__ __forceinline__ void compact_row(const double f[5], double &lo, double &di, double &up,
                                            double &rhs) {
  if (SCH == SCH_CRWENO5) crweno5_row(f, lo, di, up, rhs);
  else hccs_row(f, lo, di, up, rhs);
}

template <int DIR, int SCH, bool WHOLE = false>
__global__ void __launch_bounds__(kThreads, NUC3D_SWEEP_MINB)
compact_rows_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
                    int stage, int flags) {
  static_assert(!WHOLE || SCH == SCH_HCCS, "the whole-line system is the hccs77 form of hccs");
  using M = TileSmem<DIR, SCH>;
  constexpr int R = M::R, TW = M::TW, TL = M::TL, SP = M::SP;
  extern __shared__ double smem[];
  double *sF = smem;
  __shared__ double sRed[kThreads / 32];
  const TileCtx T = decode_tile<DIR>(blocks, tm, P);
  const bool eig = (flags & SW_EIG) != 0;
  unsigned st = 0;
  double emax = 0.0;
  unsigned nres = 0;
  phase_split<DIR, SCH>(blocks, T, P, stage, eig, sF, nullptr, st, emax, nullptr,
                        DIR == 0 ? &nres : nullptr);
  __syncthreads();
  const BlockDev &B = *T.B;
  const int L = T.G.L, ts = T.ts, f0 = WHOLE ? 0 : ts, m = L - 2 * f0 + 1;
  const long long nl = (long long)T.G.nW * T.G.nO;
  const long long S10 = 10 * nl;
  for (int e = threadIdx.x; e < TW * (TL + 1); e += kThreads) {
    const int fl = e % (TL + 1), w = e / (TL + 1);
    if (w >= T.nw || fl > T.cl) continue;
    const int f = T.c0 + fl;
    const long long line = (T.w0 + w) + (long long)T.G.nW * T.o;
#pragma unroll 1
    for (int sys = 0; sys < 10; ++sys) {
      const int v = sys >> 1, side = sys & 1;
      const double *row = sF + ((side ? 5 + v : v) * TW + w) * SP + (R - T.c0);
      auto A = [row](int c) { return row[c]; };
      const long long sidx = sys * nl + line;
      if (!WHOLE && (f < ts || f > L - ts)) {
        const double h = side ? recon_neg<SCH>(f, L, ts, T.physL, T.physR, A)
                              : recon_pos<SCH>(f, L, ts, T.physL, T.physR, false, A);
        B.fh[sidx * (L + 1) + f] = h;
        continue;
      }
      const int r = f - f0;
      double a, b, c, d;
      if (r == 0 || r == m - 1) {
        // explicit end rows: WENO5-JS (crweno5) or WENO7-Z (hccs, hccs77), the interior
        // stencil (hccs77: its faces 0 and n read the neighbour's ghost cells)
        a = 0.0; b = 1.0; c = 0.0;
        d = side ? recon_neg_in<SCH>(f, A) : recon_pos_in<SCH>(f, false, A);
      } else {
        double s5[5];
        if (side) { s5[0] = A(f + 2); s5[1] = A(f + 1); s5[2] = A(f); s5[3] = A(f - 1); s5[4] = A(f - 2); }
        else { s5[0] = A(f - 3); s5[1] = A(f - 2); s5[2] = A(f - 1); s5[3] = A(f); s5[4] = A(f + 1); }
        double lo, di, up;
        compact_row<SCH>(s5, lo, di, up, d);
        b = di;
        if (side) { a = up; c = lo; } else { a = lo; c = up; }
      }
      double *rw = B.rows + (long long)r * 4 * S10 + sidx;
      rw[0] = a;
      rw[S10] = b;
      rw[2 * S10] = c;
      rw[3 * S10] = d;
    }
  }
  if (eig) reduce_eig(emax, sRed, S);
  if (st) atomicOr(&S->status, st);
  if (nres) atomicAdd(&S->reset_cells, (unsigned long long)nres);
}

// One thread per (line, variable, split) system of one direction.
// f0: the face of the system's first row (ts; 0 for hccs77).
template <int DIR>
__global__ void __launch_bounds__(256)
compact_thomas_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, int f0) {
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const int n[3] = {B.n[0], B.n[1], B.n[2]};
  const Geo G = make_geo(DIR, n);
  const long long nl = (long long)G.nW * G.nO, S10 = 10 * nl;
  const long long s = (long long)(blockIdx.x - tm.tile_start[b]) * 256 + threadIdx.x;
  if (s >= S10) return;
  const int L = G.L, m = L - 2 * f0 + 1;
  double *rw = B.rows + s;
  double cp = rw[2 * S10], dp = rw[3 * S10];
  for (int r = 1; r < m; ++r) {
    double *x = rw + (long long)r * 4 * S10;
    const double a = x[0], bb = x[S10], c = x[2 * S10], d = x[3 * S10];
    const double den = bb - cp * a;
    cp = c / den;
    dp = (d - dp * a) / den;
    x[2 * S10] = cp;
    x[3 * S10] = dp;
  }
  double *fh = B.fh + s * (L + 1) + f0;
  double xv = dp;
  fh[m - 1] = xv;
  for (int r = m - 2; r >= 0; --r) {
    const double *x = rw + (long long)r * 4 * S10;
    xv = x[3 * S10] - x[2 * S10] * xv;
    fh[r] = xv;
  }
}

template <int DIR, int SCH>
__global__ void __launch_bounds__(kThreads, NUC3D_SWEEP_MINB)
compact_finish_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
                      int stage, int flags) {
  using M = TileSmem<DIR, SCH>;
  constexpr int TW = M::TW, TL = M::TL, SV = M::SV, SH = M::SH, SQ = M::SQ;
  extern __shared__ double smem[];
  double *sH = smem;
  double *sV = sH + 5 * TW * SH;
  const bool ns = (flags & SW_NS) != 0;
  double *sQ = sV + (ns ? 4 * TW * SV : 0);
  __shared__ double sRed[kThreads / 32];
  const TileCtx T = decode_tile<DIR>(blocks, tm, P);
  const BlockDev &B = *T.B;
  unsigned st = 0;
  if (DIR == 2 && (flags & SW_RK)) {
    // stage state of the tile's own cells (with the energy reset), as phase 1 leaves it
    for (int e = threadIdx.x; e < TW * TL; e += kThreads) {
      int c, w;
      w = e % TW; c = e / TW;
      if (w >= T.nw || c >= T.cl) continue;
      const long long idx = (T.c0 + c) * T.G.sL + (T.w0 + w) * T.G.sW + T.o * T.G.sO;
      double q[5];
      CellPrim s;
      load_q(B.q[stage], T.N, idx, q);
      con2prim(q, __ldg(B.jac + idx), P.gamma, P.mach, s, st);
      q[4] = s.q4;
#pragma unroll
      for (int v = 0; v < 5; ++v) sQ[(v * TW + w) * SQ + c] = q[v];
    }
  }
  if (ns) phase_vis<DIR, SCH>(blocks, T, P, sV);
  const int L = T.G.L;
  const long long nl = (long long)T.G.nW * T.G.nO;
  for (int e = threadIdx.x; e < TW * (TL + 1); e += kThreads) {
    const int fl = e % (TL + 1), w = e / (TL + 1);
    if (w >= T.nw || fl > T.cl) continue;
    const long long line = (T.w0 + w) + (long long)T.G.nW * T.o;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double hp = B.fh[((2 * v) * nl + line) * (L + 1) + T.c0 + fl];
      const double hn = B.fh[((2 * v + 1) * nl + line) * (L + 1) + T.c0 + fl];
      sH[(v * TW + w) * SH + fl] = hp + hn;
    }
  }
  __syncthreads();
  phase_cells<DIR, SCH>(T, P, S, stage, flags, sH, sV, sQ, st, sRed);
  if (st) atomicOr(&S->status, st);
}

#if NUC3D_FAST
// ---------------------------------------------------------------------------------
// Fused compact sweep (throughput build; crweno5 and hccs on lines of at most 256 cells).
// One CTA per line, 10 warps: phase 1 splits the line into shared memory; warp s solves
// the tridiagonal system of (variable s/2, split s%2) from those fluxes -- its rows are
// generated where they are needed, never stored to HBM -- and the explicit faces; the
// two splits are added; phase 3 as in the sweep.  The solve is the partition method
// (Wang 1981) on 32 lanes: lane l owns a chunk of 2..8 consecutive rows, eliminates it
// (forward to the chunk's first unknown, backward to its last) in registers, which leaves
// two rows per lane coupling only chunk ends; the 64-row reduced system is solved by
// parallel cyclic reduction (Hockney 1965) over warp shuffles (6 steps), and each lane
// recovers its interior unknowns.  The operation order differs from the reference's
// Thomas sweep (src/crweno5.cpp:207-218), so the results agree to round-off, not bits;
// the reference-order build keeps compact_thomas_kernel.
// ---------------------------------------------------------------------------------
constexpr int kLineThreads = 320;  // 10 warps: one per (variable, split) system
constexpr int kLineChunk = 8;      // rows per lane at most: systems of at most 256 rows

// Normalised row (a, c, d with unit diagonal) of the reduced system, for the shuffles.
struct PcrRow {
  double a, c, d;
};
__device__ __forceinline__ PcrRow pcr_shfl_up(PcrRow r, int o, int lane) {
  PcrRow x;
  x.a = __shfl_up_sync(0xffffffffu, r.a, o);
  x.c = __shfl_up_sync(0xffffffffu, r.c, o);
  x.d = __shfl_up_sync(0xffffffffu, r.d, o);
  if (lane < o) x.a = x.c = x.d = 0.0;  // beyond the system's first row: an identity row
  return x;
}
__device__ __forceinline__ PcrRow pcr_shfl_down(PcrRow r, int o, int lane) {
  PcrRow x;
  x.a = __shfl_down_sync(0xffffffffu, r.a, o);
  x.c = __shfl_down_sync(0xffffffffu, r.c, o);
  x.d = __shfl_down_sync(0xffffffffu, r.d, o);
  if (lane + o > 31) x.a = x.c = x.d = 0.0;
  return x;
}
// One cyclic-reduction update of row (a, b, c, d) from its normalised neighbours lo
// (the row s above) and hi (the row s below): the result couples rows 2s away.
__device__ __forceinline__ void pcr_update(double &a, double &b, double &c, double &d, PcrRow lo,
                                           PcrRow hi) {
  const double na = -a * lo.a, nc = -c * hi.c;
  b = b - a * lo.c - c * hi.a;
  d = d - a * lo.d - c * hi.d;
  a = na;
  c = nc;
}
__device__ __forceinline__ PcrRow pcr_norm(double a, double b, double c, double d) {
  const double r = qdiv(1.0, b);
  return PcrRow{a * r, c * r, d * r};
}

// Solve the m-row tridiagonal system row(r, a, b, c, d) (a of row 0 and c of row m-1
// zero), 2 <= m <= 32 * kLineChunk, with the 32 lanes of this warp; out(r, x) receives
// every unknown once.
template <class RowF, class OutF>
__device__ __forceinline__ void warp_tridiag(int m, RowF row, OutF out) {
  const int lane = threadIdx.x & 31;
  const int np = min(32, m >> 1);  // active lanes, each with >= 2 rows
  const int q = m / np, rem = m - q * np;
  const bool act = lane < np;
  const int r0 = lane * q + min(lane, rem);
  const int kk = act ? q + (lane < rem ? 1 : 0) : 0;
  double A[kLineChunk], C[kLineChunk], D[kLineChunk];
  // the lane's two rows of the reduced system: F (its first unknown: couples the previous
  // lane's last and its own last) and L (its last: couples its own first and the next
  // lane's first); inactive lanes hold identity rows
  double fa = 0.0, fb = 1.0, fc = 0.0, fd = 0.0, la = 0.0, lb = 1.0, lc = 0.0, ld = 0.0;
  // forward: row j becomes x_j + A_j x_first + C_j x_{j+1} = D_j (row 0 keeps its a,
  // the coupling to the previous chunk's last unknown).  The last row's values are final
  // here: L takes each valid row's in turn (no select by kk, which the compiler would
  // turn into an indexed, local-memory load).
#pragma unroll
  for (int j = 0; j < kLineChunk; ++j) {
    A[j] = C[j] = D[j] = 0.0;
    if (j < kk) {
      double a, b, c, d;
      row(r0 + j, a, b, c, d);
      if (j < 2) {
        const double r = qdiv(1.0, b);
        A[j] = a * r;
        C[j] = c * r;
        D[j] = d * r;
      } else {
        const double r = qdiv(1.0, b - a * C[j - 1]);
        A[j] = -r * a * A[j - 1];
        C[j] = r * c;
        D[j] = r * (d - a * D[j - 1]);
      }
      la = A[j];
      lc = C[j];
      ld = D[j];
    }
  }
  // backward: rows 1 .. kk-2 become x_j + A_j x_first + C_j x_last = D_j
#pragma unroll
  for (int j = kLineChunk - 3; j >= 1; --j) {
    if (j <= kk - 3) {
      A[j] = A[j] - C[j] * A[j + 1];
      D[j] = D[j] - C[j] * D[j + 1];
      C[j] = -C[j] * C[j + 1];
    }
  }
  if (act) {
    if (kk >= 3) {
      const double r = qdiv(1.0, 1.0 - C[0] * A[1]);
      fa = r * A[0];
      fc = -r * C[0] * C[1];
      fd = r * (D[0] - C[0] * D[1]);
    } else {
      fa = A[0];
      fc = C[0];
      fd = D[0];
    }
  }
  // cyclic reduction over the 64 reduced rows (row 2l = F of lane l, 2l+1 = L of lane l)
  {
    const PcrRow nf = pcr_norm(fa, fb, fc, fd), nl = pcr_norm(la, lb, lc, ld);
    const PcrRow lo = pcr_shfl_up(nl, 1, lane), hi = pcr_shfl_down(nf, 1, lane);
    pcr_update(fa, fb, fc, fd, lo, nl);
    pcr_update(la, lb, lc, ld, nf, hi);
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const PcrRow nf = pcr_norm(fa, fb, fc, fd), nl = pcr_norm(la, lb, lc, ld);
    const PcrRow flo = pcr_shfl_up(nf, o, lane), fhi = pcr_shfl_down(nf, o, lane);
    const PcrRow llo = pcr_shfl_up(nl, o, lane), lhi = pcr_shfl_down(nl, o, lane);
    pcr_update(fa, fb, fc, fd, flo, fhi);
    pcr_update(la, lb, lc, ld, llo, lhi);
  }
  if (!act) return;
  const double xf = qdiv(fd, fb), xl = qdiv(ld, lb);
  out(r0, xf);
#pragma unroll
  for (int j = 1; j < kLineChunk - 1; ++j)
    if (j < kk - 1) out(r0 + j, D[j] - A[j] * xf - C[j] * xl);
  out(r0 + kk - 1, xl);
}

// Row (a, b, c, d) of face f of one line's system from the split fluxes A(c) = rowF[c]:
// the compact row (src/crweno5.cpp:124-199, src/hccs.cpp:145-188 and their F- mirrors), or
// at the system's end rows the explicit interior reconstruction.
struct LineRow {
  double a, b, c, d;
};
template <int SCH>
__device__ __forceinline__ LineRow line_row(const double *rowF, int f, int side, bool end) {
  auto A = [rowF](int c) { return rowF[c]; };
  LineRow q;
  if (end) {
    q.a = 0.0;
    q.b = 1.0;
    q.c = 0.0;
    q.d = side ? recon_neg_in<SCH>(f, A) : recon_pos_in<SCH>(f, false, A);
    return q;
  }
  double s5[5];
  if (side) { s5[0] = A(f + 2); s5[1] = A(f + 1); s5[2] = A(f); s5[3] = A(f - 1); s5[4] = A(f - 2); }
  else { s5[0] = A(f - 3); s5[1] = A(f - 2); s5[2] = A(f - 1); s5[3] = A(f); s5[4] = A(f + 1); }
  double lo, di, up;
  compact_row<SCH>(s5, lo, di, up, q.d);
  q.b = di;
  if (side) { q.a = up; q.c = lo; } else { q.a = lo; q.c = up; }
  return q;
}

// The lines of tile t: tile = (group of TW neighbouring lanes) + groups * (outer index).
template <int DIR, int TW>
__device__ __forceinline__ TileCtx decode_line(const BlockDev *__restrict__ blocks, const TileMap &tm,
                                               const SolverParams &P) {
  TileCtx T;
  T.t = (int)blockIdx.x;
  T.b = find_block(tm, T.t);
  T.B = &blocks[T.b];
  for (int d = 0; d < 3; ++d) T.n[d] = T.B->n[d];
  T.G = make_geo(DIR, T.n);
  const int lt = T.t - tm.tile_start[T.b];
  const int ng = (T.G.nW + TW - 1) / TW;
  T.o = lt / ng;
  T.w0 = (lt - T.o * ng) * TW;
  T.nw = min(TW, T.G.nW - T.w0);
  T.c0 = 0;
  T.cl = T.G.L;
  T.N = T.B->N;
  T.ts = P.ts[DIR];
  T.physL = T.B->face[2 * DIR].type < 0;
  T.physR = T.B->face[2 * DIR + 1].type < 0;
  return T;
}

template <int DIR, int SCH>
__host__ __device__ constexpr size_t compact_line_smem_bytes(bool ns) {
  using M = TileSmem<DIR, SCH, line_shape(DIR)>;
  size_t n = (size_t)10 * M::TW * M::SP + (size_t)10 * M::TW * M::SH;
  if (ns) n += (size_t)4 * M::TW * M::SV;
  if (DIR == 2) n += (size_t)5 * M::TW * M::SQ;
  return n * sizeof(double);
}

template <int DIR, int SCH>
__global__ void __launch_bounds__(kLineThreads, DIR == 0 || kLineLanes <= 2 ? 2 : 1)
compact_line_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
                    int stage, int flags) {
  constexpr int SHP = line_shape(DIR);
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int R = M::R, TW = M::TW, SP = M::SP, SH = M::SH, SV = M::SV;
  static_assert(M::TL >= kLineMax, "whole lines per CTA");
  extern __shared__ double smem[];
  double *sF = smem;                // [10][TW][SP] split fluxes; later [5][TW][SH] face values
  double *sX = sF + 10 * TW * SP;   // [10][TW][SH] each system's solution and explicit faces
  const bool ns = (flags & SW_NS) != 0;
  double *sV = sX + 10 * TW * SH;   // [4][TW][SV] viscous fluxes (NS)
  double *sQ = sV + (ns ? 4 * TW * SV : 0);  // [5][TW][SQ] zeta: the stage state of the lines
  __shared__ double sRed[kLineThreads / 32];
  const TileCtx T = decode_line<DIR, TW>(blocks, tm, P);
  // phases 1 and 3 run on the first kThreads threads (their loops stride by kThreads and
  // phase 1 writes every item it visits); warp 9 takes part in the solve and the barriers
  // only, and in phase 3 as a tile with no lanes, which skips every item
  TileCtx Tp = T;
  if (threadIdx.x >= kThreads) Tp.nw = 0;
  const bool eig = (flags & SW_EIG) != 0;
  unsigned st = 0, nres = 0;
  double emax = 0.0;
  if (threadIdx.x < kThreads) {
    phase_split<DIR, SCH, false, SHP>(blocks, T, P, stage, eig, sF, DIR == 2 ? sQ : nullptr, st, emax,
                                      nullptr, DIR == 0 ? &nres : nullptr);
    if (ns) phase_vis<DIR, SCH, SHP>(blocks, T, P, sV);
  }
  __syncthreads();
  {
    const int sys = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v = sys >> 1, side = sys & 1;
    const int L = T.G.L, ts = T.ts, m = L - 2 * ts + 1;
    for (int w = 0; w < T.nw; ++w) {
      const double *rowF = sF + ((side ? 5 + v : v) * TW + w) * SP + R;  // c0 = 0
      auto A = [rowF](int c) { return rowF[c]; };
      double *x = sX + (sys * TW + w) * SH;
      // explicit faces next to the block edges (f < ts, f > L - ts)
      if (lane < 2 * ts) {
        const int f = lane < ts ? lane : L - 2 * ts + 1 + lane;
        x[f] = side ? recon_neg<SCH>(f, L, ts, T.physL, T.physR, A)
                    : recon_pos<SCH>(f, L, ts, T.physL, T.physR, false, A);
      }
      auto row = [&](int r, double &a, double &b, double &c, double &d) {
        const LineRow q = line_row<SCH>(rowF, ts + r, side, r == 0 || r == m - 1);
        a = q.a;
        b = q.b;
        c = q.c;
        d = q.d;
      };
      auto out = [x, ts](int r, double val) { x[ts + r] = val; };
      warp_tridiag(m, row, out);
    }
  }
  __syncthreads();
  double *sH = sF;
  const int nf = T.G.L + 1;
  for (int e = threadIdx.x; e < 5 * TW * nf; e += kLineThreads) {
    const int vw = e / nf, f = e - vw * nf, v = vw / TW, w = vw - v * TW;
    if (w < T.nw)
      sH[(v * TW + w) * SH + f] = sX[((2 * v) * TW + w) * SH + f] + sX[((2 * v + 1) * TW + w) * SH + f];
  }
  __syncthreads();
  phase_cells<DIR, SCH, SHP>(Tp, P, S, stage, flags & ~SW_EIG, sH, sV, sQ, st, sRed);
  if (eig) reduce_eig(emax, sRed, S);
  if (st) atomicOr(&S->status, st);
  if (nres) atomicAdd(&S->reset_cells, (unsigned long long)nres);
}
#endif  // NUC3D_FAST

// ---------------------------------------------------------------------------------
// Physical-face ghost fluxes: the reference's setBC (src/boundaryConditions.cpp:95-108)
// fills the ghost slabs before its sweeps; here one thread per face cell evaluates
// the slot next to the face (the only one the exterior reconstruction reads).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
bc_ghost_kernel(const BlockDev *__restrict__ blocks, const FaceJobs *__restrict__ jobs,
                SolverParams P, StepState *S, int stage, int k0 = 0, int k1 = 0x7fffffff) {
  int lo = 0, hi = jobs->njobs - 1;
  const int t = blockIdx.x;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (jobs->start[mid] <= t) lo = mid; else hi = mid - 1;
  }
  const BlockDev &B = blocks[jobs->block[lo]];
  const int f = jobs->face[lo], d = f >> 1, side = f & 1;
  const int A = d == 0 ? B.n[1] : (d == 1 ? B.n[2] : B.n[0]);
  const int Bn = d == 0 ? B.n[2] : (d == 1 ? B.n[0] : B.n[1]);
  const long long r = (long long)(t - jobs->start[lo]) * 256 + threadIdx.x;
  if (r >= (long long)A * Bn) return;
  const int a = (int)(r % A), b = (int)(r / A);
  int i, j, k;
  const int pos = side ? B.n[d] - 1 : 0;
  if (d == 0) { i = pos; j = a; k = b; }
  else if (d == 1) { i = b; j = pos; k = a; }
  else { i = a; j = b; k = pos; }
  if (k < k0 || k >= k1) return;  // a z-slab's share (nuc3d_solve_host's pipelined steps)
  const long long eidx = ((long long)k * B.n[1] + j) * B.n[0] + i;
  unsigned st = 0;
  double out[5];
  bc_ghost_flux(B, stage, d, side, eidx, P, out, st);
  double *gh = B.ghost + B.goff[f] + r;
  const long long area = (long long)A * Bn;
#pragma unroll
  for (int v = 0; v < 5; ++v) gh[v * area] = out[v];
  if (st) atomicOr(&S->status, st);
}

// ---------------------------------------------------------------------------------
// Navier-Stokes: primitives, then gradients and viscous fluxes per cell.
// ---------------------------------------------------------------------------------
constexpr int kCellTile = 256;
constexpr int kDiagChunk = 2048;  // values a reference-order sum stages at a time

// ---------------------------------------------------------------------------------
// The TVD-RK3 stage alone (tvdrk3rd::integrationAll, src/TVD-RK3.cpp:16-137), one thread
// per cell, from the right-hand side in B.rhs: q[(stage+1) mod 3] from u_i = q[stage] and
// u_n = q[0], each with con2prim's energy reset applied (src/physicsModel.cpp:324-332), as
// the reference's Q_work and Q_Euler hold them.  The fused path applies the same update in
// the zeta sweep; this kernel serves nuc3d_rk_stage.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kCellTile)
rk_stage_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S,
                int stage, double dt, int flags) {
  __shared__ double sRed[kCellTile / 32];
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const long long idx = (long long)(blockIdx.x - tm.tile_start[b]) * kCellTile + threadIdx.x;
  const long long N = B.N;
  unsigned st = 0;
  double racc = 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (stage == 0) S->dt = dt;
    if (stage == 2) S->time = S->time + dt;
  }
  if (idx < N) {
    const double jac = __ldg(B.jac + idx);
    double ui[5], un[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    load_q(B.q[stage], N, idx, ui);
    CellPrim s;
    con2prim(ui, jac, P.gamma, P.mach, s, st);
    ui[4] = s.q4;
    if (stage != 0) {
      load_q(B.q[0], N, idx, un);
      CellPrim sn;
      unsigned stn = 0;
      con2prim(un, jac, P.gamma, P.mach, sn, stn);
      un[4] = sn.q4;
    }
    double *__restrict__ qo = B.q[(stage + 1) % 3];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double x = rk3_update(stage, B.rhs[v * N + idx], ui[v], un[v], dt);
      if (!isfinite(x)) st |= ST_NONFINITE;
      qo[v * N + idx] = x;
      if (flags & SW_RES) res_value(B, v, idx, x, un[v], racc);
    }
  }
#if NUC3D_FAST
  if (flags & SW_RES) cta_sum_to(racc, sRed, kCellTile, P.res_part + blockIdx.x, [] { __syncthreads(); });
#endif
  st &= ST_NONFINITE | ST_NEG_PRESSURE;  // the reset was reported by the right-hand side
  if (st) atomicOr(&S->status, st);
}

// The step's residual from its last stage (PDEData3d::setRES, src/PDEData3d.cpp:90-122):
// per block res = |sqrt(sum (u - u_n)^2 / (5 N)) - res_last| / dt^2, res_last = that root
// (the reference keeps it in a function-static, one per rank, i.e. per block here), and
// the maximum over blocks (MPI_Allreduce MAX, :121) into S->res_bits.
__device__ __forceinline__ void residual_finish(const BlockDev &B, int b, double sum,
                                                double *__restrict__ res_last, StepState *S) {
  const double cnt = (double)((unsigned long long)B.N * 5ull);
  const double r = sqrt(sum / cnt);
  const double dt = S->dt;
  const double res = fabs(r - res_last[b]) / (dt * dt);
  res_last[b] = r;
  atomicMax(&S->res_bits, (unsigned long long)__double_as_longlong(res));
}

// Reference order: one CTA per block stages 2048 values of u - u_n at a time and thread 0
// adds their squares one by one, component by component, in cell order, as the
// reference's loops over Q_work do (src/PDEData3d.cpp:103-116).
__global__ void __launch_bounds__(256)
residual_seq_kernel(const BlockDev *__restrict__ blocks, double *__restrict__ res_last, StepState *S) {
  __shared__ double sd[kDiagChunk];
  const int b = blockIdx.x;
  const BlockDev &B = blocks[b];
  const long long n = 5 * B.N;
  double sum = 0.0;
  for (long long c0 = 0; c0 < n; c0 += kDiagChunk) {
    const int m = (int)min((long long)kDiagChunk, n - c0);
    for (int t = threadIdx.x; t < m; t += blockDim.x) sd[t] = B.dres[c0 + t];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int t = 0; t < m; ++t) sum = sum + sd[t] * sd[t];
    __syncthreads();
  }
  if (threadIdx.x == 0) residual_finish(B, b, sum, res_last, S);
}

// Throughput order: one CTA per block adds the block's per-tile sums (threads strided, then
// a fixed tree).
__global__ void __launch_bounds__(256)
residual_part_kernel(const BlockDev *__restrict__ blocks, TileMap tm, const double *__restrict__ part,
                     double *__restrict__ res_last, StepState *S) {
  __shared__ double sr[256];
  const int b = blockIdx.x;
  double acc = 0.0;
  for (int t = tm.tile_start[b] + threadIdx.x; t < tm.tile_start[b + 1]; t += blockDim.x) acc += part[t];
  sr[threadIdx.x] = acc;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sr[threadIdx.x] += sr[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) residual_finish(blocks[b], b, sr[0], res_last, S);
}

__global__ void __launch_bounds__(kCellTile)
prim_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, StepState *S, int stage) {
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const long long idx = (long long)(blockIdx.x - tm.tile_start[b]) * kCellTile + threadIdx.x;
  if (idx >= B.N) return;
  const long long N = B.N;
  unsigned st = 0;
  double q[5];
  CellPrim s;
  load_q(B.q[stage], N, idx, q);
  const double jac = __ldg(B.jac + idx);
  con2prim(q, jac, P.gamma, P.mach, s, st);
  B.prim[idx] = s.u;
  B.prim[N + idx] = s.v;
  B.prim[2 * N + idx] = s.w;
  B.prim[3 * N + idx] = temperature(s.rho, s.p, P.gamma, P.mach);
  if (st) atomicOr(&S->status, st);
}

// Value of primitive component comp at line offset g along direction d of cell (i,j,k).
__device__ __forceinline__ double prim_along(const BlockDev *__restrict__ blocks, const BlockDev &B,
                                             int d, int i, int j, int k, int g, int comp, int bfs) {
  const int L = B.n[d];
  if (g >= 0 && g < L) {
    int ii = i, jj = j, kk = k;
    if (d == 0) ii = g; else if (d == 1) jj = g; else kk = g;
    const long long idx = ((long long)kk * B.n[1] + jj) * B.n[0] + ii;
    return __ldg(B.prim + comp * B.N + idx);
  }
  const int a = d == 0 ? j : (d == 1 ? k : i);
  const int bb = d == 0 ? k : (d == 1 ? i : j);
  long long nidx;
  const int nb = ghost_cell(blocks, B, d, g, a, bb, bfs, nidx);
  if (nb < 0) return 0.0;  // never read: one-sided schemes stay inside the block
  return __ldg(blocks[nb].prim + comp * blocks[nb].N + nidx);
}

// d/d(direction d) of primitive components c0 .. c0+nc-1 of cell (i,j,k) near a block
// face: neighbour ghosts and the physical-face schemes.  Out of line, so that the
// kernels' common path (all stencil cells inside the block) stays small.
__device__ __noinline__ void prim_grad_edge(const BlockDev *__restrict__ blocks, const BlockDev &B,
                                            const SolverParams &P, int d, int i, int j, int k,
                                            int c0, int nc, double *out) {
  const int pos = d == 0 ? i : (d == 1 ? j : k);
  const bool pl = B.face[2 * d].type < 0, pr = B.face[2 * d + 1].type < 0;
  for (int c = 0; c < nc; ++c) {
    auto V = [&](int g) { return prim_along(blocks, B, d, i, j, k, g, c0 + c, P.bfs); };
    out[c] = diff_at(pos, B.n[d], P.ts[d], pl, pr, P.vis[d], V);
  }
}

// The direction's scheme_vis operator on a field with stride s from cell pointer f
// (every stencil cell inside the block).
__device__ __forceinline__ double diff_inner(const double *__restrict__ f, long long s, int vis) {
  auto V = [&](int o) { return __ldg(f + o * s); };
  if (vis == VIS_CD2) return cd2(V(-1), V(1));
  if (vis == VIS_CD8) return cd8(V(-4), V(-3), V(-2), V(-1), V(1), V(2), V(3), V(4));
  return cd6(V(-3), V(-2), V(-1), V(1), V(2), V(3));
}

// The viscous fluxes of one cell from its primitive gradients gr[u,v,w,T][xi,eta,zeta]:
// Sutherland viscosity, stresses, heat flux, contravariant fluxes / J into B.vis
// (src/NaiverStokes3d.cpp:130-326, src/physicsModel.cpp:199-234).
__device__ __forceinline__ void visc_flux_cell(const BlockDev &B, const SolverParams &P, long long idx,
                                               const double (&gr)[4][3]) {
  const long long N = B.N;
  const double jac = __ldg(B.jac + idx);
  double mx[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) mx[d][c] = __ldg(B.met[d] + c * N + idx);
  const double xi_x = mx[0][0], xi_y = mx[0][1], xi_z = mx[0][2];
  const double eta_x = mx[1][0], eta_y = mx[1][1], eta_z = mx[1][2];
  const double zeta_x = mx[2][0], zeta_y = mx[2][1], zeta_z = mx[2][2];

  double ux = gr[0][0] * xi_x + gr[0][1] * eta_x + gr[0][2] * zeta_x;
  double uy = gr[0][0] * xi_y + gr[0][1] * eta_y + gr[0][2] * zeta_y;
  double uz = gr[0][0] * xi_z + gr[0][1] * eta_z + gr[0][2] * zeta_z;
  double vx = gr[1][0] * xi_x + gr[1][1] * eta_x + gr[1][2] * zeta_x;
  double vy = gr[1][0] * xi_y + gr[1][1] * eta_y + gr[1][2] * zeta_y;
  double vz = gr[1][0] * xi_z + gr[1][1] * eta_z + gr[1][2] * zeta_z;
  double wx = gr[2][0] * xi_x + gr[2][1] * eta_x + gr[2][2] * zeta_x;
  double wy = gr[2][0] * xi_y + gr[2][1] * eta_y + gr[2][2] * zeta_y;
  double wz = gr[2][0] * xi_z + gr[2][1] * eta_z + gr[2][2] * zeta_z;
  double tx = gr[3][0] * xi_x + gr[3][1] * eta_x + gr[3][2] * zeta_x;
  double ty = gr[3][0] * xi_y + gr[3][1] * eta_y + gr[3][2] * zeta_y;
  double tz = gr[3][0] * xi_z + gr[3][1] * eta_z + gr[3][2] * zeta_z;

  const double T = __ldg(B.prim + 3 * N + idx);
  const double nd = P.t_ref / P.t_inf;
#if NUC3D_FAST
  const double miu0 = qdiv((1.0 + nd) * pow15(T), (T + nd) * P.reynolds);
  const double coeff0 = qdiv(miu0, (P.gamma - 1.0) * P.mach * P.mach * P.prandtl);
#else
  const double miu0 = (1.0 + nd) / (T + nd) * pow15(T) / P.reynolds;
  const double coeff0 = miu0 / ((P.gamma - 1.0) * P.mach * P.mach * P.prandtl);
#endif

  double grad = ux + vy + wz;
  double tau_xx = miu0 * (2.0 * ux - 2.0 / 3.0 * grad);
  double tau_xy = miu0 * (uy + vx - 2.0 / 3.0 * grad);
  double tau_xz = miu0 * (uz + wx - 2.0 / 3.0 * grad);
  double tau_yy = miu0 * (2.0 * vy - 2.0 / 3.0 * grad);
  double tau_yz = miu0 * (vz + wy - 2.0 / 3.0 * grad);
  double tau_zz = miu0 * (2.0 * wz - 2.0 / 3.0 * grad);
  double tau_tx = coeff0 * tx;
  double tau_ty = coeff0 * ty;
  double tau_tz = coeff0 * tz;
  const double u = __ldg(B.prim + idx), v = __ldg(B.prim + N + idx), w = __ldg(B.prim + 2 * N + idx);
  double fv[4] = {tau_xx, tau_xy, tau_xz, u * tau_xx + v * tau_xy + w * tau_xz + tau_tx};
  double gv[4] = {tau_xy, tau_yy, tau_yz, u * tau_xy + v * tau_yy + w * tau_yz + tau_ty};
  double hv[4] = {tau_xz, tau_yz, tau_zz, u * tau_xz + v * tau_yz + w * tau_zz + tau_tz};
#if NUC3D_FAST
  const double rj = qdiv(1.0, jac);  // one division for the twelve fluxes' 1/J
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    B.vis[(0 * 4 + c) * N + idx] = (xi_x * fv[c] + xi_y * gv[c] + xi_z * hv[c]) * rj;
    B.vis[(1 * 4 + c) * N + idx] = (eta_x * fv[c] + eta_y * gv[c] + eta_z * hv[c]) * rj;
    B.vis[(2 * 4 + c) * N + idx] = (zeta_x * fv[c] + zeta_y * gv[c] + zeta_z * hv[c]) * rj;
  }
#else
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    B.vis[(0 * 4 + c) * N + idx] = (xi_x * fv[c] + xi_y * gv[c] + xi_z * hv[c]) / jac;
    B.vis[(1 * 4 + c) * N + idx] = (eta_x * fv[c] + eta_y * gv[c] + eta_z * hv[c]) / jac;
    B.vis[(2 * 4 + c) * N + idx] = (zeta_x * fv[c] + zeta_y * gv[c] + zeta_z * hv[c]) / jac;
  }
#endif
}

// NaiverStokesData3d::solveGrads + solveViscousFlux (src/NaiverStokes3d.cpp:63-326)
// with physicsModel::sutherland (src/physicsModel.cpp:199-234).
#ifndef NUC3D_GRAD_MINB
#define NUC3D_GRAD_MINB 4  // resident CTAs per SM the gradient kernel's registers are cut for:
#endif                     // 64 registers, 7% faster than 80 (3 CTAs) despite spills
__global__ void __launch_bounds__(kCellTile, NUC3D_GRAD_MINB)
grad_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P) {
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const long long t = (long long)(blockIdx.x - tm.tile_start[b]) * kCellTile + threadIdx.x;
  if (t >= B.N) return;
  const long long N = B.N;
  const int nx = B.n[0], ny = B.n[1];
  // Threads take the cells whose xi stencil stays inside the block first (row by row), then
  // the E cells at each end of every xi row, so that a warp's lanes take the same xi
  // branch below (cell by cell in order, 3 lanes of every other warp took the edge path).
  const int E = P.ts[0], ni = nx - 2 * E;  // nx >= 2 bfsize + 2 > 2 E
  const long long nint = (long long)ni * ny * B.n[2];
  long long row;
  int i;
  if (t < nint) {
    row = t / ni;
    i = E + (int)(t - row * ni);
  } else {
    const long long e = t - nint;
    row = e / (2 * E);
    const int c = (int)(e - row * 2 * E);
    i = c < E ? c : nx - 2 * E + c;
  }
  const int j = (int)(row % ny), k = (int)(row / ny);
  const long long idx = row * nx + i;
  const int pos[3] = {i, j, k};
  const long long stride[3] = {1, nx, (long long)nx * ny};
  double gr[4][3];  // [u,v,w,T][xi,eta,zeta]
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // one-sided schemes within ts of a physical face, ghosts within reach <= ts of any face
    if (pos[d] >= P.ts[d] && pos[d] < B.n[d] - P.ts[d]) {
#pragma unroll
      for (int c = 0; c < 4; ++c) gr[c][d] = diff_inner(B.prim + c * N + idx, stride[d], P.vis[d]);
    } else {
      double g4[4];
      prim_grad_edge(blocks, B, P, d, i, j, k, 0, 4, g4);
#pragma unroll
      for (int c = 0; c < 4; ++c) gr[c][d] = g4[c];
    }
  }
  visc_flux_cell(B, P, idx, gr);
}

// ---------------------------------------------------------------------------------
// Diagnostics: postproc::solveQ (src/postproc.cpp:743-848) after block::Post's getPrim
// (src/block.cpp:601-618).  Velocity gradients use the block's difference operator
// exactly as the viscous path does (postproc::solveGrad, :1797-1820: neighbour halos,
// boundaryScheme at physical faces), then the chain rule of solveGrad_x/y/z, vorticity,
// the Q criterion, and the per-cell terms of the totals.
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kCellTile)
diag_prim_kernel(const BlockDev *__restrict__ blocks, const DiagDev *__restrict__ dd, TileMap tm,
                 SolverParams P) {
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const long long idx = (long long)(blockIdx.x - tm.tile_start[b]) * kCellTile + threadIdx.x;
  if (idx >= B.N) return;
  const long long N = B.N;
  unsigned st = 0;
  double q[5];
  CellPrim s;
  load_q(B.q[0], N, idx, q);
  con2prim(q, __ldg(B.jac + idx), P.gamma, P.mach, s, st);
  double *pr = dd[b].prim;
  pr[idx] = s.rho;
  pr[N + idx] = s.u;
  pr[2 * N + idx] = s.v;
  pr[3 * N + idx] = s.w;
}

// Component comp of the diagnostics primitives at line offset g along d of cell (i,j,k),
// across a block face from the neighbour (the raw-slab exchange of solveGrad_df).
__device__ __forceinline__ double diag_prim_along(const BlockDev *__restrict__ blocks,
                                                  const DiagDev *__restrict__ dd, int b, int d,
                                                  int i, int j, int k, int g, int comp, int bfs) {
  const BlockDev &B = blocks[b];
  const int L = B.n[d];
  if (g >= 0 && g < L) {
    int ii = i, jj = j, kk = k;
    if (d == 0) ii = g; else if (d == 1) jj = g; else kk = g;
    const long long idx = ((long long)kk * B.n[1] + jj) * B.n[0] + ii;
    return __ldg(dd[b].prim + comp * B.N + idx);
  }
  const int a = d == 0 ? j : (d == 1 ? k : i);
  const int bb = d == 0 ? k : (d == 1 ? i : j);
  long long nidx;
  const int nb = ghost_cell(blocks, B, d, g, a, bb, bfs, nidx);
  if (nb < 0) return 0.0;  // never read: one-sided schemes stay inside the block
  return __ldg(dd[nb].prim + comp * blocks[nb].N + nidx);
}

__device__ __noinline__ void diag_grad_edge(const BlockDev *__restrict__ blocks,
                                            const DiagDev *__restrict__ dd, const SolverParams &P,
                                            int b, int d, int i, int j, int k, double *out) {
  const BlockDev &B = blocks[b];
  const int pos = d == 0 ? i : (d == 1 ? j : k);
  const bool pl = B.face[2 * d].type < 0, pr = B.face[2 * d + 1].type < 0;
  for (int c = 0; c < 3; ++c) {
    auto V = [&](int g) { return diag_prim_along(blocks, dd, b, d, i, j, k, g, c + 1, P.bfs); };
    out[c] = diff_at(pos, B.n[d], P.ts[d], pl, pr, P.vis[d], V);
  }
}

__global__ void __launch_bounds__(kCellTile)
diag_kernel(const BlockDev *__restrict__ blocks, const DiagDev *__restrict__ dd, TileMap tm,
            SolverParams P) {
  const int b = find_block(tm, blockIdx.x);
  const BlockDev &B = blocks[b];
  const long long idx = (long long)(blockIdx.x - tm.tile_start[b]) * kCellTile + threadIdx.x;
  if (idx >= B.N) return;
  const long long N = B.N;
  const int nx = B.n[0], ny = B.n[1];
  const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((long long)nx * ny));
  const int pos[3] = {i, j, k};
  const long long stride[3] = {1, nx, (long long)nx * ny};
  double gr[3][3];  // [u,v,w][xi,eta,zeta]
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (pos[d] >= P.ts[d] && pos[d] < B.n[d] - P.ts[d]) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
        gr[c][d] = diff_inner(dd[b].prim + (c + 1) * N + idx, stride[d], P.vis[d]);
    } else {
      double g3[3];
      diag_grad_edge(blocks, dd, P, b, d, i, j, k, g3);
#pragma unroll
      for (int c = 0; c < 3; ++c) gr[c][d] = g3[c];
    }
  }
  double mx[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) mx[d][c] = __ldg(B.met[d] + c * N + idx);
  const double xi_x = mx[0][0], xi_y = mx[0][1], xi_z = mx[0][2];
  const double eta_x = mx[1][0], eta_y = mx[1][1], eta_z = mx[1][2];
  const double zeta_x = mx[2][0], zeta_y = mx[2][1], zeta_z = mx[2][2];
  // solveGrad_x/y/z (src/postproc.cpp:1825-1950)
  const double ux = gr[0][0] * xi_x + gr[0][1] * eta_x + gr[0][2] * zeta_x;
  const double uy = gr[0][0] * xi_y + gr[0][1] * eta_y + gr[0][2] * zeta_y;
  const double uz = gr[0][0] * xi_z + gr[0][1] * eta_z + gr[0][2] * zeta_z;
  const double vx = gr[1][0] * xi_x + gr[1][1] * eta_x + gr[1][2] * zeta_x;
  const double vy = gr[1][0] * xi_y + gr[1][1] * eta_y + gr[1][2] * zeta_y;
  const double vz = gr[1][0] * xi_z + gr[1][1] * eta_z + gr[1][2] * zeta_z;
  const double wx = gr[2][0] * xi_x + gr[2][1] * eta_x + gr[2][2] * zeta_x;
  const double wy = gr[2][0] * xi_y + gr[2][1] * eta_y + gr[2][2] * zeta_y;
  const double wz = gr[2][0] * xi_z + gr[2][1] * eta_z + gr[2][2] * zeta_z;
  // solveQ's cell body (src/postproc.cpp:807-829)
  const double w0 = wy - vz, w1 = uz - wx, w2 = vx - uy;
  const double q0 = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
  const DiagDev &D = dd[b];
  D.fields[idx] = w0;
  D.fields[N + idx] = w1;
  D.fields[2 * N + idx] = w2;
  D.fields[3 * N + idx] = (w0 * w0 + w1 * w1 + w2 * w2) * 0.5;
  D.fields[4 * N + idx] = q0;
  const double rho = D.prim[idx], u = D.prim[N + idx], v = D.prim[2 * N + idx],
               w = D.prim[3 * N + idx];
  D.dens[idx] = 0.5 * (w0 * w0 + w1 * w1 + w2 * w2);
  D.dens[N + idx] = 0.5 * rho * (u * u + v * v + w * w);
}

// Reference-order totals: one CTA per block stages 2048-cell chunks of both terms in
// shared memory and thread 0 adds them one by one in cell order, as the reference's
// k-j-i loop does.  Bitwise equal to the reference; about 2 ns per cell.
__global__ void __launch_bounds__(256)
diag_sum_seq_kernel(const BlockDev *__restrict__ blocks, const DiagDev *__restrict__ dd,
                    double *__restrict__ sums) {
  __shared__ double se[kDiagChunk], sk[kDiagChunk];
  const int b = blockIdx.x;
  const long long N = blocks[b].N;
  const double *e = dd[b].dens, *kk = e + N;
  double ens = 0.0, kin = 0.0;
  for (long long c0 = 0; c0 < N; c0 += kDiagChunk) {
    const int n = (int)min((long long)kDiagChunk, N - c0);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      se[t] = e[c0 + t];
      sk[t] = kk[c0 + t];
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int t = 0; t < n; ++t) {
        ens += se[t];
        kin += sk[t];
      }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[2 * b] = ens;
    sums[2 * b + 1] = kin;
  }
}

// Throughput totals, deterministic: kDiagParts CTAs per block each add a contiguous
// slice (threads strided, then a fixed tree), and one thread per block adds the parts in
// order.  The summation order differs from the reference's (round-off level).
__global__ void __launch_bounds__(256)
diag_sum_part_kernel(const BlockDev *__restrict__ blocks, const DiagDev *__restrict__ dd,
                     double *__restrict__ parts) {
  __shared__ double re[256], rk[256];
  const int b = blockIdx.y, part = blockIdx.x;
  const long long N = blocks[b].N;
  const long long span = (N + kDiagParts - 1) / kDiagParts;
  const long long lo = part * span, hi = min(N, lo + span);
  const double *e = dd[b].dens, *kk = e + N;
  double ens = 0.0, kin = 0.0;
  for (long long x = lo + threadIdx.x; x < hi; x += blockDim.x) {
    ens += e[x];
    kin += kk[x];
  }
  re[threadIdx.x] = ens;
  rk[threadIdx.x] = kin;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      re[threadIdx.x] += re[threadIdx.x + h];
      rk[threadIdx.x] += rk[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    parts[(2 * b) * kDiagParts + part] = re[0];
    parts[(2 * b + 1) * kDiagParts + part] = rk[0];
  }
}

__global__ void diag_sum_parts_kernel(int nblocks, const double *__restrict__ parts,
                                      double *__restrict__ sums) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nblocks) return;
  double acc = 0.0;
  for (int p = 0; p < kDiagParts; ++p) acc += parts[t * kDiagParts + p];
  sums[t] = acc;
}

// ---------------------------------------------------------------------------------
// Metrics: block::getJacobians (src/block.cpp:237-325) from the node coordinates, with the
// tile-Lagrange reconstruction of the derivatives (interpolation_derlag :327-477,
// coefficients src/block.h:36-48): every cell sums the 5x5x5 nodes of its 4x4x4-cell tile,
// xi innermost, then eta, then zeta, each sum from 0.0, as the reference does.
// ---------------------------------------------------------------------------------
__device__ constexpr double kLag[4][5] = {
    {35.0 / 128.0, 35.0 / 32.0, -35.0 / 64.0, 7.0 / 32.0, -5.0 / 128.0},
    {-5.0 / 128.0, 15.0 / 32.0, 45.0 / 64.0, -5.0 / 32.0, 3.0 / 128.0},
    {3.0 / 128.0, -5.0 / 32.0, 45.0 / 64.0, 15.0 / 32.0, -5.0 / 128.0},
    {-5.0 / 128.0, 7.0 / 32.0, -35.0 / 64.0, 35.0 / 32.0, 35.0 / 128.0}};
__device__ constexpr double kDerLag[4][5] = {
    {-11.0 / 12.0, 17.0 / 24.0, 3.0 / 8.0, -5.0 / 24.0, 1.0 / 24.0},
    {1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0, 0.0},
    {0.0, 1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0},
    {-1.0 / 24.0, 5.0 / 24.0, -3.0 / 8.0, -17.0 / 24.0, 11.0 / 12.0}};

// d(f)/d(xi, eta, zeta) of one coordinate f at cell (i,j,k): out[d]
__device__ __forceinline__ void tile_derivs(const double *__restrict__ f, int nx0, int ny0, int i,
                                            int j, int k, double out[3]) {
  const int ti = i & ~3, tj = j & ~3, tk = k & ~3, ai = i & 3, aj = j & 3, ak = k & 3;
  double vz[3] = {0.0, 0.0, 0.0};
  for (int kk = 0; kk < 5; ++kk) {
    double vy[3] = {0.0, 0.0, 0.0};
    for (int jj = 0; jj < 5; ++jj) {
      const double *row = f + ((long long)(tk + kk) * ny0 + (tj + jj)) * nx0 + ti;
      double vxd = 0.0, vxl = 0.0;  // DERLAG and LAG along xi
      for (int ii = 0; ii < 5; ++ii) {
        const double v = __ldg(row + ii);
        vxd = vxd + kDerLag[ai][ii] * v;
        vxl = vxl + kLag[ai][ii] * v;
      }
      vy[0] = vy[0] + kLag[aj][jj] * vxd;     // d/dxi:   DERLAG, LAG, LAG
      vy[1] = vy[1] + kDerLag[aj][jj] * vxl;  // d/deta:  LAG, DERLAG, LAG
      vy[2] = vy[2] + kLag[aj][jj] * vxl;     // d/dzeta: LAG, LAG, DERLAG
    }
    vz[0] = vz[0] + kLag[ak][kk] * vy[0];
    vz[1] = vz[1] + kLag[ak][kk] * vy[1];
    vz[2] = vz[2] + kDerLag[ak][kk] * vy[2];
  }
  out[0] = vz[0];
  out[1] = vz[1];
  out[2] = vz[2];
}

__global__ void __launch_bounds__(256)
metrics_kernel(const double *__restrict__ x, const double *__restrict__ y,
               const double *__restrict__ z, int nx, int ny, int nz, double *__restrict__ jac,
               double *__restrict__ met, double *__restrict__ dxyz, unsigned *__restrict__ bad) {
  const long long N = (long long)nx * ny * nz;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N) return;
  const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((long long)nx * ny));
  double dx[3], dy[3], dz[3];
  tile_derivs(x, nx + 1, ny + 1, i, j, k, dx);
  tile_derivs(y, nx + 1, ny + 1, i, j, k, dy);
  tile_derivs(z, nx + 1, ny + 1, i, j, k, dz);
  const double x_xi = dx[0], x_eta = dx[1], x_zeta = dx[2];
  const double y_xi = dy[0], y_eta = dy[1], y_zeta = dy[2];
  const double z_xi = dz[0], z_eta = dz[1], z_zeta = dz[2];
  const double jacob = 1.0 / (x_xi * (y_eta * z_zeta - y_zeta * z_eta) +
                              x_eta * (y_zeta * z_xi - y_xi * z_zeta) +
                              x_zeta * (y_xi * z_eta - y_eta * z_xi));
  if (jacob < 0.0) atomicOr(bad, 1u);  // the reference exits (src/block.cpp:314-318)
  jac[idx] = jacob;
  met[idx] = (y_eta * z_zeta - y_zeta * z_eta) * jacob;
  met[N + idx] = (x_zeta * z_eta - x_eta * z_zeta) * jacob;
  met[2 * N + idx] = (x_eta * y_zeta - x_zeta * y_eta) * jacob;
  met[3 * N + idx] = (y_zeta * z_xi - y_xi * z_zeta) * jacob;
  met[4 * N + idx] = (x_xi * z_zeta - x_zeta * z_xi) * jacob;
  met[5 * N + idx] = (x_zeta * y_xi - x_xi * y_zeta) * jacob;
  met[6 * N + idx] = (y_xi * z_eta - y_eta * z_xi) * jacob;
  met[7 * N + idx] = (x_eta * z_xi - x_xi * z_eta) * jacob;
  met[8 * N + idx] = (x_xi * y_eta - x_eta * y_xi) * jacob;
  if (dxyz) {
    const double d9[9] = {x_xi, x_eta, x_zeta, y_xi, y_eta, y_zeta, z_xi, z_eta, z_zeta};
#pragma unroll
    for (int c = 0; c < 9; ++c) dxyz[c * N + idx] = d9[c];
  }
}

// ---------------------------------------------------------------------------------
// Host-side launchers (called by the C-ABI layer).
// ---------------------------------------------------------------------------------
// Shared memory of the hybrid sweep: the plain sweep's plus rho and p per position.
template <int DIR, int SCH, int SHP = 0>
__host__ __device__ constexpr size_t hybrid_smem_bytes(bool ns) {
  using M = TileSmem<DIR, SCH, SHP>;
  return sweep_smem_bytes<DIR, SCH, SHP>(ns) + (size_t)2 * M::TW * M::SP * sizeof(double) + kHybSmem +
         (NUC3D_HYB_PREFETCH ? rhs_stage_bytes<DIR>(ns) : 0);
}

template <int DIR, int SCH, int SHP>
inline cudaError_t launch_sweep_s(const Launch &L, int stage, int flags) {
  const int ntiles = tile_range(L.tm_dir[DIR]);
  if (ntiles <= 0) return cudaSuccess;
  const bool ns = (flags & SW_NS) != 0;
#if NUC3D_FAST
  if constexpr (SCH == SCH_WENO5Z) {
    if (L.P.sensor) {
      sweep_kernel<DIR, SCH, true, SHP><<<ntiles, kThreads, hybrid_smem_bytes<DIR, SCH, SHP>(ns), L.stream>>>(
          L.d_blocks, L.tm_dir[DIR], L.P, L.d_state, stage, flags);
      return cudaGetLastError();
    }
  }
#endif
  if (L.d_maps && L.pipe_grid > 0 && ((L.pipe_dirs >> DIR) & 1)) {
    // persistent sweep fed by tensor-map loads (sweep_pipe.cuh)
    const int grid = ntiles < L.pipe_grid ? ntiles : L.pipe_grid;
    if (ns)
      pipe_sweep_kernel<DIR, SCH, SHP, true><<<grid, kPipeThreads, PipeSmem<DIR, SCH, SHP, true>::TOTAL,
                                               L.stream>>>(L.d_blocks, L.d_maps, L.tm_dir[DIR], L.P,
                                                           L.d_state, stage, flags);
    else
      pipe_sweep_kernel<DIR, SCH, SHP><<<grid, kPipeThreads, PipeSmem<DIR, SCH, SHP>::TOTAL, L.stream>>>(
          L.d_blocks, L.d_maps, L.tm_dir[DIR], L.P, L.d_state, stage, flags);
    return cudaGetLastError();
  }
  const size_t smem = sweep_smem_bytes<DIR, SCH, SHP>(ns) + rhs_stage_bytes<DIR>(ns);
  sweep_kernel<DIR, SCH, false, SHP><<<ntiles, kThreads, smem, L.stream>>>(L.d_blocks, L.tm_dir[DIR], L.P,
                                                               L.d_state, stage, flags);
  return cudaGetLastError();
}

template <int DIR, int SCH>
inline cudaError_t launch_sweep_t(const Launch &L, int stage, int flags) {
  switch (L.shape[DIR]) {
    case 0: return launch_sweep_s<DIR, SCH, 0>(L, stage, flags);
    case 1: return launch_sweep_s<DIR, SCH, 1>(L, stage, flags);
    case 2: return launch_sweep_s<DIR, SCH, 2>(L, stage, flags);
    default: return cudaErrorInvalidValue;
  }
}

template <int DIR, int SCH>
__host__ __device__ constexpr size_t compact_rows_smem_bytes() {
  using M = TileSmem<DIR, SCH>;
  return (size_t)10 * M::TW * M::SP * sizeof(double);
}
template <int DIR, int SCH>
__host__ __device__ constexpr size_t compact_finish_smem_bytes(bool ns) {
  using M = TileSmem<DIR, SCH>;
  size_t n = (size_t)5 * M::TW * M::SH;
  if (ns) n += (size_t)4 * M::TW * M::SV;
  if (DIR == 2) n += (size_t)5 * M::TW * M::SQ;
  return n * sizeof(double);
}

template <int DIR, int SCH, bool WHOLE = false>
inline cudaError_t launch_compact_t(const Launch &L, int stage, int flags) {
#if NUC3D_FAST
  if (!WHOLE && ((L.line_dirs >> DIR) & 1)) {
    const int nlines = L.tm_line[DIR].tile_start[L.tm_line[DIR].nblocks];
    compact_line_kernel<DIR, SCH><<<nlines, kLineThreads,
                                    compact_line_smem_bytes<DIR, SCH>((flags & SW_NS) != 0),
                                    L.stream>>>(L.d_blocks, L.tm_line[DIR], L.P, L.d_state, stage,
                                                flags);
    return cudaGetLastError();
  }
#endif
  const int ntiles = L.tm_dir[DIR].tile_start[L.tm_dir[DIR].nblocks];
  compact_rows_kernel<DIR, SCH, WHOLE>
      <<<ntiles, kThreads, compact_rows_smem_bytes<DIR, SCH>(), L.stream>>>(
          L.d_blocks, L.tm_dir[DIR], L.P, L.d_state, stage, flags & SW_EIG);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nsys = L.tm_sys[DIR].tile_start[L.tm_sys[DIR].nblocks];
  compact_thomas_kernel<DIR><<<nsys, 256, 0, L.stream>>>(L.d_blocks, L.tm_sys[DIR], L.P,
                                                         WHOLE ? 0 : L.P.ts[DIR]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  compact_finish_kernel<DIR, SCH><<<ntiles, kThreads,
                                    compact_finish_smem_bytes<DIR, SCH>((flags & SW_NS) != 0),
                                    L.stream>>>(L.d_blocks, L.tm_dir[DIR], L.P, L.d_state, stage,
                                                flags & ~SW_EIG);
  return cudaGetLastError();
}

template <int DIR>
inline cudaError_t launch_sweep(const Launch &L, int stage, int flags) {
  switch (L.P.scheme[DIR]) {
    case SCH_WENO5JS: return launch_sweep_t<DIR, SCH_WENO5JS>(L, stage, flags);
    case SCH_WENO5Z: return launch_sweep_t<DIR, SCH_WENO5Z>(L, stage, flags);
    case SCH_WENO7JS: return launch_sweep_t<DIR, SCH_WENO7JS>(L, stage, flags);
    case SCH_WENO3JS: return launch_sweep_t<DIR, SCH_WENO3JS>(L, stage, flags);
    case SCH_UPWIND1: return launch_sweep_t<DIR, SCH_UPWIND1>(L, stage, flags);
    case SCH_CRWENO5: return launch_compact_t<DIR, SCH_CRWENO5>(L, stage, flags);
    case SCH_HCCS: return launch_compact_t<DIR, SCH_HCCS>(L, stage, flags);
    case SCH_HCCS77: return launch_compact_t<DIR, SCH_HCCS, true>(L, stage, flags);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t run_residual(const Launch &L, bool cells);

// One right-hand-side evaluation at stage `stage`; with rk, also the stage update.
inline cudaError_t launch_stage(const Launch &L, int stage, bool rk, bool eig) {
  cudaError_t e;
  const bool ns = L.P.model == MODEL_NS;
  if (L.bc_tiles > 0) {
    bc_ghost_kernel<<<L.bc_tiles, 256, 0, L.stream>>>(L.d_blocks, L.d_jobs, L.P, L.d_state, stage);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (ns) {
    const int nt = L.tm_cells.tile_start[L.tm_cells.nblocks];
    prim_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, L.tm_cells, L.P, L.d_state, stage);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    grad_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, L.tm_cells, L.P);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  const int nsf = ns ? SW_NS : 0;
  const bool res = rk && stage == 2 && L.d_res_last;  // the step's residual at its last stage
  if ((e = launch_sweep<0>(L, stage, nsf | (eig ? SW_EIG : 0))) != cudaSuccess) return e;
  if ((e = launch_sweep<1>(L, stage, nsf)) != cudaSuccess) return e;
  if ((e = launch_sweep<2>(L, stage, nsf | (rk ? SW_RK : 0) | (res ? SW_RES : 0))) != cudaSuccess)
    return e;
  if (res) return run_residual(L, false);
  return cudaSuccess;
}

cudaError_t run_residual(const Launch &L, bool cells) {
  const int nb = L.tm_cells.nblocks;
  cudaError_t e = cudaMemsetAsync(&L.d_state->res_bits, 0, sizeof(unsigned long long), L.stream);
  if (e != cudaSuccess) return e;
#if NUC3D_FAST
  // the partial sums are per tile of the kernel that applied the last stage
  const bool line = (L.line_dirs >> 2) & 1;
  residual_part_kernel<<<nb, 256, 0, L.stream>>>(
      L.d_blocks, cells ? L.tm_cells : (line ? L.tm_line[2] : L.tm_dir[2]), L.P.res_part,
      L.d_res_last, L.d_state);
#else
  (void)cells;
  residual_seq_kernel<<<nb, 256, 0, L.stream>>>(L.d_blocks, L.d_res_last, L.d_state);
#endif
  return cudaGetLastError();
}

cudaError_t run_rk_stage(const Launch &L, int stage, double dt) {
  const bool res = stage == 2 && L.d_res_last;
  const int nt = L.tm_cells.tile_start[L.tm_cells.nblocks];
  rk_stage_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, L.tm_cells, L.P, L.d_state, stage, dt,
                                                  res ? SW_RES : 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !res) return e;
  return run_residual(L, true);
}

cudaError_t run_stage(const Launch &L, int stage, bool rk, bool eig) {
  return launch_stage(L, stage, rk, eig);
}

// Pieces of one Euler step for nuc3d_solve_host's slab pipeline; together they launch
// exactly the kernels of one_step over the same tiles (the same results):
//   stage-0 slab s (BC of k0 <= k < k1; xi and eta over the slab's tiles, xi reducing the
//   eigenvalue maximum) for every slab; then, per slab, the zeta sweep of stage 0 and
//   stages 1 and 2 (BC, xi, eta, zeta over the slab's tiles) in any order that runs a
//   slab's stage-s zeta sweep after the stage-(s-1) zeta sweeps of the slab and of the
//   slabs whose cells its stencils reach; then the residual.
static TileMap tile_part(TileMap tm, int t0, int t1) {
  tm.base = t0;
  tm.end = t1;
  return tm;
}
cudaError_t run_stage0_slab(const Launch &L, int k0, int k1, int tx0, int tx1, int ty0, int ty1) {
  cudaError_t e = run_bc(L, 0, k0, k1);
  if (e != cudaSuccess) return e;
  Launch P = L;
  P.tm_dir[0] = tile_part(L.tm_dir[0], tx0, tx1);
  if ((e = launch_sweep<0>(P, 0, SW_EIG)) != cudaSuccess) return e;
  P.tm_dir[1] = tile_part(L.tm_dir[1], ty0, ty1);
  return launch_sweep<1>(P, 0, 0);
}
// Stage 0's zeta sweep over the zeta tiles tz0 <= t < tz1 (every cell's eigenvalue must be
// in the maximum: the stage fixes dt from it).
cudaError_t run_stage0_zeta(const Launch &L, int tz0, int tz1) {
  Launch P = L;
  P.tm_dir[2] = tile_part(L.tm_dir[2], tz0, tz1);
  return launch_sweep<2>(P, 0, SW_RK);
}
// Stage 1 or 2 of one z-slab: BC, xi and eta over the slab's tiles, then zeta over its
// z-chunks (zeta reads the slab's own RHS and the stage state of its cells and of the
// neighbouring slabs' planes its stencils reach).
cudaError_t run_stage_slab(const Launch &L, int stage, int k0, int k1, int tx0, int tx1, int ty0, int ty1,
                           int tz0, int tz1) {
  cudaError_t e = run_bc(L, stage, k0, k1);
  if (e != cudaSuccess) return e;
  Launch P = L;
  P.tm_dir[0] = tile_part(L.tm_dir[0], tx0, tx1);
  P.tm_dir[1] = tile_part(L.tm_dir[1], ty0, ty1);
  P.tm_dir[2] = tile_part(L.tm_dir[2], tz0, tz1);
  if ((e = launch_sweep<0>(P, stage, 0)) != cudaSuccess) return e;
  if ((e = launch_sweep<1>(P, stage, 0)) != cudaSuccess) return e;
  return launch_sweep<2>(P, stage, SW_RK | (stage == 2 && L.d_res_last ? SW_RES : 0));
}

// Stage 1 or 2 split by blocks, for nuc3d_solve_host's multi-block pipeline: run_stage_pre
// (the ghost fluxes of every physical face; Navier-Stokes: primitives and gradients of
// every block), then run_stage_sweeps over the blocks b0 <= b < b1 in any order (their
// tiles of each direction's map; a block's sweeps read its neighbours' stage state and
// viscous fluxes, which the stage before and run_stage_pre complete).  Together: the
// kernels of launch_stage over the same tiles, without the residual.
cudaError_t run_stage_pre(const Launch &L, int stage) {
  cudaError_t e = run_bc(L, stage, 0, 0x7fffffff);
  if (e != cudaSuccess || L.P.model != MODEL_NS) return e;
  const int nt = L.tm_cells.tile_start[L.tm_cells.nblocks];
  prim_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, L.tm_cells, L.P, L.d_state, stage);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  grad_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, L.tm_cells, L.P);
  return cudaGetLastError();
}
cudaError_t run_stage_sweeps(const Launch &L, int stage, int b0, int b1) {
  Launch P = L;
  for (int d = 0; d < 3; ++d)
    P.tm_dir[d] = tile_part(L.tm_dir[d], L.tm_dir[d].tile_start[b0], L.tm_dir[d].tile_start[b1]);
  const int nsf = L.P.model == MODEL_NS ? SW_NS : 0;
  cudaError_t e;
  if ((e = launch_sweep<0>(P, stage, nsf)) != cudaSuccess) return e;
  if ((e = launch_sweep<1>(P, stage, nsf)) != cudaSuccess) return e;
  return launch_sweep<2>(P, stage, nsf | SW_RK | (stage == 2 && L.d_res_last ? SW_RES : 0));
}

cudaError_t run_bc(const Launch &L, int stage, int k0, int k1) {
  if (L.bc_tiles <= 0) return cudaSuccess;
  bc_ghost_kernel<<<L.bc_tiles, 256, 0, L.stream>>>(L.d_blocks, L.d_jobs, L.P, L.d_state, stage, k0, k1);
  return cudaGetLastError();
}

cudaError_t run_metrics(const double *x, const double *y, const double *z, const int n[3],
                        double *jac, double *met, double *dxyz, unsigned *bad, cudaStream_t st) {
  const long long N = (long long)n[0] * n[1] * n[2];
  metrics_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(x, y, z, n[0], n[1], n[2], jac, met,
                                                              dxyz, bad);
  return cudaGetLastError();
}

template <int DIR, int SHP>
inline cudaError_t launch_sensor_data(const Launch &L, float *feat, unsigned char *label,
                                      long long *where, unsigned long long *count,
                                      unsigned long long cap) {
  const int nt = L.tm_dir[DIR].tile_start[L.tm_dir[DIR].nblocks];
  using M = TileSmem<DIR, SCH_WENO5Z, SHP>;
  const size_t smem = (size_t)12 * M::TW * M::SP * sizeof(double);
  sensor_data_kernel<DIR, SHP><<<nt, kThreads, smem, L.stream>>>(L.d_blocks, L.tm_dir[DIR], L.P,
                                                                  L.d_state, 0, feat, label,
                                                                  where, count, cap);
  return cudaGetLastError();
}

template <int DIR>
inline cudaError_t launch_sensor_data_d(const Launch &L, float *feat, unsigned char *label,
                                        long long *where, unsigned long long *count,
                                        unsigned long long cap) {
  switch (L.shape[DIR]) {
    case 0: return launch_sensor_data<DIR, 0>(L, feat, label, where, count, cap);
    case 1: return launch_sensor_data<DIR, 1>(L, feat, label, where, count, cap);
    case 2: return launch_sensor_data<DIR, 2>(L, feat, label, where, count, cap);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t run_sensor_data(const Launch &L, int dir, float *feat, unsigned char *label,
                            long long *where, unsigned long long *count, unsigned long long cap) {
  if (L.P.scheme[dir] != SCH_WENO5Z) return cudaErrorInvalidValue;
  if (dir == 0) return launch_sensor_data_d<0>(L, feat, label, where, count, cap);
  if (dir == 1) return launch_sensor_data_d<1>(L, feat, label, where, count, cap);
  return launch_sensor_data_d<2>(L, feat, label, where, count, cap);
}

cudaError_t run_diag(const Launch &L, const DiagDev *dd, double *sums, double *parts) {
  const int nt = L.tm_cells.tile_start[L.tm_cells.nblocks];
  const int nb = L.tm_cells.nblocks;
  diag_prim_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, dd, L.tm_cells, L.P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  diag_kernel<<<nt, kCellTile, 0, L.stream>>>(L.d_blocks, dd, L.tm_cells, L.P);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
#if NUC3D_FAST
  diag_sum_part_kernel<<<dim3(kDiagParts, nb), 256, 0, L.stream>>>(L.d_blocks, dd, parts);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  diag_sum_parts_kernel<<<(2 * nb + 127) / 128, 128, 0, L.stream>>>(nb, parts, sums);
#else
  (void)parts;
  diag_sum_seq_kernel<<<nb, 256, 0, L.stream>>>(L.d_blocks, dd, sums);
#endif
  return cudaGetLastError();
}

cudaError_t run_sweep(const Launch &L, int dir, int stage, int flags) {
  const int f = flags | (L.P.model == MODEL_NS ? SW_NS : 0);
  if (L.bc_tiles > 0) {
    bc_ghost_kernel<<<L.bc_tiles, 256, 0, L.stream>>>(L.d_blocks, L.d_jobs, L.P, L.d_state, stage);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (dir == 0) return launch_sweep<0>(L, stage, f);
  if (dir == 1) return launch_sweep<1>(L, stage, f);
  return launch_sweep<2>(L, stage, f & ~SW_RK);
}

template <int DIR, int SCH, int SHP>
inline cudaError_t configure_s() {
#if NUC3D_FAST
  if constexpr (SCH == SCH_WENO5Z) {
    const size_t he = hybrid_smem_bytes<DIR, SCH, SHP>(false), hn = hybrid_smem_bytes<DIR, SCH, SHP>(true);
    const cudaError_t e = cudaFuncSetAttribute(sweep_kernel<DIR, SCH, true, SHP>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(he > hn ? he : hn));
    if (e != cudaSuccess) return e;
  }
#endif
  constexpr size_t euler = sweep_smem_bytes<DIR, SCH, SHP>(false) + rhs_stage_bytes<DIR>(false);
  constexpr size_t ns = sweep_smem_bytes<DIR, SCH, SHP>(true) + rhs_stage_bytes<DIR>(true);
  // every dynamic shared-memory request below fits what a CTA may opt in to
  static_assert(euler <= kSmemOptin && ns <= kSmemOptin, "sweep tile fits");
  static_assert(PipeSmem<DIR, SCH, SHP>::TOTAL <= kSmemOptin, "pipelined tile fits");
  static_assert(hybrid_smem_bytes<DIR, SCH, SHP>(true) <= kSmemOptin, "hybrid tile fits");
  cudaError_t e = cudaFuncSetAttribute(pipe_sweep_kernel<DIR, SCH, SHP>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PipeSmem<DIR, SCH, SHP>::TOTAL);
  if (e != cudaSuccess) return e;
  static_assert(PipeSmem<DIR, SCH, SHP, true>::TOTAL <= kSmemOptin, "NS pipelined tile fits");
  e = cudaFuncSetAttribute(pipe_sweep_kernel<DIR, SCH, SHP, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)PipeSmem<DIR, SCH, SHP, true>::TOTAL);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sweep_kernel<DIR, SCH, false, SHP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(euler > ns ? euler : ns));
}

template <int DIR, int SCH>
inline cudaError_t configure_t() {
  cudaError_t e;
  if ((e = configure_s<DIR, SCH, 0>()) != cudaSuccess) return e;
  if ((e = configure_s<DIR, SCH, 1>()) != cudaSuccess) return e;
  return configure_s<DIR, SCH, 2>();
}

template <int DIR, int SCH>
inline cudaError_t configure_compact_t() {
  cudaError_t e = cudaFuncSetAttribute(compact_rows_kernel<DIR, SCH>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)compact_rows_smem_bytes<DIR, SCH>());
  if (e != cudaSuccess) return e;
  if constexpr (SCH == SCH_HCCS) {
    e = cudaFuncSetAttribute(compact_rows_kernel<DIR, SCH, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)compact_rows_smem_bytes<DIR, SCH>());
    if (e != cudaSuccess) return e;
  }
#if NUC3D_FAST
  static_assert(compact_line_smem_bytes<DIR, SCH>(false) <= kSmemOptin, "Euler line tile fits");
  static_assert(compact_rows_smem_bytes<DIR, SCH>() <= kSmemOptin &&
                compact_finish_smem_bytes<DIR, SCH>(true) <= kSmemOptin, "compact tiles fit");
  // (a Navier-Stokes tile of kLineLanes lines may not fit: compact_line_smem tells the host)
  e = cudaFuncSetAttribute(compact_line_kernel<DIR, SCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)std::min<size_t>(compact_line_smem_bytes<DIR, SCH>(true), kSmemOptin));
  if (e != cudaSuccess) return e;
#endif
  return cudaFuncSetAttribute(compact_finish_kernel<DIR, SCH>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)compact_finish_smem_bytes<DIR, SCH>(true));
}

template <int DIR>
inline cudaError_t configure_dir() {
  cudaError_t e;
  if ((e = configure_t<DIR, SCH_WENO5JS>()) != cudaSuccess) return e;
  if ((e = configure_t<DIR, SCH_WENO5Z>()) != cudaSuccess) return e;
  if ((e = configure_compact_t<DIR, SCH_CRWENO5>()) != cudaSuccess) return e;
  if ((e = configure_compact_t<DIR, SCH_HCCS>()) != cudaSuccess) return e;
  if ((e = configure_t<DIR, SCH_WENO3JS>()) != cudaSuccess) return e;
  if ((e = configure_t<DIR, SCH_UPWIND1>()) != cudaSuccess) return e;
  return configure_t<DIR, SCH_WENO7JS>();
}

cudaError_t configure() {
  cudaError_t e;
  if ((e = configure_dir<0>()) != cudaSuccess) return e;
  if ((e = configure_dir<1>()) != cudaSuccess) return e;
  return configure_dir<2>();
}

// ---------------------------------------------------------------------------------
// Debug taps: the inviscid intermediates of one right-hand side at the current state,
// in the reference's EulerFlux layouts (src/euler3d.cpp:12-20, :62-83): per direction the
// split fluxes FluxL/FluxR (cells), the reconstructions reconstFluxL/R (faces) and the
// difference dfdxi/dgdeta/dhdzeta (cells), each stored line position fastest, then
// (xi: j, k; eta: k, i; zeta: i, j).  Explicit schemes: the reconstructions of the
// reference-order switch (recon_pos / recon_neg); compact schemes: the three-kernel
// path's face values (fh).
// ---------------------------------------------------------------------------------
template <int DIR>
__device__ __forceinline__ long long tap_index(int pos, int w, int o, int len, const Geo &G) {
  return DIR == 1 ? pos + (long long)len * (o + (long long)G.nO * w)
                  : pos + (long long)len * (w + (long long)G.nW * o);
}

template <int DIR, int SCH, int SHP, bool FACES>
__global__ void __launch_bounds__(kThreads)
tap_kernel(const BlockDev *__restrict__ blocks, TileMap tm, SolverParams P, int want, double *fl,
           double *fr, double *rl, double *rr, double *df) {
  using M = TileSmem<DIR, SCH, SHP>;
  constexpr int R = M::R, TW = M::TW, TL = M::TL, SP = M::SP, SH = M::SH;
  extern __shared__ double smem[];
  double *sF = smem;               // [10][TW][SP]
  double *sH = sF + 10 * TW * SP;  // [5][TW][SH]
  const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P);
  if (T.b != want) return;  // the same for the whole CTA
  unsigned st = 0;
  double emax = 0.0;
  phase_split<DIR, SCH, false, SHP>(blocks, T, P, 0, false, sF, nullptr, st, emax);
  __syncthreads();
  const Geo &G = T.G;
  const long long N = T.N, NF = (long long)(G.L + 1) * G.nW * G.nO;
  for (int e = threadIdx.x; e < TW * TL; e += kThreads) {
    const int c = e % TL, w = e / TL;
    if (w >= T.nw || c >= T.cl) continue;
    const long long i = tap_index<DIR>(T.c0 + c, T.w0 + w, T.o, G.L, G);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      fl[v * N + i] = sF[(v * TW + w) * SP + R + c];
      fr[v * N + i] = sF[((5 + v) * TW + w) * SP + R + c];
    }
  }
  if constexpr (FACES) {
    const bool compat = P.weno5z_compat != 0;
    for (int e = threadIdx.x; e < TW * (TL + 1); e += kThreads) {
      const int fc = e % (TL + 1), w = e / (TL + 1);
      if (w >= T.nw || fc > T.cl) continue;
      const int f = T.c0 + fc;
      const long long i = tap_index<DIR>(f, T.w0 + w, T.o, G.L + 1, G);
      for (int v = 0; v < 5; ++v) {
        const double *rowP = sF + (v * TW + w) * SP + (R - T.c0);
        const double *rowN = sF + ((5 + v) * TW + w) * SP + (R - T.c0);
        auto Pacc = [rowP](int cc) { return rowP[cc]; };
        auto Nacc = [rowN](int cc) { return rowN[cc]; };
        const double hp = recon_pos<SCH>(f, G.L, T.ts, T.physL, T.physR, compat, Pacc);
        const double hn = recon_neg<SCH>(f, G.L, T.ts, T.physL, T.physR, Nacc);
        rl[v * NF + i] = hp;
        rr[v * NF + i] = hn;
        sH[(v * TW + w) * SH + fc] = hp + hn;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TW * TL; e += kThreads) {
      const int c = e % TL, w = e / TL;
      if (w >= T.nw || c >= T.cl) continue;
      const long long i = tap_index<DIR>(T.c0 + c, T.w0 + w, T.o, G.L, G);
#pragma unroll
      for (int v = 0; v < 5; ++v) df[v * N + i] = sH[(v * TW + w) * SH + c + 1] - sH[(v * TW + w) * SH + c];
    }
  }
}

// Compact directions: face values of one block from fh (compact_rows + compact_thomas).
template <int DIR>
__global__ void __launch_bounds__(256)
tap_fh_kernel(const BlockDev *__restrict__ blocks, int want, double *rl, double *rr, double *df) {
  const BlockDev &B = blocks[want];
  const int n[3] = {B.n[0], B.n[1], B.n[2]};
  const Geo G = make_geo(DIR, n);
  const long long nl = (long long)G.nW * G.nO, NF = (long long)(G.L + 1) * nl;
  const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
  if (t >= 5 * nl) return;
  const int v = (int)(t / nl);
  const long long line = t - v * nl;
  const int w = (int)(line % G.nW), o = (int)(line / G.nW);
  const double *hp = B.fh + ((2 * v) * nl + line) * (G.L + 1);
  const double *hn = B.fh + ((2 * v + 1) * nl + line) * (G.L + 1);
  double prev = 0.0;
  for (int f = 0; f <= G.L; ++f) {
    const long long i = tap_index<DIR>(f, w, o, G.L + 1, G);
    rl[v * NF + i] = hp[f];
    rr[v * NF + i] = hn[f];
    const double h = hp[f] + hn[f];
    if (f > 0) df[v * B.N + tap_index<DIR>(f - 1, w, o, G.L, G)] = h - prev;
    prev = h;
  }
}

template <int DIR, int SCH, int SHP, bool FACES>
inline cudaError_t launch_tap(const Launch &L, int block, double *const out[5]) {
  using M = TileSmem<DIR, SCH, SHP>;
  const size_t smem = ((size_t)10 * M::TW * M::SP + (size_t)5 * M::TW * M::SH) * sizeof(double);
  const int ntiles = L.tm_dir[DIR].tile_start[L.tm_dir[DIR].nblocks];
  tap_kernel<DIR, SCH, SHP, FACES><<<ntiles, kThreads, smem, L.stream>>>(
      L.d_blocks, L.tm_dir[DIR], L.P, block, out[0], out[1], out[2], out[3], out[4]);
  return cudaGetLastError();
}

template <int DIR, int SCH, bool FACES>
inline cudaError_t launch_tap_s(const Launch &L, int block, double *const out[5]) {
  switch (L.shape[DIR]) {
    case 0: return launch_tap<DIR, SCH, 0, FACES>(L, block, out);
    case 1: return launch_tap<DIR, SCH, 1, FACES>(L, block, out);
    case 2: return launch_tap<DIR, SCH, 2, FACES>(L, block, out);
    default: return cudaErrorInvalidValue;
  }
}

template <int DIR, int SCH, bool WHOLE>
inline cudaError_t launch_tap_compact(const Launch &L, int block, const int nl, double *const out[5]) {
  cudaError_t e = launch_tap_s<DIR, SCH, false>(L, block, out);
  if (e != cudaSuccess) return e;
  const int ntiles = L.tm_dir[DIR].tile_start[L.tm_dir[DIR].nblocks];
  compact_rows_kernel<DIR, SCH, WHOLE><<<ntiles, kThreads, compact_rows_smem_bytes<DIR, SCH>(), L.stream>>>(
      L.d_blocks, L.tm_dir[DIR], L.P, L.d_state, 0, 0);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int nsys = L.tm_sys[DIR].tile_start[L.tm_sys[DIR].nblocks];
  compact_thomas_kernel<DIR><<<nsys, 256, 0, L.stream>>>(L.d_blocks, L.tm_sys[DIR], L.P,
                                                         WHOLE ? 0 : L.P.ts[DIR]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  tap_fh_kernel<DIR><<<(5 * nl + 255) / 256, 256, 0, L.stream>>>(L.d_blocks, block, out[2], out[3], out[4]);
  return cudaGetLastError();
}

template <int DIR>
inline cudaError_t run_taps_d(const Launch &L, int block, int nl, double *const out[5]) {
  switch (L.P.scheme[DIR]) {
    case SCH_WENO5JS: return launch_tap_s<DIR, SCH_WENO5JS, true>(L, block, out);
    case SCH_WENO5Z: return launch_tap_s<DIR, SCH_WENO5Z, true>(L, block, out);
    case SCH_WENO7JS: return launch_tap_s<DIR, SCH_WENO7JS, true>(L, block, out);
    case SCH_WENO3JS: return launch_tap_s<DIR, SCH_WENO3JS, true>(L, block, out);
    case SCH_UPWIND1: return launch_tap_s<DIR, SCH_UPWIND1, true>(L, block, out);
    case SCH_CRWENO5: return launch_tap_compact<DIR, SCH_CRWENO5, false>(L, block, nl, out);
    case SCH_HCCS: return launch_tap_compact<DIR, SCH_HCCS, false>(L, block, nl, out);
    case SCH_HCCS77: return launch_tap_compact<DIR, SCH_HCCS, true>(L, block, nl, out);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t run_taps(const Launch &L, int block, int dir, int nl, double *const out[5]) {
  if (L.bc_tiles > 0) {  // the physical faces' ghost fluxes at the current state
    bc_ghost_kernel<<<L.bc_tiles, 256, 0, L.stream>>>(L.d_blocks, L.d_jobs, L.P, L.d_state, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (dir == 0) return run_taps_d<0>(L, block, nl, out);
  if (dir == 1) return run_taps_d<1>(L, block, nl, out);
  return run_taps_d<2>(L, block, nl, out);
}

int tile_count(int dir, const int n[3], int shape) { return sweep_tiles(dir, n, shape); }

size_t compact_line_smem(int dir, int sch, bool ns) {
#if NUC3D_FAST
  if (sch != SCH_CRWENO5 && sch != SCH_HCCS) return 0;
  const bool c = sch == SCH_CRWENO5;
  if (dir == 0) return c ? compact_line_smem_bytes<0, SCH_CRWENO5>(ns) : compact_line_smem_bytes<0, SCH_HCCS>(ns);
  if (dir == 1) return c ? compact_line_smem_bytes<1, SCH_CRWENO5>(ns) : compact_line_smem_bytes<1, SCH_HCCS>(ns);
  return c ? compact_line_smem_bytes<2, SCH_CRWENO5>(ns) : compact_line_smem_bytes<2, SCH_HCCS>(ns);
#else
  (void)dir; (void)sch; (void)ns;
  return 0;
#endif
}

}  // namespace NUC3D_NS
}  // namespace nuc3d
