// sweep_pipe.cuh -- the explicit-scheme sweep as a persistent, warp-specialised kernel fed
// by the Tensor Memory Accelerator (included by kernels.cuh inside its namespace).
//
// Same arithmetic as sweep_kernel (phases split -> faces -> cells, the reference's
// operations: src/physicsModel.cpp:420-760, src/euler3d.cpp:305-366, :143-241, :368-427,
// src/TVD-RK3.cpp:16-137), different data movement:
//   * Each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ... (two CTAs per SM).
//   * Warp kProdWarp is the producer.  For tile k+2 it issues cp.async.bulk.tensor loads
//     of the tile's state Q (5 components), Jacobian and metric, halo included, into one
//     of two shared-memory slots, completing on an mbarrier with a transaction count; its
//     32 lanes also gather the cells across block faces (neighbour blocks, raw-slab
//     mapping of ghost_cell, or the BC ghost flux) into the slot with plain loads.  For
//     tile k+1 it loads the right-hand side the eta/zeta sweeps add to and, for the zeta
//     sweep's RK update at stages 1 and 2, the state u_n, into a third buffer.
//   * Warps 0..8 (kThreads = 288 threads) consume: split fluxes from the slot, faces,
//     cells; then they release the slot (mbarrier arrive) so the producer refills it.
// The consumers never wait on global memory: the loads of tile k+1 and k+2 run while tile
// k is computed.  Tensor maps are over this GPU's own arrays, plain tile mode, no
// multicast.  Every mbarrier wait gives up after kPipeWaitNs of %globaltimer and sets
// ST_PIPE_TIMEOUT: the consumers then skip their later waits (still meeting at every named
// barrier), the producer stops issuing, and it waits (bounded the same way) for the copies
// it issued before it returns.

#ifndef NUC3D_PIPE_FACE_UNROLL
#define NUC3D_PIPE_FACE_UNROLL 5  // variables per iteration of the face loop (5: 2-3% faster than 1 or 2)
#endif
constexpr int kPipeFaceUnroll = NUC3D_PIPE_FACE_UNROLL;
constexpr int kProdWarp = kThreads / 32;         // warp index of the producer
constexpr int kPipeThreads = kThreads + 32;      // 288 consumers + one producer warp
constexpr unsigned long long kPipeWaitNs = 2000000000ull;  // 2 s

// Tensor maps of one block for one direction (maps[(block * 3 + dir) * PM_COUNT + kind]).
enum PipeMap : int {
  PM_Q0 = 0, PM_Q1 = 1, PM_Q2 = 2,  // state q[s]: halo box, 5 components
  PM_JAC = 3,                       // Jacobian: halo box
  PM_MET = 4,                       // the direction's metric: halo box, 3 components
  PM_METO = 5,                      // the eta and zeta metrics (components 3..8): own cells
                                    // (the xi sweep's eigenvalue maximum, stage 0)
  PM_RHS = 6,                       // right-hand side: the tile's own cells, 5 components
  PM_QN = 7,                        // q[0] (u_n): own cells, 5 components
  PM_COUNT = 8
};

// Compile-time geometry of a pipelined sweep tile.
template <int DIR, int SCH, int SHP> struct PipeGeo {
  static constexpr int R = Halo<SCH>::R, TW = Tile<SHP>::TW, TL = Tile<SHP>::TL;
  static_assert(R == scheme_halo(SCH), "the host encodes the boxes with scheme_halo");
  static constexpr int NP = TL + 2 * R;  // split positions per line
  static constexpr int RA = pipe_ra(R);  // xi: the halo box starts RA cells before the tile
  // halo box extents (x, y, z), as pipe_box gives them to the host's tensor maps
  static constexpr int BX = DIR == 0 ? ((TL + R + RA + 1) & ~1) : TW;
  static constexpr int BY = DIR == 0 ? TW : (DIR == 1 ? NP : 1);
  static constexpr int BZ = DIR == 2 ? NP : 1;
  static constexpr int BOX = BX * BY * BZ;
  static constexpr int OWN = TL * TW;
  static constexpr int NG = 2 * R * TW;  // ghost positions: R at each line end, per lane
  __device__ static int hidx(int p, int w) { return DIR == 0 ? w * BX + (p - R + RA) : p * TW + w; }
  __device__ static int oidx(int c, int w) { return DIR == 0 ? w * TL + c : c * TW + w; }
};

__host__ __device__ constexpr size_t align128(size_t x) { return (x + 127) & ~size_t(127); }

// Shared-memory carve-up of the pipelined sweep (byte offsets from a 128-byte aligned base).
template <int DIR, int SCH, int SHP, bool NSV = false> struct PipeSmem {
  using G = PipeGeo<DIR, SCH, SHP>;
  using M = TileSmem<DIR, SCH, SHP>;
  // one slot: state, Jacobian and direction metric over the halo box, [xi] the other two
  // directions' metrics of the own cells, ghosts, [zeta] u_i's energy after the reset
  static constexpr size_t Q = 0;
  static constexpr size_t J = Q + align128((size_t)5 * G::BOX * 8);
  static constexpr size_t MET = J + align128((size_t)G::BOX * 8);
  static constexpr size_t METO = MET + align128((size_t)3 * G::BOX * 8);  // [6][OWN]
  static constexpr size_t GH = METO + (DIR == 0 ? align128((size_t)6 * G::OWN * 8) : 0);  // [NG][9]
  static constexpr size_t GT = GH + align128((size_t)G::NG * 9 * 8);     // ghost types [NG]
  static constexpr size_t Q4 = GT + align128((size_t)G::NG * 4);         // [OWN]
  static constexpr size_t SLOT = Q4 + (DIR == 2 ? align128((size_t)G::OWN * 8) : 0);
  // single buffer: [eta, zeta] the right-hand side to add to, [zeta] u_n
  static constexpr size_t RHS = 2 * SLOT;                                                // [5][OWN]
  static constexpr size_t QN = RHS + (DIR != 0 ? align128((size_t)5 * G::OWN * 8) : 0);  // [5][OWN]
  static constexpr size_t F = QN + (DIR == 2 ? align128((size_t)5 * G::OWN * 8) : 0);
  static constexpr size_t H = F + align128((size_t)10 * G::TW * M::SP * 8);
  static constexpr size_t V = H + align128((size_t)5 * G::TW * M::SH * 8);    // NS: [4][TW][SV]
  static constexpr size_t RED = V + (NSV ? align128((size_t)4 * G::TW * M::SV * 8) : 0);  // [kThreads / 32]
  static constexpr size_t BAR = RED + align128((size_t)(kThreads / 32) * 8);  // 5 mbarriers
  static constexpr size_t TOTAL = BAR + 64;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  unsigned long long st;
  asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(st) : "r"(smem_u32(b)) : "memory");
  (void)st;
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *b, unsigned bytes) {
  unsigned long long st;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
               : "=l"(st) : "r"(smem_u32(b)), "r"(bytes) : "memory");
  (void)st;
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P;\n}" : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase of parity `parity` of mbarrier b; false if it did not complete
// within kPipeWaitNs.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 0 && global_ns() - t0 > kPipeWaitNs) return false;
  }
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            int c, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(c),
      "r"(smem_u32(bar))
      : "memory");
}
// Barrier of the consumer warps only (the producer warp does not take part).
__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory");
}

// Box origin (x, y, z) of a tile's halo box or own box.
template <int DIR, int SCH, int SHP>
__device__ __forceinline__ void pipe_origin(const TileCtx &T, bool halo, int &x, int &y, int &z) {
  using G = PipeGeo<DIR, SCH, SHP>;
  const int c = halo ? T.c0 - (DIR == 0 ? G::RA : G::R) : T.c0;
  if (DIR == 0) { x = c; y = T.w0; z = T.o; }
  else if (DIR == 1) { x = T.w0; y = c; z = T.o; }
  else { x = T.w0; y = T.o; z = c; }
}

// The producer's gather of a tile's positions across block faces (g < 0 or g >= L), the
// data phase_split takes from ghost_cell / the BC ghost slab: per ghost position the
// neighbour cell's Q (5), Jacobian and direction metric (3), type 1; or the BC ghost flux
// (F+ left of the block, type 2; F- right, type 3); type 0 contributes zero fluxes.
template <int DIR, int SCH, int SHP>
__device__ __forceinline__ void pipe_gather(const BlockDev *__restrict__ blocks, const TileCtx &T,
                                            const SolverParams &P, int stage, double *gh, int *gt,
                                            int lane) {
  using G = PipeGeo<DIR, SCH, SHP>;
  constexpr int R = G::R, TW = G::TW;
  const BlockDev &B = *T.B;
  const int L = T.G.L;
  const bool lo = T.c0 - R < 0, hi = T.c0 + T.cl + R > L;
  if (!lo && !hi) return;
  for (int it = lane; it < G::NG; it += 32) {
    const int gp = it / TW, w = it - gp * TW;
    const int g = gp < R ? gp - R : L + (gp - R);
    int type = 0;
    double *o = gh + it * 9;
    const bool used = w < T.nw && ((gp < R && lo) || (gp >= R && hi)) && g >= T.c0 - R &&
                      g < T.c0 + T.cl + R;
    if (used) {
      const int wl = T.w0 + w;
      const int sa = (DIR == 1) ? T.o : wl, sb = (DIR == 1) ? wl : T.o;
      long long nidx;
      const int nb = ghost_cell(blocks, B, DIR, g, sa, sb, P.bfs, nidx);
      if (nb >= 0) {
        const BlockDev &NB = blocks[nb];
        const long long NN = NB.N;
        const double *q = NB.q[stage];
#pragma unroll
        for (int v = 0; v < 5; ++v) o[v] = __ldg(q + v * NN + nidx);
        o[5] = __ldg(NB.jac + nidx);
        const double *m = NB.met[DIR];
#pragma unroll
        for (int k = 0; k < 3; ++k) o[6 + k] = __ldg(m + k * NN + nidx);
        type = 1;
      } else if (g == -1 || g == L) {
        const int f = 2 * DIR + (g < 0 ? 0 : 1);
        const int A = DIR == 0 ? T.n[1] : (DIR == 1 ? T.n[2] : T.n[0]);
        const long long area = (long long)A * (DIR == 0 ? T.n[2] : (DIR == 1 ? T.n[0] : T.n[1]));
        const double *ghs = B.ghost + B.goff[f] + (sa + (long long)A * sb);
#pragma unroll
        for (int v = 0; v < 5; ++v) o[v] = __ldg(ghs + v * area);
        type = g < 0 ? 2 : 3;
      }
    }
    gt[it] = type;
  }
}

// NSV: the Navier-Stokes sweep: the consumers also load the direction's viscous fluxes
// (phase_vis, plain loads) and phase 3 applies the viscous differences as sweep_kernel does.
template <int DIR, int SCH, int SHP, bool NSV = false>
__global__ void __launch_bounds__(kPipeThreads, 2)
pipe_sweep_kernel(const BlockDev *__restrict__ blocks, const CUtensorMap *__restrict__ maps,
                  TileMap tm, SolverParams P, StepState *S, int stage, int flags) {
  using G = PipeGeo<DIR, SCH, SHP>;
  using M = TileSmem<DIR, SCH, SHP>;
  using L = PipeSmem<DIR, SCH, SHP, NSV>;
  constexpr int R = G::R, TW = G::TW, TL = G::TL, NP = G::NP, SP = M::SP, SH = M::SH, SV = M::SV;
  extern __shared__ __align__(128) unsigned char psm[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(psm + L::BAR);
  unsigned long long *full_q = bar, *done = bar + 2, *full_r = bar + 4;
  double *sF = reinterpret_cast<double *>(psm + L::F);
  double *sH = reinterpret_cast<double *>(psm + L::H);
  double *sRed = reinterpret_cast<double *>(psm + L::RED);
  double *rbuf = reinterpret_cast<double *>(psm + L::RHS);
  double *nbuf = reinterpret_cast<double *>(psm + L::QN);
  double *sV = reinterpret_cast<double *>(psm + L::V);  // NSV only

  const bool eig = DIR == 0 && (flags & SW_EIG) != 0;
  const bool rk = (flags & SW_RK) != 0;
  const bool need_r = DIR != 0;                      // RHS read (eta += , zeta +=)
  const bool need_n = DIR == 2 && rk && stage != 0;  // u_n read (RK stages 1, 2)
  const int ntile = tile_range(tm);  // tiles tm.base .. tm.base + ntile - 1
  const int nmine = (int)blockIdx.x < ntile ? (ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int tid = threadIdx.x;
  // The tensor copies need 128-byte aligned shared-memory destinations; every offset above
  // is a multiple of 128 from the dynamic shared-memory base, which must be too.
  if (smem_u32(psm) & 127u) {
    if (tid == 0) atomicOr(&S->status, ST_BAD_LAUNCH);
    return;
  }

  if (tid == 0) {
    mbar_init(&full_q[0], 32);
    mbar_init(&full_q[1], 32);
    mbar_init(&done[0], kThreads / 32);
    mbar_init(&done[1], kThreads / 32);
    mbar_init(&full_r[0], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (tid >= kThreads) {
    // ---------------- producer warp ----------------
    const int lane = tid & 31;
    const unsigned qbytes = (unsigned)((5 + 1 + 3) * G::BOX * 8 + (eig ? 6 * G::OWN * 8 : 0));
    const unsigned rbytes = (unsigned)((need_r ? 5 : 0) * G::OWN * 8 + (need_n ? 5 : 0) * G::OWN * 8);
    unsigned nq[2] = {0, 0}, nr = 0;  // phases armed per barrier
    bool ok = true;
    auto issue_q = [&](int k, int s) {
      const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P, tm.base + (int)blockIdx.x + k * (int)gridDim.x);
      unsigned char *slot = psm + s * L::SLOT;
      const CUtensorMap *mp = maps + ((size_t)T.b * 3 + DIR) * PM_COUNT;
      if (lane == 0) {
        mbar_expect_tx(&full_q[s], qbytes);
        int x, y, z;
        pipe_origin<DIR, SCH, SHP>(T, true, x, y, z);
        tma_load_4d(slot + L::Q, mp + PM_Q0 + stage, x, y, z, 0, &full_q[s]);
        tma_load_3d(slot + L::J, mp + PM_JAC, x, y, z, &full_q[s]);
        tma_load_4d(slot + L::MET, mp + PM_MET, x, y, z, 3 * DIR, &full_q[s]);
        if (eig) {
          pipe_origin<DIR, SCH, SHP>(T, false, x, y, z);
          tma_load_4d(slot + L::METO, mp + PM_METO, x, y, z, 3, &full_q[s]);
        }
      }
      pipe_gather<DIR, SCH, SHP>(blocks, T, P, stage, reinterpret_cast<double *>(slot + L::GH),
                                 reinterpret_cast<int *>(slot + L::GT), lane);
      __syncwarp();
      mbar_arrive(&full_q[s]);
      ++nq[s];
    };
    auto issue_r = [&](int k) {
      if (lane == 0) {
        const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P, tm.base + (int)blockIdx.x + k * (int)gridDim.x);
        const CUtensorMap *mp = maps + ((size_t)T.b * 3 + DIR) * PM_COUNT;
        int x, y, z;
        pipe_origin<DIR, SCH, SHP>(T, false, x, y, z);
        mbar_arrive_tx(&full_r[0], rbytes);  // one arrival (this one) plus the transaction bytes
        if (need_r) tma_load_4d(rbuf, mp + PM_RHS, x, y, z, 0, &full_r[0]);
        if (need_n) tma_load_4d(nbuf, mp + PM_QN, x, y, z, 0, &full_r[0]);
      }
      ++nr;
    };
    if (nmine > 0) issue_q(0, 0);
    if (nmine > 1) issue_q(1, 1);
    if (nmine > 0 && (need_r || need_n)) issue_r(0);
    for (int k = 0; k < nmine; ++k) {
      ok = mbar_wait(&done[k & 1], (unsigned)((k >> 1) & 1));
      if (!ok) break;
      if (k + 1 < nmine && (need_r || need_n)) issue_r(k + 1);
      if (k + 2 < nmine) issue_q(k + 2, k & 1);
    }
    if (!ok && lane == 0) atomicOr(&S->status, ST_PIPE_TIMEOUT);
    // before the CTA exits, every copy issued into its shared memory must have landed
    // (the consumers waited for them, unless a wait gave up): bounded waits
    for (int s = 0; s < 2; ++s)
      if (nq[s]) mbar_wait(&full_q[s], (nq[s] - 1) & 1);
    if (nr) mbar_wait(&full_r[0], (nr - 1) & 1);
    return;
  }

  // ---------------- consumer warps ----------------
  unsigned st = 0, nres = 0;
  double emax = 0.0;
  double dt = 0.0;
  if (rk) {
    if (stage == 0) dt = 1.0 / __longlong_as_double((long long)S->max_eig_bits) * P.cfl;
    else dt = S->dt;
  }
  const bool compat = P.weno5z_compat != 0;
  bool ok = true;
  for (int k = 0; k < nmine; ++k) {
    const int s = k & 1;
    const TileCtx T = decode_tile<DIR, SHP>(blocks, tm, P, tm.base + (int)blockIdx.x + k * (int)gridDim.x);
    const BlockDev &B = *T.B;
    const unsigned char *slot = psm + s * L::SLOT;
    const double *Qh = reinterpret_cast<const double *>(slot + L::Q);
    const double *Jh = reinterpret_cast<const double *>(slot + L::J);
    const double *Mh = reinterpret_cast<const double *>(slot + L::MET);
    const double *Mo = reinterpret_cast<const double *>(slot + L::METO);
    const double *Gh = reinterpret_cast<const double *>(slot + L::GH);
    const int *Gt = reinterpret_cast<const int *>(slot + L::GT);
    // u_i's energy after the reset (zeta), per slot: phase 3 of this tile reads it while
    // phase 1 of the next tile may already write the other slot's
    double *sQ4 = reinterpret_cast<double *>(psm + s * L::SLOT + L::Q4);
    // After a wait that gave up, later waits are skipped, so every consumer thread still
    // reaches every named barrier; the status word reports the failure.
    if (ok && !mbar_wait(&full_q[s], (unsigned)((k >> 1) & 1))) ok = false;

    // ---- phase 1: split fluxes of the line positions c0-R .. c0+cl+R-1 ----
    for (int e = tid; e < TW * NP; e += kThreads) {
      int p, w;
      if (DIR == 0) { p = e % NP; w = e / NP; } else { w = e % TW; p = e / TW; }
      double fp[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, fn[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      const int g = T.c0 + p - R;
      if (w < T.nw && p < T.cl + 2 * R) {
        double q[5], jac, m0, m1, m2;
        bool cell = true;
        if (g >= 0 && g < T.G.L) {
          const int h = G::hidx(p, w);
#pragma unroll
          for (int v = 0; v < 5; ++v) q[v] = Qh[v * G::BOX + h];
          jac = Jh[h];
          m0 = Mh[h];
          m1 = Mh[G::BOX + h];
          m2 = Mh[2 * G::BOX + h];
        } else {
          const int gp = g < 0 ? g + R : R + (g - T.G.L);
          const int it = gp * TW + w;
          const int type = Gt[it];
          const double *o = Gh + it * 9;
#pragma unroll
          for (int v = 0; v < 5; ++v) q[v] = o[v];
          jac = o[5]; m0 = o[6]; m1 = o[7]; m2 = o[8];
          cell = type == 1;
          if (type == 2) {
#pragma unroll
            for (int v = 0; v < 5; ++v) fp[v] = o[v];
          } else if (type == 3) {
#pragma unroll
            for (int v = 0; v < 5; ++v) fn[v] = o[v];
          }
        }
        if (cell) {
          CellPrim sp;
          con2prim(q, jac, P.gamma, P.mach, sp, st);
          q[4] = sp.q4;
          split_cell(P.riemann, q, sp, m0, m1, m2, jac, fp, fn);
          if (g >= T.c0 && g < T.c0 + T.cl) {
            if (DIR == 0 && sp.reset) ++nres;
            if (DIR == 2) sQ4[G::oidx(g - T.c0, w)] = sp.q4;
            if (eig) {
              // max(|U| + c |grad xi|) over the three directions (xi's metric is m0..m2)
              const int oi = G::oidx(g - T.c0, w);
              double ev = eigen_cell(sp, m0, m1, m2);
              emax = ev > emax ? ev : emax;
              ev = eigen_cell(sp, Mo[oi], Mo[G::OWN + oi], Mo[2 * G::OWN + oi]);
              emax = ev > emax ? ev : emax;
              ev = eigen_cell(sp, Mo[3 * G::OWN + oi], Mo[4 * G::OWN + oi], Mo[5 * G::OWN + oi]);
              emax = ev > emax ? ev : emax;
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
    consumer_sync();

    // NS: the direction's viscous fluxes of the tile's line positions into sV (after the
    // barrier above: phase 3 of the previous tile has read sV)
    if constexpr (NSV) phase_vis<DIR, SCH, SHP>(blocks, T, P, sV);

    // ---- phase 2: the ten reconstructions of each face c0 .. c0+cl ----
    {
      const int nf = T.cl + 1;
      const int lo = T.physL ? min(max(T.ts - T.c0, 0), nf) : 0;
      const int hi = T.physR ? min(max(T.G.L - T.ts + 1 - T.c0, 0), nf) : nf;
      const int ni = hi > lo ? hi - lo : 0;
      const int nl = ni > 0 ? lo : nf;
      const int ne = nf - ni;
      const int ei = TW * ni, e0 = (ei + 31) & ~31;
      const float rni = ni > 0 ? 1.0f / (float)ni : 0.0f, rne = ne > 0 ? 1.0f / (float)ne : 0.0f;
      for (int e = tid; e < e0 + TW * ne; e += kThreads) {
        int w, fl;
        bool edge;
        if (e < ei) {
          w = __float2int_rz(((float)e + 0.5f) * rni);
          fl = lo + (e - w * ni);
          edge = false;
        } else if (e >= e0) {
          const int j = e - e0;
          w = __float2int_rz(((float)j + 0.5f) * rne);
          const int kk = j - w * ne;
          fl = kk < nl ? kk : hi + (kk - nl);
          edge = true;
        } else {
          continue;
        }
        if (w >= T.nw) continue;
        const int f = T.c0 + fl;
        if (!edge) {
          const bool cz = compat && f >= T.ts && f <= T.G.L - T.ts;
#pragma unroll kPipeFaceUnroll
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
                edge_face<SCH>(f, T.G.L, T.ts, T.physR, T.c0 - R, T.c0 - R + NP - 1, Pacc, Nacc);
#else
            const double hp = recon_pos<SCH>(f, T.G.L, T.ts, T.physL, T.physR, compat, Pacc);
            const double hn = recon_neg<SCH>(f, T.G.L, T.ts, T.physL, T.physR, Nacc);
            sH[(v * TW + w) * SH + fl] = hp + hn;
#endif
          }
        }
      }
    }
    consumer_sync();

    // ---- phase 3: difference, right-hand side, RK3 stage ----
    if ((need_r || need_n) && ok && !mbar_wait(&full_r[0], (unsigned)(k & 1))) ok = false;
    if (rk && stage == 0 && T.t == 0 && tid == 0) S->dt = dt;
    if (rk && stage == 2 && T.t == 0 && tid == 0) S->time = S->time + dt;
    const long long N = T.N;
    double racc = 0.0;  // the residual's sum of (u - u_n)^2 (SW_RES)
    for (int e = tid; e < TW * TL; e += kThreads) {
      int c, w;
      if (DIR == 0) { c = e % TL; w = e / TL; } else { w = e % TW; c = e / TW; }
      if (w >= T.nw || c >= T.cl) continue;
      const int g = T.c0 + c;
      const long long idx = g * T.G.sL + (T.w0 + w) * T.G.sW + T.o * T.G.sO;
      const int oi = G::oidx(c, w);
      double d[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double *h = sH + (v * TW + w) * SH;
        d[v] = h[c + 1] - h[c];
      }
      double dv[4] = {0.0, 0.0, 0.0, 0.0};
      if constexpr (NSV) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double *row = sV + (v * TW + w) * SV + (kVisHalo - T.c0);
          auto Vacc = [row](int cc) { return row[cc]; };
          dv[v] = diff_at(g, T.G.L, T.ts, T.physL, T.physR, P.vis[DIR], Vacc);
        }
      }
      if (DIR == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) B.rhs[v * N + idx] = d[v];
        if constexpr (NSV) {
#pragma unroll
          for (int v = 0; v < 4; ++v) B.dvis[v * N + idx] = dv[v];
        }
      } else if (DIR == 1) {
#pragma unroll
        for (int v = 0; v < 5; ++v) B.rhs[v * N + idx] = rbuf[v * G::OWN + oi] + d[v];
        if constexpr (NSV) {
#pragma unroll
          for (int v = 0; v < 4; ++v) B.dvis[(4 + v) * N + idx] = dv[v];
        }
      } else if (!rk) {
        double r[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) r[v] = rbuf[v * G::OWN + oi] + d[v];
        if constexpr (NSV) {
#pragma unroll
          for (int v = 1; v < 5; ++v) {
            r[v] = r[v] - B.dvis[(v - 1) * N + idx];
            r[v] = r[v] - B.dvis[(4 + v - 1) * N + idx];
            r[v] = r[v] - dv[v - 1];
          }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) B.rhs[v * N + idx] = r[v];
      } else {
        double *__restrict__ qo = B.q[(stage + 1) % 3];
        const int h = G::hidx(c + R, w);
        double un[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (stage != 0) {
          // u_n with stage 0's energy reset, as the reference's Q_Euler holds it
#pragma unroll
          for (int v = 0; v < 5; ++v) un[v] = nbuf[v * G::OWN + oi];
          CellPrim sn;
          unsigned stn = 0;
          con2prim(un, Jh[h], P.gamma, P.mach, sn, stn);
          un[4] = sn.q4;
        }
        double r[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) r[v] = rbuf[v * G::OWN + oi] + d[v];
        if constexpr (NSV) {
          // the reference's RHS order: inviscid sum, then minus each direction's viscous
          // part (sweep_kernel's phase_cells)
#pragma unroll
          for (int v = 1; v < 5; ++v) {
            r[v] = r[v] - B.dvis[(v - 1) * N + idx];
            r[v] = r[v] - B.dvis[(4 + v - 1) * N + idx];
            r[v] = r[v] - dv[v - 1];
          }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const double ui = v < 4 ? Qh[v * G::BOX + h] : sQ4[oi];
          const double x = rk3_update(stage, r[v], ui, un[v], dt);
          if (!isfinite(x)) st |= ST_NONFINITE;
          qo[v * N + idx] = x;
          if (flags & SW_RES) res_value(B, v, idx, x, un[v], racc);
        }
      }
    }
#if NUC3D_FAST
    if (flags & SW_RES) cta_sum_to(racc, sRed, kThreads, P.res_part + T.t, [] { consumer_sync(); });
#endif
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(&done[s]);
  }
  if (!ok) atomicOr(&S->status, ST_PIPE_TIMEOUT);
  if (eig) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double x = __shfl_xor_sync(0xffffffffu, emax, off);
      emax = x > emax ? x : emax;
    }
    if ((tid & 31) == 0) sRed[tid >> 5] = emax;
    consumer_sync();
    if (tid == 0) {
      double m = sRed[0];
      for (int i = 1; i < kThreads / 32; ++i) m = sRed[i] > m ? sRed[i] : m;
      atomicMax(&S->max_eig_bits, (unsigned long long)__double_as_longlong(m));
    }
  }
  if (st) atomicOr(&S->status, st);
  if (nres) atomicAdd(&S->reset_cells, (unsigned long long)nres);
}
