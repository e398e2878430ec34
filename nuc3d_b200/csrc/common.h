// common.h -- host/device descriptors shared by the NUC3d B200 kernels and the C-ABI.
//
// Data layout in HBM (one block = one structured grid of nx*ny*nz cells):
//   every field is a plain [nz][ny][nx] array of doubles (i fastest), the layout of
//   the reference's field3d (src/field.h:11-81, index k*nx*ny + j*nx + i);
//   multi-component fields are stacked component-major: comp*N + idx.
// Direction-transposed copies of the reference (src/euler3d.cpp:75-80) are not
// materialised: each sweep kernel walks its own axis through strides.
#pragma once
#include <stdint.h>
#include <cuda.h>
#include <cuda_runtime.h>

namespace nuc3d {

enum Scheme : int {
  SCH_WENO5JS = 0, SCH_WENO5Z = 1, SCH_WENO7JS = 2, SCH_CRWENO5 = 3, SCH_HCCS = 4,
  SCH_WENO3JS = 5, SCH_UPWIND1 = 6, SCH_HCCS77 = 7
};
// Viscous difference per direction (scheme_x/y/z_vis, src/fieldOperator.cpp:286-367).
enum VisScheme : int { VIS_CD6 = 0, VIS_CD2 = 1, VIS_CD8 = 2 };
enum Riemann : int { RIE_LF = 0, RIE_AUSM = 1, RIE_AUSMP = 2 };
enum Model : int { MODEL_EULER = 0, MODEL_NS = 1 };
enum BcId : int { BC_INLET = 0, BC_OUTLET = 1, BC_WALL = 2, BC_SYMM = 3 };

// Status bits written by kernels (atomicOr) and read back by the host.
enum StatusBits : unsigned {
  ST_NEG_PRESSURE = 1u,    // EoS pressure < 0 (the reference exits, src/physicsModel.cpp:1009-1016)
  ST_ENERGY_RESET = 2u,    // internal energy < 0, E reset (src/physicsModel.cpp:324-332)
  ST_NONFINITE = 4u,       // a non-finite value was produced by the RK update
  ST_BAD_LAUNCH = 8u,      // a kernel found an inconsistent descriptor and skipped work
  ST_PIPE_TIMEOUT = 16u,   // a pipelined sweep's wait for its copies gave up (results invalid)
};

// Reference bufferSize per scheme (src/fieldOperator.cpp:127-283).
inline __host__ __device__ int scheme_tilesize(int s) {
  return (s == SCH_WENO7JS || s == SCH_HCCS || s == SCH_HCCS77) ? 4
         : s == SCH_WENO3JS ? 2 : s == SCH_UPWIND1 ? 1 : 3;
}

struct FaceDev {
  int type;        // -1: physical boundary; >= 0: neighbour block index
  int id;          // physical: BcId; neighbour: the neighbour's face 0..5
  double bcv[5];   // inlet primitive state (rho, u, v, w, p), from BC_Topo values
};

// Everything a kernel needs to know about one block.  Pointers are device pointers.
struct BlockDev {
  int n[3];              // nx, ny, nz (cells)
  int pad_;
  long long N;           // nx*ny*nz
  double *q[3];          // TVD-RK3 state buffers: q[0] = Q_n, q[1] = Q_1, q[2] = Q_2 (5*N each)
  double *rhs;           // 5*N
  const double *jac;     // N
  const double *met[3];  // met[d] = 3*N: (d_x, d_y, d_z) of computational coordinate d
  const double *dxyz;    // 9*N: x_xi, x_eta, x_zeta, y_xi, y_eta, y_zeta, z_xi, z_eta, z_zeta (or null)
  double *prim;          // NS: u, v, w, T (4*N)
  double *vis;           // NS: contravariant viscous fluxes, [dir][var 1..4] (12*N)
  double *dvis;          // NS exact mode: d(Fv)/dxi and d(Gv)/deta, vars 1..4 (8*N)
  double *ghost;         // split flux of the ghost next to each physical face: at
                         // ghost + goff[f], 5 components of A_f*B_f slab cells (F+ on
                         // left faces, F- on right faces)
  long long goff[6];     // -1 for neighbour faces
  double *fh;            // compact schemes: face fluxes [sys][line][face] of one direction
  double *rows;          // compact schemes: tridiagonal rows [row][4][sys*lines + line]
  double *dres;          // reference-order build: u - u_n of the last RK stage (5*N), summed
                         // in the reference's order for the residual; null otherwise
  FaceDev face[6];
  // Per direction d, ceil(2^40 / k) for k = tile chunks per line and k = line groups:
  // the sweep kernels divide tile indices by multiply-and-shift (set_tile_divisors).
  unsigned long long tdiv[3][2];
};

// Sweep tile shapes, chosen per direction (nuc3d_autotune): shape s is tile_w(s) lines x
// tile_l(s) cells along them; 0: 4 x 64, 1: 8 x 32, 2: 2 x 128.  All hold 256 cells, so
// every sweep CTA has the same 288 threads.  Compact schemes use shape 0.
constexpr int kTileShapes = 3;
// Shapes kLineShape (1 x 256) and kLineShape4 (kLineLanes x 256: whole lines of at most
// 256 cells) are not autotuner choices: they are the tiles of the fused compact sweep
// (compact_line_kernel), one line per CTA along xi, kLineLanes neighbouring lines along
// eta and zeta so that the strided loads fill 32-byte sectors.
constexpr int kLineShape = 3;
constexpr int kLineShape4 = 4;
#ifndef NUC3D_LINE_LANES
#define NUC3D_LINE_LANES 2  // 4: one CTA per SM, measured slower
#endif
constexpr int kLineLanes = NUC3D_LINE_LANES;
constexpr int kLineMax = 256;
// dynamic shared memory a CTA may opt in to: the 227 KB per-block maximum less 1 KB for the
// kernels' static shared memory (the attribute must leave room for it)
constexpr size_t kSmemOptin = 227 * 1024 - 1024;
__host__ __device__ constexpr int line_shape(int dir) { return dir == 0 ? kLineShape : kLineShape4; }
__host__ __device__ constexpr int tile_w(int s) {
  return s == 1 ? 8 : (s == 2 ? 2 : (s == 3 ? 1 : (s == 4 ? kLineLanes : 4)));
}
__host__ __device__ constexpr int tile_l(int s) {
  return s == 1 ? 32 : (s == 2 ? 128 : (s >= 3 ? 256 : 64));
}

// Boxes of the pipelined sweep's tensor-map loads (pipe_sweep_kernel), for direction d, a
// tile of tw lines x tl cells and a scheme reaching r cells: the halo box covers line
// positions c0-r .. c0+tl+r-1 of the tile's lanes (xi: from c0 - ra, ra = r rounded up to
// even, and x extent rounded up to even, so that the box starts and spans whole 16-byte
// units); the own box covers the tile's cells.  ext[0..2] = x, y, z extents.
__host__ __device__ constexpr int pipe_ra(int r) { return (r + 1) & ~1; }
__host__ __device__ inline void pipe_box(int d, int tw, int tl, int r, bool halo, int ext[3]) {
  const int len = halo ? (d == 0 ? ((tl + r + pipe_ra(r) + 1) & ~1) : tl + 2 * r) : tl;
  ext[0] = d == 0 ? len : tw;
  ext[1] = d == 0 ? tw : (d == 1 ? len : 1);
  ext[2] = d == 2 ? len : 1;
}
// Cells a scheme's reconstruction reaches past a face (the sweep's split halo).
__host__ __device__ constexpr int scheme_halo(int s) {
  return (s == SCH_WENO7JS || s == SCH_HCCS || s == SCH_HCCS77) ? 4
         : s == SCH_WENO3JS ? 2 : s == SCH_UPWIND1 ? 1 : 3;
}

// Fills BlockDev::tdiv from n[] and the directions' tile shapes: the two radices of the
// tile index decode (decode_tile), chunks and line groups for xi and eta, line groups and
// outer lines for zeta.  q = (x * tdiv) >> 40 equals x / k exactly for x < 2^24 (the tile
// count of a block of fewer than 2^32 cells) and k < 2^16.
inline void set_tile_divisors(BlockDev &b, const int shape[3]) {
  for (int d = 0; d < 3; ++d) {
    const unsigned long long L = (unsigned long long)b.n[d];
    const unsigned long long nW = (unsigned long long)(d == 0 ? b.n[1] : b.n[0]);
    const unsigned long long TL = (unsigned long long)tile_l(shape[d]),
                             TW = (unsigned long long)tile_w(shape[d]);
    const unsigned long long nch = (L + TL - 1) / TL, nwg = (nW + TW - 1) / TW;
    const unsigned long long k[2] = {d == 2 ? nwg : nch, d == 2 ? (unsigned long long)b.n[1] : nwg};
    for (int j = 0; j < 2; ++j) b.tdiv[d][j] = ((1ull << 40) + k[j] - 1) / k[j];
  }
}

// Physical faces of all blocks, laid end to end for the BC ghost pass.
constexpr int kMaxFaceJobs = 6 * 512;
struct FaceJobs {
  int njobs;
  int block[kMaxFaceJobs];
  unsigned char face[kMaxFaceJobs];
  int start[kMaxFaceJobs + 1];  // prefix sums of 256-cell tiles
};

// The face sensor of the hybrid WENO-Z sweep (sensor.cuh), arranged for the tensor-core
// inference: BF16 weight pairs in mma.sync m16n8k16 B-fragment order, [k-step][n-tile][lane],
// and BF16-rounded biases and output weights as floats.  zero_logit: the network's logit
// for all-zero features (a face inside a uniform region), evaluated once on the GPU by
// the same tensor-core code when the sensor is set.
struct SensorDev {
  uint32_t w1[2][4][32][2];
  float b1[32];
  uint32_t w2[2][4][32][2];
  float b2[32];
  float w3[32];
  float b3;
  float zero_logit;
};

struct SolverParams {
  int scheme[3];         // per direction
  int ts[3];             // per-direction bufferSize (scheme_tilesize)
  int bfs;               // bfsize = max ts: width of the reference's ghost slabs
  int riemann;
  int model;
  int weno5z_compat;     // 1: reproduce the interior positive is2 of src/weno5z.cpp:80
  int vis[3];            // VisScheme per direction
  double gamma, mach, reynolds, prandtl, t_ref, t_inf, t_wall, cfl;
  const SensorDev *sensor;  // hybrid WENO-Z: the face sensor, or null (plain WENO-Z)
  float sensor_threshold;   // logit below which a face takes the linear weights
  int sensor_theta;         // 1: decide by hccs's theta switch instead of the network;
                            // a face takes the linear weights where theta >= sensor_threshold
  double *res_part;         // throughput build: per-tile sums of (u - u_n)^2 of the step's
                            // last stage, for the residual (Launch::d_res_part)
};

// Per-launch work list: tiles of every block, laid end to end.
constexpr int kMaxBlocks = 512;
struct TileMap {
  int nblocks;
  int tile_start[kMaxBlocks + 1];  // prefix sums of tiles per block
  // the tiles base .. end-1 of a launch over part of the map (end 0: to the last tile);
  // kernels keep the global tile index, so per-tile outputs and "tile 0" duties are as
  // in a launch over all tiles
  int base, end;
};

// Device-resident scalars of the time loop.
struct StepState {
  unsigned long long max_eig_bits;  // max over blocks and directions of |U|+c|grad xi| (bits of a double >= 0)
  unsigned long long res_bits;      // the step's residual (PDEData3d::setRES, src/PDEData3d.cpp:
                                    // 90-122): max over blocks, bits of a double >= 0
  double dt;                        // cfl / max_eig, fixed at stage 0 of each step
  double time;                      // accumulated time
  unsigned status;                  // StatusBits
  unsigned pad_;
  unsigned long long reset_cells;   // cells whose energy con2prim reset (src/physicsModel.cpp:
                                    // 324-332), once per cell and right-hand side; the
                                    // reference prints one "negative pressure at" line for each
};

// What the host hands to a stage launch.
struct Launch {
  const BlockDev *d_blocks;
  StepState *d_state;
  SolverParams P;
  TileMap tm_dir[3];
  TileMap tm_sys[3];       // compact schemes: 256-system tiles per direction
  TileMap tm_cells;
  TileMap tm_line[3];      // fused compact sweeps: one tile per line
  int line_dirs;           // bit d: direction d's compact scheme runs compact_line_kernel
  const FaceJobs *d_jobs;  // device copy
  int bc_tiles;            // CTAs of the BC ghost pass (0: no physical faces)
  cudaStream_t stream;
  int shape[3];            // sweep tile shape per direction (tile_w / tile_l)
  // pipelined sweeps (pipe_sweep_kernel): tensor maps [block][dir][PM_COUNT] in device
  // memory and the persistent grid (CTAs); null / 0: the one-tile-per-CTA sweeps
  const CUtensorMap *d_maps;
  int pipe_grid;
  int pipe_dirs;           // bit d: direction d runs pipelined (nuc3d_autotune picks per direction)
  // each block's residual root of the previous step (the reference's static res_last);
  // null: no residual (nuc3d_rhs_noalloc)
  double *d_res_last;
};

// Diagnostics workspace of one block (postproc::solveQ, src/postproc.cpp:743-848):
// prim 4N (rho, u, v, w), fields 5N (vorticity x, y, z, 0.5|w|^2, Q), dens 2N (the
// per-cell enstrophy and kinetic-energy terms of the totals).
struct DiagDev {
  double *prim, *fields, *dens;
};
// Partial sums per block of the throughput build's two-pass reduction.
constexpr int kDiagParts = 256;

// One right-hand-side evaluation of every block at RK stage `stage`
// (state q[stage]); rk: also apply the TVD-RK3 update; eig: reduce the
// eigenvalue maximum that fixes dt.  Defined once per arithmetic mode.
// Message returned by nuc3d_last_error() for the calling thread.
void set_error_message(const char *msg);

// configure(): one-time kernel attributes (dynamic shared memory opt-in).
// run_sensor_zero(): fills S->zero_logit (one warp).
// tile_count(): CTAs of the dir-sweep over one block of n cells with tile shape `shape`.
// run_metrics(): block::getJacobians of an nx x ny x nz block from its node coordinates
// ((n+1) per axis, device arrays); *bad gets 1 for a negative Jacobian.
// run_diag(): the solveQ diagnostics of state q[0] of every block into dd[b] and the
// per-block totals sums[2b] (enstrophy), sums[2b+1] (kinetic energy); parts holds
// 2 * kDiagParts doubles per block of scratch.
// run_rk_stage(): the TVD-RK3 stage update alone (rk_stage_kernel), from the RHS array, dt
// given; at stage 2 also time += dt and the residual.
// run_residual(): the residual of the step just finished (after stage 2); cells: 1 when the
// partial sums are per cell tile (rk_stage_kernel), 0 per zeta-sweep tile.
namespace exact {
cudaError_t run_rk_stage(const Launch &L, int stage, double dt);
cudaError_t run_residual(const Launch &L, bool cells);
cudaError_t run_stage(const Launch &L, int stage, bool rk, bool eig);
// run_bc(): the physical faces' ghost fluxes at stage `stage` for the cells k0 <= k < k1.
// Pieces of one Euler step over z-slabs (nuc3d_solve_host's copy/compute pipeline).
cudaError_t run_stage0_slab(const Launch &L, int k0, int k1, int tx0, int tx1, int ty0, int ty1);
cudaError_t run_stage0_zeta(const Launch &L, int tz0, int tz1);
cudaError_t run_stage_slab(const Launch &L, int stage, int k0, int k1, int tx0, int tx1, int ty0, int ty1,
                           int tz0, int tz1);
cudaError_t run_bc(const Launch &L, int stage, int k0, int k1);
cudaError_t run_stage_pre(const Launch &L, int stage);
cudaError_t run_stage_sweeps(const Launch &L, int stage, int b0, int b1);
cudaError_t run_sensor_zero(SensorDev *S, cudaStream_t st);
cudaError_t run_sensor_data(const Launch &L, int dir, float *feat, unsigned char *label,
                            long long *where, unsigned long long *count, unsigned long long cap);
cudaError_t run_metrics(const double *x, const double *y, const double *z, const int n[3],
                        double *jac, double *met, double *dxyz, unsigned *bad, cudaStream_t st);
cudaError_t run_diag(const Launch &L, const DiagDev *dd, double *sums, double *parts);
cudaError_t run_sweep(const Launch &L, int dir, int stage, int flags);
// run_taps(): debug taps of direction dir for one block (nl: its lines along dir);
// out = FluxL, FluxR (5N), reconstFluxL, reconstFluxR (5 (L+1) nl), dF (5N), device.
cudaError_t run_taps(const Launch &L, int block, int dir, int nl, double *const out[5]);
// compact_line_smem(): dynamic shared memory of the fused compact sweep (0: none).
size_t compact_line_smem(int dir, int sch, bool ns);
cudaError_t configure();
int tile_count(int dir, const int n[3], int shape);
}
namespace fast {
cudaError_t run_rk_stage(const Launch &L, int stage, double dt);
cudaError_t run_residual(const Launch &L, bool cells);
cudaError_t run_stage(const Launch &L, int stage, bool rk, bool eig);
// run_bc(): the physical faces' ghost fluxes at stage `stage` for the cells k0 <= k < k1.
// Pieces of one Euler step over z-slabs (nuc3d_solve_host's copy/compute pipeline).
cudaError_t run_stage0_slab(const Launch &L, int k0, int k1, int tx0, int tx1, int ty0, int ty1);
cudaError_t run_stage0_zeta(const Launch &L, int tz0, int tz1);
cudaError_t run_stage_slab(const Launch &L, int stage, int k0, int k1, int tx0, int tx1, int ty0, int ty1,
                           int tz0, int tz1);
cudaError_t run_bc(const Launch &L, int stage, int k0, int k1);
cudaError_t run_stage_pre(const Launch &L, int stage);
cudaError_t run_stage_sweeps(const Launch &L, int stage, int b0, int b1);
cudaError_t run_sensor_zero(SensorDev *S, cudaStream_t st);
cudaError_t run_sensor_data(const Launch &L, int dir, float *feat, unsigned char *label,
                            long long *where, unsigned long long *count, unsigned long long cap);
cudaError_t run_metrics(const double *x, const double *y, const double *z, const int n[3],
                        double *jac, double *met, double *dxyz, unsigned *bad, cudaStream_t st);
cudaError_t run_diag(const Launch &L, const DiagDev *dd, double *sums, double *parts);
cudaError_t run_sweep(const Launch &L, int dir, int stage, int flags);
// run_taps(): debug taps of direction dir for one block (nl: its lines along dir);
// out = FluxL, FluxR (5N), reconstFluxL, reconstFluxR (5 (L+1) nl), dF (5N), device.
cudaError_t run_taps(const Launch &L, int block, int dir, int nl, double *const out[5]);
// compact_line_smem(): dynamic shared memory of the fused compact sweep (0: none).
size_t compact_line_smem(int dir, int sch, bool ns);
cudaError_t configure();
int tile_count(int dir, const int n[3], int shape);
}

}  // namespace nuc3d
