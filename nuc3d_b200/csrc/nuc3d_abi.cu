// nuc3d_abi.cu -- the C ABI (include/nuc3d_gpu.h) over the stage kernels.
//
// Owns the per-block device arrays, validates the block topology the way the
// reference's BC_Topo pairing works (src/boundaryConditions.cpp:25-93,
// src/MPICommunicator.cpp:27-34), and drives the time loop of block::solve
// (src/block.cpp:569-594): per step three stages, dt fixed at stage 0 from the
// global eigenvalue maximum (src/PDEData3d.cpp:152-170), time += dt.  A step is
// captured once as a CUDA graph and replayed.
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "common.h"
#include "nuc3d_gpu.h"

using namespace nuc3d;

// Tensor maps of the pipelined sweeps: [block][dir][kind] (the kinds of sweep_pipe.cuh).
namespace nuc3d {
enum : int { kMapQ0 = 0, kMapJac = 3, kMapMet = 4, kMapMetO = 5, kMapRhs = 6, kMapQn = 7, kMapKinds = 8 };
}

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CUDA_TRY(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return fail(NUC3D_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

struct HostBlock {
  int n[3];
  long long N;
  int bc_type[6], bc_id[6];
  double bcv[6][5];
  double *q[3] = {nullptr, nullptr, nullptr};
  double *rhs = nullptr, *jac = nullptr, *met = nullptr, *dxyz = nullptr;
  double *prim = nullptr, *vis = nullptr, *dvis = nullptr, *ghost = nullptr;
  double *fh = nullptr, *rows = nullptr;  // compact schemes
  double *dres = nullptr;                 // reference-order build: u - u_n for the residual
  long long goff[6] = {-1, -1, -1, -1, -1, -1};
  bool metrics = false;
};

int parse_scheme(const char *s, int *out) {
  if (!s) return fail(NUC3D_EINVAL, "null scheme name");
  if (!std::strcmp(s, "weno5js")) *out = SCH_WENO5JS;
  else if (!std::strcmp(s, "weno5z")) *out = SCH_WENO5Z;
  else if (!std::strcmp(s, "weno7js")) *out = SCH_WENO7JS;
  else if (!std::strcmp(s, "crweno5")) *out = SCH_CRWENO5;
  else if (!std::strcmp(s, "hccs")) *out = SCH_HCCS;
  else if (!std::strcmp(s, "weno3js")) *out = SCH_WENO3JS;
  else if (!std::strcmp(s, "upwind1st")) *out = SCH_UPWIND1;
  else if (!std::strcmp(s, "hccs77")) *out = SCH_HCCS77;
  else return fail(NUC3D_EINVAL, "unknown reconstruction scheme '%s'", s);
  return NUC3D_OK;
}

// scheme_x/y/z_vis (src/fieldOperator.cpp:286-367); null means cd6, the reference default
int parse_vis(const char *s, int *out) {
  if (!s || !std::strcmp(s, "cd6")) *out = VIS_CD6;
  else if (!std::strcmp(s, "cd2")) *out = VIS_CD2;
  else if (!std::strcmp(s, "cd8")) *out = VIS_CD8;
  else return fail(NUC3D_EINVAL, "unknown viscous scheme '%s' (cd2 | cd6 | cd8)", s);
  return NUC3D_OK;
}

// Cells the viscous stencil reaches.  The reference's difference loops start at the
// direction's tilesize (src/centraldifference6th.cpp:26-43, 8th :27-52) and take ghosts
// from slabs bfsize wide, so a reach beyond the tilesize reads outside its rows.
int vis_reach(int vis) { return vis == VIS_CD2 ? 1 : vis == VIS_CD8 ? 4 : 3; }

}  // namespace

void nuc3d::set_error_message(const char *msg) { g_err = msg; }

struct nuc3d_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool exact = true;
  SolverParams P{};
  std::vector<HostBlock> blocks;
  BlockDev *d_blocks = nullptr;
  FaceJobs *d_jobs = nullptr;
  StepState *d_state = nullptr;
  Launch L{};
  bool finalized = false;
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  // diagnostics workspace, allocated by the first nuc3d_diagnostics call
  std::vector<DiagDev> diag;
  DiagDev *d_diag = nullptr;
  double *d_dsums = nullptr, *d_dparts = nullptr;
  SensorDev *d_sensor = nullptr;  // hybrid WENO-Z face sensor (nuc3d_set_sensor)
  std::vector<BlockDev> hdesc;  // host copy of the block descriptors (tile divisors change)
  // pipelined sweeps: tensor maps of every block and direction (built by build_maps)
  bool use_pipe = true;
  int pipe_mask = 7;  // directions to run pipelined where the grid allows (bit d)
  bool compact_fused = true;  // throughput build: compact directions on compact_line_kernel
  CUtensorMap *d_maps = nullptr;
  // the residual of each step: per-tile partial sums, each block's previous residual root
  double *d_res_part = nullptr, *d_res_last = nullptr;
  // nuc3d_solve_host: copy streams and events, created by its first call
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_start = nullptr, ev_h2d = nullptr, ev_step = nullptr, ev_end = nullptr;
  std::vector<cudaEvent_t> ev_chunk;
  // nuc3d_solve_host's slab pipeline: per z-slab, upload done / stage-2 zeta done / download done
  std::vector<cudaEvent_t> ev_up, ev_zeta, ev_down;
  bool host_pipeline = true;

  cudaError_t stage(int s, bool rk, bool eig) {
    return exact ? nuc3d::exact::run_stage(L, s, rk, eig) : nuc3d::fast::run_stage(L, s, rk, eig);
  }
  cudaError_t one_step() {
    cudaError_t e = cudaMemsetAsync(&d_state->max_eig_bits, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    for (int s = 0; s < 3; ++s)
      if ((e = stage(s, true, s == 0)) != cudaSuccess) return e;
    return cudaSuccess;
  }
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    gexec = nullptr;
    graph = nullptr;
  }
};

extern "C" {

const char *nuc3d_last_error(void) { return g_err.c_str(); }

int nuc3d_create(const nuc3d_config *cfg, int device, nuc3d_ctx **out) {
  if (!cfg || !out) return fail(NUC3D_EINVAL, "null argument");
  *out = nullptr;
  SolverParams P{};
  for (int d = 0; d < 3; ++d) {
    int r = parse_scheme(cfg->scheme_ivs[d], &P.scheme[d]);
    if (r) return r;
    if ((r = parse_vis(cfg->scheme_vis[d], &P.vis[d]))) return r;
    P.ts[d] = scheme_tilesize(P.scheme[d]);
  }
  // block::initialData: bfsize = max of the three bufferSizes (src/block.cpp:506-507)
  P.bfs = P.ts[0] > P.ts[1] ? P.ts[0] : P.ts[1];
  P.bfs = P.bfs > P.ts[2] ? P.bfs : P.ts[2];
  if (!cfg->riemann) return fail(NUC3D_EINVAL, "null riemann name");
  if (!std::strcmp(cfg->riemann, "LF")) P.riemann = RIE_LF;
  else if (!std::strcmp(cfg->riemann, "AUSM")) P.riemann = RIE_AUSM;
  else if (!std::strcmp(cfg->riemann, "AUSMp")) P.riemann = RIE_AUSMP;
  else return fail(NUC3D_EINVAL, "unknown Riemann solver '%s'", cfg->riemann);
  if (!cfg->model) return fail(NUC3D_EINVAL, "null model name");
  if (!std::strcmp(cfg->model, "Euler3d")) P.model = MODEL_EULER;
  else if (!std::strcmp(cfg->model, "NavierStokes3d")) P.model = MODEL_NS;
  else return fail(NUC3D_EINVAL, "unknown model '%s' (Euler3d | NavierStokes3d)", cfg->model);
  if (P.model == MODEL_NS)
    for (int d = 0; d < 3; ++d)
      if (vis_reach(P.vis[d]) > P.ts[d])
        return fail(NUC3D_ENOTSUP,
                    "direction %d: the viscous stencil reaches %d cells but the reconstruction's "
                    "bufferSize is %d; the reference reads outside its arrays there", d,
                    vis_reach(P.vis[d]), P.ts[d]);
  P.reynolds = cfg->reynolds;
  P.mach = cfg->mach;
  P.prandtl = cfg->prandtl;
  P.gamma = cfg->gamma;
  P.t_ref = cfg->t_ref;
  P.t_inf = cfg->t_inf;
  P.t_wall = cfg->t_wall;
  P.cfl = cfg->cfl;
  P.weno5z_compat = cfg->weno5z_compat ? 1 : 0;
  if (!(P.gamma > 1.0) || !(P.mach > 0.0) || !(P.cfl > 0.0))
    return fail(NUC3D_EINVAL, "gamma > 1, mach > 0 and cfl > 0 are required");

  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(NUC3D_EINVAL, "device %d not present", device);
  CUDA_TRY(cudaSetDevice(device));
  nuc3d_ctx *c = new nuc3d_ctx();
  c->device = device;
  c->P = P;
  c->exact = cfg->exact != 0;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_state, sizeof(StepState));
  if (e == cudaSuccess) e = cudaMemset(c->d_state, 0, sizeof(StepState));
  if (e == cudaSuccess) e = c->exact ? nuc3d::exact::configure() : nuc3d::fast::configure();
  if (e != cudaSuccess) {
    if (c->d_state) cudaFree(c->d_state);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return fail(NUC3D_ECUDA, "context setup: %s", cudaGetErrorString(e));
  }
  c->own_stream = true;
  *out = c;
  return NUC3D_OK;
}

int nuc3d_destroy(nuc3d_ctx *c) {
  if (!c) return NUC3D_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->drop_graph();
  for (auto &b : c->blocks) {
    for (auto p : {b.q[0], b.q[1], b.q[2], b.rhs, b.jac, b.met, b.dxyz, b.prim, b.vis, b.dvis,
                   b.ghost, b.fh, b.rows, b.dres})
      if (p) cudaFree(p);
  }
  for (auto p : {c->d_res_part, c->d_res_last})
    if (p) cudaFree(p);
  if (c->d_maps) cudaFree(c->d_maps);
  for (auto &d : c->diag)
    for (auto p : {d.prim, d.fields, d.dens})
      if (p) cudaFree(p);
  for (auto p : {c->d_dsums, c->d_dparts})
    if (p) cudaFree(p);
  if (c->d_diag) cudaFree(c->d_diag);
  if (c->d_sensor) cudaFree(c->d_sensor);
  if (c->d_blocks) cudaFree(c->d_blocks);
  if (c->d_jobs) cudaFree(c->d_jobs);
  if (c->d_state) cudaFree(c->d_state);
  for (auto ev : c->ev_chunk) cudaEventDestroy(ev);
  for (auto *v : {&c->ev_up, &c->ev_zeta, &c->ev_down})
    for (auto ev : *v) cudaEventDestroy(ev);
  for (auto ev : {c->ev_start, c->ev_h2d, c->ev_step, c->ev_end})
    if (ev) cudaEventDestroy(ev);
  for (auto st : {c->h2d, c->d2h})
    if (st) cudaStreamDestroy(st);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return NUC3D_OK;
}

int nuc3d_block_add(nuc3d_ctx *c, int nx, int ny, int nz, const int bc_type[6], const int bc_id[6],
                    const double *bc_values, int *block_id) {
  if (!c || !bc_type || !bc_id) return fail(NUC3D_EINVAL, "null argument");
  if (c->finalized) return fail(NUC3D_ESTATE, "blocks cannot be added after nuc3d_finalize");
  if ((int)c->blocks.size() >= kMaxBlocks) return fail(NUC3D_EINVAL, "at most %d blocks", kMaxBlocks);
  const int n[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d)
    if (n[d] < 2 * c->P.bfs + 2)
      return fail(NUC3D_EINVAL, "block dimension %d = %d is below 2*bfsize+2 = %d", d, n[d],
                  2 * c->P.bfs + 2);
  HostBlock b;
  for (int d = 0; d < 3; ++d) b.n[d] = n[d];
  b.N = (long long)nx * ny * nz;
  for (int f = 0; f < 6; ++f) {
    b.bc_type[f] = bc_type[f];
    b.bc_id[f] = bc_id[f];
    if (bc_type[f] == -1) {
      if (bc_id[f] < 0 || bc_id[f] > 3)
        return fail(NUC3D_EINVAL, "face %d: physical BC id %d not in 0..3", f, bc_id[f]);
    } else if (bc_type[f] < 0) {
      return fail(NUC3D_EINVAL, "face %d: type %d (use -1 or a block index)", f, bc_type[f]);
    }
    for (int v = 0; v < 5; ++v) b.bcv[f][v] = bc_values ? bc_values[f * 5 + v] : 0.0;
    if (bc_type[f] == -1 && bc_id[f] == BC_INLET && !bc_values)
      return fail(NUC3D_EINVAL, "face %d is an inlet but no bc_values were given", f);
  }
  for (int d = 0; d < 3; ++d) {
    if (c->P.scheme[d] != SCH_HCCS77) continue;
    // hccs77 builds its rows in file-static a, b, c, d[128][128][128] (src/hccs77.hpp:15-18),
    // row n of a line at [k][j][n], and solves them only from interpolationBoundaryR
    // (src/hccs77.cpp:570-590), which the reference calls for neighbour faces alone
    // (src/fieldOperator.cpp:400-412).  A physical face would leave rows of an earlier
    // call in the system (or no solve at all), a longer line would write into the next
    // line's rows.
    if (bc_type[2 * d] == -1 || bc_type[2 * d + 1] == -1)
      return fail(NUC3D_ENOTSUP,
                  "direction %d: hccs77 with a physical face; the reference then solves rows "
                  "left from an earlier call", d);
    for (int e = 0; e < 3; ++e)
      if (n[e] > (e == d ? 127 : 128))
        return fail(NUC3D_ENOTSUP,
                    "direction %d: hccs77 keeps its rows in 128x128x128 arrays; the line "
                    "extent must be <= 127 cells and the other two <= 128 (dimension %d is %d)",
                    d, e, n[e]);
  }
  cudaSetDevice(c->device);
  const size_t nb = (size_t)b.N * sizeof(double);
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < 3 && e == cudaSuccess; ++s) e = cudaMalloc(&b.q[s], 5 * nb);
  if (e == cudaSuccess) e = cudaMalloc(&b.rhs, 5 * nb);
  if (e == cudaSuccess) e = cudaMalloc(&b.jac, nb);
  if (e == cudaSuccess) e = cudaMalloc(&b.met, 9 * nb);
  if (c->P.model == MODEL_NS) {
    if (e == cudaSuccess) e = cudaMalloc(&b.prim, 4 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&b.vis, 12 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&b.dvis, 8 * nb);
  }
  {
    long long off = 0;
    for (int f = 0; f < 6; ++f) {
      if (bc_type[f] != -1) continue;
      const int d = f >> 1;
      const long long area = d == 0 ? (long long)ny * nz : (d == 1 ? (long long)nz * nx : (long long)nx * ny);
      b.goff[f] = off;
      off += 5 * area;
    }
    if (off > 0 && e == cudaSuccess) e = cudaMalloc(&b.ghost, off * sizeof(double));
  }
  {
    // compact schemes: face fluxes of all systems of one direction and their tridiagonal
    // rows, sized for the largest compact direction of the block (directions run one
    // after the other)
    long long fh_n = 0, rows_n = 0;
    for (int d = 0; d < 3; ++d) {
      const int sc = c->P.scheme[d];
      if (sc != SCH_CRWENO5 && sc != SCH_HCCS && sc != SCH_HCCS77) continue;
      const long long nl = (long long)b.N / n[d];
      const long long m = n[d] - 2 * (sc == SCH_HCCS77 ? 0 : c->P.ts[d]) + 1;
      fh_n = std::max(fh_n, 10 * nl * (n[d] + 1));
      rows_n = std::max(rows_n, 4 * m * 10 * nl);
    }
    if (fh_n > 0 && e == cudaSuccess) e = cudaMalloc(&b.fh, fh_n * sizeof(double));
    if (rows_n > 0 && e == cudaSuccess) e = cudaMalloc(&b.rows, rows_n * sizeof(double));
  }
  if (c->exact && e == cudaSuccess) e = cudaMalloc(&b.dres, 5 * nb);
  for (int s = 0; s < 3 && e == cudaSuccess; ++s) e = cudaMemset(b.q[s], 0, 5 * nb);
  if (e == cudaSuccess) e = cudaMemset(b.rhs, 0, 5 * nb);
  if (e != cudaSuccess) {
    for (auto p : {b.q[0], b.q[1], b.q[2], b.rhs, b.jac, b.met, b.prim, b.vis, b.dvis, b.ghost,
                   b.fh, b.rows, b.dres})
      if (p) cudaFree(p);
    return fail(NUC3D_ECUDA, "block allocation (%lld cells): %s", b.N, cudaGetErrorString(e));
  }
  c->blocks.push_back(b);
  if (block_id) *block_id = (int)c->blocks.size() - 1;
  return NUC3D_OK;
}

int nuc3d_block_set_metrics(nuc3d_ctx *c, int bi, const double *jac, const double *xi_xyz,
                            const double *eta_xyz, const double *zeta_xyz, const double *dxyz) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad block index");
  if (!jac || !xi_xyz || !eta_xyz || !zeta_xyz) return fail(NUC3D_EINVAL, "null metric array");
  HostBlock &b = c->blocks[bi];
  const size_t nb = (size_t)b.N * sizeof(double);
  cudaSetDevice(c->device);
  CUDA_TRY(cudaMemcpy(b.jac, jac, nb, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(b.met, xi_xyz, 3 * nb, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(b.met + 3 * b.N, eta_xyz, 3 * nb, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(b.met + 6 * b.N, zeta_xyz, 3 * nb, cudaMemcpyHostToDevice));
  if (dxyz) {
    if (!b.dxyz) CUDA_TRY(cudaMalloc(&b.dxyz, 9 * nb));
    CUDA_TRY(cudaMemcpy(b.dxyz, dxyz, 9 * nb, cudaMemcpyHostToDevice));
  }
  b.metrics = true;
  return NUC3D_OK;
}

int nuc3d_block_set_nodes(nuc3d_ctx *c, int bi, const double *x, const double *y,
                          const double *z) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad block index");
  if (!x || !y || !z) return fail(NUC3D_EINVAL, "null node array");
  HostBlock &b = c->blocks[bi];
  for (int d = 0; d < 3; ++d)
    if (b.n[d] % 4)
      return fail(NUC3D_EINVAL, "the reference's tile-Lagrange metrics need cells per axis to be "
                  "a multiple of 4 (block %d axis %d has %d)", bi, d, b.n[d]);
  bool symm = false;
  for (int f = 0; f < 6; ++f) symm = symm || (b.bc_type[f] == -1 && b.bc_id[f] == BC_SYMM);
  const size_t nn = (size_t)(b.n[0] + 1) * (b.n[1] + 1) * (b.n[2] + 1) * sizeof(double);
  const size_t nb = (size_t)b.N * sizeof(double);
  cudaSetDevice(c->device);
  if (symm && !b.dxyz) CUDA_TRY(cudaMalloc(&b.dxyz, 9 * nb));
  double *nodes = nullptr;
  unsigned *bad = nullptr;
  CUDA_TRY(cudaMalloc(&nodes, 3 * nn + 256));
  cudaError_t e = cudaSuccess;
  unsigned h_bad = 0;
  bad = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(nodes) + 3 * nn);
  const double *src[3] = {x, y, z};
  for (int a = 0; a < 3 && e == cudaSuccess; ++a)
    e = cudaMemcpy(reinterpret_cast<char *>(nodes) + a * nn, src[a], nn, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(bad, 0, sizeof(unsigned));
  if (e == cudaSuccess) {
    const double *dx = nodes, *dy = reinterpret_cast<const double *>(reinterpret_cast<char *>(nodes) + nn),
                 *dz = reinterpret_cast<const double *>(reinterpret_cast<char *>(nodes) + 2 * nn);
    e = nuc3d::exact::run_metrics(dx, dy, dz, b.n, b.jac, b.met, symm ? b.dxyz : nullptr, bad,
                                  nullptr);
  }
  if (e == cudaSuccess) e = cudaMemcpy(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(nodes);
  if (e != cudaSuccess) return fail(NUC3D_ECUDA, "metrics: %s", cudaGetErrorString(e));
  if (h_bad) return fail(NUC3D_EINVAL, "block %d: negative Jacobian (the reference exits)", bi);
  b.metrics = true;
  return NUC3D_OK;
}

int nuc3d_block_get_metrics(nuc3d_ctx *c, int bi, double *jac, double *xi_xyz, double *eta_xyz,
                            double *zeta_xyz, double *dxyz) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad block index");
  HostBlock &b = c->blocks[bi];
  if (!b.metrics) return fail(NUC3D_ESTATE, "block %d has no metrics", bi);
  const size_t nb = (size_t)b.N * sizeof(double);
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (jac) CUDA_TRY(cudaMemcpy(jac, b.jac, nb, cudaMemcpyDeviceToHost));
  if (xi_xyz) CUDA_TRY(cudaMemcpy(xi_xyz, b.met, 3 * nb, cudaMemcpyDeviceToHost));
  if (eta_xyz) CUDA_TRY(cudaMemcpy(eta_xyz, b.met + 3 * b.N, 3 * nb, cudaMemcpyDeviceToHost));
  if (zeta_xyz) CUDA_TRY(cudaMemcpy(zeta_xyz, b.met + 6 * b.N, 3 * nb, cudaMemcpyDeviceToHost));
  if (dxyz) {
    if (!b.dxyz) return fail(NUC3D_ESTATE, "block %d has no dxyz metrics", bi);
    CUDA_TRY(cudaMemcpy(dxyz, b.dxyz, 9 * nb, cudaMemcpyDeviceToHost));
  }
  return NUC3D_OK;
}

}  // extern "C"

namespace {

PFN_cuTensorMapEncodeTiled g_encode = nullptr;
std::once_flag g_encode_once;

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  std::call_once(g_encode_once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  });
  return g_encode;
}

bool explicit_scheme(int s) {
  return s == SCH_WENO5JS || s == SCH_WENO5Z || s == SCH_WENO7JS || s == SCH_WENO3JS ||
         s == SCH_UPWIND1;
}

// A 3D (ncomp = 0) or 4D tiled map over an [ncomp][nz][ny][nx] array of doubles.
bool encode_map(CUtensorMap *m, const void *base, const int n[3], int ncomp, const int box[3],
                int box_comp) {
  const cuuint64_t dims[4] = {(cuuint64_t)n[0], (cuuint64_t)n[1], (cuuint64_t)n[2], (cuuint64_t)ncomp};
  const cuuint64_t nx8 = (cuuint64_t)n[0] * 8;
  const cuuint64_t strides[3] = {nx8, nx8 * n[1], nx8 * n[1] * n[2]};
  const cuuint32_t bdim[4] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2],
                              (cuuint32_t)box_comp};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = tensor_map_encoder()(
      m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, ncomp ? 4 : 3, const_cast<void *>(base), dims, strides,
      bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Tensor maps of the pipelined sweeps for the current tile shapes, or pipelining off
// (L.d_maps = null) where it does not apply: Navier-Stokes (its viscous tiles are not
// staged), a block with an odd nx (TMA needs 16-byte row strides), or switched off.
int build_maps(nuc3d_ctx *c) {
  Launch &L = c->L;
  L.d_maps = nullptr;
  L.pipe_grid = 0;
  bool ok = c->use_pipe;
  for (const HostBlock &b : c->blocks) ok = ok && b.n[0] % 2 == 0;
  if (!ok) return NUC3D_OK;
  if (!tensor_map_encoder()) return NUC3D_OK;  // no TMA encoder in this driver: plain sweeps
  const int nbk = (int)c->blocks.size();
  std::vector<CUtensorMap> h((size_t)nbk * 3 * kMapKinds);
  std::memset(h.data(), 0, h.size() * sizeof(CUtensorMap));
  for (int bi = 0; bi < nbk; ++bi) {
    const HostBlock &b = c->blocks[bi];
    for (int d = 0; d < 3; ++d) {
      if (!explicit_scheme(c->P.scheme[d])) continue;
      CUtensorMap *m = &h[((size_t)bi * 3 + d) * kMapKinds];
      const int tw = tile_w(L.shape[d]), tl = tile_l(L.shape[d]), r = scheme_halo(c->P.scheme[d]);
      int hb[3], ob[3];
      pipe_box(d, tw, tl, r, true, hb);
      pipe_box(d, tw, tl, r, false, ob);
      bool e = true;
      for (int s = 0; s < 3; ++s) e = e && encode_map(&m[kMapQ0 + s], b.q[s], b.n, 5, hb, 5);
      e = e && encode_map(&m[kMapJac], b.jac, b.n, 0, hb, 0);
      e = e && encode_map(&m[kMapMet], b.met, b.n, 9, hb, 3);
      e = e && encode_map(&m[kMapMetO], b.met, b.n, 9, ob, 6);
      e = e && encode_map(&m[kMapRhs], b.rhs, b.n, 5, ob, 5);
      e = e && encode_map(&m[kMapQn], b.q[0], b.n, 5, ob, 5);
      if (!e) return fail(NUC3D_ECUDA, "block %d direction %d: tensor map encoding failed", bi, d);
    }
  }
  cudaSetDevice(c->device);
  if (!c->d_maps) CUDA_TRY(cudaMalloc(&c->d_maps, h.size() * sizeof(CUtensorMap)));
  CUDA_TRY(cudaMemcpy(c->d_maps, h.data(), h.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  L.d_maps = c->d_maps;
  L.pipe_grid = 2 * sms;  // two persistent CTAs per SM
  L.pipe_dirs = c->pipe_mask;
  return NUC3D_OK;
}

}  // namespace

extern "C" {

// Directions whose compact scheme (crweno5, hccs; not the whole-line hccs77 system) runs
// the fused compact_line_kernel: the throughput build, every block's line at most
// kLineMax cells with at least 2 rows in its system, and the kernel's tile fitting in
// shared memory (a Navier-Stokes tile of several lines may not).
static void set_line_dirs(nuc3d_ctx *c) {
  int dirs = 0;
  for (int d = 0; d < 3 && !c->exact && c->compact_fused; ++d) {
    const int sc = c->P.scheme[d];
    if (sc != SCH_CRWENO5 && sc != SCH_HCCS) continue;
    bool ok = nuc3d::fast::compact_line_smem(d, sc, c->P.model == MODEL_NS) <= kSmemOptin;
    for (const HostBlock &b : c->blocks)
      ok = ok && b.n[d] <= kLineMax && b.n[d] - 2 * c->P.ts[d] + 1 >= 2;
    if (ok) dirs |= 1 << d;
  }
  c->L.line_dirs = dirs;
}

int nuc3d_finalize(nuc3d_ctx *c) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (c->finalized) return fail(NUC3D_ESTATE, "already finalized");
  const int nbk = (int)c->blocks.size();
  if (nbk == 0) return fail(NUC3D_ESTATE, "no blocks");
  const int bfs = c->P.bfs;
  for (int bi = 0; bi < nbk; ++bi) {
    const HostBlock &b = c->blocks[bi];
    if (!b.metrics) return fail(NUC3D_ESTATE, "block %d has no metrics", bi);
    for (int f = 0; f < 6; ++f) {
      const int d = f >> 1;
      if (b.bc_type[f] == -1) {
        if (b.bc_id[f] == BC_SYMM && !b.dxyz)
          return fail(NUC3D_EINVAL, "block %d face %d is a symmetry face: dxyz metrics required", bi, f);
        continue;
      }
      const int nbi = b.bc_type[f], nf = b.bc_id[f];
      if (nbi >= nbk) return fail(NUC3D_EINVAL, "block %d face %d: neighbour %d does not exist", bi, f, nbi);
      if (nf < 0 || nf > 5) return fail(NUC3D_EINVAL, "block %d face %d: neighbour face %d", bi, f, nf);
      // The reference exchanges one direction at a time (src/euler3d.cpp:318-330), so a
      // face can only pair with a face of the same direction.
      if ((nf >> 1) != d)
        return fail(NUC3D_EINVAL, "block %d face %d pairs with face %d of another direction", bi, f, nf);
      const HostBlock &o = c->blocks[nbi];
      auto area = [](const HostBlock &h, int dd) {
        return dd == 0 ? (long long)h.n[1] * h.n[2]
                       : (dd == 1 ? (long long)h.n[2] * h.n[0] : (long long)h.n[0] * h.n[1]);
      };
      if (area(b, d) != area(o, d))
        return fail(NUC3D_EINVAL, "block %d face %d and block %d face %d have different sizes", bi, f,
                    nbi, nf);
      if (o.n[d] < bfs) return fail(NUC3D_EINVAL, "block %d is thinner than the ghost width", nbi);
    }
  }
  // device descriptors
  std::vector<BlockDev> hb(nbk);
  for (int bi = 0; bi < nbk; ++bi) {
    const HostBlock &b = c->blocks[bi];
    BlockDev &d = hb[bi];
    std::memset(&d, 0, sizeof(d));
    for (int k = 0; k < 3; ++k) d.n[k] = b.n[k];
    d.N = b.N;
    for (int s = 0; s < 3; ++s) d.q[s] = b.q[s];
    d.rhs = b.rhs;
    d.jac = b.jac;
    for (int k = 0; k < 3; ++k) d.met[k] = b.met + 3 * k * b.N;
    d.dxyz = b.dxyz;
    d.prim = b.prim;
    d.vis = b.vis;
    d.dvis = b.dvis;
    d.ghost = b.ghost;
    d.fh = b.fh;
    d.rows = b.rows;
    d.dres = b.dres;
    for (int f = 0; f < 6; ++f) d.goff[f] = b.goff[f];
    for (int f = 0; f < 6; ++f) {
      d.face[f].type = b.bc_type[f];
      d.face[f].id = b.bc_id[f];
      for (int v = 0; v < 5; ++v) d.face[f].bcv[v] = b.bcv[f][v];
    }
    set_tile_divisors(d, c->L.shape);
  }
  c->hdesc = hb;
  cudaSetDevice(c->device);
  CUDA_TRY(cudaMalloc(&c->d_blocks, nbk * sizeof(BlockDev)));
  CUDA_TRY(cudaMemcpy(c->d_blocks, hb.data(), nbk * sizeof(BlockDev), cudaMemcpyHostToDevice));
  Launch &L = c->L;
  L.d_blocks = c->d_blocks;
  L.d_state = c->d_state;
  L.P = c->P;
  L.stream = c->stream;
  for (int d = 0; d < 3; ++d) {
    L.tm_dir[d].nblocks = nbk;
    L.tm_dir[d].tile_start[0] = 0;
    L.tm_sys[d].nblocks = nbk;
    L.tm_sys[d].tile_start[0] = 0;
    L.tm_line[d].nblocks = nbk;
    L.tm_line[d].tile_start[0] = 0;
  }
  L.tm_cells.nblocks = nbk;
  L.tm_cells.tile_start[0] = 0;
  for (int bi = 0; bi < nbk; ++bi) {
    const HostBlock &b = c->blocks[bi];
    for (int d = 0; d < 3; ++d) {
      L.tm_dir[d].tile_start[bi + 1] =
          L.tm_dir[d].tile_start[bi] + nuc3d::exact::tile_count(d, b.n, L.shape[d]);
      const long long nsys = 10 * (b.N / b.n[d]);
      L.tm_sys[d].tile_start[bi + 1] = L.tm_sys[d].tile_start[bi] + (int)((nsys + 255) / 256);
      {  // fused compact sweep: groups of tile_w(line_shape(d)) lanes per outer index
        const long long nW = d == 0 ? b.n[1] : b.n[0], nO = d == 2 ? b.n[1] : b.n[2];
        const long long lw = tile_w(line_shape(d));
        L.tm_line[d].tile_start[bi + 1] = L.tm_line[d].tile_start[bi] + (int)(((nW + lw - 1) / lw) * nO);
      }
    }
    L.tm_cells.tile_start[bi + 1] = L.tm_cells.tile_start[bi] + (int)((b.N + 255) / 256);
  }
  // physical faces for the BC ghost pass
  std::vector<FaceJobs> jv(1);
  FaceJobs &J = jv[0];
  std::memset(&J, 0, sizeof(J));
  for (int bi = 0; bi < nbk; ++bi) {
    const HostBlock &b = c->blocks[bi];
    for (int f = 0; f < 6; ++f) {
      if (b.bc_type[f] != -1) continue;
      const int d = f >> 1;
      const long long area = d == 0 ? (long long)b.n[1] * b.n[2]
                                    : (d == 1 ? (long long)b.n[2] * b.n[0] : (long long)b.n[0] * b.n[1]);
      J.block[J.njobs] = bi;
      J.face[J.njobs] = (unsigned char)f;
      J.start[J.njobs + 1] = J.start[J.njobs] + (int)((area + 255) / 256);
      ++J.njobs;
    }
  }
  L.bc_tiles = J.start[J.njobs];
  CUDA_TRY(cudaMalloc(&c->d_jobs, sizeof(FaceJobs)));
  CUDA_TRY(cudaMemcpy(c->d_jobs, &J, sizeof(FaceJobs), cudaMemcpyHostToDevice));
  L.d_jobs = c->d_jobs;
  set_line_dirs(c);
  // residual workspace: one partial sum per zeta tile (any tile shape, or per line of the
  // fused compact sweep) or per cell tile
  {
    long long nt = std::max(L.tm_cells.tile_start[nbk], L.tm_line[2].tile_start[nbk]);
    for (int sh = 0; sh < kTileShapes; ++sh) {
      long long z = 0;
      for (int bi = 0; bi < nbk; ++bi) z += nuc3d::exact::tile_count(2, c->blocks[bi].n, sh);
      nt = std::max(nt, z);
    }
    CUDA_TRY(cudaMalloc(&c->d_res_part, nt * sizeof(double)));
    CUDA_TRY(cudaMalloc(&c->d_res_last, nbk * sizeof(double)));
    CUDA_TRY(cudaMemset(c->d_res_last, 0, nbk * sizeof(double)));
    c->P.res_part = L.P.res_part = c->d_res_part;
    L.d_res_last = c->d_res_last;
  }
  if (int r = build_maps(c)) return r;
  c->finalized = true;
  return NUC3D_OK;
}

int nuc3d_block_set_q(nuc3d_ctx *c, int bi, const double *q) {
  if (!c || !q || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  HostBlock &b = c->blocks[bi];
  cudaSetDevice(c->device);
  CUDA_TRY(cudaMemcpyAsync(b.q[0], q, 5 * (size_t)b.N * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
  return NUC3D_OK;
}

int nuc3d_block_get_q(nuc3d_ctx *c, int bi, double *q) {
  if (!c || !q || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  HostBlock &b = c->blocks[bi];
  cudaSetDevice(c->device);
  CUDA_TRY(cudaMemcpyAsync(q, b.q[0], 5 * (size_t)b.N * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return NUC3D_OK;
}

int nuc3d_block_q_device(nuc3d_ctx *c, int bi, double **dev_q) {
  if (!c || !dev_q || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  *dev_q = c->blocks[bi].q[0];
  return NUC3D_OK;
}

static int copy_out(nuc3d_ctx *c, int bi, double *dst, const double *src, int ncomp) {
  if (!c || !dst || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  if (!src) return fail(NUC3D_ESTATE, "this field is not allocated for the configured model");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(dst, src, (size_t)ncomp * c->blocks[bi].N * sizeof(double),
                      cudaMemcpyDeviceToHost));
  return NUC3D_OK;
}

int nuc3d_block_get_rhs(nuc3d_ctx *c, int bi, double *rhs) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  return copy_out(c, bi, rhs, c->blocks[bi].rhs, 5);
}
int nuc3d_block_get_prim(nuc3d_ctx *c, int bi, double *prim) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  return copy_out(c, bi, prim, c->blocks[bi].prim, 4);
}
int nuc3d_block_get_vis(nuc3d_ctx *c, int bi, double *vis) {
  if (!c || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  return copy_out(c, bi, vis, c->blocks[bi].vis, 12);
}

int nuc3d_debug_get(nuc3d_ctx *c, int bi, int tap, double *out) {
  if (!c || !out || bi < 0 || bi >= (int)c->blocks.size() || tap < 0 || tap >= 15)
    return fail(NUC3D_EINVAL, "bad argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  const int dir = tap % 3, kind = tap / 3;
  const HostBlock &b = c->blocks[bi];
  const long long N = b.N, nl = b.N / b.n[dir], NF = (long long)(b.n[dir] + 1) * nl;
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  StepState s0;  // the taps leave the step state (status, reset count) as it was
  CUDA_TRY(cudaMemcpy(&s0, c->d_state, sizeof(s0), cudaMemcpyDeviceToHost));
  double *buf = nullptr;
  CUDA_TRY(cudaMalloc(&buf, sizeof(double) * (size_t)(15 * N + 10 * NF)));
  double *const o[5] = {buf, buf + 5 * N, buf + 10 * N, buf + 10 * N + 5 * NF, buf + 10 * N + 10 * NF};
  cudaError_t e = c->exact ? nuc3d::exact::run_taps(c->L, bi, dir, (int)nl, o)
                           : nuc3d::fast::run_taps(c->L, bi, dir, (int)nl, o);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  const size_t n = (size_t)5 * (kind == 2 || kind == 3 ? NF : N);
  if (e == cudaSuccess) e = cudaMemcpy(out, o[kind], n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_state, &s0, sizeof(s0), cudaMemcpyHostToDevice);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(NUC3D_ECUDA, "debug taps: %s", cudaGetErrorString(e));
  return NUC3D_OK;
}

static int check_status(nuc3d_ctx *c) {
  StepState s;
  CUDA_TRY(cudaMemcpy(&s, c->d_state, sizeof(s), cudaMemcpyDeviceToHost));
  if (s.status & ST_PIPE_TIMEOUT)
    return fail(NUC3D_ECUDA, "kernel status 0x%x: a pipelined sweep's wait for its loads gave up",
                s.status);
  if (s.status & (ST_NEG_PRESSURE | ST_NONFINITE | ST_BAD_LAUNCH))
    return fail(NUC3D_ENUMERIC, "kernel status 0x%x (negative pressure / non-finite state)", s.status);
  return NUC3D_OK;
}

int nuc3d_rhs(nuc3d_ctx *c, double *dt_local) { return nuc3d_rhs_stage(c, 0, dt_local); }

int nuc3d_rhs_stage(nuc3d_ctx *c, int stage, double *dt_local) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (stage < 0 || stage > 2) return fail(NUC3D_EINVAL, "stage %d not in 0..2", stage);
  cudaSetDevice(c->device);
  CUDA_TRY(cudaMemsetAsync(&c->d_state->max_eig_bits, 0, sizeof(unsigned long long), c->stream));
  CUDA_TRY(c->stage(stage, false, true));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  StepState s;
  CUDA_TRY(cudaMemcpy(&s, c->d_state, sizeof(s), cudaMemcpyDeviceToHost));
  if (dt_local) {
    double me;
    std::memcpy(&me, &s.max_eig_bits, sizeof(me));
    *dt_local = 1.0 / me;
  }
  return check_status(c);
}

int nuc3d_rk_stage(nuc3d_ctx *c, int stage, double dt) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (stage < 0 || stage > 2) return fail(NUC3D_EINVAL, "stage %d not in 0..2", stage);
  if (!(dt > 0.0)) return fail(NUC3D_EINVAL, "dt must be > 0");
  cudaSetDevice(c->device);
  CUDA_TRY(c->exact ? nuc3d::exact::run_rk_stage(c->L, stage, dt)
                    : nuc3d::fast::run_rk_stage(c->L, stage, dt));
  return NUC3D_OK;
}

int nuc3d_get_residual(nuc3d_ctx *c, double *res) {
  if (!c || !res) return fail(NUC3D_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  unsigned long long bits = 0;
  CUDA_TRY(cudaMemcpy(&bits, &c->d_state->res_bits, sizeof(bits), cudaMemcpyDeviceToHost));
  std::memcpy(res, &bits, sizeof(double));
  return NUC3D_OK;
}

int nuc3d_step(nuc3d_ctx *c, int nsteps) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (nsteps < 0) return fail(NUC3D_EINVAL, "nsteps < 0");
  cudaSetDevice(c->device);
  if (c->use_graph && !c->gexec) {
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = c->one_step();
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(NUC3D_ECUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    c->graph = g;
    CUDA_TRY(cudaGraphInstantiate(&c->gexec, c->graph, 0));
  }
  for (int s = 0; s < nsteps; ++s) {
    if (c->use_graph) CUDA_TRY(cudaGraphLaunch(c->gexec, c->stream));
    else CUDA_TRY(c->one_step());
  }
  return NUC3D_OK;
}

// Two timing events, destroyed on every way out of the scope that made them.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Copy chunks of nuc3d_solve_host: small enough that the upload of chunk j (next step)
// trails the download of chunk j (this step) by little, large enough that each copy runs
// at full PCIe speed.
#ifndef NUC3D_HOST_CHUNK_MB
#define NUC3D_HOST_CHUNK_MB 16  // measured at 256^3: 4 and 64 MiB chunks 1% slower
#endif
constexpr size_t kHostChunk = (size_t)NUC3D_HOST_CHUNK_MB << 20;

// nuc3d_solve_host for one Euler block with explicit schemes, as a copy/compute pipeline
// over z-slabs (the zeta sweep's z-chunks): the upload of slab s is followed at once by
// stage 0's BC, xi and eta work on that slab (their lines stay inside a z-plane), and
// stage 2 runs slab by slab (BC, xi, eta, then zeta over the slab: it reads the slab's own
// RHS and the stage state stage 1 completed), each slab's download following its zeta
// sweep, while the copy engines move the other slabs.  The kernels and tiles are one_step's, so the results are too.
// nuc3d_solve_host's slab pipeline runs the zeta sweep in 8 x 32 tiles whatever the
// context's zeta shape: slabs of 32 planes instead of 64 halve the stretch between a step's
// last upload and its first download, when the copy engines idle (the 256^3 Euler step:
// 17.8 against 19.6 ms; the shape changes which CTA computes a cell, not the results).
constexpr int kHostZetaShape = 1;

static bool slab_pipeline_ok(const nuc3d_ctx *c) {
  if (!c->host_pipeline || c->blocks.size() != 1 || c->P.model != MODEL_EULER || c->P.sensor)
    return false;
  for (int d = 0; d < 3; ++d)
    if (c->P.scheme[d] == SCH_CRWENO5 || c->P.scheme[d] == SCH_HCCS || c->P.scheme[d] == SCH_HCCS77)
      return false;
  return c->blocks[0].n[2] >= 2 * tile_l(kHostZetaShape);
}

#ifndef NUC3D_HOST_PIECES
#define NUC3D_HOST_PIECES 8  // copy pieces per slab (256^3: 17.45 ms per step against 17.66 with 4)
#endif
constexpr int kHostPieces = NUC3D_HOST_PIECES;

// nuc3d_solve_host's per-block stage 2 (contexts of several blocks, explicit schemes, no
// learned sensor): the block sweeps of run_stage_sweeps.
static bool block_pipeline_ok(const nuc3d_ctx *c) {
  if (!c->host_pipeline || c->blocks.size() < 2 || c->P.sensor) return false;
  for (int d = 0; d < 3; ++d)
    if (c->P.scheme[d] == SCH_CRWENO5 || c->P.scheme[d] == SCH_HCCS || c->P.scheme[d] == SCH_HCCS77)
      return false;
  return true;
}

// The slabs of nuc3d_solve_host's pipeline are whole zeta chunks; a last chunk thinner than
// kSlabMin planes joins the slab before it, so that every slab holds more planes than a
// zeta stencil reaches (4) and a slab's stencils touch only its two neighbours' cells (and
// the z faces' ghost fluxes only in the end slabs).
constexpr int kSlabMin = 8;
static int host_slab_count(const nuc3d_ctx *c) {
  const int nz = c->blocks[0].n[2], TLz = tile_l(kHostZetaShape), nchunk = (nz + TLz - 1) / TLz;
  return (nchunk > 1 && nz - (nchunk - 1) * TLz < kSlabMin) ? nchunk - 1 : nchunk;
}

static int apply_shapes(nuc3d_ctx *c, const int shape[3]);

static int solve_host_slabs(nuc3d_ctx *c, double *q_host, int nsteps) {
  const HostBlock &b = c->blocks[0];
  const int nx = b.n[0], ny = b.n[1], nz = b.n[2];
  const int *sh = c->L.shape;
  const int TLz = tile_l(sh[2]), nchunk = (nz + TLz - 1) / TLz, ns = host_slab_count(c);
  const int zper = ((nx + tile_w(sh[2]) - 1) / tile_w(sh[2])) * ny;                      // zeta tiles per chunk
  const int xper = ((nx + tile_l(sh[0]) - 1) / tile_l(sh[0])) * ((ny + tile_w(sh[0]) - 1) / tile_w(sh[0]));
  const int yper = ((ny + tile_l(sh[1]) - 1) / tile_l(sh[1])) * ((nx + tile_w(sh[1]) - 1) / tile_w(sh[1]));
  auto slab_chunks = [&](int s, int &c0, int &c1) {
    c0 = s;
    c1 = s == ns - 1 ? nchunk : s + 1;
  };
  // with both z faces physical, a slab's stage-s zeta sweep needs the stage-(s-1) state of
  // its own and its neighbours' cells only, so the stages run as a wavefront over the
  // slabs and the first slab's download starts after 3 slabs of stage 0's zeta sweep, 2 of
  // stage 1 and 1 of stage 2; a z face joined to the block itself makes every slab depend
  // on every other, and then stages 0 (zeta) and 1 run over the whole block first
  const bool wave = b.bc_type[4] < 0 && b.bc_type[5] < 0;
  // copies move pieces of kHostPieces z-ranges per slab: the upload of a piece waits only
  // for the download of the same piece, so the last slab's round trip is short
  const int np = ns * kHostPieces;
  for (auto *v : {&c->ev_up, &c->ev_zeta, &c->ev_down})
    while ((int)v->size() < np) {
      cudaEvent_t ev;
      CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      v->push_back(ev);
    }
  const size_t plane = (size_t)nx * ny;
  auto slab_range = [&](int s, int &k0, int &k1) {
    int c0, c1;
    slab_chunks(s, c0, c1);
    k0 = c0 * TLz;
    k1 = std::min(nz, c1 * TLz);
  };
  auto piece_range = [&](int p, int &k0, int &k1) {
    const int q = p % kHostPieces;
    int s0, s1;
    slab_range(p / kHostPieces, s0, s1);
    const int len = s1 - s0;
    k0 = s0 + len * q / kHostPieces;
    k1 = s0 + len * (q + 1) / kHostPieces;
  };
  auto copy_piece = [&](int p, bool up, cudaStream_t st) -> cudaError_t {
    int k0, k1;
    piece_range(p, k0, k1);
    if (k1 <= k0) return cudaSuccess;
    // the piece's planes of the five components: one strided copy (5 rows, pitch N), or
    // five copies where the pitch exceeds what the copy engines take (2^31 - 1 bytes)
    const size_t off = (size_t)k0 * plane, width = (size_t)(k1 - k0) * plane * sizeof(double);
    const size_t pitch = (size_t)b.N * sizeof(double);
    const cudaMemcpyKind kind = up ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    if (pitch <= (size_t)0x7fffffff)
      return up ? cudaMemcpy2DAsync(b.q[0] + off, pitch, q_host + off, pitch, width, 5, kind, st)
                : cudaMemcpy2DAsync(q_host + off, pitch, b.q[0] + off, pitch, width, 5, kind, st);
    for (int v = 0; v < 5; ++v) {
      const size_t o = (size_t)v * b.N + off;
      cudaError_t e = up ? cudaMemcpyAsync(b.q[0] + o, q_host + o, width, kind, st)
                         : cudaMemcpyAsync(q_host + o, b.q[0] + o, width, kind, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  const Launch &L = c->L;
  auto run = [&](auto fast_fn, auto exact_fn) { return c->exact ? exact_fn() : fast_fn(); };
  auto zeta0 = [&](int s) {
    int c0, c1;
    slab_chunks(s, c0, c1);
    return run([&] { return nuc3d::fast::run_stage0_zeta(L, c0 * zper, c1 * zper); },
               [&] { return nuc3d::exact::run_stage0_zeta(L, c0 * zper, c1 * zper); });
  };
  auto stage_slab = [&](int stage, int s) {
    int k0, k1, c0, c1;
    slab_range(s, k0, k1);
    slab_chunks(s, c0, c1);
    return run([&] { return nuc3d::fast::run_stage_slab(L, stage, k0, k1, k0 * xper, k1 * xper, k0 * yper,
                                                        k1 * yper, c0 * zper, c1 * zper); },
               [&] { return nuc3d::exact::run_stage_slab(L, stage, k0, k1, k0 * xper, k1 * xper, k0 * yper,
                                                         k1 * yper, c0 * zper, c1 * zper); });
  };
  auto stage2_slab = [&](int s) -> cudaError_t {
    cudaError_t e = stage_slab(2, s);
    if (e != cudaSuccess) return e;
    return cudaEventRecord(c->ev_zeta[s], c->stream);
  };
  CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
  CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_start, 0));
  for (int step = 0; step < nsteps; ++step) {
    for (int p = 0; p < np; ++p) {
      // the host piece is read only once the previous step's download has written it
      if (step > 0) CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_down[p], 0));
      CUDA_TRY(copy_piece(p, true, c->h2d));
      CUDA_TRY(cudaEventRecord(c->ev_up[p], c->h2d));
    }
    CUDA_TRY(cudaMemsetAsync(&c->d_state->max_eig_bits, 0, sizeof(unsigned long long), c->stream));
    // stage 0's xi/eta lines lie in z-planes: each piece's share runs as soon as it is in,
    // so only the last piece's remains between the step's last upload and its dt
    for (int p = 0; p < np; ++p) {
      int k0, k1;
      piece_range(p, k0, k1);
      if (k1 <= k0) continue;
      CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_up[p], 0));
      CUDA_TRY(run([&] { return nuc3d::fast::run_stage0_slab(L, k0, k1, k0 * xper, k1 * xper, k0 * yper, k1 * yper); },
                   [&] { return nuc3d::exact::run_stage0_slab(L, k0, k1, k0 * xper, k1 * xper, k0 * yper, k1 * yper); }));
    }
    if (wave) {
      for (int w = 0; w < ns + 2; ++w) {
        if (w < ns) CUDA_TRY(zeta0(w));
        if (w >= 1 && w - 1 < ns) CUDA_TRY(stage_slab(1, w - 1));
        if (w >= 2) CUDA_TRY(stage2_slab(w - 2));
      }
    } else {
      CUDA_TRY(run([&] { return nuc3d::fast::run_stage0_zeta(L, 0, nchunk * zper); },
                   [&] { return nuc3d::exact::run_stage0_zeta(L, 0, nchunk * zper); }));
      CUDA_TRY(run([&] { return nuc3d::fast::run_stage(L, 1, true, false); },
                   [&] { return nuc3d::exact::run_stage(L, 1, true, false); }));
      for (int s = 0; s < ns; ++s) CUDA_TRY(stage2_slab(s));
    }
    if (L.d_res_last)
      CUDA_TRY(run([&] { return nuc3d::fast::run_residual(L, false); },
                   [&] { return nuc3d::exact::run_residual(L, false); }));
    for (int p = 0; p < np; ++p) {
      if (p % kHostPieces == 0) CUDA_TRY(cudaStreamWaitEvent(c->d2h, c->ev_zeta[p / kHostPieces], 0));
      CUDA_TRY(copy_piece(p, false, c->d2h));
      CUDA_TRY(cudaEventRecord(c->ev_down[p], c->d2h));
    }
  }
  CUDA_TRY(cudaEventRecord(c->ev_end, c->d2h));
  CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_end, 0));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int nuc3d_set_host_pipeline(nuc3d_ctx *c, int on) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  c->host_pipeline = on != 0;
  return NUC3D_OK;
}

int nuc3d_get_host_pipeline(nuc3d_ctx *c, int *on) {
  if (!c || !on) return fail(NUC3D_EINVAL, "null argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  *on = slab_pipeline_ok(c) ? host_slab_count(c) : 0;
  return NUC3D_OK;
}

int nuc3d_solve_host(nuc3d_ctx *c, double *const *q_host, int nsteps) {
  if (!c || !q_host) return fail(NUC3D_EINVAL, "null argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (nsteps < 0) return fail(NUC3D_EINVAL, "nsteps < 0");
  for (size_t b = 0; b < c->blocks.size(); ++b)
    if (!q_host[b]) return fail(NUC3D_EINVAL, "q_host[%zu] is null", b);
  cudaSetDevice(c->device);
  if (!c->h2d) {
    CUDA_TRY(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
    for (cudaEvent_t *ev : {&c->ev_start, &c->ev_h2d, &c->ev_step, &c->ev_end})
      CUDA_TRY(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  }
  if (slab_pipeline_ok(c)) {
    const int keep[3] = {c->L.shape[0], c->L.shape[1], c->L.shape[2]};
    const int host[3] = {keep[0], keep[1], kHostZetaShape};
    if (keep[2] != kHostZetaShape)
      if (int r = apply_shapes(c, host)) return r;
    int r = solve_host_slabs(c, q_host[0], nsteps);
    if (keep[2] != kHostZetaShape) {
      const int r2 = apply_shapes(c, keep);
      if (r == NUC3D_OK) r = r2;
    }
    return r;
  }
  struct Chunk { int b; size_t off, bytes; };
  std::vector<Chunk> chunks;
  for (size_t b = 0; b < c->blocks.size(); ++b) {
    const size_t total = 5 * (size_t)c->blocks[b].N * sizeof(double);
    for (size_t off = 0; off < total; off += kHostChunk)
      chunks.push_back({(int)b, off, std::min(kHostChunk, total - off)});
  }
  while (c->ev_chunk.size() < chunks.size()) {
    cudaEvent_t ev;
    CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    c->ev_chunk.push_back(ev);
  }
  // several blocks (explicit schemes, no sensor): stage 2 block by block, so that each
  // block's download starts after its own zeta sweep instead of after the whole step
  const int nb = (int)c->blocks.size();
  const bool by_block = block_pipeline_ok(c);
  while (by_block && (int)c->ev_zeta.size() < nb) {
    cudaEvent_t ev;
    CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    c->ev_zeta.push_back(ev);
  }
  const Launch &L = c->L;
  auto run = [&](auto fast_fn, auto exact_fn) { return c->exact ? exact_fn() : fast_fn(); };
  auto dev = [&](const Chunk &k) { return reinterpret_cast<char *>(c->blocks[k.b].q[0]) + k.off; };
  auto host = [&](const Chunk &k) { return reinterpret_cast<char *>(q_host[k.b]) + k.off; };
  // uploads start after the work already queued on the context's stream
  CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
  CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_start, 0));
  for (int s = 0; s < nsteps; ++s) {
    for (size_t j = 0; j < chunks.size(); ++j) {
      // the host chunk is read only once the previous step's download has written it
      if (s > 0) CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_chunk[j], 0));
      CUDA_TRY(cudaMemcpyAsync(dev(chunks[j]), host(chunks[j]), chunks[j].bytes,
                               cudaMemcpyHostToDevice, c->h2d));
    }
    CUDA_TRY(cudaEventRecord(c->ev_h2d, c->h2d));
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_h2d, 0));
    if (by_block) {
      // stages 0 and 1 whole; stage 2's ghost fluxes (and NS gradients) of every block,
      // then each block's sweeps, whose last (zeta) releases that block's download
      CUDA_TRY(cudaMemsetAsync(&c->d_state->max_eig_bits, 0, sizeof(unsigned long long), c->stream));
      CUDA_TRY(c->stage(0, true, true));
      CUDA_TRY(c->stage(1, true, false));
      CUDA_TRY(run([&] { return nuc3d::fast::run_stage_pre(L, 2); },
                   [&] { return nuc3d::exact::run_stage_pre(L, 2); }));
      for (int b = 0; b < nb; ++b) {
        CUDA_TRY(run([&] { return nuc3d::fast::run_stage_sweeps(L, 2, b, b + 1); },
                     [&] { return nuc3d::exact::run_stage_sweeps(L, 2, b, b + 1); }));
        CUDA_TRY(cudaEventRecord(c->ev_zeta[b], c->stream));
      }
      if (L.d_res_last)
        CUDA_TRY(run([&] { return nuc3d::fast::run_residual(L, false); },
                     [&] { return nuc3d::exact::run_residual(L, false); }));
    } else {
      if (int r = nuc3d_step(c, 1)) return r;
      CUDA_TRY(cudaEventRecord(c->ev_step, c->stream));
      CUDA_TRY(cudaStreamWaitEvent(c->d2h, c->ev_step, 0));
    }
    for (size_t j = 0; j < chunks.size(); ++j) {
      if (by_block && (j == 0 || chunks[j].b != chunks[j - 1].b))
        CUDA_TRY(cudaStreamWaitEvent(c->d2h, c->ev_zeta[chunks[j].b], 0));
      CUDA_TRY(cudaMemcpyAsync(host(chunks[j]), dev(chunks[j]), chunks[j].bytes,
                               cudaMemcpyDeviceToHost, c->d2h));
      CUDA_TRY(cudaEventRecord(c->ev_chunk[j], c->d2h));
    }
  }
  // the context's stream (and events recorded on it) cover the last download
  CUDA_TRY(cudaEventRecord(c->ev_end, c->d2h));
  CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_end, 0));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

// Tile shapes of the sweeps: tile divisors of every block (device descriptors) and the
// per-direction tile maps; the captured step graph holds the old launches, so it goes.
static int apply_shapes(nuc3d_ctx *c, const int shape[3]) {
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int nbk = (int)c->blocks.size();
  for (int d = 0; d < 3; ++d) c->L.shape[d] = shape[d];
  for (int bi = 0; bi < nbk; ++bi) set_tile_divisors(c->hdesc[bi], c->L.shape);
  CUDA_TRY(cudaMemcpy(c->d_blocks, c->hdesc.data(), nbk * sizeof(BlockDev), cudaMemcpyHostToDevice));
  for (int bi = 0; bi < nbk; ++bi)
    for (int d = 0; d < 3; ++d)
      c->L.tm_dir[d].tile_start[bi + 1] =
          c->L.tm_dir[d].tile_start[bi] + nuc3d::exact::tile_count(d, c->blocks[bi].n, shape[d]);
  c->drop_graph();
  return build_maps(c);
}

static bool compact_scheme(int s) { return s == SCH_CRWENO5 || s == SCH_HCCS || s == SCH_HCCS77; }

int nuc3d_set_tiles(nuc3d_ctx *c, const int shape[3]) {
  if (!c || !shape) return fail(NUC3D_EINVAL, "null argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  for (int d = 0; d < 3; ++d) {
    if (shape[d] < 0 || shape[d] >= kTileShapes)
      return fail(NUC3D_EINVAL, "direction %d: tile shape %d not in 0..%d", d, shape[d], kTileShapes - 1);
    if (compact_scheme(c->P.scheme[d]) && shape[d] != 0)
      return fail(NUC3D_EINVAL, "direction %d: compact schemes run tile shape 0", d);
  }
  return apply_shapes(c, shape);
}

int nuc3d_get_tiles(nuc3d_ctx *c, int shape[3]) {
  if (!c || !shape) return fail(NUC3D_EINVAL, "null argument");
  for (int d = 0; d < 3; ++d) shape[d] = c->L.shape[d];
  return NUC3D_OK;
}

namespace {
// Tile shapes chosen by nuc3d_autotune, per grid: block extents, schemes, model, build.
std::mutex g_tune_mutex;
std::map<std::string, std::array<int, 4>> g_tune_cache;  // shapes, pipelined directions

std::string tune_key(const nuc3d_ctx *c) {
  std::string k = c->exact ? "x" : "f";
  k += c->P.model == MODEL_NS ? "ns" : "eu";
  k += c->P.sensor ? "h" : "p";
  k += c->use_pipe ? "t" : "n";
  for (int d = 0; d < 3; ++d) k += ":" + std::to_string(c->P.scheme[d]) + "." + std::to_string(c->P.vis[d]);
  for (const HostBlock &b : c->blocks)
    k += "|" + std::to_string(b.n[0]) + "x" + std::to_string(b.n[1]) + "x" + std::to_string(b.n[2]);
  return k;
}
}  // namespace

int nuc3d_autotune(nuc3d_ctx *c, int reps, int shape_out[3], double ms_out[9]) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (reps < 1) reps = 3;
  const std::string key = tune_key(c);
  std::array<int, 4> best = {0, 0, 0, 0};  // shapes, then the pipelined directions (bits)
  bool cached = false;
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) { best = it->second; cached = true; }
  }
  if (ms_out)
    for (int i = 0; i < 9; ++i) ms_out[i] = -1.0;
  if (!cached) {
    cudaSetDevice(c->device);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    unsigned status0 = 0;  // the timing sweeps must not leave status bits or resets behind
    unsigned long long resets0 = 0;
    CUDA_TRY(cudaMemcpy(&status0, &c->d_state->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&resets0, &c->d_state->reset_cells, sizeof(resets0), cudaMemcpyDeviceToHost));
    EventPair ev;
    CUDA_TRY(cudaEventCreate(&ev.a));
    CUDA_TRY(cudaEventCreate(&ev.b));
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    int cur[3] = {c->L.shape[0], c->L.shape[1], c->L.shape[2]};
    // every tile shape of every explicit direction, each pipelined and one tile per CTA
    // where the pipelined sweeps apply (the pipeline's bit for a direction is its choice)
    const int mask0 = c->pipe_mask;
    const bool can_pipe = c->L.d_maps != nullptr;
    int mask = mask0;
    for (int d = 0; d < 3; ++d) {
      if (compact_scheme(c->P.scheme[d])) { best[d] = 0; continue; }
      double tbest = 1e300;
      int best_mode = (mask0 >> d) & 1;
      // two passes over the candidates, each keeping its faster time: one disturbed
      // measurement cannot decide the choice
      for (int pass = 0; pass < 2; ++pass)
      for (int sh = 0; sh < kTileShapes; ++sh) {
        for (int mode = can_pipe ? 1 : 0; mode >= 0; --mode) {
          cur[d] = sh;
          mask = (mask & ~(1 << d)) | (mode << d);
          c->pipe_mask = mask;
          if (int r = apply_shapes(c, cur)) return r;
          auto sweep = [&]() {
            return c->exact ? nuc3d::exact::run_sweep(c->L, d, 0, 0) : nuc3d::fast::run_sweep(c->L, d, 0, 0);
          };
          CUDA_TRY(sweep());  // warm-up
          CUDA_TRY(cudaEventRecord(e0, c->stream));
          for (int r = 0; r < reps; ++r) CUDA_TRY(sweep());
          CUDA_TRY(cudaEventRecord(e1, c->stream));
          CUDA_TRY(cudaEventSynchronize(e1));
          float t = 0.0f;
          CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
          unsigned st = 0;  // a pipelined sweep that gave up waiting is a failure, not a time
          CUDA_TRY(cudaMemcpy(&st, &c->d_state->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
          if (st & ~status0 & ST_PIPE_TIMEOUT)
            return fail(NUC3D_ECUDA, "autotune: a pipelined sweep timed out");
          const double ms = (double)t / reps;
          if (ms_out && (ms_out[3 * d + sh] < 0.0 || ms < ms_out[3 * d + sh])) ms_out[3 * d + sh] = ms;
          if (ms < tbest) { tbest = ms; best[d] = sh; best_mode = mode; }
        }
      }
      cur[d] = best[d];
      mask = (mask & ~(1 << d)) | (best_mode << d);
    }
    best[3] = mask;
    CUDA_TRY(cudaMemcpy(&c->d_state->status, &status0, sizeof(unsigned), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(&c->d_state->reset_cells, &resets0, sizeof(resets0), cudaMemcpyHostToDevice));
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  const int shp[3] = {best[0], best[1], best[2]};
  if (c->use_pipe) c->pipe_mask = best[3];
  if (int r = apply_shapes(c, shp)) return r;
  if (shape_out)
    for (int d = 0; d < 3; ++d) shape_out[d] = best[d];
  return NUC3D_OK;
}

int nuc3d_sync(nuc3d_ctx *c) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int nuc3d_get_time(nuc3d_ctx *c, double *time, double *dt) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  StepState s;
  CUDA_TRY(cudaMemcpy(&s, c->d_state, sizeof(s), cudaMemcpyDeviceToHost));
  if (time) *time = s.time;
  if (dt) *dt = s.dt;
  return NUC3D_OK;
}

int nuc3d_set_time(nuc3d_ctx *c, double time) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&c->d_state->time, &time, sizeof(double), cudaMemcpyHostToDevice));
  return NUC3D_OK;
}

int nuc3d_get_status(nuc3d_ctx *c, unsigned *status) {
  if (!c || !status) return fail(NUC3D_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(status, &c->d_state->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return NUC3D_OK;
}

int nuc3d_get_energy_resets(nuc3d_ctx *c, unsigned long long *cells) {
  if (!c || !cells) return fail(NUC3D_EINVAL, "null argument");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(cells, &c->d_state->reset_cells, sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost));
  return NUC3D_OK;
}

int nuc3d_set_stream(nuc3d_ctx *c, void *stream) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->drop_graph();
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (stream) {
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  c->L.stream = c->stream;
  return NUC3D_OK;
}

int nuc3d_profile_sweep(nuc3d_ctx *c, int dir, int reps, double *ms) {
  if (!c || !ms || dir < 0 || dir > 2 || reps < 1) return fail(NUC3D_EINVAL, "bad argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  cudaSetDevice(c->device);
  auto sweep = [&]() {
    return c->exact ? nuc3d::exact::run_sweep(c->L, dir, 0, 0) : nuc3d::fast::run_sweep(c->L, dir, 0, 0);
  };
  unsigned long long resets0 = 0;  // profiling sweeps leave the reset count as it was
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&resets0, &c->d_state->reset_cells, sizeof(resets0), cudaMemcpyDeviceToHost));
  CUDA_TRY(sweep());  // warm-up
  EventPair ev;
  CUDA_TRY(cudaEventCreate(&ev.a));
  CUDA_TRY(cudaEventCreate(&ev.b));
  cudaEvent_t e0 = ev.a, e1 = ev.b;
  CUDA_TRY(cudaEventRecord(e0, c->stream));
  for (int r = 0; r < reps; ++r) CUDA_TRY(sweep());
  CUDA_TRY(cudaEventRecord(e1, c->stream));
  CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0.0f;
  CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
  *ms = (double)t / reps;
  CUDA_TRY(cudaMemcpy(&c->d_state->reset_cells, &resets0, sizeof(resets0), cudaMemcpyHostToDevice));
  return check_status(c);
}

int nuc3d_diagnostics(nuc3d_ctx *c, double *enstrophy, double *kinetic) {
  if (!c || !enstrophy || !kinetic) return fail(NUC3D_EINVAL, "bad argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  for (int d = 0; d < 3; ++d)
    if (vis_reach(c->P.vis[d]) > c->P.ts[d])
      return fail(NUC3D_ENOTSUP,
                  "direction %d: the velocity-gradient stencil reaches %d cells but the "
                  "reconstruction's bufferSize is %d; the reference reads outside its arrays there",
                  d, vis_reach(c->P.vis[d]), c->P.ts[d]);
  cudaSetDevice(c->device);
  const int nb = (int)c->blocks.size();
  if (!c->d_diag) {
    c->diag.assign(nb, DiagDev{nullptr, nullptr, nullptr});
    for (int bi = 0; bi < nb; ++bi) {
      const size_t n = (size_t)c->blocks[bi].N * sizeof(double);
      DiagDev &d = c->diag[bi];
      CUDA_TRY(cudaMalloc(&d.prim, 4 * n));
      CUDA_TRY(cudaMalloc(&d.fields, 5 * n));
      CUDA_TRY(cudaMalloc(&d.dens, 2 * n));
    }
    CUDA_TRY(cudaMalloc(&c->d_dsums, 2 * nb * sizeof(double)));
    CUDA_TRY(cudaMalloc(&c->d_dparts, 2 * (size_t)nb * kDiagParts * sizeof(double)));
    CUDA_TRY(cudaMalloc(&c->d_diag, nb * sizeof(DiagDev)));
    CUDA_TRY(cudaMemcpy(c->d_diag, c->diag.data(), nb * sizeof(DiagDev), cudaMemcpyHostToDevice));
  }
  CUDA_TRY(c->exact ? nuc3d::exact::run_diag(c->L, c->d_diag, c->d_dsums, c->d_dparts)
                    : nuc3d::fast::run_diag(c->L, c->d_diag, c->d_dsums, c->d_dparts));
  std::vector<double> sums(2 * nb);
  CUDA_TRY(cudaMemcpyAsync(sums.data(), c->d_dsums, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  // MPI_Allreduce(SUM) over the ranks, in rank order (src/postproc.cpp:832-834)
  double e = sums[0], k = sums[1];
  for (int bi = 1; bi < nb; ++bi) {
    e += sums[2 * bi];
    k += sums[2 * bi + 1];
  }
  *enstrophy = e;
  *kinetic = k;
  return NUC3D_OK;
}

int nuc3d_block_get_diag(nuc3d_ctx *c, int bi, double *fields) {
  if (!c || !fields || bi < 0 || bi >= (int)c->blocks.size()) return fail(NUC3D_EINVAL, "bad argument");
  if (!c->d_diag) return fail(NUC3D_ESTATE, "call nuc3d_diagnostics first");
  return copy_out(c, bi, fields, c->diag[bi].fields, 5);
}

int nuc3d_sensor_record(nuc3d_ctx *c, int dir, float *feat, unsigned char *label,
                        long long *where, unsigned long long cap, unsigned long long *count) {
  if (!c || !feat || !label || !count || dir < 0 || dir > 2) return fail(NUC3D_EINVAL, "bad argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (c->P.scheme[dir] != SCH_WENO5Z)
    return fail(NUC3D_ENOTSUP, "the face sensor is defined for weno5z directions");
  cudaSetDevice(c->device);
  unsigned long long *d_count = nullptr;
  CUDA_TRY(cudaMallocAsync(&d_count, sizeof(unsigned long long), c->stream));
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), c->stream);
  if (e == cudaSuccess)
    e = c->exact ? nuc3d::exact::run_sensor_data(c->L, dir, feat, label, where, d_count, cap)
                 : nuc3d::fast::run_sensor_data(c->L, dir, feat, label, where, d_count, cap);
  unsigned long long n = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&n, d_count, sizeof(n), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFreeAsync(d_count, c->stream);
  if (e != cudaSuccess) return fail(NUC3D_ECUDA, "sensor record: %s", cudaGetErrorString(e));
  *count = n < cap ? n : cap;
  return NUC3D_OK;
}

namespace {
// float -> BF16 bits, round to nearest even (NaN stays NaN)
uint32_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (u >> 16) | 0x40u;
  return (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
}
float bf16_value(float f) {
  const uint32_t u = bf16_bits(f) << 16;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}
}  // namespace

int nuc3d_set_sensor(nuc3d_ctx *c, const float *params, float logit_threshold) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (c->exact && params)
    return fail(NUC3D_ENOTSUP, "the hybrid sweep exists in the throughput build only (exact = 0)");
  cudaSetDevice(c->device);
  c->drop_graph();
  if (!params) {
    c->P.sensor = c->L.P.sensor = nullptr;
    return NUC3D_OK;
  }
  // W1[32][19] b1[32] W2[32][32] b2[32] W3[32] b3: B fragments of mma.sync m16n8k16
  // (rows k = 2q, 2q+1 and 2q+8, 2q+9 of the k-step, column n = lane / 4 of the n-tile)
  SensorDev h{};
  auto W1 = [&](int n, int k) { return k < 19 ? params[n * 19 + k] : 0.0f; };
  auto W2 = [&](int n, int k) { return params[640 + n * 32 + k]; };
  for (int ks = 0; ks < 2; ++ks)
    for (int nt = 0; nt < 4; ++nt)
      for (int lane = 0; lane < 32; ++lane) {
        const int n = nt * 8 + lane / 4, k0 = ks * 16 + 2 * (lane % 4);
        h.w1[ks][nt][lane][0] = bf16_bits(W1(n, k0)) | (bf16_bits(W1(n, k0 + 1)) << 16);
        h.w1[ks][nt][lane][1] = bf16_bits(W1(n, k0 + 8)) | (bf16_bits(W1(n, k0 + 9)) << 16);
        h.w2[ks][nt][lane][0] = bf16_bits(W2(n, k0)) | (bf16_bits(W2(n, k0 + 1)) << 16);
        h.w2[ks][nt][lane][1] = bf16_bits(W2(n, k0 + 8)) | (bf16_bits(W2(n, k0 + 9)) << 16);
      }
  for (int j = 0; j < 32; ++j) {
    h.b1[j] = bf16_value(params[608 + j]);
    h.b2[j] = bf16_value(params[1664 + j]);
    h.w3[j] = bf16_value(params[1696 + j]);
  }
  h.b3 = bf16_value(params[1728]);
  if (!c->d_sensor) CUDA_TRY(cudaMalloc(&c->d_sensor, sizeof(SensorDev)));
  CUDA_TRY(cudaMemcpy(c->d_sensor, &h, sizeof(SensorDev), cudaMemcpyHostToDevice));
  CUDA_TRY(nuc3d::fast::run_sensor_zero(c->d_sensor, c->stream));
  c->P.sensor = c->L.P.sensor = c->d_sensor;
  c->P.sensor_threshold = c->L.P.sensor_threshold = logit_threshold;
  c->P.sensor_theta = c->L.P.sensor_theta = 0;
  return NUC3D_OK;
}

int nuc3d_set_sensor_theta(nuc3d_ctx *c, float theta_min) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  if (c->exact)
    return fail(NUC3D_ENOTSUP, "the hybrid sweep exists in the throughput build only (exact = 0)");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->drop_graph();
  if (!c->d_sensor) {
    CUDA_TRY(cudaMalloc(&c->d_sensor, sizeof(SensorDev)));
    CUDA_TRY(cudaMemset(c->d_sensor, 0, sizeof(SensorDev)));
  }
  c->P.sensor = c->L.P.sensor = c->d_sensor;  // selects the hybrid sweep; weights unused
  c->P.sensor_threshold = c->L.P.sensor_threshold = theta_min;
  c->P.sensor_theta = c->L.P.sensor_theta = 1;
  return NUC3D_OK;
}

int nuc3d_kernels_per_step(nuc3d_ctx *c, int *kernels) {
  if (!c || !kernels) return fail(NUC3D_EINVAL, "bad argument");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  const Launch &L = c->L;
  int per_stage = (L.bc_tiles > 0 ? 1 : 0) + (L.P.model == MODEL_NS ? 2 : 0);
  for (int d = 0; d < 3; ++d)
    per_stage += ((L.P.scheme[d] == SCH_CRWENO5 || L.P.scheme[d] == SCH_HCCS ||
                   L.P.scheme[d] == SCH_HCCS77) && !((L.line_dirs >> d) & 1)) ? 3 : 1;
  *kernels = 3 * per_stage + (L.d_res_last ? 1 : 0);  // + the residual after the last stage
  return NUC3D_OK;
}

int nuc3d_set_pipeline(nuc3d_ctx *c, int on) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->use_pipe = on != 0;
  c->pipe_mask = on == 1 ? 7 : (on & 7);  // 1: every direction; else a bitmask of directions
  c->drop_graph();
  return build_maps(c);
}

int nuc3d_set_compact_solver(nuc3d_ctx *c, int fused) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  if (!c->finalized) return fail(NUC3D_ESTATE, "call nuc3d_finalize first");
  cudaSetDevice(c->device);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->compact_fused = fused != 0;
  c->drop_graph();
  set_line_dirs(c);
  return NUC3D_OK;
}

int nuc3d_get_compact_solver(nuc3d_ctx *c, int *dirs) {
  if (!c || !dirs) return fail(NUC3D_EINVAL, "null argument");
  *dirs = c->L.line_dirs;
  return NUC3D_OK;
}

int nuc3d_get_pipeline(nuc3d_ctx *c, int *on) {
  if (!c || !on) return fail(NUC3D_EINVAL, "null argument");
  *on = c->L.d_maps != nullptr ? c->L.pipe_dirs : 0;
  return NUC3D_OK;
}

int nuc3d_use_graph(nuc3d_ctx *c, int on) {
  if (!c) return fail(NUC3D_EINVAL, "null context");
  c->use_graph = on != 0;
  if (!c->use_graph) c->drop_graph();
  return NUC3D_OK;
}

}  // extern "C"
