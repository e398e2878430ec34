// nuc3d_noalloc.cu -- nuc3d_rhs_noalloc: one Euler right-hand side of one block,
// with every byte of working memory taken from a fixed static device array.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they evaluate
// the right-hand side -- host frameworks with their own memory pool that forbid
// foreign allocations, or real-time loops where an allocation could stall.  They bring
// their own device buffers for the inputs (state, metrics) and the output (RHS); the
// library's working memory is the file-scope array below.
//
// The array holds the block descriptor, the step state (eigenvalue maximum and
// status word), the list of physical faces and the ghost fluxes of the physical faces.
// It is device memory reserved when the library's module is loaded on a GPU and kept
// by every GPU that loads the library until the process exits.  Its host-side name is
// only a stand-in: host code takes the device address with cudaGetSymbolAddress, once
// per device, with that device current, and passes that address to the kernels.
// The descriptors reach the array through the arguments of a one-thread kernel
// (noalloc_setup), so nothing is copied from host memory.
#include <cstring>
#include <mutex>
#include <string>

#include "common.h"
#include "nuc3d_gpu.h"

using namespace nuc3d;

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;  // NUC3D_NOALLOC_SCRATCH_BYTES
static_assert(kScratchBytes == NUC3D_NOALLOC_SCRATCH_BYTES, "header and library disagree");
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_dev[kMaxDevices];   // device address of g_noalloc_scratch per device
bool g_ready[kMaxDevices][2];       // kernel attributes set (exact, fast) per device

int nfail(int code, const char *msg) {
  nuc3d::set_error_message(msg);  // read back with nuc3d_last_error()
  return code;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The physical faces of the one block (at most six), passed by value to noalloc_setup.
struct NoallocFaces {
  int njobs;
  unsigned char face[6];
  int start[7];
};

// Writes the block descriptor and the face list into the static array and clears the
// step state (eigenvalue maximum, status, counters): the call's set-up, on the GPU.
__global__ void noalloc_setup(BlockDev B, NoallocFaces F, BlockDev *dB, StepState *dS,
                              FaceJobs *dJ) {
  *dB = B;
  StepState z;
  memset(&z, 0, sizeof(z));
  *dS = z;
  dJ->njobs = F.njobs;
  for (int j = 0; j < 6; ++j) {
    dJ->block[j] = 0;
    dJ->face[j] = F.face[j];
  }
  for (int j = 0; j < 7; ++j) dJ->start[j] = F.start[j];
}

// Restores the calling thread's current device on every way out of the entry point.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int scheme_id(const char *s, int *out) {
  if (!s) return 1;
  if (!std::strcmp(s, "weno5js")) *out = SCH_WENO5JS;
  else if (!std::strcmp(s, "weno5z")) *out = SCH_WENO5Z;
  else if (!std::strcmp(s, "weno7js")) *out = SCH_WENO7JS;
  else return 1;
  return 0;
}

}  // namespace

extern "C" {

int nuc3d_rhs_noalloc(const nuc3d_config *cfg, int device, int nx, int ny, int nz,
                      const int bc_type[6], const int bc_id[6], const double *bc_values,
                      const double *q, const double *jac, const double *xi_xyz,
                      const double *eta_xyz, const double *zeta_xyz, const double *dxyz,
                      double *rhs, double *dt_local, void *stream) {
  // ---- arguments (no CUDA call before they are known good) ----
  if (!cfg || !bc_type || !bc_id || !q || !jac || !xi_xyz || !eta_xyz || !zeta_xyz || !rhs)
    return nfail(NUC3D_EINVAL, "null argument");
  if (!cfg->model || std::strcmp(cfg->model, "Euler3d"))
    return nfail(NUC3D_ENOTSUP, "nuc3d_rhs_noalloc evaluates the Euler3d model only (the "
                                "Navier-Stokes terms need O(cells) working memory)");
  SolverParams P{};
  for (int d = 0; d < 3; ++d) {
    if (scheme_id(cfg->scheme_ivs[d], &P.scheme[d]))
      return nfail(NUC3D_EINVAL, "scheme must be weno5js, weno5z or weno7js");
    P.ts[d] = scheme_tilesize(P.scheme[d]);
  }
  P.bfs = P.ts[0] > P.ts[1] ? P.ts[0] : P.ts[1];
  P.bfs = P.bfs > P.ts[2] ? P.bfs : P.ts[2];
  if (!cfg->riemann) return nfail(NUC3D_EINVAL, "null riemann name");
  if (!std::strcmp(cfg->riemann, "LF")) P.riemann = RIE_LF;
  else if (!std::strcmp(cfg->riemann, "AUSM")) P.riemann = RIE_AUSM;
  else if (!std::strcmp(cfg->riemann, "AUSMp")) P.riemann = RIE_AUSMP;
  else return nfail(NUC3D_EINVAL, "riemann must be LF, AUSM or AUSMp");
  P.model = MODEL_EULER;
  P.gamma = cfg->gamma;
  P.mach = cfg->mach;
  P.reynolds = cfg->reynolds;
  P.prandtl = cfg->prandtl;
  P.t_ref = cfg->t_ref;
  P.t_inf = cfg->t_inf;
  P.t_wall = cfg->t_wall;
  P.cfl = cfg->cfl;
  P.weno5z_compat = cfg->weno5z_compat ? 1 : 0;
  if (!(P.gamma > 1.0) || !(P.mach > 0.0)) return nfail(NUC3D_EINVAL, "gamma > 1 and mach > 0 required");
  const int n[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d)
    if (n[d] < 2 * P.bfs + 2) return nfail(NUC3D_EINVAL, "block dimension below 2*bfsize+2");
  if ((long long)nx * ny * nz > 2000000000LL) return nfail(NUC3D_EINVAL, "block too large");
  long long ghost_doubles = 0;
  long long goff[6];
  for (int f = 0; f < 6; ++f) {
    goff[f] = -1;
    const int d = f >> 1;
    if (bc_type[f] == -1) {
      if (bc_id[f] < 0 || bc_id[f] > 3) return nfail(NUC3D_EINVAL, "physical BC id not in 0..3");
      if (bc_id[f] == BC_INLET && !bc_values) return nfail(NUC3D_EINVAL, "inlet face needs bc_values");
      if (bc_id[f] == BC_SYMM && !dxyz) return nfail(NUC3D_EINVAL, "symmetry face needs dxyz");
      const long long area = d == 0 ? (long long)ny * nz : (d == 1 ? (long long)nz * nx : (long long)nx * ny);
      goff[f] = ghost_doubles;
      ghost_doubles += 5 * area;
    } else if (bc_type[f] == 0) {
      // the block is its own neighbour (periodic): the paired face must be in the same direction
      if (bc_id[f] < 0 || bc_id[f] > 5 || (bc_id[f] >> 1) != d)
        return nfail(NUC3D_EINVAL, "a neighbour face must pair with a face of the same direction");
    } else {
      return nfail(NUC3D_EINVAL, "nuc3d_rhs_noalloc takes one block: bc_type must be -1 or 0");
    }
  }
  const size_t off_state = align256(sizeof(BlockDev));
  const size_t off_jobs = off_state + align256(sizeof(StepState));
  const size_t off_ghost = off_jobs + align256(sizeof(FaceJobs));
  const size_t need = off_ghost + (size_t)ghost_doubles * sizeof(double);
  if (need > kScratchBytes)
    return nfail(NUC3D_EINVAL, "the physical faces of this block need more than the 8 MiB of "
                               "static working memory (40 bytes per face cell)");
  if (device < 0 || device >= kMaxDevices) return nfail(NUC3D_EINVAL, "bad device index");

  // ---- one-time set-up on this device: the array's device address, kernel attributes ----
  DeviceGuard keep_device;  // the caller's current device is restored on return
  if (cudaSetDevice(device) != cudaSuccess) return nfail(NUC3D_ECUDA, "cudaSetDevice failed");
  const int mode = cfg->exact ? 0 : 1;
  {
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    if (!g_scratch_dev[device]) {
      void *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return nfail(NUC3D_ECUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
      g_scratch_dev[device] = ptr;
    }
    if (!g_ready[device][mode]) {
      cudaError_t e = mode == 0 ? nuc3d::exact::configure() : nuc3d::fast::configure();
      if (e != cudaSuccess) return nfail(NUC3D_ECUDA, cudaGetErrorString(e));
      g_ready[device][mode] = true;
    }
  }
  unsigned char *base = static_cast<unsigned char *>(g_scratch_dev[device]);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // ---- descriptors, built on the host and written into the static array by a kernel ----
  BlockDev B;
  std::memset(&B, 0, sizeof(B));
  for (int d = 0; d < 3; ++d) B.n[d] = n[d];
  B.N = (long long)nx * ny * nz;
  B.q[0] = const_cast<double *>(q);  // read only: stage 0 of a right-hand side
  B.rhs = rhs;
  B.jac = jac;
  B.met[0] = xi_xyz;
  B.met[1] = eta_xyz;
  B.met[2] = zeta_xyz;
  B.dxyz = dxyz;
  B.ghost = reinterpret_cast<double *>(base + off_ghost);
  for (int f = 0; f < 6; ++f) {
    B.goff[f] = goff[f];
    B.face[f].type = bc_type[f];
    B.face[f].id = bc_id[f];
    for (int v = 0; v < 5; ++v) B.face[f].bcv[v] = bc_values ? bc_values[f * 5 + v] : 0.0;
  }
  const int shape0[3] = {0, 0, 0};  // default tile shape in every direction
  set_tile_divisors(B, shape0);
  NoallocFaces J;
  std::memset(&J, 0, sizeof(J));
  for (int f = 0; f < 6; ++f) {
    if (bc_type[f] != -1) continue;
    const int d = f >> 1;
    const long long area = d == 0 ? (long long)ny * nz : (d == 1 ? (long long)nz * nx : (long long)nx * ny);
    J.face[J.njobs] = (unsigned char)f;
    J.start[J.njobs + 1] = J.start[J.njobs] + (int)((area + 255) / 256);
    ++J.njobs;
  }
  noalloc_setup<<<1, 1, 0, st>>>(B, J, reinterpret_cast<BlockDev *>(base),
                                 reinterpret_cast<StepState *>(base + off_state),
                                 reinterpret_cast<FaceJobs *>(base + off_jobs));
  if (cudaGetLastError() != cudaSuccess) return nfail(NUC3D_ECUDA, "descriptor set-up launch failed");

  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.d_blocks = reinterpret_cast<const BlockDev *>(base);
  L.d_state = reinterpret_cast<StepState *>(base + off_state);
  L.d_jobs = reinterpret_cast<const FaceJobs *>(base + off_jobs);
  L.bc_tiles = J.start[J.njobs];
  L.P = P;
  L.stream = st;
  for (int d = 0; d < 3; ++d) {
    L.tm_dir[d].nblocks = 1;
    L.tm_dir[d].tile_start[0] = 0;
    L.tm_dir[d].tile_start[1] = nuc3d::exact::tile_count(d, n, 0);
  }
  L.tm_cells.nblocks = 1;
  L.tm_cells.tile_start[1] = (int)((B.N + 255) / 256);
  cudaError_t e = mode == 0 ? nuc3d::exact::run_stage(L, 0, false, true)
                            : nuc3d::fast::run_stage(L, 0, false, true);
  if (e != cudaSuccess) return nfail(NUC3D_ECUDA, cudaGetErrorString(e));
  if (dt_local) {
    StepState S;
    if (cudaMemcpyAsync(&S, base + off_state, sizeof(S), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return nfail(NUC3D_ECUDA, "reading the step state failed");
    double me;
    std::memcpy(&me, &S.max_eig_bits, sizeof(me));
    *dt_local = 1.0 / me;
    if (S.status & (ST_NEG_PRESSURE | ST_NONFINITE))
      return nfail(NUC3D_ENUMERIC, "negative pressure or non-finite value in the right-hand side");
  }
  return NUC3D_OK;
}

}  // extern "C"
