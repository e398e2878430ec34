/*
 * nuc3d_gpu.h -- C ABI of the B200 implementation of NUC3d's per-block right-hand
 * side and TVD-RK3 update (libnuc3d_b200.so).
 *
 * Plain C types only.  Every entry point returns 0 (NUC3D_OK) or an error code;
 * nuc3d_last_error() gives a message for the calling thread.  Host arrays are
 * the reference's field3d layout: [nz][ny][nx] doubles, i fastest
 * (src/field.h:11-81, index k*nx*ny + j*nx + i); multi-component arrays are
 * stacked component-major (component c of cell idx at c*N + idx).
 *
 * What each entry point replaces in juncas/NUC3d (paths relative to the project):
 *   nuc3d_create            fieldOperator3d (src/fieldOperator.cpp:20-87, Method.in),
 *                           physicsModel (src/physicsModel.cpp:13-112, PhysModel.in)
 *   nuc3d_block_add         block::initial's per-rank block + BC_Topo
 *                           (src/block.cpp:31-100, src/boundaryConditions.cpp:25-93)
 *   nuc3d_block_set_nodes   block::getJacobians on the GPU (src/block.cpp:237-477)
 *   nuc3d_block_set_metrics block::getJacobians output (src/block.cpp:237-325):
 *                           EulerData3D::jacobian, xi_xyz, eta_xyz, zeta_xyz, dx, dy, dz
 *                           (src/euler3d.h:38-46)
 *   nuc3d_block_set_q/get_q PDEData3d::Q_work = U/J (src/PDEData3d.hpp:39-44),
 *                           restart read/write (src/block.cpp:754-855)
 *   nuc3d_rhs, nuc3d_rhs_stage  EulerData3D::solve / NaiverStokesData3d::solve
 *                           (src/euler3d.cpp:248-262, src/NaiverStokes3d.cpp:36-49) + getDt
 *   nuc3d_rk_stage          tvdrk3rd::integrationAll (src/TVD-RK3.cpp:16-137)
 *   nuc3d_get_residual      PDEData3d::setRES / getRes (src/PDEData3d.cpp:90-122)
 *   nuc3d_block_get_rhs     PDEData3d::RHS (src/PDEData3d.hpp:44)
 *   nuc3d_step              block::solve: 3 x (RHS; PDEData3d::solve -> tvdrk3rd)
 *                           (src/block.cpp:569-594, src/PDEData3d.cpp:152-170,
 *                           src/TVD-RK3.cpp:16-137), time += dt
 *   nuc3d_solve_host        the same on host arrays, in place, every step
 *   (MPI halo exchange, src/MPICommunicator.cpp:36-115, has no entry point: blocks
 *    added to one context read each other's cells directly on the device.)
 */
#ifndef NUC3D_GPU_H
#define NUC3D_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  NUC3D_OK = 0,
  NUC3D_EINVAL = 1,    /* bad argument or configuration */
  NUC3D_ECUDA = 2,     /* CUDA runtime error */
  NUC3D_ESTATE = 3,    /* call out of order (e.g. stepping before finalize) */
  NUC3D_ENUMERIC = 4,  /* a kernel flagged negative pressure or a non-finite state */
  NUC3D_ENOTSUP = 5    /* configuration the library does not implement */
};

/* status bits returned by nuc3d_get_status */
enum {
  NUC3D_ST_NEG_PRESSURE = 1, /* EoS pressure < 0: the reference exits (src/physicsModel.cpp:1009-1016) */
  NUC3D_ST_ENERGY_RESET = 2, /* internal energy < 0 was reset (src/physicsModel.cpp:324-332) */
  NUC3D_ST_NONFINITE = 4,    /* the RK update produced a NaN or Inf */
  NUC3D_ST_BAD_LAUNCH = 8,
  NUC3D_ST_PIPE_TIMEOUT = 16 /* a pipelined sweep gave up waiting for its loads (2 s); the
                                results of that evaluation are invalid (NUC3D_ECUDA) */
};

typedef struct nuc3d_ctx nuc3d_ctx;

typedef struct {
  /* Method.in: scheme_{x,y,z}_ivs and scheme_{x,y,z}_vis (src/fieldOperator.cpp:20-33).
     ivs: "weno5js" | "weno5z" | "weno7js" | "crweno5" | "hccs" | "hccs77" | "weno3js" |
     "upwind1st"; vis: "cd6" (NULL) | "cd2" | "cd8". */
  const char *scheme_ivs[3];
  const char *scheme_vis[3];
  /* PhysModel.in positional entries (src/physicsModel.cpp:65-69):
     riemann "LF" | "AUSM" | "AUSMp"; model "Euler3d" | "NavierStokes3d". */
  const char *riemann;
  const char *model;
  /* PhysModel.in key/values (src/physicsModel.cpp:41-51) */
  double reynolds, mach, prandtl, gamma, t_ref, t_inf, t_wall;
  /* IOController.in cfl (src/IOcontroller.cpp:22-29) */
  double cfl;
  /* 1: reference operation order, no FMA contraction (bit-comparable with the
        reference on x86-64); 0: throughput arithmetic (agrees to round-off). */
  int exact;
  /* 1: reproduce the interior positive-split WENO5-Z smoothness indicator of
        src/weno5z.cpp:80 (reference behaviour); 0: textbook WENO5-Z. */
  int weno5z_compat;
} nuc3d_config;

const char *nuc3d_last_error(void);

int nuc3d_create(const nuc3d_config *cfg, int device, nuc3d_ctx **out);
int nuc3d_destroy(nuc3d_ctx *ctx);

/* Add a block of nx*ny*nz cells.  Faces are ordered xi-, xi+, eta-, eta+, zeta-, zeta+
   as in BC_Topo_<rank>.in (src/boundaryConditions.cpp:69-93):
     bc_type[f] = -1 for a physical face, else the index of the neighbour block;
     bc_id[f]   = physical: 0 inlet, 1 outlet, 2 wall, 3 symmetry; else the neighbour's face.
   bc_values: 6*5 doubles (rho, u, v, w, p per face, used by inlet faces); may be NULL.
   NUC3D_ENOTSUP for an hccs77 direction with a physical face, or with more than 127 cells
   along it or more than 128 across it: the reference's hccs77 is defined only for
   neighbour faces and lines that fit its 128^3 row arrays (src/hccs77.hpp:15-18). */
int nuc3d_block_add(nuc3d_ctx *ctx, int nx, int ny, int nz, const int bc_type[6],
                    const int bc_id[6], const double *bc_values, int *block_id);

/* Metrics of a block (host arrays, N doubles per component):
   jac: 1/det(d(x,y,z)/d(xi,eta,zeta)); xi_xyz, eta_xyz, zeta_xyz: 3N each;
   dxyz: 9N (x_xi, x_eta, x_zeta, y_xi, y_eta, y_zeta, z_xi, z_eta, z_zeta), needed
   only by symmetry faces, may be NULL otherwise. */
int nuc3d_block_set_metrics(nuc3d_ctx *ctx, int block, const double *jac, const double *xi_xyz,
                            const double *eta_xyz, const double *zeta_xyz, const double *dxyz);

/* Metrics computed on the GPU from the block's node coordinates: block::getJacobians
   (src/block.cpp:237-325) with its tile-Lagrange derivatives (:327-477).  x, y, z: host
   arrays of (nx+1)(ny+1)(nz+1) nodes, i fastest (mesh_<r>.x, src/block.cpp:42-81); cells
   per axis must be multiples of 4, as in the reference.  Bitwise the reference's metrics;
   a negative Jacobian returns NUC3D_EINVAL (the reference exits). */
int nuc3d_block_set_nodes(nuc3d_ctx *ctx, int block, const double *x, const double *y,
                          const double *z);
/* Copy a block's metrics back (any pointer may be NULL; dxyz exists for blocks with a
   symmetry face or when given to nuc3d_block_set_metrics). */
int nuc3d_block_get_metrics(nuc3d_ctx *ctx, int block, double *jac, double *xi_xyz,
                            double *eta_xyz, double *zeta_xyz, double *dxyz);

/* Validate the block topology and upload the descriptors.  Call once, after all
   blocks are added and before any evaluation. */
int nuc3d_finalize(nuc3d_ctx *ctx);

/* Conservative state Q = U/J of a block (5N doubles, host memory). */
int nuc3d_block_set_q(nuc3d_ctx *ctx, int block, const double *q);
int nuc3d_block_get_q(nuc3d_ctx *ctx, int block, double *q);
/* Device pointer of the block's current state (5N doubles), for callers that keep
   their data in HBM. */
int nuc3d_block_q_device(nuc3d_ctx *ctx, int block, double **dev_q);

/* One right-hand-side evaluation of every block at the current state (no update).
   dt_local receives min over blocks and directions of 1/max(|U|+c|grad xi|),
   the reference's dt before the cfl factor (src/euler3d.cpp:429-435). */
int nuc3d_rhs(nuc3d_ctx *ctx, double *dt_local);
int nuc3d_block_get_rhs(nuc3d_ctx *ctx, int block, double *rhs);

/* The stages of block::solve one call at a time, for a host that drives the reference's
   loop itself (src/block.cpp:579-580: EulerData3D::solve, then PDEData3d::solve).
   nuc3d_rhs_stage: the right-hand side of every block at the state of RK stage `stage`
   (0: the step's state; 1, 2: the states nuc3d_rk_stage(stage - 1) produced), as
   EulerData3D::solve / NaiverStokesData3d::solve evaluate it on Q_work; dt_local as in
   nuc3d_rhs.  nuc3d_rhs(ctx, dt) is nuc3d_rhs_stage(ctx, 0, dt).
   nuc3d_rk_stage: tvdrk3rd::integrationAll (src/TVD-RK3.cpp:16-137) for stage `stage` with
   the step size dt the caller fixed at stage 0 (PDEData3d::solve, src/PDEData3d.cpp:70-88:
   cfl times the minimum over ranks of dt_local), from the right-hand side the last
   nuc3d_rhs_stage(stage) left; the stage state and the step's state enter with con2prim's
   energy reset applied, as Q_work and Q_Euler hold them.  Stage 2 leaves the new state as
   the block's current state, adds dt to the time and computes the residual. */
int nuc3d_rhs_stage(nuc3d_ctx *ctx, int stage, double *dt_local);
int nuc3d_rk_stage(nuc3d_ctx *ctx, int stage, double dt);
/* The residual of the last step (PDEData3d::setRES, src/PDEData3d.cpp:90-122, which
   block::printStatus prints: src/block.cpp:593-598): per block
   |sqrt(sum over components and cells of (u - u_n)^2 / (5N)) - that root one step earlier|
   / dt^2, the maximum over blocks.  The reference-order build sums in the reference's order
   (bit for bit); the throughput build sums per tile (round-off apart). */
int nuc3d_get_residual(nuc3d_ctx *ctx, double *res);

/* nsteps TVD-RK3 steps (each: three stages; dt fixed at stage 0 as cfl/max eigenvalue).
   Asynchronous on the context's stream; nuc3d_sync waits and checks the status. */
int nuc3d_step(nuc3d_ctx *ctx, int nsteps);
/* block::solve on host arrays (src/block.cpp:569-594, which updates Q_work in place):
   nsteps steps, each reading every block's Q = U/J from q_host[block] (5N doubles, the
   nuc3d_block_set_q layout) and writing the new Q back there.  The download of a step and
   the upload of the next run at the same time in 16 MiB chunks (PCIe is full duplex), so
   q_host should be pinned (cudaHostAlloc / cudaHostRegister).  Synchronous: returns
   when q_host holds the last step's state, with nuc3d_sync's status check.
   A context of one Euler block with explicit schemes and at least 64 z-planes runs the
   steps as a pipeline over z-slabs of 32 planes instead (the zeta sweep in 8 x 32 tiles
   for the call, whatever the context's zeta shape, which is restored): stage 0's work
   on each uploaded piece of a slab follows its upload at once (the xi and eta lines lie
   in a z-plane); with both z faces physical the three stages then advance slab by slab
   as a wavefront (a slab's zeta sweep needs the previous stage's state of its
   neighbours only), and each slab's download follows stage 2's zeta sweep over it, so
   the copy engines move the other slabs while the GPU computes; the kernels are those
   of nuc3d_step and the state is bitwise the same (in the throughput build the
   residual's partial sums follow the zeta tiles, so its last bits can differ from
   nuc3d_step's with another zeta shape).  A last z-chunk thinner than 8 planes joins
   the slab before it.  A context of several blocks (explicit schemes, no learned sensor)
   runs stage 2 block by block instead, each block's download following its own zeta
   sweep (bitwise the same).  nuc3d_set_host_pipeline(ctx, 0) turns both off;
   nuc3d_get_host_pipeline gives the slab count in use (0: the chunked copies). */
int nuc3d_solve_host(nuc3d_ctx *ctx, double *const *q_host, int nsteps);
int nuc3d_set_host_pipeline(nuc3d_ctx *ctx, int on);
int nuc3d_get_host_pipeline(nuc3d_ctx *ctx, int *slabs);
int nuc3d_sync(nuc3d_ctx *ctx);
/* time accumulated over the steps and the dt of the last step */
int nuc3d_get_time(nuc3d_ctx *ctx, double *time, double *dt);
int nuc3d_set_time(nuc3d_ctx *ctx, double time);
int nuc3d_get_status(nuc3d_ctx *ctx, unsigned *status);
/* Cells whose energy con2prim reset because their internal energy was negative
   (physicsModel::con2prim, src/physicsModel.cpp:324-332), counted once per cell and
   right-hand-side evaluation and summed since the context was created: the number of
   "negative pressure at" lines the reference prints for the same evaluations.  Profiling
   and autotuning sweeps leave it unchanged. */
int nuc3d_get_energy_resets(nuc3d_ctx *ctx, unsigned long long *cells);

/* CUDA stream (cudaStream_t) the context launches on; NULL = its own stream. */
int nuc3d_set_stream(nuc3d_ctx *ctx, void *stream);
/* 1: replay the three stages of a step as one CUDA graph (default); 0: launch directly. */
int nuc3d_use_graph(nuc3d_ctx *ctx, int on);

/* Profiling: launch the dir-sweep kernel (0 xi, 1 eta, 2 zeta; right-hand side
   only, at the current state) `reps` times back to back on the context's stream and
   return the mean device time per launch in milliseconds (CUDA events). */
int nuc3d_profile_sweep(nuc3d_ctx *ctx, int dir, int reps, double *ms_per_launch);

/* Flow diagnostics of the current state of every block: postproc::solveQ after
   block::Post (src/postproc.cpp:743-848, src/block.cpp:601-618), which the reference runs
   every postStep steps when PostProc.in has SimutaneousData 1 and appends to
   enstrophy.dat.  Velocity gradients by the block's difference operator, vorticity w,
   Q criterion; *enstrophy = sum over cells of 0.5|w|^2, *kinetic = sum of 0.5 rho |u|^2
   (per block in cell order, then over the blocks in order, as the reference's
   MPI_Allreduce).  The reference-order build reproduces the reference's totals bit for
   bit; the throughput build sums in a different, fixed order.  The first call allocates
   88 bytes per cell of workspace. */
int nuc3d_diagnostics(nuc3d_ctx *ctx, double *enstrophy, double *kinetic);
/* Fields of the last nuc3d_diagnostics call for one block: 5N doubles, w_x, w_y, w_z,
   0.5|w|^2, Q (TemporalQField[9..13] of the reference). */
int nuc3d_block_get_diag(nuc3d_ctx *ctx, int block, double *fields);

/* ---- Learned face sensor (hybrid WENO-Z) --------------------------------------------
   No counterpart in the reference.  A 19 -> 32 -> 32 -> 1 MLP decides per face whether
   WENO-Z needs its nonlinear weights; parameters are NUC3D_SENSOR_PARAMS floats, in the
   order W1[32][19], b1[32], W2[32][32], b2[32], W3[32], b3. */
#define NUC3D_SENSOR_PARAMS 1729
/* Features (19 floats per face) and labels (1: some WENO-Z weight is more than 0.05 from
   its linear weight) of the interior faces of direction dir at the current state, written
   to device buffers in no particular order; where (may be NULL) gets each face's index in
   its block's face grid (n[dir]+1 faces along dir, i fastest); *count = faces written (at
   most cap).  dir must use weno5z. */
int nuc3d_sensor_record(nuc3d_ctx *ctx, int dir, float *feat, unsigned char *label,
                        long long *where, unsigned long long cap, unsigned long long *count);
/* Training, on device buffers and the given CUDA stream: loss (BCE on the logit, positives
   weighted by pos_weight, mean over n) and its gradient w.r.t. the parameters (grad is
   overwritten); logits (n floats) may be NULL.  Then one Adam step (step >= 1). */
int nuc3d_sensor_loss_grad(const float *params, const float *feat, const unsigned char *label,
                           long long n, float pos_weight, float *grad, float *loss, float *logits,
                           void *stream);
int nuc3d_sensor_adam(float *params, const float *grad, float *m, float *v, float lr, float beta1,
                      float beta2, float eps, int step, void *stream);
/* Hybrid WENO-Z (throughput build only): from now on every interior face of a weno5z
   direction whose sensor logit is below logit_threshold takes the linear weights
   (0.1, 0.6, 0.3); the others, and the faces of the boundary schemes, are unchanged.
   params: NUC3D_SENSOR_PARAMS floats (copied, rounded to BF16 as in the training), or
   NULL to return to plain WENO-Z. */
int nuc3d_set_sensor(nuc3d_ctx *ctx, const float *params, float logit_threshold);
/* The same hybrid with the hand-made decision of the reference's hybrid compact scheme
   instead of the network: theta = 1 / (1 + (sum_k alpha_k - 1)^2) of CRWENO5-Z weights
   (src/hccs.cpp:154-181), evaluated on the face's density and pressure stencils (both
   splits); a face takes the linear weights where the smallest of the four thetas is at
   least theta_min.  nuc3d_set_sensor(ctx, NULL, 0) returns to plain WENO-Z. */
int nuc3d_set_sensor_theta(nuc3d_ctx *ctx, float theta_min);

/* ---- Sweep tile shapes (after nuc3d_finalize) ----------------------------------------
   No counterpart in the reference.  Each direction's sweep runs tiles of one of
   NUC3D_TILE_SHAPES shapes (lines x cells along them): 0 = 4 x 64 (default), 1 = 8 x 32,
   2 = 2 x 128; compact-scheme directions run shape 0.  The results do not depend on the
   shape (same arithmetic), only the speed does. */
#define NUC3D_TILE_SHAPES 3
int nuc3d_set_tiles(nuc3d_ctx *ctx, const int shape[3]);
int nuc3d_get_tiles(nuc3d_ctx *ctx, int shape[3]);
/* Time every shape of every explicit-scheme direction's right-hand-side sweep on the
   current state, pipelined and not where the pipelined sweeps apply (two passes of reps
   launches each, a candidate's faster pass counting; the state and the status word are
   left as they were, the RHS array is overwritten) and keep the fastest per direction;
   a pipelined sweep that gives up waiting for its loads returns NUC3D_ECUDA.  The choice is cached in the process per grid (block
   extents, schemes, model, build, hybrid or plain): a later context of the same grid takes
   it without timing.  shape_out (may be NULL): the shapes chosen; ms_out (may be NULL):
   9 doubles, ms per launch of direction d with shape s at [3d + s], -1 where not timed
   (a cached choice, a compact direction). */
int nuc3d_autotune(nuc3d_ctx *ctx, int reps, int shape_out[3], double ms_out[9]);

/* Pipelined sweeps (after nuc3d_finalize; on by default).  No counterpart in the reference.
   With it on, each explicit-scheme sweep is a persistent kernel (two CTAs per SM) whose
   producer warp loads the next tiles' state, Jacobian and metric with tensor-map (TMA)
   copies while the other warps compute (Navier-Stokes: the viscous fluxes by plain loads);
   results are identical either way.  It applies to contexts whose blocks all have an even
   nx (16-byte rows), for the explicit-scheme directions; elsewhere, or with
   on = 0, every sweep CTA loads its own tile.  on = 1: every direction; on > 1: the
   directions of its bits 0..2 (bit d: direction d).  nuc3d_autotune also chooses, per
   direction, between the two.  nuc3d_get_pipeline: the directions that run pipelined
   (bit d), 0 for none. */
int nuc3d_set_pipeline(nuc3d_ctx *ctx, int on);
int nuc3d_get_pipeline(nuc3d_ctx *ctx, int *on);

/* Line solver of the compact schemes (after nuc3d_finalize).  The reference solves each
   line's tridiagonal system with the Thomas algorithm (src/crweno5.cpp:207-218,
   src/hccs.cpp:252-264).  The reference-order build always does the same, in three
   kernels per direction: rows to device memory, one thread per system, faces back.
   The throughput build by default (fused = 1) runs crweno5 and hccs directions whose
   lines have at most 256 cells in one kernel per direction: a CTA per line generates the
   rows in shared memory and solves each system with one warp (partition method and
   cyclic reduction), agreeing with Thomas to round-off.  fused = 0 selects the
   three-kernel path there too.  nuc3d_get_compact_solver: the directions that run
   fused (bit d). */
int nuc3d_set_compact_solver(nuc3d_ctx *ctx, int fused);
int nuc3d_get_compact_solver(nuc3d_ctx *ctx, int *dirs);

/* Kernels one nuc3d_step(ctx, 1) launches (after nuc3d_finalize): per RK stage the BC
   ghost pass (when a block has a physical face), the NS primitive and gradient passes,
   and one sweep per direction (three kernels for a compact-scheme direction); then the
   residual kernel after the last stage.  No counterpart in the reference. */
int nuc3d_kernels_per_step(nuc3d_ctx *ctx, int *kernels);

/* Debug taps: NS primitives (u, v, w, T: 4N) and contravariant viscous fluxes
   ([dir][var 1..4]: 12N) of the last evaluation. */
int nuc3d_block_get_prim(nuc3d_ctx *ctx, int block, double *prim);
int nuc3d_block_get_vis(nuc3d_ctx *ctx, int block, double *vis);

/* Debug taps of the inviscid path: one right-hand side's intermediates at the block's
   current state (stage 0), for parity work against the reference's EulerFlux members
   (src/euler3d.h:16-31, allocated at src/euler3d.cpp:12-20 and :62-83).  tap =
   3 * kind + direction; out: 5 components, each in the reference's layout for that
   direction: line position fastest, then (xi: j, k; eta: k, i; zeta: i, j).
     FLUXL / FLUXR   Flux_<dir>.FluxL / FluxR, the split fluxes: 5N doubles
     RFLUXL / RFLUXR Flux_<dir>.reconstFluxL / R, the reconstructions: 5 (n_dir + 1) N / n_dir
     DF              dfdxi / dgdeta / dhdzeta, the flux differences: 5N
   The step state (status bits, energy-reset count) is left as it was.  Explicit schemes
   use the reference-order boundary switch in either build; compact schemes the
   three-kernel solve. */
enum {
  NUC3D_TAP_FLUXL_XI = 0, NUC3D_TAP_FLUXL_ETA = 1, NUC3D_TAP_FLUXL_ZETA = 2,
  NUC3D_TAP_FLUXR_XI = 3, NUC3D_TAP_FLUXR_ETA = 4, NUC3D_TAP_FLUXR_ZETA = 5,
  NUC3D_TAP_RFLUXL_XI = 6, NUC3D_TAP_RFLUXL_ETA = 7, NUC3D_TAP_RFLUXL_ZETA = 8,
  NUC3D_TAP_RFLUXR_XI = 9, NUC3D_TAP_RFLUXR_ETA = 10, NUC3D_TAP_RFLUXR_ZETA = 11,
  NUC3D_TAP_DF_XI = 12, NUC3D_TAP_DF_ETA = 13, NUC3D_TAP_DF_ZETA = 14
};
int nuc3d_debug_get(nuc3d_ctx *ctx, int block, int tap, double *out);

/* ---- Allocation-free right-hand side -------------------------------------------
   No counterpart in the reference: it exists for callers that cannot allocate device
   memory where they evaluate the right-hand side (a host framework that owns every
   device buffer and forbids allocations by libraries, a loop where an allocation could
   stall).  One Euler3d block.  Device pointers, owned by the caller: q (5N), jac (N),
   xi_xyz, eta_xyz, zeta_xyz (3N each, as in nuc3d_block_set_metrics), dxyz (9N; only
   read by symmetry faces, may be NULL otherwise) and the output rhs (5N).  Host
   pointers: bc_type and bc_id (6 ints; bc_type[f] is -1 for a physical face or 0 for a
   face joined to the block itself, i.e. periodic), bc_values (NULL, or 6 x 5 doubles
   rho, u, v, w, p per face, read for inlet faces) and dt_local (NULL or one double).
   It calls no cudaMalloc/cudaFree: its working memory (block descriptor, step state,
   face list, 40 bytes per cell of every physical face) is a static device array of
   NUC3D_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until the process
   exits; blocks whose physical faces need more are rejected with NUC3D_EINVAL.  The first
   call on a device looks up that array's device address and sets kernel attributes, so
   make that first call before any stream capture.  All calls share the array and each
   call overwrites it: calls that overlap on the GPU (different streams, or threads
   without ordering) race and must be serialised by the caller.  With dt_local non-NULL
   the call waits for the stream, returns 1/max eigenvalue in *dt_local and reports
   negative pressure or non-finite values as NUC3D_ENUMERIC; with NULL it only queues the
   work on `stream` (a cudaStream_t, NULL = legacy default stream) and reports no numeric
   status.  The calling thread's current device is the same on return as on entry. */
#define NUC3D_NOALLOC_SCRATCH_BYTES (8u << 20)
int nuc3d_rhs_noalloc(const nuc3d_config *cfg, int device, int nx, int ny, int nz,
                      const int bc_type[6], const int bc_id[6], const double *bc_values,
                      const double *q, const double *jac, const double *xi_xyz,
                      const double *eta_xyz, const double *zeta_xyz, const double *dxyz,
                      double *rhs, double *dt_local, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NUC3D_GPU_H */
