// ref_taps.cpp -- oracle harness: drives the unmodified NUC3d reference classes and
// dumps their state, so the GPU path and the C restatement can be pinned to it.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the reference
// sources in place (read-only); the binary lands in oracle/_ref/.
//
// It constructs the same objects, in the same order, as the reference driver
// singleBlock (src/singleBlock.h:31-38, src/singleBlock.cpp:10-43) and then,
// instead of the file-output loop of src/singleBlock.cpp:51-71, exposes:
//
//   nuc3d_ref_taps init  OUT   metrics + Q after block::initial (src/block.cpp:31-100)
//   nuc3d_ref_taps rhs   OUT   one right-hand side: EulerData3D::solve or its NS override
//                              (src/euler3d.cpp:248-262, src/NaiverStokes3d.cpp:36-49)
//   nuc3d_ref_taps steps N OUT  N TVD-RK3 steps of block::solve (src/block.cpp:569-594):
//                              Q, and per step dt, time and the residual block::RES
//   nuc3d_ref_taps time  N W    W untimed + N timed steps; prints the reference's own
//                              per-step wall time (src/block.cpp:576-584) as JSON
//   nuc3d_ref_taps post  N OUT  N steps, then block::Post (src/block.cpp:601-618), whose
//                              postproc::solveQ (src/postproc.cpp:743-848) needs
//                              SimutaneousData 1 in inp/PostProc.in: enstrophy and kinetic
//                              energy totals and the vorticity / enstrophy / Q fields
//
// OUT gets the rank number appended ("OUT.r<rank>").  Format: "NUCT" then records
// {u32 name_len, name, u32 ndim, i64 dims[ndim], f64 data[prod(dims)]}.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "mpi.h"

// The reference keeps the state we tap in protected/private members; widen
// access for this translation unit only (the reference objects are unchanged).
#define private public
#define protected public
#include "singleBlock.h"
#include "block.h"
#include "euler3d.h"
#include "NaiverStokes3d.h"
#include "PDEData3d.hpp"
#include "boundaryConditions.hpp"
#include "bufferData.hpp"
#include "physicsModel.h"
#include "IOcontroller.h"
#include "fieldOperator.h"
#include "postproc.hpp"
#undef private
#undef protected

using nuc3d::Field;
using nuc3d::VectorField;

// postproc keeps its totals and fields under the class's default (private) access,
// which the #define above cannot widen.  An explicit instantiation may name a private
// member ([temp.spec]/6), so these tags hand out member pointers to them.
namespace taps_access {
template <typename Tag, typename Tag::type M>
struct Grant {
  friend typename Tag::type member(Tag) { return M; }
};
struct EnsGlb { typedef double nuc3d::postproc::*type; friend type member(EnsGlb); };
struct KinGlb { typedef double nuc3d::postproc::*type; friend type member(KinGlb); };
struct Ens { typedef double nuc3d::postproc::*type; friend type member(Ens); };
struct Kin { typedef double nuc3d::postproc::*type; friend type member(Kin); };
struct QField { typedef VectorField nuc3d::postproc::*type; friend type member(QField); };
template struct Grant<EnsGlb, &nuc3d::postproc::enstrophy_glb>;
template struct Grant<KinGlb, &nuc3d::postproc::kinetic_glb>;
template struct Grant<Ens, &nuc3d::postproc::enstrophy>;
template struct Grant<Kin, &nuc3d::postproc::kinetic>;
template struct Grant<QField, &nuc3d::postproc::TemporalQField>;
}  // namespace taps_access

namespace {

struct Writer {
  std::FILE *f = nullptr;
  explicit Writer(const std::string &path) {
    f = std::fopen(path.c_str(), "wb");
    if (!f) {
      std::perror(path.c_str());
      std::exit(2);
    }
    std::fwrite("NUCT", 1, 4, f);
  }
  ~Writer() {
    if (f) std::fclose(f);
  }
  void rec(const std::string &name, const std::vector<long long> &dims, const double *data) {
    unsigned nl = (unsigned)name.size();
    std::fwrite(&nl, 4, 1, f);
    std::fwrite(name.data(), 1, nl, f);
    unsigned nd = (unsigned)dims.size();
    std::fwrite(&nd, 4, 1, f);
    long long n = 1;
    for (long long d : dims) {
      std::fwrite(&d, 8, 1, f);
      n *= d;
    }
    std::fwrite(data, 8, (size_t)n, f);
  }
  void field(const std::string &name, const Field &fl) {
    // stored with the field's own layout: dims listed slowest first
    rec(name, {fl.getSizeZ(), fl.getSizeY(), fl.getSizeX()}, fl.getDataPtr());
  }
  void fields(const std::string &name, const VectorField &v) {
    for (size_t i = 0; i < v.size(); ++i) field(name + "." + std::to_string(i), v[i]);
  }
  void scalar(const std::string &name, double x) { rec(name, {1}, &x); }
};

struct Harness {
  // same members, same declaration order as nuc3d::singleBlock
  nuc3d::MPIComunicator3d_nonblocking myMPI;
  nuc3d::IOController myIO;
  nuc3d::physicsModel myPhys;
  nuc3d::fieldOperator3d myOperator;
  nuc3d::boundaryCondition myBC;
  nuc3d::block myBlock;

  void init() { myBlock.initial(myOperator, myPhys, myMPI, myBC, myIO); }

  void dump_geometry(Writer &w) {
    nuc3d::EulerData3D &e = *myBlock.myFluxes;
    w.field("jac", e.jacobian);
    w.fields("xi_xyz", e.xi_xyz);
    w.fields("eta_xyz", e.eta_xyz);
    w.fields("zeta_xyz", e.zeta_xyz);
    w.fields("dx", e.dx);
    w.fields("dy", e.dy);
    w.fields("dz", e.dz);
    w.fields("xyz_center", myBlock.xyz_center);
  }

  void dump_rhs(Writer &w) {
    nuc3d::EulerData3D &e = *myBlock.myFluxes;
    w.fields("Q", myBlock.myPDE.getQ());
    w.fields("RHS", myBlock.myPDE.getRHS());
    w.scalar("dt_local", myBlock.myPDE.dt_local);
    w.scalar("maxEigen_xi", e.Flux_xi.maxEigen);
    w.scalar("maxEigen_eta", e.Flux_eta.maxEigen);
    w.scalar("maxEigen_zeta", e.Flux_zeta.maxEigen);
    w.fields("W", e.W_Euler);
    w.fields("W0", e.W0_Euler);
    w.fields("FluxL_xi", e.Flux_xi.FluxL);
    w.fields("FluxR_xi", e.Flux_xi.FluxR);
    w.fields("FluxL_eta", e.Flux_eta.FluxL);
    w.fields("FluxR_eta", e.Flux_eta.FluxR);
    w.fields("FluxL_zeta", e.Flux_zeta.FluxL);
    w.fields("FluxR_zeta", e.Flux_zeta.FluxR);
    w.fields("rFluxL_xi", e.Flux_xi.reconstFluxL);
    w.fields("rFluxR_xi", e.Flux_xi.reconstFluxR);
    w.fields("rFluxL_eta", e.Flux_eta.reconstFluxL);
    w.fields("rFluxR_eta", e.Flux_eta.reconstFluxR);
    w.fields("rFluxL_zeta", e.Flux_zeta.reconstFluxL);
    w.fields("rFluxR_zeta", e.Flux_zeta.reconstFluxR);
    w.fields("dfdxi", e.dfdxi);
    w.fields("dgdeta", e.dgdeta);
    w.fields("dhdzeta", e.dhdzeta);
    if (auto *ns = dynamic_cast<nuc3d::NaiverStokesData3d *>(&e)) {
      w.field("du_dxi", ns->du.getdxi());
      w.field("du_deta", ns->du.getdeta());
      w.field("du_dzeta", ns->du.getdzeta());
      w.field("dT_dxi", ns->dT.getdxi());
      w.field("dT_deta", ns->dT.getdeta());
      w.field("dT_dzeta", ns->dT.getdzeta());
      w.field("miu", ns->miu);
      w.fields("Fv_xi", ns->Flux_xi_vis);
      w.fields("Fv_eta", ns->Flux_eta_vis);
      w.fields("Fv_zeta", ns->Flux_zeta_vis);
      w.fields("dfvdxi", ns->dfvdxi);
      w.fields("dgvdeta", ns->dgvdeta);
      w.fields("dhvdzeta", ns->dhvdzeta);
    }
  }

  void one_rhs() {
    myBlock.myFluxes->solve(myBlock.myPDE, myOperator, myBlock.mybuffer, myPhys, myMPI, myBC);
  }
};

std::string ranked(const std::string &out, int rank) { return out + ".r" + std::to_string(rank); }

}  // namespace

int main(int argc, char **argv) {
  if (MPI_Init(&argc, &argv)) return 99;
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s init|rhs OUT | steps N OUT | time N W\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  {
    Harness h;
    h.init();
    MPI_Barrier(MPI_COMM_WORLD);
    if (mode == "init") {
      Writer w(ranked(argv[2], rank));
      h.dump_geometry(w);
      w.fields("Q", h.myBlock.myPDE.getQ());
      w.scalar("time", h.myBlock.time);
    } else if (mode == "rhs") {
      h.one_rhs();
      Writer w(ranked(argv[2], rank));
      h.dump_rhs(w);
    } else if (mode == "steps") {
      if (argc < 4) return 2;
      int n = std::atoi(argv[2]);
      std::vector<double> dts, times, res;
      for (int s = 0; s < n; ++s) {
        h.myBlock.solve(h.myOperator, h.myPhys, h.myMPI, h.myBC, h.myIO);
        dts.push_back(h.myBlock.dt);
        times.push_back(h.myBlock.time);
        res.push_back(h.myBlock.RES);  // PDEData3d::setRES via block::solve (src/block.cpp:593)
      }
      Writer w(ranked(argv[3], rank));
      w.fields("Q", h.myBlock.myPDE.getQ());
      if (n > 0) {
        w.rec("dt", {(long long)n}, dts.data());
        w.rec("time", {(long long)n}, times.data());
        w.rec("res", {(long long)n}, res.data());
      }
    } else if (mode == "post") {
      if (argc < 4) return 2;
      int n = std::atoi(argv[2]);
      for (int s = 0; s < n; ++s) h.myBlock.solve(h.myOperator, h.myPhys, h.myMPI, h.myBC, h.myIO);
      h.myBlock.Post(h.myOperator, h.myPhys, h.myMPI, h.myBC, h.myIO);
      nuc3d::postproc &pp = *h.myBlock.myPost;
      Writer w(ranked(argv[3], rank));
      w.fields("Q", h.myBlock.myPDE.getQ());
      using namespace taps_access;
      w.scalar("enstrophy_glb", pp.*member(EnsGlb()));
      w.scalar("kinetic_glb", pp.*member(KinGlb()));
      w.scalar("enstrophy", pp.*member(Ens()));
      w.scalar("kinetic", pp.*member(Kin()));
      w.fields("qfield", pp.*member(QField()));
    } else if (mode == "time") {
      if (argc < 4) return 2;
      int n = std::atoi(argv[2]);
      int warm = std::atoi(argv[3]);
      for (int s = 0; s < warm; ++s) h.myBlock.solve(h.myOperator, h.myPhys, h.myMPI, h.myBC, h.myIO);
      double sum = 0.0;
      for (int s = 0; s < n; ++s) {
        h.myBlock.solve(h.myOperator, h.myPhys, h.myMPI, h.myBC, h.myIO);
        double wt = h.myBlock.wall_time, wmax = 0.0;
        MPI_Allreduce(&wt, &wmax, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
        sum += wmax;
      }
      if (rank == 0) {
        std::printf("{\"steps\": %d, \"warmup\": %d, \"solve_seconds\": %.9g}\n", n, warm, sum);
        std::fflush(stdout);
      }
    } else {
      std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
      return 2;
    }
    MPI_Barrier(MPI_COMM_WORLD);
  }
  return 0;
}
