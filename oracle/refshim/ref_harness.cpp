// Test infrastructure only: the main() of the oracle build of MPulse.
//
// It replaces mpulse.cpp:18-78 and drives MPulse's own objects exactly like
// Process::run (process.cpp:17-31) does, with three additions that the
// reference cannot express by itself and that the parity tests need:
//
//  1. "fdtd-plrc-masked-lin" / "fdtd-plrc-masked-nonlin": MPulse's own
//     FDTD_PLRCSolver<> (fdtd_plrc.t) over a core that restricts the Lorentz
//     medium (eps, chi, poles) to the z-planes [medium_z0, medium_z1] and treats
//     the other cells as a background of permittivity eps_bg with no poles and no
//     Kerr term.  Per cell it delegates to the reference's own plrcStepD
//     (fdtd_plrc.cpp:94-261 / :304-427) after swapping eps / chi / plrcData.
//  2. "raw_init { file F }": reads initial Ex..Bz (full ghost range, C order)
//     from a raw double file, so parity cases can start from seeded random
//     fields instead of only the analytic initialisers.
//  3. Output: after the run every full-size grid named on the command line is
//     written as raw doubles (C order, ghost cells included), and the wall time
//     of the step loop alone is printed as one JSON line.
//  4. "slab_xy_periodic { z0 Z0 z1 Z1 }": the single_xy_periodic boundary
//     (periodic_bound.cpp:87-130) over the z-planes Z0..Z1 of the global grid
//     only (plus one ghost plane each side), the slab one process of MPulse's
//     z-split MPI run holds (mpi_bound.cpp:66-109), with no halo exchange.
//     Storage::getBorderExtent (storage.cpp:208-318) then gives the CPML faces
//     and the injection plane only to the slabs that contain them, so a set
//     of slab processes does the per-cell work of the whole grid; used to time
//     the reference on the host cores (the fields at slab edges are not those
//     of the whole grid).
//
// Usage: mpulse_ref SETUP OUTDIR [grid names...]
// Environment: MPULSE_REF_WARMUP=W times only the steps after the first W.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <list>
#include <map>
#include <sstream>
#include <string>
#include <vector>

// Process keeps its field simulation and globals private (process.h:23-35);
// the harness needs to create a FieldSimulation subclass and read its grids.
#define private public
#define protected public
#include "process.h"
#include "fieldsim.h"
#include "storage.h"
#include "diagnostic.h"
#include "fdtd_plrc.h"
#include "init.h"
#include "periodic_bound.h"
#include "globals.h"
#undef private
#undef protected

#ifdef MPB_WITH_GPU
// MPulse with the B200 FieldSolver plug-in registered beside its own solvers
#include "fdtd_gpu.h"
#endif

namespace {

template <class Base>
class MaskedCore : public Base {
 protected:
  int medium_z0, medium_z1;
  double eps_bg;

  bool inMedium(int k) const { return k >= medium_z0 && k <= medium_z1; }

 public:
  void plrcStepD(double dt, int i, int j, int k, double dx, double dy, double dz,
                 double Jx, double Jy, double Jz) {
    if (inMedium(k)) {
      Base::plrcStepD(dt, i, j, k, dx, dy, dz, Jx, Jy, Jz);
      return;
    }
    const double epsSave = this->eps;
    const typename Base::PLRCData dataSave = this->plrcData;
    this->eps = eps_bg;
    for (int n = 0; n < 3; ++n) {
      this->plrcData.dchi0[n] = 0.0;
      this->plrcData.dxi0[n] = 0.0;
      this->plrcData.Crec[n] = 0.0;
    }
    this->plrcData.sumChi0 = 0.0;
    this->plrcData.sumXi0 = 0.0;
    callBase(dt, i, j, k, dx, dy, dz, Jx, Jy, Jz);
    this->eps = epsSave;
    this->plrcData = dataSave;
  }

  void plrcStepB(double dt, int i, int j, int k, double dx, double dy, double dz,
                 double Jx, double Jy, double Jz) {
    Base::plrcStepB(dt, i, j, k, dx, dy, dz, Jx, Jy, Jz);
  }

  ParameterMap *CustomParamMap(ParameterMap *pm) {
    pm = Base::CustomParamMap(pm);
    (*pm)["medium_z0"] = WParameter(new ParameterValue<int>(&medium_z0, 0));
    (*pm)["medium_z1"] = WParameter(new ParameterValue<int>(&medium_z1, 1 << 30));
    (*pm)["eps_bg"] = WParameter(new ParameterValue<double>(&eps_bg, 1.0));
    return pm;
  }

 private:
  void callBase(double dt, int i, int j, int k, double dx, double dy, double dz,
                double Jx, double Jy, double Jz);
};

// The linear core has no Kerr term; the nonlinear core's chi is zeroed outside
// the medium.
template <>
void MaskedCore<FDTD_PLRCLinCore>::callBase(double dt, int i, int j, int k, double dx,
                                            double dy, double dz, double Jx, double Jy,
                                            double Jz) {
  FDTD_PLRCLinCore::plrcStepD(dt, i, j, k, dx, dy, dz, Jx, Jy, Jz);
}

template <>
void MaskedCore<FDTD_PLRCNonlinCore>::callBase(double dt, int i, int j, int k, double dx,
                                               double dy, double dz, double Jx, double Jy,
                                               double Jz) {
  const double chiSave = this->chi;
  this->chi = 0.0;
  FDTD_PLRCNonlinCore::plrcStepD(dt, i, j, k, dx, dy, dz, Jx, Jy, Jz);
  this->chi = chiSave;
}

class SlabXYPeriodicBoundary : public SingleXYPeriodicBoundary {
 public:
  int z0 = 1, z1 = 1;
  GridIndex lo, hi;
  void init() {
    lo = Globals::instance().gridLow();
    hi = Globals::instance().gridHigh();
    const int g0 = lo[2], g1 = hi[2];
    lo[2] = std::max(g0, z0 - 1);
    hi[2] = std::min(g1, z1 + 1);
  }
  const GridIndex &RegionLow() const { return lo; }
  const GridIndex &RegionHigh() const { return hi; }

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm) {
    pm = Rebuildable::MakeParamMap(pm);
    (*pm)["z0"] = WParameter(new ParameterValue<int>(&z0, 1));
    (*pm)["z1"] = WParameter(new ParameterValue<int>(&z1, 1));
    return pm;
  }
};

typedef FDTD_PLRCSolver<MaskedCore<FDTD_PLRCLinCore> > MaskedLin;
typedef FDTD_PLRCSolver<MaskedCore<FDTD_PLRCNonlinCore> > MaskedNonlin;

// Reads Ex, Ey, Ez, Bx, By, Bz (in that order) over the full storage range.
class RawInit : public FieldSimInit {
 public:
  std::string file;
  void init(Storage &fields) {
    std::ifstream in(file.c_str(), std::ios::binary);
    if (!in) {
      std::cerr << "raw_init: cannot open " << file << "\n";
      std::exit(-1);
    }
    const char *names[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};
    for (int f = 0; f < 6; ++f) {
      DataGrid &g = fields.getGrid(names[f]);
      in.read(reinterpret_cast<char *>(g.getRawData()), std::streamsize(g.getSize() * sizeof(double)));
      if (!in) {
        std::cerr << "raw_init: short file " << file << "\n";
        std::exit(-1);
      }
    }
  }

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm) {
    pm = Rebuildable::MakeParamMap(pm);
    (*pm)["file"] = WParameter(new ParameterValue<std::string>(&file, "init.bin"));
    return pm;
  }
};

class HarnessFieldSim : public FieldSimulation {
 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm) {
    pm = FieldSimulation::MakeParamMap(pm);
    (*pm)["fdtd-plrc-masked-lin"] =
        WParameter(new ParameterRebuild<MaskedLin, FieldSolver>(&solver));
    (*pm)["fdtd-plrc-masked-nonlin"] =
        WParameter(new ParameterRebuild<MaskedNonlin, FieldSolver>(&solver));
    (*pm)["raw_init"] =
        WParameter(new ParameterRebuild<RawInit, FieldSimInit>(&initializers));
    (*pm)["slab_xy_periodic"] =
        WParameter(new ParameterRebuild<SlabXYPeriodicBoundary, Boundary>(&boundary));
#ifdef MPB_WITH_GPU
    registerGpuSolvers(pm, &solver);
#endif
    return pm;
  }
};

class HarnessProcess : public Process {
 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm) {
    pm = Rebuildable::MakeParamMap(pm);
    (*pm)["globals"] = WParameter(new ParameterRebuild<Globals, Globals>(&globals));
    (*pm)["fieldsim"] =
        WParameter(new ParameterRebuild<HarnessFieldSim, FieldSimulation>(&fieldSim));
    return pm;
  }
};

void writeGrid(const std::string &dir, const std::string &name, DataGrid &g) {
  const std::string path = dir + "/" + name + ".bin";
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::cerr << "cannot write " << path << "\n";
    std::exit(-1);
  }
  std::fwrite(g.getRawData(), sizeof(double), g.getSize(), f);
  std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::cerr << "usage: mpulse_ref SETUP OUTDIR [grid names...]\n";
    return 2;
  }
  Globals::setArgc(argc);
  Globals::setArgv(argv);
  std::ifstream setup(argv[1]);
  if (!setup) {
    std::cerr << "cannot open " << argv[1] << "\n";
    return 2;
  }
  // MPulse prints a line per cycle to stdout (process.cpp:24-25); keep stdout
  // for the JSON result by sending the chatter to stderr.
  std::streambuf *coutBuf = std::cout.rdbuf(std::cerr.rdbuf());

  HarnessProcess *process = new HarnessProcess();
  process->Rebuild(setup);
  process->init();

  // MPULSE_REF_WARMUP=W leaves the first W steps out of the timing.
  const int T = Globals::instance().totalTime();
  const char *w = std::getenv("MPULSE_REF_WARMUP");
  const int warm = w ? std::atoi(w) : 0;
  auto t0 = std::chrono::steady_clock::now();
  for (process->time = 0; process->time < T; ++process->time) {
    if (process->time == warm) t0 = std::chrono::steady_clock::now();
    process->fieldSim->execute();
    DiagnosticManager::instance().execute();
  }
  const auto t1 = std::chrono::steady_clock::now();
  const double seconds = std::chrono::duration<double>(t1 - t0).count();
  const int timed = T > warm ? T - warm : T;

  Storage &st = *process->fieldSim;
  for (int a = 3; a < argc; ++a) writeGrid(argv[2], argv[a], st.getGrid(argv[a]));

  const GridIndex lo = st.getLow(), hi = st.getHigh();
  const long long cells = (long long)(hi[0] - lo[0] - 1) * (hi[1] - lo[1] - 1) * (hi[2] - lo[2] - 1);
  std::cout.rdbuf(coutBuf);
  std::printf("{\"steps\": %d, \"timed_steps\": %d, \"cells\": %lld, \"seconds\": %.9f, \"low\": [%d, %d, %d], \"high\": [%d, %d, %d]}\n",
              T, timed, cells, seconds, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
  std::fflush(stdout);
  // The reference never frees its plug-ins; skip teardown the same way.
  std::_Exit(0);
}
