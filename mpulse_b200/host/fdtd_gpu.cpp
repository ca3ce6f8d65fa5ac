// fdtd_gpu.cpp - see fdtd_gpu.h.
#include "fdtd_gpu.h"

#include "globals.h"
#include "parameter.h"
#include "periodic_bound.h"
#include "process.h"
#include "storage.h"

#include <cmath>
#include <cstdlib>
#include <iostream>
#include <vector>

namespace {

const char *kFieldNames[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};

}  // namespace

// --------------------------------------------------------------------------
// plug-in parameter blocks

ParameterMap *GpuCpmlBlock::MakeParamMap(ParameterMap *pm) {
  pm = CurrentFactory::MakeParamMap(pm);
  (*pm)["d"] = WParameter(new ParameterValue<int>(&thickness, 8));
  (*pm)["kappaMax"] = WParameter(new ParameterValue<double>(&kappaMax, 15));
  (*pm)["aMax"] = WParameter(new ParameterValue<double>(&aMax, 0.25));
  (*pm)["sigmaMax"] = WParameter(new ParameterValue<double>(&sigmaMax, 3));
  return pm;
}

ParameterMap *GpuPlasmaBlock::MakeParamMap(ParameterMap *pm) {
  pm = CurrentFactory::MakeParamMap(pm);
  if (current) {
    (*pm)["em"] = WParameter(new ParameterValue<double>(&em, 1.0));
    (*pm)["gamma"] = WParameter(new ParameterValue<double>(&gamma, 0.1));
    (*pm)["rho_bg"] = WParameter(new ParameterValue<double>(&rho_bg, 0.0));
  } else {
    (*pm)["nu"] = WParameter(new ParameterValue<double>(&nu, 1.0));
    (*pm)["mpa"] = WParameter(new ParameterValue<double>(&mpa, 1.0));
    (*pm)["Wion"] = WParameter(new ParameterValue<double>(&Wion, 1.0));
    (*pm)["K"] = WParameter(new ParameterValue<int>(&K, 5));
  }
  return pm;
}

ParameterMap *GpuSourceBlock::MakeParamMap(ParameterMap *pm) {
  pm = CurrentFactory::MakeParamMap(pm);
  (*pm)["d"] = WParameter(new ParameterValue<int>(&distance, 15));
  if (kind == MP_SOURCE_PLANE_WAVE || kind == MP_SOURCE_PLANE_GAUSS) {
    (*pm)["kx"] = WParameter(new ParameterValue<double>(&kx, 0));
    (*pm)["ky"] = WParameter(new ParameterValue<double>(&ky, 0));
    (*pm)["kz"] = WParameter(new ParameterValue<double>(&kz, 1));
    (*pm)["Hx"] = WParameter(new ParameterValue<double>(&Hx, 0));
    (*pm)["Hy"] = WParameter(new ParameterValue<double>(&Hy, 0));
    (*pm)["Hz"] = WParameter(new ParameterValue<double>(&Hz, 0));
    (*pm)["eps"] = WParameter(new ParameterValue<double>(&eps, 1));
  }
  if (kind == MP_SOURCE_PLANE_WAVE) {
    (*pm)["Hx_bg"] = WParameter(new ParameterValue<double>(&Hx_bg, 0));
    (*pm)["Hy_bg"] = WParameter(new ParameterValue<double>(&Hy_bg, 0));
    (*pm)["Hz_bg"] = WParameter(new ParameterValue<double>(&Hz_bg, 0));
    (*pm)["Ex_bg"] = WParameter(new ParameterValue<double>(&Ex_bg, 0));
    (*pm)["Ey_bg"] = WParameter(new ParameterValue<double>(&Ey_bg, 0));
    (*pm)["Ez_bg"] = WParameter(new ParameterValue<double>(&Ez_bg, 0));
    (*pm)["ramp"] = WParameter(new ParameterValue<double>(&ramp, 0.5));
  }
  if (kind == MP_SOURCE_PLANE_GAUSS) {
    (*pm)["width"] = WParameter(new ParameterValue<double>(&width, 10));
    (*pm)["offset"] = WParameter(new ParameterValue<double>(&offset, 40));
  }
  if (kind == MP_SOURCE_SHORT_PULSE || kind == MP_SOURCE_FOCUSED_PULSE) {
    (*pm)["length"] = WParameter(new ParameterValue<double>(&length, 1.));
    (*pm)["width"] = WParameter(new ParameterValue<double>(&waist, 1.));
    (*pm)["om0"] = WParameter(new ParameterValue<double>(&om0, 2 * M_PI));
    (*pm)["TShift"] = WParameter(new ParameterValue<double>(&TShift, 0));
    (*pm)["ZShift"] = WParameter(new ParameterValue<double>(&ZShift, 0));
    (*pm)["Phase"] = WParameter(new ParameterValue<double>(&Phase, 0));
    (*pm)["amp"] = WParameter(new ParameterValue<double>(&amp, 1));
    (*pm)["eps"] = WParameter(new ParameterValue<double>(&eps, 1));
  }
  if (kind == MP_SOURCE_FOCUSED_PULSE) {
    // FocusedPulseInject::MakeParamMap (focusedpulseinject.cpp:39-57): the
    // angular-spectrum oversampling has no meaning for the closed form
    (*pm)["OversampleX"] = WParameter(new ParameterValue<int>(&oversampleX, 1));
    (*pm)["OversampleY"] = WParameter(new ParameterValue<int>(&oversampleY, 1));
  }
  if (kind == MP_SOURCE_GAUSS_BEAM) {  // GaussInject::MakeParamMap (gaussinject.cpp:33-49)
    (*pm)["SizeT"] = WParameter(new ParameterValue<int>(&SizeT, 4096));
    (*pm)["length"] = WParameter(new ParameterValue<double>(&length, 1.));
    (*pm)["width"] = WParameter(new ParameterValue<double>(&width, 1.));
    (*pm)["k0"] = WParameter(new ParameterValue<double>(&k0, 2 * M_PI));
    (*pm)["Shift"] = WParameter(new ParameterValue<double>(&Shift, 0));
    (*pm)["Time"] = WParameter(new ParameterValue<double>(&Time, 0));
    (*pm)["amp"] = WParameter(new ParameterValue<double>(&amp, 1));
    (*pm)["eps"] = WParameter(new ParameterValue<double>(&eps, 1));
    (*pm)["toff"] = WParameter(new ParameterValue<int>(&toff, 0));
  }
  return pm;
}

void GpuSourceBlock::fill(mp_source &s) const {
  s.kind = kind;
  s.distance = distance;
  if (kind == MP_SOURCE_PLANE_WAVE || kind == MP_SOURCE_PLANE_GAUSS) {
    s.k[0] = kx; s.k[1] = ky; s.k[2] = kz;
    s.H[0] = Hx; s.H[1] = Hy; s.H[2] = Hz;
    s.eps = eps;
  }
  if (kind == MP_SOURCE_PLANE_WAVE) {
    s.H_bg[0] = Hx_bg; s.H_bg[1] = Hy_bg; s.H_bg[2] = Hz_bg;
    s.E_bg[0] = Ex_bg; s.E_bg[1] = Ey_bg; s.E_bg[2] = Ez_bg;
    s.ramp = ramp;
  }
  if (kind == MP_SOURCE_PLANE_GAUSS) {
    s.width = width;
    s.offset = offset;
  }
  if (kind == MP_SOURCE_SHORT_PULSE || kind == MP_SOURCE_FOCUSED_PULSE) {
    s.length = length; s.waist = waist; s.om0 = om0;
    s.t_shift = TShift; s.z_shift = ZShift; s.phase = Phase; s.amp = amp; s.eps = eps;
  }
  if (kind == MP_SOURCE_GAUSS_BEAM) {
    s.t_size = SizeT; s.length = length; s.width = width; s.k0 = k0; s.shift = Shift;
    s.time = Time; s.amp = amp; s.eps = eps; s.t_off = toff;
  }
}

// --------------------------------------------------------------------------
// the solver

FDTD_GPU::FDTD_GPU(int solver_)
    : solver(solver_), storage(0), ctx(0), hostDirty(true), stepsSinceSync(0) {
  for (int f = 0; f < 6; ++f) pF[f] = 0;
  for (int q = 0; q < 4; ++q) pPlasma[q] = 0;
}

FDTD_GPU::~FDTD_GPU() { mp_destroy(ctx); }

ParameterMap *FDTD_GPU::MakeParamMap(ParameterMap *pm) {
  pm = FieldSolver::MakeParamMap(pm);
  (*pm)["eps"] = WParameter(new ParameterValue<double>(&eps, 1.0));
  (*pm)["chi"] = WParameter(new ParameterValue<double>(&chi, 0.1));
  const char *le[3] = {"L1eps", "L2eps", "L3eps"};
  const char *ld[3] = {"L1delta", "L2delta", "L3delta"};
  const char *lo[3] = {"L1Om2", "L2Om2", "L3Om2"};
  for (int n = 0; n < 3; ++n) {
    (*pm)[le[n]] = WParameter(new ParameterValue<double>(&LEps[n], 0.0));
    (*pm)[ld[n]] = WParameter(new ParameterValue<double>(&LDelta[n], 0.0));
    (*pm)[lo[n]] = WParameter(new ParameterValue<double>(&LOm2[n], 1.0));
  }
  (*pm)["medium_z0"] = WParameter(new ParameterValue<int>(&mediumZ0, 0));
  (*pm)["medium_z1"] = WParameter(new ParameterValue<int>(&mediumZ1, 1 << 30));
  (*pm)["eps_bg"] = WParameter(new ParameterValue<double>(&epsBg, 1.0));
  (*pm)["fp32"] = WParameter(new ParameterValue<int>(&fp32, 0));
  (*pm)["sync_interval"] = WParameter(new ParameterValue<int>(&syncInterval, 1));
  (*pm)["device"] = WParameter(new ParameterValue<int>(&device, 0));
  (*pm)["cpml_border"] =
      WParameter(new ParameterRebuild<GpuCpmlBlockT<MP_CPML_ALL>, CurrentFactory>(&blocks));
  (*pm)["cpml_border_1d"] =
      WParameter(new ParameterRebuild<GpuCpmlBlockT<MP_CPML_Z>, CurrentFactory>(&blocks));
  (*pm)["wave_inject"] =
      WParameter(new ParameterRebuild<GpuSourceBlockT<MP_SOURCE_PLANE_WAVE>, CurrentFactory>(&blocks));
  (*pm)["plane_gauss_inject"] =
      WParameter(new ParameterRebuild<GpuSourceBlockT<MP_SOURCE_PLANE_GAUSS>, CurrentFactory>(&blocks));
  (*pm)["short_pulse_inject"] =
      WParameter(new ParameterRebuild<GpuSourceBlockT<MP_SOURCE_SHORT_PULSE>, CurrentFactory>(&blocks));
  (*pm)["gauss_inject"] =
      WParameter(new ParameterRebuild<GpuSourceBlockT<MP_SOURCE_GAUSS_BEAM>, CurrentFactory>(&blocks));
  (*pm)["focused_pulse_inject"] =
      WParameter(new ParameterRebuild<GpuSourceBlockT<MP_SOURCE_FOCUSED_PULSE>, CurrentFactory>(&blocks));
  (*pm)["plasma"] = WParameter(new ParameterRebuild<GpuPlasmaBlockT<0>, CurrentFactory>(&blocks));
  (*pm)["plasma_current"] = WParameter(new ParameterRebuild<GpuPlasmaBlockT<1>, CurrentFactory>(&blocks));
  return pm;
}

void FDTD_GPU::check(int rc, const char *what) {
  if (rc == MP_OK) return;
  char msg[512];
  mp_last_error(ctx, msg, sizeof msg);
  std::cerr << "FDTD_GPU: " << what << " failed (" << rc << "): " << (ctx ? msg : mp_create_error()) << "\n";
  exit(-1);
}

void FDTD_GPU::initStorage(Storage *storage_) {
  storage = storage_;
  Globals &g = Globals::instance();
  mp_config_defaults(&cfg);
  cfg.nx = g.gridX();
  cfg.ny = g.gridY();
  cfg.nz = g.gridZ();
  cfg.dx = g.gridDX();
  cfg.dy = g.gridDY();
  cfg.dz = g.gridDZ();
  cfg.dt = g.dt();
  cfg.precision = fp32 ? MP_FP32 : MP_FP64;
  cfg.solver = solver;
  const Boundary &b = storage->getBoundary();
  if (dynamic_cast<const SingleXYPeriodicBoundary *>(&b)) cfg.boundary = MP_BOUNDARY_XY_PERIODIC;
  else if (dynamic_cast<const SinglePeriodicBoundary *>(&b)) cfg.boundary = MP_BOUNDARY_PERIODIC;
  else {
    std::cerr << "FDTD_GPU: only single_periodic and single_xy_periodic are supported on one GPU\n";
    exit(-1);
  }
  cfg.eps = eps;
  cfg.chi = chi;
  for (int n = 0; n < 3; ++n) {
    cfg.poles[n].eps = LEps[n];
    cfg.poles[n].delta = LDelta[n];
    cfg.poles[n].om2 = LOm2[n];
  }
  cfg.medium_z0 = mediumZ0;
  cfg.medium_z1 = mediumZ1;
  cfg.eps_bg = epsBg;
  cfg.device = device;
  cfg.n_sources = 0;
  for (std::list<CurrentFactory *>::iterator it = blocks.begin(); it != blocks.end(); ++it) {
    if (GpuCpmlBlock *cp = dynamic_cast<GpuCpmlBlock *>(*it)) {
      cfg.cpml = cp->kind;
      cfg.cpml_d = cp->thickness;
      cfg.cpml_kappa_max = cp->kappaMax;
      cfg.cpml_a_max = cp->aMax;
      cfg.cpml_sigma_max = cp->sigmaMax;
    } else if (GpuSourceBlock *sb = dynamic_cast<GpuSourceBlock *>(*it)) {
      if (cfg.n_sources == MP_MAX_SOURCES) {
        std::cerr << "FDTD_GPU: at most " << MP_MAX_SOURCES << " injectors\n";
        exit(-1);
      }
      sb->fill(cfg.sources[cfg.n_sources++]);
    } else if (GpuPlasmaBlock *pb = dynamic_cast<GpuPlasmaBlock *>(*it)) {
      if (pb->current) {
        cfg.plasma_current = 1;
        cfg.plasma_em = pb->em;
        cfg.plasma_gamma = pb->gamma;
        cfg.plasma_rho_bg = pb->rho_bg;
      } else {
        cfg.plasma = 1;
        cfg.plasma_nu = pb->nu;
        cfg.plasma_mpa = pb->mpa;
        cfg.plasma_wion = pb->Wion;
        cfg.plasma_k = pb->K;
      }
    }
  }
  check(mp_create(&cfg, &ctx), "mp_create");
  // the plasma plug-ins' grids (plasmadensity.cpp:17, plasmacurrent.cpp:35-39)
  const char *plasmaNames[4] = {"PlasmaDensity", "PlasmaJx", "PlasmaJy", "PlasmaJz"};
  for (int q = 0; q < 4; ++q)
    pPlasma[q] = (cfg.plasma || cfg.plasma_current) ? storage->addGrid(plasmaNames[q]) : 0;
  // the grids the rest of MPulse sees (FDTD_PLRCCore::coreInitStorage,
  // fdtd_plrc.cpp:17-23, :59-65)
  for (int f = 0; f < 6; ++f) pF[f] = storage->addGrid(kFieldNames[f]);
  storage->addToGroup("E", "Ex");
  storage->addToGroup("E", "Ey");
  storage->addToGroup("E", "Ez");
  storage->addToGroup("B", "Bx");
  storage->addToGroup("B", "By");
  storage->addToGroup("B", "Bz");
  hostDirty = true;
}

void FDTD_GPU::upload() {
  const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
  std::vector<double> h(size_t(nz + 2) * ny * nx);
  for (int f = 0; f < 6; ++f) {
    DataGrid &G = *pF[f];
    for (int k = 0; k <= nz + 1; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) h[(size_t(k) * ny + (j - 1)) * nx + (i - 1)] = G(i, j, k);
    check(mp_upload(ctx, kFieldNames[f], &h[0], h.size()), "mp_upload");
  }
  hostDirty = false;
}

void FDTD_GPU::download() {
  const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
  std::vector<double> h(size_t(nz + 2) * ny * nx);
  const char *plasmaNames[4] = {"PlasmaDensity", "PlasmaJx", "PlasmaJy", "PlasmaJz"};
  for (int f = 0; f < 10; ++f) {
    DataGrid *pG = f < 6 ? pF[f] : pPlasma[f - 6];
    if (!pG) continue;
    check(mp_download(ctx, f < 6 ? kFieldNames[f] : plasmaNames[f - 6], &h[0], h.size()), "mp_download");
    DataGrid &G = *pG;
    for (int k = 0; k <= nz + 1; ++k)
      for (int j = 0; j <= ny + 1; ++j)
        for (int i = 0; i <= nx + 1; ++i) {
          // x/y ghosts are the periodic images (periodic_bound.cpp:10-51)
          const int ii = i == 0 ? nx : (i == nx + 1 ? 1 : i);
          const int jj = j == 0 ? ny : (j == ny + 1 ? 1 : j);
          G(i, j, k) = h[(size_t(k) * ny + (jj - 1)) * nx + (ii - 1)];
        }
  }
}

void FDTD_GPU::stepSchemeInit(double) {
  // MPulse never calls it (fieldsim.cpp:109-112 only calls stepScheme).
}

void FDTD_GPU::stepScheme(double) {
  if (hostDirty) upload();
  check(mp_set_time(ctx, Process::instance().getTime()), "mp_set_time");
  check(mp_step(ctx, 1), "mp_step");
  if (syncInterval > 0 && ++stepsSinceSync >= syncInterval) {
    download();
    stepsSinceSync = 0;
  }
}

void registerGpuSolvers(ParameterMap *pm, FieldSolver **solver) {
  (*pm)["fdtd-gpu-plain"] = WParameter(new ParameterRebuild<FDTD_GPU_Plain, FieldSolver>(solver));
  (*pm)["fdtd-gpu-nl"] = WParameter(new ParameterRebuild<FDTD_GPU_Nonlinear, FieldSolver>(solver));
  (*pm)["fdtd-gpu-plrc-lin"] = WParameter(new ParameterRebuild<FDTD_GPU_PLRCLin, FieldSolver>(solver));
  (*pm)["fdtd-gpu-plrc-nonlin"] = WParameter(new ParameterRebuild<FDTD_GPU_PLRCNonlin, FieldSolver>(solver));
}
