// fdtd_gpu.h - MPulse FieldSolver plug-in that runs MPulse's time step on a
// B200 through the C ABI of include/mpulse_b200.h.
//
// It is the host side of the drop-in: a FieldSolver (src/fieldsolver.h:10-37)
// registered beside MPulse's own solvers, reading the same setup-file keys with
// the same defaults as FDTD_PLRCSolver (src/fdtd_plrc.t:411-473,
// src/fdtd_plrc.cpp:461-465), FDTD_Plain (src/fdtd_plain.cpp) and
// FDTD_Nonlinear (src/fdtd_nl.cpp:146-153), including the nested plug-in blocks
// cpml_border, cpml_border_1d, wave_inject, plane_gauss_inject,
// short_pulse_inject, gauss_inject, focused_pulse_inject, plasma and
// plasma_current.  Those blocks do not create host Currents here: their
// parameters configure the device context, which computes the CPML psi fields
// and the TF/SF planes inside the step kernels.
//
// The Storage grids Ex..Bz stay the interface to the rest of MPulse: the
// initialisers write them before the first step (src/fieldsim.cpp:91-106), the
// solver uploads them once, and it downloads them back into Storage every
// `sync_interval` steps for the diagnostics (src/fielddiag.cpp:255-286).
//
// Errors follow MPulse's convention (message on std::cerr, exit(-1)), e.g.
// src/fdtd_plrc.t:20-24; the C ABI underneath never exits.
#ifndef MPULSE_B200_FDTD_GPU_H
#define MPULSE_B200_FDTD_GPU_H

#include "currentfactory.h"
#include "fieldsolver.h"
#include "mpulse.h"
#include "mpulse_b200.h"

#include <list>

class Storage;

// Parameters of cpml_border (CPMLBorder::MakeParamMap, cpml_border.cpp:142-151)
// and cpml_border_1d (cpml_border.cpp:246-255).
class GpuCpmlBlock : public CurrentFactory {
 public:
  explicit GpuCpmlBlock(int kind_) : kind(kind_) {}
  void initCurrents(Storage *, FieldSolver *) {}
  int kind;
  int thickness;
  double kappaMax, aMax, sigmaMax;

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm = NULL);
};

template <int KIND>
class GpuCpmlBlockT : public GpuCpmlBlock {
 public:
  GpuCpmlBlockT() : GpuCpmlBlock(KIND) {}
};

// Parameters of the injectors: wave_inject / plane_gauss_inject
// (sources.cpp:58-82, :225-241) and short_pulse_inject
// (shortpulseinject.cpp:33-49), with IncidentSource's "d"
// (incsource.cpp:80-86).
class GpuSourceBlock : public CurrentFactory {
 public:
  explicit GpuSourceBlock(int kind_) : kind(kind_) {}
  void initCurrents(Storage *, FieldSolver *) {}
  int kind;
  int distance;
  double kx, ky, kz, Hx, Hy, Hz, Hx_bg, Hy_bg, Hz_bg, Ex_bg, Ey_bg, Ez_bg;
  double ramp, width, offset, eps;
  double length, waist, om0, TShift, ZShift, Phase, amp;
  int SizeT, toff;
  int oversampleX, oversampleY;  // focused_pulse_inject keys, read and not used
  double k0, Shift, Time;
  void fill(mp_source &s) const;

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm = NULL);
};

template <int KIND>
class GpuSourceBlockT : public GpuSourceBlock {
 public:
  GpuSourceBlockT() : GpuSourceBlock(KIND) {}
};

// Parameters of the plasma plug-ins of FDTD_PLRCSolver (fdtd_plrc.t:431-436):
// "plasma" (PlasmaDensity::MakeParamMap, plasmadensity.cpp:52-61) and
// "plasma_current" (PlasmaCurrentFactory::MakeParamMap,
// plasmacurrent.cpp:6-15).  The device context computes both inside the E
// half-step kernel.
class GpuPlasmaBlock : public CurrentFactory {
 public:
  explicit GpuPlasmaBlock(int current_) : current(current_) {}
  void initCurrents(Storage *, FieldSolver *) {}
  int current;  // 0: plasma (density), 1: plasma_current
  double nu, mpa, Wion;
  int K;
  double em, gamma, rho_bg;

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm = NULL);
};

template <int CURRENT>
class GpuPlasmaBlockT : public GpuPlasmaBlock {
 public:
  GpuPlasmaBlockT() : GpuPlasmaBlock(CURRENT) {}
};

class FDTD_GPU : public FieldSolver {
 public:
  explicit FDTD_GPU(int solver_);
  virtual ~FDTD_GPU();

  void initStorage(Storage *storage_);
  void stepSchemeInit(double dt);
  void stepScheme(double dt);

 protected:
  ParameterMap *MakeParamMap(ParameterMap *pm = NULL);

 private:
  void upload();
  void download();
  void check(int rc, const char *what);

  int solver;
  Storage *storage;
  mp_ctx *ctx;
  mp_config cfg;
  bool hostDirty;
  int stepsSinceSync;

  // setup-file parameters
  double eps, chi;
  double LEps[3], LDelta[3], LOm2[3];
  int mediumZ0, mediumZ1;
  double epsBg;
  int fp32;
  int syncInterval;
  int device;
  std::list<CurrentFactory *> blocks;

  DataGrid *pF[6];
  DataGrid *pPlasma[4];  // PlasmaDensity, PlasmaJx..z (when the plug-ins are on)
};

template <int SOLVER>
class FDTD_GPU_T : public FDTD_GPU {
 public:
  FDTD_GPU_T() : FDTD_GPU(SOLVER) {}
};

typedef FDTD_GPU_T<MP_SOLVER_PLAIN> FDTD_GPU_Plain;
typedef FDTD_GPU_T<MP_SOLVER_NL> FDTD_GPU_Nonlinear;
typedef FDTD_GPU_T<MP_SOLVER_PLRC_LIN> FDTD_GPU_PLRCLin;
typedef FDTD_GPU_T<MP_SOLVER_PLRC_NONLIN> FDTD_GPU_PLRCNonlin;

// Adds "fdtd-gpu-plain", "fdtd-gpu-nl", "fdtd-gpu-plrc-lin" and
// "fdtd-gpu-plrc-nonlin" to a FieldSimulation's parameter map; the one line a
// maintainer adds to FieldSimulation::MakeParamMap (src/fieldsim.cpp:174-195).
void registerGpuSolvers(ParameterMap *pm, FieldSolver **solver);

#endif
