/*
 * mpulse_b200.h - C ABI of the B200 time-stepping path of MPulse.
 *
 * One context (mp_ctx) owns the device state of one simulation: the six Yee
 * field components, the PLRC accumulators of the Lorentz poles, the CPML psi
 * layers and the per-step injection planes.  The host calls mp_step() once per
 * MPulse time step (or once for many steps); everything in between stays in HBM.
 *
 * What each entry point replaces in MPulse (paths relative to the MPulse tree):
 *
 *   mp_create      FieldSimulation::init (src/fieldsim.cpp:31-107) as far as the
 *                  solver is concerned: FDTD_PLRCSolver::initStorage
 *                  (src/fdtd_plrc.t:18-76), FDTD_PLRCCore::coreInitStorage
 *                  (src/fdtd_plrc.cpp:13-86), CPMLBorder[OneD]::initCurrents /
 *                  initCoefficients (src/cpml_border.cpp:14-139, :158-243),
 *                  CPMLBorderCurrent::makeCoeff (src/cpml_border.cpp:287-339),
 *                  IncidentSource::initCurrents (src/incsource.cpp:16-77).
 *   mp_step        FieldSolver::stepScheme (src/fieldsolver.h:218-219) as
 *                  implemented by FDTD_PLRCSolver::stepScheme
 *                  (src/fdtd_plrc.t:127-168), FDTD_Plain::stepScheme
 *                  (src/fdtd_plain.cpp:31-35) and FDTD_Nonlinear::stepScheme
 *                  (src/fdtd_nl.cpp:32-36), including the boundary exchange of
 *                  Storage::applyBoundary (src/storage.cpp:194-204) done by
 *                  SinglePeriodicBoundary / SingleXYPeriodicBoundary
 *                  (src/periodic_bound.cpp:10-130), which becomes an index wrap.
 *                  One call advances n_steps steps; Process::time
 *                  (src/process.cpp:22) is kept in the context.
 *   mp_upload /    direct access to the Storage grids by name
 *   mp_download    (Storage::getGrid, src/storage.cpp:48-51), e.g. by the field
 *                  initialisers (src/pulseinit.cpp:22-27) and the diagnostics
 *                  (src/fielddiag.cpp:255-286).
 *   mp_last_error  replaces std::cerr + exit(-1) (e.g. src/fdtd_plrc.t:20-24).
 *
 * Conventions
 *   - Every function returns 0 (MP_OK) or a negative mp_status; none exits.
 *     The message of the last failure is available from mp_last_error().
 *   - Host buffers are caller-owned and always double precision; the device
 *     form (FP32 or FP64) is chosen by mp_config.precision.
 *   - Field layout on the host side ("plane layout"): nz+2 z-planes, index
 *     k = 0 .. nz+1 exactly as MPulse's global z index (src/globals.cpp:74-75);
 *     x and y hold the interior only (MPulse indices 1..n), x fastest:
 *         h[((size_t)k * ny + (j - 1)) * nx + (i - 1)]   for MPulse cell (i, j, k)
 *     MPulse's x/y ghost cells are periodic images in both boundaries it
 *     supports on one process and are not stored.  In the z-periodic boundary
 *     the planes 0 and nz+1 are images of nz and 1; they are ignored on upload
 *     and filled on download.
 *   - A context is used by one host thread at a time; all device work goes to
 *     the context's stream (mp_set_stream), so calls are asynchronous except
 *     mp_download, mp_sync and the status check at the end of mp_step.
 */
#ifndef MPULSE_B200_H
#define MPULSE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MP_ABI_VERSION 2
#define MP_MAX_POLES 3
#define MP_MAX_SOURCES 4

typedef enum mp_status {
  MP_OK = 0,
  MP_ERR_INVALID = -1,      /* bad argument or configuration */
  MP_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  MP_ERR_NO_MEMORY = -3,    /* device allocation failed */
  MP_ERR_NEWTON = -4,       /* Kerr Newton solve did not converge in a cell */
  MP_ERR_NONFINITE = -5,    /* a field value became NaN or Inf */
  MP_ERR_UNSUPPORTED = -6,  /* the configuration names a part that is not built */
  MP_ERR_NAME = -7,         /* unknown field name */
  MP_ERR_BOUNDS = -8        /* checked build only: a kernel index fell outside its array (access skipped) */
} mp_status;

typedef enum mp_precision { MP_FP64 = 0, MP_FP32 = 1 } mp_precision;

/* The solvers MPulse registers in FieldSimulation::MakeParamMap
 * (src/fieldsim.cpp:177-195). */
typedef enum mp_solver_kind {
  MP_SOLVER_PLAIN = 0,       /* "fdtd-plain"       src/fdtd_plain.cpp */
  MP_SOLVER_NL = 1,          /* "fdtd-nl"          src/fdtd_nl.cpp */
  MP_SOLVER_PLRC_LIN = 2,    /* "fdtd-plrc-lin"    src/fdtd_plrc.cpp:94-293 */
  MP_SOLVER_PLRC_NONLIN = 3  /* "fdtd-plrc-nonlin" src/fdtd_plrc.cpp:304-459 */
} mp_solver_kind;

/* The single-process boundaries (src/fieldsim.cpp:198-204). */
typedef enum mp_boundary_kind {
  MP_BOUNDARY_PERIODIC = 0,     /* "single_periodic"    periodic_bound.cpp:10-71 */
  MP_BOUNDARY_XY_PERIODIC = 1   /* "single_xy_periodic" periodic_bound.cpp:87-130 */
} mp_boundary_kind;

/* CPML plug-ins (src/fdtd_plrc.t:439-445). */
typedef enum mp_cpml_kind {
  MP_CPML_NONE = 0,
  MP_CPML_ALL = 1,   /* "cpml_border":    all six faces, cpml_border.cpp:14-139 */
  MP_CPML_Z = 2      /* "cpml_border_1d": z faces only, cpml_border.cpp:158-243 */
} mp_cpml_kind;

/* Incident-source plug-ins (src/fdtd_plrc.t:447-469). */
typedef enum mp_source_kind {
  MP_SOURCE_NONE = 0,
  MP_SOURCE_PLANE_WAVE = 1,     /* "wave_inject"        sources.cpp:8-173 */
  MP_SOURCE_PLANE_GAUSS = 2,    /* "plane_gauss_inject" sources.cpp:179-331 */
  MP_SOURCE_SHORT_PULSE = 3,    /* "short_pulse_inject" shortpulseinject.cpp */
  MP_SOURCE_FOCUSED_PULSE = 4,  /* "focused_pulse_inject" (see mp_source) */
  MP_SOURCE_GAUSS_BEAM = 5      /* "gauss_inject"       gaussinject.cpp */
} mp_source_kind;

/* Kernel form of the step.  All forms run the same cell arithmetic and agree
 * to the last bit, or within rounding (FP64: 1e-14 relative) where a kernel's
 * own vector code leaves a multiply-add to the compiler.  GLOBAL reads
 * global memory directly (L1/L2 serve the neighbours), one kernel per half
 * step; TMA stages each z-plane in a shared-memory ring with TMA tile loads
 * (needs nx a multiple of 32 and ny of 8, else mp_create fails with
 * MP_ERR_UNSUPPORTED); FUSED runs both half steps of a tile of columns in one
 * z-march and the cells on the tiles' edges in a second, small kernel (not
 * with a design region or the plasma plug-ins: MP_ERR_UNSUPPORTED); AUTO
 * picks the form measured fastest on B200 for the configuration. */
typedef enum mp_staging {
  MP_STAGING_AUTO = 0,
  MP_STAGING_GLOBAL = 1,
  MP_STAGING_TMA = 2,
  MP_STAGING_FUSED = 3
} mp_staging;

/* One Lorentz pole: MPulse's L<n>eps, L<n>delta, L<n>Om2
 * (src/fdtd_plrc.t:419-429, src/fdtd_plrc.h:85-90). */
typedef struct mp_lorentz_pole {
  double eps;    /* Delta epsilon of the pole */
  double delta;  /* damping delta (e-folding rate of chi(t)) */
  double om2;    /* resonance omega^2; must be > delta^2 and != 0 */
} mp_lorentz_pole;

/* One incident-source plug-in.  Only the fields of its kind are read. */
typedef struct mp_source {
  int kind;          /* mp_source_kind */
  int distance;      /* "d": TF/SF plane index, incsource.cpp:84 (default 15) */
  /* wave_inject, plane_gauss_inject (sources.cpp:58-82, :225-241) */
  double k[3];       /* kx ky kz */
  double H[3];       /* Hx Hy Hz */
  double H_bg[3];    /* Hx_bg.. (wave_inject only) */
  double E_bg[3];    /* Ex_bg.. (wave_inject only) */
  double ramp;       /* wave_inject ramp (default 0.5) */
  double width;      /* plane_gauss_inject width (default 10) */
  double offset;     /* plane_gauss_inject offset (default 40) */
  double eps;        /* background permittivity of the source (default 1) */
  /* short_pulse_inject (shortpulseinject.cpp:33-49).  focused_pulse_inject
   * takes the same keys (focusedpulseinject.cpp:39-57); its plug-in does not
   * compile in MPulse, and here it is defined as the same paraxial closed form
   * injected on the down face (OversampleX/Y have no meaning for it). */
  double length;     /* pulse duration parameter T */
  double waist;      /* "width": beam waist w0 */
  double om0;        /* carrier frequency (default 2 pi) */
  double t_shift;    /* TShift */
  double z_shift;    /* ZShift (focus offset from the grid centre) */
  double phase;      /* Phase, in units of 2 pi */
  double amp;        /* short pulse: peak Re Ex at the focus; gauss_inject: amp */
  /* gauss_inject (gaussinject.cpp:33-48); also uses length, width, amp, eps */
  int t_size;        /* SizeT: samples of the time transform (default 4096) */
  int t_off;         /* toff: first step of the injection (default 0) */
  double k0;         /* k0: central wavenumber (default 2 pi) */
  double shift;      /* Shift: focal shift along z */
  double time;       /* Time: time shift of the spectrum */
} mp_source;

typedef struct mp_config {
  int abi_version;          /* must be MP_ABI_VERSION */
  int nx, ny, nz;           /* grid-x, grid-y, grid-z (globals.cpp:53-55) */
  double dx, dy, dz;        /* grid-dx, grid-dy, grid-dz */
  double dt;                /* dt */
  int precision;            /* mp_precision of the device state */
  int solver;               /* mp_solver_kind */
  int boundary;             /* mp_boundary_kind */

  /* medium (fdtd_plrc.t:417-429, fdtd_plrc.cpp:461-465, fdtd_nl.cpp:146-153) */
  double eps;               /* eps_infinity of the medium */
  double chi;               /* Kerr chi (PLRC_NONLIN and NL) */
  mp_lorentz_pole poles[MP_MAX_POLES];
  /* The medium fills the z-planes medium_z0..medium_z1 (MPulse z index,
   * inclusive); cells outside are a background of permittivity eps_bg without
   * poles or Kerr term.  MPulse itself has a uniform medium: medium_z0 = 0,
   * medium_z1 = nz + 1. */
  int medium_z0, medium_z1;
  double eps_bg;

  /* CPML (cpml_border.cpp:142-151) */
  int cpml;                 /* mp_cpml_kind */
  int cpml_d;               /* d: layer thickness (default 8) */
  double cpml_kappa_max;    /* kappaMax (default 15) */
  double cpml_a_max;        /* aMax (default 0.25) */
  double cpml_sigma_max;    /* sigmaMax (default 3) */

  int n_sources;
  mp_source sources[MP_MAX_SOURCES];

  /* Kerr Newton solve: MPulse iterates until |E - E_old| <= 1e-9 with no cap
   * (fdtd_plrc.cpp:409-414).  Here the loop is capped; a cell that does not
   * converge makes mp_step return MP_ERR_NEWTON. */
  int newton_max_iter;      /* default 64 */
  double newton_tol;        /* default 1e-9 */

  int staging;              /* mp_staging: kernel form (results are the same) */
  int device;               /* CUDA device ordinal */

  /* Design region, an addition to MPulse (whose medium parameters are global
   * scalars, src/fdtd_plrc.h:82-90): in the box of MPulse cells
   * design_box = {x0, x1, y0, y1, z0, z1} (inclusive; empty when x0 > x1)
   * every cell has its own eps_infinity, a factor on the Delta epsilon of
   * every pole and a factor on chi.  They are uploaded by name as "DesignEps",
   * "DesignDepsScale" and "DesignChiScale", box-sized arrays with x fastest
   * (defaults: eps, 1, 1).  PLRC solvers only; the box lies inside the medium
   * planes and the interior.  A cell with factors 1 and eps_infinity = eps
   * gives the same results as a cell outside the box. */
  int design_box[6];

  /* Plasma plug-ins of the PLRC solvers (src/fdtd_plrc.t:431-436), PLRC
   * solvers only, global-load staging only, no design box, no adjoint.
   * "plasma" (PlasmaDensity, src/plasmadensity.cpp:18-61): every step, before
   * the E half, from I = |E^n|^2: rho <- (rho (1 + n I) + m I^K) / (1 - n I)
   * with n = dt nu / 2, m = dt mpa, and the conductivity Sigma = mpa Wion
   * I^(K-1) of the E update (numer - Sigma dt / 2, denom + Sigma dt / 2).
   * "plasma_current" (PlasmaCurrent, src/plasmacurrent.cpp:42-74): the
   * current J <- (J (1 - gamma dt / 2) - em dt E^n (rho + rho_bg)) /
   * (1 + gamma dt / 2), added to the E update after the other currents.
   * The density and the current are device state, named "PlasmaDensity" and
   * "PlasmaJx" / "PlasmaJy" / "PlasmaJz" as in MPulse's Storage, kept on the
   * planes 1..nz the E half updates (MPulse also evolves them on its ghost
   * cells, where they never reach the fields). */
  int plasma;               /* 1: the "plasma" plug-in */
  double plasma_nu;         /* nu: avalanche ionisation (default 1) */
  double plasma_mpa;        /* mpa: multi-photon ionisation (default 1) */
  double plasma_wion;       /* Wion: ionisation energy (default 1) */
  int plasma_k;             /* K: order of the multi-photon term (default 5) */
  int plasma_current;       /* 1: the "plasma_current" plug-in */
  double plasma_em;         /* em: e/m of the carriers (default 1) */
  double plasma_gamma;      /* gamma: friction (default 0.1) */
  double plasma_rho_bg;     /* rho_bg: constant background density (default 0) */
} mp_config;

/* Objectives of mp_objective / mp_adjoint (additions to MPulse). */
typedef enum mp_objective_kind {
  /* J = dt * sum over the steps n = 1..T of the sum over the cells of box of
   * Ex^2 + Ey^2 + Ez^2 after step n */
  MP_OBJ_E2_BOX = 1,
  /* J = dt * dx * dy * sum over n = 1..T of the sum over the x-y range of box
   * at the plane z = box[4] of Ex By - Ey Bx after step n (cell-centred
   * product of the stored components, no Yee interpolation) */
  MP_OBJ_SZ_PLANE = 2
} mp_objective_kind;

typedef struct mp_adjoint_config {
  int kind;               /* mp_objective_kind */
  int box[6];             /* x0, x1, y0, y1, z0, z1, MPulse cells, inclusive */
  int steps;              /* T: steps of the forward run */
  /* The forward state is saved every checkpoint_every steps; the reverse pass
   * recomputes each segment from its checkpoint, keeping E of every step of
   * the segment.  0 chooses the segment length from mem_budget (bytes of
   * device memory for checkpoints and the segment's E history; 0 = no limit,
   * which keeps all steps in one segment). */
  int checkpoint_every;
  double mem_budget;
} mp_adjoint_config;

typedef struct mp_ctx mp_ctx;

/* Fills *cfg with MPulse's parameter defaults (the ParameterValue defaults of
 * the MakeParamMap functions cited above) and a 32^3 grid. */
void mp_config_defaults(mp_config *cfg);

/* Allocates and zero-initialises all device state of a simulation.
 * MPulse: FDTD_PLRCSolver::initStorage and the plug-ins' initStorage. */
int mp_create(const mp_config *cfg, mp_ctx **out);

/* Releases everything mp_create allocated.  Accepts NULL. */
void mp_destroy(mp_ctx *ctx);

/* Runs all further device work of ctx on the given cudaStream_t (NULL: the
 * context's own stream). */
int mp_set_stream(mp_ctx *ctx, void *cuda_stream);

/* Number of doubles of the host buffer for field `name`.  Names follow
 * MPulse's Storage: "Ex" "Ey" "Ez" "Bx" "By" "Bz" (fdtd_plrc.cpp:17-23), the
 * PLRC accumulators "PsiR<n><c>" / "PsiI<n><c>" with n = 1..3, c = x, y, z
 * (fdtd_plrc.cpp:35-57) and, with the plasma plug-ins, "PlasmaDensity" and
 * "PlasmaJx" / "PlasmaJy" / "PlasmaJz" (plasmadensity.cpp:17,
 * plasmacurrent.cpp:35-39), all in the plane layout described above. */
int mp_field_size(mp_ctx *ctx, const char *name, size_t *count);

/* Copies a host field into the device state (converted to the device form). */
int mp_upload(mp_ctx *ctx, const char *name, const double *host, size_t count);

/* Copies a device field to the host.  Synchronises the context's stream. */
int mp_download(mp_ctx *ctx, const char *name, double *host, size_t count);

/* Advances the simulation by n_steps MPulse time steps, each the stepScheme
 * order of fdtd_plrc.t:127-168: E-side currents (CPML psi_E, TF/SF J), the D
 * update with PLRC / Kerr, the E boundary, H-side currents (CPML psi_H, TF/SF
 * M), the B update, the B boundary.  Synchronises once at the end to read the
 * device status word (Newton failures, non-finite values). */
int mp_step(mp_ctx *ctx, int n_steps);

/* Same as mp_step, without the synchronisation and status check; the status
 * is accumulated and returned by the next mp_check_status(). */
int mp_step_async(mp_ctx *ctx, int n_steps);
int mp_check_status(mp_ctx *ctx);

/* Process::time of the next step (src/process.cpp:22); starts at 0. */
int mp_get_time(mp_ctx *ctx, long long *time);
int mp_set_time(mp_ctx *ctx, long long time);

/* Waits for all work queued on the context's stream. */
int mp_sync(mp_ctx *ctx);

/* Device pointer, element count and element size (4 or 8 bytes) of a field's
 * device array, for zero-copy use by a caller that already lives on the GPU.
 * The device array has the plane layout above. */
int mp_device_field(mp_ctx *ctx, const char *name, void **dptr, size_t *count,
                    int *elem_bytes);

/* Total field energy as FieldEnergyDiag::calculate (src/fielddiag.cpp:255-286)
 * computes it: dx dy dz times the sum over the interior cells of
 * Ex^2 + Ey^2 + Ez^2 + Bx^2 + By^2 + Bz^2, accumulated in FP64 whatever the
 * field precision.  Synchronises the context's stream. */
int mp_field_energy(mp_ctx *ctx, double *energy);

/* Largest nz that mp_field_energy_noalloc accepts. */
#define MP_NOALLOC_MAX_PLANES 16384

/* The field energy of mp_field_energy for callers that cannot allocate device
 * memory.  No counterpart in MPulse.
 *
 * Who needs it: code that owns all of its device memory itself - an
 * application that runs its own pool or allocator and hands this library only
 * pointers into it, a process held to a fixed device-memory budget, or a
 * caller that must not enter cudaMalloc / cudaFree (they can synchronise the
 * whole device and stall work queued by others).  Such a caller cannot create
 * an mp_ctx (mp_create allocates) and so cannot use mp_field_energy, whose
 * scratch lives in the context.
 *
 * What it does: the same two kernels as mp_field_energy on caller-owned
 * device arrays.  fields[0..5] are Ex Ey Ez Bx By Bz in the plane layout
 * above ((nz+2) * ny * nx elements each, elem_bytes 4 for FP32 or 8 for FP64),
 * on the current device or one it can read as a peer; a pointer that is not
 * device or managed memory is rejected with MP_ERR_INVALID before anything
 * is launched.  The interior planes 1..nz are summed, times dx dy dz, in FP64.
 * Work goes to cuda_stream and the call blocks until that stream has drained
 * (cudaStreamSynchronize), then writes the result to the host double *energy.
 * A NULL cuda_stream is the legacy default stream, which also waits for and
 * holds up the other blocking streams of the device.  Because it blocks, it
 * cannot be used while cuda_stream is being captured into a CUDA graph.
 *
 * Limit: the scratch is a fixed array compiled into the library
 * (MP_NOALLOC_MAX_PLANES + 32 doubles, about 130 KB, held by every GPU that
 * loads the library until the process exits), one partial sum per z-plane, so
 * nz above MP_NOALLOC_MAX_PLANES is rejected with MP_ERR_INVALID and a message
 * from mp_last_error(NULL, ..).  It allocates nothing: no cudaMalloc, no
 * cudaFree, no allocating library call.  Every call looks up the array's
 * device address on the current device (cudaGetSymbolAddress, which neither
 * allocates nor synchronises), so it stays valid across cudaDeviceReset.
 * All calls share the array and it keeps the last call's contents (nothing in
 * it needs to start at zero); calls whose work overlaps on the GPU race on it
 * and must be serialised by the caller. */
int mp_field_energy_noalloc(const void *const fields[6], int elem_bytes, int nx, int ny, int nz,
                            double dx, double dy, double dz, void *cuda_stream, double *energy);

/* Number of CUDA kernel launches the context has issued so far. */
long long mp_launch_count(mp_ctx *ctx);

/* Advances the simulation by n_steps steps like mp_step while timing every
 * kernel with CUDA events on the context's stream; returns the average device
 * time of one launch of the E half-step kernel, of the B half-step kernel and
 * of all source-plane kernels of one step together, in milliseconds.  Used for
 * the per-kernel roofline; no counterpart in MPulse. */
int mp_kernel_times(mp_ctx *ctx, int n_steps, double *e_half_ms, double *b_half_ms,
                    double *sources_ms);

/* The Kerr solves of the E half-steps run since the previous call (or since
 * mp_create), read from counters the E-half kernel keeps on the device: the
 * cell updates in which the Newton solve for |E| ran (FDTD_PLRCNonlinCore::
 * plrcStepD, src/fdtd_plrc.cpp:406-419, skips it where c = 0; the solve of
 * FDTD_Nonlinear::stepD, src/fdtd_nl.cpp:86-92, is skipped here where D = 0)
 * and the Newton iterations they took, summed.  Resets both counters; synchronises the context's stream.
 * Zero for the linear solvers.  No counterpart in MPulse (a diagnostic that
 * shows how much of a run's work was the nonlinear solve). */
int mp_kerr_counts(mp_ctx *ctx, long long *solves, long long *iterations);

/* Field initialisers (FieldSimulation's "pulse_init", "gauss_init",
 * "wave_init", src/fieldsim.cpp:157-168), evaluated on the device in FP64
 * over the stored cells: the interior x / y columns of every z plane.  MPulse
 * also writes the x / y ghost cells; here they are the periodic images. */
typedef enum mp_init_kind {
  MP_INIT_PULSE = 1,        /* GaussPulseInit::init, src/pulseinit.cpp:7-74:
                               keys k (= k[2]), r0, z0, zc, C, Bx, By, bound */
  MP_INIT_PLANE_GAUSS = 2,  /* PlaneGaussPulseInit::init, src/gaussinit.cpp:7-82:
                               keys kx, ky, kz (whole numbers), Bx, By, Bz */
  MP_INIT_WAVE = 3          /* PlaneWaveInit::init, src/waveinit.cpp:9-60 (adds to
                               the fields): kx, ky, kz (whole numbers), Bx, By, Bz, eps */
} mp_init_kind;

typedef struct mp_init {
  int kind;       /* mp_init_kind */
  double k[3];    /* kx ky kz */
  double B[3];    /* Bx By Bz */
  double r0, z0, zc, C, eps;
  int bound;      /* pulse_init: planes 0..bound-1 and nz+2-bound..nz+1 are left as they are */
} mp_init;

/* Fills *init with the MakeParamMap defaults of `kind` (pulseinit.cpp:77-89,
 * gaussinit.cpp:85-95, waveinit.cpp:63-74). */
void mp_init_defaults(int kind, mp_init *init);
int mp_initialize(mp_ctx *ctx, const mp_init *init);

/* FollowMax::calculate (src/followmax.cpp:73-113) on the device state: from
 * the integer position *ipos along axis dim (0 x, 1 y, 2 z) of the line
 * through MPulse cell pos[3], climb to a local maximum of the field (periodic
 * wrap inside 1..n), return it in *ipos and the vertex of the parabola through
 * it and its two neighbours in *position.  field: "Ex".."Bz". */
int mp_follow_max(mp_ctx *ctx, const char *field, int dim, const int pos[3], int *ipos, double *position);

/* HDF5 field dumps: the output of MPulse's "fielddiag" (FieldDiag,
 * src/fielddiag.cpp:17-24 and src/diagnostic.t:1-30) through HDFostream
 * (src/hdfstream.cpp:189-212, src/hdfstream.t:87-187), written from the device
 * state by this library's own HDF5 encoder (HDF5 is not a dependency): the
 * version 0 superblock, the root group as a symbol table, one contiguous
 * dataset of IEEE doubles per field.
 *
 * mp_diag_file_name: DiagnosticInterface::parsedFileName
 * (src/diagnostic.cpp:52-70): pattern with its first "#p" replaced by proc_id
 * and its first "#t" by time, into out (n bytes).
 *
 * mp_hdf5_create: creates (truncates) the file mp_diag_file_name names.
 * mp_hdf5_write_field: adds the field `name` of ctx (any name mp_download
 * accepts that has the full-grid plane layout) as the next dataset, named as
 * HDFstream::getNextBlockName names them after HDFostream::open
 * (src/hdfstream.cpp:70-81, :189-212): "data0", "data1", "data2", ...; the
 * dataset is MPulse's full grid with its ghost
 * cells (x / y ghosts are the periodic images), dims {nz+2, ny+2, nx+2}: the
 * element of MPulse cell (i, j, k) is dataset[k][j][i], as the reversed dims
 * of src/hdfstream.t:110 make it.  Synchronises ctx's stream.  At most 256
 * datasets per file.  "fielddiag" with append = "y" keeps one file and adds a
 * dataset per output step; with "n" it creates a file per output step.
 * mp_hdf5_close: writes the file's metadata and closes it (a file that is
 * not closed is not a valid HDF5 file). */
typedef struct mp_hdf5 mp_hdf5;
int mp_diag_file_name(const char *pattern, int proc_id, long long time, char *out, size_t n);
int mp_hdf5_create(const char *pattern, int proc_id, long long time, mp_hdf5 **out);
int mp_hdf5_write_field(mp_hdf5 *file, mp_ctx *ctx, const char *name);
/* Adds a host array of doubles with dims {dims[0], dims[1], dims[2]}, C
 * order (dims[2] fastest), as the next dataset (what mp_hdf5_write_field
 * writes after assembling the grid). */
int mp_hdf5_write_grid(mp_hdf5 *file, const double *data, const size_t dims[3]);
/* FieldSliceDiag::write (src/fielddiag.cpp:56-115, "slicediag" with keys
 * field, plane, pos): the plane of field `name` through MPulse index `pos`
 * along axis `normal` (0: plane "x", 1: "y", 2: "z") over the full index
 * range, as the next dataset of rank 2 with the dims reversed: for normal x
 * the element of (j, k) is dataset[k][j], for y (i, k) -> [k][i], for z
 * (i, j) -> [j][i].  Nothing is written when pos is not strictly inside the
 * range (0 < pos < n + 1); MPulse's stream is then inactive and does not even
 * create the file, so a caller following slicediag skips mp_hdf5_create for
 * such a plane.  Synchronises ctx's stream. */
int mp_hdf5_write_slice(mp_hdf5 *file, mp_ctx *ctx, const char *name, int normal, int pos);
int mp_hdf5_close(mp_hdf5 *file);

/* Checkpoint / restart of the whole device state: the six fields, the PLRC
 * accumulators, the CPML psi of every face and the time (the injector state
 * is a function of the time).  The buffer is opaque, in the device precision,
 * with a header that mp_load_state checks against the context (grid,
 * precision, solver, boundary, CPML, medium planes).  MPulse itself has no
 * restart (Globals::IsRestart is never read, src/globals.h:45,90-92). */
int mp_state_size(mp_ctx *ctx, size_t *bytes);
int mp_save_state(mp_ctx *ctx, void *host, size_t bytes);
int mp_load_state(mp_ctx *ctx, const void *host, size_t bytes);

/* Runs adj->steps steps like mp_step and returns the objective J of adj over
 * them in *J (FP64 accumulation).  No counterpart in MPulse. */
int mp_objective(mp_ctx *ctx, const mp_adjoint_config *adj, double *J);

/* Like mp_objective, then the gradient of J with respect to the design
 * parameters by the discrete adjoint of the steps run: the transposed curls,
 * the reverse CPML and PLRC recursions and the linearised Kerr solve, run
 * backwards over the steps, with the forward recomputed segment by segment
 * from checkpoints (mp_adjoint_config).  grad_eps, grad_deps_scale and
 * grad_chi_scale receive dJ/d DesignEps, dJ/d DesignDepsScale and
 * dJ/d DesignChiScale per design cell (host arrays of the design box's size,
 * x fastest; NULL skips one).  The state ends as after mp_objective.  Needs a
 * PLRC solver, the xy-periodic boundary, the global-load staging and a
 * non-empty design box; the sources must not depend on the design (they do
 * not).  No counterpart in MPulse. */
int mp_adjoint(mp_ctx *ctx, const mp_adjoint_config *adj, double *J, double *grad_eps,
               double *grad_deps_scale, double *grad_chi_scale);

/* mp_adjoint in two calls, as an autograd tape: mp_objective_record runs the
 * forward part of mp_adjoint for adj (the steps, J in *J, and the checkpoints
 * of mp_adjoint's schedule, with the E history of the last segment) and keeps
 * them in the context: the device memory mp_adjoint would use, beside the
 * state.  mp_adjoint_reverse then runs the rest (the reverse pass, recomputing
 * the other segments from their checkpoints) and releases the record; J (may
 * be NULL) and the gradients are those mp_adjoint gives for the same run, to
 * the last bit, and the state ends as after mp_objective_record.  A record is
 * released by mp_release_record, by the next mp_objective_record, and by
 * every call that steps the context or writes its state, time, design maps,
 * stream or host checkpoint buffers (mp_step, mp_step_async, mp_kernel_times,
 * mp_upload, mp_set_time, mp_load_state, mp_initialize, mp_objective,
 * mp_adjoint, mp_set_stream, mp_set_host_checkpoint_budget, mp_destroy);
 * mp_adjoint_reverse without a record returns MP_ERR_INVALID.  Writes through
 * mp_device_field pointers are not seen: the reverse pass reads only the
 * record and the design maps.  No counterpart in MPulse. */
int mp_objective_record(mp_ctx *ctx, const mp_adjoint_config *adj, double *J);
int mp_adjoint_reverse(mp_ctx *ctx, double *J, double *grad_eps, double *grad_deps_scale, double *grad_chi_scale);
int mp_release_record(mp_ctx *ctx);

/* Reserves pinned host memory for mp_adjoint's checkpoints: as many buffers
 * of one forward state each as fit in `bytes` (allocated and pinned now, which
 * takes seconds for tens of GB; freed by the next call or mp_destroy; 0 frees
 * them).  With a device budget (mem_budget, checkpoint_every = 0) and at least
 * two such buffers, mp_adjoint may add a second level to its schedule: the
 * first forward run copies the state at the start of every segment of L steps
 * to host memory, and each segment is then reversed, last first, on the
 * device schedule for L steps, starting from its host copy.  It does so when
 * that runs fewer forward steps, counting each host copy as the steps that
 * take as long.  The results are the same as with any other schedule.
 * MP_ERR_NO_MEMORY when the host memory cannot be pinned (nothing is kept). */
int mp_set_host_checkpoint_budget(mp_ctx *ctx, double bytes);

/* Copies the message of the last failure (or "") into buf. */
int mp_last_error(mp_ctx *ctx, char *buf, size_t n);

/* Message of the last mp_create failure (no context exists then). */
const char *mp_create_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MPULSE_B200_H */
