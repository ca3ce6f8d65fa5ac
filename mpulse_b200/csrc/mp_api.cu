// mp_api.cu - host side of the C ABI declared in include/mpulse_b200.h.
//
// It builds, once per context, everything MPulse recomputes or re-derives on
// the host: the kappa lines (CPMLBorder[OneD]::initCoefficients,
// cpml_border.cpp:58-139, :179-243), the CPML b/c coefficients
// (CPMLBorderCurrent::makeCoeff, cpml_border.cpp:287-339), the PLRC recursion
// coefficients (fdtd_plrc.t:181-216, FP64, identical every step because dt is
// fixed) and the injector constants (sources.cpp:14-56,
// shortpulseinject.cpp:56-113), and then drives the kernels of
// mp_step_kernels.cu / mp_source_kernels.cu in MPulse's per-step order.
#include "mpulse_b200.h"

#include "mp_device.h"
#include "mp_gauss.h"
#include "mp_pulse_math.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>  // header-only NVTX: ranges for Nsight timelines, no cost without a tool

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <sys/mman.h>

namespace mpb {
template <typename T> cudaError_t launch_e_half(const EParams<T> &, int, int, cudaStream_t);
template <typename T> cudaError_t launch_b_half(const BParams<T> &, cudaStream_t);
template <typename T>
cudaError_t launch_source_batch(const SourceEvalParams &, const SourceEvalParams &, long long, int, T *, cudaStream_t);
cudaError_t launch_convert_in(const double *src, void *dst, int fp32, long long n, int stride, int offset,
                              cudaStream_t st);
cudaError_t launch_convert_out(const void *src, double *dst, int fp32, long long n, int stride, int offset,
                               cudaStream_t st);
cudaError_t launch_field_energy(const void *const fields[6], int elem_bytes, int nx, int ny, int nz, double dV,
                                double *partial, double *out_dev, cudaStream_t st);
template <typename T>
cudaError_t launch_e_half_tma(const EParams<T> &, const ETmaMaps &, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_b_half_tma(const BParams<T> &, const BTmaMaps &, cudaStream_t);
template <typename T>
cudaError_t launch_step_fused(const EParams<T> &, const BParams<T> &, int, int, int, cudaStream_t);
void tma_boxes(int esz, int e_box[7][2], int b_box[6][2]);
#ifndef MPB_ADJ_E_BPSM
#define MPB_ADJ_E_BPSM 8
#endif
#ifndef MPB_ADJ_B_BPSM
#define MPB_ADJ_B_BPSM 8
#endif
template <typename T> cudaError_t launch_adj_e(const AdjParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_adj_b(const AdjParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_adj_init(const AdjParams<T> &, cudaStream_t);
template <typename T>
cudaError_t launch_objective_term(const T *const E[3], const T *const B[3], int nx, int ny, long long plane, int kind,
                                  const int box0[6], double f, double *out, cudaStream_t st);
cudaError_t launch_sum_terms(const double *terms, long long n, double *out, cudaStream_t st);
}  // namespace mpb

using namespace mpb;

namespace {

constexpr int kFaceOrderAll[6] = {FACE_NORTH, FACE_SOUTH, FACE_EAST, FACE_WEST, FACE_UP, FACE_DOWN};
const int kFaceOrderZ[2] = {FACE_UP, FACE_DOWN};
thread_local char g_create_err[512];

constexpr int face_dim(int f) {
  return (f == FACE_EAST || f == FACE_WEST) ? 0 : (f == FACE_NORTH || f == FACE_SOUTH) ? 1 : 2;
}
// slot q of the kernels' face arrays holds kFaceOrderAll[q], whose axis the
// kernels take as y, y, x, x, z, z
static_assert(face_dim(kFaceOrderAll[0]) == 1 && face_dim(kFaceOrderAll[1]) == 1 &&
                  face_dim(kFaceOrderAll[2]) == 0 && face_dim(kFaceOrderAll[3]) == 0 &&
                  face_dim(kFaceOrderAll[4]) == 2 && face_dim(kFaceOrderAll[5]) == 2,
              "face slots");
bool face_low(int f) { return f == FACE_WEST || f == FACE_SOUTH || f == FACE_DOWN; }

struct LayerHost {
  int active = 0, dim = 0, lo = 0, hi = -1, zlo = 0, ex = 0, ey = 0;
  size_t n = 0;
  void *psi0 = nullptr, *psi1 = nullptr;
  size_t b_off = 0, c_off = 0;  // offsets (elements) into the line buffer
};

}  // namespace

struct AdjRecord;

struct mp_ctx {
  mp_config cfg;
  int fp32 = 0;
  int esz = 8;
  int mode = MODE_PLRC_LIN;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  long long plane = 0;
  size_t fcount = 0;
  void *F[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int np = 0;
  int slot_of_pole[3] = {-1, -1, -1};
  int mz0 = 1, mz1 = 0;
  size_t psi_cells = 0;
  void *psi[3][3] = {{nullptr}};
  void *lines = nullptr;
  LayerHost cpE[6], cpH[6];
  int nsrc = 0;
  int src_mult = 0;
  SourceEvalParams sq[MP_MAX_SOURCES][2];
  int src_plane[MP_MAX_SOURCES][2];
  void *src_buf = nullptr;   // injection planes of up to src_batch steps
  int src_batch = 1;
  // Source batches computed ahead (every injector but gauss_inject): buffer b
  // (src_buf, src_buf2) holds the planes of steps [pre_t0[b], pre_t0[b] +
  // pre_k[b]); while one is stepped, the next batch is computed into the other
  // on src_stream, so the FP64 source arithmetic overlaps the step kernels.
  void *src_buf2 = nullptr;
  cudaStream_t src_stream = nullptr;
  cudaEvent_t src_done[2] = {nullptr, nullptr};  // the side stream's write of buffer b is done
  cudaEvent_t src_free[2] = {nullptr, nullptr};  // the steps reading buffer b are done
  long long pre_t0[2] = {0, 0};
  int pre_k[2] = {0, 0};
  bool pre_pending[2] = {false, false};  // a side-stream write of buffer b may be in flight
  GaussBeam *gauss = nullptr;  // gauss_inject state when the last injector is one
  double *d_wcoef = nullptr;
  void *plasma[4] = {nullptr, nullptr, nullptr, nullptr};  // PlasmaDensity, PlasmaJx, PlasmaJy, PlasmaJz
  int *d_status = nullptr;
  int *h_status = nullptr;
  unsigned long long *d_kerr = nullptr;  // Kerr solves and Newton iterations since the last mp_kerr_counts
  unsigned long long *h_kerr = nullptr;
  double *staging = nullptr;
  double *d_diag = nullptr;   // diagnostics scratch: per-plane partials, then the result
  double *h_diag = nullptr;   // pinned results (two doubles)
  size_t staging_n = 0;
  long long time = 0;
  long long launches = 0;
  int pending_status = MP_OK;
  std::string err;
  EParams<float> epf;
  BParams<float> bpf;
  EParams<double> epd;
  BParams<double> bpd;
  bool tma = false;    // TMA-staged kernels in use
  bool fused = false;  // the fused step kernel and its border kernel in use
  std::vector<void *> host_ckpt;  // pinned host buffers of one state each (mp_set_host_checkpoint_budget)
  AdjRecord *rec = nullptr;       // the run mp_objective_record kept for mp_adjoint_reverse
  // CUDA graphs of K steps whose injection planes start at `planes` (small
  // grids, where the launch gaps between the short half-step kernels cost)
  struct StepGraph {
    const void *planes;
    int K;
    cudaGraphExec_t exec;
  };
  std::vector<StepGraph> graphs;
  bool use_graphs = false;
  ETmaMaps etma;
  BTmaMaps btma;
  // design region (mp_config.design_box): FP64 maps eps, Delta-eps factor, chi factor
  bool design = false;
  size_t dcells = 0;
  double *d_design[3] = {nullptr, nullptr, nullptr};
  DesignParams dp;
  // FP64 PLRC constants of the active poles: [D, dxi0, Crec][slot][re, im]
  double coef[3][3][2] = {{{0}}};
  double sumChi0 = 0, sumXi0 = 0;
  std::vector<void *> allocs;
};

namespace {

// An NVTX range over a scope (the host side of one phase).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int set_err(mp_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  else snprintf(g_create_err, sizeof g_create_err, "%s", buf);
  return code;
}

int cuda_err(mp_ctx *c, cudaError_t e, const char *what) {
  return set_err(c, e == cudaErrorMemoryAllocation ? MP_ERR_NO_MEMORY : MP_ERR_CUDA, "%s: %s", what,
                 cudaGetErrorString(e));
}

cudaError_t dalloc(mp_ctx *c, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return e;
  c->allocs.push_back(*p);
  return cudaMemsetAsync(*p, 0, bytes, c->stream);
}

// Kappa lines exactly as CPMLBorder::initCoefficients (cpml_border.cpp:100-139)
// and CPMLBorderOneD::initCoefficients (cpml_border.cpp:208-243).
void kappa_lines(const mp_config &c, std::vector<double> kapE[3], std::vector<double> kapH[3]) {
  const int n[3] = {c.nx, c.ny, c.nz};
  const int d = c.cpml_d;
  for (int a = 0; a < 3; ++a) {
    kapE[a].assign(n[a] + 2, 1.0);
    kapH[a].assign(n[a] + 2, 1.0);
  }
  auto grade = [&](double x) { return 1 + (c.cpml_kappa_max - 1) * x * x * x; };
  if (c.cpml == MP_CPML_ALL) {
    for (int a = 0; a < 3; ++a) {
      const int low = 0, high = n[a] + 1;
      for (int i = 0; i <= d; ++i) kapE[a][low + i] = grade(1 - double(i) / double(d));
      for (int i = 0; i < d; ++i) kapH[a][low + i] = grade(1 - (double(i) + 0.5) / double(d));
      for (int i = 0; i <= d; ++i) kapH[a][high - i] = grade(1 - double(i) / double(d));
      for (int i = 0; i < d; ++i) kapE[a][high - i] = grade(1 - (double(i) + 0.5) / double(d));
    }
  } else if (c.cpml == MP_CPML_Z) {
    const int low = 0, high = n[2] + 1;
    for (int i = 0; i < d; ++i) kapE[2][low + i + 1] = grade(1 - double(i) / double(d));
    for (int i = 0; i < d; ++i) kapH[2][low + i] = grade(1 - (double(i) + 0.5) / double(d));
    for (int i = 0; i < d; ++i) kapE[2][high - i - 1] = grade(1 - double(i) / double(d));
    for (int i = 0; i < d; ++i) kapH[2][high - i - 1] = grade(1 - double(i + 0.5) / double(d));
  }
}

int validate(const mp_config *c) {
  if (!c) return set_err(nullptr, MP_ERR_INVALID, "config is NULL");
  if (c->abi_version != MP_ABI_VERSION)
    return set_err(nullptr, MP_ERR_INVALID, "abi_version %d, library speaks %d", c->abi_version, MP_ABI_VERSION);
  if (c->nx < 2 || c->ny < 2 || c->nz < 2) return set_err(nullptr, MP_ERR_INVALID, "grid must be at least 2 cells per axis");
  if (!(c->dx > 0 && c->dy > 0 && c->dz > 0 && c->dt > 0))
    return set_err(nullptr, MP_ERR_INVALID, "grid spacings and dt must be positive");
  if (c->precision != MP_FP64 && c->precision != MP_FP32) return set_err(nullptr, MP_ERR_INVALID, "unknown precision");
  if (c->solver < MP_SOLVER_PLAIN || c->solver > MP_SOLVER_PLRC_NONLIN)
    return set_err(nullptr, MP_ERR_INVALID, "unknown solver %d", c->solver);
  if (c->boundary != MP_BOUNDARY_PERIODIC && c->boundary != MP_BOUNDARY_XY_PERIODIC)
    return set_err(nullptr, MP_ERR_INVALID, "unknown boundary %d", c->boundary);
  const bool plrc = c->solver == MP_SOLVER_PLRC_LIN || c->solver == MP_SOLVER_PLRC_NONLIN;
  if (!plrc && (c->cpml != MP_CPML_NONE || c->n_sources > 0))
    return set_err(nullptr, MP_ERR_INVALID,
                   "additional currents cannot be used with this field solver (fieldsolver.h:198-216)");
  if (plrc) {
    for (int n = 0; n < MP_MAX_POLES; ++n) {
      if (c->poles[n].om2 == 0)
        return set_err(nullptr, MP_ERR_INVALID, "FDTD_PLRCSolver: Omega should not be zero! (pole %d)", n + 1);
      if (!(c->poles[n].om2 > c->poles[n].delta * c->poles[n].delta))
        return set_err(nullptr, MP_ERR_INVALID, "pole %d needs om2 > delta^2", n + 1);
    }
    if (!(c->eps_bg != 0) || !std::isfinite(c->eps_bg)) return set_err(nullptr, MP_ERR_INVALID, "eps_bg must be non-zero");
  }
  if (c->cpml != MP_CPML_NONE) {
    if (c->cpml != MP_CPML_ALL && c->cpml != MP_CPML_Z) return set_err(nullptr, MP_ERR_INVALID, "unknown cpml kind");
    if (c->cpml_d < 1) return set_err(nullptr, MP_ERR_INVALID, "cpml_d must be >= 1");
    const int lim = c->cpml == MP_CPML_Z ? c->nz : std::min(c->nx, std::min(c->ny, c->nz));
    if (c->cpml_d > lim) return set_err(nullptr, MP_ERR_INVALID, "CPML thicker (%d) than the domain (%d)", c->cpml_d, lim);
    if (c->cpml_sigma_max == 0 && c->cpml_a_max == 0)
      return set_err(nullptr, MP_ERR_INVALID, "CPML with sigmaMax = aMax = 0 has undefined c = 0/0 (cpml_border.cpp:333)");
  }
  if (c->n_sources < 0 || c->n_sources > MP_MAX_SOURCES) return set_err(nullptr, MP_ERR_INVALID, "n_sources out of range");
  for (int s = 0; s < c->n_sources; ++s) {
    const mp_source &q = c->sources[s];
    if (q.kind < MP_SOURCE_PLANE_WAVE || q.kind > MP_SOURCE_GAUSS_BEAM)
      return set_err(nullptr, MP_ERR_INVALID, "source %d: unknown kind %d", s, q.kind);
    if (q.kind == MP_SOURCE_GAUSS_BEAM && (q.t_size < 1 || q.t_size > (1 << 22)))
      return set_err(nullptr, MP_ERR_INVALID, "source %d: t_size %d outside 1..2^22", s, q.t_size);
    if (q.distance < 1 || q.distance > c->nz)
      return set_err(nullptr, MP_ERR_INVALID, "source %d: distance %d outside 1..nz", s, q.distance);
    if (!(q.eps > 0)) return set_err(nullptr, MP_ERR_INVALID, "source %d: eps must be positive", s);
  }
  if (c->newton_max_iter < 1) return set_err(nullptr, MP_ERR_INVALID, "newton_max_iter must be >= 1");
  if (c->staging != MP_STAGING_AUTO && c->staging != MP_STAGING_GLOBAL && c->staging != MP_STAGING_TMA &&
      c->staging != MP_STAGING_FUSED)
    return set_err(nullptr, MP_ERR_INVALID, "unknown staging %d", c->staging);
  const int *db = c->design_box;
  if (db[0] <= db[1]) {
    if (!plrc) return set_err(nullptr, MP_ERR_INVALID, "a design region needs a PLRC solver");
    if (db[0] < 1 || db[1] > c->nx || db[2] < 1 || db[2] > db[3] || db[3] > c->ny || db[4] < 1 || db[4] > db[5] ||
        db[5] > c->nz)
      return set_err(nullptr, MP_ERR_INVALID, "design box outside the interior");
    if (db[4] < c->medium_z0 || db[5] > c->medium_z1)
      return set_err(nullptr, MP_ERR_INVALID, "design box outside the medium planes %d..%d", c->medium_z0,
                     c->medium_z1);
    if (c->staging == MP_STAGING_TMA || c->staging == MP_STAGING_FUSED)
      return set_err(nullptr, MP_ERR_UNSUPPORTED, "design regions use the global-load kernels (staging GLOBAL/AUTO)");
  }
  if (c->plasma || c->plasma_current) {
    if (!plrc) return set_err(nullptr, MP_ERR_INVALID, "the plasma plug-ins belong to the PLRC solvers (fdtd_plrc.t:431-436)");
    if (c->plasma && (c->plasma_k < 1 || c->plasma_k > 64))
      return set_err(nullptr, MP_ERR_INVALID, "plasma K %d outside 1..64", c->plasma_k);
    if (c->staging == MP_STAGING_TMA || c->staging == MP_STAGING_FUSED)
      return set_err(nullptr, MP_ERR_UNSUPPORTED, "the plasma plug-ins use the global-load kernels (staging GLOBAL/AUTO)");
    if (db[0] <= db[1]) return set_err(nullptr, MP_ERR_UNSUPPORTED, "the plasma plug-ins and a design region together");
  }
  if (c->staging == MP_STAGING_TMA && (c->nx % kTmaTileX != 0 || c->ny % kTmaTileY != 0))
    return set_err(nullptr, MP_ERR_UNSUPPORTED, "TMA staging needs nx a multiple of %d and ny of %d", kTmaTileX,
                   kTmaTileY);
  return MP_OK;
}

template <typename T>
void fill_face(CpmlFace<T> &F, const LayerHost &L, const T *lines) {
  F.active = L.active;
  F.dim = L.dim;
  F.lo = L.lo;
  F.hi = L.hi;
  F.zlo = L.zlo;
  F.ex = L.ex;
  F.ey = L.ey;
  F.psi0 = static_cast<T *>(L.psi0);
  F.psi1 = static_cast<T *>(L.psi1);
  F.n = int(L.n);
  F.b = lines + L.b_off;
  F.c = lines + L.c_off;
}

template <typename T>
void build_params(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, const std::vector<size_t> &ikE_off,
                  const std::vector<size_t> &ikH_off, size_t bzy_off, const double coef[3][3][2], double numer,
                  double denom) {
  const mp_config &g = c->cfg;
  const T *lines = static_cast<const T *>(c->lines);
  ep = EParams<T>();
  bp = BParams<T>();
  ep.nx = bp.nx = g.nx;
  ep.ny = bp.ny = g.ny;
  ep.nz = bp.nz = g.nz;
  ep.plane = bp.plane = c->plane;
  for (int a = 0; a < 3; ++a) {
    ep.E[a] = static_cast<T *>(c->F[a]);
    ep.B[a] = static_cast<const T *>(c->F[3 + a]);
    bp.E[a] = static_cast<const T *>(c->F[a]);
    bp.B[a] = static_cast<T *>(c->F[3 + a]);
    ep.ik[a] = lines + ikE_off[a];
    bp.ik[a] = lines + ikH_off[a];
  }
  bp.ik_bz_y = lines + bzy_off;
  const bool zper = g.boundary == MP_BOUNDARY_PERIODIC;
  ep.zperiodic = bp.zperiodic = zper ? 1 : 0;
  ep.k_first = 1;
  ep.k_last = (c->mode == MODE_PLAIN || c->mode == MODE_NL) && !zper ? g.nz + 1 : g.nz;
  bp.k_first = zper ? 1 : 0;
  bp.k_last = g.nz;
  ep.dt = bp.dt = T(g.dt);
  ep.dt_lo = bp.dt_lo = T(g.dt - double(T(g.dt)));
  ep.mz0 = c->mz0;
  ep.mz1 = c->mz1;
  for (int s = 0; s < c->np; ++s)
    for (int a = 0; a < 3; ++a) ep.psi[s][a] = static_cast<T *>(c->psi[s][a]);
  for (int s = 0; s < 3; ++s)
    for (int q = 0; q < 2; ++q) {
      ep.pD[s][q] = T(coef[0][s][q]);
      ep.pxi[s][q] = T(coef[1][s][q]);
      ep.pC[s][q] = T(coef[2][s][q]);
    }
  if (c->plasma[0]) {
    // PlasmaDensity (plasmadensity.cpp:31-35) and PlasmaCurrent
    // (plasmacurrent.cpp:57-59) constants
    ep.rho = static_cast<T *>(c->plasma[0]);
    for (int a = 0; a < 3; ++a) ep.pj[a] = static_cast<T *>(c->plasma[1 + a]);
    ep.pl_density = g.plasma ? 1 : 0;
    ep.pl_current = g.plasma_current ? 1 : 0;
    ep.pl_km = g.plasma_k - 1;
    ep.pl_n = T(0.5 * g.dt * g.plasma_nu);
    ep.pl_m = T(g.dt * g.plasma_mpa);
    ep.pl_w = T(g.plasma_mpa * g.plasma_wion);
    ep.pl_gdtn = T(1 - 0.5 * g.plasma_gamma * g.dt);
    ep.pl_gdtd = T(1 + 0.5 * g.plasma_gamma * g.dt);
    ep.pl_emdt = T(g.plasma_em * g.dt);
    ep.pl_rho_bg = T(g.plasma_rho_bg);
  }
  ep.denom_t = T(denom);
  ep.denom_d = denom;
  ep.chi_raw = g.chi;
  ep.numer = T(numer);
  ep.inv_denom = T(1.0 / denom);
  ep.numer_lo = T(numer - double(ep.numer));
  ep.inv_denom_lo = T(1.0 / denom - double(ep.inv_denom));
  ep.eps_bg = T(g.eps_bg);
  ep.inv_eps_bg = T(1.0 / g.eps_bg);
  ep.chi_over_denom = g.chi / denom;
  ep.chi = T(g.chi);
  ep.eps_d = g.eps;
  ep.chi_d = g.chi;
  ep.newton_tol = g.newton_tol;
  ep.newton_max = g.newton_max_iter;
  for (int f = 0; f < 6; ++f) {
    fill_face(ep.cpml[f], c->cpE[f], lines);
    fill_face(bp.cpml[f], c->cpH[f], lines);
  }
  ep.design.x0 = 1;  // none; set by create_impl when the config has a design box
  ep.design.x1 = 0;
  ep.n_src = bp.n_src = c->nsrc;
  ep.src_mult = bp.src_mult = c->src_mult;
  const size_t pl = size_t(c->plane);
  for (int s = 0; s < c->nsrc; ++s) {
    T *base = static_cast<T *>(c->src_buf) + size_t(s) * 4 * pl;
    ep.src[s].plane = c->src_plane[s][0];
    ep.src[s].v0 = base;
    ep.src[s].v1 = base + pl;
    bp.src[s].plane = c->src_plane[s][1];
    bp.src[s].v0 = base + 2 * pl;
    bp.src[s].v1 = base + 3 * pl;
  }
  ep.status = c->d_status;
  ep.kerr_count = c->d_kerr;
  bp.status = c->d_status;
  ep.n_field = bp.n_field = (long long)c->fcount;
  ep.n_psi = (long long)c->psi_cells;
  // planes per block of the scalar B half (and a default the global-load E
  // half replaces with its own, launch_e_np): enough blocks to fill 148 SMs
  // several times over
  const long long blocks_xy = (long long)((g.nx + 31) / 32) * ((g.ny + 7) / 8);
  const long long target = 148LL * 8;
  const int ne = ep.k_last - ep.k_first + 1, nb = bp.k_last - bp.k_first + 1;
  const long long chunks = std::max(1LL, (target + blocks_xy - 1) / blocks_xy);
  ep.kchunk = int(std::max(1LL, (ne + chunks - 1) / chunks));
  bp.kchunk = int(std::max(1LL, (nb + chunks - 1) / chunks));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 3-D map over an array of `dz` planes of dy rows of dx elements, box bx x by x 1.
bool encode_map(CUtensorMap *m, void *base, int esz, long long dx, long long dy, long long dz, int bx, int by) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || !base) return false;
  const cuuint64_t dims[3] = {cuuint64_t(dx), cuuint64_t(dy), cuuint64_t(dz)};
  const cuuint64_t strides[2] = {cuuint64_t(dx * esz), cuuint64_t(dx * dy * esz)};
  const cuuint32_t box[3] = {cuuint32_t(bx), cuuint32_t(by), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(m, esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides,
            box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of the TMA-staged kernels; false (global-load kernels are used)
// if the driver cannot encode them.
bool setup_tma(mp_ctx *c) {
  const mp_config &g = c->cfg;
  int eb[7][2], bb[6][2];
  tma_boxes(c->esz, eb, bb);
  const long long nx = g.nx, ny = g.ny, nzp = g.nz + 2;
  bool ok = true;
  ok = ok && encode_map(&c->etma.bx, c->F[3], c->esz, nx, ny, nzp, eb[0][0], eb[0][1]);
  ok = ok && encode_map(&c->etma.by, c->F[4], c->esz, nx, ny, nzp, eb[1][0], eb[1][1]);
  ok = ok && encode_map(&c->etma.bz, c->F[5], c->esz, nx, ny, nzp, eb[2][0], eb[2][1]);
  ok = ok && encode_map(&c->etma.ex, c->F[0], c->esz, nx, ny, nzp, eb[3][0], eb[3][1]);
  ok = ok && encode_map(&c->etma.ey, c->F[1], c->esz, nx, ny, nzp, eb[4][0], eb[4][1]);
  ok = ok && encode_map(&c->etma.ez, c->F[2], c->esz, nx, ny, nzp, eb[5][0], eb[5][1]);
  for (int s = 0; s < c->np && ok; ++s)
    for (int a = 0; a < 3 && ok; ++a)
      ok = encode_map(&c->etma.psi[s][a], c->psi[s][a], c->esz, 2 * nx, ny, c->mz1 - c->mz0 + 1, eb[6][0], eb[6][1]);
  ok = ok && encode_map(&c->btma.ex, c->F[0], c->esz, nx, ny, nzp, bb[0][0], bb[0][1]);
  ok = ok && encode_map(&c->btma.ey, c->F[1], c->esz, nx, ny, nzp, bb[1][0], bb[1][1]);
  ok = ok && encode_map(&c->btma.ez, c->F[2], c->esz, nx, ny, nzp, bb[2][0], bb[2][1]);
  ok = ok && encode_map(&c->btma.bx, c->F[3], c->esz, nx, ny, nzp, bb[3][0], bb[3][1]);
  ok = ok && encode_map(&c->btma.by, c->F[4], c->esz, nx, ny, nzp, bb[4][0], bb[4][1]);
  ok = ok && encode_map(&c->btma.bz, c->F[5], c->esz, nx, ny, nzp, bb[5][0], bb[5][1]);
  c->tma = ok;
  return ok;
}

int create_impl(const mp_config *cfg, mp_ctx **out) {
  int rc = validate(cfg);
  if (rc != MP_OK) return rc;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) return set_err(nullptr, MP_ERR_CUDA, "cudaSetDevice(%d): %s", cfg->device, cudaGetErrorString(e));

  mp_ctx *c = new (std::nothrow) mp_ctx();
  if (!c) return set_err(nullptr, MP_ERR_NO_MEMORY, "out of host memory");
  c->cfg = *cfg;
  const mp_config &g = c->cfg;
  c->fp32 = g.precision == MP_FP32;
  c->esz = c->fp32 ? 4 : 8;
  c->mode = g.solver == MP_SOLVER_PLAIN ? MODE_PLAIN
            : g.solver == MP_SOLVER_NL  ? MODE_NL
            : g.solver == MP_SOLVER_PLRC_LIN ? MODE_PLRC_LIN
                                             : MODE_PLRC_NONLIN;
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { rc = cuda_err(nullptr, e, "cudaStreamCreate"); delete c; return rc; }
  c->stream = c->own_stream;
  c->plane = (long long)g.nx * g.ny;
  c->fcount = size_t(g.nz + 2) * size_t(c->plane);

  auto fail = [&](int code) {
    snprintf(g_create_err, sizeof g_create_err, "%s", c->err.c_str());
    mp_destroy(c);
    return code;
  };
#define MPB_TRY(expr, what)                          \
  do {                                               \
    cudaError_t e_ = (expr);                         \
    if (e_ != cudaSuccess) return fail(cuda_err(c, e_, what)); \
  } while (0)

  for (int f = 0; f < 6; ++f) MPB_TRY(dalloc(c, &c->F[f], c->fcount * c->esz), "field allocation");
  if (g.plasma || g.plasma_current)
    for (int q = 0; q < 4; ++q) MPB_TRY(dalloc(c, &c->plasma[q], c->fcount * c->esz), "plasma allocation");

  const bool plrc = c->mode == MODE_PLRC_LIN || c->mode == MODE_PLRC_NONLIN;
  // PLRC: active poles (Delta eps != 0) and their accumulators over the medium
  // planes the E update touches.  A pole with Delta eps = 0 has dchi0 = dxi0 = 0
  // and an accumulator that stays 0 from MPulse's zero start, so it is skipped.
  double coef[3][3][2] = {{{0}}};  // [D, dxi0, Crec][slot][re, im]
  double numer = g.eps, denom = g.eps;
  if (plrc) {
    c->mz0 = std::max(g.medium_z0, 1);
    c->mz1 = std::min(g.medium_z1, g.nz);
    // FDTD_PLRCSolver::stepD coefficient block (fdtd_plrc.t:181-216)
    const std::complex<double> I(0, 1);
    std::complex<double> sumChi = 0.0, sumXi = 0.0;
    for (int n = 0; n < 3; ++n) {
      const mp_lorentz_pole &P = g.poles[n];
      const double beta = std::sqrt(P.om2 - P.delta * P.delta);
      const double gamma = P.eps * P.om2 / beta;
      const std::complex<double> phasor = P.delta - I * beta;
      const std::complex<double> Crec = std::exp(-phasor * g.dt);
      const std::complex<double> chi0 = (I * gamma * (Crec - 1.0) / phasor);
      const std::complex<double> xi0 = I * gamma * (Crec * (phasor * g.dt + 1.0) - 1.0) / (phasor * phasor * g.dt);
      const std::complex<double> dchi0 = chi0 * (1.0 - Crec), dxi0 = xi0 * (1.0 - Crec);
      sumChi += chi0;
      sumXi += xi0;
      if (P.eps != 0.0 && c->mz0 <= c->mz1) {
        const int s = c->np++;
        c->slot_of_pole[n] = s;
        const std::complex<double> D = dchi0 - dxi0;
        coef[0][s][0] = D.real(); coef[0][s][1] = D.imag();
        coef[1][s][0] = dxi0.real(); coef[1][s][1] = dxi0.imag();
        coef[2][s][0] = Crec.real(); coef[2][s][1] = Crec.imag();
      }
    }
    const double sumChi0 = sumChi.real(), sumXi0 = sumXi.real();
    c->sumChi0 = sumChi0;
    c->sumXi0 = sumXi0;
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 3; ++s)
        for (int r = 0; r < 2; ++r) c->coef[a][s][r] = coef[a][s][r];
    numer = g.eps - sumXi0 - 0.0;
    denom = (c->mode == MODE_PLRC_LIN) ? g.eps + (sumChi0 - sumXi0) + 0.0 : g.eps + sumChi0 - sumXi0 + 0.0;
    if (c->mz0 <= c->mz1) {
      c->psi_cells = size_t(c->mz1 - c->mz0 + 1) * size_t(c->plane);
      for (int s = 0; s < c->np; ++s)
        for (int a = 0; a < 3; ++a) MPB_TRY(dalloc(c, &c->psi[s][a], 2 * c->psi_cells * c->esz), "psi allocation");
    }
  }

  // Lines: ikE[3], ikH[3], bz_y, then b/c per CPML face (E 6, H 6), each the
  // full axis length n+2, all in one buffer of T.
  std::vector<double> kapE[3], kapH[3];
  kappa_lines(g, kapE, kapH);
  const int n3[3] = {g.nx, g.ny, g.nz};
  const double d3[3] = {g.dx, g.dy, g.dz};
  std::vector<double> host_lines;
  std::vector<size_t> ikE_off(3), ikH_off(3);
  for (int a = 0; a < 3; ++a) {
    ikE_off[a] = host_lines.size();
    for (int i = 0; i < n3[a] + 2; ++i) host_lines.push_back(1.0 / (kapE[a][i] * d3[a]));
  }
  for (int a = 0; a < 3; ++a) {
    ikH_off[a] = host_lines.size();
    for (int i = 0; i < n3[a] + 2; ++i) host_lines.push_back(1.0 / (kapH[a][i] * d3[a]));
  }
  const size_t bzy_off = host_lines.size();
  for (int i = 0; i < g.ny + 2; ++i)
    host_lines.push_back(plrc ? 1.0 / (kapH[1][i] * g.dy) : 1.0 / g.dx);  // fdtd_plain.cpp:115 divides by dx

  const int kb0 = g.boundary == MP_BOUNDARY_PERIODIC ? 1 : 0;
  if (g.cpml != MP_CPML_NONE) {
    const int *order = g.cpml == MP_CPML_ALL ? kFaceOrderAll : kFaceOrderZ;
    const int nface = g.cpml == MP_CPML_ALL ? 6 : 2;
    const int d = g.cpml_d;
    for (int q = 0; q < nface; ++q) {
      const int f = order[q];
      const int dim = face_dim(f);
      const int n = n3[dim];
      // the kernels find a face's axis from its slot: the order of kFaceOrderAll
      const int slot = g.cpml == MP_CPML_ALL ? q : q + 4;
      for (int isH = 0; isH < 2; ++isH) {
        LayerHost &L = isH ? c->cpH[slot] : c->cpE[slot];
        // the reference layer along dim (getBorderExtent with the distances of
        // cpml_border.cpp:353 and :441-450)
        const int distance = (isH && face_low(f)) ? 0 : 1;
        int rlo, rhi;
        if (face_low(f)) { rlo = distance; rhi = d - 1 + distance; }
        else { rlo = n + 1 - d + 1 - distance; rhi = n + 1 - distance; }
        // b and c (makeCoeff), positions counted from the outer edge
        std::vector<double> bl(n + 2, 0.0), cl(n + 2, 0.0);
        const double offset = isH ? 0.5 : 0.0;
        for (int k = 0; k < d; ++k) {
          const double x = 1 - (double(k) - offset) / double(d);
          const double x3 = x * x * x;
          const int pos = face_low(f) ? (rlo + k) : (rhi - k);
          const double sigma = x3 * g.cpml_sigma_max;
          const double kappa = 1 + (g.cpml_kappa_max - 1) * x3;
          const double a = g.cpml_a_max * (1 - x);
          const double b = std::exp(-(sigma / kappa + a) * g.dt / 1.0);
          const double cc = sigma * (b - 1) / (kappa * (sigma + kappa * a));
          bl[pos] = b;
          cl[pos] = cc / d3[dim];
        }
        // restrict to the cells the kernels update
        int ulo, uhi;
        if (dim == 2) { ulo = isH ? kb0 : 1; uhi = g.nz; }
        else { ulo = 1; uhi = n; }
        L.dim = dim;
        L.lo = std::max(rlo, ulo);
        L.hi = std::min(rhi, uhi);
        L.active = L.lo <= L.hi;
        if (!L.active) continue;
        L.zlo = isH ? kb0 : 1;
        const int zdepth = g.nz - L.zlo + 1;
        L.ex = dim == 0 ? L.hi - L.lo + 1 : g.nx;
        L.ey = dim == 1 ? L.hi - L.lo + 1 : g.ny;
        const int ez = dim == 2 ? L.hi - L.lo + 1 : zdepth;
        L.n = size_t(L.ex) * L.ey * ez;
        if (L.n >= (size_t(1) << 31))
          return fail(set_err(c, MP_ERR_UNSUPPORTED, "CPML layer of %zu cells exceeds 2^31 (32-bit layer index)", L.n));
        MPB_TRY(dalloc(c, &L.psi0, L.n * c->esz), "CPML allocation");
        MPB_TRY(dalloc(c, &L.psi1, L.n * c->esz), "CPML allocation");
        L.b_off = host_lines.size();
        host_lines.insert(host_lines.end(), bl.begin(), bl.end());
        L.c_off = host_lines.size();
        host_lines.insert(host_lines.end(), cl.begin(), cl.end());
      }
    }
  }

  // Incident sources.
  std::vector<double> wcoef(kFaddeevaTerms);
  double wL = 0;
  faddeeva_coefficients(wcoef.data(), &wL);
  MPB_TRY(dalloc(c, reinterpret_cast<void **>(&c->d_wcoef), wcoef.size() * sizeof(double)), "source allocation");
  MPB_TRY(cudaMemcpyAsync(c->d_wcoef, wcoef.data(), wcoef.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream),
          "cudaMemcpy");
  // All built injector kinds use the `down` face, and every injector on a face
  // shares the border-layer grids "IncidentEJx".. / "IncidentHJx".. of the first
  // one (Storage::addBorderLayer returns the grid already registered under the
  // name, storage.cpp:129-141).  Each injector's stepScheme overwrites the shared
  // grid over the first injector's extent, and sumCurrents adds the grid once
  // per injector: the step sees the LAST injector's field on the FIRST one's
  // planes, n_sources times.  One plane pair is evaluated and added src_mult
  // times.
  c->nsrc = g.n_sources > 0 ? 1 : 0;
  c->src_mult = g.n_sources;
  for (int s = 0; s < c->nsrc; ++s) {
    const mp_source &q = g.sources[g.n_sources - 1];
    const mp_source &first = g.sources[0];
    for (int isH = 0; isH < 2; ++isH) {
      SourceEvalParams &p = c->sq[s][isH];
      p = SourceEvalParams();
      p.kind = q.kind;
      p.nx = g.nx;
      p.ny = g.ny;
      p.isH = isH;
      p.l = first.distance - 1;
      p.dx = g.dx; p.dy = g.dy; p.dz = g.dz; p.dt = g.dt;
      p.DX = g.dz;
      if (q.kind == MP_SOURCE_PLANE_WAVE || q.kind == MP_SOURCE_PLANE_GAUSS) {
        // PlaneWaveSource::makeECurrent (sources.cpp:14-34)
        const double *k = q.k, *H = q.H;
        double E[3] = {k[1] * H[2] - k[2] * H[1], k[2] * H[0] - k[0] * H[2], k[0] * H[1] - k[1] * H[0]};
        const double bmag = std::sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
        const double factor = -bmag / std::sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
        for (int a = 0; a < 3; ++a) {
          p.k[a] = k[a];
          p.amp3[a] = isH ? E[a] * (factor / std::sqrt(q.eps)) : H[a];
          p.bg[a] = isH ? q.E_bg[a] : q.H_bg[a];
        }
        p.om = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]) / std::sqrt(q.eps);
        p.ramp = q.ramp;
        p.width = q.width;
        p.offset = q.offset;
      } else if (q.kind == MP_SOURCE_GAUSS_BEAM) {
        // getHField scales Bx by sqrt(eps) amp, getEField Ex / Ey by amp
        // (gaussinject.cpp:204-222); the planes are set per block in step_impl
        p.g_scale = isH ? q.amp : std::sqrt(q.eps) * q.amp;
      } else {
        // ShortPulseInjectSourceFunc::setParam (shortpulseinject.cpp:56-113)
        p.centre[0] = 0.5 * double(g.nx + 1);
        p.centre[1] = 0.5 * double(g.ny + 1);
        p.centre[2] = 0.5 * double(g.nz + 1);
        p.lightspeed = std::sqrt(1 / q.eps);
        p.ZRl = 0.5 * q.om0 * q.waist * q.waist / p.lightspeed;
        p.length = q.length;
        p.om0 = q.om0;
        ShortPulse sp;
        sp.c = p.lightspeed; sp.ZRl = p.ZRl; sp.phase = 0.0; sp.T = q.length; sp.om0 = q.om0;
        sp.coef = wcoef.data(); sp.L = wL;
        short_pulse_constants(sp);
        const double Exmax = short_pulse_e(sp, 0, 0, 0, 0).re;
        p.amp = q.amp / Exmax;
        p.phase = 2 * M_PI * q.phase;
        sp.phase = p.phase;
        short_pulse_constants(sp);
        p.sp_eiphi[0] = sp.eiphi.re; p.sp_eiphi[1] = sp.eiphi.im;
        p.sp_emip[0] = sp.emip.re; p.sp_emip[1] = sp.emip.im;
        p.sp_g = sp.g;
        p.tshift = q.t_shift;
        p.zshift = q.z_shift;
        p.w_coef = c->d_wcoef;
        p.w_L = wL;
      }
    }
    c->src_plane[s][0] = first.distance;      // E current layer z = d
    c->src_plane[s][1] = first.distance - 1;  // H current layer z = d - 1 (incsource.t:91)
    if (q.kind == MP_SOURCE_GAUSS_BEAM) {
      c->gauss = new (std::nothrow) GaussBeam();
      if (!c->gauss) return fail(set_err(c, MP_ERR_NO_MEMORY, "gauss_inject state"));
      const int grc = gauss_create(*c->gauss, q, g, &c->err);
      if (grc != MP_OK) {
        delete c->gauss;
        c->gauss = nullptr;
        return fail(grc);
      }
      c->sq[s][0].g_f1 = c->gauss->bx;
      c->sq[s][1].g_f1 = c->gauss->ex;
      c->sq[s][1].g_f2 = c->gauss->ey;
    }
  }
  if (c->nsrc) {
    // plane pairs for up to 64 steps ahead, at most 256 MB
    const size_t per_step = 4 * size_t(c->plane) * c->esz;
    c->src_batch = int(std::max<size_t>(1, std::min<size_t>(64, (size_t(256) << 20) / per_step)));
    MPB_TRY(dalloc(c, &c->src_buf, size_t(c->src_batch) * per_step), "source allocation");
    if (!c->gauss) {
      MPB_TRY(dalloc(c, &c->src_buf2, size_t(c->src_batch) * per_step), "source allocation");
      MPB_TRY(cudaStreamCreateWithFlags(&c->src_stream, cudaStreamNonBlocking), "cudaStreamCreate");
      for (int b = 0; b < 2; ++b) {
        MPB_TRY(cudaEventCreateWithFlags(&c->src_done[b], cudaEventDisableTiming), "cudaEventCreate");
        MPB_TRY(cudaEventCreateWithFlags(&c->src_free[b], cudaEventDisableTiming), "cudaEventCreate");
      }
    }
  }

  // upload the lines
  MPB_TRY(dalloc(c, &c->lines, host_lines.size() * c->esz), "line allocation");
  if (c->fp32) {
    std::vector<float> hf(host_lines.begin(), host_lines.end());
    MPB_TRY(cudaMemcpyAsync(c->lines, hf.data(), hf.size() * 4, cudaMemcpyHostToDevice, c->stream), "cudaMemcpy");
    MPB_TRY(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  } else {
    MPB_TRY(cudaMemcpyAsync(c->lines, host_lines.data(), host_lines.size() * 8, cudaMemcpyHostToDevice, c->stream),
            "cudaMemcpy");
    MPB_TRY(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  }
  MPB_TRY(dalloc(c, reinterpret_cast<void **>(&c->d_status), ST_COUNT * sizeof(int)), "status allocation");
  MPB_TRY(cudaMallocHost(reinterpret_cast<void **>(&c->h_status), ST_COUNT * sizeof(int)), "pinned allocation");
  MPB_TRY(dalloc(c, reinterpret_cast<void **>(&c->d_kerr), 2 * sizeof(unsigned long long)), "counter allocation");
  MPB_TRY(cudaMallocHost(reinterpret_cast<void **>(&c->h_kerr), 2 * sizeof(unsigned long long)), "pinned allocation");
  MPB_TRY(dalloc(c, reinterpret_cast<void **>(&c->d_diag), size_t(g.nz + 3) * sizeof(double)), "diagnostics allocation");
  MPB_TRY(cudaMallocHost(reinterpret_cast<void **>(&c->h_diag), 2 * sizeof(double)), "pinned allocation");

  if (c->fp32) build_params<float>(c, c->epf, c->bpf, ikE_off, ikH_off, bzy_off, coef, numer, denom);
  else build_params<double>(c, c->epd, c->bpd, ikE_off, ikH_off, bzy_off, coef, numer, denom);

  // design region: FP64 maps with the defaults eps, 1, 1
  if (g.design_box[0] <= g.design_box[1]) {
    const int *db = g.design_box;
    DesignParams &d = c->dp;
    d.x0 = db[0] - 1; d.x1 = db[1] - 1;
    d.y0 = db[2] - 1; d.y1 = db[3] - 1;
    d.z0 = db[4]; d.z1 = db[5];
    d.bx = db[1] - db[0] + 1;
    d.by = db[3] - db[2] + 1;
    c->dcells = size_t(d.bx) * d.by * (db[5] - db[4] + 1);
    const double init[3] = {g.eps, 1.0, 1.0};
    for (int a = 0; a < 3; ++a) {
      MPB_TRY(dalloc(c, reinterpret_cast<void **>(&c->d_design[a]), c->dcells * sizeof(double)), "design allocation");
      std::vector<double> h(c->dcells, init[a]);
      MPB_TRY(cudaMemcpyAsync(c->d_design[a], h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream),
              "cudaMemcpy");
      MPB_TRY(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    }
    d.eps = c->d_design[0];
    d.dscale = c->d_design[1];
    d.chiscale = c->d_design[2];
    for (int s = 0; s < 3; ++s)
      for (int r = 0; r < 2; ++r) {
        d.pD[s][r] = coef[0][s][r];
        d.pxi[s][r] = coef[1][s][r];
      }
    d.sumChi0 = c->sumChi0;
    d.sumXi0 = c->sumXi0;
    d.chi = g.chi;
    d.lin = c->mode == MODE_PLRC_LIN;
    c->design = true;
    if (c->fp32) c->epf.design = d;
    else c->epd.design = d;
  }
  // AUTO = GLOBAL: on the 256x256x512 PLRC + Kerr workload the global-load
  // kernels (E 0.92 ms, B 0.47 ms per launch) beat the TMA-staged ones
  // (E 1.12 ms, B 0.61 ms), whose 12 small tile copies per plane and block
  // serialise in the copy engine.
  c->fused = g.staging == MP_STAGING_FUSED;
  // CUDA graphs for grids of up to 4 M cells, whose half steps take a few
  // microseconds, so that the gaps between launches matter
  c->use_graphs = (long long)g.nx * g.ny * g.nz <= (4LL << 20);
  if (g.staging == MP_STAGING_TMA) {
    if (!setup_tma(c)) return fail(set_err(c, MP_ERR_UNSUPPORTED, "TMA tensor maps could not be encoded"));
    // TMA kernels: two resident blocks per SM; about four waves of blocks so
    // each block's pipeline runs over a long chunk of planes
    const long long tiles = (long long)(g.nx / kTmaTileX) * (g.ny / kTmaTileY);
    const long long chunks = std::max(1LL, (148LL * 8 + tiles - 1) / tiles);
    const int ne = g.nz + 2, nb = g.nz + 2;
    const int ke = int(std::max(1LL, (ne + chunks - 1) / chunks)), kb = int(std::max(1LL, (nb + chunks - 1) / chunks));
    if (c->fp32) { c->epf.kchunk = ke; c->bpf.kchunk = kb; }
    else { c->epd.kchunk = ke; c->bpd.kchunk = kb; }
  }
  MPB_TRY(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
#undef MPB_TRY
  *out = c;
  return MP_OK;
}

// Resolves a field name to (device pointer, stride, offset, first plane,
// number of planes) of its device array.
struct FieldView {
  void *base = nullptr;
  int stride = 1, offset = 0;
  int k0 = 0, nk = 0;
  bool zero = false;  // a pole without state: reads as zeros
};

int resolve(mp_ctx *c, const char *name, FieldView &v) {
  static const char *fn[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};
  if (!name) return set_err(c, MP_ERR_NAME, "field name is NULL");
  for (int f = 0; f < 6; ++f)
    if (!strcmp(name, fn[f])) {
      v.base = c->F[f];
      v.k0 = 0;
      v.nk = c->cfg.nz + 2;
      return MP_OK;
    }
  static const char *pn[4] = {"PlasmaDensity", "PlasmaJx", "PlasmaJy", "PlasmaJz"};
  for (int q = 0; q < 4; ++q)
    if (!strcmp(name, pn[q])) {
      if (!c->plasma[q]) return set_err(c, MP_ERR_NAME, "%s: no plasma plug-in in this configuration", name);
      v.base = c->plasma[q];
      v.k0 = 0;
      v.nk = c->cfg.nz + 2;
      return MP_OK;
    }
  if (!strncmp(name, "Psi", 3) && (name[3] == 'R' || name[3] == 'I') && name[4] >= '1' && name[4] <= '3' &&
      name[5] >= 'x' && name[5] <= 'z' && name[6] == 0) {
    const bool plrc = c->mode == MODE_PLRC_LIN || c->mode == MODE_PLRC_NONLIN;
    if (!plrc) return set_err(c, MP_ERR_NAME, "%s: solver has no PLRC accumulators", name);
    const int pole = name[4] - '1', comp = name[5] - 'x';
    const int s = c->slot_of_pole[pole];
    v.stride = 2;
    v.offset = name[3] == 'R' ? 0 : 1;
    if (s < 0) {
      v.zero = true;
      return MP_OK;
    }
    v.base = c->psi[s][comp];
    v.k0 = c->mz0;
    v.nk = c->mz1 - c->mz0 + 1;
    return MP_OK;
  }
  return set_err(c, MP_ERR_NAME, "unknown field name '%s'", name);
}

int ensure_staging(mp_ctx *c, size_t n) {
  if (c->staging_n >= n) return MP_OK;
  if (c->staging) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_n = 0;
  }
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&c->staging), n * sizeof(double));
  if (e != cudaSuccess) return cuda_err(c, e, "staging allocation");
  c->staging_n = n;
  return MP_OK;
}

const size_t kStagingChunk = size_t(1) << 24;  // doubles per host<->device chunk

// Optional per-kernel event timing (mp_kernel_times): events recorded before
// and after each group of launches of one step.
struct StepTimer {
  cudaEvent_t ev[6];
  bool on = false;
};

// Per-step callbacks of step_impl: `before(n)` runs before the launches of the
// n-th step of the call, `after(n)` after them (both may launch work on the
// stream and return an mp_status).
struct StepHooks {
  std::function<int(long long)> before, after;
};

// The injection planes of the steps from c->time on, from the buffers that
// src_stream fills ahead; launches the next batch into the other buffer.
// Returns the planes of step c->time in *planes and the steps they cover.
template <typename T>
int sources_ahead(mp_ctx *c, int want, const T **planes, int *steps) {
  T *bufs[2] = {static_cast<T *>(c->src_buf), static_cast<T *>(c->src_buf2)};
  const size_t per_step = 4 * size_t(c->plane);
  cudaError_t e;
  int u = -1;
  for (int b = 0; b < 2; ++b)
    if (c->pre_k[b] > 0 && c->time >= c->pre_t0[b] && c->time < c->pre_t0[b] + c->pre_k[b]) u = b;
  if (u < 0) {
    // nothing ahead covers this step: compute a batch here, into buffer 0
    u = 0;
    if (c->pre_pending[0] && (e = cudaStreamWaitEvent(c->stream, c->src_done[0], 0)) != cudaSuccess)
      return cuda_err(c, e, "cudaStreamWaitEvent");
    e = launch_source_batch<T>(c->sq[0][0], c->sq[0][1], c->time, c->src_batch, bufs[0], c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "source kernel");
    c->launches++;
    c->pre_t0[0] = c->time;
    c->pre_k[0] = c->src_batch;
    c->pre_pending[0] = false;
  } else if (c->pre_pending[u]) {
    if ((e = cudaStreamWaitEvent(c->stream, c->src_done[u], 0)) != cudaSuccess)
      return cuda_err(c, e, "cudaStreamWaitEvent");
    c->pre_pending[u] = false;
  }
  const int off = int(c->time - c->pre_t0[u]);
  *planes = bufs[u] + size_t(off) * per_step;
  *steps = std::min(want, c->pre_k[u] - off);
  // the batch after this buffer's, into the other one once the steps that
  // read it (all launched before now) are done
  const int w = 1 - u;
  const long long nt0 = c->pre_t0[u] + c->pre_k[u];
  if (!(c->pre_k[w] > 0 && c->pre_t0[w] == nt0)) {
    if ((e = cudaEventRecord(c->src_free[w], c->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(c->src_stream, c->src_free[w], 0)) != cudaSuccess)
      return cuda_err(c, e, "event");
    e = launch_source_batch<T>(c->sq[0][0], c->sq[0][1], nt0, c->src_batch, bufs[w], c->src_stream);
    if (e != cudaSuccess) return cuda_err(c, e, "source kernel");
    if ((e = cudaEventRecord(c->src_done[w], c->src_stream)) != cudaSuccess) return cuda_err(c, e, "event");
    c->launches++;
    c->pre_t0[w] = nt0;
    c->pre_k[w] = c->src_batch;
    c->pre_pending[w] = true;
  }
  return MP_OK;
}

// Per step: E half, B half.  The injection planes of a block of up to
// src_batch steps are computed ahead in one launch (they depend on
// Process::time only), and each half step reads its step's plane pair.
// Without gauss_inject and the per-kernel timer the next block is computed on
// a second stream while the current one is stepped (sources_ahead).
// The launches of K steps whose injection planes start at `planes` (plane q
// of the batch at planes + 4 q plane).
template <typename T>
cudaError_t launch_steps(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, const T *planes, int K) {
  const size_t pl = size_t(c->plane);
  for (int q = 0; q < K; ++q) {
    if (c->nsrc) {
      const T *base = planes + size_t(q) * 4 * pl;
      ep.src[0].v0 = base;
      ep.src[0].v1 = base + pl;
      bp.src[0].v0 = base + 2 * pl;
      bp.src[0].v1 = base + 3 * pl;
    }
    cudaError_t e = c->fused ? launch_step_fused<T>(ep, bp, c->mode, c->np, 1, c->stream)
                    : c->tma ? launch_e_half_tma<T>(ep, c->etma, c->mode, c->np, c->stream)
                             : launch_e_half<T>(ep, c->mode, c->np, c->stream);
    if (e != cudaSuccess) return e;
    e = c->fused ? launch_step_fused<T>(ep, bp, c->mode, c->np, 2, c->stream)
        : c->tma ? launch_b_half_tma<T>(bp, c->btma, c->stream)
                 : launch_b_half<T>(bp, c->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The graph of K steps from `planes`, captured on first use (the kernels'
// parameters are fixed for the context but for the injection planes; the
// plane buffers are read when the graph runs).  *exec = nullptr when the
// stream is being captured by the caller (the steps are then launched one by
// one, into the caller's graph).
template <typename T>
int step_graph(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, const T *planes, int K, cudaGraphExec_t *exec) {
  *exec = nullptr;
  cudaStreamCaptureStatus cs;
  cudaError_t e = cudaStreamIsCapturing(c->stream, &cs);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaStreamIsCapturing");
  if (cs != cudaStreamCaptureStatusNone) return MP_OK;
  for (const auto &g : c->graphs)
    if (g.planes == planes && g.K == K) {
      *exec = g.exec;
      return MP_OK;
    }
  if (c->graphs.size() >= 16) {  // keep the most recent ones
    cudaGraphExecDestroy(c->graphs.front().exec);
    c->graphs.erase(c->graphs.begin());
  }
  cudaGraph_t graph = nullptr;
  if ((e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return cuda_err(c, e, "cudaStreamBeginCapture");
  const cudaError_t le = launch_steps<T>(c, ep, bp, planes, K);
  e = cudaStreamEndCapture(c->stream, &graph);
  if (le != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_err(c, le, "step kernels (graph capture)");
  }
  if (e != cudaSuccess) return cuda_err(c, e, "cudaStreamEndCapture");
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaGraphInstantiate");
  c->graphs.push_back({planes, K, x});
  *exec = x;
  return MP_OK;
}

template <typename T>
int step_impl(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, int n_steps, StepTimer *tm = nullptr,
              double *acc = nullptr, const StepHooks *hooks = nullptr) {
  const size_t pl = size_t(c->plane);
  const bool ahead = c->src_stream && !tm;
  int t = 0;
  while (t < n_steps) {
    int K = c->nsrc ? std::min(c->src_batch, n_steps - t) : n_steps - t;
    cudaError_t e;
    const T *planes = static_cast<const T *>(c->src_buf);
    if (c->nsrc && ahead) {
      NvtxRange nv("mp sources");
      const int rc = sources_ahead<T>(c, K, &planes, &K);
      if (rc != MP_OK) return rc;
    } else if (c->nsrc) {
      // computed here into buffer 0: what the buffers held ahead is void
      if (c->pre_pending[0] && (e = cudaStreamWaitEvent(c->stream, c->src_done[0], 0)) != cudaSuccess)
        return cuda_err(c, e, "cudaStreamWaitEvent");
      c->pre_k[0] = c->pre_k[1] = 0;
      c->pre_pending[0] = false;
      NvtxRange nv("mp sources");
      if (tm) cudaEventRecord(tm->ev[4], c->stream);
      if (c->gauss) {
        // the block holding this step (computed here when it changes); the
        // batch ends where the source's state changes next
        bool active;
        long long toff, until;
        const int rc = gauss_prepare(*c->gauss, c->time, c->stream, &active, &toff, &until, &c->launches, &c->err);
        if (rc != MP_OK) return rc;
        if (until > c->time) K = int(std::min<long long>(K, until - c->time));
        for (int side = 0; side < 2; ++side) {
          c->sq[0][side].g_active = active ? 1 : 0;
          c->sq[0][side].g_toff = toff;
        }
      }
      e = launch_source_batch<T>(c->sq[0][0], c->sq[0][1], c->time, K, static_cast<T *>(c->src_buf), c->stream);
      if (e != cudaSuccess) return cuda_err(c, e, "source kernel");
      c->launches++;
      if (tm) {
        cudaEventRecord(tm->ev[5], c->stream);
        e = cudaEventSynchronize(tm->ev[5]);
        if (e != cudaSuccess) return cuda_err(c, e, "event synchronize");
        float ms;
        cudaEventElapsedTime(&ms, tm->ev[4], tm->ev[5]);
        acc[2] += ms;  // sources, all steps of the block
      }
    }
    if (c->use_graphs && !tm && !hooks) {
      // the batch as one CUDA graph (at most 64 steps per graph)
      const int Kg = std::min(K, 64);
      cudaGraphExec_t g;
      const int rc = step_graph<T>(c, ep, bp, planes, Kg, &g);
      if (rc != MP_OK) return rc;
      if (g) {
        NvtxRange nv("mp steps (graph)");
        if ((e = cudaGraphLaunch(g, c->stream)) != cudaSuccess) return cuda_err(c, e, "cudaGraphLaunch");
        c->launches += 2 * Kg;
        c->time += Kg;
        t += Kg;
        continue;
      }
    }
    for (int q = 0; q < K; ++q) {
      if (c->nsrc) {
        const T *base = planes + size_t(q) * 4 * pl;
        ep.src[0].v0 = base;
        ep.src[0].v1 = base + pl;
        bp.src[0].v0 = base + 2 * pl;
        bp.src[0].v1 = base + 3 * pl;
      }
      if (hooks && hooks->before) {
        const int rc = hooks->before(t + q);
        if (rc != MP_OK) return rc;
      }
      NvtxRange nv("mp step");
      if (tm) cudaEventRecord(tm->ev[0], c->stream);
      // (the fused form: its step kernel in the E slot, the border kernel in the B slot)
      e = c->fused ? launch_step_fused<T>(ep, bp, c->mode, c->np, 1, c->stream)
          : c->tma ? launch_e_half_tma<T>(ep, c->etma, c->mode, c->np, c->stream)
                   : launch_e_half<T>(ep, c->mode, c->np, c->stream);
      if (e != cudaSuccess) return cuda_err(c, e, "E half-step kernel");
      c->launches++;
      if (tm) cudaEventRecord(tm->ev[1], c->stream);
      e = c->fused ? launch_step_fused<T>(ep, bp, c->mode, c->np, 2, c->stream)
          : c->tma ? launch_b_half_tma<T>(bp, c->btma, c->stream)
                   : launch_b_half<T>(bp, c->stream);
      if (e != cudaSuccess) return cuda_err(c, e, "B half-step kernel");
      c->launches++;
      if (tm) {
        cudaEventRecord(tm->ev[2], c->stream);
        e = cudaEventSynchronize(tm->ev[2]);
        if (e != cudaSuccess) return cuda_err(c, e, "event synchronize");
        float ms[2];
        cudaEventElapsedTime(&ms[0], tm->ev[0], tm->ev[1]);
        cudaEventElapsedTime(&ms[1], tm->ev[1], tm->ev[2]);
        acc[0] += ms[0];  // E half
        acc[1] += ms[1];  // B half
      }
      c->time++;
      if (hooks && hooks->after) {
        const int rc = hooks->after(t + q);
        if (rc != MP_OK) return rc;
      }
    }
    t += K;
  }
  return MP_OK;
}

// "DesignEps", "DesignDepsScale", "DesignChiScale": index of the map, or -1
int design_map(const mp_ctx *c, const char *name) {
  if (!c->design || !name) return -1;
  static const char *dn[3] = {"DesignEps", "DesignDepsScale", "DesignChiScale"};
  for (int a = 0; a < 3; ++a)
    if (!strcmp(name, dn[a])) return a;
  return -1;
}

}  // namespace

extern "C" {

void mp_config_defaults(mp_config *c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->abi_version = MP_ABI_VERSION;
  c->nx = c->ny = c->nz = 32;
  c->dx = c->dy = c->dz = 0.1;  // grid-dx.. default (globals.cpp:57-59)
  c->dt = 1e-2;                 // dt default (globals.cpp:61)
  c->precision = MP_FP64;
  c->solver = MP_SOLVER_PLRC_LIN;
  c->boundary = MP_BOUNDARY_PERIODIC;
  c->eps = 1.0;   // fdtd_plrc.t:417
  c->chi = 0.1;   // fdtd_plrc.cpp:463, fdtd_nl.cpp:151
  for (int n = 0; n < MP_MAX_POLES; ++n) {
    c->poles[n].eps = 0.0;    // fdtd_plrc.t:419-421
    c->poles[n].delta = 0.0;  // :423-425
    c->poles[n].om2 = 1.0;    // :427-429
  }
  c->medium_z0 = 0;
  c->medium_z1 = 1 << 30;
  c->eps_bg = 1.0;
  c->cpml = MP_CPML_NONE;
  c->cpml_d = 8;              // cpml_border.cpp:146-149
  c->cpml_kappa_max = 15.0;
  c->cpml_a_max = 0.25;
  c->cpml_sigma_max = 3.0;
  c->n_sources = 0;
  for (int s = 0; s < MP_MAX_SOURCES; ++s) {
    mp_source &q = c->sources[s];
    q.kind = MP_SOURCE_NONE;
    q.distance = 15;          // incsource.cpp:84
    q.k[2] = 1.0;             // sources.cpp:64
    q.ramp = 0.5;             // sources.cpp:78
    q.width = 10.0;           // sources.cpp:237
    q.offset = 40.0;          // sources.cpp:238
    q.eps = 1.0;
    q.length = 1.0;           // shortpulseinject.cpp:38-46
    q.waist = 1.0;
    q.om0 = 2 * M_PI;
    q.amp = 1.0;
    q.t_size = 4096;          // gaussinject.cpp:38-47
    q.t_off = 0;
    q.k0 = 2 * M_PI;
  }
  c->newton_max_iter = 64;
  c->newton_tol = 1e-9;       // fdtd_plrc.cpp:414
  c->device = 0;
  c->design_box[0] = c->design_box[2] = c->design_box[4] = 1;  // empty: x0 > x1
  c->plasma = 0;
  c->plasma_nu = c->plasma_mpa = c->plasma_wion = 1.0;  // plasmadensity.cpp:55-58
  c->plasma_k = 5;
  c->plasma_current = 0;
  c->plasma_em = 1.0;                                   // plasmacurrent.cpp:10-12
  c->plasma_gamma = 0.1;
  c->plasma_rho_bg = 0.0;
}

int mp_create(const mp_config *cfg, mp_ctx **out) {
  if (!out) return set_err(nullptr, MP_ERR_INVALID, "out is NULL");
  *out = nullptr;
  g_create_err[0] = 0;
  return create_impl(cfg, out);
}

const char *mp_create_error(void) { return g_create_err; }

// The pinned host checkpoint buffers of mp_set_host_checkpoint_budget.
static void free_host_ckpt(mp_ctx *c) {
  for (void *p : c->host_ckpt) {
    cudaHostUnregister(p);
    std::free(p);
  }
  c->host_ckpt.clear();
}

// Frees what mp_objective_record kept (defined with the adjoint below).  Every
// call that steps the context or writes its state, time, design maps, stream or
// host checkpoint buffers releases it first.
static void release_record(mp_ctx *c);

void mp_destroy(mp_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->src_stream) {
    cudaStreamSynchronize(c->src_stream);
    cudaStreamDestroy(c->src_stream);
  }
  for (int b = 0; b < 2; ++b) {
    if (c->src_done[b]) cudaEventDestroy(c->src_done[b]);
    if (c->src_free[b]) cudaEventDestroy(c->src_free[b]);
  }
  for (void *p : c->allocs) cudaFree(p);
  if (c->gauss) {
    gauss_destroy(*c->gauss);
    delete c->gauss;
  }
  if (c->staging) cudaFree(c->staging);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->h_kerr) cudaFreeHost(c->h_kerr);
  if (c->h_diag) cudaFreeHost(c->h_diag);
  free_host_ckpt(c);
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int mp_set_stream(mp_ctx *c, void *s) {
  if (!c) return MP_ERR_INVALID;
  release_record(c);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "cudaStreamSynchronize");
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
  return MP_OK;
}

int mp_field_size(mp_ctx *c, const char *name, size_t *count) {
  if (!c || !count) return MP_ERR_INVALID;
  if (design_map(c, name) >= 0) {
    *count = c->dcells;
    return MP_OK;
  }
  FieldView v;
  int rc = resolve(c, name, v);
  if (rc != MP_OK) return rc;
  *count = c->fcount;
  return MP_OK;
}

int mp_upload(mp_ctx *c, const char *name, const double *host, size_t count) {
  if (!c || !host) return MP_ERR_INVALID;
  release_record(c);
  const int dm = design_map(c, name);
  if (dm >= 0) {
    if (count != c->dcells) return set_err(c, MP_ERR_INVALID, "%s: %zu values, expected %zu", name, count, c->dcells);
    cudaSetDevice(c->cfg.device);
    cudaError_t e = cudaMemcpyAsync(c->d_design[dm], host, count * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? MP_OK : cuda_err(c, e, "design upload");
  }
  FieldView v;
  int rc = resolve(c, name, v);
  if (rc != MP_OK) return rc;
  if (count != c->fcount) return set_err(c, MP_ERR_INVALID, "%s: %zu values, expected %zu", name, count, c->fcount);
  cudaSetDevice(c->cfg.device);
  if (v.zero) {
    for (size_t q = 0; q < count; ++q)
      if (host[q] != 0.0) return set_err(c, MP_ERR_INVALID, "%s: this pole has Delta eps = 0 and keeps no state", name);
    return MP_OK;
  }
  const size_t pl = size_t(c->plane);
  const size_t n = size_t(v.nk) * pl;
  const double *src = host + size_t(v.k0) * pl;
  rc = ensure_staging(c, std::min(n, kStagingChunk));
  if (rc != MP_OK) return rc;
  for (size_t off = 0; off < n; off += kStagingChunk) {
    const size_t m = std::min(kStagingChunk, n - off);
    cudaError_t e = cudaMemcpyAsync(c->staging, src + off, m * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "upload copy");
    char *dst = static_cast<char *>(v.base) + off * size_t(v.stride) * c->esz;
    e = launch_convert_in(c->staging, dst, c->fp32, (long long)m, v.stride, v.offset, c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "upload convert");
    c->launches++;
  }
  return MP_OK;
}

int mp_download(mp_ctx *c, const char *name, double *host, size_t count) {
  if (!c || !host) return MP_ERR_INVALID;
  const int dm = design_map(c, name);
  if (dm >= 0) {
    if (count != c->dcells) return set_err(c, MP_ERR_INVALID, "%s: %zu values, expected %zu", name, count, c->dcells);
    cudaSetDevice(c->cfg.device);
    cudaError_t e = cudaMemcpyAsync(host, c->d_design[dm], count * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? MP_OK : cuda_err(c, e, "design download");
  }
  FieldView v;
  int rc = resolve(c, name, v);
  if (rc != MP_OK) return rc;
  if (count != c->fcount) return set_err(c, MP_ERR_INVALID, "%s: %zu values, expected %zu", name, count, c->fcount);
  cudaSetDevice(c->cfg.device);
  const size_t pl = size_t(c->plane);
  if (v.zero || v.nk < int(c->cfg.nz + 2)) memset(host, 0, count * sizeof(double));
  if (!v.zero) {
    const size_t n = size_t(v.nk) * pl;
    double *dstbase = host + size_t(v.k0) * pl;
    rc = ensure_staging(c, std::min(n, kStagingChunk));
    if (rc != MP_OK) return rc;
    for (size_t off = 0; off < n; off += kStagingChunk) {
      const size_t m = std::min(kStagingChunk, n - off);
      const char *src = static_cast<const char *>(v.base) + off * size_t(v.stride) * c->esz;
      cudaError_t e = launch_convert_out(src, c->staging, c->fp32, (long long)m, v.stride, v.offset, c->stream);
      if (e != cudaSuccess) return cuda_err(c, e, "download convert");
      c->launches++;
      e = cudaMemcpyAsync(dstbase + off, c->staging, m * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) return cuda_err(c, e, "download copy");
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "download");
  }
  // z-periodic grids: the ghost planes are images (periodic_bound.cpp:53-71)
  const bool field = name[0] == 'E' || name[0] == 'B';
  if (field && c->cfg.boundary == MP_BOUNDARY_PERIODIC) {
    const int nz = c->cfg.nz;
    memcpy(host, host + size_t(nz) * pl, pl * sizeof(double));
    memcpy(host + size_t(nz + 1) * pl, host + pl, pl * sizeof(double));
  }
  return MP_OK;
}

int mp_step_async(mp_ctx *c, int n_steps) {
  if (!c || n_steps < 0) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  return c->fp32 ? step_impl<float>(c, c->epf, c->bpf, n_steps) : step_impl<double>(c, c->epd, c->bpd, n_steps);
}

int mp_check_status(mp_ctx *c) {
  if (!c) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  cudaError_t e = cudaMemcpyAsync(c->h_status, c->d_status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "status read");
  const int newton = c->h_status[ST_NEWTON], nonfin = c->h_status[ST_NONFINITE];
  const int timeout = c->h_status[ST_TIMEOUT], bounds = c->h_status[ST_BOUNDS];
  if (newton || nonfin || timeout || bounds) {
    cudaMemsetAsync(c->d_status, 0, ST_COUNT * sizeof(int), c->stream);
    if (bounds)
      return set_err(c, MP_ERR_BOUNDS, "%d state accesses fell outside their arrays and were skipped (checked build)",
                     bounds);
    if (timeout)
      return set_err(c, MP_ERR_CUDA, "%d blocks gave up waiting for their TMA plane loads; the step is incomplete",
                     timeout);
    if (nonfin) return set_err(c, MP_ERR_NONFINITE, "%d field values became NaN or Inf", nonfin);
    return set_err(c, MP_ERR_NEWTON, "Kerr Newton solve did not converge in %d cell updates (max %d iterations)",
                   newton, c->cfg.newton_max_iter);
  }
  return MP_OK;
}

int mp_step(mp_ctx *c, int n_steps) {
  int rc = mp_step_async(c, n_steps);
  if (rc != MP_OK) return rc;
  return mp_check_status(c);
}

int mp_get_time(mp_ctx *c, long long *t) {
  if (!c || !t) return MP_ERR_INVALID;
  *t = c->time;
  return MP_OK;
}

int mp_set_time(mp_ctx *c, long long t) {
  if (!c) return MP_ERR_INVALID;
  release_record(c);
  c->time = t;
  return MP_OK;
}

int mp_sync(mp_ctx *c) {
  if (!c) return MP_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? MP_OK : cuda_err(c, e, "cudaStreamSynchronize");
}

int mp_device_field(mp_ctx *c, const char *name, void **dptr, size_t *count, int *elem_bytes) {
  if (!c || !dptr || !count || !elem_bytes) return MP_ERR_INVALID;
  FieldView v;
  int rc = resolve(c, name, v);
  if (rc != MP_OK) return rc;
  if (v.stride != 1) return set_err(c, MP_ERR_NAME, "%s: accumulators are stored complex-interleaved", name);
  *dptr = v.base;
  *count = c->fcount;
  *elem_bytes = c->esz;
  return MP_OK;
}

long long mp_launch_count(mp_ctx *c) { return c ? c->launches : -1; }

}  // extern "C"

namespace mpb {
void set_global_error(const char *msg) { snprintf(g_create_err, sizeof g_create_err, "%s", msg); }

// The grid of a context (for the HDF5 writer of mp_hdf5.cu).
int ctx_grid(const mp_ctx *c, int *nx, int *ny, int *nz) {
  if (!c) return MP_ERR_INVALID;
  *nx = c->cfg.nx;
  *ny = c->cfg.ny;
  *nz = c->cfg.nz;
  return MP_OK;
}
}  // namespace mpb

extern "C" {

int mp_field_energy(mp_ctx *c, double *energy) {
  if (!c || !energy) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  const mp_config &g = c->cfg;
  const void *f[6];
  for (int q = 0; q < 6; ++q) f[q] = c->F[q];
  double *result = c->d_diag + (g.nz + 2);
  cudaError_t e = launch_field_energy(f, c->esz, g.nx, g.ny, g.nz, g.dx * g.dy * g.dz, c->d_diag, result, c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "energy kernels");
  c->launches += 2;
  e = cudaMemcpyAsync(c->h_diag, result, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "energy read");
  *energy = *c->h_diag;
  return MP_OK;
}

int mp_kernel_times(mp_ctx *c, int n_steps, double *e_ms, double *b_ms, double *s_ms) {
  if (!c || n_steps < 1 || !e_ms || !b_ms || !s_ms) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  StepTimer tm;
  for (int q = 0; q < 6; ++q) {
    cudaError_t e = cudaEventCreate(&tm.ev[q]);
    if (e != cudaSuccess) return cuda_err(c, e, "cudaEventCreate");
  }
  double acc[3] = {0, 0, 0};
  int rc = c->fp32 ? step_impl<float>(c, c->epf, c->bpf, n_steps, &tm, acc)
                   : step_impl<double>(c, c->epd, c->bpd, n_steps, &tm, acc);
  for (int q = 0; q < 6; ++q) cudaEventDestroy(tm.ev[q]);
  if (rc != MP_OK) return rc;
  *e_ms = acc[0] / n_steps;
  *b_ms = acc[1] / n_steps;
  *s_ms = acc[2] / n_steps;
  return mp_check_status(c);
}

int mp_kerr_counts(mp_ctx *c, long long *solves, long long *iterations) {
  if (!c || !solves || !iterations) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  cudaError_t e = cudaMemcpyAsync(c->h_kerr, c->d_kerr, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_kerr, 0, 2 * sizeof(unsigned long long), c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "Kerr counter read");
  *solves = (long long)c->h_kerr[0];
  *iterations = (long long)c->h_kerr[1];
  return MP_OK;
}

int mp_last_error(mp_ctx *c, char *buf, size_t n) {
  if (!buf || n == 0) return MP_ERR_INVALID;
  const char *m = c ? c->err.c_str() : g_create_err;
  snprintf(buf, n, "%s", m);
  return MP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// mp_objective / mp_adjoint

namespace {

// Device buffers of one call, freed (after the stream drains) when it returns.
struct DevBufs {
  cudaStream_t st;
  std::vector<void *> p;
  explicit DevBufs(cudaStream_t s) : st(s) {}
  ~DevBufs() {
    cudaStreamSynchronize(st);
    for (void *q : p) cudaFree(q);
  }
  cudaError_t alloc(void **out, size_t bytes) {
    *out = nullptr;
    if (!bytes) return cudaSuccess;
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) return e;
    p.push_back(*out);
    return cudaMemsetAsync(*out, 0, bytes, st);
  }
};

// The arrays that make up the forward state: fields, PLRC accumulators, CPML psi.
std::vector<std::pair<void *, size_t>> state_regions(const mp_ctx *c) {
  std::vector<std::pair<void *, size_t>> r;
  for (int f = 0; f < 6; ++f) r.emplace_back(c->F[f], c->fcount * c->esz);
  for (int q = 0; q < 4; ++q)
    if (c->plasma[q]) r.emplace_back(c->plasma[q], c->fcount * c->esz);
  for (int s = 0; s < c->np; ++s)
    for (int a = 0; a < 3; ++a) r.emplace_back(c->psi[s][a], 2 * c->psi_cells * c->esz);
  for (int f = 0; f < 6; ++f)
    for (const LayerHost *L : {&c->cpE[f], &c->cpH[f]})
      if (L->active) {
        r.emplace_back(L->psi0, L->n * c->esz);
        r.emplace_back(L->psi1, L->n * c->esz);
      }
  return r;
}

// The adjoint face entry per axis of the E (isH false) or H CPML currents: the
// low and the high face of the axis together (their layers must not overlap,
// so that a cell is in at most one face per axis).
template <typename T>
int adj_faces(mp_ctx *c, DevBufs &buf, bool isH, const CpmlFace<T> *fw, AdjFace<T> out[3]) {
  const mp_config &g = c->cfg;
  const int n3[3] = {g.nx, g.ny, g.nz};
  for (int dim = 0; dim < 3; ++dim) {
    AdjFace<T> &F = out[dim];
    F = AdjFace<T>();
    int fl[2], nf = 0;
    for (int f = 0; f < 6; ++f) {
      const LayerHost &L = isH ? c->cpH[f] : c->cpE[f];
      if (L.active && L.dim == dim && nf < 2) fl[nf++] = f;
    }
    if (!nf) continue;
    const LayerHost *A = isH ? &c->cpH[fl[0]] : &c->cpE[fl[0]];
    const LayerHost *B = nf == 2 ? (isH ? &c->cpH[fl[1]] : &c->cpE[fl[1]]) : nullptr;
    int fa = fl[0], fb = nf == 2 ? fl[1] : -1;
    if (B && B->lo < A->lo) {
      std::swap(A, B);
      std::swap(fa, fb);
    }
    if (B && B->lo <= A->hi)
      return set_err(c, MP_ERR_UNSUPPORTED, "mp_adjoint: the two CPML layers along axis %d overlap", dim);
    F.active = 1;
    F.lo0 = A->lo;
    F.hi0 = A->hi;
    F.n0 = A->hi - A->lo + 1;
    F.lo1 = B ? B->lo : 1;
    F.hi1 = B ? B->hi : 0;
    const int ntot = F.n0 + (B ? B->hi - B->lo + 1 : 0);
    F.zlo = A->zlo;
    F.ex = dim == 0 ? ntot : g.nx;
    F.ey = dim == 1 ? ntot : g.ny;
    const size_t zdepth = size_t(g.nz - F.zlo + 1);
    const size_t cells = dim == 2 ? size_t(ntot) * size_t(c->plane) : zdepth * size_t(F.ex) * size_t(F.ey);
    if (cells >= (size_t(1) << 31))  // the adjoint kernels index face arrays in 32 bits
      return set_err(c, MP_ERR_UNSUPPORTED, "mp_adjoint: CPML face array of %zu cells exceeds 2^31", cells);
    void *a0, *a1;
    cudaError_t e;
    if ((e = buf.alloc(&a0, cells * sizeof(T))) != cudaSuccess || (e = buf.alloc(&a1, cells * sizeof(T))) != cudaSuccess)
      return cuda_err(c, e, "adjoint allocation");
    F.a0 = static_cast<T *>(a0);
    F.a1 = static_cast<T *>(a1);
    F.n = (long long)cells;
    if (!B) {
      F.b = fw[fa].b;
      F.c = fw[fa].c;
      continue;
    }
    // the two faces' b and c lines are zero outside their layers: add them
    const size_t len = size_t(n3[dim]) + 2;
    std::vector<T> hb(len), hc(len), tb(len), tc(len);
    if ((e = cudaMemcpy(hb.data(), fw[fa].b, len * sizeof(T), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(hc.data(), fw[fa].c, len * sizeof(T), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(tb.data(), fw[fb].b, len * sizeof(T), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(tc.data(), fw[fb].c, len * sizeof(T), cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_err(c, e, "line read");
    for (size_t q = 0; q < len; ++q) {
      hb[q] += tb[q];
      hc[q] += tc[q];
    }
    void *lb, *lc;
    if ((e = buf.alloc(&lb, len * sizeof(T))) != cudaSuccess || (e = buf.alloc(&lc, len * sizeof(T))) != cudaSuccess ||
        (e = cudaMemcpyAsync(lb, hb.data(), len * sizeof(T), cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(lc, hc.data(), len * sizeof(T), cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
      return cuda_err(c, e, "line upload");
    F.b = static_cast<const T *>(lb);
    F.c = static_cast<const T *>(lc);
  }
  return MP_OK;
}

int check_objective(mp_ctx *c, const mp_adjoint_config *a) {
  const mp_config &g = c->cfg;
  if (a->kind != MP_OBJ_E2_BOX && a->kind != MP_OBJ_SZ_PLANE)
    return set_err(c, MP_ERR_INVALID, "unknown objective kind %d", a->kind);
  if (a->steps < 1) return set_err(c, MP_ERR_INVALID, "steps must be >= 1");
  const int *b = a->box;
  if (b[0] < 1 || b[0] > b[1] || b[1] > g.nx || b[2] < 1 || b[2] > b[3] || b[3] > g.ny || b[4] < 1 || b[4] > b[5] ||
      b[5] > g.nz)
    return set_err(c, MP_ERR_INVALID, "objective box outside the interior");
  return MP_OK;
}

// 0-based x/y, MPulse z box of the objective (the Sz plane is box[4])
void objective_box(const mp_adjoint_config *a, int b0[6]) {
  b0[0] = a->box[0] - 1;
  b0[1] = a->box[1] - 1;
  b0[2] = a->box[2] - 1;
  b0[3] = a->box[3] - 1;
  b0[4] = a->box[4];
  b0[5] = a->kind == MP_OBJ_E2_BOX ? a->box[5] : a->box[4];
}

template <typename T>
int objective_term(mp_ctx *c, const mp_adjoint_config *a, double *out) {
  const mp_config &g = c->cfg;
  const T *E[3] = {static_cast<const T *>(c->F[0]), static_cast<const T *>(c->F[1]), static_cast<const T *>(c->F[2])};
  const T *B[3] = {static_cast<const T *>(c->F[3]), static_cast<const T *>(c->F[4]), static_cast<const T *>(c->F[5])};
  int b0[6];
  objective_box(a, b0);
  const double f = a->kind == MP_OBJ_E2_BOX ? g.dt : g.dt * g.dx * g.dy;
  cudaError_t e = launch_objective_term<T>(E, B, g.nx, g.ny, c->plane, a->kind, b0, f, out, c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "objective kernel");
  c->launches++;
  return MP_OK;
}

int read_sum(mp_ctx *c, double *terms, long long n, double *J) {
  cudaError_t e = launch_sum_terms(terms, n, terms + n, c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "sum kernel");
  c->launches++;
  e = cudaMemcpyAsync(c->h_diag, terms + n, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "objective read");
  *J = *c->h_diag;
  return MP_OK;
}

template <typename T>
int objective_impl(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, const mp_adjoint_config *a, double *J) {
  DevBufs buf(c->stream);
  double *terms;
  cudaError_t e = buf.alloc(reinterpret_cast<void **>(&terms), (size_t(a->steps) + 1) * sizeof(double));
  if (e != cudaSuccess) return cuda_err(c, e, "objective allocation");
  StepHooks h;
  h.after = [&](long long n) { return objective_term<T>(c, a, terms + n); };
  int rc = step_impl<T>(c, ep, bp, a->steps, nullptr, nullptr, &h);
  if (rc != MP_OK) return rc;
  rc = read_sum(c, terms, a->steps, J);
  return rc != MP_OK ? rc : mp_check_status(c);
}

// The checkpoint schedule of the reverse pass.  The steps are cut into chunks
// of Kh steps whose E history fits the history buffer; a chunk is reversed by
// running it forward from its start keeping E of every step ("leaf") and then
// stepping back.  Chunk starts are kept as state checkpoints where slots allow,
// placed by the binomial rule of revolve (Griewank): with s free slots and r
// the smallest number of sweeps with C(s + r, s) >= m chunks, the next
// checkpoint leaves C(s + r - 1, s) chunks to its left; with no free slot left
// the chunks are run again from the last checkpoint, last chunk first.
struct RevolveOps {
  std::function<int(long long, int)> restore;    // live state := checkpoint slot, at step
  std::function<int(long long, int)> save;       // checkpoint slot := live state
  std::function<int(long long, long long)> advance;  // run from -> to, no history
  std::function<int(long long, long long)> leaf;     // live at n0: run n0 -> n1 keeping E, step back
};

double binom_sr(int s, int r) {  // C(s + r, s)
  double v = 1;
  for (int q = 1; q <= s; ++q) v = v * double(r + q) / double(q);
  return v;
}

int revolve(long long a, long long b, int slot_a, std::vector<int> &free_slots, long long Kh, RevolveOps &ops,
            long long &live) {
  int rc;
  const long long m = (b - a + Kh - 1) / Kh;
  if (m <= 1) {
    if (live != a && (rc = ops.restore(a, slot_a)) != MP_OK) return rc;
    if ((rc = ops.leaf(a, b)) != MP_OK) return rc;
    live = b;
    return MP_OK;
  }
  if (free_slots.empty()) {
    for (long long e = b; e > a;) {
      const long long c0 = std::max(a, e - Kh);
      if (live != a && (rc = ops.restore(a, slot_a)) != MP_OK) return rc;
      live = a;
      if (c0 > a && (rc = ops.advance(a, c0)) != MP_OK) return rc;
      if ((rc = ops.leaf(c0, e)) != MP_OK) return rc;
      live = e;
      e = c0;
    }
    return MP_OK;
  }
  const int s = int(free_slots.size());
  int r = 1;
  while (binom_sr(s, r) < double(m)) ++r;
  const long long left = std::max(1LL, std::min(m - 1, (long long)binom_sr(s, r - 1)));
  const long long cpos = a + left * Kh;
  if (live != a && (rc = ops.restore(a, slot_a)) != MP_OK) return rc;
  if ((rc = ops.advance(a, cpos)) != MP_OK) return rc;
  live = cpos;
  const int sc = free_slots.back();
  free_slots.pop_back();
  if ((rc = ops.save(cpos, sc)) != MP_OK) return rc;
  if ((rc = revolve(cpos, b, sc, free_slots, Kh, ops, live)) != MP_OK) return rc;
  free_slots.push_back(sc);
  return revolve(a, cpos, slot_a, free_slots, Kh, ops, live);
}

// Steps the schedule runs forward in all (first pass and recomputation).
long long schedule_steps(long long Tn, long long Kh, int slots) {
  long long steps = 0;
  RevolveOps ops;
  ops.restore = [](long long, int) { return MP_OK; };
  ops.save = [](long long, int) { return MP_OK; };
  ops.advance = [&](long long f, long long t) { steps += t - f; return MP_OK; };
  ops.leaf = [&](long long f, long long t) { steps += t - f; return MP_OK; };
  std::vector<int> free_slots;
  for (int q = slots - 1; q >= 1; --q) free_slots.push_back(q);
  long long live = 0;
  revolve(0, Tn, 0, free_slots, Kh, ops, live);
  return steps;
}

// History chunk Kh, checkpoint slots and history buffers for Tn steps:
// checkpoint_every K > 0 gives chunks of K with a checkpoint at every chunk
// start; a memory budget (bytes for (slots + 1) states and Kh + 1 steps of
// history per buffer) gives the plan with the fewest forward steps; neither
// keeps the whole history.  A second history buffer, which lets the forward
// run of one chunk overlap the reverse pass of the last, is taken when there
// are several chunks and (under a budget) it fits beside the chosen plan.
bool plan_schedule(long long Tn, long long every, double budget, size_t S, size_t H, long long *Kh, int *slots,
                   int *nbuf) {
  if (every > 0) {
    *Kh = std::min(every, Tn);
    *slots = int((Tn + *Kh - 1) / *Kh);
    *nbuf = *Kh < Tn ? 2 : 1;
    return true;
  }
  if (!(budget > 0)) {
    *Kh = Tn;
    *slots = 1;
    *nbuf = 1;
    return true;
  }
  long long best = -1;
  for (long long kh = Tn; kh >= 1; kh = std::min(kh - 1, (long long)(kh * 0.9))) {
    const double room = budget - double(kh + 1) * double(H) - double(S);  // one slot for the final state
    if (room < double(S)) continue;
    const long long m = (Tn + kh - 1) / kh;
    const int s = int(std::min<double>(double(m), std::floor(room / double(S))));
    const long long cost = schedule_steps(Tn, kh, s);
    if (best < 0 || cost < best) {
      best = cost;
      *Kh = kh;
      *slots = s;
      *nbuf = m > 1 && room - double(s) * double(S) >= double(kh + 1) * double(H) ? 2 : 1;
    }
  }
  return best >= 0;
}

// Two-level schedule under a device budget and a host budget: the first
// forward run keeps the state at the start of every segment of L steps in
// pinned host memory (one state of S bytes per segment), and each segment is
// then reversed, last first, on the device schedule plan_schedule gives for L
// steps, starting from its host copy.  Taken when its forward steps plus the
// host copies (two per segment but the last, each counted as the steps that
// take as long: a step moves about 2.5 S through HBM at 4 TB/s and costs at
// least two launches of 10 us, a copy moves S through PCIe at 20 GB/s after
// 20 us) are fewer than the steps of the device schedule alone.
struct TwoLevel {
  long long L = 0, nseg = 0, Kh = 0;
  int slots = 0, nbuf = 1;
};

bool plan_two_level(long long Tn, double budget, double host_budget, size_t S, size_t H, long long one_level_steps,
                    TwoLevel *out) {
  if (!(host_budget > 0) || !(budget > 0) || S == 0) return false;
  const long long host_slots = (long long)std::floor(host_budget / double(S));
  if (host_slots < 2) return false;
  const double t_step = std::max(2.5 * double(S) / 4e12, 20e-6), t_copy = double(S) / 20e9 + 20e-6;
  const double copy_steps = t_copy / t_step;  // one host copy, in steps
  bool found = false;
  double best = double(one_level_steps);
  // fewer, longer segments than the host allows when that is cheaper
  for (long long nseg = host_slots; nseg >= 2; nseg = std::min(nseg - 1, (long long)(nseg * 0.8))) {
    const long long L = (Tn + nseg - 1) / nseg;
    const long long ns = (Tn + L - 1) / L;
    if (ns < 2) continue;
    long long Kh;
    int slots, nbuf;
    if (!plan_schedule(L, 0, budget, S, H, &Kh, &slots, &nbuf)) continue;
    // first run up to the last segment, then every segment on its schedule
    const long long last = Tn - (ns - 1) * L;
    const double steps = double((ns - 1) * L) + double(ns - 1) * double(schedule_steps(L, Kh, slots)) +
                         double(schedule_steps(last, Kh, slots)) + copy_steps * double(2 * ns - 1);
    if (steps < best) {
      best = steps;
      out->L = L;
      out->nseg = ns;
      out->Kh = Kh;
      out->slots = slots;
      out->nbuf = nbuf;
      found = true;
    }
  }
  return found;
}

// Phases of adjoint_impl: the whole of mp_adjoint; the forward part alone
// (mp_objective_record), which stops once the first run has reached the end;
// the reverse part alone (mp_adjoint_reverse), from what the forward part kept.
enum AdjPhase { kAdjAll = 0, kAdjRecord = 1, kAdjReverse = 2 };
const int kAdjStop = 1 << 20;  // returned through revolve when the forward part is done

}  // namespace

// What mp_objective_record keeps for mp_adjoint_reverse: the objective, the
// schedule, the checkpoint slots (the run's start and chunk starts, and its end
// state), the history buffers (the last chunk's E history in buffer 0) and the
// objective terms, in device memory freed with the record.
struct AdjRecord {
  DevBufs buf;
  mp_adjoint_config a;
  long long t0 = 0;  // the time the run started at
  double J = 0;
  long long Kh = 0;
  int slots = 0, nbuf = 1;
  bool two = false;
  TwoLevel tl;
  char *ckpt = nullptr, *hist[2] = {nullptr, nullptr};
  double *terms = nullptr;
  explicit AdjRecord(cudaStream_t s) : buf(s) {}
};

static void release_record(mp_ctx *c) {
  if (!c->rec) return;
  cudaSetDevice(c->cfg.device);
  delete c->rec;  // waits for the stream, frees the buffers
  c->rec = nullptr;
}

namespace {

// The forward run and the reverse pass on the schedule of plan_schedule /
// revolve: each chunk [n0, n1) is run forward from the live state or a
// checkpoint keeping E (and, for the Sz objective, Bx and By on the plane) of
// every state n0..n1, then stepped back with adj_e / adj_b from n1 - 1 down to
// n0.  The last chunk is reversed straight after the first run reaches it, so
// with one chunk nothing is recomputed.  The reverse phase runs the same
// schedule from the record and skips what the recorded run did (the saves, the
// advances and the forward run of the last chunk), so both phases together do
// what the whole does, in the same order.
template <typename T>
int adjoint_impl(mp_ctx *c, EParams<T> &ep, BParams<T> &bp, const mp_adjoint_config *a, double *J, double *gout[3],
                 AdjPhase phase = kAdjAll) {
  const mp_config &g = c->cfg;
  AdjRecord *rec = phase == kAdjReverse ? c->rec : nullptr;
  if (phase == kAdjReverse && !rec) return set_err(c, MP_ERR_INVALID, "no recorded run");
  if (rec) a = &rec->a;
  const long long Tn = a->steps;
  const auto regions = state_regions(c);
  size_t S = 0;
  for (const auto &r : regions) S += r.second;
  const bool sz = a->kind == MP_OBJ_SZ_PLANE;
  const size_t fbytes = c->fcount * sizeof(T), pbytes = size_t(c->plane) * sizeof(T);
  const size_t H = 3 * fbytes + (sz ? 2 * pbytes : 0);
  long long Kh = 0;  // steps per history chunk
  int slots = 0;     // state checkpoints (the initial state included)
  int nbuf = 1;      // history buffers
  TwoLevel tl;       // segments whose starts go to host memory
  bool two = false;
  if (rec) {
    Kh = rec->Kh;
    slots = rec->slots;
    nbuf = rec->nbuf;
    two = rec->two;
    tl = rec->tl;
  } else {
    if (!plan_schedule(Tn, a->checkpoint_every, a->mem_budget, S, H, &Kh, &slots, &nbuf))
      return set_err(c, MP_ERR_NO_MEMORY,
                     "mem_budget %.4g B holds no schedule (state %zu B per checkpoint, %zu B per step of history)",
                     a->mem_budget, S, H);
    // two levels only under a budget (not with an explicit checkpoint_every)
    two = a->checkpoint_every <= 0 && Kh < Tn &&
          plan_two_level(Tn, a->mem_budget, double(c->host_ckpt.size()) * double(S), S, H,
                         schedule_steps(Tn, Kh, slots), &tl);
    if (two) {
      Kh = tl.Kh;
      slots = tl.slots;
      nbuf = tl.nbuf;
    }
  }
  const long long K = Kh;

  DevBufs buf(c->stream);  // the buffers of this call
  // the forward part's buffers go to the record it makes
  std::unique_ptr<AdjRecord> made(phase == kAdjRecord ? new AdjRecord(c->stream) : nullptr);
  DevBufs &sbuf = made ? made->buf : buf;
  cudaError_t e;
  char *ckpt, *hist[2] = {nullptr, nullptr};
  double *terms;
  if (rec) {
    ckpt = rec->ckpt;
    hist[0] = rec->hist[0];
    hist[1] = rec->hist[1];
    terms = rec->terms;
  } else {
    if ((e = sbuf.alloc(reinterpret_cast<void **>(&ckpt), size_t(slots + 1) * S)) != cudaSuccess ||
        (e = sbuf.alloc(reinterpret_cast<void **>(&hist[0]), size_t(K + 1) * H)) != cudaSuccess ||
        (e = sbuf.alloc(reinterpret_cast<void **>(&terms), (size_t(Tn) + 1) * sizeof(double))) != cudaSuccess)
      return cuda_err(c, e, "checkpoint allocation");
    if (nbuf == 2 && sbuf.alloc(reinterpret_cast<void **>(&hist[1]), size_t(K + 1) * H) != cudaSuccess) {
      cudaGetLastError();  // no room for the second buffer: chunks run forward and back in turn
      nbuf = 1;
    }
  }
  // The reverse pass runs on a second stream: the adjoint kernels of one chunk
  // overlap the forward run of the next, which only shares the history buffer
  // the chunk reads (events order the two).
  struct RevStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fwd[2] = {nullptr, nullptr}, rev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    ~RevStream() {
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
      for (int q = 0; q < 2; ++q) {
        if (fwd[q]) cudaEventDestroy(fwd[q]);
        if (rev[q]) cudaEventDestroy(rev[q]);
      }
    }
  } rs;
  if ((e = cudaStreamCreateWithFlags(&rs.s, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_err(c, e, "cudaStreamCreate");
  for (int q = 0; q < 2; ++q)
    if ((e = cudaEventCreateWithFlags(&rs.fwd[q], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&rs.rev[q], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_err(c, e, "cudaEventCreate");
  int cur = 0;  // history buffer of the chunk being run forward
  AdjParams<T> p = AdjParams<T>();
  for (int q = 0; q < 3 && phase != kAdjRecord; ++q) {
    void *eb, *bb, *gg;
    double *gr;
    if ((e = buf.alloc(&eb, fbytes)) != cudaSuccess || (e = buf.alloc(&bb, fbytes)) != cudaSuccess ||
        (e = buf.alloc(&gg, fbytes)) != cudaSuccess ||
        (e = buf.alloc(reinterpret_cast<void **>(&gr), c->dcells * sizeof(double))) != cudaSuccess)
      return cuda_err(c, e, "adjoint allocation");
    p.Eb[q] = static_cast<T *>(eb);
    p.Bb[q] = static_cast<T *>(bb);
    p.G[q] = static_cast<T *>(gg);
    p.grad[q] = gr;
  }
  for (int s = 0; s < c->np && phase != kAdjRecord; ++s)
    for (int q = 0; q < 3; ++q) {
      void *ps;
      if ((e = buf.alloc(&ps, 2 * c->psi_cells * sizeof(T))) != cudaSuccess) return cuda_err(c, e, "adjoint allocation");
      p.psib[s][q] = static_cast<T *>(ps);
    }
  if (phase != kAdjRecord) {
    void *dp = nullptr;
    if (c->np > 0 && (e = buf.alloc(&dp, c->dcells * c->np * 6 * sizeof(T))) != cudaSuccess)
      return cuda_err(c, e, "adjoint allocation");
    p.dpsi = static_cast<T *>(dp);
  }
  for (int isH = 0; isH < 2 && phase != kAdjRecord; ++isH) {
    const int rc = adj_faces<T>(c, buf, isH != 0, isH ? bp.cpml : ep.cpml, isH ? p.fh : p.fe);
    if (rc != MP_OK) return rc;
  }
  p.nx = g.nx; p.ny = g.ny; p.nz = g.nz;
  p.status = c->d_status;
  p.n_field = (long long)c->fcount;
  p.n_psi = (long long)c->psi_cells;
  p.n_design = (long long)c->dcells;
  {
    // planes per block: about MPB_ADJ_E_BPSM / MPB_ADJ_B_BPSM blocks of 32 x 4
    // columns per SM (measured on the 96^3 adjoint workload, FP32: for adj_e
    // 6 planes per block beat 3 and 2)
    const long long blocks_xy = (long long)((g.nx + 31) / 32) * ((g.ny + 3) / 4);
    const long long ce = std::max(1LL, (148LL * MPB_ADJ_E_BPSM + blocks_xy - 1) / blocks_xy);
    const long long cb = std::max(1LL, (148LL * MPB_ADJ_B_BPSM + blocks_xy - 1) / blocks_xy);
    p.kchunk_e = int(std::max(1LL, (g.nz + ce - 1) / ce));
    p.kchunk_b = int(std::max(1LL, (g.nz + 1 + cb - 1) / cb));
#ifdef MPB_ADJ_KCHUNK
    p.kchunk_e = p.kchunk_b = MPB_ADJ_KCHUNK;
#endif
  }
  p.plane = c->plane;
  p.dt = g.dt;
  for (int q = 0; q < 3; ++q) {
    p.ikE[q] = ep.ik[q];
    p.ikH[q] = bp.ik[q];
  }
  p.ikH_bzy = bp.ik_bz_y;
  for (int s = 0; s < 3; ++s)
    for (int r = 0; r < 2; ++r) {
      p.pD[s][r] = c->coef[0][s][r];
      p.pxi[s][r] = c->coef[1][s][r];
      p.pC[s][r] = c->coef[2][s][r];
    }
  p.sumChi0 = c->sumChi0;
  p.sumXi0 = c->sumXi0;
  p.chi = g.chi;
  p.eps = g.eps;
  p.eps_bg = g.eps_bg;
  {
    const double denom0 = c->mode == MODE_PLRC_LIN ? g.eps + (c->sumChi0 - c->sumXi0) : g.eps + c->sumChi0 - c->sumXi0;
    p.inv_eps_bg = 1.0 / g.eps_bg;
    p.numer0 = g.eps - c->sumXi0;
    p.inv_denom0 = 1.0 / denom0;
    p.A0 = c->mode == MODE_PLRC_NONLIN ? g.chi / denom0 : 0.0;
  }
  p.np = c->np;
  p.mz0 = c->mz0;
  p.mz1 = c->mz1;
  p.nonlin = c->mode == MODE_PLRC_NONLIN;
  p.design = c->dp;
  p.obj_kind = a->kind;
  int b0[6];
  objective_box(a, b0);
  p.ox0 = b0[0]; p.ox1 = b0[1]; p.oy0 = b0[2]; p.oy1 = b0[3]; p.oz0 = b0[4]; p.oz1 = b0[5];
  p.obj_f = a->kind == MP_OBJ_E2_BOX ? 2.0 * g.dt : g.dt * g.dx * g.dy;
  for (int s = 0; s < 3; ++s)
    for (int r = 0; r < 2; ++r) {
      p.pDt[s][r] = T(p.pD[s][r]);
      p.pxit[s][r] = T(p.pxi[s][r]);
      p.pCt[s][r] = T(p.pC[s][r]);
    }
  p.inv_eps_bg_t = T(p.inv_eps_bg);
  p.eps_bg_t = T(p.eps_bg);
  p.numer0_t = T(p.numer0);
  p.inv_denom0_t = T(p.inv_denom0);
  p.chi_nl_t = T(p.nonlin ? p.chi : 0.0);
  p.obj_f_t = T(p.obj_f);

  auto copy_state = [&](long long slot, bool save) -> cudaError_t {
    size_t off = 0;
    for (const auto &r : regions) {
      char *ck = ckpt + size_t(slot) * S + off;
      cudaError_t err = save ? cudaMemcpyAsync(ck, r.first, r.second, cudaMemcpyDeviceToDevice, c->stream)
                             : cudaMemcpyAsync(r.first, ck, r.second, cudaMemcpyDeviceToDevice, c->stream);
      if (err != cudaSuccess) return err;
      off += r.second;
    }
    return cudaSuccess;
  };
  // E of a state into a history slot (copied, or, via ep.hist, stored by the E
  // kernel of the step that produces it); Bx, By on the Sz plane are copied
  auto record = [&](long long slot, bool withE) -> cudaError_t {
    char *h = hist[cur] + size_t(slot) * H;
    for (int q = 0; q < 3 && withE; ++q) {
      cudaError_t err = cudaMemcpyAsync(h + q * fbytes, c->F[q], fbytes, cudaMemcpyDeviceToDevice, c->stream);
      if (err != cudaSuccess) return err;
    }
    if (sz)
      for (int q = 0; q < 2; ++q) {
        const char *src = static_cast<const char *>(c->F[3 + q]) + size_t(b0[4]) * pbytes;
        cudaError_t err = cudaMemcpyAsync(h + 3 * fbytes + q * pbytes, src, pbytes, cudaMemcpyDeviceToDevice, c->stream);
        if (err != cudaSuccess) return err;
      }
    return cudaSuccess;
  };
  auto slot_e = [&](long long slot, int q) {
    return reinterpret_cast<const T *>(hist[cur] + size_t(slot) * H + q * fbytes);
  };
  auto slot_b = [&](long long slot, int q) {
    return sz ? reinterpret_cast<const T *>(hist[cur] + size_t(slot) * H + 3 * fbytes + q * pbytes) : nullptr;
  };
  auto hist_into = [&](long long slot) {
    for (int q = 0; q < 3; ++q) ep.hist[q] = slot < 0 ? nullptr : const_cast<T *>(slot_e(slot, q));
  };
  // The E kernel stores the history where the reverse kernels read it: every
  // cell for the Kerr linearisation, otherwise the design cells (adj_e's E^{n+1}
  // and the gradients) and the objective's box or plane; the other cells of a
  // slot are never read.  (Slot 0 of a chunk is a copy of the whole E.)
  ep.hist_all = p.nonlin;
  const int hb[2][6] = {{c->dp.x0, c->dp.x1, c->dp.y0, c->dp.y1, c->dp.z0, c->dp.z1},
                        {b0[0], b0[1], b0[2], b0[3], b0[4], b0[5]}};
  memcpy(ep.hist_box, hb, sizeof hb);
  // ---- forward and reverse on the checkpoint schedule
  const long long t0 = rec ? rec->t0 : c->time;
  long long reached = 0;  // steps whose objective term is computed
  bool at_end = false;
  bool skipping = rec != nullptr;  // replaying what the recorded run did
  // With a checkpoint at every chunk start and two history buffers, the first
  // run also keeps the history of the chunk before the last, [prev0, last0),
  // in buffer 1: that chunk is then reversed without being run again.
  const bool keep2 = nbuf == 2 && a->checkpoint_every > 0 && !two;
  const long long last0 = ((Tn - 1) / K) * K, prev0 = last0 - K;
  bool prev_kept = false;  // its history is in buffer 1 and not yet reversed
  // Forward steps n0..n1-1 from the live state in one batched call: the E
  // kernel of step n stores the new E into history slot n + 1 - h0 when
  // n >= h0 (h0 < 0: no history), the Sz planes are copied after it, and the
  // objective term of every step not run before goes to terms[n].
  auto run = [&](long long n0, long long n1, long long h0) -> int {
    StepHooks hk;
    hk.before = [&](long long q) {
      const long long n = n0 + q;
      hist_into(h0 >= 0 && n >= h0 ? n + 1 - h0 : -1);
      return MP_OK;
    };
    hk.after = [&](long long q) {
      const long long n = n0 + q;
      if (h0 >= 0 && n >= h0 && sz) {
        const cudaError_t err = record(n + 1 - h0, false);
        if (err != cudaSuccess) return cuda_err(c, err, "history copy");
      }
      return n >= reached ? objective_term<T>(c, a, terms + n) : MP_OK;
    };
    const int r = step_impl<T>(c, ep, bp, int(n1 - n0), nullptr, nullptr, &hk);
    hist_into(-1);
    reached = std::max(reached, n1);
    return r;
  };
  RevolveOps ops;
  ops.restore = [&](long long at, int slot) -> int {
    if (skipping || (prev_kept && at == prev0)) return MP_OK;
    const cudaError_t err = copy_state(slot, false);
    c->time = t0 + at;
    return err == cudaSuccess ? MP_OK : cuda_err(c, err, "checkpoint restore");
  };
  ops.save = [&](long long, int slot) -> int {
    if (skipping) return MP_OK;
    const cudaError_t err = copy_state(slot, true);
    return err == cudaSuccess ? MP_OK : cuda_err(c, err, "checkpoint copy");
  };
  ops.advance = [&](long long from, long long to) -> int {
    // the first run's advance to the last chunk runs the chunk before it
    // into history buffer 1
    const bool split = keep2 && !at_end && to == last0 && from <= prev0;
    if (split) prev_kept = true;
    if (skipping) {
      reached = std::max(reached, to);
      return MP_OK;
    }
    NvtxRange nv("mp_adjoint forward");
    const long long mid = split ? prev0 : to;
    int r = mid > from ? run(from, mid, -1) : MP_OK;
    if (r != MP_OK || !split) return r;
    cur = 1;
    const cudaError_t err = record(0, true);
    r = err == cudaSuccess ? run(prev0, to, prev0) : cuda_err(c, err, "history copy");
    cur = 0;
    return r;
  };
  ops.leaf = [&](long long n0, long long n1) -> int {
    NvtxRange nv("mp_adjoint chunk");
    cudaError_t err;
    const bool first = n1 == Tn && !at_end;
    if (prev_kept && n0 == prev0) {
      // its history is in buffer 1 from the first run (the buffer the last
      // chunk's reverse pass left next)
      if (cur != 1 || rs.used[1]) return set_err(c, MP_ERR_INVALID, "kept history out of order");
      prev_kept = false;
    } else if (skipping) {
      // the recorded run ended with this chunk's forward run: its history is
      // in buffer 0, J and the final state are kept
      if (!first || cur != 0) return set_err(c, MP_ERR_INVALID, "recorded schedule does not replay");
      skipping = false;
      at_end = true;
      reached = Tn;
      if (J) *J = rec->J;
    } else {
      // the buffer is free once the reverse pass of the chunk that used it is done
      if (rs.used[cur] && (err = cudaStreamWaitEvent(c->stream, rs.rev[cur], 0)) != cudaSuccess)
        return cuda_err(c, err, "cudaStreamWaitEvent");
      if ((err = record(0, true)) != cudaSuccess) return cuda_err(c, err, "history copy");
      int r = run(n0, n1, n0);
      if (r != MP_OK) return r;
      if (first) {
        // the first time the run reaches the end: J, the final state
        at_end = true;
        if ((err = copy_state(slots, true)) != cudaSuccess) return cuda_err(c, err, "checkpoint copy");
        if ((r = read_sum(c, terms, Tn, J)) != MP_OK || (r = mp_check_status(c)) != MP_OK) return r;
        if (phase == kAdjRecord) return kAdjStop;
      }
    }
    if ((err = cudaEventRecord(rs.fwd[cur], c->stream)) != cudaSuccess ||
        (err = cudaStreamWaitEvent(rs.s, rs.fwd[cur], 0)) != cudaSuccess)
      return cuda_err(c, err, "event");
    if (first) {
      // the start of the adjoint
      for (int q = 0; q < 3; ++q) p.En[q] = slot_e(n1 - n0, q);
      p.obx = slot_b(n1 - n0, 0);
      p.oby = slot_b(n1 - n0, 1);
      if ((err = launch_adj_init<T>(p, rs.s)) != cudaSuccess) return cuda_err(c, err, "adjoint init kernel");
      c->launches++;
    }
    for (long long n = n1 - 1; n >= n0; --n) {
      for (int q = 0; q < 3; ++q) {
        p.En[q] = slot_e(n - n0, q);
        p.En1[q] = slot_e(n - n0 + 1, q);
      }
      p.obx = slot_b(n - n0, 0);
      p.oby = slot_b(n - n0, 1);
      p.add_obj = n >= 1;
      // adj_e, then adj_b with the step's design gradients, chained by
      // programmatic dependent launch
      if ((err = launch_adj_e<T>(p, rs.s)) != cudaSuccess) return cuda_err(c, err, "adjoint E kernel");
      if ((err = launch_adj_b<T>(p, rs.s)) != cudaSuccess) return cuda_err(c, err, "adjoint B kernel");
      c->launches += 2;
    }
    if ((err = cudaEventRecord(rs.rev[cur], rs.s)) != cudaSuccess) return cuda_err(c, err, "event");
    rs.used[cur] = true;
    cur = (cur + 1) % nbuf;
    return MP_OK;
  };
  long long live = 0;
  // the whole schedule, on one level or two (kAdjStop: the forward part is done)
  auto run_schedule = [&]() -> int {
    if (!two) {
      if (!skipping && (e = copy_state(0, true)) != cudaSuccess) return cuda_err(c, e, "checkpoint copy");
      std::vector<int> free_slots;
      for (int q = slots - 1; q >= 1; --q) free_slots.push_back(q);
      return revolve(0, Tn, 0, free_slots, K, ops, live);
    }
    // the live state to / from the host copy of segment k, on the stream
    auto host_copy = [&](long long k, bool save) -> cudaError_t {
      size_t off = 0;
      for (const auto &r : regions) {
        char *hc = static_cast<char *>(c->host_ckpt[size_t(k)]) + off;
        cudaError_t err = save ? cudaMemcpyAsync(hc, r.first, r.second, cudaMemcpyDeviceToHost, c->stream)
                               : cudaMemcpyAsync(r.first, hc, r.second, cudaMemcpyHostToDevice, c->stream);
        if (err != cudaSuccess) return err;
        off += r.second;
      }
      return cudaSuccess;
    };
    int r;
    // first run: the start of every segment to host memory
    for (long long k = 0; k < tl.nseg; ++k) {
      if (!skipping && (e = host_copy(k, true)) != cudaSuccess) return cuda_err(c, e, "host checkpoint copy");
      if (k + 1 < tl.nseg && (r = ops.advance(k * tl.L, (k + 1) * tl.L)) != MP_OK) return r;
      live = k * tl.L + (k + 1 < tl.nseg ? tl.L : 0);
    }
    // segments last first, each from its host copy on the device schedule
    for (long long k = tl.nseg - 1; k >= 0; --k) {
      const long long a0 = k * tl.L, a1 = std::min(Tn, a0 + tl.L);
      if (live != a0) {
        if ((e = host_copy(k, false)) != cudaSuccess) return cuda_err(c, e, "host checkpoint restore");
        c->time = t0 + a0;
        live = a0;
      }
      if (!skipping && (e = copy_state(0, true)) != cudaSuccess) return cuda_err(c, e, "checkpoint copy");
      std::vector<int> free_slots;
      for (int q = slots - 1; q >= 1; --q) free_slots.push_back(q);
      if ((r = revolve(a0, a1, 0, free_slots, K, ops, live)) != MP_OK) return r;
    }
    return MP_OK;
  };
  const int rc = run_schedule();
  if (phase == kAdjRecord) {
    if (rc != kAdjStop) return rc == MP_OK ? set_err(c, MP_ERR_INVALID, "the run did not reach its end") : rc;
    // the live state is the end state at time t0 + Tn; J is read
    made->a = *a;
    made->t0 = t0;
    made->J = *J;
    made->Kh = Kh;
    made->slots = slots;
    made->nbuf = nbuf;
    made->two = two;
    made->tl = tl;
    made->ckpt = ckpt;
    made->hist[0] = hist[0];
    made->hist[1] = hist[1];
    made->terms = terms;
    c->rec = made.release();
    return MP_OK;
  }
  if (rc != MP_OK) return rc;
  if ((e = cudaStreamSynchronize(rs.s)) != cudaSuccess) return cuda_err(c, e, "adjoint");
  if ((e = copy_state(slots, false)) != cudaSuccess) return cuda_err(c, e, "checkpoint restore");
  c->time = t0 + Tn;
  for (int q = 0; q < 3; ++q)
    if (gout[q] && (e = cudaMemcpyAsync(gout[q], p.grad[q], c->dcells * sizeof(double), cudaMemcpyDeviceToHost,
                                        c->stream)) != cudaSuccess)
      return cuda_err(c, e, "gradient read");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return cuda_err(c, e, "adjoint");
  return mp_check_status(c);
}

}  // namespace

extern "C" {

int mp_objective(mp_ctx *c, const mp_adjoint_config *a, double *J) {
  if (!c || !a || !J) return MP_ERR_INVALID;
  int rc = check_objective(c, a);
  if (rc != MP_OK) return rc;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  return c->fp32 ? objective_impl<float>(c, c->epf, c->bpf, a, J) : objective_impl<double>(c, c->epd, c->bpd, a, J);
}

}  // extern "C"

namespace {
// What the adjoint needs of the context and the objective.
int adjoint_supported(mp_ctx *c, const mp_adjoint_config *a) {
  int rc = check_objective(c, a);
  if (rc != MP_OK) return rc;
  if (c->mode != MODE_PLRC_LIN && c->mode != MODE_PLRC_NONLIN)
    return set_err(c, MP_ERR_UNSUPPORTED, "mp_adjoint needs a PLRC solver");
  if (c->plasma[0]) return set_err(c, MP_ERR_UNSUPPORTED, "the adjoint of the plasma plug-ins is not built");
  if (c->cfg.boundary != MP_BOUNDARY_XY_PERIODIC)
    return set_err(c, MP_ERR_UNSUPPORTED, "mp_adjoint needs the xy-periodic boundary");
  if (!c->design) return set_err(c, MP_ERR_INVALID, "mp_adjoint needs a design region (mp_config.design_box)");
  if (c->tma) return set_err(c, MP_ERR_UNSUPPORTED, "mp_adjoint uses the global-load kernels");
  return MP_OK;
}
}  // namespace

extern "C" {

int mp_adjoint(mp_ctx *c, const mp_adjoint_config *a, double *J, double *grad_eps, double *grad_deps_scale,
               double *grad_chi_scale) {
  if (!c || !a || !J) return MP_ERR_INVALID;
  NvtxRange nv("mp_adjoint");
  int rc = adjoint_supported(c, a);
  if (rc != MP_OK) return rc;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  double *g[3] = {grad_eps, grad_deps_scale, grad_chi_scale};
  return c->fp32 ? adjoint_impl<float>(c, c->epf, c->bpf, a, J, g) : adjoint_impl<double>(c, c->epd, c->bpd, a, J, g);
}

int mp_objective_record(mp_ctx *c, const mp_adjoint_config *a, double *J) {
  if (!c || !a || !J) return MP_ERR_INVALID;
  NvtxRange nv("mp_objective_record");
  int rc = adjoint_supported(c, a);
  if (rc != MP_OK) return rc;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  double *g[3] = {nullptr, nullptr, nullptr};
  return c->fp32 ? adjoint_impl<float>(c, c->epf, c->bpf, a, J, g, kAdjRecord)
                 : adjoint_impl<double>(c, c->epd, c->bpd, a, J, g, kAdjRecord);
}

int mp_adjoint_reverse(mp_ctx *c, double *J, double *grad_eps, double *grad_deps_scale, double *grad_chi_scale) {
  if (!c) return MP_ERR_INVALID;
  NvtxRange nv("mp_adjoint_reverse");
  if (!c->rec)
    return set_err(c, MP_ERR_INVALID,
                   "mp_adjoint_reverse: no recorded run (mp_objective_record; calls that change the state release it)");
  cudaSetDevice(c->cfg.device);
  double *g[3] = {grad_eps, grad_deps_scale, grad_chi_scale};
  const int rc = c->fp32 ? adjoint_impl<float>(c, c->epf, c->bpf, nullptr, J, g, kAdjReverse)
                         : adjoint_impl<double>(c, c->epd, c->bpd, nullptr, J, g, kAdjReverse);
  release_record(c);
  return rc;
}

int mp_release_record(mp_ctx *c) {
  if (!c) return MP_ERR_INVALID;
  release_record(c);
  return MP_OK;
}

int mp_set_host_checkpoint_budget(mp_ctx *c, double bytes) {
  if (!c) return MP_ERR_INVALID;
  if (!(bytes >= 0) || !std::isfinite(bytes)) return set_err(c, MP_ERR_INVALID, "host checkpoint budget %g", bytes);
  cudaSetDevice(c->cfg.device);
  release_record(c);
  free_host_ckpt(c);
  size_t S = 0;
  for (const auto &r : state_regions(c)) S += r.second;
  const long long n = S ? (long long)std::floor(bytes / double(S)) : 0;
  // Each buffer: 2 MB-aligned memory marked for transparent huge pages, its
  // pages faulted in by one thread per buffer (the host kernel zeroes them in
  // parallel), then registered with the driver (fewer, larger pages to pin;
  // cudaHostAlloc of 115 GB took 44-50 s).
  const size_t align = size_t(2) << 20, len = (S + align - 1) / align * align;
  std::vector<void *> bufs(size_t(n), nullptr);
  std::vector<std::thread> th;
  for (long long k = 0; k < n; ++k)
    th.emplace_back([&, k] {
      void *p = std::aligned_alloc(align, len);
      if (!p) return;
      madvise(p, len, MADV_HUGEPAGE);
      std::memset(p, 0, len);
      bufs[size_t(k)] = p;
    });
  for (auto &t : th) t.join();
  long long k = 0;
  cudaError_t e = cudaSuccess;
  for (; k < n && bufs[size_t(k)]; ++k)
    if ((e = cudaHostRegister(bufs[size_t(k)], len, cudaHostRegisterDefault)) != cudaSuccess) break;
  if (k < n) {
    cudaGetLastError();
    for (long long q = 0; q < n; ++q) {
      if (q < k) cudaHostUnregister(bufs[size_t(q)]);
      std::free(bufs[size_t(q)]);
    }
    return set_err(c, MP_ERR_NO_MEMORY, "pinned host memory for checkpoint %lld of %lld (%zu B each): %s", k, n, S,
                   e != cudaSuccess ? cudaGetErrorString(e) : "allocation failed");
  }
  c->host_ckpt = bufs;
  return MP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// mp_state_size / mp_save_state / mp_load_state

namespace {

struct StateHeader {
  char magic[8];  // "MPB200ST"
  int abi_version, precision, solver, boundary, cpml, cpml_d;
  int nx, ny, nz, mz0, mz1, np, nregions;
  long long time;
  unsigned long long payload;
};

void fill_header(const mp_ctx *c, const std::vector<std::pair<void *, size_t>> &regions, StateHeader &h) {
  memset(&h, 0, sizeof h);
  memcpy(h.magic, "MPB200ST", 8);
  h.abi_version = MP_ABI_VERSION;
  h.precision = c->cfg.precision;
  h.solver = c->cfg.solver;
  h.boundary = c->cfg.boundary;
  h.cpml = c->cfg.cpml;
  h.cpml_d = c->cfg.cpml_d;
  h.nx = c->cfg.nx;
  h.ny = c->cfg.ny;
  h.nz = c->cfg.nz;
  h.mz0 = c->mz0;
  h.mz1 = c->mz1;
  h.np = c->np;
  h.nregions = int(regions.size());
  h.time = c->time;
  for (const auto &r : regions) h.payload += r.second;
}

}  // namespace

extern "C" {

int mp_state_size(mp_ctx *c, size_t *bytes) {
  if (!c || !bytes) return MP_ERR_INVALID;
  StateHeader h;
  fill_header(c, state_regions(c), h);
  *bytes = sizeof(StateHeader) + size_t(h.payload);
  return MP_OK;
}

int mp_save_state(mp_ctx *c, void *host, size_t bytes) {
  if (!c || !host) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  const auto regions = state_regions(c);
  StateHeader h;
  fill_header(c, regions, h);
  if (bytes != sizeof h + size_t(h.payload))
    return set_err(c, MP_ERR_INVALID, "state buffer of %zu bytes, expected %zu", bytes, sizeof h + size_t(h.payload));
  memcpy(host, &h, sizeof h);
  char *dst = static_cast<char *>(host) + sizeof h;
  for (const auto &r : regions) {
    cudaError_t e = cudaMemcpyAsync(dst, r.first, r.second, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "state copy");
    dst += r.second;
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? MP_OK : cuda_err(c, e, "state copy");
}

int mp_load_state(mp_ctx *c, const void *host, size_t bytes) {
  if (!c || !host) return MP_ERR_INVALID;
  cudaSetDevice(c->cfg.device);
  release_record(c);
  const auto regions = state_regions(c);
  StateHeader want, got;
  fill_header(c, regions, want);
  if (bytes < sizeof got) return set_err(c, MP_ERR_INVALID, "state buffer too short");
  memcpy(&got, host, sizeof got);
  want.time = got.time;
  if (memcmp(&want, &got, sizeof got) != 0 || bytes != sizeof got + size_t(got.payload))
    return set_err(c, MP_ERR_INVALID, "state buffer does not match this context (grid, precision, solver, "
                                      "boundary, CPML or medium differ)");
  const char *src = static_cast<const char *>(host) + sizeof got;
  for (const auto &r : regions) {
    cudaError_t e = cudaMemcpyAsync(r.first, src, r.second, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_err(c, e, "state copy");
    src += r.second;
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "state copy");
  c->time = got.time;
  return MP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// mp_initialize, mp_follow_max

namespace mpb {
template <typename T> cudaError_t launch_init(const InitParams &, void *const[6], cudaStream_t);
template <typename T>
cudaError_t launch_follow_max(const void *, int, int, int, long long, int, const int[3], int *, double *,
                              cudaStream_t);
}  // namespace mpb

extern "C" {

void mp_init_defaults(int kind, mp_init *q) {
  if (!q) return;
  memset(q, 0, sizeof(*q));
  q->kind = kind;
  for (int a = 0; a < 3; ++a) {
    q->k[a] = 1.0;  // k / kx ky kz (pulseinit.cpp:79, gaussinit.cpp:87-89, waveinit.cpp:65-67)
    q->B[a] = 1.0;  // Bx By Bz
  }
  q->r0 = q->z0 = q->zc = q->C = 1.0;  // pulseinit.cpp:80-83
  q->eps = 1.0;                        // waveinit.cpp:71
  q->bound = 0;                        // pulseinit.cpp:86
}

int mp_initialize(mp_ctx *c, const mp_init *q) {
  if (!c || !q) return MP_ERR_INVALID;
  release_record(c);
  const mp_config &g = c->cfg;
  InitParams p;
  memset(&p, 0, sizeof p);
  p.kind = q->kind;
  p.nx = g.nx; p.ny = g.ny; p.nz = g.nz;
  p.plane = c->plane;
  p.dx = g.dx; p.dy = g.dy; p.dz = g.dz;
  // Globals::gridLow / gridHigh are 0 and n + 1 per axis (globals.cpp:44-45)
  p.xh = 0.5 * double(g.nx + 1);
  p.yh = 0.5 * double(g.ny + 1);
  p.zh = 0.5 * double(g.nz + 1);
  if (q->kind == MP_INIT_PULSE) {
    // GaussPulseInit::init (pulseinit.cpp:7-31)
    p.ex = q->B[1];
    p.ey = -q->B[0];
    p.bx = q->B[0];
    p.by = q->B[1];
    p.kz = q->k[2];
    p.r0 = q->r0; p.z0 = q->z0; p.zc = q->zc; p.C = q->C;
    p.k_lo = q->bound;
    p.k_hi = g.nz + 1 - q->bound;
  } else if (q->kind == MP_INIT_PLANE_GAUSS || q->kind == MP_INIT_WAVE) {
    // PlaneGaussPulseInit::init (gaussinit.cpp:7-41), PlaneWaveInit::init (waveinit.cpp:9-36):
    // kx, ky, kz are int parameters in MPulse
    const int kx = int(q->k[0]), ky = int(q->k[1]), kz = int(q->k[2]);
    const double bx = q->B[0], by = q->B[1], bz = q->B[2];
    double ex = ky * bz - kz * by, ey = kz * bx - kx * bz, ez = kx * by - ky * bx;
    const double bmag = std::sqrt(bx * bx + by * by + bz * bz);
    const double factor = -bmag / std::sqrt(ex * ex + ey * ey + ez * ez);
    if (q->kind == MP_INIT_PLANE_GAUSS) {
      ex *= factor; ey *= factor; ez *= factor;
      p.kx = kx / double(g.nx);
      p.ky = ky / double(g.ny);
      p.kz = kz / double(g.nz);
      p.k_lo = 12;  // offsetz (gaussinit.cpp:42)
      p.k_hi = g.nz + 1 - 12;
    } else {
      if (!(q->eps > 0)) return set_err(c, MP_ERR_INVALID, "wave_init: eps must be positive");
      ex *= factor / std::sqrt(q->eps);
      ey *= factor / std::sqrt(q->eps);
      ez *= factor / std::sqrt(q->eps);
      p.kx = 2 * M_PI * kx / double(g.nx);
      p.ky = 2 * M_PI * ky / double(g.ny);
      p.kz = 2 * M_PI * kz / double(g.nz);
      p.k_lo = 0;
      p.k_hi = g.nz + 1;
    }
    p.ex = ex; p.ey = ey; p.ez = ez;
    p.bx = bx; p.by = by; p.bz = bz;
  } else {
    return set_err(c, MP_ERR_INVALID, "unknown initialiser kind %d", q->kind);
  }
  p.k_lo = std::max(p.k_lo, 0);
  p.k_hi = std::min(p.k_hi, g.nz + 1);
  cudaSetDevice(g.device);
  cudaError_t e = c->fp32 ? launch_init<float>(p, c->F, c->stream) : launch_init<double>(p, c->F, c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "initialiser kernel");
  c->launches++;
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? MP_OK : cuda_err(c, e, "initialiser");
}

int mp_follow_max(mp_ctx *c, const char *field, int dim, const int pos[3], int *ipos, double *position) {
  if (!c || !field || !pos || !ipos || !position) return MP_ERR_INVALID;
  static const char *fn[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};
  int f = -1;
  for (int q = 0; q < 6; ++q)
    if (!strcmp(field, fn[q])) f = q;
  if (f < 0) return set_err(c, MP_ERR_NAME, "follow_max: unknown field '%s'", field);
  const mp_config &g = c->cfg;
  const int n3[3] = {g.nx, g.ny, g.nz};
  if (dim < 0 || dim > 2) return set_err(c, MP_ERR_INVALID, "follow_max: dim must be 0, 1 or 2");
  if (pos[0] < 1 || pos[0] > g.nx || pos[1] < 1 || pos[1] > g.ny || pos[2] < 0 || pos[2] > g.nz + 1)
    return set_err(c, MP_ERR_INVALID, "follow_max: position outside the stored cells");
  if (*ipos < 1 || *ipos > n3[dim]) return set_err(c, MP_ERR_INVALID, "follow_max: start index outside 1..%d", n3[dim]);
  cudaSetDevice(g.device);
  // the diagnostics scratch: the start index in, the result out
  int *d_ip = reinterpret_cast<int *>(c->d_diag);
  double *d_out = c->d_diag + 1;
  cudaError_t e = cudaMemcpyAsync(d_ip, ipos, sizeof(int), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = c->fp32 ? launch_follow_max<float>(c->F[f], g.nx, g.ny, g.nz, c->plane, dim, pos, d_ip, d_out, c->stream)
                : launch_follow_max<double>(c->F[f], g.nx, g.ny, g.nz, c->plane, dim, pos, d_ip, d_out, c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "follow_max kernel");
  c->launches++;
  e = cudaMemcpyAsync(c->h_diag, c->d_diag, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_err(c, e, "follow_max read");
  memcpy(ipos, c->h_diag, sizeof(int));
  *position = c->h_diag[1];
  return MP_OK;
}

}  // extern "C"
