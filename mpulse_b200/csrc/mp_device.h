// mp_device.h - launch parameters shared by the host side (mp_api.cu) and the
// kernels (mp_step_kernels.cu, mp_source_kernels.cu).
//
// Device data layout ("plane layout", identical to the host buffers of
// include/mpulse_b200.h): every full-size array holds nz+2 z-planes
// k = 0 .. nz+1 (MPulse's global z index) of ny*nx interior cells, x fastest:
//     a[(k * ny + (j-1)) * nx + (i-1)]
// x and y are periodic in every boundary MPulse supports on one process, so
// their ghost cells are index wraps; the z ghost planes are stored because the
// xy-periodic boundary keeps them as state (E at 0 and nz+1 stay fixed, B at 0
// is updated every step, periodic_bound.cpp:129-130).
#ifndef MPB_MP_DEVICE_H
#define MPB_MP_DEVICE_H

#include <cuda.h>  // CUtensorMap (a type only; no driver call is linked)

#include <cstddef>
#include <cstdint>

namespace mpb {

enum Mode { MODE_PLAIN = 0, MODE_NL = 1, MODE_PLRC_LIN = 2, MODE_PLRC_NONLIN = 3 };

enum Face { FACE_NORTH = 0, FACE_SOUTH, FACE_WEST, FACE_EAST, FACE_UP, FACE_DOWN };

// Device status word, read back after mp_step.
// ST_BOUNDS counts the accesses a checked build (MPB_CHECKED=1) found outside
// their array and skipped.
enum StatusSlot { ST_NEWTON = 0, ST_NONFINITE = 1, ST_TIMEOUT = 2, ST_BOUNDS = 3, ST_COUNT = 4 };

// Tile of the TMA-staged kernels (mp_step_tma.cu): 32 x 8 columns.
static const int kTmaTileX = 32, kTmaTileY = 8;

// Tensor maps of the TMA-staged kernels, one per array and halo shape.
struct ETmaMaps {
  CUtensorMap bx, by, bz, ex, ey, ez;
  CUtensorMap psi[3][3];
};
struct BTmaMaps {
  CUtensorMap ex, ey, ez, bx, by, bz;
};

// One CPML current (CPMLBorderECurrent / CPMLBorderHCurrent,
// cpml_border.cpp:345-527) restricted to the cells the kernels update.  Its two
// psi arrays cover the box [lo, hi] (MPulse indices); along `dim` the box is the
// layer, across it the whole interior.  Index within the box, x fastest.
template <typename T>
struct CpmlFace {
  int active;
  int dim;          // 0 x, 1 y, 2 z
  int lo, hi;       // extent along dim (inclusive)
  int zlo;          // first z plane of the box (for x/y faces)
  int ex, ey;       // box extents in x and y (for the index)
  T *psi0, *psi1;   // psi components as in cpml_border.cpp:361-383 / :460-482
  int n;            // elements of psi0 / psi1 (checked builds test indices against it)
  const T *b;       // b coefficient per index along dim (full axis length)
  const T *c;       // c / Delta per index along dim
};

// One incident-source plane: the J (E side) or M (H side) values of the two
// transverse components of one TF/SF current (incsource.t:40-73, :112-145).
template <typename T>
struct SourcePlane {
  int plane;        // MPulse z index the current lives on
  const T *v0;      // component transverse1 (x)
  const T *v1;      // component transverse2 (y)
};

// Per-cell design parameters (mp_config.design_box): eps_infinity, a factor
// on every pole's Delta epsilon and a factor on chi, box-sized FP64 maps with x
// fastest.  x0..x1, y0..y1 are 0-based interior indices, z0..z1 MPulse planes.
struct DesignParams {
  int x0, x1, y0, y1, z0, z1;  // inclusive; x0 > x1: no design region
  int bx, by;                  // box extents in x and y
  const double *eps, *dscale, *chiscale;
  double pD[3][2], pxi[3][2];  // dchi0 - dxi0 and dxi0 of the active poles, FP64
  double sumChi0, sumXi0, chi;
  int lin;                     // PLRC_LIN: denominator eps + (sumChi0 - sumXi0)
};

template <typename T>
struct EParams {
  int nx, ny, nz;
  long long plane;        // nx * ny
  T *E[3];
  const T *B[3];
  int k_first, k_last;    // planes updated (1..nz, or 1..nz+1 for plain / NL)
  int zperiodic;
  int kchunk;             // planes per block
  T dt;
  // FP32 form: the rounding error of dt, numer and inv_denom as floats
  // (x - float(x)), so that the updates apply the FP64 coefficients (hi + lo)
  // and the FP32 rounding of the coefficients does not add up step after
  // step; zero in the FP64 form
  T dt_lo, numer_lo, inv_denom_lo;

  // PLRC (fdtd_plrc.t:198-216), active poles only, in T; psi is complex
  // (re, im interleaved) over the medium planes mz0..mz1.
  int mz0, mz1;
  T *psi[3][3];           // [pole][component] -> pairs
  T pD[3][2];             // dchi0 - dxi0
  T pxi[3][2];            // dxi0
  T pC[3][2];             // Crec
  T numer, inv_denom;     // medium
  T eps_bg, inv_eps_bg;   // background
  double chi_over_denom;  // Kerr A (PLRC nonlinear)
  double eps_d, chi_d;    // fdtd_nl
  T chi;                  // Kerr chi in the constitutive term
  double newton_tol;
  int newton_max;

  const T *ik[3];         // 1 / (kappa_E * d) per index, per axis

  CpmlFace<T> cpml[6];    // E-side CPML currents in MPulse's current order
  DesignParams design;
  T *hist[3];             // with a design region: also store the new E here (adjoint history), if set
  // the cells whose history the reverse pass reads: all (hist_all) or those in
  // either box (0-based x0, x1, y0, y1, MPulse z0, z1; x0 > x1: empty)
  int hist_all;
  int hist_box[2][6];
  int n_src;
  int src_mult;           // how many injectors share the plane (each adds it once)
  SourcePlane<T> src[4];
  int *status;
  unsigned long long *kerr_count;  // [0] Kerr solves, [1] their Newton iterations (accumulated)
  long long n_field;      // elements of each field and history array
  long long n_psi;        // pairs of each PLRC accumulator array

  // Plasma plug-ins: PlasmaDensity (plasmadensity.cpp:18-49) and PlasmaCurrent
  // (plasmacurrent.cpp:42-74), state in the field layout (planes 1..nz used);
  // rho == nullptr: no plasma
  T *rho, *pj[3];
  int pl_density, pl_current;
  int pl_km;                        // K - 1
  T pl_n, pl_m, pl_w;               // dt nu / 2, dt mpa, mpa Wion
  T pl_gdtn, pl_gdtd, pl_emdt, pl_rho_bg;  // 1 - gamma dt / 2, 1 + gamma dt / 2, em dt, rho_bg
  T denom_t;                        // the medium's denominator without the conductivity
  double denom_d, chi_raw;          // the same in FP64, and chi
};

template <typename T>
struct BParams {
  int nx, ny, nz;
  long long plane;
  const T *E[3];
  T *B[3];
  int k_first, k_last;    // 0..nz (xy periodic) or 1..nz (periodic)
  int zperiodic;
  int kchunk;
  T dt, dt_lo;            // dt_lo as in EParams
  const T *ik[3];         // 1 / (kappa_H * d)
  const T *ik_bz_y;       // line used for dEx/dy in the Bz update
  CpmlFace<T> cpml[6];
  int n_src;
  int src_mult;           // how many injectors share the plane (each adds it once)
  SourcePlane<T> src[4];
  int *status;
  long long n_field;      // elements of each field array
};

// ---------------------------------------------------------------------------
// Adjoint (mp_adjoint): the discrete adjoint of one PLRC step, run backwards.

// The adjoint totals of the CPML faces along one axis: for an E face the
// adjoint of its psi after the E half plus dt times the adjoint of the E
// numerator component it feeds; for an H face the adjoint of its psi after the
// B half plus dt times the adjoint of the B component it feeds.  The low and
// the high face of the axis share the entry (their layers must not overlap):
// positions lo0..hi0 map to 0..n0-1 and lo1..hi1 to n0.. (lo1 > hi1: one
// face).  Layout like CpmlFace with the merged extent along the axis: z
// entries [pos][ny][nx]; x entries [k - zlo][ny][ex]; y entries [k - zlo][ey][nx].
template <typename T>
struct AdjFace {
  int active, lo0, hi0, lo1, hi1, n0, zlo, ex, ey;
  T *a0, *a1;
  long long n;     // elements of a0 / a1
  const T *b, *c;  // b and c / Delta along the axis (full axis length, both faces)
};

template <typename T>
struct AdjParams {
  int nx, ny, nz;
  long long plane;
  double dt;
  T *Eb[3], *Bb[3];       // adjoint of E and B (full plane layout)
  T *G[3];                // adjoint of the E numerator of the step (planes 1..nz; 0 elsewhere)
  T *psib[3][3];          // adjoint of the PLRC accumulators, pairs over planes mz0..mz1
  const T *En[3];         // E before the step
  const T *En1[3];        // E after the step
  const T *ikE[3], *ikH[3], *ikH_bzy;
  double pD[3][2], pxi[3][2], pC[3][2];  // active poles, FP64
  double sumChi0, sumXi0, chi, eps, eps_bg;
  double inv_eps_bg, numer0, inv_denom0, A0;  // background and uniform-medium constants
  // the same constants rounded to the state precision once (cells outside the
  // design region use these; no per-cell conversions)
  T pDt[3][2], pxit[3][2], pCt[3][2];
  T inv_eps_bg_t, eps_bg_t, numer0_t, inv_denom0_t, chi_nl_t, obj_f_t;
  int np, mz0, mz1, nonlin;
  int kchunk_e, kchunk_b;  // planes per block of adj_e (1..nz) / adj_b (0..nz)
  AdjFace<T> fe[3], fh[3];  // per axis x, y, z
  DesignParams design;
  double *grad[3];        // dJ/d eps, dJ/d Delta-eps factor, dJ/d chi factor (box-sized, FP64)
  // objective term of the state before the step (added when add_obj)
  int obj_kind, add_obj;
  int ox0, ox1, oy0, oy1, oz0, oz1;  // 0-based x/y, MPulse z
  double obj_f;           // 2 dt (E^2 box) or dt dx dy (Sz plane)
  const T *obx, *oby;     // Bx, By of that state on the Sz plane (plane-sized)
  int *status;            // the context's status word
  long long n_field, n_psi, n_design;  // elements of a field array, pairs of a PLRC array, design cells
  // the PLRC accumulator adjoints of the design cells before the step's E
  // half, saved by adj_e for adj_grad: box-sized, [cell][pole][component][re, im]
  T *dpsi;
};

// Field initialisers (mp_init_kernels.cu).
struct InitParams {
  int kind, nx, ny, nz;
  long long plane;
  double dx, dy, dz;
  double ex, ey, ez, bx, by, bz;  // amplitudes after the reference's normalisation
  double kx, ky, kz;              // pulse_init: kz; gauss_init / wave_init: the scaled nk*
  double r0, z0, zc, C;
  double xh, yh, zh;              // grid centre (MPulse index)
  int k_lo, k_hi;                 // planes written
};

// Incident-source plane evaluation.
struct SourceEvalParams {
  int kind;               // mp_source_kind
  int nx, ny;
  int isH;                // 0: getHField for the E current, 1: getEField for the H current
  int l;                  // z argument of getHField / getEField
  long long time;         // Process::time
  double dx, dy, dz, dt, DX;
  // plane sources
  double k[3], amp3[3], bg[3], om, ramp, width, offset;
  // short pulse
  double lightspeed, ZRl, amp, phase, tshift, zshift, length, om0;
  double sp_eiphi[2], sp_emip[2], sp_g;  // exp(2 i phase), exp(-i phase), exp(-(om0 length / 2)^2)
  double centre[3];
  const double *w_coef;   // Faddeeva expansion coefficients (highest power first)
  double w_L;
  // gauss_inject: the planes [Nt][ny][nx] of the block that starts at g_toff
  // (getHField: Bx in g_f1; getEField: Ex in g_f1, Ey in g_f2), scaled by
  // g_scale; zero fields while g_active is 0
  const double *g_f1, *g_f2;
  double g_scale;
  long long g_toff;
  int g_active;
};

}  // namespace mpb

#endif
