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
enum StatusSlot { ST_NEWTON = 0, ST_NONFINITE = 1, ST_TIMEOUT = 2, ST_COUNT = 4 };

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
  int n_src;
  int src_mult;           // how many injectors share the plane (each adds it once)
  SourcePlane<T> src[4];
  int *status;
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
  T dt;
  const T *ik[3];         // 1 / (kappa_H * d)
  const T *ik_bz_y;       // line used for dEx/dy in the Bz update
  CpmlFace<T> cpml[6];
  int n_src;
  int src_mult;           // how many injectors share the plane (each adds it once)
  SourcePlane<T> src[4];
  int *status;
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
