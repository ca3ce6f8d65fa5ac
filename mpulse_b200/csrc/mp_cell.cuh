// mp_cell.cuh - the arithmetic of one cell's E update and B update, shared by
// the global-load kernels (mp_step_kernels.cu) and the TMA-staged kernels
// (mp_step_tma.cu).  The caller loads the field values (from global memory or
// from shared memory) and the PLRC accumulators, calls e_cell / b_cell, and
// stores the results; the CPML psi of the faces containing the cell and the
// injection-plane values are loaded and stored here with plain global accesses
// (a minority of cells).
//
// Order of operations per cell: every load before any store.  The arrays may
// alias as far as the compiler can tell, so a load written after a store would
// wait for that store to complete.
#ifndef MPB_MP_CELL_CUH
#define MPB_MP_CELL_CUH

#include "mp_checked.cuh"
#include "mp_device.h"

#include <cuda_runtime.h>

namespace mpb {

template <typename T> struct Vec2;
template <> struct Vec2<float> { typedef float2 type; };
template <> struct Vec2<double> { typedef double2 type; };

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }


// A value is finite in T exactly when it is finite after widening: test it
// in T (no conversions in the FP32 form).
template <typename T>
__device__ __forceinline__ bool finite3(T a, T b, T c) {
  return isfinite(a) && isfinite(b) && isfinite(c);
}

// CPML faces sit in fixed slots of EParams::cpml / BParams::cpml, in MPulse's
// current order (north, south, east, west, up, down): slots 0-1 are y faces,
// 2-3 x faces, 4-5 z faces.  With the slot known at compile time the axis of
// every face is too.
__host__ __device__ constexpr int face_axis(int f) { return f < 2 ? 1 : (f < 4 ? 0 : 2); }

// Bit f (f < 4) set when the x / y face in slot f contains column (i, j):
// computed once per thread, outside the z-march.
template <typename T>
__device__ __forceinline__ unsigned face_column_mask(const CpmlFace<T> (&cpml)[6], int i, int j) {
  unsigned m = 0;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const int idx = face_axis(f) == 0 ? i + 1 : j + 1;
    if (cpml[f].active && idx >= cpml[f].lo && idx <= cpml[f].hi) m |= 1u << f;
  }
  return m;
}

// True when plane k lies in one of the z faces (slots 4, 5).
template <typename T>
__device__ __forceinline__ bool z_face_plane(const CpmlFace<T> (&cpml)[6], int k) {
  return (cpml[4].active && k >= cpml[4].lo && k <= cpml[4].hi) ||
         (cpml[5].active && k >= cpml[5].lo && k <= cpml[5].hi);
}

// The range of planes holding an injection plane (empty: lo > hi).
template <typename P>
__device__ __forceinline__ int2 source_plane_range(const P &p) {
  int2 r = make_int2(1 << 30, -(1 << 30));
#pragma unroll
  for (int s = 0; s < 4; ++s)
    if (s < p.n_src) {
      r.x = min(r.x, p.src[s].plane);
      r.y = max(r.y, p.src[s].plane);
    }
  return r;
}

// 1/d for 1e-30 < d < 1e30: a single-precision estimate refined by two
// Newton-Raphson steps r <- r + r (1 - d r) in FP64, each squaring the relative
// error (the Newton-Raphson iteration for the reciprocal, e.g. Muller et al.,
// Handbook of Floating-Point Arithmetic): about 1e-7, then 1e-14, then below
// FP64 rounding.  Other d (a diverging field) fall back to the division.  The
// Newton denominators below are at least 1 (Kerr) or eps (FDTD_Nonlinear).
__device__ __forceinline__ double rcp_pos(double d) {
  if (!(d > 1e-30 && d < 1e30)) return 1.0 / d;
  double r = (double)__fdividef(1.0f, (float)d);
  r = fma(r, fma(-d, r, 1.0), r);
  r = fma(r, fma(-d, r, 1.0), r);
  return r;
}

// The same with one Newton-Raphson step (relative error about 1e-14), for
// the FP32 form, whose results are rounded to single precision.
__device__ __forceinline__ double rcp_pos1(double d) {
  if (!(d > 1e-30 && d < 1e30)) return 1.0 / d;
  const double r = (double)__fdividef(1.0f, (float)d);
  return fma(r, fma(-d, r, 1.0), r);
}

// Newton solve of |E| + A |E|^3 = C, FDTD_PLRCNonlinCore::plrcStepD
// (fdtd_plrc.cpp:406-419), in FP64 whatever the field precision; capped at
// maxit iterations.  Adds the iterations it ran to *iters.  FP32 = true: the
// reciprocal of each step to about 1e-14 (rcp_pos1), enough for a result
// rounded to single precision.
template <bool FP32 = false>
__device__ __forceinline__ double kerr_newton(double E, double A, double C, double tol, int maxit,
                                              int *status, unsigned *iters) {
  double Eold;
  int it = 0;
  do {
    Eold = E;
    const double E2 = E * E;
    const double d = 3.0 * A * E2 + 1.0;
    E = (2.0 * A * E2 * E + C) * (FP32 ? rcp_pos1(d) : rcp_pos(d));
    ++it;
  } while (fabs(E - Eold) > tol && it < maxit);
  if (fabs(E - Eold) > tol) atomicAdd(status + ST_NEWTON, 1);
  *iters += unsigned(it);
  return E;
}

// FDTD_Nonlinear's Newton for eps E + chi E^3 = D (fdtd_nl.cpp:86-92).
__device__ __forceinline__ double nl_newton(double E, double eps, double chi, double D, double tol,
                                            int maxit, int *status, unsigned *iters) {
  double Eold;
  int it = 0;
  do {
    Eold = E;
    const double E2 = E * E;
    E = (2.0 * chi * E2 * E + D) * rcp_pos(3.0 * chi * E2 + eps);
    ++it;
  } while (fabs(E - Eold) > tol && it < maxit);
  if (fabs(E - Eold) > tol) atomicAdd(status + ST_NEWTON, 1);
  *iters += unsigned(it);
  return E;
}

// Per-thread counts of the Kerr solves a thread ran ([0]: cells in which the
// Newton solve ran, [1]: the iterations they took), added to the context's
// counters once per warp when the thread's z-march ends.
struct KerrCount {
  unsigned solves = 0, iters = 0;
};

template <int MODE>
__device__ __forceinline__ void flush_kerr_count(unsigned long long *dst, const KerrCount &kc) {
  if (MODE != MODE_PLRC_NONLIN && MODE != MODE_NL) return;
  const unsigned m = __activemask();
  const unsigned a = __reduce_add_sync(m, kc.solves);
  const unsigned b = __reduce_add_sync(m, kc.iters);
  const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
  if (lane == __ffs(m) - 1 && a != 0u) {
    atomicAdd(dst, (unsigned long long)a);
    atomicAdd(dst + 1, (unsigned long long)b);
  }
}

// dt * u with the FP32 form's compensated step (hi + lo): the exact product
// dt * u plus dt_lo * u, rounded once.  FP64: dt * u.
template <typename T>
__device__ __forceinline__ T dt_mul(T dt, T dt_lo, T u) {
  return sizeof(T) == 4 ? fma(dt, u, dt_lo * u) : dt * u;
}

// numer * e + a and x * inv_denom with the compensated coefficients of the
// FP32 form; in FP64 the plain products.
template <typename T>
__device__ __forceinline__ T numer_mul_add(T numer, T numer_lo, T e, T a) {
  return sizeof(T) == 4 ? fma(numer, e, fma(numer_lo, e, a)) : numer * e + a;
}
template <typename T>
__device__ __forceinline__ T inv_denom_mul(T x, T idn, T idn_lo) {
  return sizeof(T) == 4 ? fma(x, idn, x * idn_lo) : x * idn;
}

// Sums of two products spelled out as one FMA: a b + c d, a b - c d, and
// a^2 + b^2 + c^2.  Left to the compiler, either product of such a sum may be
// fused, and the choice differs between kernels that inline the same cell
// code (it did between the fused step kernel, whose neighbours come from
// shared memory, and the half-step kernels); spelled out, every kernel form
// rounds alike.  A lone a b + c is fused the same way everywhere.
template <typename T>
__device__ __forceinline__ T fma_pp(T a, T b, T c, T d) {
  return fma(a, b, c * d);
}
template <typename T>
__device__ __forceinline__ T fma_pm(T a, T b, T c, T d) {
  return fma(a, b, -(c * d));
}
template <typename T>
__device__ __forceinline__ T sq3(T a, T b, T c) {
  return fma(c, c, fma(b, b, a * a));
}

// e + dt u with the FP32 form's compensated step; in FP64 one FMA.
template <typename T>
__device__ __forceinline__ T add_dt(T e, T dt, T dt_lo, T u) {
  return sizeof(T) == 4 ? e + fma(dt, u, dt_lo * u) : fma(dt, u, e);
}

// The plasma plug-ins at one cell, from E^n (before the E update):
// PlasmaDensity::stepScheme (plasmadensity.cpp:18-49) gives the new density
// and the conductivity Sigma = mpa Wion I^(K-1) of this step (Sigma is reset
// every step, fdtd_plrc.t:129), of which the E update takes sig = Sigma dt / 2
// (fdtd_plrc.cpp:188, :356); PlasmaCurrent::stepScheme
// (plasmacurrent.cpp:42-74) gives the new current from E^n and the new
// density.  Same operations and order as the reference.
template <typename T>
struct PlasmaCell {
  T rho, j[3], sig;
};

template <typename T>
__device__ __forceinline__ void plasma_cell(const EParams<T> &p, T ex, T ey, T ez, T rho, T j0, T j1, T j2,
                                            PlasmaCell<T> &pc) {
  pc.rho = rho;
  pc.sig = T(0);
  if (p.pl_density) {
    const T I = sq3(ex, ey, ez);
    T IKm = T(1);  // util.h ipow: K - 1 products
    for (int q = 0; q < p.pl_km; ++q) IKm *= I;
    const T IK = I * IKm;
    pc.rho = fma_pp(rho, T(1) + p.pl_n * I, p.pl_m, IK) / (T(1) - p.pl_n * I);
    pc.sig = T(0.5) * (p.pl_w * IKm) * p.dt;
  }
  if (p.pl_current) {
    const T r = pc.rho + p.pl_rho_bg;
    pc.j[0] = fma_pm(j0, p.pl_gdtn, p.pl_emdt * ex, r) / p.pl_gdtd;
    pc.j[1] = fma_pm(j1, p.pl_gdtn, p.pl_emdt * ey, r) / p.pl_gdtd;
    pc.j[2] = fma_pm(j2, p.pl_gdtn, p.pl_emdt * ez, r) / p.pl_gdtd;
  } else {
    pc.j[0] = pc.j[1] = pc.j[2] = T(0);
  }
}

// Values one E update reads: B at the cell and its x-1, y-1, z-1 neighbours
// (the ones the curl uses) and the old E.
template <typename T>
struct EIn {
  T bx, by, bz;
  T bz_xm, by_xm, bz_ym, bx_ym, bx_km, by_km;
  T ex, ey, ez;
};

// Values one B update reads: E at the cell and its x+1, y+1, z+1 neighbours
// and the old B.
template <typename T>
struct BIn {
  T ex, ey, ez;
  T ez_xp, ey_xp, ez_yp, ex_yp, ex_kp, ey_kp;
  T bx, by, bz;
};

// One cell of the E half: CPML psi_E (cpml_border.cpp:398-425), the current sum
// in MPulse's order (fdtd_plrc.t:352-373), the PLRC recursion and the E update
// of plrcStepD (fdtd_plrc.cpp:94-261, :304-427), FDTD_Plain::stepD
// (fdtd_plain.cpp:37-77) or FDTD_Nonlinear::stepD (fdtd_nl.cpp:38-100).
// i, j are 0-based interior indices (MPulse i+1, j+1); k is MPulse's z index.
// q holds the cell's PLRC accumulators on entry and their new values on exit.
// The medium coefficients of one cell: the kernel parameters, or for a cell of
// the design region the same formulas with its eps_infinity, Delta-eps factor s
// and chi factor u (FP64, then rounded to T like the host's).  Factors 1 and
// eps_infinity = eps reproduce the kernel parameters bit for bit.
template <typename T, int NP>
struct CellCoef {
  T numer, inv_denom, chi;
  T numer_lo, inv_denom_lo;  // FP32 form: the rounding errors of numer and inv_denom (zero in FP64)
  double chi_over_denom;
  T pD[NP > 0 ? NP : 1][2], pxi[NP > 0 ? NP : 1][2];
};

template <typename T, int NP, bool DESIGN>
__device__ __forceinline__ void cell_coef(const EParams<T> &p, int i, int j, int k, bool med, CellCoef<T, NP> &cc) {
  cc.numer = p.numer;
  cc.inv_denom = p.inv_denom;
  cc.numer_lo = p.numer_lo;
  cc.inv_denom_lo = p.inv_denom_lo;
  cc.chi = p.chi;
  cc.chi_over_denom = p.chi_over_denom;
#pragma unroll
  for (int n = 0; n < (NP > 0 ? NP : 1); ++n)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      cc.pD[n][r] = p.pD[n][r];
      cc.pxi[n][r] = p.pxi[n][r];
    }
  if (DESIGN) {
    const DesignParams &d = p.design;
    if (med && i >= d.x0 && i <= d.x1 && j >= d.y0 && j <= d.y1 && k >= d.z0 && k <= d.z1) {
      const long long di = ((long long)(k - d.z0) * d.by + (j - d.y0)) * d.bx + (i - d.x0);
      const double e = d.eps[di], s = d.dscale[di], u = d.chiscale[di];
      const double denom = d.lin ? e + s * (d.sumChi0 - d.sumXi0) : e + s * d.sumChi0 - s * d.sumXi0;
      const double nm = e - s * d.sumXi0, idn = 1.0 / denom;
      cc.numer = T(nm);
      cc.inv_denom = T(idn);
      cc.numer_lo = T(nm - double(cc.numer));
      cc.inv_denom_lo = T(idn - double(cc.inv_denom));
      cc.chi = T(u * d.chi);
      cc.chi_over_denom = u * d.chi / denom;
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          cc.pD[n][r] = T(s * d.pD[n][r]);
          cc.pxi[n][r] = T(s * d.pxi[n][r]);
        }
    }
  }
}

// SPECIAL = false: the caller guarantees that no CPML face contains the cell
// and that k is no injection plane; the face and source code is left out.
// PLASMA: *pc holds the plasma plug-ins' values of the cell (plasma_cell).
template <typename T, int MODE, int NP, bool DESIGN = false, bool SPECIAL = true, bool PLASMA = false>
__device__ __forceinline__ void e_cell(const EParams<T> &p, int i, int j, int k, long long col, bool med,
                                       unsigned cmask, const EIn<T> &v, T ikx, T iky, T ikz,
                                       typename Vec2<T>::type (&q)[NP > 0 ? NP : 1][3], T &exn, T &eyn,
                                       T &ezn, KerrCount &kc, const PlasmaCell<T> *pc = nullptr) {
  const T dt = p.dt;
  CellCoef<T, NP> lc;
  cell_coef<T, NP, DESIGN>(p, i, j, k, med, lc);
  if (PLASMA && med && p.pl_density) {
    // numer - sig and denom + sig (fdtd_plrc.cpp:188-196, :356-359)
    lc.numer = lc.numer - pc->sig;
    lc.inv_denom = T(1) / (p.denom_t + pc->sig);
    lc.inv_denom_lo = T(0);
    lc.chi_over_denom = p.chi_raw / (p.denom_d + (double)pc->sig);
  }
  // ---- loads of the CPML psi of the faces containing the cell, and of the
  // injection plane
  T cp0[6], cp1[6], cb[6], cc[6];
  int cli[6];  // layer arrays hold < 2^31 cells (checked by mp_create)
  bool cin[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const CpmlFace<T> &F = p.cpml[f];
    const int idx = face_axis(f) == 0 ? i + 1 : face_axis(f) == 1 ? j + 1 : k;
    cin[f] = SPECIAL && (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) &&
             (f < 4 ? ((cmask >> f) & 1u) != 0 : (F.active && k >= F.lo && k <= F.hi));
    if (cin[f]) {
      if (face_axis(f) == 2) cli[f] = ((k - F.lo) * p.ny + j) * p.nx + i;
      else if (face_axis(f) == 0) cli[f] = ((k - F.zlo) * p.ny + j) * F.ex + (i + 1 - F.lo);
      else cli[f] = ((k - F.zlo) * F.ey + (j + 1 - F.lo)) * p.nx + i;
      cp0[f] = ld_c(F.psi0, cli[f], F.n, p.status);
      cp1[f] = ld_c(F.psi1, cli[f], F.n, p.status);
      cb[f] = ld(F.b + idx);
      cc[f] = ld(F.c + idx);
    }
  }
  T sa = T(0), sb = T(0);
  bool on_src = false;
  if (SPECIAL && (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN)) {
    for (int s = 0; s < p.n_src; ++s) {
      if (k == p.src[s].plane) {
        sa = ldg_c(p.src[s].v0, col, p.plane, p.status);
        sb = ldg_c(p.src[s].v1, col, p.plane, p.status);
        on_src = true;
      }
    }
  }

  // ---- E-side currents: CPML faces, then the injector plane
  T jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (!cin[f]) continue;
    const int dim = face_axis(f);
    T d0, d1;  // differences of B along dim for psi0, psi1
    if (dim == 2) { d0 = -(v.by - v.by_km); d1 = v.bx - v.bx_km; }
    else if (dim == 0) { d0 = -(v.bz - v.bz_xm); d1 = v.by - v.by_xm; }
    else { d0 = -(v.bx - v.bx_ym); d1 = v.bz - v.bz_ym; }
    cp0[f] = fma_pp(cb[f], cp0[f], cc[f], d0);
    cp1[f] = fma_pp(cb[f], cp1[f], cc[f], d1);
    if (dim == 2) { jx += cp0[f]; jy += cp1[f]; }
    else if (dim == 0) { jy += cp0[f]; jz += cp1[f]; }
    else { jz += cp0[f]; jx += cp1[f]; }
  }
  if (on_src) {
    for (int m = 0; m < p.src_mult; ++m) {
      jx += sa;
      jy += sb;
    }
  }
  if (PLASMA) {  // the plasma current, after the other currents
    jx += pc->j[0];
    jy += pc->j[1];
    jz += pc->j[2];
  }

  // curl_kappa B (fdtd_plrc.cpp:207-244)
  const T cbx = fma_pm(v.bz - v.bz_ym, iky, v.by - v.by_km, ikz);
  const T cby = fma_pm(v.bx - v.bx_km, ikz, v.bz - v.bz_xm, ikx);
  const T cbz = fma_pm(v.by - v.by_xm, ikx, v.bx - v.bx_ym, iky);
  const T ex = v.ex, ey = v.ey, ez = v.ez;

  const T dtl = p.dt_lo;
  if (MODE == MODE_PLAIN) {
    exn = add_dt(ex, dt, dtl, cbx);
    eyn = add_dt(ey, dt, dtl, cby);
    ezn = add_dt(ez, dt, dtl, cbz);
  } else if (MODE == MODE_NL) {
    const double E2 = sq3((double)ex, (double)ey, (double)ez);
    const T f = T(p.eps_d + p.chi_d * E2);
    const T Dx = fma(f, ex, dt_mul(dt, dtl, cbx)), Dy = fma(f, ey, dt_mul(dt, dtl, cby)),
            Dz = fma(f, ez, dt_mul(dt, dtl, cbz));
    const double D2 = sq3((double)Dx, (double)Dy, (double)Dz);
    if (D2 > 0) {
      const double rD = rsqrt(D2);  // as in the PLRC Kerr update below
      const double D = D2 * rD;
      const double E0 = E2 > 0 ? E2 * rsqrt(E2) : 0.0;
      const double E = nl_newton(E0, p.eps_d, p.chi_d, D, p.newton_tol, p.newton_max, p.status, &kc.iters);
      ++kc.solves;
      const double sc = E * rD;
      exn = T(sc * Dx);
      eyn = T(sc * Dy);
      ezn = T(sc * Dz);
    } else {
      exn = eyn = ezn = T(0);
    }
  } else if (!med) {
    // background: no poles, no Kerr term
    if (PLASMA && p.pl_density) {
      const T nb = p.eps_bg - pc->sig, ib = T(1) / (p.eps_bg + pc->sig);
      exn = fma(nb, ex, dt_mul(dt, dtl, cbx + jx)) * ib;
      eyn = fma(nb, ey, dt_mul(dt, dtl, cby + jy)) * ib;
      ezn = fma(nb, ez, dt_mul(dt, dtl, cbz + jz)) * ib;
    } else {
      exn = fma(p.eps_bg, ex, dt_mul(dt, dtl, cbx + jx)) * p.inv_eps_bg;
      eyn = fma(p.eps_bg, ey, dt_mul(dt, dtl, cby + jy)) * p.inv_eps_bg;
      ezn = fma(p.eps_bg, ez, dt_mul(dt, dtl, cbz + jz)) * p.inv_eps_bg;
    }
  } else {
    T Px = T(0), Py = T(0), Pz = T(0);
    if (NP > 0) {
      const T e3[3] = {ex, ey, ez};
      T P3[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int n = 0; n < NP; ++n) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          // psi~ = (dchi0 - dxi0) e + psi ; Psi += Re psi~
          const T ar = lc.pD[n][0] * e3[c] + q[n][c].x;
          const T ai = lc.pD[n][1] * e3[c] + q[n][c].y;
          P3[c] += ar;
          // psi <- dxi0 e + Crec psi~
          q[n][c].x = fma(lc.pxi[n][0], e3[c], fma_pm(p.pC[n][0], ar, p.pC[n][1], ai));
          q[n][c].y = fma(lc.pxi[n][1], e3[c], fma_pp(p.pC[n][0], ai, p.pC[n][1], ar));
        }
      }
      Px = P3[0];
      Py = P3[1];
      Pz = P3[2];
    }
    if (MODE == MODE_PLRC_LIN) {
      exn = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ex, dt_mul(dt, dtl, cbx + jx) + Px), lc.inv_denom,
                          lc.inv_denom_lo);
      eyn = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ey, dt_mul(dt, dtl, cby + jy) + Py), lc.inv_denom,
                          lc.inv_denom_lo);
      ezn = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ez, dt_mul(dt, dtl, cbz + jz) + Pz), lc.inv_denom,
                          lc.inv_denom_lo);
    } else {
      // |E^n|^2: in FP64 for the FP64 form; the FP32 form needs it only for
      // the single-precision Kerr term and the start of the Newton solve
      double E2;
      T E2t;
      if (sizeof(T) == 4) {
        E2t = sq3(ex, ey, ez);
        E2 = E2t;
      } else {
        E2 = sq3((double)ex, (double)ey, (double)ez);
        E2t = T(E2);
      }
      const T f = lc.numer + lc.chi * E2t;
      T cx, cy, cz;
      if (sizeof(T) == 4) {
        // (numer + chi |E|^2) E + dt u + P with the compensated numer and dt
        const T kf = lc.chi * E2t;
        cx = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ex, fma(kf, ex, dt_mul(dt, dtl, cbx + jx) + Px)),
                           lc.inv_denom, lc.inv_denom_lo);
        cy = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ey, fma(kf, ey, dt_mul(dt, dtl, cby + jy) + Py)),
                           lc.inv_denom, lc.inv_denom_lo);
        cz = inv_denom_mul(numer_mul_add(lc.numer, lc.numer_lo, ez, fma(kf, ez, dt_mul(dt, dtl, cbz + jz) + Pz)),
                           lc.inv_denom, lc.inv_denom_lo);
      } else {
        cx = fma(f, ex, fma(dt, cbx + jx, Px)) * lc.inv_denom;
        cy = fma(f, ey, fma(dt, cby + jy, Py)) * lc.inv_denom;
        cz = fma(f, ez, fma(dt, cbz + jz, Pz)) * lc.inv_denom;
      }
      // |c|, 1/|c| and the start |E^n| from reciprocal square roots: no FP64
      // square root or division here (equal to sqrt and / up to rounding).
      // The FP32 form takes 1/|c| from the single-precision estimate refined
      // by one FP64 Newton-Raphson step r <- r (3/2 - C2 r^2 / 2) (relative
      // error about 1e-14, far below the FP32 rounding of the result) and the
      // start |E^n| of the Newton solve in single precision (the solve
      // converges to the same root from any start near it); outside the
      // normal single-precision range it takes the FP64 path.
      const double C2 = sq3((double)cx, (double)cy, (double)cz);
      if (C2 > 0) {
        double rC, E0;
        if (sizeof(T) == 4 && C2 > 1e-30 && C2 < 1e30) {
          rC = (double)rsqrtf((float)C2);
          rC = rC * fma(-0.5 * C2, rC * rC, 1.5);
          E0 = (double)sqrtf((float)E2t);
        } else {
          rC = rsqrt(C2);
          E0 = E2 > 0 ? E2 * rsqrt(E2) : 0.0;
        }
        const double C = C2 * rC;
        const double E = kerr_newton<sizeof(T) == 4>(E0, lc.chi_over_denom, C, p.newton_tol, p.newton_max, p.status,
                                                      &kc.iters);
        ++kc.solves;
        const double sc = E * rC;
        exn = T(sc * cx);
        eyn = T(sc * cy);
        ezn = T(sc * cz);
      } else {
        exn = eyn = ezn = T(0);
      }
    }
  }
  if (!finite3(exn, eyn, ezn)) atomicAdd(p.status + ST_NONFINITE, 1);
  // ---- CPML stores
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (!cin[f]) continue;
    st_c(p.cpml[f].psi0, cli[f], p.cpml[f].n, p.status, cp0[f]);
    st_c(p.cpml[f].psi1, cli[f], p.cpml[f].n, p.status, cp1[f]);
  }
}

// One cell of the B half: CPML psi_H (cpml_border.cpp:499-527), the magnetic
// current sum and plrcStepB (fdtd_plrc.cpp:263-293) / FDTD_Plain::stepB.
// Returns the new B in bxn, byn, bzn.
template <typename T, bool SPECIAL = true>
__device__ __forceinline__ void b_cell(const BParams<T> &p, int i, int j, int k, long long col, unsigned cmask,
                                       const BIn<T> &v, T ikx, T iky, T iky_bz, T ikz, T &bxn, T &byn, T &bzn) {
  const T dt = p.dt;
  T cp0[6], cp1[6], cb[6], cc[6];
  int cli[6];
  bool cin[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const CpmlFace<T> &F = p.cpml[f];
    const int idx = face_axis(f) == 0 ? i + 1 : face_axis(f) == 1 ? j + 1 : k;
    cin[f] = SPECIAL && (f < 4 ? ((cmask >> f) & 1u) != 0 : (F.active && k >= F.lo && k <= F.hi));
    if (cin[f]) {
      if (face_axis(f) == 2) cli[f] = ((k - F.lo) * p.ny + j) * p.nx + i;
      else if (face_axis(f) == 0) cli[f] = ((k - F.zlo) * p.ny + j) * F.ex + (i + 1 - F.lo);
      else cli[f] = ((k - F.zlo) * F.ey + (j + 1 - F.lo)) * p.nx + i;
      cp0[f] = ld_c(F.psi0, cli[f], F.n, p.status);
      cp1[f] = ld_c(F.psi1, cli[f], F.n, p.status);
      cb[f] = ld(F.b + idx);
      cc[f] = ld(F.c + idx);
    }
  }
  T sa = T(0), sb = T(0);
  bool on_src = false;
  for (int s = 0; SPECIAL && s < p.n_src; ++s) {
    if (k == p.src[s].plane) {
      sa = ldg_c(p.src[s].v0, col, p.plane, p.status);
      sb = ldg_c(p.src[s].v1, col, p.plane, p.status);
      on_src = true;
    }
  }

  // ---- H-side currents (cpml_border.cpp:499-527, incsource.t:112-145)
  T mx = T(0), my = T(0), mz = T(0);
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (!cin[f]) continue;
    const int dim = face_axis(f);
    T d0, d1;
    if (dim == 2) { d0 = v.ey_kp - v.ey; d1 = -(v.ex_kp - v.ex); }
    else if (dim == 0) { d0 = v.ez_xp - v.ez; d1 = -(v.ey_xp - v.ey); }
    else { d0 = v.ex_yp - v.ex; d1 = -(v.ez_yp - v.ez); }
    cp0[f] = fma_pp(cb[f], cp0[f], cc[f], d0);
    cp1[f] = fma_pp(cb[f], cp1[f], cc[f], d1);
    if (dim == 2) { mx += cp0[f]; my += cp1[f]; }
    else if (dim == 0) { my += cp0[f]; mz += cp1[f]; }
    else { mz += cp0[f]; mx += cp1[f]; }
  }
  if (on_src) {
    for (int m = 0; m < p.src_mult; ++m) {
      mx += sa;
      my += sb;
    }
  }

  // ---- plrcStepB (fdtd_plrc.cpp:263-293)
  bxn = add_dt(v.bx, dt, p.dt_lo, fma_pm(v.ey_kp - v.ey, ikz, v.ez_yp - v.ez, iky) + mx);
  byn = add_dt(v.by, dt, p.dt_lo, fma_pm(v.ez_xp - v.ez, ikx, v.ex_kp - v.ex, ikz) + my);
  bzn = add_dt(v.bz, dt, p.dt_lo, fma_pm(v.ex_yp - v.ex, iky_bz, v.ey_xp - v.ey, ikx) + mz);
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (!cin[f]) continue;
    st_c(p.cpml[f].psi0, cli[f], p.cpml[f].n, p.status, cp0[f]);
    st_c(p.cpml[f].psi1, cli[f], p.cpml[f].n, p.status, cp1[f]);
  }
}

}  // namespace mpb

#endif
