// mp_step_kernels.cu - the two half-step kernels of one MPulse time step.
//
// e_half: FDTD_PLRCSolver::stepScheme's E side (fdtd_plrc.t:129-146) in one
//   pass: the CPML psi_E recursions (CPMLBorderECurrent::stepScheme,
//   cpml_border.cpp:398-425), the TF/SF J plane (incsource.t:40-73, values from
//   mp_source_kernels.cu), the current sum (fdtd_plrc.t:342-374, never
//   materialised), the PLRC recursion and D -> E update of plrcStepD
//   (fdtd_plrc.cpp:94-261, nonlinear :304-427) or of FDTD_Plain / FDTD_Nonlinear
//   (fdtd_plain.cpp:37-77, fdtd_nl.cpp:38-100), and the periodic boundary as an
//   index wrap (periodic_bound.cpp:10-71).
// b_half: the H side (fdtd_plrc.t:148-167): CPML psi_H
//   (cpml_border.cpp:499-527), TF/SF M plane (incsource.t:112-145) and plrcStepB
//   (fdtd_plrc.cpp:263-293).
//
// Thread mapping: one thread per (x, y) column, 32 x 8 columns per block; a
// block marches up a chunk of z-planes so the z-neighbour of the previous plane
// is carried in registers and every field element is read from HBM once per
// half step (x/y neighbours are re-read through L1/L2).  The medium test, the
// CPML z-faces and the source planes depend on z only and are uniform per
// iteration.  The stencil has no contraction, so no tensor cores are involved;
// both kernels are HBM-bandwidth bound.
#include "mp_device.h"

#include <cuda_runtime.h>

// Minimum resident blocks per SM asked of the register allocator.  Measured
// on the 256x256x512 PLRC + Kerr workload (FP32): E half 1.083 ms with no
// bound (114 registers), 0.917 ms with 3 blocks (80 registers, 28 B spilled),
// 1.17 ms with 4 (64 registers, more spills); the B half does not move.
#ifndef MPB_E_MIN_BLOCKS
#define MPB_E_MIN_BLOCKS 3
#endif
#ifndef MPB_B_MIN_BLOCKS
#define MPB_B_MIN_BLOCKS 1
#endif

namespace mpb {

template <typename T> struct Vec2;
template <> struct Vec2<float> { typedef float2 type; };
template <> struct Vec2<double> { typedef double2 type; };

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

__device__ __forceinline__ bool finite3(double a, double b, double c) {
  return isfinite(a) && isfinite(b) && isfinite(c);
}

// Newton solve of |E| + A |E|^3 = C, FDTD_PLRCNonlinCore::plrcStepD
// (fdtd_plrc.cpp:406-419), in FP64 whatever the field precision; capped.
__device__ __forceinline__ double kerr_newton(double E, double A, double C, double tol, int maxit,
                                              int *status) {
  double Eold;
  int it = 0;
  do {
    Eold = E;
    const double E2 = E * E;
    E = (2.0 * A * E2 * E + C) / (3.0 * A * E2 + 1.0);
  } while (fabs(E - Eold) > tol && ++it < maxit);
  if (fabs(E - Eold) > tol) atomicAdd(status + ST_NEWTON, 1);
  return E;
}

// FDTD_Nonlinear's Newton for eps E + chi E^3 = D (fdtd_nl.cpp:86-92).
__device__ __forceinline__ double nl_newton(double E, double eps, double chi, double D, double tol,
                                            int maxit, int *status) {
  double Eold;
  int it = 0;
  do {
    Eold = E;
    const double E2 = E * E;
    E = (2.0 * chi * E2 * E + D) / (3.0 * chi * E2 + eps);
  } while (fabs(E - Eold) > tol && ++it < maxit);
  if (fabs(E - Eold) > tol) atomicAdd(status + ST_NEWTON, 1);
  return E;
}

template <typename T, int MODE, int NP>
__global__ void __launch_bounds__(256, MPB_E_MIN_BLOCKS) e_half_kernel(const EParams<T> p) {
  typedef typename Vec2<T>::type T2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // 0-based: MPulse i + 1
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= p.nx || j >= p.ny) return;
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  if (k0 > k1) return;

  const long long plane = p.plane;
  const int im = (i == 0) ? p.nx - 1 : i - 1;
  const int jm = (j == 0) ? p.ny - 1 : j - 1;
  const long long col = (long long)j * p.nx + i;
  const long long colxm = (long long)j * p.nx + im;
  const long long colym = (long long)jm * p.nx + i;
  const T *__restrict__ Bx = p.B[0];
  const T *__restrict__ By = p.B[1];
  const T *__restrict__ Bz = p.B[2];
  T *__restrict__ Ex = p.E[0];
  T *__restrict__ Ey = p.E[1];
  T *__restrict__ Ez = p.E[2];
  const T ikx = ld(p.ik[0] + i + 1);
  const T iky = ld(p.ik[1] + j + 1);
  const T dt = p.dt;

  int km = k0 - 1;
  if (p.zperiodic && km == 0) km = p.nz;
  T bx_km = ld(Bx + km * plane + col);
  T by_km = ld(By + km * plane + col);

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    // ---- all loads of this cell first: the arrays may alias as far as the
    // compiler knows, so a load placed after a store would wait for it
    const T bx = ld(Bx + base + col), by = ld(By + base + col), bz = ld(Bz + base + col);
    const T bz_xm = ld(Bz + base + colxm), by_xm = ld(By + base + colxm);
    const T bz_ym = ld(Bz + base + colym), bx_ym = ld(Bx + base + colym);
    const T ex = Ex[base + col], ey = Ey[base + col], ez = Ez[base + col];
    const T ikz = ld(p.ik[2] + k);
    const bool med = (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) && k >= p.mz0 && k <= p.mz1;
    const long long pi = ((long long)(k - p.mz0) * p.ny + j) * p.nx + i;
    T2 q[NP > 0 ? NP : 1][3];
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) q[n][c] = reinterpret_cast<const T2 *>(p.psi[n][c])[pi];
    }
    T cp0[6], cp1[6], cb[6], cc[6];
    int cli[6];  // layer arrays hold < 2^31 cells (checked by mp_create)
    bool cin[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const CpmlFace<T> &F = p.cpml[f];
      const int idx = F.dim == 0 ? i + 1 : F.dim == 1 ? j + 1 : k;
      cin[f] = (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) && F.active && idx >= F.lo && idx <= F.hi;
      if (cin[f]) {
        if (F.dim == 2) cli[f] = ((k - F.lo) * p.ny + j) * p.nx + i;
        else if (F.dim == 0) cli[f] = ((k - F.zlo) * p.ny + j) * F.ex + (i + 1 - F.lo);
        else cli[f] = ((k - F.zlo) * F.ey + (j + 1 - F.lo)) * p.nx + i;
        cp0[f] = F.psi0[cli[f]];
        cp1[f] = F.psi1[cli[f]];
        cb[f] = ld(F.b + idx);
        cc[f] = ld(F.c + idx);
      }
    }
    T sa = T(0), sb = T(0);
    bool on_src = false;
    for (int s = 0; s < p.n_src; ++s) {
      if (k == p.src[s].plane) {
        sa = ld(p.src[s].v0 + col);
        sb = ld(p.src[s].v1 + col);
        on_src = true;
      }
    }

    // ---- E-side currents, summed in MPulse's current order
    // (fdtd_plrc.t:352-373): CPML faces (cpml_border.cpp:398-425), then the
    // injector plane
    T jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!cin[f]) continue;
      const int dim = p.cpml[f].dim;
      T d0, d1;  // differences of B along dim for psi0, psi1
      if (dim == 2) { d0 = -(by - by_km); d1 = bx - bx_km; }
      else if (dim == 0) { d0 = -(bz - bz_xm); d1 = by - by_xm; }
      else { d0 = -(bx - bx_ym); d1 = bz - bz_ym; }
      cp0[f] = cb[f] * cp0[f] + cc[f] * d0;
      cp1[f] = cb[f] * cp1[f] + cc[f] * d1;
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

    // curl_kappa B (fdtd_plrc.cpp:207-244)
    const T cbx = (bz - bz_ym) * iky - (by - by_km) * ikz;
    const T cby = (bx - bx_km) * ikz - (bz - bz_xm) * ikx;
    const T cbz = (by - by_xm) * ikx - (bx - bx_ym) * iky;

    T exn, eyn, ezn;
    if (MODE == MODE_PLAIN) {
      exn = ex + dt * cbx;
      eyn = ey + dt * cby;
      ezn = ez + dt * cbz;
    } else if (MODE == MODE_NL) {
      const double E2 = (double)ex * ex + (double)ey * ey + (double)ez * ez;
      const T f = T(p.eps_d + p.chi_d * E2);
      const T Dx = f * ex + dt * cbx, Dy = f * ey + dt * cby, Dz = f * ez + dt * cbz;
      const double D = sqrt((double)Dx * Dx + (double)Dy * Dy + (double)Dz * Dz);
      if (D > 0) {
        const double E = nl_newton(sqrt(E2), p.eps_d, p.chi_d, D, p.newton_tol, p.newton_max, p.status);
        exn = T(E * Dx / D);
        eyn = T(E * Dy / D);
        ezn = T(E * Dz / D);
      } else {
        exn = eyn = ezn = T(0);
      }
    } else {
      if (!med) {
        // background: no poles, no Kerr term
        exn = (p.eps_bg * ex + dt * (cbx + jx)) * p.inv_eps_bg;
        eyn = (p.eps_bg * ey + dt * (cby + jy)) * p.inv_eps_bg;
        ezn = (p.eps_bg * ez + dt * (cbz + jz)) * p.inv_eps_bg;
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
              const T ar = p.pD[n][0] * e3[c] + q[n][c].x;
              const T ai = p.pD[n][1] * e3[c] + q[n][c].y;
              P3[c] += ar;
              // psi <- dxi0 e + Crec psi~
              q[n][c].x = p.pxi[n][0] * e3[c] + (p.pC[n][0] * ar - p.pC[n][1] * ai);
              q[n][c].y = p.pxi[n][1] * e3[c] + (p.pC[n][0] * ai + p.pC[n][1] * ar);
            }
          }
          Px = P3[0]; Py = P3[1]; Pz = P3[2];
        }
        if (MODE == MODE_PLRC_LIN) {
          exn = (p.numer * ex + (dt * (cbx + jx) + Px)) * p.inv_denom;
          eyn = (p.numer * ey + (dt * (cby + jy) + Py)) * p.inv_denom;
          ezn = (p.numer * ez + (dt * (cbz + jz) + Pz)) * p.inv_denom;
        } else {
          const double E2 = (double)ex * ex + (double)ey * ey + (double)ez * ez;
          const T f = p.numer + p.chi * T(E2);
          const T cx = (f * ex + dt * (cbx + jx) + Px) * p.inv_denom;
          const T cy = (f * ey + dt * (cby + jy) + Py) * p.inv_denom;
          const T cz = (f * ez + dt * (cbz + jz) + Pz) * p.inv_denom;
          const double C = sqrt((double)cx * cx + (double)cy * cy + (double)cz * cz);
          if (C > 0) {
            const double E = kerr_newton(sqrt(E2), p.chi_over_denom, C, p.newton_tol, p.newton_max, p.status);
            exn = T(E * cx / C);
            eyn = T(E * cy / C);
            ezn = T(E * cz / C);
          } else {
            exn = eyn = ezn = T(0);
          }
        }
      }
    }
    if (!finite3((double)exn, (double)eyn, (double)ezn)) atomicAdd(p.status + ST_NONFINITE, 1);
    // ---- all stores last
    Ex[base + col] = exn;
    Ey[base + col] = eyn;
    Ez[base + col] = ezn;
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) reinterpret_cast<T2 *>(p.psi[n][c])[pi] = q[n][c];
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!cin[f]) continue;
      p.cpml[f].psi0[cli[f]] = cp0[f];
      p.cpml[f].psi1[cli[f]] = cp1[f];
    }
    bx_km = bx;
    by_km = by;
  }
}

template <typename T>
__global__ void __launch_bounds__(256, MPB_B_MIN_BLOCKS) b_half_kernel(const BParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= p.nx || j >= p.ny) return;
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  if (k0 > k1) return;

  const long long plane = p.plane;
  const int ip = (i == p.nx - 1) ? 0 : i + 1;
  const int jp = (j == p.ny - 1) ? 0 : j + 1;
  const long long col = (long long)j * p.nx + i;
  const long long colxp = (long long)j * p.nx + ip;
  const long long colyp = (long long)jp * p.nx + i;
  const T *__restrict__ Ex = p.E[0];
  const T *__restrict__ Ey = p.E[1];
  const T *__restrict__ Ez = p.E[2];
  T *__restrict__ Bx = p.B[0];
  T *__restrict__ By = p.B[1];
  T *__restrict__ Bz = p.B[2];
  const T ikx = ld(p.ik[0] + i + 1);
  const T iky = ld(p.ik[1] + j + 1);
  const T iky_bz = ld(p.ik_bz_y + j + 1);
  const T dt = p.dt;

  T ex_k = ld(Ex + (long long)k0 * plane + col);
  T ey_k = ld(Ey + (long long)k0 * plane + col);

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    int kp = k + 1;
    if (p.zperiodic && kp == p.nz + 1) kp = 1;
    const long long basep = (long long)kp * plane;
    const T ex_kp = ld(Ex + basep + col), ey_kp = ld(Ey + basep + col);
    const T ez = ld(Ez + base + col);
    const T ez_xp = ld(Ez + base + colxp), ey_xp = ld(Ey + base + colxp);
    const T ez_yp = ld(Ez + base + colyp), ex_yp = ld(Ex + base + colyp);
    const T ikz = ld(p.ik[2] + k);
    // ---- all loads first (see e_half_kernel)
    const T bx = Bx[base + col], by = By[base + col], bz = Bz[base + col];
    T cp0[6], cp1[6], cb[6], cc[6];
    int cli[6];  // layer arrays hold < 2^31 cells (checked by mp_create)
    bool cin[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const CpmlFace<T> &F = p.cpml[f];
      const int idx = F.dim == 0 ? i + 1 : F.dim == 1 ? j + 1 : k;
      cin[f] = F.active && idx >= F.lo && idx <= F.hi;
      if (cin[f]) {
        if (F.dim == 2) cli[f] = ((k - F.lo) * p.ny + j) * p.nx + i;
        else if (F.dim == 0) cli[f] = ((k - F.zlo) * p.ny + j) * F.ex + (i + 1 - F.lo);
        else cli[f] = ((k - F.zlo) * F.ey + (j + 1 - F.lo)) * p.nx + i;
        cp0[f] = F.psi0[cli[f]];
        cp1[f] = F.psi1[cli[f]];
        cb[f] = ld(F.b + idx);
        cc[f] = ld(F.c + idx);
      }
    }
    T sa = T(0), sb = T(0);
    bool on_src = false;
    for (int s = 0; s < p.n_src; ++s) {
      if (k == p.src[s].plane) {
        sa = ld(p.src[s].v0 + col);
        sb = ld(p.src[s].v1 + col);
        on_src = true;
      }
    }

    // ---- H-side currents (cpml_border.cpp:499-527, incsource.t:112-145)
    T mx = T(0), my = T(0), mz = T(0);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!cin[f]) continue;
      const int dim = p.cpml[f].dim;
      T d0, d1;
      if (dim == 2) { d0 = ey_kp - ey_k; d1 = -(ex_kp - ex_k); }
      else if (dim == 0) { d0 = ez_xp - ez; d1 = -(ey_xp - ey_k); }
      else { d0 = ex_yp - ex_k; d1 = -(ez_yp - ez); }
      cp0[f] = cb[f] * cp0[f] + cc[f] * d0;
      cp1[f] = cb[f] * cp1[f] + cc[f] * d1;
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

    // ---- plrcStepB (fdtd_plrc.cpp:263-293), stores last
    Bx[base + col] = bx + dt * ((ey_kp - ey_k) * ikz - (ez_yp - ez) * iky + mx);
    By[base + col] = by + dt * ((ez_xp - ez) * ikx - (ex_kp - ex_k) * ikz + my);
    Bz[base + col] = bz + dt * ((ex_yp - ex_k) * iky_bz - (ey_xp - ey_k) * ikx + mz);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!cin[f]) continue;
      p.cpml[f].psi0[cli[f]] = cp0[f];
      p.cpml[f].psi1[cli[f]] = cp1[f];
    }
    ex_k = ex_kp;
    ey_k = ey_kp;
  }
}

// ---------------------------------------------------------------------------
// Launchers (called from mp_api.cu)

template <typename T>
static dim3 grid_for(int nx, int ny, int nk, int kchunk) {
  return dim3((nx + 31) / 32, (ny + 7) / 8, (nk + kchunk - 1) / kchunk);
}

template <typename T, int MODE>
static cudaError_t launch_e_np(const EParams<T> &p, int np, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  const dim3 g = grid_for<T>(p.nx, p.ny, nk, p.kchunk), b(32, 8, 1);
  switch (np) {
    case 0: e_half_kernel<T, MODE, 0><<<g, b, 0, st>>>(p); break;
    case 1: e_half_kernel<T, MODE, 1><<<g, b, 0, st>>>(p); break;
    case 2: e_half_kernel<T, MODE, 2><<<g, b, 0, st>>>(p); break;
    default: e_half_kernel<T, MODE, 3><<<g, b, 0, st>>>(p); break;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_e_half(const EParams<T> &p, int mode, int np, cudaStream_t st) {
  switch (mode) {
    case MODE_PLAIN: return launch_e_np<T, MODE_PLAIN>(p, 0, st);
    case MODE_NL: return launch_e_np<T, MODE_NL>(p, 0, st);
    case MODE_PLRC_LIN: return launch_e_np<T, MODE_PLRC_LIN>(p, np, st);
    default: return launch_e_np<T, MODE_PLRC_NONLIN>(p, np, st);
  }
}

template <typename T>
cudaError_t launch_b_half(const BParams<T> &p, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  b_half_kernel<T><<<grid_for<T>(p.nx, p.ny, nk, p.kchunk), dim3(32, 8, 1), 0, st>>>(p);
  return cudaGetLastError();
}

template cudaError_t launch_e_half<float>(const EParams<float> &, int, int, cudaStream_t);
template cudaError_t launch_e_half<double>(const EParams<double> &, int, int, cudaStream_t);
template cudaError_t launch_b_half<float>(const BParams<float> &, cudaStream_t);
template cudaError_t launch_b_half<double>(const BParams<double> &, cudaStream_t);

}  // namespace mpb
