// mp_step_kernels.cu - the two half-step kernels of one MPulse time step,
// global-load form (any grid size; mp_step_tma.cu has the TMA-staged form used
// when the tile divides the grid).
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
// Thread mapping: one thread per (x, y) column, 32 x 4 columns per block; a
// block marches up a chunk of z-planes so the z-neighbour of the previous plane
// is carried in registers and every field element is read from HBM once per
// half step (x/y neighbours are re-read through L1/L2).  The medium test, the
// CPML z-faces and the source planes depend on z only and are uniform per
// iteration.  The stencil has no contraction, so no tensor cores are involved;
// both kernels are HBM-bandwidth bound.
#include "mp_cell.cuh"

// Block shape 32 x BLOCK_Y columns (a warp is one row of 32 columns) and the
// minimum resident threads per SM asked of the register allocator, 768 (80
// registers).  Measured on the 256x256x512 PLRC + Kerr workload (FP32), with
// 32 x 8 blocks: E half 1.083 ms with no bound (114 registers), 0.917 ms with
// 768 threads (80 registers, 28 B spilled), 1.17 ms with 1024 (64 registers,
// more spills); 32 x 4 blocks then took the E half from 0.872 to 0.859 ms and
// the B half from 0.462 to 0.440 ms (32 x 2: no further gain).
#ifndef MPB_E_BLOCK_Y
#define MPB_E_BLOCK_Y 4
#endif
#ifndef MPB_B_BLOCK_Y
#define MPB_B_BLOCK_Y 4
#endif
#ifndef MPB_E_MIN_THREADS
#define MPB_E_MIN_THREADS 768
#endif
#ifndef MPB_B_MIN_THREADS
#define MPB_B_MIN_THREADS 768
#endif
// B half: issue the next plane's loads before the current plane's arithmetic.
#ifndef MPB_B_PREFETCH
#define MPB_B_PREFETCH 1
#endif

namespace mpb {

template <typename T, int MODE, int NP, bool DESIGN>
__global__ void __launch_bounds__(32 * MPB_E_BLOCK_Y, MPB_E_MIN_THREADS / (32 * MPB_E_BLOCK_Y))
    e_half_kernel(const EParams<T> p) {
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
  // CPML faces: the x / y faces of this warp's columns are fixed through the
  // z-march; warps with none skip the face code on planes outside the z faces
  const unsigned cmask = face_column_mask(p.cpml, i, j);
  const bool warp_xy = __any_sync(__activemask(), cmask != 0u);
  const int2 srck = source_plane_range(p);

  int km = k0 - 1;
  if (p.zperiodic && km == 0) km = p.nz;
  T bx_km = ld(Bx + km * plane + col);
  T by_km = ld(By + km * plane + col);

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    // ---- loads of this cell (the rest are in e_cell, still before any store)
    EIn<T> v;
    v.bx = ld(Bx + base + col);
    v.by = ld(By + base + col);
    v.bz = ld(Bz + base + col);
    v.bz_xm = ld(Bz + base + colxm);
    v.by_xm = ld(By + base + colxm);
    v.bz_ym = ld(Bz + base + colym);
    v.bx_ym = ld(Bx + base + colym);
    v.bx_km = bx_km;
    v.by_km = by_km;
    v.ex = Ex[base + col];
    v.ey = Ey[base + col];
    v.ez = Ez[base + col];
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
    T exn, eyn, ezn;
    if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
      e_cell<T, MODE, NP, DESIGN, true>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn);
    else
      e_cell<T, MODE, NP, DESIGN, false>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn);
    // ---- stores
    Ex[base + col] = exn;
    Ey[base + col] = eyn;
    Ez[base + col] = ezn;
    if (DESIGN && p.hist[0]) {
      p.hist[0][base + col] = exn;
      p.hist[1][base + col] = eyn;
      p.hist[2][base + col] = ezn;
    }
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) reinterpret_cast<T2 *>(p.psi[n][c])[pi] = q[n][c];
    }
    bx_km = v.bx;
    by_km = v.by;
  }
}

template <typename T>
__global__ void __launch_bounds__(32 * MPB_B_BLOCK_Y, MPB_B_MIN_THREADS / (32 * MPB_B_BLOCK_Y))
    b_half_kernel(const BParams<T> p) {
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
  const unsigned cmask = face_column_mask(p.cpml, i, j);
  const bool warp_xy = __any_sync(__activemask(), cmask != 0u);
  const int2 srck = source_plane_range(p);

  // loads of plane k (ex, ey of plane k are carried from the previous plane)
  auto load = [&](int k, T ex_k, T ey_k, BIn<T> &v) {
    const long long base = (long long)k * plane;
    int kp = k + 1;
    if (p.zperiodic && kp == p.nz + 1) kp = 1;
    const long long basep = (long long)kp * plane;
    v.ex = ex_k;
    v.ey = ey_k;
    v.ex_kp = ld(Ex + basep + col);
    v.ey_kp = ld(Ey + basep + col);
    v.ez = ld(Ez + base + col);
    v.ez_xp = ld(Ez + base + colxp);
    v.ey_xp = ld(Ey + base + colxp);
    v.ez_yp = ld(Ez + base + colyp);
    v.ex_yp = ld(Ex + base + colyp);
    v.bx = Bx[base + col];
    v.by = By[base + col];
    v.bz = Bz[base + col];
  };

  BIn<T> v;
  load(k0, ld(Ex + (long long)k0 * plane + col), ld(Ey + (long long)k0 * plane + col), v);
  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
#if MPB_B_PREFETCH
    // the next plane's loads go out before this plane's arithmetic and stores
    // (they never alias them: B of plane k+1, E is read-only here)
    BIn<T> vn;
    if (k < k1) load(k + 1, v.ex_kp, v.ey_kp, vn);
#endif
    const T ikz = ld(p.ik[2] + k);
    T bxn, byn, bzn;
    if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
      b_cell<T, true>(p, i, j, k, col, cmask, v, ikx, iky, iky_bz, ikz, bxn, byn, bzn);
    else
      b_cell<T, false>(p, i, j, k, col, cmask, v, ikx, iky, iky_bz, ikz, bxn, byn, bzn);
    Bx[base + col] = bxn;
    By[base + col] = byn;
    Bz[base + col] = bzn;
#if MPB_B_PREFETCH
    v = vn;
#else
    if (k < k1) load(k + 1, v.ex_kp, v.ey_kp, v);
#endif
  }
}

// ---------------------------------------------------------------------------
// Launchers (called from mp_api.cu)


template <typename T, int MODE, bool DESIGN>
static cudaError_t launch_e_np(const EParams<T> &p, int np, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  const dim3 g((p.nx + 31) / 32, (p.ny + MPB_E_BLOCK_Y - 1) / MPB_E_BLOCK_Y, (nk + p.kchunk - 1) / p.kchunk),
      b(32, MPB_E_BLOCK_Y, 1);
  switch (np) {
    case 0: e_half_kernel<T, MODE, 0, DESIGN><<<g, b, 0, st>>>(p); break;
    case 1: e_half_kernel<T, MODE, 1, DESIGN><<<g, b, 0, st>>>(p); break;
    case 2: e_half_kernel<T, MODE, 2, DESIGN><<<g, b, 0, st>>>(p); break;
    default: e_half_kernel<T, MODE, 3, DESIGN><<<g, b, 0, st>>>(p); break;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_e_half(const EParams<T> &p, int mode, int np, cudaStream_t st) {
  // design regions exist only with the PLRC solvers
  const bool design = p.design.x0 <= p.design.x1;
  switch (mode) {
    case MODE_PLAIN: return launch_e_np<T, MODE_PLAIN, false>(p, 0, st);
    case MODE_NL: return launch_e_np<T, MODE_NL, false>(p, 0, st);
    case MODE_PLRC_LIN:
      return design ? launch_e_np<T, MODE_PLRC_LIN, true>(p, np, st) : launch_e_np<T, MODE_PLRC_LIN, false>(p, np, st);
    default:
      return design ? launch_e_np<T, MODE_PLRC_NONLIN, true>(p, np, st)
                    : launch_e_np<T, MODE_PLRC_NONLIN, false>(p, np, st);
  }
}

template <typename T>
cudaError_t launch_b_half(const BParams<T> &p, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  const dim3 g((p.nx + 31) / 32, (p.ny + MPB_B_BLOCK_Y - 1) / MPB_B_BLOCK_Y, (nk + p.kchunk - 1) / p.kchunk);
  b_half_kernel<T><<<g, dim3(32, MPB_B_BLOCK_Y, 1), 0, st>>>(p);
  return cudaGetLastError();
}

template cudaError_t launch_e_half<float>(const EParams<float> &, int, int, cudaStream_t);
template cudaError_t launch_e_half<double>(const EParams<double> &, int, int, cudaStream_t);
template cudaError_t launch_b_half<float>(const BParams<float> &, cudaStream_t);
template cudaError_t launch_b_half<double>(const BParams<double> &, cudaStream_t);

}  // namespace mpb
