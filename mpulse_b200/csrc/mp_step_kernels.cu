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

#include <algorithm>

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
// FP32 E half: resident threads per SM (the FP64 form keeps MPB_E_MIN_THREADS).
// On the 256x256x512 workload with the pulse in the Kerr medium (FP32, where
// the E half is latency- and issue-bound) 1024 threads (64 registers, 40 B
// spilled) took the E half from 0.855 to 0.839 ms.
#ifndef MPB_E_MIN_THREADS_F
#define MPB_E_MIN_THREADS_F 1024
#endif
#ifndef MPB_B_MIN_THREADS
#define MPB_B_MIN_THREADS 768
#endif
// E half z-chunks: planes per block chosen for about this many blocks of
// 32 x MPB_E_BLOCK_Y columns per SM, so that the last, partly filled wave of
// blocks is a small part of the launch, and at least MPB_E_MIN_PLANES planes
// per block (the z-march carries the plane below in registers).  Measured on
// the 256x256x512 PLRC + Kerr workload with the pulse in the Kerr medium
// (FP32, E half): 103 planes per block (2560 blocks, 2.2 waves of the 1184
// resident) 0.847 ms, 47 / 32 / 23 / 16 / 8 planes 0.774 / 0.772 / 0.757 /
// 0.769 / 0.774 ms; blocks per SM 64 / 80 / 112: 0.765 / 0.758 / 0.753 ms.
// FP64 (768 resident threads), 103 planes 1.695 ms, 24 / 48 / 80 blocks per
// SM 1.632 / 1.563 / 1.540 ms.  On the 96^3 adjoint workload the forward run
// takes the same time with at least 1, 2, 4 or 8 planes per block (±3%).
#ifndef MPB_E_BLOCKS_PER_SM_F
#define MPB_E_BLOCKS_PER_SM_F 80
#endif
#ifndef MPB_E_BLOCKS_PER_SM_D
#define MPB_E_BLOCKS_PER_SM_D 80
#endif
#ifndef MPB_E_MIN_PLANES
#define MPB_E_MIN_PLANES 2
#endif
// B half: two cells per thread with vector loads along x where nx allows,
// with its own occupancy and z-chunks (half the threads), per precision.
// Measured on the 256x256x512 workload (FP32, B half): scalar kernel 0.440
// ms; four cells per thread (float4), 768 threads, chunks for 24 blocks per SM
// 0.354 ms; two cells per thread (float2) with 768 / 1024 / 1280 / 1536
// threads 0.335 / 0.293 / 0.304 / 0.302 ms, 1024 threads and 32 / 48 blocks
// per SM 0.290 / 0.285 ms (32 x 2 blocks: 0.284 ms, 32 x 8: 0.307 ms).  FP64 (double2), B half with 512 / 640 / 768 / 1024 threads:
// 0.553 / 0.488 / 0.538 / 0.560 ms.  Re-measured with the pulse in the Kerr
// medium and the E half's z-chunks for 80 blocks per SM: FP32 48 / 80 / 128
// blocks per SM 0.295 / 0.281 / 0.286 ms, FP64 24 / 48 / 80 blocks per SM
// 0.510 / 0.495 / 0.468 ms; at least 4 instead of 8 planes per block: no
// change.
#ifndef MPB_B_VECTOR
#define MPB_B_VECTOR 1
#endif
#ifndef MPB_BV_MIN_THREADS_F
#define MPB_BV_MIN_THREADS_F 1024
#endif
#ifndef MPB_BV_MIN_THREADS_D
#define MPB_BV_MIN_THREADS_D 640
#endif
#ifndef MPB_BV_BLOCKS_PER_SM_F
#define MPB_BV_BLOCKS_PER_SM_F 80
#endif
#ifndef MPB_BV_BLOCKS_PER_SM_D
#define MPB_BV_BLOCKS_PER_SM_D 80
#endif
#ifndef MPB_BV_MIN_PLANES
#define MPB_BV_MIN_PLANES 8
#endif
// B half, scalar kernel: issue the next plane's loads before the current
// plane's arithmetic.
#ifndef MPB_B_PREFETCH
#define MPB_B_PREFETCH 1
#endif

namespace mpb {

// Whether the adjoint history of cell (i, j, k) is stored (EParams::hist_box).
template <typename T>
__device__ __forceinline__ bool hist_cell(const EParams<T> &p, int i, int j, int k) {
  if (p.hist_all) return true;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const int *h = p.hist_box[b];
    if (i >= h[0] && i <= h[1] && j >= h[2] && j <= h[3] && k >= h[4] && k <= h[5]) return true;
  }
  return false;
}

template <typename T, int MODE, int NP, bool DESIGN, bool PLASMA = false>
__global__ void __launch_bounds__(32 * MPB_E_BLOCK_Y,
                                  (sizeof(T) == 4 ? MPB_E_MIN_THREADS_F : MPB_E_MIN_THREADS) / (32 * MPB_E_BLOCK_Y))
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
  const long long nf = p.n_field;
  int *const st = p.status;
  T bx_km = ldg_c(Bx, km * plane + col, nf, st);
  T by_km = ldg_c(By, km * plane + col, nf, st);
  KerrCount kc;

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    // ---- loads of this cell (the rest are in e_cell, still before any store)
    EIn<T> v;
    v.bx = ldg_c(Bx, base + col, nf, st);
    v.by = ldg_c(By, base + col, nf, st);
    v.bz = ldg_c(Bz, base + col, nf, st);
    v.bz_xm = ldg_c(Bz, base + colxm, nf, st);
    v.by_xm = ldg_c(By, base + colxm, nf, st);
    v.bz_ym = ldg_c(Bz, base + colym, nf, st);
    v.bx_ym = ldg_c(Bx, base + colym, nf, st);
    v.bx_km = bx_km;
    v.by_km = by_km;
    v.ex = ld_c(Ex, base + col, nf, st);
    v.ey = ld_c(Ey, base + col, nf, st);
    v.ez = ld_c(Ez, base + col, nf, st);
    const T ikz = ld(p.ik[2] + k);
    const bool med = (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) && k >= p.mz0 && k <= p.mz1;
    const long long pi = ((long long)(k - p.mz0) * p.ny + j) * p.nx + i;
    T2 q[NP > 0 ? NP : 1][3];
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) q[n][c] = ld_c(reinterpret_cast<const T2 *>(p.psi[n][c]), pi, p.n_psi, st);
    }
    PlasmaCell<T> pc;
    if (PLASMA) {
      const T r0 = ld_c(p.rho, base + col, nf, st);
      T j0 = T(0), j1 = T(0), j2 = T(0);
      if (p.pl_current) {
        j0 = ld_c(p.pj[0], base + col, nf, st);
        j1 = ld_c(p.pj[1], base + col, nf, st);
        j2 = ld_c(p.pj[2], base + col, nf, st);
      }
      plasma_cell(p, v.ex, v.ey, v.ez, r0, j0, j1, j2, pc);
    }
    T exn, eyn, ezn;
    if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
      e_cell<T, MODE, NP, DESIGN, true, PLASMA>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn, kc,
                                                &pc);
    else
      e_cell<T, MODE, NP, DESIGN, false, PLASMA>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn,
                                                 kc, &pc);
    // ---- stores
    st_c(Ex, base + col, nf, st, exn);
    st_c(Ey, base + col, nf, st, eyn);
    st_c(Ez, base + col, nf, st, ezn);
    if (PLASMA) {
      st_c(p.rho, base + col, nf, st, pc.rho);
      if (p.pl_current) {
        st_c(p.pj[0], base + col, nf, st, pc.j[0]);
        st_c(p.pj[1], base + col, nf, st, pc.j[1]);
        st_c(p.pj[2], base + col, nf, st, pc.j[2]);
      }
    }
    if (DESIGN && p.hist[0] && hist_cell(p, i, j, k)) {
      st_c(p.hist[0], base + col, nf, st, exn);
      st_c(p.hist[1], base + col, nf, st, eyn);
      st_c(p.hist[2], base + col, nf, st, ezn);
    }
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) st_c(reinterpret_cast<T2 *>(p.psi[n][c]), pi, p.n_psi, st, q[n][c]);
    }
    bx_km = v.bx;
    by_km = v.by;
  }
  flush_kerr_count<MODE>(p.kerr_count, kc);
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
  const long long nf = p.n_field;
  int *const st = p.status;
  auto load = [&](int k, T ex_k, T ey_k, BIn<T> &v) {
    const long long base = (long long)k * plane;
    int kp = k + 1;
    if (p.zperiodic && kp == p.nz + 1) kp = 1;
    const long long basep = (long long)kp * plane;
    v.ex = ex_k;
    v.ey = ey_k;
    v.ex_kp = ldg_c(Ex, basep + col, nf, st);
    v.ey_kp = ldg_c(Ey, basep + col, nf, st);
    v.ez = ldg_c(Ez, base + col, nf, st);
    v.ez_xp = ldg_c(Ez, base + colxp, nf, st);
    v.ey_xp = ldg_c(Ey, base + colxp, nf, st);
    v.ez_yp = ldg_c(Ez, base + colyp, nf, st);
    v.ex_yp = ldg_c(Ex, base + colyp, nf, st);
    v.bx = ld_c(Bx, base + col, nf, st);
    v.by = ld_c(By, base + col, nf, st);
    v.bz = ld_c(Bz, base + col, nf, st);
  };

  BIn<T> v;
  load(k0, ldg_c(Ex, (long long)k0 * plane + col, nf, st), ldg_c(Ey, (long long)k0 * plane + col, nf, st), v);
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
    st_c(Bx, base + col, nf, st, bxn);
    st_c(By, base + col, nf, st, byn);
    st_c(Bz, base + col, nf, st, bzn);
#if MPB_B_PREFETCH
    v = vn;
#else
    if (k < k1) load(k + 1, v.ex_kp, v.ey_kp, v);
#endif
  }
}

// The B half with vector loads along x: each thread owns V = 2 consecutive
// cells of a row (nx a multiple of 64), so a plane's loads are 8 float2 /
// double2 vectors and two scalars (the x+1 neighbour of the second cell), and
// the z+1 plane of E is carried to the next plane.  The CPML faces add their
// currents cell by cell (y faces hold whole rows, x faces single cells, z
// faces whole planes).
template <typename T> struct VecB;
template <> struct VecB<float> { typedef float2 type; };
template <> struct VecB<double> { typedef double2 type; };
constexpr int kBV = 2;  // cells per thread

template <typename T>
struct RowV {
  T v[kBV];
};

template <typename T>
__device__ __forceinline__ RowV<T> ldv(const T *p) {
  typedef typename VecB<T>::type VT;
  const VT x = __ldg(reinterpret_cast<const VT *>(p));
  RowV<T> r;
  memcpy(r.v, &x, sizeof(VT));
  return r;
}

template <typename T>
__device__ __forceinline__ RowV<T> ldv_rw(const T *p) {
  typedef typename VecB<T>::type VT;
  const VT x = *reinterpret_cast<const VT *>(p);
  RowV<T> r;
  memcpy(r.v, &x, sizeof(VT));
  return r;
}

template <typename T>
__device__ __forceinline__ void stv(T *p, const RowV<T> &r) {
  typedef typename VecB<T>::type VT;
  VT x;
  memcpy(&x, r.v, sizeof(VT));
  *reinterpret_cast<VT *>(p) = x;
}

// The vector accesses at element i of an array of n elements, checked like
// ldg_c / ld_c / st_c (both elements must lie inside).
template <typename T>
__device__ __forceinline__ RowV<T> ldv_c(const T *a, long long i, long long n, int *status) {
  if (in_bounds(i + kBV - 1, n, status) && in_bounds(i, n, status)) return ldv(a + i);
  RowV<T> r;
#pragma unroll
  for (int c = 0; c < kBV; ++c) r.v[c] = T(0);
  return r;
}
template <typename T>
__device__ __forceinline__ RowV<T> ldv_rw_c(const T *a, long long i, long long n, int *status) {
  if (in_bounds(i + kBV - 1, n, status) && in_bounds(i, n, status)) return ldv_rw(a + i);
  RowV<T> r;
#pragma unroll
  for (int c = 0; c < kBV; ++c) r.v[c] = T(0);
  return r;
}
template <typename T>
__device__ __forceinline__ void stv_c(T *a, long long i, long long n, int *status, const RowV<T> &r) {
  if (in_bounds(i + kBV - 1, n, status) && in_bounds(i, n, status)) stv(a + i, r);
}

// psi_H of the face in slot F at one cell (cpml_border.cpp:499-527): updates
// the layer arrays and adds the face's currents to m (MPulse's order: slots
// in turn, as b_cell sums them).  d0 / d1: the differences of E along the
// face's axis for psi0 / psi1.
template <typename T, int F>
__device__ __forceinline__ void b_face(const BParams<T> &p, int i, int j, int k, T d0, T d1, T (&m)[3]) {
  constexpr int dim = face_axis(F);
  const CpmlFace<T> &L = p.cpml[F];
  const int idx = dim == 0 ? i + 1 : dim == 1 ? j + 1 : k;
  int li;
  if (dim == 2) li = ((k - L.lo) * p.ny + j) * p.nx + i;
  else if (dim == 0) li = ((k - L.zlo) * p.ny + j) * L.ex + (i + 1 - L.lo);
  else li = ((k - L.zlo) * L.ey + (j + 1 - L.lo)) * p.nx + i;
  const T b = ld(L.b + idx), c = ld(L.c + idx);
  const T c0 = b * ld_c(L.psi0, li, L.n, p.status) + c * d0;
  const T c1 = b * ld_c(L.psi1, li, L.n, p.status) + c * d1;
  st_c(L.psi0, li, L.n, p.status, c0);
  st_c(L.psi1, li, L.n, p.status, c1);
  if (dim == 2) { m[0] += c0; m[1] += c1; }
  else if (dim == 0) { m[1] += c0; m[2] += c1; }
  else { m[2] += c0; m[0] += c1; }
}

template <typename T>
__global__ void __launch_bounds__(32 * MPB_B_BLOCK_Y,
                                  (sizeof(T) == 4 ? MPB_BV_MIN_THREADS_F : MPB_BV_MIN_THREADS_D) / (32 * MPB_B_BLOCK_Y))
    b_half_vec_kernel(const BParams<T> p) {
  constexpr int V = kBV;
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i0 >= p.nx || j >= p.ny) return;
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  if (k0 > k1) return;

  const long long plane = p.plane;
  const int jp = (j == p.ny - 1) ? 0 : j + 1;
  const int il = (i0 + V == p.nx) ? 0 : i0 + V;  // x+1 of the last cell
  const long long col = (long long)j * p.nx + i0;
  const long long colyp = (long long)jp * p.nx + i0;
  const long long colxl = (long long)j * p.nx + il;
  const T *__restrict__ Ex = p.E[0];
  const T *__restrict__ Ey = p.E[1];
  const T *__restrict__ Ez = p.E[2];
  T *__restrict__ Bx = p.B[0];
  T *__restrict__ By = p.B[1];
  T *__restrict__ Bz = p.B[2];
  T ikx[V];
#pragma unroll
  for (int c = 0; c < V; ++c) ikx[c] = ld(p.ik[0] + i0 + c + 1);
  const T iky = ld(p.ik[1] + j + 1);
  const T iky_bz = ld(p.ik_bz_y + j + 1);
  // y faces (slots 0, 1) hold whole rows: warp-uniform; x faces (slots 2, 3)
  // per cell, bits 2c and 2c + 1
  const unsigned ybits = face_column_mask(p.cpml, i0, j) & 3u;
  unsigned xbits = 0;
#pragma unroll
  for (int c = 0; c < V; ++c) xbits |= ((face_column_mask(p.cpml, i0 + c, j) >> 2) & 3u) << (2 * c);
  const int2 srck = source_plane_range(p);

  const long long nf = p.n_field;
  int *const st = p.status;
  RowV<T> ex = ldv_c(Ex, (long long)k0 * plane + col, nf, st), ey = ldv_c(Ey, (long long)k0 * plane + col, nf, st);
  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    int kp = k + 1;
    if (p.zperiodic && kp == p.nz + 1) kp = 1;
    const long long basep = (long long)kp * plane;
    // ---- every load of this plane first
    const RowV<T> ex_kp = ldv_c(Ex, basep + col, nf, st), ey_kp = ldv_c(Ey, basep + col, nf, st);
    const RowV<T> ez = ldv_c(Ez, base + col, nf, st);
    const T ez_xl = ldg_c(Ez, base + colxl, nf, st), ey_xl = ldg_c(Ey, base + colxl, nf, st);
    const RowV<T> ez_yp = ldv_c(Ez, base + colyp, nf, st), ex_yp = ldv_c(Ex, base + colyp, nf, st);
    const RowV<T> bx = ldv_rw_c(Bx, base + col, nf, st), by = ldv_rw_c(By, base + col, nf, st),
                  bz = ldv_rw_c(Bz, base + col, nf, st);
    const T ikz = ld(p.ik[2] + k);
    // ---- H-side currents, in MPulse's order: faces by slot, then the injector
    T m[V][3];
#pragma unroll
    for (int c = 0; c < V; ++c) m[c][0] = m[c][1] = m[c][2] = T(0);
    if (ybits) {
#pragma unroll
      for (int c = 0; c < V; ++c) {
        const T d0 = ex_yp.v[c] - ex.v[c], d1 = -(ez_yp.v[c] - ez.v[c]);
        if (ybits & 1u) b_face<T, 0>(p, i0 + c, j, k, d0, d1, m[c]);
        if (ybits & 2u) b_face<T, 1>(p, i0 + c, j, k, d0, d1, m[c]);
      }
    }
    if (xbits) {
#pragma unroll
      for (int c = 0; c < V; ++c) {
        const T ezx = c + 1 < V ? ez.v[c + 1 < V ? c + 1 : 0] : ez_xl;
        const T eyx = c + 1 < V ? ey.v[c + 1 < V ? c + 1 : 0] : ey_xl;
        const T d0 = ezx - ez.v[c], d1 = -(eyx - ey.v[c]);
        if (xbits & (1u << (2 * c))) b_face<T, 2>(p, i0 + c, j, k, d0, d1, m[c]);
        if (xbits & (2u << (2 * c))) b_face<T, 3>(p, i0 + c, j, k, d0, d1, m[c]);
      }
    }
    if (z_face_plane(p.cpml, k)) {
      const bool z4 = p.cpml[4].active && k >= p.cpml[4].lo && k <= p.cpml[4].hi;
      const bool z5 = p.cpml[5].active && k >= p.cpml[5].lo && k <= p.cpml[5].hi;
#pragma unroll
      for (int c = 0; c < V; ++c) {
        const T d0 = ey_kp.v[c] - ey.v[c], d1 = -(ex_kp.v[c] - ex.v[c]);
        if (z4) b_face<T, 4>(p, i0 + c, j, k, d0, d1, m[c]);
        if (z5) b_face<T, 5>(p, i0 + c, j, k, d0, d1, m[c]);
      }
    }
    if (k >= srck.x && k <= srck.y) {
      for (int s = 0; s < p.n_src; ++s) {
        if (k != p.src[s].plane) continue;
#pragma unroll
        for (int c = 0; c < V; ++c) {
          const T sa = ldg_c(p.src[s].v0, col + c, p.plane, st), sb = ldg_c(p.src[s].v1, col + c, p.plane, st);
          for (int q = 0; q < p.src_mult; ++q) {
            m[c][0] += sa;
            m[c][1] += sb;
          }
        }
      }
    }
    // ---- plrcStepB (fdtd_plrc.cpp:263-293)
    const T dt = p.dt;
    RowV<T> bxn, byn, bzn;
#pragma unroll
    for (int c = 0; c < V; ++c) {
      const T ezx = c + 1 < V ? ez.v[c + 1 < V ? c + 1 : 0] : ez_xl;
      const T eyx = c + 1 < V ? ey.v[c + 1 < V ? c + 1 : 0] : ey_xl;
      // (the sums of two products are left to the compiler here: spelled out
      // as in b_cell they cost this kernel six registers and 7% of its time;
      // the results agree with b_cell's to the last bit or within rounding)
      bxn.v[c] = bx.v[c] + dt_mul(dt, p.dt_lo, (ey_kp.v[c] - ey.v[c]) * ikz - (ez_yp.v[c] - ez.v[c]) * iky + m[c][0]);
      byn.v[c] = by.v[c] + dt_mul(dt, p.dt_lo, (ezx - ez.v[c]) * ikx[c] - (ex_kp.v[c] - ex.v[c]) * ikz + m[c][1]);
      bzn.v[c] = bz.v[c] + dt_mul(dt, p.dt_lo, (ex_yp.v[c] - ex.v[c]) * iky_bz - (eyx - ey.v[c]) * ikx[c] + m[c][2]);
    }
    stv_c(Bx, base + col, nf, st, bxn);
    stv_c(By, base + col, nf, st, byn);
    stv_c(Bz, base + col, nf, st, bzn);
    ex = ex_kp;
    ey = ey_kp;
  }
}

// ---------------------------------------------------------------------------
// Launchers (called from mp_api.cu)


template <typename T, int MODE, bool DESIGN, bool PLASMA = false>
static cudaError_t launch_e_np(const EParams<T> &p, int np, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  const long long bxy = (long long)((p.nx + 31) / 32) * ((p.ny + MPB_E_BLOCK_Y - 1) / MPB_E_BLOCK_Y);
  const long long per_sm = sizeof(T) == 4 ? MPB_E_BLOCKS_PER_SM_F : MPB_E_BLOCKS_PER_SM_D;
  const long long chunks = std::max(1LL, (148LL * per_sm + bxy - 1) / bxy);
  EParams<T> q = p;
  q.kchunk = int(std::min<long long>(nk, std::max<long long>(MPB_E_MIN_PLANES, (nk + chunks - 1) / chunks)));
  const dim3 g((p.nx + 31) / 32, (p.ny + MPB_E_BLOCK_Y - 1) / MPB_E_BLOCK_Y, (nk + q.kchunk - 1) / q.kchunk),
      b(32, MPB_E_BLOCK_Y, 1);
  switch (np) {
    case 0: e_half_kernel<T, MODE, 0, DESIGN, PLASMA><<<g, b, 0, st>>>(q); break;
    case 1: e_half_kernel<T, MODE, 1, DESIGN, PLASMA><<<g, b, 0, st>>>(q); break;
    case 2: e_half_kernel<T, MODE, 2, DESIGN, PLASMA><<<g, b, 0, st>>>(q); break;
    default: e_half_kernel<T, MODE, 3, DESIGN, PLASMA><<<g, b, 0, st>>>(q); break;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_e_half(const EParams<T> &p, int mode, int np, cudaStream_t st) {
  // design regions and the plasma plug-ins exist only with the PLRC solvers
  // (and not together)
  const bool design = p.design.x0 <= p.design.x1;
  const bool plasma = p.rho != nullptr;
  switch (mode) {
    case MODE_PLAIN: return launch_e_np<T, MODE_PLAIN, false>(p, 0, st);
    case MODE_NL: return launch_e_np<T, MODE_NL, false>(p, 0, st);
    case MODE_PLRC_LIN:
      return design   ? launch_e_np<T, MODE_PLRC_LIN, true>(p, np, st)
             : plasma ? launch_e_np<T, MODE_PLRC_LIN, false, true>(p, np, st)
                      : launch_e_np<T, MODE_PLRC_LIN, false>(p, np, st);
    default:
      return design   ? launch_e_np<T, MODE_PLRC_NONLIN, true>(p, np, st)
             : plasma ? launch_e_np<T, MODE_PLRC_NONLIN, false, true>(p, np, st)
                      : launch_e_np<T, MODE_PLRC_NONLIN, false>(p, np, st);
  }
}

template <typename T>
cudaError_t launch_b_half(const BParams<T> &p, cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
#if MPB_B_VECTOR
  constexpr int V = kBV;
  // rows of whole warps only: on narrow grids (nx = 96: 48 threads a row)
  // the scalar kernel keeps every lane busy
  if (p.nx % (32 * V) == 0) {
    // V cells per thread: z-chunks sized for a number of blocks per SM, at
    // least 8 planes each
    const int tx = p.nx / V;
    const long long per_sm = sizeof(T) == 4 ? MPB_BV_BLOCKS_PER_SM_F : MPB_BV_BLOCKS_PER_SM_D;
    const long long bxy = (long long)(tx / 32) * ((p.ny + MPB_B_BLOCK_Y - 1) / MPB_B_BLOCK_Y);
    const long long chunks = std::max(1LL, (148LL * per_sm + bxy - 1) / bxy);
    BParams<T> q = p;
    q.kchunk = int(std::max<long long>(MPB_BV_MIN_PLANES, (nk + chunks - 1) / chunks));
    const dim3 g((tx + 31) / 32, (p.ny + MPB_B_BLOCK_Y - 1) / MPB_B_BLOCK_Y, (nk + q.kchunk - 1) / q.kchunk);
    b_half_vec_kernel<T><<<g, dim3(32, MPB_B_BLOCK_Y, 1), 0, st>>>(q);
    return cudaGetLastError();
  }
#endif
  const dim3 g((p.nx + 31) / 32, (p.ny + MPB_B_BLOCK_Y - 1) / MPB_B_BLOCK_Y, (nk + p.kchunk - 1) / p.kchunk);
  b_half_kernel<T><<<g, dim3(32, MPB_B_BLOCK_Y, 1), 0, st>>>(p);
  return cudaGetLastError();
}

template cudaError_t launch_e_half<float>(const EParams<float> &, int, int, cudaStream_t);
template cudaError_t launch_e_half<double>(const EParams<double> &, int, int, cudaStream_t);
template cudaError_t launch_b_half<float>(const BParams<float> &, cudaStream_t);
template cudaError_t launch_b_half<double>(const BParams<double> &, cudaStream_t);

}  // namespace mpb
