// mp_step_fused.cu - one MPulse time step as one z-march: the E half and the
// B half of a block's tile of columns in the same pass, so that the B half
// reads neither E nor B back from HBM for most cells.
//
// A block owns a tile of 32 x MPB_F_BLOCK_Y columns (a warp is one row) and a
// chunk of E planes k0..k1.  At plane k it runs the E half of its cells
// (e_cell, as e_half_kernel does), keeps the new E of the plane in a ring of
// three planes in shared memory, and then runs the B half of plane k - 1
// (b_cell, as the B-half kernels do): B at plane k - 1 needs the new E at
// k - 1 (own cell, x + 1, y + 1: from the ring) and at k (own cell: just
// computed), and the old B of its own cell (loaded again: it is still in L1 or
// L2 from the E half of plane k - 1).
//
// The state is updated in place, so a block must not write an old value that
// another block still reads, and must not read a new E from another block.
// Both hold when the block leaves out the B half of (a) the last column and
// the last row of its tile, whose x + 1 / y + 1 neighbours belong to other
// tiles (and whose old B those tiles' E halves read as their x - 1 / y - 1
// neighbours), and (b) its top plane k1, which needs the new E of k1 + 1 and
// whose old B the block above reads as the z - 1 neighbour.  The cells left
// out are updated afterwards by b_border_kernel from global memory: the
// tiles' last rows and last columns over all planes, and the top plane of
// every chunk.  Every cell of the B half is updated exactly once, by the
// same b_cell arithmetic, so the results equal those of the two half-step
// kernels bit for bit.
//
// One __syncthreads per plane: the ring has three slots, so the slot written
// at plane k + 1 is not the one read at plane k, and the one written at k + 2
// is read at k only before the barrier of k + 1.
#include "mp_cell.cuh"

#include <algorithm>

// Tile height, resident threads per SM asked of the register allocator, and
// z-chunks sized for about MPB_F_BLOCKS_PER_SM blocks per SM (at least
// MPB_F_MIN_PLANES planes: each chunk's top plane goes to the border kernel).
#ifndef MPB_F_BLOCK_Y
#define MPB_F_BLOCK_Y 8
#endif
#ifndef MPB_F_MIN_THREADS_F
#define MPB_F_MIN_THREADS_F 1024
#endif
#ifndef MPB_F_MIN_THREADS_D
#define MPB_F_MIN_THREADS_D 768
#endif
#ifndef MPB_F_BLOCKS_PER_SM
#define MPB_F_BLOCKS_PER_SM 40
#endif
#ifndef MPB_F_MIN_PLANES
#define MPB_F_MIN_PLANES 8
#endif

namespace mpb {

// Chunks of the fused launch: E planes k_first.. in chunks of kchunk.
struct FusedChunks {
  int kchunk, nchunks;
};

template <typename T, int MODE, int NP>
__global__ void __launch_bounds__(32 * MPB_F_BLOCK_Y,
                                  (sizeof(T) == 4 ? MPB_F_MIN_THREADS_F : MPB_F_MIN_THREADS_D) / (32 * MPB_F_BLOCK_Y))
    step_fused_kernel(const EParams<T> p, const BParams<T> q) {
  typedef typename Vec2<T>::type T2;
  constexpr int BY = MPB_F_BLOCK_Y;
  __shared__ T ring[3][3][BY][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx;
  const int j = blockIdx.y * BY + ty;
  const bool act = i < p.nx && j < p.ny;  // threads off the grid keep to the barriers
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  // this thread's B cells: off the tile's last row and column (and off the
  // grid's last row and column, whose neighbours wrap)
  const bool bown = act && tx != 31 && ty != BY - 1 && i != p.nx - 1 && j != p.ny - 1;

  const long long plane = p.plane;
  const int ia = act ? i : 0, ja = act ? j : 0;
  const int im = (ia == 0) ? p.nx - 1 : ia - 1;
  const int jm = (ja == 0) ? p.ny - 1 : ja - 1;
  // offsets inside a plane (a plane holds fewer than 2^31 cells)
  const int col = ja * p.nx + ia, colxm = ja * p.nx + im, colym = jm * p.nx + ia;
  // B is written in this kernel too: plain (coherent) loads, no __restrict__
  const T *Bx = p.B[0];
  const T *By = p.B[1];
  const T *Bz = p.B[2];
  T *Ex = p.E[0];
  T *Ey = p.E[1];
  T *Ez = p.E[2];
  const T ikx = ld(p.ik[0] + ia + 1);
  const T iky = ld(p.ik[1] + ja + 1);
  const unsigned cmask = act ? face_column_mask(p.cpml, ia, ja) : 0u;
  const bool warp_xy = __any_sync(0xffffffffu, cmask != 0u);
  const int2 srck = source_plane_range(p);
  // the B side's faces (its coefficient lines and injection planes are read
  // where used: fewer registers live through the march)
  const unsigned hmask = act ? face_column_mask(q.cpml, ia, ja) : 0u;
  const bool warp_xy_h = __any_sync(0xffffffffu, hmask != 0u);

  int km = k0 - 1;
  if (p.zperiodic && km == 0) km = p.nz;
  const long long nf = p.n_field;
  int *const st = p.status;
  T bx_km = T(0), by_km = T(0);
  if (act) {
    bx_km = ld_c(Bx, km * plane + col, nf, st);
    by_km = ld_c(By, km * plane + col, nf, st);
  }
  KerrCount kc;

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * plane;
    const int slot = (k - k0) % 3;
    T exn = T(0), eyn = T(0), ezn = T(0);
    EIn<T> v;
    if (act) {
      // ---- the E half of this cell at plane k (e_half_kernel's body)
      v.bx = ld_c(Bx, base + col, nf, st);
      v.by = ld_c(By, base + col, nf, st);
      v.bz = ld_c(Bz, base + col, nf, st);
      v.bz_xm = ld_c(Bz, base + colxm, nf, st);
      v.by_xm = ld_c(By, base + colxm, nf, st);
      v.bz_ym = ld_c(Bz, base + colym, nf, st);
      v.bx_ym = ld_c(Bx, base + colym, nf, st);
      v.bx_km = bx_km;
      v.by_km = by_km;
      v.ex = ld_c(Ex, base + col, nf, st);
      v.ey = ld_c(Ey, base + col, nf, st);
      v.ez = ld_c(Ez, base + col, nf, st);
      const T ikz = ld(p.ik[2] + k);
      const bool med = (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) && k >= p.mz0 && k <= p.mz1;
      const long long pi = ((long long)(k - p.mz0) * p.ny + ja) * p.nx + ia;
      T2 qq[NP > 0 ? NP : 1][3];
      if (NP > 0 && med) {
#pragma unroll
        for (int n = 0; n < NP; ++n)
#pragma unroll
          for (int c = 0; c < 3; ++c) qq[n][c] = ld_c(reinterpret_cast<const T2 *>(p.psi[n][c]), pi, p.n_psi, st);
      }
      if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
        e_cell<T, MODE, NP, false, true>(p, ia, ja, k, col, med, cmask, v, ikx, iky, ikz, qq, exn, eyn, ezn, kc);
      else
        e_cell<T, MODE, NP, false, false>(p, ia, ja, k, col, med, cmask, v, ikx, iky, ikz, qq, exn, eyn, ezn, kc);
      st_c(Ex, base + col, nf, st, exn);
      st_c(Ey, base + col, nf, st, eyn);
      st_c(Ez, base + col, nf, st, ezn);
      if (NP > 0 && med) {
#pragma unroll
        for (int n = 0; n < NP; ++n)
#pragma unroll
          for (int c = 0; c < 3; ++c) st_c(reinterpret_cast<T2 *>(p.psi[n][c]), pi, p.n_psi, st, qq[n][c]);
      }
      bx_km = v.bx;
      by_km = v.by;
    }
    ring[slot][0][ty][tx] = exn;
    ring[slot][1][ty][tx] = eyn;
    ring[slot][2][ty][tx] = ezn;
    __syncthreads();
    // ---- the B half of this cell at plane k - 1: the new E of that plane
    // from the ring, its old B again from global memory (no other thread
    // writes it; L1 / L2 still hold it from the E half of plane k - 1)
    const int kb = k - 1;
    if (k > k0 && bown && kb >= q.k_first && kb <= q.k_last) {
      const int ps = (k - 1 - k0) % 3;
      const long long bb = (long long)kb * plane + col;
      BIn<T> w;
      w.bx = ld_c(q.B[0], bb, nf, st);
      w.by = ld_c(q.B[1], bb, nf, st);
      w.bz = ld_c(q.B[2], bb, nf, st);
      w.ex = ring[ps][0][ty][tx];
      w.ey = ring[ps][1][ty][tx];
      w.ez = ring[ps][2][ty][tx];
      w.ez_xp = ring[ps][2][ty][tx + 1];
      w.ey_xp = ring[ps][1][ty][tx + 1];
      w.ez_yp = ring[ps][2][ty + 1][tx];
      w.ex_yp = ring[ps][0][ty + 1][tx];
      w.ex_kp = ring[slot][0][ty][tx];
      w.ey_kp = ring[slot][1][ty][tx];
      const T hkx = ld(q.ik[0] + ia + 1), hky = ld(q.ik[1] + ja + 1), hky_bz = ld(q.ik_bz_y + ja + 1);
      const T hkz = ld(q.ik[2] + kb);
      const int2 srch = source_plane_range(q);
      T bxn, byn, bzn;
      if (warp_xy_h || z_face_plane(q.cpml, kb) || (kb >= srch.x && kb <= srch.y))
        b_cell<T, true>(q, ia, ja, kb, col, hmask, w, hkx, hky, hky_bz, hkz, bxn, byn, bzn);
      else
        b_cell<T, false>(q, ia, ja, kb, col, hmask, w, hkx, hky, hky_bz, hkz, bxn, byn, bzn);
      st_c(q.B[0], bb, nf, st, bxn);
      st_c(q.B[1], bb, nf, st, byn);
      st_c(q.B[2], bb, nf, st, bzn);
    }
  }
  flush_kerr_count<MODE>(p.kerr_count, kc);
}

// The B half of one cell from global memory (b_half_kernel's loads and
// b_cell).
template <typename T>
__device__ __forceinline__ void b_cell_global(const BParams<T> &q, int i, int j, int k) {
  const long long plane = q.plane;
  const int ip = (i == q.nx - 1) ? 0 : i + 1;
  const int jp = (j == q.ny - 1) ? 0 : j + 1;
  const long long col = (long long)j * q.nx + i;
  const long long colxp = (long long)j * q.nx + ip;
  const long long colyp = (long long)jp * q.nx + i;
  int kp = k + 1;
  if (q.zperiodic && kp == q.nz + 1) kp = 1;
  const long long base = (long long)k * plane, basep = (long long)kp * plane;
  const long long nf = q.n_field;
  int *const st = q.status;
  BIn<T> v;
  v.ex = ldg_c(q.E[0], base + col, nf, st);
  v.ey = ldg_c(q.E[1], base + col, nf, st);
  v.ez = ldg_c(q.E[2], base + col, nf, st);
  v.ex_kp = ldg_c(q.E[0], basep + col, nf, st);
  v.ey_kp = ldg_c(q.E[1], basep + col, nf, st);
  v.ez_xp = ldg_c(q.E[2], base + colxp, nf, st);
  v.ey_xp = ldg_c(q.E[1], base + colxp, nf, st);
  v.ez_yp = ldg_c(q.E[2], base + colyp, nf, st);
  v.ex_yp = ldg_c(q.E[0], base + colyp, nf, st);
  v.bx = ld_c(q.B[0], base + col, nf, st);
  v.by = ld_c(q.B[1], base + col, nf, st);
  v.bz = ld_c(q.B[2], base + col, nf, st);
  const T ikx = ld(q.ik[0] + i + 1), iky = ld(q.ik[1] + j + 1), iky_bz = ld(q.ik_bz_y + j + 1);
  const T ikz = ld(q.ik[2] + k);
  T bxn, byn, bzn;
  b_cell<T, true>(q, i, j, k, col, face_column_mask(q.cpml, i, j), v, ikx, iky, iky_bz, ikz, bxn, byn, bzn);
  st_c(q.B[0], base + col, nf, st, bxn);
  st_c(q.B[1], base + col, nf, st, byn);
  st_c(q.B[2], base + col, nf, st, bzn);
}

// Row of border row r (the last row of y-tile r, or the grid's last row).
__device__ __forceinline__ int border_row(int r, int ny) { return min(r * MPB_F_BLOCK_Y + MPB_F_BLOCK_Y - 1, ny - 1); }
__device__ __forceinline__ bool is_border_row(int j, int ny) {
  return (j % MPB_F_BLOCK_Y) == MPB_F_BLOCK_Y - 1 || j == ny - 1;
}
__device__ __forceinline__ bool is_border_col(int i, int nx) { return (i % 32) == 31 || i == nx - 1; }

// The B cells step_fused_kernel leaves out, in one launch of 128-thread
// blocks (a 1-D grid):
//   [0, na)          the tiles' last rows, all B planes: 32 columns x 4
//                    border rows per block, a chunk of kb planes each;
//   [na, na + nb)    the tiles' last columns off those rows, all B planes:
//                    128 (tile, row) pairs per block, a chunk of kb planes;
//   [na + nb, ...)   the remaining cells of the planes the fused launch does
//                    not reach: B planes below its first E plane and the top
//                    plane of each of its chunks (one plane per block row of
//                    32 x 4 cells).
template <typename T>
__global__ void __launch_bounds__(128) b_border_kernel(const BParams<T> q, const int ek_first, const int ek_last,
                                                       const FusedChunks fc, const int kb, const int na,
                                                       const int nb) {
  const int b = blockIdx.x, t = threadIdx.x;
  const int nkb = q.k_last - q.k_first + 1, zch = (nkb + kb - 1) / kb;
  if (b < na) {
    const int gx = (q.nx + 31) / 32;
    const int nbr = (q.ny + MPB_F_BLOCK_Y - 1) / MPB_F_BLOCK_Y, gy = (nbr + 3) / 4;
    const int z = b / (gx * gy), r0 = b % (gx * gy);
    const int i = (r0 % gx) * 32 + (t & 31), r = (r0 / gx) * 4 + (t >> 5);
    if (i >= q.nx || r >= nbr) return;
    const int j = border_row(r, q.ny);
    const int k0 = q.k_first + z * kb, k1 = min(k0 + kb - 1, q.k_last);
    for (int k = k0; k <= k1; ++k) b_cell_global(q, i, j, k);
    (void)zch;
  } else if (b < na + nb) {
    const int gx = (q.nx + 31) / 32;
    const int pairs = gx * q.ny, gp = (pairs + 127) / 128;
    const int z = (b - na) / gp, pr = ((b - na) % gp) * 128 + t;
    if (pr >= pairs) return;
    const int tile = pr % gx, j = pr / gx;
    if (is_border_row(j, q.ny)) return;
    const int i = min(tile * 32 + 31, q.nx - 1);
    const int k0 = q.k_first + z * kb, k1 = min(k0 + kb - 1, q.k_last);
    for (int k = k0; k <= k1; ++k) b_cell_global(q, i, j, k);
  } else {
    const int gx = (q.nx + 31) / 32, gy = (q.ny + 3) / 4;
    const int c = b - na - nb;
    const int d = c / (gx * gy), r0 = c % (gx * gy);
    const int i = (r0 % gx) * 32 + (t & 31), j = (r0 / gx) * 4 + (t >> 5);
    if (i >= q.nx || j >= q.ny || is_border_row(j, q.ny) || is_border_col(i, q.nx)) return;
    // plane d: first the B planes below the first E plane, then the chunks'
    // top planes
    const int below = max(0, ek_first - q.k_first);
    int k;
    if (d < below) {
      k = q.k_first + d;
    } else {
      k = min(ek_first + (d - below + 1) * fc.kchunk - 1, ek_last);
      if (k > q.k_last) return;
    }
    b_cell_global(q, i, j, k);
  }
}

template <typename T, int MODE>
static cudaError_t launch_fused_np(const EParams<T> &p, const BParams<T> &q, int np, const FusedChunks &fc,
                                   cudaStream_t st) {
  EParams<T> pe = p;
  pe.kchunk = fc.kchunk;
  const dim3 g((p.nx + 31) / 32, (p.ny + MPB_F_BLOCK_Y - 1) / MPB_F_BLOCK_Y, fc.nchunks), b(32, MPB_F_BLOCK_Y, 1);
  switch (np) {
    case 0: step_fused_kernel<T, MODE, 0><<<g, b, 0, st>>>(pe, q); break;
    case 1: step_fused_kernel<T, MODE, 1><<<g, b, 0, st>>>(pe, q); break;
    case 2: step_fused_kernel<T, MODE, 2><<<g, b, 0, st>>>(pe, q); break;
    default: step_fused_kernel<T, MODE, 3><<<g, b, 0, st>>>(pe, q); break;
  }
  return cudaGetLastError();
}

// One time step with the fused kernel and the border kernel.  `which`: 1 the
// fused launch only, 2 the border launch only, 3 both (the step's per-kernel
// timing launches them one at a time).
template <typename T>
cudaError_t launch_step_fused(const EParams<T> &p, const BParams<T> &q, int mode, int np, int which,
                              cudaStream_t st) {
  const int nk = p.k_last - p.k_first + 1;
  const long long bxy = (long long)((p.nx + 31) / 32) * ((p.ny + MPB_F_BLOCK_Y - 1) / MPB_F_BLOCK_Y);
  const long long chunks = std::max(1LL, (148LL * MPB_F_BLOCKS_PER_SM + bxy - 1) / bxy);
  FusedChunks fc;
  fc.kchunk = int(std::min<long long>(nk, std::max<long long>(MPB_F_MIN_PLANES, (nk + chunks - 1) / chunks)));
  fc.nchunks = (nk + fc.kchunk - 1) / fc.kchunk;
  cudaError_t e = cudaSuccess;
  if (which & 1) {
    switch (mode) {
      case MODE_PLAIN: e = launch_fused_np<T, MODE_PLAIN>(p, q, 0, fc, st); break;
      case MODE_NL: e = launch_fused_np<T, MODE_NL>(p, q, 0, fc, st); break;
      case MODE_PLRC_LIN: e = launch_fused_np<T, MODE_PLRC_LIN>(p, q, np, fc, st); break;
      default: e = launch_fused_np<T, MODE_PLRC_NONLIN>(p, q, np, fc, st); break;
    }
    if (e != cudaSuccess) return e;
  }
  if (which & 2) {
    // border rows and columns in chunks of 16 B planes; the planes the fused
    // launch does not reach: those below its first E plane and one per chunk
    const int kb = 16;
    const int nkb = q.k_last - q.k_first + 1, zch = (nkb + kb - 1) / kb;
    const int gx = (q.nx + 31) / 32;
    const int nbr = (q.ny + MPB_F_BLOCK_Y - 1) / MPB_F_BLOCK_Y;
    const int na = gx * ((nbr + 3) / 4) * zch;
    const int nb = ((gx * q.ny + 127) / 128) * zch;
    const int nd = std::max(0, p.k_first - q.k_first) + fc.nchunks;
    const int nc = gx * ((q.ny + 3) / 4) * nd;
    b_border_kernel<T><<<na + nb + nc, 128, 0, st>>>(q, p.k_first, p.k_last, fc, kb, na, nb);
    e = cudaGetLastError();
  }
  return e;
}

template cudaError_t launch_step_fused<float>(const EParams<float> &, const BParams<float> &, int, int, int,
                                              cudaStream_t);
template cudaError_t launch_step_fused<double>(const EParams<double> &, const BParams<double> &, int, int, int,
                                               cudaStream_t);

}  // namespace mpb
