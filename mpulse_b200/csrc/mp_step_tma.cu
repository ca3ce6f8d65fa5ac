// mp_step_tma.cu - the E and B half-step kernels with the z-planes staged in
// shared memory by TMA (cp.async.bulk.tensor), for grids whose x extent is a
// multiple of 32 and y extent a multiple of 8 (otherwise mp_step_kernels.cu's
// global-load kernels run).  The arithmetic per cell is the same code
// (mp_cell.cuh), so both forms give bit-identical results.
//
// A block owns a 32 x 8 tile of columns and marches up a chunk of z-planes.
// It is warp-specialised: warp 8 is the producer, whose lane 0 issues, for
// every plane, 3-D TMA tile loads of all the arrays the cells read - with the
// x-1 / y-1 (E half) or x+1 / y+1 (B half) halo - into one stage of a ring in
// shared memory, completing on that stage's "full" mbarrier; warps 0..7 are
// the consumers (one tile row each), which copy their values out of the stage,
// release it on its "empty" mbarrier and compute while the producer refills
// it.  The ring is S planes deep, so the copy engine keeps tens of KB per SM
// in flight however few warps are resident.  Results go straight to global
// memory.  x halos start 16 bytes before / at the tile (the TMA x coordinate
// must be a multiple of 16 bytes); a halo that falls outside the grid reads as
// zero and the few cells that need the periodic image read it from global
// memory instead.  Each CTA loads its own tiles; no thread-block clusters.
//
// Every wait on an mbarrier is bounded: after ~4M polls the warp records a
// timeout in the status word and leaves; mp_step then reports MP_ERR_CUDA.
#include "mp_cell.cuh"

#include <cuda.h>

#include <cstdint>

namespace mpb {

static const int kTX = kTmaTileX, kTY = kTmaTileY;
static const int kConsumerWarps = kTY;           // one tile row per consumer warp
static const int kThreads = 32 * (kConsumerWarps + 1);
static const int kStageBudget = 110 * 1024;      // ring bytes per block: two blocks per SM

// ---- PTX wrappers -----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false after ~4M polls (each poll may suspend briefly).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int n = 0; n < (1 << 22); ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__host__ __device__ constexpr int round128(int b) { return (b + 127) / 128 * 128; }
__host__ __device__ constexpr int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---- shared-memory layout of one stage ---------------------------------------

template <typename T, int NP>
struct ELayout {
  static constexpr int H = 16 / int(sizeof(T));  // x halo: 16 bytes
  static constexpr int WB = kTX + H;             // row length of the haloed tiles
  static constexpr int BX = kTX * (kTY + 1) * sizeof(T);
  static constexpr int BY = WB * kTY * sizeof(T);
  static constexpr int BZ = WB * (kTY + 1) * sizeof(T);
  static constexpr int EE = kTX * kTY * sizeof(T);
  static constexpr int PS = 2 * kTX * kTY * sizeof(T);
  static constexpr int oBX = 0;
  static constexpr int oBY = oBX + round128(BX);
  static constexpr int oBZ = oBY + round128(BY);
  static constexpr int oEX = oBZ + round128(BZ);
  static constexpr int oEY = oEX + round128(EE);
  static constexpr int oEZ = oEY + round128(EE);
  static constexpr int oPS = oEZ + round128(EE);
  static constexpr int STAGE = oPS + 3 * NP * round128(PS);
  static constexpr int FIELD_BYTES = BX + BY + BZ + 3 * EE;  // transaction bytes without psi
  static constexpr int PSI_BYTES = 3 * NP * PS;
  static constexpr int S = clampi(kStageBudget / STAGE, 2, 8);
  static constexpr int SMEM = S * STAGE + 2 * S * 8;  // ring, then full[S], empty[S]
};

template <typename T>
struct BLayout {
  static constexpr int H = 16 / int(sizeof(T));
  static constexpr int WB = kTX + H;
  static constexpr int EX = kTX * (kTY + 1) * sizeof(T);
  static constexpr int EY = WB * kTY * sizeof(T);
  static constexpr int EZ = WB * (kTY + 1) * sizeof(T);
  static constexpr int BB = kTX * kTY * sizeof(T);
  static constexpr int oEX = 0;
  static constexpr int oEY = oEX + round128(EX);
  static constexpr int oEZ = oEY + round128(EY);
  static constexpr int oBX = oEZ + round128(EZ);
  static constexpr int oBY = oBX + round128(BB);
  static constexpr int oBZ = oBY + round128(BB);
  static constexpr int STAGE = oBZ + round128(BB);
  static constexpr int BYTES = EX + EY + EZ + 3 * BB;
  static constexpr int S = clampi(kStageBudget / STAGE, 3, 8);
  static constexpr int SMEM = S * STAGE + 2 * S * 8;
};

// ---- E half -----------------------------------------------------------------

template <typename T, int MODE, int NP>
__global__ void __launch_bounds__(kThreads, 2)
    e_half_tma_kernel(const EParams<T> p, const __grid_constant__ ETmaMaps maps) {
  typedef typename Vec2<T>::type T2;
  typedef ELayout<T, NP> L;
  constexpr int S = L::S;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S * L::STAGE);
  uint64_t *empty = full + S;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  if (k0 > k1) return;  // whole block
  const int nplanes = k1 - k0 + 1;
  if (smem_u32(smem) & 127) {  // tile copies need 128-byte aligned destinations
    if (tx == 0 && ty == 0) atomicAdd(p.status + ST_TIMEOUT, 1);
    return;
  }
  if (tx == 0 && ty == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    mbar_fence_init();
  }
  __syncthreads();

  // medium cell (PLRC / Kerr update) and whether accumulators exist there
  auto is_med = [&](int k) {
    return (MODE == MODE_PLRC_LIN || MODE == MODE_PLRC_NONLIN) && k >= p.mz0 && k <= p.mz1;
  };

  if (ty == kConsumerWarps) {
    // ---------------- producer warp
    if (tx != 0) return;
    for (int m = 0; m < nplanes; ++m) {
      const int s = m % S;
      if (m >= S && !mbar_wait(&empty[s], ((m / S) + 1) & 1)) {
        atomicAdd(p.status + ST_TIMEOUT, 1);
        return;
      }
      const int k = k0 + m;
      unsigned char *st = smem + s * L::STAGE;
      const bool med = NP > 0 && is_med(k);
      mbar_expect_tx(&full[s], L::FIELD_BYTES + (med ? L::PSI_BYTES : 0));
      tma_load_3d(st + L::oBX, &maps.bx, x0, y0 - 1, k, &full[s]);
      tma_load_3d(st + L::oBY, &maps.by, x0 - L::H, y0, k, &full[s]);
      tma_load_3d(st + L::oBZ, &maps.bz, x0 - L::H, y0 - 1, k, &full[s]);
      tma_load_3d(st + L::oEX, &maps.ex, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oEY, &maps.ey, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oEZ, &maps.ez, x0, y0, k, &full[s]);
      if (med) {
#pragma unroll
        for (int n = 0; n < (NP > 0 ? NP : 1); ++n)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            tma_load_3d(st + L::oPS + (3 * n + c) * round128(L::PS), &maps.psi[n][c], 2 * x0, y0, k - p.mz0,
                        &full[s]);
      }
    }
    return;
  }

  // ---------------- consumer warps: cell (i, j), one tile row per warp
  const int i = x0 + tx, j = y0 + ty;
  const long long plane = p.plane;
  const long long col = (long long)j * p.nx + i;
  const T *__restrict__ Bx = p.B[0];
  const T *__restrict__ By = p.B[1];
  const T *__restrict__ Bz = p.B[2];
  const T ikx = ld(p.ik[0] + i + 1);
  const T iky = ld(p.ik[1] + j + 1);
  const unsigned cmask = face_column_mask(p.cpml, i, j);
  const bool warp_xy = __any_sync(__activemask(), cmask != 0u);
  const int2 srck = source_plane_range(p);
  const bool wrap_x = (x0 == 0 && tx == 0);  // x-1 is the periodic image nx-1
  const bool wrap_y = (y0 == 0 && ty == 0);  // y-1 is the periodic image ny-1
  const long long colxm = (long long)j * p.nx + (p.nx - 1);
  const long long colym = (long long)(p.ny - 1) * p.nx + i;

  int km = k0 - 1;
  if (p.zperiodic && km == 0) km = p.nz;
  T bx_km = ld(Bx + km * plane + col);
  T by_km = ld(By + km * plane + col);
  KerrCount kc;

  for (int m = 0; m < nplanes; ++m) {
    const int k = k0 + m;
    const int s = m % S;
    if (!mbar_wait(&full[s], (m / S) & 1)) {
      if (tx == 0) atomicAdd(p.status + ST_TIMEOUT, 1);
      return;
    }
    const unsigned char *st = smem + s * L::STAGE;
    const T *sbx = reinterpret_cast<const T *>(st + L::oBX);
    const T *sby = reinterpret_cast<const T *>(st + L::oBY);
    const T *sbz = reinterpret_cast<const T *>(st + L::oBZ);
    EIn<T> v;
    v.bx = sbx[(ty + 1) * kTX + tx];
    v.bx_ym = sbx[ty * kTX + tx];
    v.by = sby[ty * L::WB + tx + L::H];
    v.by_xm = sby[ty * L::WB + tx + L::H - 1];
    v.bz = sbz[(ty + 1) * L::WB + tx + L::H];
    v.bz_xm = sbz[(ty + 1) * L::WB + tx + L::H - 1];
    v.bz_ym = sbz[ty * L::WB + tx + L::H];
    v.ex = reinterpret_cast<const T *>(st + L::oEX)[ty * kTX + tx];
    v.ey = reinterpret_cast<const T *>(st + L::oEY)[ty * kTX + tx];
    v.ez = reinterpret_cast<const T *>(st + L::oEZ)[ty * kTX + tx];
    const bool med = is_med(k);
    T2 q[NP > 0 ? NP : 1][3];
    if (NP > 0 && med) {
#pragma unroll
      for (int n = 0; n < (NP > 0 ? NP : 1); ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          q[n][c] = reinterpret_cast<const T2 *>(st + L::oPS + (3 * n + c) * round128(L::PS))[ty * kTX + tx];
    }
    __syncwarp();
    if (tx == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s

    const long long base = (long long)k * plane;
    if (wrap_x) {
      v.by_xm = ld(By + base + colxm);
      v.bz_xm = ld(Bz + base + colxm);
    }
    if (wrap_y) {
      v.bx_ym = ld(Bx + base + colym);
      v.bz_ym = ld(Bz + base + colym);
    }
    v.bx_km = bx_km;
    v.by_km = by_km;
    const T ikz = ld(p.ik[2] + k);
    T exn, eyn, ezn;
    if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
      e_cell<T, MODE, NP, false, true>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn, kc);
    else
      e_cell<T, MODE, NP, false, false>(p, i, j, k, col, med, cmask, v, ikx, iky, ikz, q, exn, eyn, ezn, kc);
    p.E[0][base + col] = exn;
    p.E[1][base + col] = eyn;
    p.E[2][base + col] = ezn;
    if (NP > 0 && med) {
      const long long pi = ((long long)(k - p.mz0) * p.ny + j) * p.nx + i;
#pragma unroll
      for (int n = 0; n < (NP > 0 ? NP : 1); ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) reinterpret_cast<T2 *>(p.psi[n][c])[pi] = q[n][c];
    }
    bx_km = v.bx;
    by_km = v.by;
  }
  flush_kerr_count<MODE>(p.kerr_count, kc);
}

// ---- B half -----------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(kThreads, 2)
    b_half_tma_kernel(const BParams<T> p, const __grid_constant__ BTmaMaps maps) {
  typedef BLayout<T> L;
  constexpr int S = L::S;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S * L::STAGE);
  uint64_t *empty = full + S;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int k0 = p.k_first + blockIdx.z * p.kchunk;
  const int k1 = min(k0 + p.kchunk - 1, p.k_last);
  if (k0 > k1) return;
  // planes k0 .. k1 + 1 are loaded (the last only for its Ex, Ey)
  const int nload = k1 - k0 + 2;
  if (smem_u32(smem) & 127) {
    if (tx == 0 && ty == 0) atomicAdd(p.status + ST_TIMEOUT, 1);
    return;
  }
  if (tx == 0 && ty == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (ty == kConsumerWarps) {
    // ---------------- producer warp
    if (tx != 0) return;
    for (int m = 0; m < nload; ++m) {
      const int s = m % S;
      if (m >= S && !mbar_wait(&empty[s], ((m / S) + 1) & 1)) {
        atomicAdd(p.status + ST_TIMEOUT, 1);
        return;
      }
      int k = k0 + m;
      if (p.zperiodic && k == p.nz + 1) k = 1;
      unsigned char *st = smem + s * L::STAGE;
      mbar_expect_tx(&full[s], L::BYTES);
      tma_load_3d(st + L::oEX, &maps.ex, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oEY, &maps.ey, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oEZ, &maps.ez, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oBX, &maps.bx, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oBY, &maps.by, x0, y0, k, &full[s]);
      tma_load_3d(st + L::oBZ, &maps.bz, x0, y0, k, &full[s]);
    }
    return;
  }

  // ---------------- consumer warps
  const int i = x0 + tx, j = y0 + ty;
  const long long plane = p.plane;
  const long long col = (long long)j * p.nx + i;
  const T *__restrict__ Ex = p.E[0];
  const T *__restrict__ Ey = p.E[1];
  const T *__restrict__ Ez = p.E[2];
  const T ikx = ld(p.ik[0] + i + 1);
  const T iky = ld(p.ik[1] + j + 1);
  const T iky_bz = ld(p.ik_bz_y + j + 1);
  const unsigned cmask = face_column_mask(p.cpml, i, j);
  const bool warp_xy = __any_sync(__activemask(), cmask != 0u);
  const int2 srck = source_plane_range(p);
  const bool wrap_x = (x0 + kTX == p.nx && tx == kTX - 1);  // x+1 is the image 0
  const bool wrap_y = (y0 + kTY == p.ny && ty == kTY - 1);  // y+1 is the image 0
  const long long colxp = (long long)j * p.nx;
  const long long colyp = (long long)i;

  // plane k0's centre values of Ex, Ey, carried as "this plane" into the loop
  if (!mbar_wait(&full[0], 0)) {
    if (tx == 0) atomicAdd(p.status + ST_TIMEOUT, 1);
    return;
  }
  T ex_k = reinterpret_cast<const T *>(smem + L::oEX)[ty * kTX + tx];
  T ey_k = reinterpret_cast<const T *>(smem + L::oEY)[ty * L::WB + tx];

  for (int m = 0; m + 1 < nload; ++m) {
    const int k = k0 + m;
    const int s = m % S, sn = (m + 1) % S;
    // stage s (plane k) is complete since the previous iteration; wait for k+1
    if (!mbar_wait(&full[sn], ((m + 1) / S) & 1)) {
      if (tx == 0) atomicAdd(p.status + ST_TIMEOUT, 1);
      return;
    }
    const unsigned char *st = smem + s * L::STAGE;
    const unsigned char *stn = smem + sn * L::STAGE;
    const T *sex = reinterpret_cast<const T *>(st + L::oEX);
    const T *sey = reinterpret_cast<const T *>(st + L::oEY);
    const T *sez = reinterpret_cast<const T *>(st + L::oEZ);
    BIn<T> v;
    v.ex = ex_k;
    v.ey = ey_k;
    v.ex_yp = sex[(ty + 1) * kTX + tx];
    v.ey_xp = sey[ty * L::WB + tx + 1];
    v.ez = sez[ty * L::WB + tx];
    v.ez_xp = sez[ty * L::WB + tx + 1];
    v.ez_yp = sez[(ty + 1) * L::WB + tx];
    v.bx = reinterpret_cast<const T *>(st + L::oBX)[ty * kTX + tx];
    v.by = reinterpret_cast<const T *>(st + L::oBY)[ty * kTX + tx];
    v.bz = reinterpret_cast<const T *>(st + L::oBZ)[ty * kTX + tx];
    v.ex_kp = reinterpret_cast<const T *>(stn + L::oEX)[ty * kTX + tx];
    v.ey_kp = reinterpret_cast<const T *>(stn + L::oEY)[ty * L::WB + tx];
    __syncwarp();
    if (tx == 0) mbar_arrive(&empty[s]);  // plane k is no longer needed

    const long long base = (long long)k * plane;
    if (wrap_x) {
      v.ey_xp = ld(Ey + base + colxp);
      v.ez_xp = ld(Ez + base + colxp);
    }
    if (wrap_y) {
      v.ex_yp = ld(Ex + base + colyp);
      v.ez_yp = ld(Ez + base + colyp);
    }
    const T ikz = ld(p.ik[2] + k);
    T bxn, byn, bzn;
    if (warp_xy || z_face_plane(p.cpml, k) || (k >= srck.x && k <= srck.y))
      b_cell<T, true>(p, i, j, k, col, cmask, v, ikx, iky, iky_bz, ikz, bxn, byn, bzn);
    else
      b_cell<T, false>(p, i, j, k, col, cmask, v, ikx, iky, iky_bz, ikz, bxn, byn, bzn);
    p.B[0][base + col] = bxn;
    p.B[1][base + col] = byn;
    p.B[2][base + col] = bzn;
    ex_k = v.ex_kp;
    ey_k = v.ey_kp;
  }
  // the stage of the extra plane k1+1 is released too, so that a producer
  // waiting on it (it never does: it issued its last load) has nothing pending
}

// ---- launchers ----------------------------------------------------------------

// Raises one kernel's dynamic shared-memory limit once per device; `done` is
// the kernel's own flag array.
template <typename K>
static cudaError_t smem_attribute(K kernel, int bytes, bool *done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

template <typename T, int MODE, int NP>
static cudaError_t launch_e_tma_np(const EParams<T> &p, const ETmaMaps &maps, cudaStream_t st) {
  typedef ELayout<T, NP> L;
  static bool done[64] = {false};  // one per template instance
  cudaError_t e = smem_attribute(e_half_tma_kernel<T, MODE, NP>, L::SMEM, done);
  if (e != cudaSuccess) return e;
  const int nk = p.k_last - p.k_first + 1;
  const dim3 g(p.nx / kTX, p.ny / kTY, (nk + p.kchunk - 1) / p.kchunk), b(32, kConsumerWarps + 1, 1);
  e_half_tma_kernel<T, MODE, NP><<<g, b, L::SMEM, st>>>(p, maps);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_e_half_tma(const EParams<T> &p, const ETmaMaps &maps, int mode, int np, cudaStream_t st) {
  switch (mode) {
    case MODE_PLAIN: return launch_e_tma_np<T, MODE_PLAIN, 0>(p, maps, st);
    case MODE_NL: return launch_e_tma_np<T, MODE_NL, 0>(p, maps, st);
    case MODE_PLRC_LIN:
      switch (np) {
        case 0: return launch_e_tma_np<T, MODE_PLRC_LIN, 0>(p, maps, st);
        case 1: return launch_e_tma_np<T, MODE_PLRC_LIN, 1>(p, maps, st);
        case 2: return launch_e_tma_np<T, MODE_PLRC_LIN, 2>(p, maps, st);
        default: return launch_e_tma_np<T, MODE_PLRC_LIN, 3>(p, maps, st);
      }
    default:
      switch (np) {
        case 0: return launch_e_tma_np<T, MODE_PLRC_NONLIN, 0>(p, maps, st);
        case 1: return launch_e_tma_np<T, MODE_PLRC_NONLIN, 1>(p, maps, st);
        case 2: return launch_e_tma_np<T, MODE_PLRC_NONLIN, 2>(p, maps, st);
        default: return launch_e_tma_np<T, MODE_PLRC_NONLIN, 3>(p, maps, st);
      }
  }
}

template <typename T>
cudaError_t launch_b_half_tma(const BParams<T> &p, const BTmaMaps &maps, cudaStream_t st) {
  typedef BLayout<T> L;
  static bool done[64] = {false};
  cudaError_t e = smem_attribute(b_half_tma_kernel<T>, L::SMEM, done);
  if (e != cudaSuccess) return e;
  const int nk = p.k_last - p.k_first + 1;
  const dim3 g(p.nx / kTX, p.ny / kTY, (nk + p.kchunk - 1) / p.kchunk), b(32, kConsumerWarps + 1, 1);
  b_half_tma_kernel<T><<<g, b, L::SMEM, st>>>(p, maps);
  return cudaGetLastError();
}

template cudaError_t launch_e_half_tma<float>(const EParams<float> &, const ETmaMaps &, int, int, cudaStream_t);
template cudaError_t launch_e_half_tma<double>(const EParams<double> &, const ETmaMaps &, int, int, cudaStream_t);
template cudaError_t launch_b_half_tma<float>(const BParams<float> &, const BTmaMaps &, cudaStream_t);
template cudaError_t launch_b_half_tma<double>(const BParams<double> &, const BTmaMaps &, cudaStream_t);

// Box sizes (elements) of the tensor maps, innermost first, for the host.
void tma_boxes(int esz, int e_box[7][2], int b_box[6][2]) {
  const int H = 16 / esz;
  // E half: bx, by, bz, ex, ey, ez, psi (psi counts T elements: 2 per complex)
  const int eb[7][2] = {{kTX, kTY + 1}, {kTX + H, kTY}, {kTX + H, kTY + 1}, {kTX, kTY}, {kTX, kTY}, {kTX, kTY},
                        {2 * kTX, kTY}};
  // B half: ex, ey, ez, bx, by, bz
  const int bb[6][2] = {{kTX, kTY + 1}, {kTX + H, kTY}, {kTX + H, kTY + 1}, {kTX, kTY}, {kTX, kTY}, {kTX, kTY}};
  for (int q = 0; q < 7; ++q) { e_box[q][0] = eb[q][0]; e_box[q][1] = eb[q][1]; }
  for (int q = 0; q < 6; ++q) { b_box[q][0] = bb[q][0]; b_box[q][1] = bb[q][1]; }
}

}  // namespace mpb
