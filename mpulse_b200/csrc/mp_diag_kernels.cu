// mp_diag_kernels.cu - field energy of FieldEnergyDiag::calculate
// (fielddiag.cpp:255-286): sum over the interior cells [1, n]^3 of
// Ex^2 + Ey^2 + Ez^2 + Bx^2 + By^2 + Bz^2, times dx dy dz, accumulated in FP64
// whatever the field precision.
//
// Two passes, both deterministic: one block per z-plane sums that plane into a
// per-plane partial (fixed tree order), then one block sums the partials in
// plane order.  The per-plane partials are scratch memory: mp_field_energy uses
// a buffer the context allocated; mp_field_energy_noalloc uses the file-scope
// array below instead.
#include "mpulse_b200.h"

#include "mp_device.h"

#include <cuda_runtime.h>

#include <cstdio>

namespace mpb {

static const int kDiagThreads = 256;

template <typename T>
struct FieldPtrs {
  const T *f[6];
};

__device__ __forceinline__ double block_sum(double v, double *smem) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  v = threadIdx.x < (blockDim.x >> 5) ? smem[threadIdx.x] : 0.0;
  if (warp == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// partial[b] = sum over plane k = k0 + b of the six squared components
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) plane_energy_kernel(FieldPtrs<T> p, long long plane, int k0,
                                                                    double *partial) {
  __shared__ double smem[kDiagThreads / 32];
  const long long base = (long long)(k0 + blockIdx.x) * plane;
  double s = 0.0;
  for (long long q = threadIdx.x; q < plane; q += blockDim.x) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const double v = (double)p.f[c][base + q];
      s += v * v;
    }
  }
  s = block_sum(s, smem);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// out[0] = scale * sum of partial[0 .. n-1]
__global__ void __launch_bounds__(kDiagThreads) sum_partials_kernel(const double *partial, int n, double scale,
                                                                    double *out) {
  __shared__ double smem[kDiagThreads / 32];
  double s = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) s += partial[q];
  s = block_sum(s, smem);
  if (threadIdx.x == 0) out[0] = s * scale;
}

// Queues the energy of the interior planes 1..nz into *out_dev, using
// partial[0 .. nz-1] as scratch.
cudaError_t launch_field_energy(const void *const fields[6], int elem_bytes, int nx, int ny, int nz, double dV,
                                double *partial, double *out_dev, cudaStream_t st) {
  const long long plane = (long long)nx * ny;
  if (elem_bytes == 4) {
    FieldPtrs<float> p;
    for (int c = 0; c < 6; ++c) p.f[c] = static_cast<const float *>(fields[c]);
    plane_energy_kernel<float><<<nz, kDiagThreads, 0, st>>>(p, plane, 1, partial);
  } else {
    FieldPtrs<double> p;
    for (int c = 0; c < 6; ++c) p.f[c] = static_cast<const double *>(fields[c]);
    plane_energy_kernel<double><<<nz, kDiagThreads, 0, st>>>(p, plane, 1, partial);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sum_partials_kernel<<<1, kDiagThreads, 0, st>>>(partial, nz, dV, out_dev);
  return cudaGetLastError();
}

void set_global_error(const char *msg);  // mp_api.cu: message for mp_last_error(NULL, ..)

}  // namespace mpb

// ---------------------------------------------------------------------------
// mp_field_energy without allocating.
//
// The scratch of the two passes (one partial sum per z-plane, then the result)
// lives in this fixed file-scope array instead of a context buffer.  It holds
// MP_NOALLOC_MAX_PLANES partials plus the result slot (about 130 KB); every GPU
// that loads the library keeps it until the process exits.  All calls on a
// device share it and it keeps the last call's contents; nothing in it has to
// start at zero, because a call writes every slot it reads before reading it.
// Two calls whose work overlaps on the GPU (different streams, or different
// host threads) race on it.
static __device__ __align__(256) double g_energy_scratch[MP_NOALLOC_MAX_PLANES + 32];

namespace {

// The host-side name g_energy_scratch is a stand-in, not a device address;
// the address comes from cudaGetSymbolAddress with the device current.  It is
// looked up on every call (no allocation, no device synchronisation), so a
// call after cudaDeviceReset, which reloads the module, gets the new address.
cudaError_t scratch_for_current_device(double **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_energy_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<double *>(p);
  return cudaSuccess;
}

// True when ptr is device (or managed) memory that the current device can
// read: a host pointer handed to the kernel would fault the GPU, so it is
// turned into MP_ERR_INVALID here, before any launch.
bool device_readable(const void *ptr, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();  // the failed query leaves a (non-sticky) error behind: clear it
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  if (a.type != cudaMemoryTypeDevice) return false;
  if (a.device == dev) return true;
  int peer = 0;
  return cudaDeviceCanAccessPeer(&peer, dev, a.device) == cudaSuccess && peer;
}

}  // namespace

extern "C" int mp_field_energy_noalloc(const void *const fields[6], int elem_bytes, int nx, int ny, int nz,
                                       double dx, double dy, double dz, void *cuda_stream, double *energy) {
  char msg[256];
  if (!fields || !energy) {
    mpb::set_global_error("mp_field_energy_noalloc: fields and energy must not be NULL");
    return MP_ERR_INVALID;
  }
  for (int c = 0; c < 6; ++c)
    if (!fields[c]) {
      mpb::set_global_error("mp_field_energy_noalloc: a field pointer is NULL");
      return MP_ERR_INVALID;
    }
  if (elem_bytes != 4 && elem_bytes != 8) {
    mpb::set_global_error("mp_field_energy_noalloc: elem_bytes must be 4 (FP32) or 8 (FP64)");
    return MP_ERR_INVALID;
  }
  if (nx < 1 || ny < 1 || nz < 1) {
    mpb::set_global_error("mp_field_energy_noalloc: nx, ny, nz must be positive");
    return MP_ERR_INVALID;
  }
  if (nz > MP_NOALLOC_MAX_PLANES) {
    snprintf(msg, sizeof msg,
             "mp_field_energy_noalloc: nz = %d exceeds the %d planes of its fixed scratch array; "
             "use mp_field_energy", nz, MP_NOALLOC_MAX_PLANES);
    mpb::set_global_error(msg);
    return MP_ERR_INVALID;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) {
    for (int c = 0; c < 6; ++c)
      if (!device_readable(fields[c], dev)) {
        snprintf(msg, sizeof msg,
                 "mp_field_energy_noalloc: fields[%d] is not device memory readable by device %d", c, dev);
        mpb::set_global_error(msg);
        return MP_ERR_INVALID;
      }
  }
  double *scratch = nullptr;
  if (e == cudaSuccess) e = scratch_for_current_device(&scratch);
  if (e == cudaSuccess) {
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    double *result = scratch + MP_NOALLOC_MAX_PLANES;
    e = mpb::launch_field_energy(fields, elem_bytes, nx, ny, nz, dx * dy * dz, scratch, result, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(energy, result, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) {
    snprintf(msg, sizeof msg, "mp_field_energy_noalloc: %s", cudaGetErrorString(e));
    mpb::set_global_error(msg);
    return MP_ERR_CUDA;
  }
  return MP_OK;
}
