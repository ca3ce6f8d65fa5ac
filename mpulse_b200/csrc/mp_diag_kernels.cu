// mp_diag_kernels.cu - field energy of FieldEnergyDiag::calculate
// (fielddiag.cpp:255-286): sum over the interior cells [1, n]^3 of
// Ex^2 + Ey^2 + Ez^2 + Bx^2 + By^2 + Bz^2, times dx dy dz, accumulated in FP64
// whatever the field precision.
//
// Two passes, both deterministic: one block per z-plane sums that plane into a
// per-plane partial (fixed tree order), then one block sums the partials in
// plane order.  The per-plane partials are scratch memory: mp_field_energy uses
// a buffer the context allocated.
#include "mpulse_b200.h"

#include "mp_device.h"

#include <cuda_runtime.h>


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

}  // namespace mpb
