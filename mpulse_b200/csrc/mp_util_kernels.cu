// mp_util_kernels.cu - conversion between the host's double buffers and the
// device form (FP32 or FP64), with a stride / offset for the complex-interleaved
// PLRC accumulators.  Used by mp_upload / mp_download only.
#include <cuda_runtime.h>

namespace mpb {

template <typename T>
__global__ void convert_in_kernel(const double *__restrict__ src, T *__restrict__ dst, long long n, int stride,
                                  int offset) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q * stride + offset] = T(src[q]);
}

template <typename T>
__global__ void convert_out_kernel(const T *__restrict__ src, double *__restrict__ dst, long long n, int stride,
                                   int offset) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = double(src[q * stride + offset]);
}

static dim3 conv_grid(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  if (b < 1) b = 1;
  return dim3((unsigned)b);
}

cudaError_t launch_convert_in(const double *src, void *dst, int fp32, long long n, int stride, int offset,
                              cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (fp32) convert_in_kernel<float><<<conv_grid(n), 256, 0, st>>>(src, static_cast<float *>(dst), n, stride, offset);
  else convert_in_kernel<double><<<conv_grid(n), 256, 0, st>>>(src, static_cast<double *>(dst), n, stride, offset);
  return cudaGetLastError();
}

cudaError_t launch_convert_out(const void *src, double *dst, int fp32, long long n, int stride, int offset,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (fp32)
    convert_out_kernel<float><<<conv_grid(n), 256, 0, st>>>(static_cast<const float *>(src), dst, n, stride, offset);
  else
    convert_out_kernel<double><<<conv_grid(n), 256, 0, st>>>(static_cast<const double *>(src), dst, n, stride, offset);
  return cudaGetLastError();
}

}  // namespace mpb
