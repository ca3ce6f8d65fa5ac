// mp_checked.cuh - the state accesses of the step and adjoint kernels, plain
// or bounds-checked (MPB_CHECKED=1).
#ifndef MPB_MP_CHECKED_CUH
#define MPB_MP_CHECKED_CUH

#include "mp_device.h"

#include <cuda_runtime.h>

namespace mpb {

// A checked build (MPB_CHECKED=1, the library libmpulse_b200_checked.so)
// tests every element index against the size of its array; an index outside
// is counted in the status word (ST_BOUNDS, reported by mp_step / mp_adjoint
// as MP_ERR_BOUNDS) and the access is skipped, a load reading 0, so nothing
// faults.  The default build compiles these to plain accesses.
#ifndef MPB_CHECKED
#define MPB_CHECKED 0
#endif
__device__ __forceinline__ bool in_bounds(long long i, long long n, int *status) {
#if MPB_CHECKED
  if ((unsigned long long)i < (unsigned long long)n) return true;
  atomicAdd(status + ST_BOUNDS, 1);
  return false;
#else
  (void)i;
  (void)n;
  (void)status;
  return true;
#endif
}
template <typename T>
__device__ __forceinline__ T ldg_c(const T *a, long long i, long long n, int *status) {
  return in_bounds(i, n, status) ? __ldg(a + i) : T{};
}
template <typename T>
__device__ __forceinline__ T ld_c(const T *a, long long i, long long n, int *status) {
  return in_bounds(i, n, status) ? a[i] : T{};
}
template <typename T>
__device__ __forceinline__ void st_c(T *a, long long i, long long n, int *status, T v) {
  if (in_bounds(i, n, status)) a[i] = v;
}

}  // namespace mpb

#endif
