// mp_init_kernels.cu - the field initialisers and FollowMax on the device.
//
// pulse_init (GaussPulseInit::init, pulseinit.cpp:7-74), gauss_init
// (PlaneGaussPulseInit::init, gaussinit.cpp:7-82) and wave_init
// (PlaneWaveInit::init, waveinit.cpp:9-60): one thread per stored cell (the
// interior x / y columns of every z plane), FP64 arithmetic in the
// reference's order, stored in the state precision.  FollowMax
// (followmax.cpp:73-113) is a short sequential hill climb along one grid line:
// one thread.
#include "mp_device.h"

#include <cuda_runtime.h>

namespace mpb {

template <typename T>
__global__ void __launch_bounds__(256) init_kernel(const InitParams q, T *Ex, T *Ey, T *Ez, T *Bx, T *By, T *Bz) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = q.k_lo + blockIdx.z;
  if (ii >= q.nx || jj >= q.ny || k > q.k_hi) return;
  const int i = ii + 1, j = jj + 1;  // MPulse indices
  const long long c = (long long)k * q.plane + (long long)jj * q.nx + ii;
  if (q.kind == 1) {
    // GaussPulseInit::init (pulseinit.cpp:33-71)
    const double dx2 = q.dx * q.dx, dy2 = q.dy * q.dy;
    const double nkz = q.dz * q.kz;
    const double rr0 = q.r0 * q.r0, zz0 = q.z0 * q.z0;
    const double iie = i - q.xh, jje = j - q.yh;
    const double rre = (iie * iie * dx2 + jje * jje * dy2) / rr0;
    const double iib = i + 0.5 - q.xh, jjb = j + 0.5 - q.yh;
    const double rrb = (iib * iib * dx2 + jjb * jjb * dy2) / rr0;
    const double nze = k * q.dz - q.zc, nzb = (k + 0.5) * q.dz - q.zc;
    const double kze = k * nkz, kzb = (k + 0.5) * nkz;
    const double ampe = cos(kze - q.C * rre) * exp(-nze * nze / zz0 - rre);
    const double ampb = cos(kzb - q.C * rrb) * exp(-nzb * nzb / zz0 - rrb);
    Ex[c] = T(q.ex * ampe);
    Ey[c] = T(q.ey * ampe);
    Ez[c] = T(0);
    Bx[c] = T(q.bx * ampb);
    By[c] = T(q.by * ampb);
    Bz[c] = T(0);
  } else if (q.kind == 2) {
    // PlaneGaussPulseInit::init (gaussinit.cpp:43-78)
    const double delta = 0.5;
    const double pose = (i - q.xh) * q.kx + (j - q.yh) * q.ky + (k - q.zh) * q.kz;
    const double posb = (i + delta - q.xh) * q.kx + (j + delta - q.yh) * q.ky + (k + delta - q.zh) * q.kz;
    const double ampe = exp(-pose * pose);
    const double ampb = exp(-posb * posb);
    Ex[c] = T(q.ex * ampe);
    Ey[c] = T(q.ey * ampe);
    Ez[c] = T(q.ez * ampe);
    Bx[c] = T(-q.bx * ampb);
    By[c] = T(-q.by * ampb);
    Bz[c] = T(-q.bz * ampb);
  } else {
    // PlaneWaveInit::init (waveinit.cpp:38-57): added to the fields
    const int i1 = i - 1, j1 = j - 1, k1 = k - 1;
    const double ampex = cos((i1 + 0.5) * q.kx + j1 * q.ky + k1 * q.kz);
    const double ampey = cos(i1 * q.kx + (j1 + 0.5) * q.ky + k1 * q.kz);
    const double ampez = cos(i1 * q.kx + j1 * q.ky + (k1 + 0.5) * q.kz);
    const double ampbx = cos(i1 * q.kx + (j1 + 0.5) * q.ky + (k1 + 0.5) * q.kz);
    const double ampby = cos((i1 + 0.5) * q.kx + j1 * q.ky + (k1 + 0.5) * q.kz);
    const double ampbz = cos((i1 + 0.5) * q.kx + (j1 + 0.5) * q.ky + k1 * q.kz);
    Ex[c] = T((double)Ex[c] + q.ex * ampex);
    Ey[c] = T((double)Ey[c] + q.ey * ampey);
    Ez[c] = T((double)Ez[c] + q.ez * ampez);
    Bx[c] = T((double)Bx[c] + q.bx * ampbx);
    By[c] = T((double)By[c] + q.by * ampby);
    Bz[c] = T((double)Bz[c] + q.bz * ampbz);
  }
}

template <typename T>
cudaError_t launch_init(const InitParams &q, void *const F[6], cudaStream_t st) {
  if (q.k_hi < q.k_lo) return cudaSuccess;
  const dim3 b(32, 8, 1), g((q.nx + 31) / 32, (q.ny + 7) / 8, q.k_hi - q.k_lo + 1);
  init_kernel<T><<<g, b, 0, st>>>(q, static_cast<T *>(F[0]), static_cast<T *>(F[1]), static_cast<T *>(F[2]),
                                  static_cast<T *>(F[3]), static_cast<T *>(F[4]), static_cast<T *>(F[5]));
  return cudaGetLastError();
}

template cudaError_t launch_init<float>(const InitParams &, void *const[6], cudaStream_t);
template cudaError_t launch_init<double>(const InitParams &, void *const[6], cudaStream_t);

// FollowMax::calculate (followmax.cpp:73-113): the line through MPulse cell
// pos along dim; indices wrap inside 1..n (low = 0, high = n + 1).  At most n
// moves (each one goes to a strictly larger value).
template <typename T>
__global__ void follow_max_kernel(const T *G, int nx, int ny, int nz, long long plane, int dim, int px, int py,
                                  int pz, int *ipos, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int n = dim == 0 ? nx : dim == 1 ? ny : nz;
  int p[3] = {px, py, pz};
  auto at = [&](int v) {
    p[dim] = v;
    return (double)G[(long long)p[2] * plane + (long long)(p[1] - 1) * nx + (p[0] - 1)];
  };
  int ip = *ipos;
  double mid = 0, left = 0, right = 0;
  for (int it = 0; it <= n; ++it) {
    int pm = ip - 1, pp = ip + 1;
    if (pm <= 0) pm = n;
    if (pp >= n + 1) pp = 1;
    mid = at(ip);
    left = at(pm);
    right = at(pp);
    if (right > mid) ip = pp;
    else if (left > mid) ip = pm;
    else break;
  }
  *ipos = ip;
  out[0] = ip + (left - right) / (2 * (left - 2 * mid + right));  // vertex of the parabola
}

template <typename T>
cudaError_t launch_follow_max(const void *G, int nx, int ny, int nz, long long plane, int dim, const int pos[3],
                              int *ipos, double *out, cudaStream_t st) {
  follow_max_kernel<T><<<1, 32, 0, st>>>(static_cast<const T *>(G), nx, ny, nz, plane, dim, pos[0], pos[1], pos[2],
                                         ipos, out);
  return cudaGetLastError();
}

template cudaError_t launch_follow_max<float>(const void *, int, int, int, long long, int, const int[3], int *,
                                              double *, cudaStream_t);
template cudaError_t launch_follow_max<double>(const void *, int, int, int, long long, int, const int[3], int *,
                                               double *, cudaStream_t);

}  // namespace mpb
