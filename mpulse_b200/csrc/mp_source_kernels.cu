// mp_source_kernels.cu - per-step values of the TF/SF injection planes.
//
// For every built injector kind MPulse adds currents on the `down` face only
// (PlaneWaveSource / PlaneGaussSource::needCurrent, sources.cpp:8-11, :179-182;
// ShortPulseInject::needCurrent, shortpulseinject.cpp:28-31).  Per step:
//   E side (IncidentSourceECurrent::stepScheme, incsource.t:40-73): on plane
//     z = d, J_x = H_inc,y(i, j, d-1, t) / dz and J_y = H_inc,x / dz;
//   H side (IncidentSourceHCurrent::stepScheme, incsource.t:112-145): on plane
//     z = d-1, M_x = E_inc,y(i, j, d-1, t) / dz and M_y = E_inc,x / dz,
// with t = Process::time.  One thread per interior (i, j); the step kernels
// read the two planes written here.
#include "mp_device.h"
#include "mp_pulse_math.h"

#include <cuda_runtime.h>

namespace mpb {

// getHField of PlaneWaveSourceEFunc / PlaneGaussSourceEFunc (sources.cpp:107-125,
// :266-284) and getEField of the H functions (sources.cpp:150-173, :308-331).
__device__ void plane_source_field(const SourceEvalParams &q, int i, int j, int l, double out[3]) {
  const double *k = q.k;
  double pos[3];
  if (!q.isH) {
    const double realtime = q.dt * ((double)q.time - 0.5);
    pos[0] = k[0] * i * q.dx + k[1] * (j + 0.5) * q.dy + k[2] * (l + 0.5) * q.dz + q.om * realtime;
    pos[1] = k[0] * (i + 0.5) * q.dx + k[1] * j * q.dy + k[2] * (l + 0.5) * q.dz + q.om * realtime;
    pos[2] = k[0] * (i + 0.5) * q.dx + k[1] * (j + 0.5) * q.dy + k[2] * l * q.dz + q.om * realtime;
  } else {
    const double realtime = q.dt * (double)q.time;
    pos[0] = k[0] * (i + 0.5) * q.dx + k[1] * j * q.dy + k[2] * l * q.dz + q.om * realtime;
    pos[1] = k[0] * i * q.dx + k[1] * (j + 0.5) * q.dy + k[2] * l * q.dz + q.om * realtime;
    pos[2] = k[0] * i * q.dx + k[1] * j * q.dy + k[2] * (l + 0.5) * q.dz + q.om * realtime;
  }
  for (int c = 0; c < 3; ++c) {
    if (q.kind == 1) {  // MP_SOURCE_PLANE_WAVE
      double v = q.amp3[c] * sin(pos[c]) + q.bg[c];
      if (pos[c] < q.ramp) v *= pos[c] / q.ramp;
      out[c] = v;
    } else {            // MP_SOURCE_PLANE_GAUSS
      const double a = (pos[c] - q.offset) / q.width;
      out[c] = q.amp3[c] * exp(-(a * a)) * sin(pos[c]);
    }
  }
}

// ShortPulseInjectSourceFunc::getHField / getEField (shortpulseinject.cpp:126-178).
__device__ void short_pulse_field(const SourceEvalParams &q, int i, int j, int l, double out[3]) {
  ShortPulse sp;
  sp.c = q.lightspeed; sp.ZRl = q.ZRl; sp.phase = q.phase; sp.T = q.length; sp.om0 = q.om0;
  sp.coef = q.w_coef; sp.L = q.w_L;
  sp.eiphi = cd(q.sp_eiphi[0], q.sp_eiphi[1]);
  sp.emip = cd(q.sp_emip[0], q.sp_emip[1]);
  sp.g = q.sp_g;
  out[2] = 0.0;
  if (q.isH) {
    const double posxh = (i + 0.5 - q.centre[0]) * q.dx;
    const double posyo = (j - q.centre[1]) * q.dy;
    const double poszo = (l - q.centre[2]) * q.dz - q.zshift;
    const double t = (double)q.time * q.dt - q.tshift;
    out[0] = q.amp * short_pulse_e(sp, posxh, posyo, poszo, t).re;
    out[1] = 0.0;
  } else {
    const double posxo = (i - q.centre[0]) * q.dx;
    const double posxh = (i + 0.5 - q.centre[0]) * q.dx;
    const double posyo = (j - q.centre[1]) * q.dy;
    const double posyh = (j + 0.5 - q.centre[1]) * q.dy;
    const double poszh = (l - 0.5 - q.centre[2]) * q.dz - q.zshift;
    const double t = ((double)q.time - 0.5) * q.dt - q.tshift;
    out[0] = q.amp * short_pulse_b(sp, posxo, posyh, poszh, t, true).re;
    out[1] = q.amp * short_pulse_b(sp, posxh, posyo, poszh, t, false).re;
  }
}

// GaussInjectSourceFunc::getHField / getEField (gaussinject.cpp:204-222) on
// the block precomputed by mp_gauss_kernels.cu.
__device__ void gauss_beam_field(const SourceEvalParams &q, int i, int j, double out[3]) {
  out[0] = out[1] = out[2] = 0.0;
  if (!q.g_active) return;
  const long long o = (q.time - q.g_toff) * ((long long)q.nx * q.ny) + (long long)j * q.nx + i;
  out[0] = q.g_scale * q.g_f1[o];
  if (q.isH) out[1] = q.g_scale * q.g_f2[o];
}

// The incident field at interior column (i, j) (0-based; MPulse i + 1, j + 1).
__device__ void source_field(const SourceEvalParams &q, int i, int j, double f[3]) {
  if (q.kind == 3 || q.kind == 4) short_pulse_field(q, i + 1, j + 1, q.l, f);  // short / focused pulse
  else if (q.kind == 5) gauss_beam_field(q, i, j, f);
  else plane_source_field(q, i + 1, j + 1, q.l, f);
}

template <typename T>
__global__ void __launch_bounds__(256) source_plane_kernel(const SourceEvalParams q, T *v0, T *v1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= q.nx || j >= q.ny) return;
  double f[3];
  source_field(q, i, j, f);
  const long long col = (long long)j * q.nx + i;
  // J0 = F[t2] / DX, J1 = F[t1] / DX with (t1, t2) = (x, y) on z faces
  v0[col] = T(f[1] / q.DX);
  v1[col] = T(f[0] / q.DX);
}

template <typename T>
cudaError_t launch_source_plane(const SourceEvalParams &q, T *v0, T *v1, cudaStream_t st) {
  const dim3 b(32, 8, 1), g((q.nx + 31) / 32, (q.ny + 7) / 8, 1);
  source_plane_kernel<T><<<g, b, 0, st>>>(q, v0, v1);
  return cudaGetLastError();
}

// The planes of `nsteps` consecutive steps in one launch: the values depend
// only on Process::time, so step t0 + q's E-side pair goes to
// out + (4 q + 0, 1) * plane and its H-side pair to out + (4 q + 2, 3) * plane.
// The short-pulse closed forms are long FP64 expressions (about 240 registers
// unbounded, one block of 256 threads per SM): asking for MPB_SRC_MIN_BLOCKS
// blocks per SM trades spills for occupancy.  Measured on the 256 x 256 plane
// of the PLRC + Kerr workload: 1 / 2 / 3 blocks per SM 0.042 / 0.025 / 0.022
// ms per step; with the one-division Faddeeva function 2 / 3 / 4 blocks
// 0.0196 / 0.0183 / 0.0194 ms.
#ifndef MPB_SRC_MIN_BLOCKS
#define MPB_SRC_MIN_BLOCKS 3
#endif
template <typename T>
__global__ void __launch_bounds__(256, MPB_SRC_MIN_BLOCKS) source_batch_kernel(const SourceEvalParams qe, const SourceEvalParams qh,
                                                          long long t0, T *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= qe.nx || j >= qe.ny) return;
  const int step = blockIdx.z >> 1, side = blockIdx.z & 1;
  SourceEvalParams q = side ? qh : qe;
  q.time = t0 + step;
  double f[3];
  source_field(q, i, j, f);
  const long long plane = (long long)qe.nx * qe.ny;
  const long long col = (long long)j * qe.nx + i;
  T *v0 = out + (4LL * step + 2 * side) * plane;
  v0[col] = T(f[1] / q.DX);
  v0[plane + col] = T(f[0] / q.DX);
}

template <typename T>
cudaError_t launch_source_batch(const SourceEvalParams &qe, const SourceEvalParams &qh, long long t0, int nsteps,
                                T *out, cudaStream_t st) {
  const dim3 b(32, 8, 1), g((qe.nx + 31) / 32, (qe.ny + 7) / 8, 2 * nsteps);
  source_batch_kernel<T><<<g, b, 0, st>>>(qe, qh, t0, out);
  return cudaGetLastError();
}

template cudaError_t launch_source_plane<float>(const SourceEvalParams &, float *, float *, cudaStream_t);
template cudaError_t launch_source_plane<double>(const SourceEvalParams &, double *, double *, cudaStream_t);
template cudaError_t launch_source_batch<float>(const SourceEvalParams &, const SourceEvalParams &, long long, int,
                                                float *, cudaStream_t);
template cudaError_t launch_source_batch<double>(const SourceEvalParams &, const SourceEvalParams &, long long, int,
                                                 double *, cudaStream_t);

}  // namespace mpb
