// mp_gauss_kernels.cu - the block precompute of gauss_inject (mp_gauss.h).
//
// Per field and block:
//   spectrum_kernel  A(kx, ky, om) of fillEx / fillEy / fillBx
//                    (gaussinject.cpp:329-482), written for a slab of x rows in
//                    transformT's input order (uo[k] = A[(k + SizeT/2) % SizeT],
//                    :257-267);
//   cuFFT inverse    over om, batched over the slab's (x, y) columns (:269);
//   select_kernel    the block's Nt times, f = 2 pi length / BoxT (:271-277),
//                    stored in transformY's input order (:284-291);
//   cuFFT forward    over ky, batched over (x, t) (:292);
//   swap_kernel      f = width / BoxY (:293-297), into transformX's input order
//                    (:307-314);
//   cuFFT forward    over kx, batched over (y, t) (:316);
//   extract_kernel   f = width / BoxX, real part (:318-322), interior columns
//                    into the t-major planes the source kernel reads.
// Everything is FP64 whatever the step precision; the spectrum and the shuffles
// are memory-bound elementwise kernels, the transforms are library FFTs.
#include "mp_gauss.h"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace mpb {

namespace {

enum GaussComp { GC_EX = 0, GC_EY = 1, GC_BX = 2 };

struct SpecArgs {
  int SizeT, SizeX, SizeY, SizeTH, SizeXH, SizeYH;
  double BoxX, BoxY, BoxT;
  double k0, length, width;  // GaussFunc (gaussinject.h:166-203)
  double sx, sy, sz;         // GaussFunc::setShift
  double Time;
  int comp;
  int i0, rows;
};

// GaussFunc::gauss / shift / excomp / eycomp / bxcomp (gaussinject.h:176-201)
__device__ double gf_gauss(const SpecArgs &a, double x, double y, double z) {
  const double zoff = z - a.k0;
  return exp(-0.25 * zoff * zoff * a.length * a.length - 0.25 * (x * x + y * y) * a.width * a.width);
}

__device__ double gf_comp(int comp, double x, double y, double z) {
  if (comp == GC_EX) {
    const double D = sqrt(x * x + y * y + z * z) * sqrt(x * x + z * z);
    return D == 0 ? 0 : (-x * y / D);
  }
  if (comp == GC_EY) {
    const double D = sqrt(x * x + y * y + z * z);
    return D == 0 ? 0 : (sqrt(x * x + z * z) / D);
  }
  const double D = sqrt(x * x + z * z);
  return D == 0 ? 0 : (-z / D);
}

__global__ void __launch_bounds__(256) spectrum_kernel(const SpecArgs a, double2 *__restrict__ out) {
  const long long n = (long long)a.rows * a.SizeY * a.SizeT;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = int(idx % a.SizeT);  // position in transformT's input
    const long long r = idx / a.SizeT;
    const int j = int(r % a.SizeY);
    const int i = a.i0 + int(r / a.SizeY);
    const int kh = (k + a.SizeTH) % a.SizeT;  // frequency index
    const double kx = 2 * M_PI * (i - a.SizeXH) / (a.BoxX);
    const double ky = 2 * M_PI * (j - a.SizeYH) / (a.BoxY);
    const double om = 2 * M_PI * (kh - a.SizeTH) / (a.BoxT);
    // K = om^2 - ky^2 - kx^2 rounded term by term: the |K| < 1e-9 and K < 0
    // tests decide which modes propagate
    double K = __dsub_rn(__dsub_rn(__dmul_rn(om, om), __dmul_rn(ky, ky)), __dmul_rn(kx, kx));
    if (fabs(K) < 1e-9) K = 0;
    double2 v = make_double2(0.0, 0.0);
    if (!(K < 0)) {
      const double kz = sqrt(K) * (om > 0 ? 1 : (om < 0 ? -1 : 0));
      const double amp = gf_comp(a.comp, kx, ky, kz) * gf_gauss(a, kx, ky, kz);
      const double ph = -(kx * a.sx + ky * a.sy + kz * a.sz) + 0.5 * M_PI;
      double s, c;
      sincos(ph + a.Time * om, &s, &c);
      v = make_double2(amp * c, -amp * s);  // a exp(-i (ph + Time om))
    }
    out[idx] = v;
  }
}

// tmpField_TY(j, kh) = f ut[(kh + blockmin + SizeT/2) % SizeT], stored at
// y-transform input position (j + SizeY/2) % SizeY of batch (i, kh)
__global__ void __launch_bounds__(256) select_kernel(const double2 *__restrict__ spec, double2 *__restrict__ ybuf,
                                                     int SizeT, int SizeTH, int SizeY, int SizeYH, int Nt, int i0,
                                                     int rows, long long blockmin, double f) {
  const long long n = (long long)rows * SizeY * Nt;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int kh = int(idx % Nt);
    const long long r = idx / Nt;
    const int j = int(r % SizeY);
    const int il = int(r / SizeY);
    const int k = int((kh + blockmin + SizeTH) % SizeT);
    const double2 u = spec[((long long)il * SizeY + j) * SizeT + k];
    ybuf[((long long)(i0 + il) * Nt + kh) * SizeY + (j + SizeYH) % SizeY] = make_double2(f * u.x, f * u.y);
  }
}

// tmpField_TX(i, j, k) = f uy[(j + SizeY/2) % SizeY], stored at x-transform
// input position (i + SizeX/2) % SizeX of batch (j, k)
__global__ void __launch_bounds__(256) swap_kernel(const double2 *__restrict__ ybuf, double2 *__restrict__ xbuf,
                                                   int SizeX, int SizeXH, int SizeY, int SizeYH, int Nt, double f) {
  const long long n = (long long)SizeX * SizeY * Nt;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ip = int(idx % SizeX);  // output position
    const long long r = idx / SizeX;
    const int k = int(r % Nt);
    const int j = int(r / Nt);
    const int i = (ip - SizeXH + SizeX) % SizeX;  // (i + SizeXH) % SizeX == ip
    const double2 u = ybuf[((long long)i * Nt + k) * SizeY + (j + SizeYH) % SizeY];
    xbuf[idx] = make_double2(f * u.x, f * u.y);
  }
}

// F(i, j, k) = f Re ux[(i + SizeX/2) % SizeX] for the interior columns,
// t-major: out[(k ny + j - 1) nx + i - 1]
__global__ void __launch_bounds__(256) extract_kernel(const double2 *__restrict__ xbuf, double *__restrict__ out,
                                                      int nx, int ny, int SizeX, int SizeXH, int Nt, double f) {
  const long long n = (long long)nx * ny * Nt;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = int(idx % nx) + 1;
    const long long r = idx / nx;
    const int j = int(r % ny) + 1;
    const int k = int(r / ny);
    out[idx] = f * xbuf[((long long)j * Nt + k) * SizeX + (i + SizeXH) % SizeX].x;
  }
}

int grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return int(std::min<long long>(b, 148LL * 16));
}

int fail(std::string *err, int code, const char *what, const char *detail) {
  if (err) {
    char buf[256];
    snprintf(buf, sizeof buf, "gauss_inject %s: %s", what, detail);
    *err = buf;
  }
  return code;
}

int cufail(std::string *err, cufftResult r, const char *what) {
  char buf[64];
  snprintf(buf, sizeof buf, "cuFFT error %d", int(r));
  return fail(err, r == CUFFT_ALLOC_FAILED ? MP_ERR_NO_MEMORY : MP_ERR_CUDA, what, buf);
}

int cudafail(std::string *err, cudaError_t e, const char *what) {
  return fail(err, e == cudaErrorMemoryAllocation ? MP_ERR_NO_MEMORY : MP_ERR_CUDA, what, cudaGetErrorString(e));
}

cufftResult make_plan(cufftHandle *h, int n, int batch) {
  int nn[1] = {n};
  return cufftPlanMany(h, 1, nn, nullptr, 1, n, nullptr, 1, n, CUFFT_Z2Z, batch);
}

// Scratch for one slab of the spectrum, at most this many bytes (at least one x row).
const size_t kSlabBytes = size_t(512) << 20;

}  // namespace

int gauss_create(GaussBeam &g, const mp_source &q, const mp_config &c, std::string *err) {
  g = GaussBeam();
  g.SizeT = q.t_size;
  g.length = q.length;
  g.width = q.width;
  g.k0 = q.k0;
  g.Shift = q.shift;
  g.Time = q.time;
  g.amp = q.amp;
  g.eps = q.eps;
  g.toff = q.t_off;
  const double lightspeed = std::sqrt(1 / g.eps);
  g.SizeX = c.nx + 2;
  g.SizeY = c.ny + 2;
  g.SizeTH = g.SizeT / 2;
  g.SizeXH = g.SizeX / 2;
  g.SizeYH = g.SizeY / 2;
  g.DX = c.dx;
  g.DY = c.dy;
  g.DT = c.dt * lightspeed;
  g.BoxX = g.SizeX * g.DX;
  g.BoxY = g.SizeY * g.DY;
  g.BoxT = g.SizeT * g.DT;
  g.nx = c.nx;
  g.ny = c.ny;
  // initSourceFunc (gaussinject.cpp:134): the storage's z range is 0..nz+1
  g.Nt = 1 << int(std::round(std::log(double(c.nz + 1)) / std::log(2.0) + 1e-6));
  g.nblocks = (g.SizeT + g.Nt - 1) / g.Nt;

  const size_t col_bytes = size_t(g.SizeY) * g.SizeT * sizeof(double2);
  g.slab_rows = int(std::max<size_t>(1, std::min<size_t>(size_t(g.SizeX), kSlabBytes / col_bytes)));
  const size_t stage = size_t(g.SizeX) * g.SizeY * g.Nt;
  const size_t fplane = size_t(g.nx) * g.ny * g.Nt;
  cudaError_t e;
  if ((e = cudaMalloc(&g.spec, size_t(g.slab_rows) * col_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&g.ybuf, stage * sizeof(double2))) != cudaSuccess ||
      (e = cudaMalloc(&g.xbuf, stage * sizeof(double2))) != cudaSuccess ||
      (e = cudaMalloc(&g.bx, fplane * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&g.ex, fplane * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&g.ey, fplane * sizeof(double))) != cudaSuccess) {
    gauss_destroy(g);
    return cudafail(err, e, "allocation");
  }
  cufftResult r;
  if ((r = make_plan(&g.plan_t, g.SizeT, g.slab_rows * g.SizeY)) != CUFFT_SUCCESS) {
    gauss_destroy(g);
    return cufail(err, r, "plan over t");
  }
  g.have_t = true;
  const int last = g.SizeX % g.slab_rows;
  if (last) {
    if ((r = make_plan(&g.plan_t_last, g.SizeT, last * g.SizeY)) != CUFFT_SUCCESS) {
      gauss_destroy(g);
      return cufail(err, r, "plan over t");
    }
    g.have_t_last = true;
  }
  if ((r = make_plan(&g.plan_y, g.SizeY, g.SizeX * g.Nt)) != CUFFT_SUCCESS) {
    gauss_destroy(g);
    return cufail(err, r, "plan over y");
  }
  g.have_y = true;
  if ((r = make_plan(&g.plan_x, g.SizeX, g.SizeY * g.Nt)) != CUFFT_SUCCESS) {
    gauss_destroy(g);
    return cufail(err, r, "plan over x");
  }
  g.have_x = true;
  return MP_OK;
}

void gauss_destroy(GaussBeam &g) {
  if (g.have_t) cufftDestroy(g.plan_t);
  if (g.have_t_last) cufftDestroy(g.plan_t_last);
  if (g.have_y) cufftDestroy(g.plan_y);
  if (g.have_x) cufftDestroy(g.plan_x);
  cudaFree(g.spec);
  cudaFree(g.ybuf);
  cudaFree(g.xbuf);
  cudaFree(g.bx);
  cudaFree(g.ex);
  cudaFree(g.ey);
  g = GaussBeam();
}

namespace {

// One of fillEx / fillEy / fillBx for block b into `out`.
int fill(GaussBeam &g, int comp, double sx, double sy, double sz, double Time, long long b, double *out,
         cudaStream_t st, long long *launches, std::string *err) {
  SpecArgs a;
  a.SizeT = g.SizeT; a.SizeX = g.SizeX; a.SizeY = g.SizeY;
  a.SizeTH = g.SizeTH; a.SizeXH = g.SizeXH; a.SizeYH = g.SizeYH;
  a.BoxX = g.BoxX; a.BoxY = g.BoxY; a.BoxT = g.BoxT;
  a.k0 = g.k0; a.length = g.length; a.width = g.width;
  a.sx = sx; a.sy = sy; a.sz = sz;
  a.Time = Time;
  a.comp = comp;
  const long long blockmin = b * g.Nt;
  cufftResult r;
  cudaError_t e;
  for (int i0 = 0; i0 < g.SizeX; i0 += g.slab_rows) {
    a.i0 = i0;
    a.rows = std::min(g.slab_rows, g.SizeX - i0);
    const long long n = (long long)a.rows * g.SizeY * g.SizeT;
    spectrum_kernel<<<grid_for(n), 256, 0, st>>>(a, g.spec);
    if ((e = cudaGetLastError()) != cudaSuccess) return cudafail(err, e, "spectrum kernel");
    ++*launches;
    cufftHandle p = a.rows == g.slab_rows ? g.plan_t : g.plan_t_last;
    if ((r = cufftSetStream(p, st)) != CUFFT_SUCCESS) return cufail(err, r, "stream");
    if ((r = cufftExecZ2Z(p, reinterpret_cast<cufftDoubleComplex *>(g.spec),
                          reinterpret_cast<cufftDoubleComplex *>(g.spec), CUFFT_INVERSE)) != CUFFT_SUCCESS)
      return cufail(err, r, "transform over t");
    const long long m = (long long)a.rows * g.SizeY * g.Nt;
    select_kernel<<<grid_for(m), 256, 0, st>>>(g.spec, g.ybuf, g.SizeT, g.SizeTH, g.SizeY, g.SizeYH, g.Nt, i0,
                                               a.rows, blockmin, (2 * M_PI * g.length / g.BoxT));
    if ((e = cudaGetLastError()) != cudaSuccess) return cudafail(err, e, "select kernel");
    ++*launches;
  }
  if ((r = cufftSetStream(g.plan_y, st)) != CUFFT_SUCCESS) return cufail(err, r, "stream");
  if ((r = cufftExecZ2Z(g.plan_y, reinterpret_cast<cufftDoubleComplex *>(g.ybuf),
                        reinterpret_cast<cufftDoubleComplex *>(g.ybuf), CUFFT_FORWARD)) != CUFFT_SUCCESS)
    return cufail(err, r, "transform over y");
  const long long s = (long long)g.SizeX * g.SizeY * g.Nt;
  swap_kernel<<<grid_for(s), 256, 0, st>>>(g.ybuf, g.xbuf, g.SizeX, g.SizeXH, g.SizeY, g.SizeYH, g.Nt,
                                           (g.width / g.BoxY));
  if ((e = cudaGetLastError()) != cudaSuccess) return cudafail(err, e, "swap kernel");
  ++*launches;
  if ((r = cufftSetStream(g.plan_x, st)) != CUFFT_SUCCESS) return cufail(err, r, "stream");
  if ((r = cufftExecZ2Z(g.plan_x, reinterpret_cast<cufftDoubleComplex *>(g.xbuf),
                        reinterpret_cast<cufftDoubleComplex *>(g.xbuf), CUFFT_FORWARD)) != CUFFT_SUCCESS)
    return cufail(err, r, "transform over x");
  const long long x = (long long)g.nx * g.ny * g.Nt;
  extract_kernel<<<grid_for(x), 256, 0, st>>>(g.xbuf, out, g.nx, g.ny, g.SizeX, g.SizeXH, g.Nt,
                                              (g.width / g.BoxX));
  if ((e = cudaGetLastError()) != cudaSuccess) return cudafail(err, e, "extract kernel");
  ++*launches;
  return MP_OK;
}

}  // namespace

int gauss_prepare(GaussBeam &g, long long time, cudaStream_t st, bool *active, long long *block_toff,
                  long long *until, long long *launches, std::string *err) {
  // setTime (gaussinject.cpp:152-184) for a time that steps by one: off before
  // toff, block b = (t - toff) / Nt while b Nt < SizeT, off afterwards
  *block_toff = 0;
  if (time < g.toff) {
    *active = false;
    *until = g.toff;
    return MP_OK;
  }
  const long long b = (time - g.toff) / g.Nt;
  if (b >= g.nblocks) {
    *active = false;
    *until = -1;  // never changes again
    return MP_OK;
  }
  *active = true;
  *block_toff = g.toff + b * g.Nt;
  *until = *block_toff + g.Nt;
  if (g.computed == b) return MP_OK;
  g.computed = -1;
  int rc;
  // E current: fillBx with the shift (0, DX/2, Shift + DX/2) (:163-166)
  if ((rc = fill(g, GC_BX, 0, 0.5 * g.DX, g.Shift + 0.5 * g.DX, g.Time, b, g.bx, st, launches, err)) != MP_OK)
    return rc;
  // H current: Time - DT/2 (:169-175).  The reference subtracts and adds DT/2
  // back once per block, which moves Time by rounding; repeated here so block b
  // sees the same value.
  double T = g.Time;
  for (long long n = 0; n < b; ++n) T = (T - 0.5 * g.DT) + 0.5 * g.DT;
  const double Th = T - 0.5 * g.DT;
  if ((rc = fill(g, GC_EX, 0.5 * g.DX, 0, g.Shift, Th, b, g.ex, st, launches, err)) != MP_OK) return rc;
  if ((rc = fill(g, GC_EY, 0, 0.5 * g.DX, g.Shift, Th, b, g.ey, st, launches, err)) != MP_OK) return rc;
  g.computed = b;
  return MP_OK;
}

}  // namespace mpb
