// mp_adjoint_kernels.cu - the discrete adjoint of one PLRC step and the
// objective kernels of mp_objective / mp_adjoint.
//
// The forward step (mp_step_kernels.cu) maps the state (E, B, PLRC
// accumulators psi, CPML psi) of step n to that of step n+1:
//   E half  psiE' = b psiE + c d(B);  X = (numer + chi|E|^2) E + dt (curl_E B +
//           J) + Re sum psi~;  E' = X / denom (linear) or the Kerr solve
//           |E'| + A |E'|^3 = |X / denom| along X (nonlinear);
//           psi' = s dxi0 E + Crec psi~, psi~ = s (dchi0 - dxi0) E + psi;
//   B half  psiH' = b psiH + c d(E');  B' = B + dt (curl_H E' + M).
// Its adjoint runs the two halves backwards.  The adjoint of a CPML psi is
// carried as a "total" (its own adjoint after the half plus dt times the
// adjoint of the component it feeds), so that every kernel writes only its
// own cell:
//   adj_e_kernel (E cells, planes 1..nz)  gathers the adjoint of E' from the
//     adjoint of B' through the transposed curl_H and the H-face totals, then
//     undoes the E half locally (linearised Kerr, reverse PLRC recursion),
//     accumulates the design gradients, stores the numerator adjoint G and
//     advances its E-face totals;
//   adj_b_kernel (B cells, planes 0..nz)  gathers the adjoint of B from G
//     through the transposed curl_E and the E-face totals, adds the
//     objective's B term and advances its H-face totals.
// All arithmetic is FP64; the adjoint state is stored in the precision of the
// forward state and the gradients in FP64.  Memory-bound, one thread per cell.
#include "mp_device.h"

#include <cuda_runtime.h>

namespace mpb {

namespace {

template <typename T>
__device__ __forceinline__ bool face_at(const AdjFace<T> &F, int i, int j, int k, int nx, int ny, int nz,
                                        long long &li, int &idx) {
  if (!F.active) return false;
  idx = F.dim == 0 ? i + 1 : F.dim == 1 ? j + 1 : k;
  if (idx < F.lo || idx > F.hi) return false;
  if (F.dim == 2) {
    li = ((long long)(k - F.lo) * ny + j) * nx + i;
    return true;
  }
  if (k < F.zlo || k > nz) return false;  // x / y faces cover planes zlo..nz
  if (F.dim == 0) li = ((long long)(k - F.zlo) * ny + j) * F.ex + (i + 1 - F.lo);
  else li = ((long long)(k - F.zlo) * F.ey + (j + 1 - F.lo)) * nx + i;
  return true;
}

// c * total of a face at (i, j, k), zero outside the face
template <typename T>
__device__ __forceinline__ void face_w(const AdjFace<T> &F, int i, int j, int k, int nx, int ny, int nz, double &w0,
                                       double &w1) {
  long long li;
  int idx;
  if (face_at(F, i, j, k, nx, ny, nz, li, idx)) {
    const double c = (double)F.c[idx];
    w0 = c * (double)F.a0[li];
    w1 = c * (double)F.a1[li];
  } else {
    w0 = w1 = 0.0;
  }
}

// components fed by psi0 / psi1 of a face along dim (cpml_border.cpp:357-386)
__device__ __forceinline__ void face_comps(int dim, int &c0, int &c1) {
  if (dim == 2) { c0 = 0; c1 = 1; }
  else if (dim == 0) { c0 = 1; c1 = 2; }
  else { c0 = 2; c1 = 0; }
}

}  // namespace

template <typename T, int NP>
__global__ void __launch_bounds__(256) adj_e_kernel(const AdjParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z + 1;
  if (i >= p.nx || j >= p.ny) return;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int im = i == 0 ? nx - 1 : i - 1;
  const int jm = j == 0 ? ny - 1 : j - 1;
  const long long pl = p.plane, col = (long long)j * nx + i;
  const long long c0 = (long long)k * pl + col;
  const long long cxm = (long long)k * pl + (long long)j * nx + im;
  const long long cym = (long long)k * pl + (long long)jm * nx + i;
  const long long czm = c0 - pl;
  const double dt = p.dt;

  // ---- adjoint of E' (B half transposed)
  double a[3] = {(double)p.Eb[0][c0], (double)p.Eb[1][c0], (double)p.Eb[2][c0]};
  {
    const double kxi = p.ikH[0][i + 1], kxm = p.ikH[0][im + 1];
    const double kyj = p.ikH[1][j + 1], kym = p.ikH[1][jm + 1];
    const double kzk = p.ikH[2][k], kzm = p.ikH[2][k - 1];
    const double bzj = p.ikH_bzy[j + 1], bzm = p.ikH_bzy[jm + 1];
    const T *Bx = p.Bb[0], *By = p.Bb[1], *Bz = p.Bb[2];
    // Bx' = .. + dt ((ey(k+1) - ey) ikz - (ez(j+1) - ez) iky)
    a[1] += dt * (kzm * (double)Bx[czm] - kzk * (double)Bx[c0]);
    a[2] += dt * (-kym * (double)Bx[cym] + kyj * (double)Bx[c0]);
    // By' = .. + dt ((ez(i+1) - ez) ikx - (ex(k+1) - ex) ikz)
    a[2] += dt * (kxm * (double)By[cxm] - kxi * (double)By[c0]);
    a[0] += dt * (-kzm * (double)By[czm] + kzk * (double)By[c0]);
    // Bz' = .. + dt ((ex(j+1) - ex) iky_bz - (ey(i+1) - ey) ikx)
    a[0] += dt * (bzm * (double)Bz[cym] - bzj * (double)Bz[c0]);
    a[1] += dt * (-kxm * (double)Bz[cxm] + kxi * (double)Bz[c0]);
  }
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const AdjFace<T> &F = p.fh[f];
    if (!F.active) continue;
    double w0o, w1o, w0m, w1m;
    face_w(F, i, j, k, nx, ny, nz, w0o, w1o);
    if (F.dim == 2) {
      face_w(F, i, j, k - 1, nx, ny, nz, w0m, w1m);
      a[1] += w0m - w0o;
      a[0] += w1o - w1m;
    } else if (F.dim == 0) {
      face_w(F, im, j, k, nx, ny, nz, w0m, w1m);
      a[2] += w0m - w0o;
      a[1] += w1o - w1m;
    } else {
      face_w(F, i, jm, k, nx, ny, nz, w0m, w1m);
      a[0] += w0m - w0o;
      a[2] += w1o - w1m;
    }
  }

  // ---- E half, locally
  const double En[3] = {(double)p.En[0][c0], (double)p.En[1][c0], (double)p.En[2][c0]};
  double g[3], ne[3];
  const bool med = k >= p.mz0 && k <= p.mz1;
  if (!med) {
    // background: E' = (eps_bg E + dt (curl + J)) / eps_bg
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      g[c] = a[c] / p.eps_bg;
      ne[c] = p.eps_bg * g[c];
    }
  } else {
    const DesignParams &d = p.design;
    const bool dcell = i >= d.x0 && i <= d.x1 && j >= d.y0 && j <= d.y1 && k >= d.z0 && k <= d.z1;
    long long di = 0;
    double e = p.eps, s = 1.0, u = 1.0;
    if (dcell) {
      di = ((long long)(k - d.z0) * d.by + (j - d.y0)) * d.bx + (i - d.x0);
      e = d.eps[di];
      s = d.dscale[di];
      u = d.chiscale[di];
    }
    const double dD = p.sumChi0 - p.sumXi0;
    const double numer = e - s * p.sumXi0;
    const double denom = d.lin ? e + s * dD : e + s * p.sumChi0 - s * p.sumXi0;
    const double chi = p.nonlin ? u * p.chi : 0.0;
    const double A = chi / denom;
    const double En1[3] = {(double)p.En1[0][c0], (double)p.En1[1][c0], (double)p.En1[2][c0]};
    double cbar[3], cvec[3], Abar = 0.0;
    if (p.nonlin) {
      // E' = r c/|c| with r + A r^3 = |c|: dE'/dc = (I - e e^T) / (1 + A r^2)
      // + e e^T / (1 + 3 A r^2), dr/dA = -r^3 / (1 + 3 A r^2), c = E' (1 + A r^2)
      const double r2 = En1[0] * En1[0] + En1[1] * En1[1] + En1[2] * En1[2];
      const double r = sqrt(r2);
      const double al = 1.0 / (1.0 + A * r2), be = 1.0 / (1.0 + 3.0 * A * r2);
      double eh[3] = {0.0, 0.0, 0.0};
      if (r > 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) eh[c] = En1[c] / r;
      }
      const double ea = eh[0] * a[0] + eh[1] * a[1] + eh[2] * a[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cbar[c] = al * (a[c] - eh[c] * ea) + be * eh[c] * ea;
        cvec[c] = En1[c] * (1.0 + A * r2);
      }
      Abar = -ea * r * r2 * be;
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cbar[c] = a[c];
        cvec[c] = En1[c];
      }
    }
    const double E2 = En[0] * En[0] + En[1] * En[1] + En[2] * En[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] = cbar[c] / denom;
    const double Eg = En[0] * g[0] + En[1] * g[1] + En[2] * g[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) ne[c] = (numer + chi * E2) * g[c] + 2.0 * chi * En[c] * Eg;
    // reverse PLRC recursion (pairs over the medium planes)
    double gs = 0.0, SD = 0.0;
    const long long pi = ((long long)(k - p.mz0) * ny + j) * nx + i;
#pragma unroll
    for (int n = 0; n < NP; ++n) {
      const double Dr = p.pD[n][0], Di = p.pD[n][1];
      const double Xr = p.pxi[n][0], Xi = p.pxi[n][1];
      const double Cr = p.pC[n][0], Ci = p.pC[n][1];
      const double CDr = Cr * Dr - Ci * Di, CDi = Cr * Di + Ci * Dr;
      SD += Dr;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T *q = p.psib[n][c] + 2 * pi;
        const double pr = (double)q[0], pim = (double)q[1];
        // psi~bar = conj(Crec) psibar + g
        const double tr = Cr * pr + Ci * pim + g[c];
        const double ti = Cr * pim - Ci * pr;
        ne[c] += s * (Dr * tr + Di * ti) + s * (Xr * pr + Xi * pim);
        gs += pr * (Xr + CDr) * En[c] + pim * (Xi + CDi) * En[c];
        q[0] = T(tr);
        q[1] = T(ti);
      }
    }
    if (dcell) {
      double ge = -Abar * A / denom, gu = 0.0;
      gs -= Abar * A * dD / denom;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ge += g[c] * (En[c] - cvec[c]);
        gs += g[c] * ((SD - p.sumXi0) * En[c] - cvec[c] * dD);
      }
      if (p.nonlin) {
        gu = Abar * p.chi / denom;
#pragma unroll
        for (int c = 0; c < 3; ++c) gu += g[c] * p.chi * E2 * En[c];
      }
      p.grad[0][di] += ge;
      p.grad[1][di] += gs;
      p.grad[2][di] += gu;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) p.G[c][c0] = T(g[c]);
  // ---- the objective's E term of the state before the step
  if (p.add_obj) {
    if (p.obj_kind == 1) {
      if (i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1 && k >= p.oz0 && k <= p.oz1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) ne[c] += p.obj_f * En[c];
      }
    } else if (k == p.oz0 && i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1) {
      ne[0] += p.obj_f * (double)p.oby[col];
      ne[1] -= p.obj_f * (double)p.obx[col];
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) p.Eb[c][c0] = T(ne[c]);
  // ---- E-face totals of this cell: b * total + dt * G
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const AdjFace<T> &F = p.fe[f];
    long long li;
    int idx;
    if (!face_at(F, i, j, k, nx, ny, nz, li, idx)) continue;
    int q0, q1;
    face_comps(F.dim, q0, q1);
    const double b = (double)F.b[idx];
    F.a0[li] = T(b * (double)F.a0[li] + dt * g[q0]);
    F.a1[li] = T(b * (double)F.a1[li] + dt * g[q1]);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) adj_b_kernel(const AdjParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;  // 0..nz
  if (i >= p.nx || j >= p.ny) return;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int ip = i == nx - 1 ? 0 : i + 1;
  const int jp = j == ny - 1 ? 0 : j + 1;
  const long long pl = p.plane, col = (long long)j * nx + i;
  const long long c0 = (long long)k * pl + col;
  const long long cxp = (long long)k * pl + (long long)j * nx + ip;
  const long long cyp = (long long)k * pl + (long long)jp * nx + i;
  const long long czp = c0 + pl;
  const double dt = p.dt;
  double b[3] = {(double)p.Bb[0][c0], (double)p.Bb[1][c0], (double)p.Bb[2][c0]};
  {
    const T *gx = p.G[0], *gy = p.G[1], *gz = p.G[2];
    const double kxi = p.ikE[0][i + 1], kxp = p.ikE[0][ip + 1];
    const double kyj = p.ikE[1][j + 1], kyp = p.ikE[1][jp + 1];
    const double kzk = p.ikE[2][k], kzp = p.ikE[2][k + 1];
    // cbx = (bz - bz(j-1)) iky - (by - by(k-1)) ikz
    b[2] += dt * (kyj * (double)gx[c0] - kyp * (double)gx[cyp]);
    b[1] += dt * (-kzk * (double)gx[c0] + kzp * (double)gx[czp]);
    // cby = (bx - bx(k-1)) ikz - (bz - bz(i-1)) ikx
    b[0] += dt * (kzk * (double)gy[c0] - kzp * (double)gy[czp]);
    b[2] += dt * (-kxi * (double)gy[c0] + kxp * (double)gy[cxp]);
    // cbz = (by - by(i-1)) ikx - (bx - bx(j-1)) iky
    b[1] += dt * (kxi * (double)gz[c0] - kxp * (double)gz[cxp]);
    b[0] += dt * (-kyj * (double)gz[c0] + kyp * (double)gz[cyp]);
  }
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const AdjFace<T> &F = p.fe[f];
    if (!F.active) continue;
    double w0o, w1o, w0p, w1p;
    face_w(F, i, j, k, nx, ny, nz, w0o, w1o);
    if (F.dim == 2) {
      face_w(F, i, j, k + 1, nx, ny, nz, w0p, w1p);
      b[1] += -w0o + w0p;
      b[0] += w1o - w1p;
    } else if (F.dim == 0) {
      face_w(F, ip, j, k, nx, ny, nz, w0p, w1p);
      b[2] += -w0o + w0p;
      b[1] += w1o - w1p;
    } else {
      face_w(F, i, jp, k, nx, ny, nz, w0p, w1p);
      b[0] += -w0o + w0p;
      b[2] += w1o - w1p;
    }
  }
  // the objective's B term of the state before the step (Sz plane)
  if (p.add_obj && p.obj_kind == 2 && k == p.oz0 && i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1) {
    b[0] -= p.obj_f * (double)p.En[1][c0];
    b[1] += p.obj_f * (double)p.En[0][c0];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) p.Bb[c][c0] = T(b[c]);
  // H-face totals for the step before: b * total + dt * adjoint of B
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const AdjFace<T> &F = p.fh[f];
    long long li;
    int idx;
    if (!face_at(F, i, j, k, nx, ny, nz, li, idx)) continue;
    int q0, q1;
    face_comps(F.dim, q0, q1);
    const double bb = (double)F.b[idx];
    F.a0[li] = T(bb * (double)F.a0[li] + dt * b[q0]);
    F.a1[li] = T(bb * (double)F.a1[li] + dt * b[q1]);
  }
}

// Start of the reverse pass (state T): the adjoint of E and B is the
// objective's derivative with respect to that state, the H-face totals dt times
// the adjoint of B, everything else zero (the arrays arrive zeroed).
template <typename T>
__global__ void __launch_bounds__(256) adj_init_kernel(const AdjParams<T> p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;  // 0..nz
  if (i >= p.nx || j >= p.ny) return;
  const long long col = (long long)j * p.nx + i, c0 = (long long)k * p.plane + col;
  double e[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
  const bool inxy = i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1;
  if (p.obj_kind == 1) {
    if (inxy && k >= p.oz0 && k <= p.oz1)
      for (int c = 0; c < 3; ++c) e[c] = p.obj_f * (double)p.En[c][c0];
  } else if (inxy && k == p.oz0) {
    e[0] = p.obj_f * (double)p.oby[col];
    e[1] = -p.obj_f * (double)p.obx[col];
    b[0] = -p.obj_f * (double)p.En[1][c0];
    b[1] = p.obj_f * (double)p.En[0][c0];
  }
  for (int c = 0; c < 3; ++c) {
    p.Eb[c][c0] = T(e[c]);
    p.Bb[c][c0] = T(b[c]);
  }
  for (int f = 0; f < 6; ++f) {
    const AdjFace<T> &F = p.fh[f];
    long long li;
    int idx;
    if (!face_at(F, i, j, k, p.nx, p.ny, p.nz, li, idx)) continue;
    int q0, q1;
    face_comps(F.dim, q0, q1);
    F.a0[li] = T(p.dt * b[q0]);
    F.a1[li] = T(p.dt * b[q1]);
  }
}

// One step's objective term into out[slot]: one block, FP64, fixed order.
template <typename T>
__global__ void __launch_bounds__(256) objective_term_kernel(const T *Ex, const T *Ey, const T *Ez, const T *Bx,
                                                             const T *By, int nx, int ny, long long plane, int kind,
                                                             int x0, int x1, int y0, int y1, int z0, int z1,
                                                             double f, double *out) {
  __shared__ double red[256];
  const int bx = x1 - x0 + 1, by = y1 - y0 + 1, bz = z1 - z0 + 1;
  const long long n = (long long)bx * by * bz;
  double acc = 0.0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const int i = x0 + int(q % bx);
    const long long r = q / bx;
    const int j = y0 + int(r % by);
    const int k = z0 + int(r / by);
    const long long c = (long long)k * plane + (long long)j * nx + i;
    if (kind == 1) {
      const double ex = Ex[c], ey = Ey[c], ez = Ez[c];
      acc += ex * ex + ey * ey + ez * ez;
    } else {
      acc += (double)Ex[c] * (double)By[c] - (double)Ey[c] * (double)Bx[c];
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = f * red[0];
}

__global__ void __launch_bounds__(256) sum_terms_kernel(const double *terms, long long n, double *out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) acc += terms[q];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// ---------------------------------------------------------------------------
// Launchers

template <typename T>
cudaError_t launch_adj_e(const AdjParams<T> &p, cudaStream_t st) {
  const dim3 b(32, 8, 1), g((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz);
  switch (p.np) {
    case 0: adj_e_kernel<T, 0><<<g, b, 0, st>>>(p); break;
    case 1: adj_e_kernel<T, 1><<<g, b, 0, st>>>(p); break;
    case 2: adj_e_kernel<T, 2><<<g, b, 0, st>>>(p); break;
    default: adj_e_kernel<T, 3><<<g, b, 0, st>>>(p); break;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adj_b(const AdjParams<T> &p, cudaStream_t st) {
  const dim3 b(32, 8, 1), g((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz + 1);
  adj_b_kernel<T><<<g, b, 0, st>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adj_init(const AdjParams<T> &p, cudaStream_t st) {
  const dim3 b(32, 8, 1), g((p.nx + 31) / 32, (p.ny + 7) / 8, p.nz + 1);
  adj_init_kernel<T><<<g, b, 0, st>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_objective_term(const T *const E[3], const T *const B[3], int nx, int ny, long long plane, int kind,
                                  const int box0[6], double f, double *out, cudaStream_t st) {
  objective_term_kernel<T><<<1, 256, 0, st>>>(E[0], E[1], E[2], B[0], B[1], nx, ny, plane, kind, box0[0], box0[1],
                                              box0[2], box0[3], box0[4], box0[5], f, out);
  return cudaGetLastError();
}

cudaError_t launch_sum_terms(const double *terms, long long n, double *out, cudaStream_t st) {
  sum_terms_kernel<<<1, 256, 0, st>>>(terms, n, out);
  return cudaGetLastError();
}

template cudaError_t launch_adj_e<float>(const AdjParams<float> &, cudaStream_t);
template cudaError_t launch_adj_e<double>(const AdjParams<double> &, cudaStream_t);
template cudaError_t launch_adj_b<float>(const AdjParams<float> &, cudaStream_t);
template cudaError_t launch_adj_b<double>(const AdjParams<double> &, cudaStream_t);
template cudaError_t launch_adj_init<float>(const AdjParams<float> &, cudaStream_t);
template cudaError_t launch_adj_init<double>(const AdjParams<double> &, cudaStream_t);
template cudaError_t launch_objective_term<float>(const float *const[3], const float *const[3], int, int, long long,
                                                  int, const int[6], double, double *, cudaStream_t);
template cudaError_t launch_objective_term<double>(const double *const[3], const double *const[3], int, int,
                                                   long long, int, const int[6], double, double *, cudaStream_t);

}  // namespace mpb
