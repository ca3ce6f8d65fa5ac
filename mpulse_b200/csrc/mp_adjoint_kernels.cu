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
//     objective's B term and advances its H-face totals;
//   the design gradients of the step (design cells only), accumulated from
//     G, E before and after the step and the PLRC accumulator adjoints adj_e
//     saved for the design cells, by extra blocks of the adj_b launch, so
//     that adj_e, which every cell runs, carries none of the FP64 gradient
//     arithmetic.
// The kernels of the reverse pass are launched with programmatic dependent
// launch: a kernel's blocks may start while the previous kernel's last blocks
// run, do their set-up, and wait (griddepcontrol.wait) for the previous
// kernel's writes before reading anything it produced.
// The Kerr linearisation and the gradient accumulation are FP64; the rest is
// in the precision of the forward state.  Latency-bound at small grids; one
// thread per (x, y) column and chunk of planes.
#include "mp_checked.cuh"
#include "mp_device.h"

#include <cuda_runtime.h>

// Blocks of 32 x MPB_ADJ_BLOCK_Y columns; resident threads per SM asked of
// the register allocator, per precision.
#ifndef MPB_ADJ_BLOCK_Y
#define MPB_ADJ_BLOCK_Y 4
#endif
#ifndef MPB_ADJ_E_MIN_F
#define MPB_ADJ_E_MIN_F 640
#endif
#ifndef MPB_ADJ_E_MIN_D
#define MPB_ADJ_E_MIN_D 512
#endif
#ifndef MPB_ADJ_B_MIN_F
#define MPB_ADJ_B_MIN_F 768
#endif
#ifndef MPB_ADJ_B_MIN_D
#define MPB_ADJ_B_MIN_D 512
#endif
#define MPB_ADJ_THREADS (32 * MPB_ADJ_BLOCK_Y)

namespace mpb {

namespace {

// Position of axis index idx in a face entry (-1: outside its layers).
template <typename T>
__device__ __forceinline__ int face_pos(const AdjFace<T> &F, int idx) {
  if (!F.active) return -1;
  if (idx >= F.lo0 && idx <= F.hi0) return idx - F.lo0;
  if (idx >= F.lo1 && idx <= F.hi1) return F.n0 + idx - F.lo1;
  return -1;
}

// Element of the x (D = 0) or y (D = 1) entry at axis position pos, column
// (i, j) and plane k: face_col(..) + face_plane(.., k).  32-bit: the host
// keeps every face array below 2^31 elements.
template <int D, typename T>
__device__ __forceinline__ int face_col(const AdjFace<T> &F, int pos, int i, int j, int nx) {
  return pos < 0 ? 0 : (D == 0 ? j * F.ex + pos : pos * nx + i);
}
template <int D, typename T>
__device__ __forceinline__ int face_plane(const AdjFace<T> &F, int k, int nx, int ny) {
  return D == 0 ? (k - F.zlo) * ny * F.ex : (k - F.zlo) * F.ey * nx;
}

// The components fed by psi0 / psi1 of a face along D (cpml_border.cpp:357-386):
// x faces (y, z), y faces (z, x), z faces (x, y).
template <int D, typename R>
__device__ __forceinline__ R comp0(const R v[3]) {
  return D == 0 ? v[1] : (D == 1 ? v[2] : v[0]);
}
template <int D, typename R>
__device__ __forceinline__ R comp1(const R v[3]) {
  return D == 0 ? v[2] : (D == 1 ? v[0] : v[1]);
}

// c * total at element li of an entry, or zero for pos < 0
template <typename T, typename R>
__device__ __forceinline__ void face_w(const AdjFace<T> &F, int pos, int li, R c, R &w0, R &w1, int *st) {
  if (pos >= 0) {
    w0 = c * R(ld_c(F.a0, li, F.n, st));
    w1 = c * R(ld_c(F.a1, li, F.n, st));
  } else {
    w0 = w1 = R(0);
  }
}

// Programmatic dependent launch: let the next kernel of the stream start its
// blocks, and wait until the previous kernel's writes are visible.  Both are
// no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace

// Arithmetic is in T (the precision of the state); the Kerr linearisation and
// the design gradients are FP64.  One thread per (x, y) column marches up a
// chunk of planes, carrying the z-neighbours in registers.  Arrays a kernel
// only reads (the B adjoint in adj_e, G in adj_b, the E history) go through
// the read-only data path (ldg_c).  NL: the Kerr medium (PLRC nonlinear); the
// linear form leaves out the Kerr linearisation, whose terms are zero there.
template <typename T, int NP, bool NL>
__global__ void __launch_bounds__(MPB_ADJ_THREADS, (sizeof(T) == 4 ? MPB_ADJ_E_MIN_F : MPB_ADJ_E_MIN_D) / MPB_ADJ_THREADS)
    adj_e_kernel(const AdjParams<T> p) {
  typedef T R;
  pdl_launch_dependents();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= p.nx || j >= p.ny) return;
  const int k0 = 1 + blockIdx.z * p.kchunk_e;
  const int k1 = min(k0 + p.kchunk_e - 1, p.nz);
  if (k0 > k1) return;
  const int nx = p.nx, ny = p.ny;
  const int im = i == 0 ? nx - 1 : i - 1;
  const int jm = j == 0 ? ny - 1 : j - 1;
  const long long pl = p.plane;
  const int col = j * nx + i, colxm = j * nx + im, colym = jm * nx + i;
  const R dt = R(p.dt);
  const long long nf = p.n_field;
  int *const st = p.status;
  const R kxi = p.ikH[0][i + 1], kxm = p.ikH[0][im + 1];
  const R kyj = p.ikH[1][j + 1], kym = p.ikH[1][jm + 1];
  const R bzj = p.ikH_bzy[j + 1], bzm = p.ikH_bzy[jm + 1];
  const T *Bx = p.Bb[0], *By = p.Bb[1], *Bz = p.Bb[2];
  const AdjFace<T> &HX = p.fh[0], &HY = p.fh[1], &HZ = p.fh[2];
  const AdjFace<T> &EX = p.fe[0], &EY = p.fe[1], &EZ = p.fe[2];
  const int plane = int(pl);
  // warps whose columns lie in no x / y face skip the face code on planes
  // outside the z faces; the face positions are recomputed where used
  const bool warp_xy = __any_sync(__activemask(), (face_pos(HX, i + 1) >= 0) || (face_pos(HX, im + 1) >= 0) ||
                                                      (face_pos(HY, j + 1) >= 0) || (face_pos(HY, jm + 1) >= 0) ||
                                                      (face_pos(EX, i + 1) >= 0) || (face_pos(EY, j + 1) >= 0));
  // everything below reads what the previous reverse kernel wrote
  pdl_wait();
  // the z H face's c * total at plane k - 1, carried
  R cw0, cw1;
  bool cw_on;
  {
    const int pz = face_pos(HZ, k0 - 1);
    cw_on = pz >= 0;
    face_w(HZ, pz, pz * plane + col, pz >= 0 ? R(HZ.c[k0 - 1]) : R(0), cw0, cw1, st);
  }
  const DesignParams &d = p.design;
  const bool dxy = i >= d.x0 && i <= d.x1 && j >= d.y0 && j <= d.y1;
  const bool oxy = i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1;
  R bx_km = ldg_c(Bx, (long long)(k0 - 1) * pl + col, nf, st);
  R by_km = ldg_c(By, (long long)(k0 - 1) * pl + col, nf, st);

  const bool plrc_nl = NL;
  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * pl;
    const long long c0 = base + col;
    const bool med = k >= p.mz0 && k <= p.mz1;
    const bool dcell = med && dxy && k >= d.z0 && k <= d.z1;
    // ---- every load of this plane first, so that their latencies overlap
    const R bx = ldg_c(Bx, c0, nf, st), by = ldg_c(By, c0, nf, st), bz = ldg_c(Bz, c0, nf, st);
    const R bx_ym = ldg_c(Bx, base + colym, nf, st), by_xm = ldg_c(By, base + colxm, nf, st),
            bz_ym = ldg_c(Bz, base + colym, nf, st), bz_xm = ldg_c(Bz, base + colxm, nf, st);
    const R kzk = p.ikH[2][k], kzm = p.ikH[2][k - 1];
    R a[3] = {R(ld_c(p.Eb[0], c0, nf, st)), R(ld_c(p.Eb[1], c0, nf, st)), R(ld_c(p.Eb[2], c0, nf, st))};
    // E^n enters here only through the Kerr term (its coefficient is zero in
    // a linear medium) and the |E|^2 objective's box: elsewhere it is not read
    R En[3] = {R(0), R(0), R(0)};
    if (plrc_nl || (p.add_obj && oxy && p.obj_kind == 1 && k >= p.oz0 && k <= p.oz1)) {
#pragma unroll
      for (int c = 0; c < 3; ++c) En[c] = R(ldg_c(p.En[c], c0, nf, st));
    }
    R En1[3] = {R(0), R(0), R(0)};
    if (med && (plrc_nl || dcell)) {
#pragma unroll
      for (int c = 0; c < 3; ++c) En1[c] = R(ldg_c(p.En1[c], c0, nf, st));
    }
    const long long pi = ((long long)(k - p.mz0) * ny + j) * nx + i;
    R pq[NP > 0 ? NP : 1][3][2];
    if (med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          pq[n][c][0] = ld_c(p.psib[n][c], 2 * pi, 2 * p.n_psi, st);
          pq[n][c][1] = ld_c(p.psib[n][c], 2 * pi + 1, 2 * p.n_psi, st);
        }
    }
    long long di = 0;
    double e = p.eps, s = 1.0, u = 1.0;
    if (dcell) {
      di = ((long long)(k - d.z0) * d.by + (j - d.y0)) * d.bx + (i - d.x0);
      e = ld_c(d.eps, di, p.n_design, st);
      s = ld_c(d.dscale, di, p.n_design, st);
      u = ld_c(d.chiscale, di, p.n_design, st);
    }
    // H-face totals (x, y at this column and x-1 / y-1; z at this plane) and
    // E-face totals of this cell, on warps and planes that touch a face
    const int hzp = face_pos(HZ, k), ezp = face_pos(EZ, k);
    const bool fpl = warp_xy || cw_on || hzp >= 0 || ezp >= 0;
    R hx0o = R(0), hx1o = R(0), hx0m = R(0), hx1m = R(0), hy0o = R(0), hy1o = R(0), hy0m = R(0), hy1m = R(0);
    R hz0 = R(0), hz1 = R(0);
    R ex0 = R(0), ex1 = R(0), ey0 = R(0), ey1 = R(0), ez0 = R(0), ez1 = R(0), ezb = R(0);
    int lexo = 0, leyo = 0, lezo = 0;
    if (fpl) {
      const int hxo = face_pos(HX, i + 1), hxm = face_pos(HX, im + 1);
      const int hyo = face_pos(HY, j + 1), hym = face_pos(HY, jm + 1);
      const R hxco = hxo >= 0 ? R(HX.c[i + 1]) : R(0), hxcm = hxm >= 0 ? R(HX.c[im + 1]) : R(0);
      const R hyco = hyo >= 0 ? R(HY.c[j + 1]) : R(0), hycm = hym >= 0 ? R(HY.c[jm + 1]) : R(0);
      const int exo = face_pos(EX, i + 1), eyo = face_pos(EY, j + 1);
      const int chxo = face_col<0>(HX, hxo, i, j, nx), chxm = face_col<0>(HX, hxm, im, j, nx);
      const int chyo = face_col<1>(HY, hyo, i, j, nx), chym = face_col<1>(HY, hym, i, jm, nx);
      const int cexo = face_col<0>(EX, exo, i, j, nx), ceyo = face_col<1>(EY, eyo, i, j, nx);
      const int shx = face_plane<0>(HX, k, nx, ny), shy = face_plane<1>(HY, k, nx, ny);
      face_w(HX, hxo, chxo + shx, hxco, hx0o, hx1o, st);
      face_w(HX, hxm, chxm + shx, hxcm, hx0m, hx1m, st);
      face_w(HY, hyo, chyo + shy, hyco, hy0o, hy1o, st);
      face_w(HY, hym, chym + shy, hycm, hy0m, hy1m, st);
      face_w(HZ, hzp, hzp * plane + col, hzp >= 0 ? R(HZ.c[k]) : R(0), hz0, hz1, st);
      lexo = exo >= 0 ? cexo + face_plane<0>(EX, k, nx, ny) : -1;
      leyo = eyo >= 0 ? ceyo + face_plane<1>(EY, k, nx, ny) : -1;
      lezo = ezp * plane + col;
      if (lexo >= 0) { ex0 = ld_c(EX.a0, lexo, EX.n, st); ex1 = ld_c(EX.a1, lexo, EX.n, st); }
      if (leyo >= 0) { ey0 = ld_c(EY.a0, leyo, EY.n, st); ey1 = ld_c(EY.a1, leyo, EY.n, st); }
      if (ezp >= 0) { ez0 = ld_c(EZ.a0, lezo, EZ.n, st); ez1 = ld_c(EZ.a1, lezo, EZ.n, st); ezb = EZ.b[k]; }
    }
    R obx = R(0), oby = R(0);
    if (p.add_obj && oxy && p.obj_kind == 2 && k == p.oz0) {
      obx = ld_c(p.obx, col, pl, st);
      oby = ld_c(p.oby, col, pl, st);
    }

    // ---- adjoint of E' (B half transposed)
    // Bx' = .. + dt ((ey(k+1) - ey) ikz - (ez(j+1) - ez) iky)
    a[1] += dt * (kzm * bx_km - kzk * bx);
    a[2] += dt * (-kym * bx_ym + kyj * bx);
    // By' = .. + dt ((ez(i+1) - ez) ikx - (ex(k+1) - ex) ikz)
    a[2] += dt * (kxm * by_xm - kxi * by);
    a[0] += dt * (-kzm * by_km + kzk * by);
    // Bz' = .. + dt ((ex(j+1) - ex) iky_bz - (ey(i+1) - ey) ikx)
    a[0] += dt * (bzm * bz_ym - bzj * bz);
    a[1] += dt * (-kxm * bz_xm + kxi * bz);
    // H faces: psi0 / psi1 feed (y, z) on x faces, (z, x) on y faces, (x, y) on
    // z faces; their differences of E run forward along the axis
    if (fpl) {
      a[2] += hx0m - hx0o;
      a[1] += hx1o - hx1m;
      a[0] += hy0m - hy0o;
      a[2] += hy1o - hy1m;
      a[1] += cw0 - hz0;
      a[0] += hz1 - cw1;
    }
    cw0 = hz0;
    cw1 = hz1;
    cw_on = hzp >= 0;

    // ---- E half, locally
    R g[3], ne[3];
    if (!med) {
      // background: E' = (eps_bg E + dt (curl + J)) / eps_bg
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        g[c] = a[c] * p.inv_eps_bg_t;
        ne[c] = p.eps_bg_t * g[c];
      }
    } else {
      double A = NL ? p.A0 : 0.0;
      R idn = p.inv_denom0_t, numer = p.numer0_t, Rchi = NL ? p.chi_nl_t : R(0);
      if (dcell) {
        const double denom = d.lin ? e + s * (p.sumChi0 - p.sumXi0) : e + s * p.sumChi0 - s * p.sumXi0;
        A = NL ? u * p.chi / denom : 0.0;
        idn = R(1.0 / denom);
        numer = R(e - s * p.sumXi0);
        Rchi = NL ? R(u * p.chi) : R(0);
      }
      R cb[3] = {a[0], a[1], a[2]};
      if (NL) {
        // E' = r c/|c| with r + A r^3 = |c|: dE'/dc = (I - e e^T) / (1 + A r^2)
        // + e e^T / (1 + 3 A r^2), dr/dA = -r^3 / (1 + 3 A r^2), c = E' (1 + A r^2)
        const double r2 = (double)En1[0] * En1[0] + (double)En1[1] * En1[1] + (double)En1[2] * En1[2];
        const double r = sqrt(r2);
        const double al = 1.0 / (1.0 + A * r2), be = 1.0 / (1.0 + 3.0 * A * r2);
        const double ir = r > 0 ? 1.0 / r : 0.0;
        double eh[3], ea = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          eh[c] = En1[c] * ir;
          ea += eh[c] * a[c];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) cb[c] = R(al * (a[c] - eh[c] * ea) + be * eh[c] * ea);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) g[c] = cb[c] * idn;
      if (NL) {
        const R E2 = En[0] * En[0] + En[1] * En[1] + En[2] * En[2];
        const R Eg = En[0] * g[0] + En[1] * g[1] + En[2] * g[2];
        const R f = numer + Rchi * E2;
#pragma unroll
        for (int c = 0; c < 3; ++c) ne[c] = f * g[c] + R(2) * Rchi * En[c] * Eg;
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) ne[c] = numer * g[c];
      }
      // the design cells' accumulator adjoints before the reverse recursion,
      // for adj_grad
      if (dcell) {
#pragma unroll
        for (int n = 0; n < NP; ++n)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const long long q = ((di * NP + n) * 3 + c) * 2;
            st_c(p.dpsi, q, p.n_design * NP * 6, st, T(pq[n][c][0]));
            st_c(p.dpsi, q + 1, p.n_design * NP * 6, st, T(pq[n][c][1]));
          }
      }
      // reverse PLRC recursion: psi~bar = conj(Crec) psibar + g
      const R Rs = dcell ? R(s) : R(1);
#pragma unroll
      for (int n = 0; n < NP; ++n) {
        const R Dr = p.pDt[n][0], Di = p.pDt[n][1];
        const R Xr = p.pxit[n][0], Xi = p.pxit[n][1];
        const R Cr = p.pCt[n][0], Ci = p.pCt[n][1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const R pr = pq[n][c][0], pim = pq[n][c][1];
          const R tr = Cr * pr + Ci * pim + g[c];
          const R ti = Cr * pim - Ci * pr;
          ne[c] += Rs * (Dr * tr + Di * ti + Xr * pr + Xi * pim);
          pq[n][c][0] = tr;
          pq[n][c][1] = ti;
        }
      }
    }
    // the objective's E term of the state before the step
    if (p.add_obj && oxy) {
      if (p.obj_kind == 1) {
        if (k >= p.oz0 && k <= p.oz1) {
#pragma unroll
          for (int c = 0; c < 3; ++c) ne[c] += p.obj_f_t * En[c];
        }
      } else if (k == p.oz0) {
        ne[0] += p.obj_f_t * oby;
        ne[1] -= p.obj_f_t * obx;
      }
    }

    // ---- stores
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      st_c(p.G[c], c0, nf, st, T(g[c]));
      st_c(p.Eb[c], c0, nf, st, T(ne[c]));
    }
    if (med) {
#pragma unroll
      for (int n = 0; n < NP; ++n)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          st_c(p.psib[n][c], 2 * pi, 2 * p.n_psi, st, T(pq[n][c][0]));
          st_c(p.psib[n][c], 2 * pi + 1, 2 * p.n_psi, st, T(pq[n][c][1]));
        }
    }
    // E-face totals of this cell: b * total + dt * G
    if (fpl) {
      if (lexo >= 0) {
        const R exb = R(EX.b[i + 1]);
        st_c(EX.a0, lexo, EX.n, st, T(exb * ex0 + dt * comp0<0>(g)));
        st_c(EX.a1, lexo, EX.n, st, T(exb * ex1 + dt * comp1<0>(g)));
      }
      if (leyo >= 0) {
        const R eyb = R(EY.b[j + 1]);
        st_c(EY.a0, leyo, EY.n, st, T(eyb * ey0 + dt * comp0<1>(g)));
        st_c(EY.a1, leyo, EY.n, st, T(eyb * ey1 + dt * comp1<1>(g)));
      }
      if (ezp >= 0) {
        st_c(EZ.a0, lezo, EZ.n, st, T(ezb * ez0 + dt * comp0<2>(g)));
        st_c(EZ.a1, lezo, EZ.n, st, T(ezb * ez1 + dt * comp1<2>(g)));
      }
    }
    bx_km = bx;
    by_km = by;
  }
}

// The design gradients of one step, one thread per design cell (the design
// box lies inside the medium planes and the interior).  From the E half
// X = (numer + chi |E|^2) E + dt (curl + J) + Re sum psi~ with numer = e - s
// sumXi0, denom = e + s (sumChi0 - sumXi0), psi~ = s (dchi0 - dxi0) E + psi,
// psi' = s dxi0 E + Crec psi~ and (nonlinear) A = u chi / denom, with g the
// adjoint of X / denom that adj_e stored in G:
//   dJ/de += g . (E - c) - Abar A / denom
//   dJ/ds += sum_n,c psibar_nc . (dxi0 + Crec (dchi0 - dxi0)) E_c
//            + g . ((sum_n Re(dchi0 - dxi0) - sumXi0) E - c dD) - Abar A dD / denom
//   dJ/du += g . chi |E|^2 E + Abar chi / denom
// where c = E' (1 + A |E'|^2) is X / denom, dD = sumChi0 - sumXi0 and Abar,
// the adjoint of A through the Kerr solve, is -(e^ . c_bar) r^3 with r = |E'|,
// e^ = E' / r and c_bar = g denom the adjoint of c (the Kerr linearisation of
// adj_e gives e^ . c_bar = be (e^ . a) with be = 1 / (1 + 3 A r^2)).
template <typename T, int NP, bool NL>
__device__ __forceinline__ void adj_grad_cells(const AdjParams<T> &p, int gbx, int gby, int kk) {
  const DesignParams &d = p.design;
  const int ii = gbx * blockDim.x + threadIdx.x, jj = gby * blockDim.y + threadIdx.y;
  if (ii >= d.bx || jj >= d.by) return;
  pdl_wait();
  const int i = d.x0 + ii, j = d.y0 + jj, k = d.z0 + kk;
  const long long nf = p.n_field;
  int *const st = p.status;
  const long long di = ((long long)kk * d.by + jj) * d.bx + ii;
  const long long c0 = (long long)k * p.plane + (long long)j * p.nx + i;
  const double e = ld_c(d.eps, di, p.n_design, st), s = ld_c(d.dscale, di, p.n_design, st),
               u = ld_c(d.chiscale, di, p.n_design, st);
  T g[3], En[3], En1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    g[c] = ld_c(p.G[c], c0, nf, st);
    En[c] = ldg_c(p.En[c], c0, nf, st);
    En1[c] = ldg_c(p.En1[c], c0, nf, st);
  }
  const double dD = p.sumChi0 - p.sumXi0;
  const double denom = d.lin ? e + s * dD : e + s * p.sumChi0 - s * p.sumXi0;
  const double A = NL ? u * p.chi / denom : 0.0;
  const double r2 = NL ? (double)En1[0] * En1[0] + (double)En1[1] * En1[1] + (double)En1[2] * En1[2] : 0.0;
  double Abar = 0.0;
  if (NL && r2 > 0) {
    const double r = sqrt(r2);
    double ecb = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) ecb += (double)En1[c] / r * ((double)g[c] * denom);
    Abar = -ecb * r * r2;
  }
  double gs = 0.0, SD = 0.0;
#pragma unroll
  for (int n = 0; n < NP; ++n) {
    SD += p.pD[n][0];
    const double CDr = p.pC[n][0] * p.pD[n][0] - p.pC[n][1] * p.pD[n][1];
    const double CDi = p.pC[n][0] * p.pD[n][1] + p.pC[n][1] * p.pD[n][0];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long q = ((di * NP + n) * 3 + c) * 2;
      const double pr = ld_c(p.dpsi, q, p.n_design * NP * 6, st), pim = ld_c(p.dpsi, q + 1, p.n_design * NP * 6, st);
      gs += (pr * (p.pxi[n][0] + CDr) + pim * (p.pxi[n][1] + CDi)) * (double)En[c];
    }
  }
  double ge = NL ? -Abar * A / denom : 0.0, gu = 0.0;
  if (NL) gs -= Abar * A * dD / denom;
  const double grow = NL ? 1.0 + A * r2 : 1.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double cv = (double)En1[c] * grow;
    ge += (double)g[c] * ((double)En[c] - cv);
    gs += (double)g[c] * ((SD - p.sumXi0) * (double)En[c] - cv * dD);
  }
  if (NL) {
    const T E2 = En[0] * En[0] + En[1] * En[1] + En[2] * En[2];
    gu = Abar * p.chi / denom;
#pragma unroll
    for (int c = 0; c < 3; ++c) gu += (double)g[c] * p.chi * (double)E2 * (double)En[c];
  }
  st_c(p.grad[0], di, p.n_design, st, ld_c(p.grad[0], di, p.n_design, st) + ge);
  st_c(p.grad[1], di, p.n_design, st, ld_c(p.grad[1], di, p.n_design, st) + gs);
  st_c(p.grad[2], di, p.n_design, st, ld_c(p.grad[2], di, p.n_design, st) + gu);
}

template <typename T>
__device__ __forceinline__ void adj_b_cells(const AdjParams<T> &p, int bxi, int byi, int bzi) {
  typedef T R;
  const int i = bxi * blockDim.x + threadIdx.x;
  const int j = byi * blockDim.y + threadIdx.y;
  if (i >= p.nx || j >= p.ny) return;
  const int k0 = bzi * p.kchunk_b;
  const int k1 = min(k0 + p.kchunk_b - 1, p.nz);
  if (k0 > k1) return;
  const int nx = p.nx, ny = p.ny;
  const int ip = i == nx - 1 ? 0 : i + 1;
  const int jp = j == ny - 1 ? 0 : j + 1;
  const long long pl = p.plane;
  const int col = j * nx + i, colxp = j * nx + ip, colyp = jp * nx + i;
  const R dt = R(p.dt);
  const long long nf = p.n_field;
  int *const st = p.status;
  const R kxi = p.ikE[0][i + 1], kxp = p.ikE[0][ip + 1];
  const R kyj = p.ikE[1][j + 1], kyp = p.ikE[1][jp + 1];
  const T *gx = p.G[0], *gy = p.G[1], *gz = p.G[2];
  const AdjFace<T> &HX = p.fh[0], &HY = p.fh[1], &HZ = p.fh[2];
  const AdjFace<T> &EX = p.fe[0], &EY = p.fe[1], &EZ = p.fe[2];
  // E faces at this column and at x+1 / y+1; H faces at this column
  const int exo = face_pos(EX, i + 1), exp_ = face_pos(EX, ip + 1);
  const int eyo = face_pos(EY, j + 1), eyp = face_pos(EY, jp + 1);
  const R exco = exo >= 0 ? R(EX.c[i + 1]) : R(0), excp = exp_ >= 0 ? R(EX.c[ip + 1]) : R(0);
  const R eyco = eyo >= 0 ? R(EY.c[j + 1]) : R(0), eycp = eyp >= 0 ? R(EY.c[jp + 1]) : R(0);
  const int hxo = face_pos(HX, i + 1), hyo = face_pos(HY, j + 1);
  const R hxb = hxo >= 0 ? R(HX.b[i + 1]) : R(0), hyb = hyo >= 0 ? R(HY.b[j + 1]) : R(0);
  const bool oxy = p.add_obj && p.obj_kind == 2 && i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1;
  const int plane = int(pl);
  const int cexo = face_col<0>(EX, exo, i, j, nx), cexp = face_col<0>(EX, exp_, ip, j, nx);
  const int ceyo = face_col<1>(EY, eyo, i, j, nx), ceyp = face_col<1>(EY, eyp, i, jp, nx);
  const int chxo = face_col<0>(HX, hxo, i, j, nx), chyo = face_col<1>(HY, hyo, i, j, nx);
  // warps whose columns lie in no x / y face skip the face code on planes
  // outside the z faces
  const bool warp_xy =
      __any_sync(__activemask(), (exo >= 0) || (exp_ >= 0) || (eyo >= 0) || (eyp >= 0) || (hxo >= 0) || (hyo >= 0));
  // everything below reads what adj_e wrote
  pdl_wait();
  // G and the z E face's c * total at plane k, carried from the previous plane's k + 1
  R gx_k = ldg_c(gx, (long long)k0 * pl + col, nf, st), gy_k = ldg_c(gy, (long long)k0 * pl + col, nf, st);
  R zw0, zw1;
  bool zw_on;
  {
    const int pz = face_pos(EZ, k0);
    zw_on = pz >= 0;
    face_w(EZ, pz, pz * plane + col, pz >= 0 ? R(EZ.c[k0]) : R(0), zw0, zw1, st);
  }

  for (int k = k0; k <= k1; ++k) {
    const long long base = (long long)k * pl;
    const long long c0 = base + col;
    // ---- every load of this plane first
    const R gx_kp = ldg_c(gx, c0 + pl, nf, st), gy_kp = ldg_c(gy, c0 + pl, nf, st);
    const R gzk = ldg_c(gz, c0, nf, st);
    const R gx_yp = ldg_c(gx, base + colyp, nf, st), gy_xp = ldg_c(gy, base + colxp, nf, st),
            gz_xp = ldg_c(gz, base + colxp, nf, st), gz_yp = ldg_c(gz, base + colyp, nf, st);
    const R kzk = p.ikE[2][k], kzp = p.ikE[2][k + 1];
    R b[3] = {R(ld_c(p.Bb[0], c0, nf, st)), R(ld_c(p.Bb[1], c0, nf, st)), R(ld_c(p.Bb[2], c0, nf, st))};
    // faces on warps and planes that touch one: E faces (x / y hold planes
    // 1..nz; z at plane k + 1, plane k carried) and the H-face totals of this cell
    const int ezq = face_pos(EZ, k + 1), hzp = face_pos(HZ, k);
    const bool fpl = warp_xy || zw_on || ezq >= 0 || hzp >= 0;
    R ex0o = R(0), ex1o = R(0), ex0p = R(0), ex1p = R(0), ey0o = R(0), ey1o = R(0), ey0p = R(0), ey1p = R(0);
    R ez0p = R(0), ez1p = R(0);
    const bool hxk = hxo >= 0 && k >= HX.zlo, hyk = hyo >= 0 && k >= HY.zlo;
    int lhx = 0, lhy = 0, lhz = 0;
    R hx0 = R(0), hx1 = R(0), hy0 = R(0), hy1 = R(0), hz0 = R(0), hz1 = R(0), hzb = R(0);
    if (fpl) {
      if (k >= 1) {
        const int sex = face_plane<0>(EX, k, nx, ny), sey = face_plane<1>(EY, k, nx, ny);
        face_w(EX, exo, cexo + sex, exco, ex0o, ex1o, st);
        face_w(EX, exp_, cexp + sex, excp, ex0p, ex1p, st);
        face_w(EY, eyo, ceyo + sey, eyco, ey0o, ey1o, st);
        face_w(EY, eyp, ceyp + sey, eycp, ey0p, ey1p, st);
      }
      face_w(EZ, ezq, ezq * plane + col, ezq >= 0 ? R(EZ.c[k + 1]) : R(0), ez0p, ez1p, st);
      lhx = chxo + face_plane<0>(HX, k, nx, ny);
      lhy = chyo + face_plane<1>(HY, k, nx, ny);
      lhz = hzp * plane + col;
      if (hxk) { hx0 = ld_c(HX.a0, lhx, HX.n, st); hx1 = ld_c(HX.a1, lhx, HX.n, st); }
      if (hyk) { hy0 = ld_c(HY.a0, lhy, HY.n, st); hy1 = ld_c(HY.a1, lhy, HY.n, st); }
      if (hzp >= 0) { hz0 = ld_c(HZ.a0, lhz, HZ.n, st); hz1 = ld_c(HZ.a1, lhz, HZ.n, st); hzb = HZ.b[k]; }
    }
    const bool obj = oxy && k == p.oz0;
    R oex = R(0), oey = R(0);
    if (obj) {
      oex = ldg_c(p.En[0], c0, nf, st);
      oey = ldg_c(p.En[1], c0, nf, st);
    }

    // ---- transposed curl_E and E faces
    // cbx = (bz - bz(j-1)) iky - (by - by(k-1)) ikz
    b[2] += dt * (kyj * gx_k - kyp * gx_yp);
    b[1] += dt * (-kzk * gx_k + kzp * gx_kp);
    // cby = (bx - bx(k-1)) ikz - (bz - bz(i-1)) ikx
    b[0] += dt * (kzk * gy_k - kzp * gy_kp);
    b[2] += dt * (-kxi * gy_k + kxp * gy_xp);
    // cbz = (by - by(i-1)) ikx - (bx - bx(j-1)) iky
    b[1] += dt * (kxi * gzk - kxp * gz_xp);
    b[0] += dt * (-kyj * gzk + kyp * gz_yp);
    // E faces: psi0 / psi1 feed (y, z) on x faces, (z, x) on y faces, (x, y) on
    // z faces; their differences of B run backward along the axis
    if (fpl) {
      b[2] += -ex0o + ex0p;
      b[1] += ex1o - ex1p;
      b[0] += -ey0o + ey0p;
      b[2] += ey1o - ey1p;
      b[1] += -zw0 + ez0p;
      b[0] += zw1 - ez1p;
    }
    zw0 = ez0p;
    zw1 = ez1p;
    zw_on = ezq >= 0;
    // the objective's B term of the state before the step (Sz plane)
    if (obj) {
      b[0] -= p.obj_f_t * oey;
      b[1] += p.obj_f_t * oex;
    }

    // ---- stores: B adjoint, H-face totals for the step before (b * total + dt * B adjoint)
#pragma unroll
    for (int c = 0; c < 3; ++c) st_c(p.Bb[c], c0, nf, st, T(b[c]));
    if (fpl) {
      if (hxk) {
        st_c(HX.a0, lhx, HX.n, st, T(hxb * hx0 + dt * comp0<0>(b)));
        st_c(HX.a1, lhx, HX.n, st, T(hxb * hx1 + dt * comp1<0>(b)));
      }
      if (hyk) {
        st_c(HY.a0, lhy, HY.n, st, T(hyb * hy0 + dt * comp0<1>(b)));
        st_c(HY.a1, lhy, HY.n, st, T(hyb * hy1 + dt * comp1<1>(b)));
      }
      if (hzp >= 0) {
        st_c(HZ.a0, lhz, HZ.n, st, T(hzb * hz0 + dt * comp0<2>(b)));
        st_c(HZ.a1, lhz, HZ.n, st, T(hzb * hz1 + dt * comp1<2>(b)));
      }
    }
    gx_k = gx_kp;
    gy_k = gy_kp;
  }
}

// The B half of the reverse step (blocks 0 .. nb-1 of a one-dimensional grid,
// x fastest over gx x gy x z-chunks) and the design gradients of the step
// (the blocks after them, over the design box in 32 x 4 tiles, one plane
// each).
template <typename T, int NP, bool NL>
__global__ void __launch_bounds__(MPB_ADJ_THREADS, (sizeof(T) == 4 ? MPB_ADJ_B_MIN_F : MPB_ADJ_B_MIN_D) / MPB_ADJ_THREADS)
    adj_b_kernel(const AdjParams<T> p, const int gx, const int gy, const int nb) {
  pdl_launch_dependents();
  const int b = blockIdx.x;
  if (b < nb) {
    adj_b_cells<T>(p, b % gx, (b / gx) % gy, b / (gx * gy));
  } else {
    const int q = b - nb;
    const int tx = (p.design.bx + 31) / 32, ty = (p.design.by + MPB_ADJ_BLOCK_Y - 1) / MPB_ADJ_BLOCK_Y;
    adj_grad_cells<T, NP, NL>(p, q % tx, (q / tx) % ty, q / (tx * ty));
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
  const long long nf = p.n_field;
  int *const st = p.status;
  double e[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
  const bool inxy = i >= p.ox0 && i <= p.ox1 && j >= p.oy0 && j <= p.oy1;
  if (p.obj_kind == 1) {
    if (inxy && k >= p.oz0 && k <= p.oz1)
      for (int c = 0; c < 3; ++c) e[c] = p.obj_f * (double)ld_c(p.En[c], c0, nf, st);
  } else if (inxy && k == p.oz0) {
    e[0] = p.obj_f * (double)ld_c(p.oby, col, p.plane, st);
    e[1] = -p.obj_f * (double)ld_c(p.obx, col, p.plane, st);
    b[0] = -p.obj_f * (double)ld_c(p.En[1], c0, nf, st);
    b[1] = p.obj_f * (double)ld_c(p.En[0], c0, nf, st);
  }
  for (int c = 0; c < 3; ++c) {
    st_c(p.Eb[c], c0, nf, st, T(e[c]));
    st_c(p.Bb[c], c0, nf, st, T(b[c]));
  }
  // H-face totals: dt times the adjoint of B
  const int hxo = face_pos(p.fh[0], i + 1), hyo = face_pos(p.fh[1], j + 1), hzo = face_pos(p.fh[2], k);
  if (hxo >= 0 && k >= p.fh[0].zlo) {
    const int li = face_col<0>(p.fh[0], hxo, i, j, p.nx) + face_plane<0>(p.fh[0], k, p.nx, p.ny);
    st_c(p.fh[0].a0, li, p.fh[0].n, st, T(p.dt * comp0<0>(b)));
    st_c(p.fh[0].a1, li, p.fh[0].n, st, T(p.dt * comp1<0>(b)));
  }
  if (hyo >= 0 && k >= p.fh[1].zlo) {
    const int li = face_col<1>(p.fh[1], hyo, i, j, p.nx) + face_plane<1>(p.fh[1], k, p.nx, p.ny);
    st_c(p.fh[1].a0, li, p.fh[1].n, st, T(p.dt * comp0<1>(b)));
    st_c(p.fh[1].a1, li, p.fh[1].n, st, T(p.dt * comp1<1>(b)));
  }
  if (hzo >= 0) {
    const long long li = (long long)hzo * p.plane + col;
    st_c(p.fh[2].a0, li, p.fh[2].n, st, T(p.dt * comp0<2>(b)));
    st_c(p.fh[2].a1, li, p.fh[2].n, st, T(p.dt * comp1<2>(b)));
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

// A launch with programmatic stream serialisation (the kernel's blocks may
// start before the previous kernel in the stream has finished; the kernel
// orders its reads with griddepcontrol.wait).
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 g, dim3 b, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename T>
cudaError_t launch_adj_e(const AdjParams<T> &p, cudaStream_t st) {
  const dim3 b(32, MPB_ADJ_BLOCK_Y, 1),
      g((p.nx + 31) / 32, (p.ny + MPB_ADJ_BLOCK_Y - 1) / MPB_ADJ_BLOCK_Y, (p.nz + p.kchunk_e - 1) / p.kchunk_e);
  const bool nl = p.nonlin != 0;
  switch (p.np) {
    case 0: return nl ? launch_pdl(adj_e_kernel<T, 0, true>, g, b, st, p) : launch_pdl(adj_e_kernel<T, 0, false>, g, b, st, p);
    case 1: return nl ? launch_pdl(adj_e_kernel<T, 1, true>, g, b, st, p) : launch_pdl(adj_e_kernel<T, 1, false>, g, b, st, p);
    case 2: return nl ? launch_pdl(adj_e_kernel<T, 2, true>, g, b, st, p) : launch_pdl(adj_e_kernel<T, 2, false>, g, b, st, p);
    default: return nl ? launch_pdl(adj_e_kernel<T, 3, true>, g, b, st, p) : launch_pdl(adj_e_kernel<T, 3, false>, g, b, st, p);
  }
}

// adj_b of the step, with the design gradients (when there is a design box) in
// extra blocks of the same launch.
template <typename T>
cudaError_t launch_adj_b(const AdjParams<T> &p, cudaStream_t st) {
  const int gx = (p.nx + 31) / 32, gy = (p.ny + MPB_ADJ_BLOCK_Y - 1) / MPB_ADJ_BLOCK_Y,
            gz = (p.nz + 1 + p.kchunk_b - 1) / p.kchunk_b;
  const int nb = gx * gy * gz;
  const DesignParams &d = p.design;
  const int ng = d.x0 <= d.x1 ? ((d.bx + 31) / 32) * ((d.by + MPB_ADJ_BLOCK_Y - 1) / MPB_ADJ_BLOCK_Y) * (d.z1 - d.z0 + 1)
                              : 0;
  const dim3 b(32, MPB_ADJ_BLOCK_Y, 1), g(nb + ng, 1, 1);
  const bool nl = p.nonlin != 0;
  switch (p.np) {
    case 0: return nl ? launch_pdl(adj_b_kernel<T, 0, true>, g, b, st, p, gx, gy, nb) : launch_pdl(adj_b_kernel<T, 0, false>, g, b, st, p, gx, gy, nb);
    case 1: return nl ? launch_pdl(adj_b_kernel<T, 1, true>, g, b, st, p, gx, gy, nb) : launch_pdl(adj_b_kernel<T, 1, false>, g, b, st, p, gx, gy, nb);
    case 2: return nl ? launch_pdl(adj_b_kernel<T, 2, true>, g, b, st, p, gx, gy, nb) : launch_pdl(adj_b_kernel<T, 2, false>, g, b, st, p, gx, gy, nb);
    default: return nl ? launch_pdl(adj_b_kernel<T, 3, true>, g, b, st, p, gx, gy, nb) : launch_pdl(adj_b_kernel<T, 3, false>, g, b, st, p, gx, gy, nb);
  }
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
