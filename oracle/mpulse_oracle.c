/*
 * mpulse_oracle.c - TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded, FP64 restatement of MPulse's time-stepping hot
 * path, used as the checker of the CUDA path (tests/, __graft_entry__.smoke and
 * bench.py's cpu_baseline leg).  Nothing in the product links or calls it.
 *
 * It keeps MPulse's own data layout and loop structure on purpose: grids span
 * the global index range [0, n+1] per axis with ghost cells
 * (src/globals.cpp:74-75), currents are summed into full-grid J/M totals
 * (src/fdtd_plrc.t:342-409), the boundary is an explicit ghost copy after each
 * half step (src/storage.cpp:194-204, src/periodic_bound.cpp:10-130), and the
 * CPML / TF-SF layers have the extents of Storage::getBorderExtent
 * (src/storage.cpp:208-318).  Each function cites the part of MPulse it
 * follows.  Arithmetic is written in the same order as the reference so that,
 * compiled with -ffp-contract=off, it reproduces the reference bit for bit
 * (except through the Faddeeva function, see oracle_faddeeva).
 *
 * The configuration is the mp_config of include/mpulse_b200.h, so one struct
 * drives both the oracle and the CUDA path.  Host buffers use the plane layout
 * of that header.
 */
#include "mpulse_b200.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { DIR_NORTH = 0, DIR_SOUTH, DIR_WEST, DIR_EAST, DIR_UP, DIR_DOWN }; /* mpulse.h:28 */

typedef struct {
  int lo[3], hi[3];
  int dims[3];
} box3;

static size_t box_size(const box3 *b) {
  return (size_t)b->dims[0] * b->dims[1] * b->dims[2];
}
static size_t box_index(const box3 *b, int i, int j, int k) {
  return ((size_t)(k - b->lo[2]) * b->dims[1] + (size_t)(j - b->lo[1])) * b->dims[0] +
         (size_t)(i - b->lo[0]);
}

/* One CPML current: CPMLBorderCurrent (cpml_border.cpp:262-339) with its two
 * psi components and 1-D b/c coefficient lines along `dim`. */
typedef struct {
  int dir, dim, isH;
  box3 box;
  double *psi[2];      /* psi0, psi1 as in cpml_border.cpp:361-383 / :460-482 */
  double *b, *c;       /* indexed by position - box.lo[dim] */
  double delta;        /* grid spacing along dim */
} cpml_layer;

/* One TF/SF current (IncidentSourceCurrent, incsource.cpp:93-136). */
typedef struct {
  int src, dir, dim, t1, t2, isH;
  box3 box;
  double DX;
  int off[3];
} inc_layer;

/* One GaussInjectSourceFunc (gaussinject.cpp:56-482): an angular-spectrum
 * Gaussian beam whose injection-plane fields are precomputed for blocks of Nt
 * steps by transforms over t, y and x.  isH = 0 holds Bx (for the E current's
 * getHField), isH = 1 holds Ex in F1 and Ey in F2 (for the H current). */
typedef struct {
  int isH;
  int SizeT, SizeX, SizeY, SizeTH, SizeXH, SizeYH, Nt, toff, blockCount, blockToff, active;
  long long computed; /* block held in F1/F2, -1 for none */
  double length, width, k0, Shift, Time, Time0, amp, eps, lightspeed, DX, DY, DT, BoxX, BoxY, BoxT;
  double sx, sy, sz;
  double *F1, *F2; /* [SizeX][SizeY][Nt] */
} gauss_state;

typedef struct {
  /* precomputed per source (sources.cpp:14-56, shortpulseinject.cpp:56-113) */
  double E[3];       /* plane sources: E amplitude vector */
  double om;
  /* short pulse */
  double lightspeed, ZRl, amp, phase, tshift, zshift, centre[3];
  /* gauss_inject: [0] the E current's state, [1] the H current's */
  gauss_state gs[2];
} src_state;

typedef struct mpo_sim {
  mp_config cfg;
  int NX, NY, NZ;       /* n + 2 */
  double *F[6];         /* Ex Ey Ez Bx By Bz */
  double *psiR[3][3], *psiI[3][3];
  double *Jt[3], *Mt[3];
  double *kapE[3], *kapH[3];
  int nE, nH;
  cpml_layer Elay[12], Hlay[12];
  int nIE, nIH;
  inc_layer IElay[6 * MP_MAX_SOURCES], IHlay[6 * MP_MAX_SOURCES];
  src_state src[MP_MAX_SOURCES];
  double complex dchi0[3], dxi0[3], crec[3];
  double sumChi0, sumXi0;
  /* design region: per-cell eps_infinity, Delta-eps factor, chi factor */
  int design;
  box3 dbox;
  double *deps, *dscale, *dchi;
  /* plasma plug-ins (fdtd_plrc.t:431-436): density, conductivity Sigma
   * (reset every step, fdtd_plrc.t:129), plasma current; full ghost grids */
  double *rho, *Sig, *PJ[3];
  long long time;
  int newton_fail;
  char err[256];
} mpo_sim;

static char g_create_err[256];

#define IDX(s, i, j, k) (((size_t)(k) * (size_t)(s)->NY + (size_t)(j)) * (size_t)(s)->NX + (size_t)(i))

/* ------------------------------------------------------------------------ */
/* Faddeeva function w(z) = exp(-z^2) erfc(-iz) for Im z >= 0.
 *
 * MPulse calls Faddeeva_2 (specfunc.cpp:57-157, Matpack; its licence forbids
 * redistribution), always with Im z >= 0 (shortpulsefunctions.cpp:77-91).  This
 * oracle uses J.A.C. Weideman's rational expansion instead ("Computation of the
 * complex error function", SIAM J. Numer. Anal. 31 (1994) 1497-1518):
 *     w(z) = 2 p(Z) / (L - iz)^2 + 1 / (sqrt(pi) (L - iz)),  Z = (L+iz)/(L-iz),
 * p a polynomial of degree N-1 whose coefficients are the Fourier coefficients
 * of f(t) = exp(-t^2) (L^2 + t^2) at t = L tan(theta/2), L = sqrt(N / sqrt 2).
 * With N = 40 the relative error is about 1e-14 in the upper half plane, so the
 * oracle agrees with the reference's short-pulse fields to about that level
 * rather than bit for bit. */
#define W_N 40
static double w_coef[W_N];
static double w_L;
static int w_ready;

static void oracle_faddeeva_init(void) {
  if (w_ready) return;
  const int N = W_N, M = 2 * N, M2 = 2 * M;
  w_L = sqrt(N / sqrt(2.0));
  double f[4 * W_N];
  /* samples at theta_k = k pi / M, k = -M+1 .. M-1, plus f(-M) = 0, arranged
   * for an FFT of length 2M with the k = 0 sample first */
  for (int n = 0; n < M2; ++n) {
    int k = n <= M ? n : n - M2; /* wrap to -M..M-1 */
    if (k == -M || k == M) { f[n] = 0.0; continue; }
    double t = w_L * tan(0.5 * k * M_PI / M);
    f[n] = exp(-t * t) * (w_L * w_L + t * t);
  }
  /* a_n = Re(FFT(f))_n / 2M for n = 1 .. N, stored highest power first */
  for (int n = 1; n <= N; ++n) {
    double s = 0.0;
    for (int m = 0; m < M2; ++m) s += f[m] * cos(2.0 * M_PI * (double)n * m / M2);
    w_coef[N - n] = s / M2;
  }
  w_ready = 1;
}

static double complex oracle_faddeeva(double complex z) {
  const double complex Lmz = w_L - I * z;
  const double complex Z = (w_L + I * z) / Lmz;
  double complex p = w_coef[0];
  for (int n = 1; n < W_N; ++n) p = p * Z + w_coef[n];
  return 2.0 * p / (Lmz * Lmz) + (1.0 / sqrt(M_PI)) / Lmz;
}

/* ------------------------------------------------------------------------ */
/* Short-pulse closed form: ShortPulseInjectSourceFunc::Efunc / Bfunc
 * (shortpulsefunctions.cpp:28-226), paraxial focused pulse with complex beam
 * parameter q = z + i ZRl.  The expressions follow the reference term by term. */
static double complex sp_efunc(const src_state *st, const mp_source *s, double x, double y,
                               double z, double t) {
  const double c = st->lightspeed;
  const double p = st->phase;
  const double T = s->length, T2 = T * T, T4 = T2 * T2, tb = 0.5 * s->om0 * T;
  const double r2 = x * x + y * y;
  const double complex q = CMPLX(z, st->ZRl);
  const double complex rT = st->ZRl / q;
  const double complex rpiT = sqrt(M_PI) * rT;
  const double complex rpT = -st->ZRl / (q * q);
  const double complex eiphi = cexp(2.0 * I * p);
  const double complex tpT = t - z / c - r2 / (2. * c * q);
  const double complex tpT2 = tpT * tpT;
  const double complex tpzT = -1 / c - r2 / (2. * c * q * q);
  double complex an = -I * tb + tpT / T;
  double complex ap = I * tb + tpT / T;
  const double complex A = cexp(-I * p) / (rpiT * T4);
  const double complex B =
      rT * T * (I * (1.0 + eiphi) * rpT * T2 -
                rT * (T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) + 2.0 * I * (1.0 + eiphi) * tpT) * tpzT);
  double complex C = I * eiphi * rpiT * (T * tb + I * tpT) *
                     (rpT * T2 + 2.0 * I * rT * T * tb * tpzT - 2.0 * rT * tpT * tpzT);
  double complex D = rpiT * (T * tb - I * tpT) * (I * rpT * T2 + 2.0 * rT * (T * tb - I * tpT) * tpzT);
  double complex S = 0;
  if (cimag(an) < 0) {
    S += 2.0 * A * C * cexp(2.0 * I * tpT * tb / T - tpT2 / T2);
    an = -an;
    C = -C;
  }
  if (cimag(ap) < 0) {
    S += 2.0 * A * D * cexp(-2.0 * I * tpT * tb / T - tpT2 / T2);
    ap = -ap;
    D = -D;
  }
  const double complex Ef = S + A * exp(-tb * tb) * (B + C * oracle_faddeeva(an) - D * oracle_faddeeva(ap));
  return -I * Ef;
}

/* Bfunc with YComp = 0 (shortpulseinject.cpp:96): bx -> i BfA, by -> i (BfD - BfB). */
static double complex sp_bfunc(const src_state *st, const mp_source *s, double x, double y,
                               double z, double t, int bx) {
  const double c = st->lightspeed;
  const double p = st->phase;
  const double T = s->length, T2 = T * T, T4 = T2 * T2, tb = 0.5 * s->om0 * T;
  const double r2 = x * x + y * y;
  const double complex q = CMPLX(z, st->ZRl);
  const double complex rT = st->ZRl / q;
  const double complex rT2 = rT * rT;
  const double complex rT4T = rT * T4;
  const double complex rpiT = sqrt(M_PI) * rT;
  const double complex rpT = -st->ZRl / (q * q);
  const double complex rppT = 2. * st->ZRl / (q * q * q);
  const double complex eiphi = cexp(2.0 * I * p);
  const double complex tpT = t - z / c - r2 / (2. * c * q);
  const double complex tpT2 = tpT * tpT;
  const double complex tpzT = -1 / c + r2 / (2. * c * q * q);
  const double complex tpzT2 = tpzT * tpzT;
  const double complex tpxT = -x / (c * q);
  const double complex tpyT = -y / (c * q);
  const double complex tpxxT = -1. / (c * q);
  const double complex tpzzT = -r2 / (c * q * q * q);
  const double complex tpxT2 = tpxT * tpxT;
  const double complex aip = T * tb + I * tpT;
  const double complex ain = T * tb - I * tpT;
  const double complex aip2 = aip * aip;
  const double complex ain2 = ain * ain;
  double complex an = -I * tb + tpT / T;
  double complex ap = I * tb + tpT / T;
  const double complex common = T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) + 2.0 * I * (1.0 + eiphi) * tpT;

  /* A terms (tpxyT = 0 in the reference) */
  const double complex AA = cexp(-I * p) / (sqrt(M_PI) * T4);
  const double complex AB = -tpxT * tpyT * rT * T * common;
  double complex AC = -tpxT * tpyT * 2.0 * eiphi * rpiT * aip2;
  double complex AD = -tpxT * tpyT * 2.0 * rpiT * ain2;
  double complex AS = 0;
  /* B terms */
  const double complex BA = cexp(-I * p) / (sqrt(M_PI) * T4);
  const double complex BB = -tpxT2 * (rT * T * common) + I * T2 * tpxxT * (1.0 + eiphi) * rT * T;
  double complex BC = -tpxT2 * 2.0 * eiphi * rpiT * aip2 + I * T2 * tpxxT * eiphi * rpiT * aip;
  double complex BD = -tpxT2 * 2.0 * rpiT * ain2 + I * T2 * tpxxT * rpiT * (-(T * tb) + I * tpT);
  double complex BS = 0;
  /* D terms */
  const double complex DA = cexp(-I * p) / (2. * sqrt(M_PI) * T4);
  const double complex DB =
      2.0 * T * (2.0 * I * (1.0 + eiphi) * rpT * T2 * tpzT -
                 rT * (T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) * tpzT2 +
                       I * (1.0 + eiphi) * (2.0 * tpT * tpzT2 - T2 * tpzzT)));
  double complex DC = (eiphi * rpiT *
                       (rppT * rT4T + 2.0 * I * rT * aip *
                                          (2.0 * rpT * T2 * tpzT +
                                           rT * (2.0 * I * T * tb * tpzT2 - 2.0 * tpT * tpzT2 + T2 * tpzzT)))) /
                      rT2;
  double complex DD = (rpiT * (rppT * rT4T - 2.0 * rT * ain *
                                                  (2.0 * I * rpT * T2 * tpzT +
                                                   rT * (2.0 * T * tb * tpzT2 - 2.0 * I * tpT * tpzT2 +
                                                         I * T2 * tpzzT)))) /
                      rT2;
  double complex DS = 0;

  if (cimag(an) < 0) {
    const double complex e = cexp(2.0 * I * tpT * tb / T - tpT2 / T2);
    AS += 2.0 * AA * AC * e;
    BS += 2.0 * BA * BC * e;
    DS += 2.0 * DA * DC * e;
    AC = -AC; BC = -BC; DC = -DC;
    an = -an;
  }
  if (cimag(ap) < 0) {
    const double complex e = cexp(-2.0 * I * tpT * tb / T - tpT2 / T2);
    AS += 2.0 * AA * AD * e;
    BS += 2.0 * BA * BD * e;
    DS += 2.0 * DA * DD * e;
    AD = -AD; BD = -BD; DD = -DD;
    ap = -ap;
  }
  const double complex wn = oracle_faddeeva(an);
  const double complex wp = oracle_faddeeva(ap);
  const double g = exp(-tb * tb);
  const double complex fA = AS + AA * g * (AB + AC * wn - AD * wp);
  if (bx) return I * fA;
  const double complex fB = BS + BA * g * (BB + BC * wn - BD * wp);
  const double complex fD = DS + DA * g * (DB + DC * wn - DD * wp);
  return I * (fD - fB);
}

/* ------------------------------------------------------------------------ */
/* gauss_inject: GaussInjectSourceFunc (gaussinject.cpp:56-482) and its
 * GaussFunc helpers (gaussinject.h:166-203). */

static double gf_gauss(const gauss_state *g, double x, double y, double z) {
  const double zoff = z - g->k0;
  return exp(-0.25 * zoff * zoff * g->length * g->length - 0.25 * (x * x + y * y) * g->width * g->width);
}
static double gf_shift(const gauss_state *g, double x, double y, double z) {
  return -(x * g->sx + y * g->sy + z * g->sz);
}
static double gf_kp(double x, double z) { return sqrt(x * x + z * z); }
static double gf_k(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }
static double gf_comp(int which, double x, double y, double z) {
  if (which == 0) { /* excomp */
    const double D = gf_k(x, y, z) * gf_kp(x, z);
    return D == 0 ? 0 : (-x * y / D);
  }
  if (which == 1) { /* eycomp */
    const double D = gf_k(x, y, z);
    return D == 0 ? 0 : (gf_kp(x, z) / D);
  }
  const double D = gf_kp(x, z); /* bxcomp */
  return D == 0 ? 0 : (-z / D);
}
static int gf_sign(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

/* Unnormalised DFT with FFTW's conventions: out[k] = sum_j in[j] e^{sign 2 pi i jk/n}. */
static void dft(const double complex *in, double complex *out, int n, int sign) {
  for (int k = 0; k < n; ++k) {
    double complex s = 0;
    for (int j = 0; j < n; ++j) {
      const double a = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / n;
      s += in[j] * CMPLX(cos(a), sin(a));
    }
    out[k] = s;
  }
}

/* fillEx / fillEy / fillBx (gaussinject.cpp:329-482) with transformT / Y / X
 * (:257-327): the angular spectrum at (kx, ky, omega), backward transform over
 * omega (only the Nt samples of the current block kept), forward transforms
 * over ky and kx, real part. */
static void gauss_fill(gauss_state *g, int which, double *F) {
  const int SX = g->SizeX, SY = g->SizeY, ST = g->SizeT, Nt = g->Nt;
  double complex *A = malloc(sizeof(double complex) * ST);
  double complex *uo = malloc(sizeof(double complex) * ST), *ut = malloc(sizeof(double complex) * ST);
  double complex *uy_in = malloc(sizeof(double complex) * SY), *uy = malloc(sizeof(double complex) * SY);
  double complex *ux_in = malloc(sizeof(double complex) * SX), *ux = malloc(sizeof(double complex) * SX);
  double complex *tmpTY = malloc(sizeof(double complex) * SY * Nt);
  double complex *tmpTX = malloc(sizeof(double complex) * SX * SY * Nt);
  const int blockmin = g->blockCount * Nt;
  for (int i = 0; i < SX; ++i) {
    for (int j = 0; j < SY; ++j) {
      for (int k = 0; k < ST; ++k) {
        const double kx = 2 * M_PI * (i - g->SizeXH) / (g->BoxX);
        const double ky = 2 * M_PI * (j - g->SizeYH) / (g->BoxY);
        const double om = 2 * M_PI * (k - g->SizeTH) / (g->BoxT);
        double K = om * om - ky * ky - kx * kx;
        if (fabs(K) < 1e-9) K = 0;
        if (K < 0) A[k] = 0;
        else {
          const double kz = sqrt(K) * gf_sign(om);
          const double a = gf_comp(which, kx, ky, kz) * gf_gauss(g, kx, ky, kz);
          const double ph = gf_shift(g, kx, ky, kz) + 0.5 * M_PI;
          A[k] = a * cexp(-I * (ph + g->Time * om));
        }
      }
      /* transformT */
      const double fT = (2 * M_PI * g->length / g->BoxT);
      for (int k = 0; k < ST; ++k) uo[k] = A[(k + g->SizeTH) % ST];
      dft(uo, ut, ST, +1);
      for (int kh = 0; kh < Nt; ++kh) tmpTY[j * Nt + kh] = fT * ut[(kh + blockmin + g->SizeTH) % ST];
    }
    /* transformY */
    const double fY = (g->width / g->BoxY);
    for (int k = 0; k < Nt; ++k) {
      for (int j = 0; j < SY; ++j) uy_in[(j + g->SizeYH) % SY] = tmpTY[j * Nt + k];
      dft(uy_in, uy, SY, -1);
      for (int j = 0; j < SY; ++j) tmpTX[((size_t)i * SY + j) * Nt + k] = fY * uy[(j + g->SizeYH) % SY];
    }
  }
  /* transformX */
  const double fX = (g->width / g->BoxX);
  for (int j = 0; j < SY; ++j)
    for (int k = 0; k < Nt; ++k) {
      for (int i = 0; i < SX; ++i) ux_in[(i + g->SizeXH) % SX] = tmpTX[((size_t)i * SY + j) * Nt + k];
      dft(ux_in, ux, SX, -1);
      for (int i = 0; i < SX; ++i) F[((size_t)i * SY + j) * Nt + k] = fX * creal(ux[(i + g->SizeXH) % SX]);
    }
  free(A); free(uo); free(ut); free(uy_in); free(uy); free(ux_in); free(ux); free(tmpTY); free(tmpTX);
}

/* GaussInjectSourceFunc::setTime (gaussinject.cpp:152-184).  The reference
 * computes block c = 0, 1, .. when the time reaches toff + c Nt and switches
 * off at the first block start at or past toff + SizeT, so for times that step
 * by one the state at time t is: inactive before toff, block
 * b = (t - toff) / Nt while b Nt < SizeT, inactive after.  That function of t
 * is what is computed here; it also covers times set directly, where the
 * reference's block counter would index outside its block. */
static void gauss_set_time(gauss_state *g, long long time) {
  if (time < g->toff) {
    g->active = 0;
    return;
  }
  const long long b = (time - g->toff) / g->Nt;
  if (b * g->Nt >= g->SizeT) {
    g->active = 0;
    return;
  }
  g->active = 1;
  if (g->computed == b) return;
  g->blockCount = (int)b;
  if (!g->isH) {
    g->sx = 0; g->sy = 0.5 * g->DX; g->sz = g->Shift + 0.5 * g->DX;
    gauss_fill(g, 2, g->F1);
  } else {
    /* Time -= DT/2 for the fills and += DT/2 after them, once per block: block
     * b sees Time moved by b such round trips */
    double T = g->Time0;
    for (long long n = 0; n < b; ++n) T = (T - 0.5 * g->DT) + 0.5 * g->DT;
    g->Time = T - 0.5 * g->DT;
    g->sx = 0.5 * g->DX; g->sy = 0; g->sz = g->Shift;
    gauss_fill(g, 0, g->F1);
    g->sx = 0; g->sy = 0.5 * g->DX; g->sz = g->Shift;
    gauss_fill(g, 1, g->F2);
  }
  g->blockToff = g->toff + g->blockCount * g->Nt;
  g->computed = b;
}

/* GaussInjectSourceFunc::setParam / initSourceFunc (gaussinject.cpp:56-150). */
static void gauss_init(gauss_state *g, const mp_source *p, const mp_config *c, int isH) {
  memset(g, 0, sizeof(*g));
  g->isH = isH;
  g->SizeT = p->t_size;
  g->length = p->length;
  g->width = p->width;
  g->k0 = p->k0;
  g->Shift = p->shift;
  g->Time = p->time;
  g->Time0 = p->time;
  g->amp = p->amp;
  g->eps = p->eps;
  g->toff = p->t_off;
  g->lightspeed = sqrt(1 / g->eps);
  g->SizeX = c->nx + 2;
  g->SizeY = c->ny + 2;
  g->SizeTH = g->SizeT / 2;
  g->SizeXH = g->SizeX / 2;
  g->SizeYH = g->SizeY / 2;
  g->DX = c->dx;
  g->DY = c->dy;
  g->DT = c->dt * g->lightspeed;
  g->BoxX = g->SizeX * g->DX;
  g->BoxY = g->SizeY * g->DY;
  g->BoxT = g->SizeT * g->DT;
  g->blockCount = 0;
  g->blockToff = g->toff;
  g->active = 0;
  g->computed = -1;
  /* initSourceFunc (gaussinject.cpp:142): high[2] - low[2] of the storage,
   * whose z range is 0..nz+1 */
  g->Nt = 1 << (int)round(log((double)(c->nz + 1)) / log(2.0) + 1e-6);
  const size_t n = (size_t)g->SizeX * g->SizeY * g->Nt;
  g->F1 = calloc(n, sizeof(double));
  g->F2 = calloc(n, sizeof(double));
}

static double gauss_value(const gauss_state *g, const double *F, int i, int j, long long time) {
  const long long t = time - g->blockToff;
  return F[((size_t)i * g->SizeY + j) * g->Nt + (size_t)t];
}

/* ------------------------------------------------------------------------ */
/* Source functions: the field a TF/SF current needs at cell (i, j, l). */

/* PlaneWaveSourceEFunc::getHField (sources.cpp:107-125) and
 * PlaneGaussSourceEFunc::getHField (sources.cpp:266-284). */
static void src_hfield(const mpo_sim *s, int n, int i, int j, int l, long long time, double h[3]) {
  const mp_source *p = &s->cfg.sources[n];
  const src_state *st = &s->src[n];
  const double dx = s->cfg.dx, dy = s->cfg.dy, dz = s->cfg.dz, dt = s->cfg.dt;
  if (p->kind == MP_SOURCE_PLANE_WAVE || p->kind == MP_SOURCE_PLANE_GAUSS) {
    const double realtime = dt * ((double)time - 0.5);
    const double *k = p->k;
    const double pos[3] = {
        k[0] * i * dx + k[1] * (j + 0.5) * dy + k[2] * (l + 0.5) * dz + st->om * realtime,
        k[0] * (i + 0.5) * dx + k[1] * j * dy + k[2] * (l + 0.5) * dz + st->om * realtime,
        k[0] * (i + 0.5) * dx + k[1] * (j + 0.5) * dy + k[2] * l * dz + st->om * realtime};
    for (int c = 0; c < 3; ++c) {
      if (p->kind == MP_SOURCE_PLANE_WAVE) {
        double v = p->H[c] * sin(pos[c]) + p->H_bg[c];
        if (pos[c] < p->ramp) v *= pos[c] / p->ramp;
        h[c] = v;
      } else {
        const double a = (pos[c] - p->offset) / p->width;
        const double amp = p->H[c] * exp(-(a * a));
        h[c] = amp * sin(pos[c]);
      }
    }
    return;
  }
  if (p->kind == MP_SOURCE_SHORT_PULSE || p->kind == MP_SOURCE_FOCUSED_PULSE) {
    /* ShortPulseInjectSourceFunc::getHField (shortpulseinject.cpp:151-178) */
    const double posxo = (i - st->centre[0]) * dx;
    const double posxh = (i + 0.5 - st->centre[0]) * dx;
    const double posyo = (j - st->centre[1]) * dy;
    const double posyh = (j + 0.5 - st->centre[1]) * dy;
    const double poszh = (l - 0.5 - st->centre[2]) * dz - st->zshift;
    const double posTime = ((double)time - 0.5) * dt - st->tshift;
    h[0] = st->amp * creal(sp_bfunc(st, p, posxo, posyh, poszh, posTime, 1));
    h[1] = st->amp * creal(sp_bfunc(st, p, posxh, posyo, poszh, posTime, 0));
    h[2] = 0.0;
    return;
  }
  if (p->kind == MP_SOURCE_GAUSS_BEAM) {
    /* GaussInjectSourceFunc::getHField (gaussinject.cpp:215-223) */
    const gauss_state *g = &st->gs[0];
    h[0] = g->active ? sqrt(g->eps) * g->amp * gauss_value(g, g->F1, i, j, time) : 0.0;
    h[1] = 0.0;
    h[2] = 0.0;
    return;
  }
  h[0] = h[1] = h[2] = 0.0;
}

/* PlaneWaveSourceHFunc::getEField (sources.cpp:150-173),
 * PlaneGaussSourceHFunc::getEField (sources.cpp:308-331),
 * ShortPulseInjectSourceFunc::getEField (shortpulseinject.cpp:126-149). */
static void src_efield(const mpo_sim *s, int n, int i, int j, int l, long long time, double e[3]) {
  const mp_source *p = &s->cfg.sources[n];
  const src_state *st = &s->src[n];
  const double dx = s->cfg.dx, dy = s->cfg.dy, dz = s->cfg.dz, dt = s->cfg.dt;
  if (p->kind == MP_SOURCE_PLANE_WAVE || p->kind == MP_SOURCE_PLANE_GAUSS) {
    const double realtime = dt * (double)time;
    const double *k = p->k;
    const double pos[3] = {
        k[0] * (i + 0.5) * dx + k[1] * j * dy + k[2] * l * dz + st->om * realtime,
        k[0] * i * dx + k[1] * (j + 0.5) * dy + k[2] * l * dz + st->om * realtime,
        k[0] * i * dx + k[1] * j * dy + k[2] * (l + 0.5) * dz + st->om * realtime};
    for (int c = 0; c < 3; ++c) {
      if (p->kind == MP_SOURCE_PLANE_WAVE) {
        double v = st->E[c] * sin(pos[c]) + p->E_bg[c];
        if (pos[c] < p->ramp) v *= pos[c] / p->ramp;
        e[c] = v;
      } else {
        const double a = (pos[c] - p->offset) / p->width;
        const double amp = st->E[c] * exp(-(a * a));
        e[c] = amp * sin(pos[c]);
      }
    }
    return;
  }
  if (p->kind == MP_SOURCE_SHORT_PULSE || p->kind == MP_SOURCE_FOCUSED_PULSE) {
    const double posxh = (i + 0.5 - st->centre[0]) * dx;
    const double posyo = (j - st->centre[1]) * dy;
    const double poszo = (l - st->centre[2]) * dz - st->zshift;
    const double posTime = (double)time * dt - st->tshift;
    e[0] = st->amp * creal(sp_efunc(st, p, posxh, posyo, poszo, posTime));
    e[1] = 0.0;
    e[2] = 0.0;
    return;
  }
  if (p->kind == MP_SOURCE_GAUSS_BEAM) {
    /* GaussInjectSourceFunc::getEField (gaussinject.cpp:205-213) */
    const gauss_state *g = &st->gs[1];
    e[0] = g->active ? g->amp * gauss_value(g, g->F1, i, j, time) : 0.0;
    e[1] = g->active ? g->amp * gauss_value(g, g->F2, i, j, time) : 0.0;
    e[2] = 0.0;
    return;
  }
  e[0] = e[1] = e[2] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Storage::getBorderExtent (storage.cpp:208-318) with bordercells = 0. */
static int border_extent(const mpo_sim *s, int dir, int thickness, int distance, box3 *b) {
  const int glow[3] = {0, 0, 0};
  const int ghigh[3] = {s->cfg.nx + 1, s->cfg.ny + 1, s->cfg.nz + 1};
  int have = 0;
  for (int d = 0; d < 3; ++d) { b->lo[d] = glow[d]; b->hi[d] = ghigh[d]; }
  switch (dir) {
    case DIR_WEST:
      if (glow[0] < glow[0] + thickness + distance) {
        b->hi[0] = glow[0] + thickness - 1 + distance; b->lo[0] = glow[0] + distance; have = 1;
      }
      break;
    case DIR_SOUTH:
      if (glow[1] < glow[1] + thickness + distance) {
        b->hi[1] = glow[1] + thickness - 1 + distance; b->lo[1] = glow[1] + distance; have = 1;
      }
      break;
    case DIR_DOWN:
      if (glow[2] < glow[2] + thickness + distance && ghigh[2] >= glow[2] + thickness) {
        b->hi[2] = glow[2] + thickness - 1 + distance; b->lo[2] = glow[2] + distance; have = 1;
      }
      break;
    case DIR_EAST:
      if (ghigh[0] > ghigh[0] - thickness - distance) {
        b->lo[0] = ghigh[0] - thickness + 1 - distance; b->hi[0] = ghigh[0] - distance; have = 1;
      }
      break;
    case DIR_NORTH:
      if (ghigh[1] > ghigh[1] - thickness - distance) {
        b->lo[1] = ghigh[1] - thickness + 1 - distance; b->hi[1] = ghigh[1] - distance; have = 1;
      }
      break;
    case DIR_UP:
      if (ghigh[2] > ghigh[2] - thickness - distance) {
        b->lo[2] = ghigh[2] - thickness + 1 - distance; b->hi[2] = ghigh[2] - distance; have = 1;
      }
      break;
  }
  for (int d = 0; d < 3; ++d) b->dims[d] = b->hi[d] - b->lo[d] + 1;
  return have;
}

static int dir_dim(int dir) {
  return (dir == DIR_EAST || dir == DIR_WEST) ? 0 : (dir == DIR_NORTH || dir == DIR_SOUTH) ? 1 : 2;
}

/* CPMLBorderCurrent::makeCoeff (cpml_border.cpp:287-339). */
static void cpml_make_coeff(const mpo_sim *s, cpml_layer *L) {
  const mp_config *c = &s->cfg;
  const int d = c->cpml_d;
  const int reverse = (L->dir == DIR_WEST || L->dir == DIR_SOUTH || L->dir == DIR_DOWN);
  const int lowk = L->box.lo[L->dim], highk = L->box.hi[L->dim];
  const double offset = L->isH ? 0.5 : 0.0;
  const int n = highk - lowk + 1;
  L->b = calloc((size_t)n, sizeof(double));
  L->c = calloc((size_t)n, sizeof(double));
  for (int k = 0; k < d; ++k) {
    const double x = 1 - ((double)k - offset) / (double)d;
    const double x3 = x * x * x;
    const int pos = reverse ? (lowk + k) : (highk - k);
    const double sigma = x3 * c->cpml_sigma_max;
    const double kappa = 1 + (c->cpml_kappa_max - 1) * x3;
    const double a = c->cpml_a_max * (1 - x);
    const double b = exp(-(sigma / kappa + a) * c->dt / 1.0);
    const double cc = sigma * (b - 1) / (kappa * (sigma + kappa * a));
    L->b[pos - lowk] = b;
    L->c[pos - lowk] = cc;
  }
}

static int add_cpml_layer(mpo_sim *s, int dir, int isH) {
  cpml_layer *L = isH ? &s->Hlay[s->nH] : &s->Elay[s->nE];
  memset(L, 0, sizeof(*L));
  L->dir = dir;
  L->dim = dir_dim(dir);
  L->isH = isH;
  /* distances: E layers 1 (cpml_border.cpp:353), H layers 1 for east/north/up
   * and 0 for west/south/down (cpml_border.cpp:441-450) */
  int distance = 1;
  if (isH && (dir == DIR_WEST || dir == DIR_SOUTH || dir == DIR_DOWN)) distance = 0;
  if (!border_extent(s, dir, s->cfg.cpml_d, distance, &L->box)) return 0;
  const size_t n = box_size(&L->box);
  L->psi[0] = calloc(n, sizeof(double));
  L->psi[1] = calloc(n, sizeof(double));
  L->delta = L->dim == 0 ? s->cfg.dx : L->dim == 1 ? s->cfg.dy : s->cfg.dz;
  cpml_make_coeff(s, L);
  if (isH) s->nH++; else s->nE++;
  return 0;
}

/* Kappa lines: CPMLBorder::initCoefficients (cpml_border.cpp:58-139) and
 * CPMLBorderOneD::initCoefficients (cpml_border.cpp:179-243). */
static void init_kappa(mpo_sim *s) {
  const mp_config *c = &s->cfg;
  const int n[3] = {c->nx, c->ny, c->nz};
  const int d = c->cpml_d;
  for (int dim = 0; dim < 3; ++dim) {
    for (int i = 0; i < n[dim] + 2; ++i) s->kapE[dim][i] = s->kapH[dim][i] = 1.0;
  }
  if (c->cpml == MP_CPML_ALL) {
    for (int dim = 0; dim < 3; ++dim) {
      const int low = 0, high = n[dim] + 1;
      for (int i = 0; i <= d; ++i) {
        const double x = 1 - (double)i / (double)d, x3 = x * x * x;
        s->kapE[dim][low + i] = 1 + (c->cpml_kappa_max - 1) * x3;
      }
      for (int i = 0; i < d; ++i) {
        const double x = 1 - ((double)i + 0.5) / (double)d, x3 = x * x * x;
        s->kapH[dim][low + i] = 1 + (c->cpml_kappa_max - 1) * x3;
      }
      for (int i = 0; i <= d; ++i) {
        const double x = 1 - (double)i / (double)d, x3 = x * x * x;
        s->kapH[dim][high - i] = 1 + (c->cpml_kappa_max - 1) * x3;
      }
      for (int i = 0; i < d; ++i) {
        const double x = 1 - ((double)i + 0.5) / (double)d, x3 = x * x * x;
        s->kapE[dim][high - i] = 1 + (c->cpml_kappa_max - 1) * x3;
      }
    }
  } else if (c->cpml == MP_CPML_Z) {
    const int low = 0, high = n[2] + 1;
    for (int i = 0; i < d; ++i) {
      const double x = 1 - (double)i / (double)d, x3 = x * x * x;
      s->kapE[2][low + i + 1] = 1 + (c->cpml_kappa_max - 1) * x3;
    }
    for (int i = 0; i < d; ++i) {
      const double x = 1 - ((double)i + 0.5) / (double)d, x3 = x * x * x;
      s->kapH[2][low + i] = 1 + (c->cpml_kappa_max - 1) * x3;
    }
    for (int i = 0; i < d; ++i) {
      const double x = 1 - (double)i / (double)d, x3 = x * x * x;
      s->kapE[2][high - i - 1] = 1 + (c->cpml_kappa_max - 1) * x3;
    }
    for (int i = 0; i < d; ++i) {
      const double x = 1 - (double)(i + 0.5) / (double)d, x3 = x * x * x;
      s->kapH[2][high - i - 1] = 1 + (c->cpml_kappa_max - 1) * x3;
    }
  }
}

/* IncidentSource::initCurrents (incsource.cpp:16-77) for the faces the source
 * needs (all of the built kinds inject on `down` only: sources.cpp:8-11,
 * :179-182, shortpulseinject.cpp:28-31) and IncidentSourceCurrent
 * (incsource.cpp:93-136), IncidentSourceE/HCurrent::initStorage
 * (incsource.t:14-32, :88-104). */
static void add_inc_layers(mpo_sim *s, int n) {
  const mp_source *p = &s->cfg.sources[n];
  const int dir = DIR_DOWN;
  for (int isH = 0; isH < 2; ++isH) {
    inc_layer *L = isH ? &s->IHlay[s->nIH] : &s->IElay[s->nIE];
    memset(L, 0, sizeof(*L));
    L->src = n;
    L->dir = dir;
    L->isH = isH;
    L->dim = 2; L->t1 = 0; L->t2 = 1;
    L->DX = s->cfg.dz;
    const int reverse = (dir == DIR_EAST || dir == DIR_NORTH || dir == DIR_UP);
    int distance = p->distance;
    if (isH && !reverse) distance = distance - 1;
    if (!border_extent(s, dir, 1, distance, &L->box)) continue;
    /* Storage::addBorderLayer (storage.cpp:129-141) returns the grid already
     * registered under "IncidentEJx" / "IncidentHJx" for this face: every
     * injector on the face shares the first one's grid, and its extent. */
    const int nl = isH ? s->nIH : s->nIE;
    for (int q = 0; q < nl; ++q) {
      const inc_layer *F = isH ? &s->IHlay[q] : &s->IElay[q];
      if (F->dir == dir) { L->box = F->box; break; }
    }
    L->off[L->dim] = isH ? (reverse ? +1 : 0) : -1;
    if (isH) s->nIH++; else s->nIE++;
  }
}

/* ------------------------------------------------------------------------ */
/* PLRC coefficients, FDTD_PLRCSolver::stepD (fdtd_plrc.t:181-216). */
static void plrc_coefficients(mpo_sim *s) {
  const double dt = s->cfg.dt;
  double complex sumChi = 0.0, sumXi = 0.0;
  for (int n = 0; n < 3; ++n) {
    const mp_lorentz_pole *P = &s->cfg.poles[n];
    const double beta = sqrt(P->om2 - P->delta * P->delta);
    const double gamma = P->eps * P->om2 / beta;
    const double complex phasor = P->delta - I * beta;
    s->crec[n] = cexp(-phasor * dt);
    const double complex chi0 = (I * gamma * (s->crec[n] - 1.0) / phasor);
    const double complex xi0 = I * gamma * (s->crec[n] * (phasor * dt + 1.0) - 1.0) / (phasor * phasor * dt);
    s->dchi0[n] = chi0 * (1.0 - s->crec[n]);
    s->dxi0[n] = xi0 * (1.0 - s->crec[n]);
    sumChi += chi0;
    sumXi += xi0;
  }
  s->sumChi0 = creal(sumChi);
  s->sumXi0 = creal(sumXi);
}

/* ------------------------------------------------------------------------ */
/* Boundaries: SinglePeriodicBoundary / SingleXYPeriodicBoundary exchange
 * (periodic_bound.cpp:10-130), applied per field after each half step. */
static void exchange(mpo_sim *s, double *f) {
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  for (int k = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j) {
      f[IDX(s, 0, j, k)] = f[IDX(s, NX - 2, j, k)];
      f[IDX(s, NX - 1, j, k)] = f[IDX(s, 1, j, k)];
    }
  for (int k = 0; k < NZ; ++k)
    for (int i = 0; i < NX; ++i) {
      f[IDX(s, i, 0, k)] = f[IDX(s, i, NY - 2, k)];
      f[IDX(s, i, NY - 1, k)] = f[IDX(s, i, 1, k)];
    }
  if (s->cfg.boundary == MP_BOUNDARY_PERIODIC) {
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i) {
        f[IDX(s, i, j, 0)] = f[IDX(s, i, j, NZ - 2)];
        f[IDX(s, i, j, NZ - 1)] = f[IDX(s, i, j, 1)];
      }
  }
}

/* ------------------------------------------------------------------------ */
/* E-side currents. */

/* CPMLBorderECurrent::stepScheme (cpml_border.cpp:398-425).  Component map
 * from CPMLBorderECurrent::initStorage (cpml_border.cpp:357-386). */
static void cpml_e_step(mpo_sim *s, cpml_layer *L) {
  int b0, b1; /* B components: pB[0], pB[1] */
  switch (L->dim) {
    case 0: b0 = 4; b1 = 5; break;  /* By, Bz */
    case 1: b0 = 5; b1 = 3; break;  /* Bz, Bx */
    default: b0 = 3; b1 = 4; break; /* Bx, By */
  }
  const double *B0 = s->F[b0], *B1 = s->F[b1];
  const box3 *b = &L->box;
  for (int k = b->lo[2]; k <= b->hi[2]; ++k)
    for (int j = b->lo[1]; j <= b->hi[1]; ++j)
      for (int i = b->lo[0]; i <= b->hi[0]; ++i) {
        int ind[3] = {i, j, k};
        const int jj = ind[L->dim];
        int m[3] = {i, j, k};
        --m[L->dim];
        const size_t li = box_index(b, i, j, k);
        const size_t c0 = IDX(s, i, j, k), cm = IDX(s, m[0], m[1], m[2]);
        const double bc = L->b[jj - b->lo[L->dim]], cc = L->c[jj - b->lo[L->dim]];
        L->psi[0][li] = bc * L->psi[0][li] - cc * (B1[c0] - B1[cm]) / L->delta;
        L->psi[1][li] = bc * L->psi[1][li] + cc * (B0[c0] - B0[cm]) / L->delta;
      }
}

/* CPMLBorderHCurrent::stepScheme (cpml_border.cpp:499-527); component map
 * cpml_border.cpp:456-485. */
static void cpml_h_step(mpo_sim *s, cpml_layer *L) {
  int e0, e1;
  switch (L->dim) {
    case 0: e0 = 1; e1 = 2; break;  /* Ey, Ez */
    case 1: e0 = 2; e1 = 0; break;  /* Ez, Ex */
    default: e0 = 0; e1 = 1; break; /* Ex, Ey */
  }
  const double *E0 = s->F[e0], *E1 = s->F[e1];
  const box3 *b = &L->box;
  for (int k = b->lo[2]; k <= b->hi[2]; ++k)
    for (int j = b->lo[1]; j <= b->hi[1]; ++j)
      for (int i = b->lo[0]; i <= b->hi[0]; ++i) {
        int ind[3] = {i, j, k};
        const int jj = ind[L->dim];
        int p[3] = {i, j, k};
        ++p[L->dim];
        const size_t li = box_index(b, i, j, k);
        const size_t c0 = IDX(s, i, j, k), cp = IDX(s, p[0], p[1], p[2]);
        const double bc = L->b[jj - b->lo[L->dim]], cc = L->c[jj - b->lo[L->dim]];
        L->psi[0][li] = bc * L->psi[0][li] + cc * (E1[cp] - E1[c0]) / L->delta;
        L->psi[1][li] = bc * L->psi[1][li] - cc * (E0[cp] - E0[c0]) / L->delta;
      }
}

/* The components of a CPML current's J grid that are its psi arrays
 * (cpml_border.cpp:361-383): returns the field component index of psi[0],
 * psi[1]. */
static void cpml_components(int dim, int *c0, int *c1) {
  switch (dim) {
    case 0: *c0 = 1; *c1 = 2; break;
    case 1: *c0 = 2; *c1 = 0; break;
    default: *c0 = 0; *c1 = 1; break;
  }
}

/* Adds a layer's values into the J (or M) totals: the inner loop of
 * sumCurrents (fdtd_plrc.t:352-373). */
static void add_layer(mpo_sim *s, double **tot, const box3 *b, int comp[2], double *val[2]) {
  for (int k = b->lo[2]; k <= b->hi[2]; ++k)
    for (int j = b->lo[1]; j <= b->hi[1]; ++j)
      for (int i = b->lo[0]; i <= b->hi[0]; ++i) {
        const size_t li = box_index(b, i, j, k), g = IDX(s, i, j, k);
        tot[comp[0]][g] += val[0][li];
        tot[comp[1]][g] += val[1][li];
      }
}

/* IncidentSourceECurrent::stepScheme (incsource.t:40-73) /
 * IncidentSourceHCurrent::stepScheme (incsource.t:112-145), written straight
 * into the totals.  Injectors on one face share one grid (add_inc_layers), so
 * after all their stepScheme calls it holds the values of the last of them,
 * and sumCurrents adds that grid once per injector: `writer` is the source
 * whose values the shared grid holds. */
static void inc_add(mpo_sim *s, inc_layer *L, int writer, double **tot) {
  const box3 *b = &L->box;
  /* SourceFunc::setTime at the start of stepScheme (incsource.t:52-53, :124-125) */
  if (s->cfg.sources[writer].kind == MP_SOURCE_GAUSS_BEAM) gauss_set_time(&s->src[writer].gs[L->isH], s->time);
  for (int k = b->lo[2]; k <= b->hi[2]; ++k)
    for (int j = b->lo[1]; j <= b->hi[1]; ++j)
      for (int i = b->lo[0]; i <= b->hi[0]; ++i) {
        const int x = i + L->off[0], y = j + L->off[1], z = k + L->off[2];
        double f[3];
        if (L->isH) src_efield(s, writer, x, y, z, s->time, f);
        else src_hfield(s, writer, x, y, z, s->time, f);
        const size_t g = IDX(s, i, j, k);
        tot[L->t1][g] += f[L->t2] / L->DX;
        tot[L->t2][g] += f[L->t1] / L->DX;
      }
}

static int has_currents(const mpo_sim *s) { return s->nE + s->nIE > 0 || s->cfg.plasma_current; }
static int has_mag_currents(const mpo_sim *s) { return s->nH + s->nIH > 0; }

static void sum_currents(mpo_sim *s, int mag) {
  double **tot = mag ? s->Mt : s->Jt;
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  for (int c = 0; c < 3; ++c) memset(tot[c], 0, n * sizeof(double));
  /* current order: the CPML factory's currents (cpml_border.cpp:16-52 /
   * :161-173), then the sources' (incsource.cpp:16-77), as when cpml_border is
   * listed before the injector in the setup file */
  const int nl = mag ? s->nH : s->nE;
  for (int l = 0; l < nl; ++l) {
    cpml_layer *L = mag ? &s->Hlay[l] : &s->Elay[l];
    int comp[2];
    cpml_components(L->dim, &comp[0], &comp[1]);
    add_layer(s, tot, &L->box, comp, L->psi);
  }
  const int ni = mag ? s->nIH : s->nIE;
  for (int l = 0; l < ni; ++l) {
    inc_layer *L = mag ? &s->IHlay[l] : &s->IElay[l];
    int writer = L->src;
    for (int q = 0; q < ni; ++q) {
      const inc_layer *F = mag ? &s->IHlay[q] : &s->IElay[q];
      if (F->dir == L->dir) writer = F->src;
    }
    inc_add(s, L, writer, tot);
  }
  /* the plasma current last, over its full grid (plasma_current listed after
   * the CPML and injector blocks) */
  if (!mag && s->cfg.plasma_current)
    for (int c = 0; c < 3; ++c)
      for (size_t g = 0; g < n; ++g) tot[c][g] += s->PJ[c][g];
}

/* util.h ipow: r = 1, then K times r *= x. */
static double plasma_ipow(double x, int e) {
  double r = 1.0;
  for (int q = 0; q < e; ++q) r *= x;
  return r;
}

/* PlasmaDensity::stepScheme (plasmadensity.cpp:18-49): over every stored cell
 * (ghosts included), from E^n. */
static void plasma_density_step(mpo_sim *s) {
  const mp_config *c = &s->cfg;
  const double dt = c->dt;
  const double nn = 0.5 * dt * c->plasma_nu;
  const double m = dt * c->plasma_mpa;
  const double w = c->plasma_mpa * c->plasma_wion;
  const int Km = c->plasma_k - 1;
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  for (size_t g = 0; g < n; ++g) {
    const double ex = s->F[0][g], ey = s->F[1][g], ez = s->F[2][g];
    const double In = ex * ex + ey * ey + ez * ez;  /* I of the reference (I is complex.h's unit) */
    const double IKm = plasma_ipow(In, Km);
    const double IK = In * IKm;
    s->rho[g] = (s->rho[g] * (1 + nn * In) + m * IK) / (1 - nn * In);
    s->Sig[g] += w * IKm;
  }
}

/* PlasmaCurrent::stepScheme (plasmacurrent.cpp:42-74): cells low..high-1 of
 * every axis, from E^n and the density of this step. */
static void plasma_current_step(mpo_sim *s) {
  const mp_config *c = &s->cfg;
  const double dt = c->dt;
  const double gdtn = 1 - 0.5 * c->plasma_gamma * dt;
  const double gdtd = 1 + 0.5 * c->plasma_gamma * dt;
  const double emdt = c->plasma_em * dt;
  for (int i = 0; i < s->NX - 1; ++i)
    for (int j = 0; j < s->NY - 1; ++j)
      for (int k = 0; k < s->NZ - 1; ++k) {
        const size_t g = IDX(s, i, j, k);
        const double rho = s->rho[g] + c->plasma_rho_bg;
        s->PJ[0][g] = (s->PJ[0][g] * gdtn - emdt * s->F[0][g] * rho) / gdtd;
        s->PJ[1][g] = (s->PJ[1][g] * gdtn - emdt * s->F[1][g] * rho) / gdtd;
        s->PJ[2][g] = (s->PJ[2][g] * gdtn - emdt * s->F[2][g] * rho) / gdtd;
      }
}

/* ------------------------------------------------------------------------ */
/* The D / E update of one cell. */

static int in_medium(const mpo_sim *s, int k) {
  return k >= s->cfg.medium_z0 && k <= s->cfg.medium_z1;
}

/* FDTD_PLRCLinCore::plrcStepD (fdtd_plrc.cpp:94-261) and
 * FDTD_PLRCNonlinCore::plrcStepD (fdtd_plrc.cpp:304-427); outside the medium
 * eps = eps_bg, no poles, chi = 0. */
static void plrc_step_d(mpo_sim *s, int i, int j, int k, double Jx, double Jy, double Jz) {
  const mp_config *c = &s->cfg;
  const int med = in_medium(s, k);
  const double dt = c->dt;
  double *Ex = s->F[0], *Ey = s->F[1], *Ez = s->F[2];
  const double *Bx = s->F[3], *By = s->F[4], *Bz = s->F[5];
  const size_t g = IDX(s, i, j, k);
  const double ex = Ex[g], ey = Ey[g], ez = Ez[g];
  const double kappaEdx = s->kapE[0][i] * c->dx;
  const double kappaEdy = s->kapE[1][j] * c->dy;
  const double kappaEdz = s->kapE[2][k] * c->dz;
  /* a design cell scales every pole's coefficients by its Delta-eps factor
   * and has its own eps_infinity and chi factor (all 1 / eps elsewhere, which
   * leaves the arithmetic of the reference unchanged) */
  int dcell = 0;
  double eps_c = c->eps, sc = 1.0, uc = 1.0;
  if (s->design && i >= s->dbox.lo[0] && i <= s->dbox.hi[0] && j >= s->dbox.lo[1] && j <= s->dbox.hi[1] &&
      k >= s->dbox.lo[2] && k <= s->dbox.hi[2]) {
    const size_t di = box_index(&s->dbox, i, j, k);
    dcell = 1;
    eps_c = s->deps[di];
    sc = s->dscale[di];
    uc = s->dchi[di];
  }
  double Psix = 0, Psiy = 0, Psiz = 0;
  if (med) {
    for (int n = 0; n < 3; ++n) {
      const double complex D = dcell ? sc * (s->dchi0[n] - s->dxi0[n]) : s->dchi0[n] - s->dxi0[n];
      const double complex Xi = dcell ? sc * s->dxi0[n] : s->dxi0[n];
      double complex px = D * ex + CMPLX(s->psiR[n][0][g], s->psiI[n][0][g]);
      double complex py = D * ey + CMPLX(s->psiR[n][1][g], s->psiI[n][1][g]);
      double complex pz = D * ez + CMPLX(s->psiR[n][2][g], s->psiI[n][2][g]);
      Psix += creal(px);
      Psiy += creal(py);
      Psiz += creal(pz);
      px = Xi * ex + s->crec[n] * px;
      py = Xi * ey + s->crec[n] * py;
      pz = Xi * ez + s->crec[n] * pz;
      s->psiR[n][0][g] = creal(px); s->psiI[n][0][g] = cimag(px);
      s->psiR[n][1][g] = creal(py); s->psiI[n][1][g] = cimag(py);
      s->psiR[n][2][g] = creal(pz); s->psiI[n][2][g] = cimag(pz);
    }
  }
  const double eps = med ? eps_c : c->eps_bg;
  const double sumChi0 = med ? sc * s->sumChi0 : 0.0, sumXi0 = med ? sc * s->sumXi0 : 0.0;
  /* Sigma: zero each step (fdtd_plrc.t:129) plus the plasma density's term */
  const double sigma = 0.5 * (s->Sig ? s->Sig[g] : 0.0) * dt;
  const double cbx = (Bz[g] - Bz[IDX(s, i, j - 1, k)]) / kappaEdy - (By[g] - By[IDX(s, i, j, k - 1)]) / kappaEdz;
  const double cby = (Bx[g] - Bx[IDX(s, i, j, k - 1)]) / kappaEdz - (Bz[g] - Bz[IDX(s, i - 1, j, k)]) / kappaEdx;
  const double cbz = (By[g] - By[IDX(s, i - 1, j, k)]) / kappaEdx - (Bx[g] - Bx[IDX(s, i, j - 1, k)]) / kappaEdy;
  if (c->solver == MP_SOLVER_PLRC_LIN) {
    const double denom = dcell ? eps + sc * (s->sumChi0 - s->sumXi0) + sigma : eps + (sumChi0 - sumXi0) + sigma;
    const double numer = eps - sumXi0 - sigma;
    Ex[g] = (numer * ex + (dt * (cbx + Jx) + Psix)) / denom;
    Ey[g] = (numer * ey + (dt * (cby + Jy) + Psiy)) / denom;
    Ez[g] = (numer * ez + (dt * (cbz + Jz) + Psiz)) / denom;
    return;
  }
  /* nonlinear core */
  const double chi = med ? uc * c->chi : 0.0;
  const double denom = eps + sumChi0 - sumXi0 + sigma;
  const double numer = eps - sumXi0 - sigma;
  double E2 = ex * ex + ey * ey + ez * ez;
  const double cx = ((numer + chi * E2) * ex + dt * (cbx + Jx) + Psix) / denom;
  const double cy = ((numer + chi * E2) * ey + dt * (cby + Jy) + Psiy) / denom;
  const double cz = ((numer + chi * E2) * ez + dt * (cbz + Jz) + Psiz) / denom;
  double E = sqrt(E2);
  const double A = chi / denom;
  const double C = sqrt(cx * cx + cy * cy + cz * cz);
  if (C > 0) {
    double Eold;
    int it = 0;
    do {
      Eold = E;
      E2 = E * E;
      E = (2 * A * E2 * E + C) / (3 * A * E2 + 1);
    } while (fabs(E - Eold) > c->newton_tol && ++it < c->newton_max_iter);
    if (fabs(E - Eold) > c->newton_tol) s->newton_fail++;
    Ex[g] = E * cx / C;
    Ey[g] = E * cy / C;
    Ez[g] = E * cz / C;
  } else {
    Ex[g] = 0.0;
    Ey[g] = 0.0;
    Ez[g] = 0.0;
  }
}

/* FDTD_PLRCSolver::stepD (fdtd_plrc.t:171-237). */
static void plrc_step_d_all(mpo_sim *s) {
  if (has_currents(s)) sum_currents(s, 0);
  const int n[3] = {s->cfg.nx, s->cfg.ny, s->cfg.nz};
  for (int k = 1; k <= n[2]; ++k)
    for (int j = 1; j <= n[1]; ++j)
      for (int i = 1; i <= n[0]; ++i) {
        double jx = 0, jy = 0, jz = 0;
        if (has_currents(s)) {
          const size_t g = IDX(s, i, j, k);
          jx = s->Jt[0][g]; jy = s->Jt[1][g]; jz = s->Jt[2][g];
        }
        plrc_step_d(s, i, j, k, jx, jy, jz);
      }
  for (int c = 0; c < 3; ++c) exchange(s, s->F[c]);
}

/* FDTD_PLRCSolver::stepB (fdtd_plrc.t:312-339) with plrcStepB
 * (fdtd_plrc.cpp:263-293, identical in the nonlinear core :429-459). */
static void plrc_step_b_all(mpo_sim *s) {
  const mp_config *c = &s->cfg;
  if (has_mag_currents(s)) sum_currents(s, 1);
  const double dt = c->dt;
  const double *Ex = s->F[0], *Ey = s->F[1], *Ez = s->F[2];
  double *Bx = s->F[3], *By = s->F[4], *Bz = s->F[5];
  for (int k = 0; k <= c->nz; ++k)
    for (int j = 0; j <= c->ny; ++j)
      for (int i = 0; i <= c->nx; ++i) {
        const size_t g = IDX(s, i, j, k);
        double jx = 0, jy = 0, jz = 0;
        if (has_mag_currents(s)) { jx = s->Mt[0][g]; jy = s->Mt[1][g]; jz = s->Mt[2][g]; }
        const double kappaHdx = s->kapH[0][i] * c->dx;
        const double kappaHdy = s->kapH[1][j] * c->dy;
        const double kappaHdz = s->kapH[2][k] * c->dz;
        Bx[g] = Bx[g] + dt * ((Ey[IDX(s, i, j, k + 1)] - Ey[g]) / kappaHdz -
                              (Ez[IDX(s, i, j + 1, k)] - Ez[g]) / kappaHdy + jx);
        By[g] = By[g] + dt * ((Ez[IDX(s, i + 1, j, k)] - Ez[g]) / kappaHdx -
                              (Ex[IDX(s, i, j, k + 1)] - Ex[g]) / kappaHdz + jy);
        Bz[g] = Bz[g] + dt * ((Ex[IDX(s, i, j + 1, k)] - Ex[g]) / kappaHdy -
                              (Ey[IDX(s, i + 1, j, k)] - Ey[g]) / kappaHdx + jz);
      }
  for (int c3 = 3; c3 < 6; ++c3) exchange(s, s->F[c3]);
}

/* FDTD_PLRCSolver::stepScheme (fdtd_plrc.t:127-168). */
static void plrc_step(mpo_sim *s) {
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  if (s->Sig) memset(s->Sig, 0, n * sizeof(double));
  if (s->cfg.plasma) plasma_density_step(s);
  for (int l = 0; l < s->nE; ++l) cpml_e_step(s, &s->Elay[l]);
  if (s->cfg.plasma_current) plasma_current_step(s);
  plrc_step_d_all(s);
  for (int l = 0; l < s->nH; ++l) cpml_h_step(s, &s->Hlay[l]);
  plrc_step_b_all(s);
}

/* FDTD_Plain::stepD / stepB (fdtd_plain.cpp:37-120) and
 * FDTD_Nonlinear::stepD / stepB (fdtd_nl.cpp:38-143).  Both update E over
 * [1, n+1] per axis.  FDTD_Nonlinear divides by |D| without a guard
 * (fdtd_nl.cpp:94-96) and gives NaN where D = 0; here such a cell gets E = 0,
 * like the C > 0 guard of fdtd_plrc.cpp:406-425. */
static void simple_step(mpo_sim *s) {
  const mp_config *c = &s->cfg;
  const double dt = c->dt, dx = c->dx, dy = c->dy, dz = c->dz;
  double *Ex = s->F[0], *Ey = s->F[1], *Ez = s->F[2];
  double *Bx = s->F[3], *By = s->F[4], *Bz = s->F[5];
  for (int k = 1; k <= c->nz + 1; ++k)
    for (int j = 1; j <= c->ny + 1; ++j)
      for (int i = 1; i <= c->nx + 1; ++i) {
        const size_t g = IDX(s, i, j, k);
        const double cbx = (Bz[g] - Bz[IDX(s, i, j - 1, k)]) / dy - (By[g] - By[IDX(s, i, j, k - 1)]) / dz;
        const double cby = (Bx[g] - Bx[IDX(s, i, j, k - 1)]) / dz - (Bz[g] - Bz[IDX(s, i - 1, j, k)]) / dx;
        const double cbz = (By[g] - By[IDX(s, i - 1, j, k)]) / dx - (Bx[g] - Bx[IDX(s, i, j - 1, k)]) / dy;
        if (c->solver == MP_SOLVER_PLAIN) {
          Ex[g] = Ex[g] + dt * cbx;
          Ey[g] = Ey[g] + dt * cby;
          Ez[g] = Ez[g] + dt * cbz;
        } else {
          const double ex = Ex[g], ey = Ey[g], ez = Ez[g];
          double E2 = ex * ex + ey * ey + ez * ez;
          const double Dx = (c->eps + c->chi * E2) * ex + dt * cbx;
          const double Dy = (c->eps + c->chi * E2) * ey + dt * cby;
          const double Dz = (c->eps + c->chi * E2) * ez + dt * cbz;
          double E = sqrt(E2);
          const double D = sqrt(Dx * Dx + Dy * Dy + Dz * Dz);
          if (D > 0) {
            double Eold;
            int it = 0;
            do {
              Eold = E;
              E2 = E * E;
              E = (2 * c->chi * E2 * E + D) / (3 * c->chi * E2 + c->eps);
            } while (fabs(E - Eold) > c->newton_tol && ++it < c->newton_max_iter);
            if (fabs(E - Eold) > c->newton_tol) s->newton_fail++;
            Ex[g] = E * Dx / D;
            Ey[g] = E * Dy / D;
            Ez[g] = E * Dz / D;
          } else {
            Ex[g] = 0.0;
            Ey[g] = 0.0;
            Ez[g] = 0.0;
          }
        }
      }
  for (int f = 0; f < 3; ++f) exchange(s, s->F[f]);
  for (int k = 0; k <= c->nz; ++k)
    for (int j = 0; j <= c->ny; ++j)
      for (int i = 0; i <= c->nx; ++i) {
        const size_t g = IDX(s, i, j, k);
        Bx[g] = Bx[g] + dt * ((Ey[IDX(s, i, j, k + 1)] - Ey[g]) / dz - (Ez[IDX(s, i, j + 1, k)] - Ez[g]) / dy);
        By[g] = By[g] + dt * ((Ez[IDX(s, i + 1, j, k)] - Ez[g]) / dx - (Ex[IDX(s, i, j, k + 1)] - Ex[g]) / dz);
        Bz[g] = Bz[g] + dt * ((Ex[IDX(s, i, j + 1, k)] - Ex[g]) / dx - (Ey[IDX(s, i + 1, j, k)] - Ey[g]) / dx);
      }
  for (int f = 3; f < 6; ++f) exchange(s, s->F[f]);
}

/* ------------------------------------------------------------------------ */
/* Public oracle API (names prefixed mpo_; the CUDA library exports mp_*). */

static int fail(char *buf, const char *msg) {
  snprintf(buf, 256, "%s", msg);
  return MP_ERR_INVALID;
}

void mpo_destroy(mpo_sim *s);

int mpo_create(const mp_config *cfg, mpo_sim **out) {
  *out = NULL;
  g_create_err[0] = 0;
  if (cfg->abi_version != MP_ABI_VERSION) return fail(g_create_err, "abi_version mismatch");
  if (cfg->nx < 2 || cfg->ny < 2 || cfg->nz < 2) return fail(g_create_err, "grid must be at least 2 cells per axis");
  if (cfg->solver < 0 || cfg->solver > 3) return fail(g_create_err, "unknown solver");
  const int plrc = cfg->solver == MP_SOLVER_PLRC_LIN || cfg->solver == MP_SOLVER_PLRC_NONLIN;
  if (!plrc && (cfg->cpml != MP_CPML_NONE || cfg->n_sources > 0))
    return fail(g_create_err, "additional currents cannot be used with this field solver (fieldsolver.h:198-216)");
  if (plrc)
    for (int n = 0; n < 3; ++n)
    {
      if (cfg->poles[n].om2 == 0) return fail(g_create_err, "FDTD_PLRCSolver: Omega should not be zero! (fdtd_plrc.t:20-24)");
      if (!(cfg->poles[n].om2 > cfg->poles[n].delta * cfg->poles[n].delta))
        return fail(g_create_err, "Lorentz pole needs om2 > delta^2 (beta = sqrt(om2 - delta^2), fdtd_plrc.t:200)");
    }
  if (cfg->cpml != MP_CPML_NONE && cfg->cpml_d < 1) return fail(g_create_err, "cpml_d must be >= 1");

  mpo_sim *s = calloc(1, sizeof(mpo_sim));
  s->cfg = *cfg;
  s->NX = cfg->nx + 2; s->NY = cfg->ny + 2; s->NZ = cfg->nz + 2;
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  for (int f = 0; f < 6; ++f) s->F[f] = calloc(n, sizeof(double));
  if (plrc)
    for (int p = 0; p < 3; ++p)
      for (int c = 0; c < 3; ++c) {
        s->psiR[p][c] = calloc(n, sizeof(double));
        s->psiI[p][c] = calloc(n, sizeof(double));
      }
  const int nn[3] = {cfg->nx, cfg->ny, cfg->nz};
  for (int d = 0; d < 3; ++d) {
    s->kapE[d] = calloc((size_t)nn[d] + 2, sizeof(double));
    s->kapH[d] = calloc((size_t)nn[d] + 2, sizeof(double));
  }
  init_kappa(s);
  if (cfg->cpml == MP_CPML_ALL) {
    const int order[6] = {DIR_NORTH, DIR_SOUTH, DIR_EAST, DIR_WEST, DIR_UP, DIR_DOWN};
    for (int d = 0; d < 6; ++d) add_cpml_layer(s, order[d], 0);
    for (int d = 0; d < 6; ++d) add_cpml_layer(s, order[d], 1);
  } else if (cfg->cpml == MP_CPML_Z) {
    add_cpml_layer(s, DIR_UP, 0); add_cpml_layer(s, DIR_DOWN, 0);
    add_cpml_layer(s, DIR_UP, 1); add_cpml_layer(s, DIR_DOWN, 1);
  }
  oracle_faddeeva_init();
  for (int q = 0; q < cfg->n_sources; ++q) {
    const mp_source *p = &cfg->sources[q];
    src_state *st = &s->src[q];
    if (p->kind == MP_SOURCE_PLANE_WAVE || p->kind == MP_SOURCE_PLANE_GAUSS) {
      /* PlaneWaveSource::makeECurrent (sources.cpp:14-34) */
      const double *k = p->k, *H = p->H;
      double E[3] = {k[1] * H[2] - k[2] * H[1], k[2] * H[0] - k[0] * H[2], k[0] * H[1] - k[1] * H[0]};
      const double bmag = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
      const double factor = -bmag / sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
      for (int c = 0; c < 3; ++c) st->E[c] = E[c] * (factor / sqrt(p->eps));
      st->om = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]) / sqrt(p->eps);
    } else if (p->kind == MP_SOURCE_SHORT_PULSE || p->kind == MP_SOURCE_FOCUSED_PULSE) {
      /* ShortPulseInjectSourceFunc::setParam (shortpulseinject.cpp:56-113); the
       * focused pulse is defined as the same closed form (its reference plug-in,
       * focusedpulseinject.cpp, does not compile) */
      st->centre[0] = 0.5 * (double)(cfg->nx + 1);
      st->centre[1] = 0.5 * (double)(cfg->ny + 1);
      st->centre[2] = 0.5 * (double)(cfg->nz + 1);
      st->lightspeed = sqrt(1 / p->eps);
      st->ZRl = 0.5 * p->om0 * p->waist * p->waist / st->lightspeed;
      st->phase = 0.0; st->tshift = 0.0; st->zshift = 0.0;
      const double Exmax = creal(sp_efunc(st, p, 0, 0, 0, 0));
      st->amp = p->amp / Exmax;
      st->phase = 2 * M_PI * p->phase;
      st->tshift = p->t_shift;
      st->zshift = p->z_shift;
    } else if (p->kind == MP_SOURCE_GAUSS_BEAM) {
      if (p->t_size < 2 || p->eps <= 0) {
        snprintf(g_create_err, sizeof g_create_err, "gauss beam needs t_size >= 2 and eps > 0");
        mpo_destroy(s);
        return MP_ERR_INVALID;
      }
      gauss_init(&st->gs[0], p, cfg, 0);
      gauss_init(&st->gs[1], p, cfg, 1);
    } else {
      snprintf(g_create_err, sizeof g_create_err, "source kind %d is not available in the oracle", p->kind);
      mpo_destroy(s);
      return MP_ERR_UNSUPPORTED;
    }
    add_inc_layers(s, q);
  }
  if (cfg->plasma || cfg->plasma_current) {
    if (!plrc) {
      mpo_destroy(s);
      return fail(g_create_err, "the plasma plug-ins belong to the PLRC solvers");
    }
    s->rho = calloc(n, sizeof(double));
    s->Sig = calloc(n, sizeof(double));
    for (int c = 0; c < 3; ++c) s->PJ[c] = calloc(n, sizeof(double));
  }
  if (has_currents(s))
    for (int c = 0; c < 3; ++c) s->Jt[c] = calloc(n, sizeof(double));
  if (has_mag_currents(s))
    for (int c = 0; c < 3; ++c) s->Mt[c] = calloc(n, sizeof(double));
  if (plrc) plrc_coefficients(s);
  const int *db = cfg->design_box;
  if (db[0] <= db[1]) {
    if (!plrc) {
      mpo_destroy(s);
      return fail(g_create_err, "a design region needs a PLRC solver");
    }
    if (db[0] < 1 || db[1] > cfg->nx || db[2] < 1 || db[2] > db[3] || db[3] > cfg->ny || db[4] < 1 ||
        db[4] > db[5] || db[5] > cfg->nz || db[4] < cfg->medium_z0 || db[5] > cfg->medium_z1) {
      mpo_destroy(s);
      return fail(g_create_err, "design box outside the interior or the medium");
    }
    s->design = 1;
    for (int d = 0; d < 3; ++d) {
      s->dbox.lo[d] = db[2 * d];
      s->dbox.hi[d] = db[2 * d + 1];
      s->dbox.dims[d] = db[2 * d + 1] - db[2 * d] + 1;
    }
    const size_t nd = box_size(&s->dbox);
    s->deps = malloc(nd * sizeof(double));
    s->dscale = malloc(nd * sizeof(double));
    s->dchi = malloc(nd * sizeof(double));
    for (size_t q = 0; q < nd; ++q) {
      s->deps[q] = cfg->eps;
      s->dscale[q] = 1.0;
      s->dchi[q] = 1.0;
    }
  }
  *out = s;
  return MP_OK;
}

void mpo_destroy(mpo_sim *s) {
  if (!s) return;
  for (int f = 0; f < 6; ++f) free(s->F[f]);
  for (int p = 0; p < 3; ++p)
    for (int c = 0; c < 3; ++c) { free(s->psiR[p][c]); free(s->psiI[p][c]); }
  for (int c = 0; c < 3; ++c) { free(s->Jt[c]); free(s->Mt[c]); free(s->kapE[c]); free(s->kapH[c]); }
  for (int l = 0; l < s->nE; ++l) { free(s->Elay[l].psi[0]); free(s->Elay[l].psi[1]); free(s->Elay[l].b); free(s->Elay[l].c); }
  for (int l = 0; l < s->nH; ++l) { free(s->Hlay[l].psi[0]); free(s->Hlay[l].psi[1]); free(s->Hlay[l].b); free(s->Hlay[l].c); }
  for (int q = 0; q < MP_MAX_SOURCES; ++q)
    for (int h = 0; h < 2; ++h) { free(s->src[q].gs[h].F1); free(s->src[q].gs[h].F2); }
  free(s->deps);
  free(s->dscale);
  free(s->dchi);
  free(s->rho);
  free(s->Sig);
  for (int c = 0; c < 3; ++c) free(s->PJ[c]);
  free(s);
}

const char *mpo_create_error(void) { return g_create_err; }

static double *field_by_name(mpo_sim *s, const char *name) {
  static const char *fn[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};
  for (int f = 0; f < 6; ++f)
    if (!strcmp(name, fn[f])) return s->F[f];
  if ((name[0] == 'P' && name[1] == 's' && name[2] == 'i') && (name[3] == 'R' || name[3] == 'I') &&
      name[4] >= '1' && name[4] <= '3' && name[5] >= 'x' && name[5] <= 'z' && name[6] == 0) {
    const int p = name[4] - '1', c = name[5] - 'x';
    return name[3] == 'R' ? s->psiR[p][c] : s->psiI[p][c];
  }
  if (s->rho) {
    if (!strcmp(name, "PlasmaDensity")) return s->rho;
    if (!strcmp(name, "PlasmaJx")) return s->PJ[0];
    if (!strcmp(name, "PlasmaJy")) return s->PJ[1];
    if (!strcmp(name, "PlasmaJz")) return s->PJ[2];
  }
  return NULL;
}

size_t mpo_field_size(const mpo_sim *s) {
  return (size_t)(s->cfg.nz + 2) * s->cfg.ny * s->cfg.nx;
}

/* Plane layout <-> ghost layout.  Upload fills the x/y ghosts with their
 * periodic images (the state after Storage::applyBoundary). */
static double *design_by_name(mpo_sim *s, const char *name) {
  if (!s->design) return NULL;
  if (!strcmp(name, "DesignEps")) return s->deps;
  if (!strcmp(name, "DesignDepsScale")) return s->dscale;
  if (!strcmp(name, "DesignChiScale")) return s->dchi;
  return NULL;
}

int mpo_upload(mpo_sim *s, const char *name, const double *h, size_t count) {
  double *d = design_by_name(s, name);
  if (d) {
    if (count != box_size(&s->dbox)) return MP_ERR_INVALID;
    memcpy(d, h, count * sizeof(double));
    return MP_OK;
  }
  double *f = field_by_name(s, name);
  if (!f) return MP_ERR_NAME;
  if (count != mpo_field_size(s)) return MP_ERR_INVALID;
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  for (int k = 0; k < s->NZ; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        f[IDX(s, i, j, k)] = h[((size_t)k * ny + (j - 1)) * nx + (i - 1)];
  if (s->cfg.boundary == MP_BOUNDARY_PERIODIC) {
    /* the z ghosts of a periodic grid are images too */
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        f[IDX(s, i, j, 0)] = f[IDX(s, i, j, s->NZ - 2)];
        f[IDX(s, i, j, s->NZ - 1)] = f[IDX(s, i, j, 1)];
      }
  }
  /* x/y images */
  const int bsave = s->cfg.boundary;
  s->cfg.boundary = MP_BOUNDARY_XY_PERIODIC;
  exchange(s, f);
  s->cfg.boundary = bsave;
  return MP_OK;
}

int mpo_download(mpo_sim *s, const char *name, double *h, size_t count) {
  double *d = design_by_name(s, name);
  if (d) {
    if (count != box_size(&s->dbox)) return MP_ERR_INVALID;
    memcpy(h, d, count * sizeof(double));
    return MP_OK;
  }
  double *f = field_by_name(s, name);
  if (!f) return MP_ERR_NAME;
  if (count != mpo_field_size(s)) return MP_ERR_INVALID;
  const int nx = s->cfg.nx, ny = s->cfg.ny;
  for (int k = 0; k < s->NZ; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        h[((size_t)k * ny + (j - 1)) * nx + (i - 1)] = f[IDX(s, i, j, k)];
  return MP_OK;
}

/* Process::run (process.cpp:17-31): stepScheme with Process::time = n. */
int mpo_step(mpo_sim *s, int n_steps) {
  for (int t = 0; t < n_steps; ++t) {
    if (s->cfg.solver == MP_SOLVER_PLAIN || s->cfg.solver == MP_SOLVER_NL) simple_step(s);
    else plrc_step(s);
    s->time++;
  }
  return s->newton_fail ? MP_ERR_NEWTON : MP_OK;
}

long long mpo_get_time(const mpo_sim *s) { return s->time; }
void mpo_set_time(mpo_sim *s, long long t) { s->time = t; }

/* FieldEnergyDiag::calculate (fielddiag.cpp:255-286): sum over the interior of
 * E^2 + B^2 in MPulse's loop order (i slowest, k fastest), times dx dy dz. */
double mpo_field_energy(const mpo_sim *s) {
  double energy = 0;
  for (int i = 1; i <= s->cfg.nx; ++i)
    for (int j = 1; j <= s->cfg.ny; ++j)
      for (int k = 1; k <= s->cfg.nz; ++k) {
        const size_t g = IDX(s, i, j, k);
        const double ex = s->F[0][g], ey = s->F[1][g], ez = s->F[2][g];
        const double bx = s->F[3][g], by = s->F[4][g], bz = s->F[5][g];
        energy += ex * ex + ey * ey + ez * ez + bx * bx + by * by + bz * bz;
      }
  return energy * (s->cfg.dx * s->cfg.dy * s->cfg.dz);
}

/* The Faddeeva evaluator on its own, for tests against scipy / the reference. */
void mpo_faddeeva(const double *re, const double *im, double *wre, double *wim, size_t n) {
  oracle_faddeeva_init();
  for (size_t q = 0; q < n; ++q) {
    const double complex w = oracle_faddeeva(CMPLX(re[q], im[q]));
    wre[q] = creal(w);
    wim[q] = cimag(w);
  }
}

/* The incident field a source injects, for tests of the source kernels:
 * which = 0 -> getHField (E current), 1 -> getEField (H current). */
/* The short-pulse closed forms at one point, for the reference's own table of
 * them (test/testshortpulse.cpp: ShortPulseInjectSourceFunc::setParam(length,
 * width, om0, Shift = 0, Phase, amp, eps), then Efunc and Bfunc at (x, y, z, t),
 * printed without the amplitude): out = Re, Im of Efunc, Bfunc(bx = true),
 * Bfunc(bx = false). */
void mpo_short_pulse(double length, double width, double om0, double phase, double eps, double x, double y,
                     double z, double t, double out[6]) {
  oracle_faddeeva_init();
  src_state st;
  memset(&st, 0, sizeof st);
  mp_source p;
  memset(&p, 0, sizeof p);
  p.length = length;
  p.om0 = om0;
  st.lightspeed = sqrt(1 / eps);
  st.ZRl = 0.5 * om0 * width * width / st.lightspeed;
  st.phase = 2 * M_PI * phase;
  const double complex e = sp_efunc(&st, &p, x, y, z, t);
  const double complex bx = sp_bfunc(&st, &p, x, y, z, t, 1);
  const double complex by = sp_bfunc(&st, &p, x, y, z, t, 0);
  out[0] = creal(e); out[1] = cimag(e);
  out[2] = creal(bx); out[3] = cimag(bx);
  out[4] = creal(by); out[5] = cimag(by);
}

int mpo_source_field(mpo_sim *s, int src, int which, int i, int j, int l, long long time, double out[3]) {
  if (src < 0 || src >= s->cfg.n_sources) return MP_ERR_INVALID;
  if (s->cfg.sources[src].kind == MP_SOURCE_GAUSS_BEAM) gauss_set_time(&s->src[src].gs[which ? 1 : 0], time);
  if (which) src_efield(s, src, i, j, l, time, out);
  else src_hfield(s, src, i, j, l, time, out);
  return MP_OK;
}

/* ------------------------------------------------------------------------ */
/* Objectives of mp_objective (additions to MPulse, no reference counterpart):
 * J = dt sum_n sum_box |E|^2 or dt dx dy sum_n sum_plane (Ex By - Ey Bx),
 * after each step, accumulated in FP64 in x-fastest order. */
static double objective_term(const mpo_sim *s, const mp_adjoint_config *a) {
  const double *Ex = s->F[0], *Ey = s->F[1], *Ez = s->F[2], *Bx = s->F[3], *By = s->F[4];
  double acc = 0;
  if (a->kind == MP_OBJ_E2_BOX) {
    for (int k = a->box[4]; k <= a->box[5]; ++k)
      for (int j = a->box[2]; j <= a->box[3]; ++j)
        for (int i = a->box[0]; i <= a->box[1]; ++i) {
          const size_t g = IDX(s, i, j, k);
          acc += Ex[g] * Ex[g] + Ey[g] * Ey[g] + Ez[g] * Ez[g];
        }
    return s->cfg.dt * acc;
  }
  const int k = a->box[4];
  for (int j = a->box[2]; j <= a->box[3]; ++j)
    for (int i = a->box[0]; i <= a->box[1]; ++i) {
      const size_t g = IDX(s, i, j, k);
      acc += Ex[g] * By[g] - Ey[g] * Bx[g];
    }
  return s->cfg.dt * s->cfg.dx * s->cfg.dy * acc;
}

int mpo_objective(mpo_sim *s, const mp_adjoint_config *a, double *J) {
  if (a->kind != MP_OBJ_E2_BOX && a->kind != MP_OBJ_SZ_PLANE) return MP_ERR_INVALID;
  double acc = 0;
  for (int n = 0; n < a->steps; ++n) {
    const int rc = mpo_step(s, 1);
    if (rc != MP_OK) return rc;
    acc += objective_term(s, a);
  }
  *J = acc;
  return MP_OK;
}

/* Coefficient access for the test harness's adjoint restatement. */
int mpo_kappa(const mpo_sim *s, int isH, int dim, double *out, size_t n) {
  const int nn[3] = {s->cfg.nx, s->cfg.ny, s->cfg.nz};
  if (dim < 0 || dim > 2 || n != (size_t)nn[dim] + 2) return MP_ERR_INVALID;
  memcpy(out, isH ? s->kapH[dim] : s->kapE[dim], n * sizeof(double));
  return MP_OK;
}

int mpo_cpml_count(const mpo_sim *s, int isH) { return isH ? s->nH : s->nE; }

/* info: dir, dim, lo[3], hi[3]; b and c have hi[dim] - lo[dim] + 1 entries
 * (c not yet divided by delta).  With another n only info is filled. */
int mpo_cpml_layer(const mpo_sim *s, int isH, int l, int info[8], double *b, double *c, size_t n, double *delta) {
  const int cnt = isH ? s->nH : s->nE;
  if (l < 0 || l >= cnt) return MP_ERR_INVALID;
  const cpml_layer *L = isH ? &s->Hlay[l] : &s->Elay[l];
  const size_t len = (size_t)L->box.dims[L->dim];
  info[0] = L->dir;
  info[1] = L->dim;
  for (int d = 0; d < 3; ++d) {
    info[2 + d] = L->box.lo[d];
    info[5 + d] = L->box.hi[d];
  }
  if (n != len) return MP_ERR_INVALID; /* info is filled; n tells the caller's buffer length */
  memcpy(b, L->b, len * sizeof(double));
  memcpy(c, L->c, len * sizeof(double));
  *delta = L->delta;
  return MP_OK;
}

/* dchi0, dxi0, crec (re, im) for the 3 pole slots, then sumChi0, sumXi0. */
void mpo_plrc_coefficients(const mpo_sim *s, double out[20]) {
  for (int n = 0; n < 3; ++n) {
    out[2 * n] = creal(s->dchi0[n]);
    out[2 * n + 1] = cimag(s->dchi0[n]);
    out[6 + 2 * n] = creal(s->dxi0[n]);
    out[6 + 2 * n + 1] = cimag(s->dxi0[n]);
    out[12 + 2 * n] = creal(s->crec[n]);
    out[12 + 2 * n + 1] = cimag(s->crec[n]);
  }
  out[18] = s->sumChi0;
  out[19] = s->sumXi0;
}

/* ------------------------------------------------------------------------ */
/* Field initialisers over the whole grid, ghost cells included, as MPulse
 * writes them: GaussPulseInit::init (pulseinit.cpp:7-74),
 * PlaneGaussPulseInit::init (gaussinit.cpp:7-82), PlaneWaveInit::init
 * (waveinit.cpp:9-60). */
int mpo_initialize(mpo_sim *s, const mp_init *q) {
  const mp_config *c = &s->cfg;
  double *Ex = s->F[0], *Ey = s->F[1], *Ez = s->F[2], *Bx = s->F[3], *By = s->F[4], *Bz = s->F[5];
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  /* Globals::gridLow / gridHigh: 0 and n + 1 per axis */
  const double xh = 0.5 * (double)(c->nx + 1), yh = 0.5 * (double)(c->ny + 1), zh = 0.5 * (double)(c->nz + 1);
  if (q->kind == MP_INIT_PULSE) {
    const double ex = q->B[1], ey = -q->B[0], bx = q->B[0], by = q->B[1];
    const double dx2 = c->dx * c->dx, dy2 = c->dy * c->dy;
    const double nkz = c->dz * q->k[2];
    const double rr0 = q->r0 * q->r0, zz0 = q->z0 * q->z0;
    for (int i = 0; i < NX; ++i)
      for (int j = 0; j < NY; ++j) {
        const double iie = i - xh, jje = j - yh;
        const double rre = (iie * iie * dx2 + jje * jje * dy2) / rr0;
        const double iib = i + 0.5 - xh, jjb = j + 0.5 - yh;
        const double rrb = (iib * iib * dx2 + jjb * jjb * dy2) / rr0;
        for (int k = q->bound; k <= NZ - 1 - q->bound; ++k) {
          const double nze = k * c->dz - q->zc, nzb = (k + 0.5) * c->dz - q->zc;
          const double kze = k * nkz, kzb = (k + 0.5) * nkz;
          const double ampe = cos(kze - q->C * rre) * exp(-nze * nze / zz0 - rre);
          const double ampb = cos(kzb - q->C * rrb) * exp(-nzb * nzb / zz0 - rrb);
          const size_t g = IDX(s, i, j, k);
          Ex[g] = ex * ampe; Ey[g] = ey * ampe; Ez[g] = 0;
          Bx[g] = bx * ampb; By[g] = by * ampb; Bz[g] = 0;
        }
      }
    return MP_OK;
  }
  if (q->kind != MP_INIT_PLANE_GAUSS && q->kind != MP_INIT_WAVE) return MP_ERR_INVALID;
  const int kx = (int)q->k[0], ky = (int)q->k[1], kz = (int)q->k[2];
  const double bx = q->B[0], by = q->B[1], bz = q->B[2];
  double ex = ky * bz - kz * by, ey = kz * bx - kx * bz, ez = kx * by - ky * bx;
  const double bmag = sqrt(bx * bx + by * by + bz * bz);
  const double factor = -bmag / sqrt(ex * ex + ey * ey + ez * ez);
  if (q->kind == MP_INIT_PLANE_GAUSS) {
    ex *= factor; ey *= factor; ez *= factor;
    const double nkx = kx / (double)(c->nx), nky = ky / (double)(c->ny), nkz = kz / (double)(c->nz);
    for (int i = 0; i < NX; ++i)
      for (int j = 0; j < NY; ++j)
        for (int k = 12; k <= NZ - 1 - 12; ++k) {
          const double delta = 0.5;
          const double pose = (i - xh) * nkx + (j - yh) * nky + (k - zh) * nkz;
          const double posb = (i + delta - xh) * nkx + (j + delta - yh) * nky + (k + delta - zh) * nkz;
          const double ampe = exp(-pose * pose), ampb = exp(-posb * posb);
          const size_t g = IDX(s, i, j, k);
          Ex[g] = ex * ampe; Ey[g] = ey * ampe; Ez[g] = ez * ampe;
          Bx[g] = -bx * ampb; By[g] = -by * ampb; Bz[g] = -bz * ampb;
        }
    return MP_OK;
  }
  if (!(q->eps > 0)) return MP_ERR_INVALID;
  ex *= factor / sqrt(q->eps); ey *= factor / sqrt(q->eps); ez *= factor / sqrt(q->eps);
  const double nkx = 2 * M_PI * kx / (double)(c->nx), nky = 2 * M_PI * ky / (double)(c->ny),
               nkz = 2 * M_PI * kz / (double)(c->nz);
  for (int i = 0; i < NX; ++i)
    for (int j = 0; j < NY; ++j)
      for (int k = 0; k < NZ; ++k) {
        const int ii = i - 1, jj = j - 1, kk = k - 1;
        const size_t g = IDX(s, i, j, k);
        Ex[g] += ex * cos((ii + 0.5) * nkx + jj * nky + kk * nkz);
        Ey[g] += ey * cos(ii * nkx + (jj + 0.5) * nky + kk * nkz);
        Ez[g] += ez * cos(ii * nkx + jj * nky + (kk + 0.5) * nkz);
        Bx[g] += bx * cos(ii * nkx + (jj + 0.5) * nky + (kk + 0.5) * nkz);
        By[g] += by * cos((ii + 0.5) * nkx + jj * nky + (kk + 0.5) * nkz);
        Bz[g] += bz * cos((ii + 0.5) * nkx + (jj + 0.5) * nky + kk * nkz);
      }
  return MP_OK;
}

/* FollowMax::calculate (followmax.cpp:73-113) on the oracle grid: low = 0 and
 * high = n + 1 along dim. */
int mpo_follow_max(mpo_sim *s, const char *field, int dim, const int pos[3], int *ipos, double *position) {
  const double *G = field_by_name(s, field);
  if (!G || dim < 0 || dim > 2) return MP_ERR_INVALID;
  const int n = dim == 0 ? s->cfg.nx : dim == 1 ? s->cfg.ny : s->cfg.nz;
  const int low = 0, high = n + 1;
  int p[3] = {pos[0], pos[1], pos[2]};
  int ip = *ipos;
  double mid, left, right;
  int found;
  do {
    int pm = ip - 1, pp = ip + 1;
    if (pm <= low) pm = high - 1;
    if (pp >= high) pp = low + 1;
    p[dim] = ip; mid = G[IDX(s, p[0], p[1], p[2])];
    p[dim] = pm; left = G[IDX(s, p[0], p[1], p[2])];
    p[dim] = pp; right = G[IDX(s, p[0], p[1], p[2])];
    if (right > mid) { ip = pp; found = 0; }
    else if (left > mid) { ip = pm; found = 0; }
    else found = 1;
  } while (!found);
  *ipos = ip;
  *position = ip + (left - right) / (2 * (left - 2 * mid + right));
  return MP_OK;
}
