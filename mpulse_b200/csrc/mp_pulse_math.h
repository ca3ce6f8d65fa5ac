// mp_pulse_math.h - FP64 complex arithmetic, the Faddeeva function and the
// paraxial short-pulse fields, usable on host and device.
//
// The short-pulse fields are the closed forms of ShortPulseInjectSourceFunc::
// Efunc / Bfunc (shortpulsefunctions.cpp:28-226): a focused Gaussian pulse of
// duration parameter T and waist w0 with complex beam parameter
// q = z + i ZRl, ZRl = om0 w0^2 / (2 c).  They need the Faddeeva function
// w(z) = exp(-z^2) erfc(-iz) for Im z >= 0.  MPulse uses the Matpack routine
// (specfunc.cpp:57-157), whose licence forbids redistribution; this file uses
// J.A.C. Weideman's rational expansion ("Computation of the complex error
// function", SIAM J. Numer. Anal. 31 (1994) 1497-1518) with N = 40 terms,
// relative error about 1e-14 in the upper half plane.  The N coefficients are
// computed once on the host (faddeeva_coefficients) and passed in.
#ifndef MPB_MP_PULSE_MATH_H
#define MPB_MP_PULSE_MATH_H

#include <cmath>

#ifdef __CUDACC__
#define MPB_HD __host__ __device__ __forceinline__
#else
#define MPB_HD inline
#endif

namespace mpb {

static const int kFaddeevaTerms = 40;

struct cd {
  double re, im;
  MPB_HD cd() : re(0), im(0) {}
  MPB_HD cd(double r) : re(r), im(0) {}
  MPB_HD cd(double r, double i) : re(r), im(i) {}
};

MPB_HD cd operator+(cd a, cd b) { return cd(a.re + b.re, a.im + b.im); }
MPB_HD cd operator-(cd a, cd b) { return cd(a.re - b.re, a.im - b.im); }
MPB_HD cd operator-(cd a) { return cd(-a.re, -a.im); }
MPB_HD cd operator*(cd a, cd b) { return cd(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
MPB_HD cd operator*(cd a, double s) { return cd(a.re * s, a.im * s); }
MPB_HD cd operator*(double s, cd a) { return cd(s * a.re, s * a.im); }
MPB_HD cd operator+(cd a, double s) { return cd(a.re + s, a.im); }
MPB_HD cd operator+(double s, cd a) { return cd(s + a.re, a.im); }
MPB_HD cd operator-(cd a, double s) { return cd(a.re - s, a.im); }
MPB_HD cd operator-(double s, cd a) { return cd(s - a.re, -a.im); }
// Smith's algorithm for complex division.
MPB_HD cd operator/(cd a, cd b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, den = b.re + b.im * r;
    return cd((a.re + a.im * r) / den, (a.im - a.re * r) / den);
  }
  const double r = b.re / b.im, den = b.re * r + b.im;
  return cd((a.re * r + a.im) / den, (a.im * r - a.re) / den);
}
MPB_HD cd operator/(cd a, double s) { return cd(a.re / s, a.im / s); }
MPB_HD cd operator/(double s, cd b) { return cd(s) / b; }
MPB_HD cd cexp_(cd z) {
  const double e = exp(z.re);
  return cd(e * cos(z.im), e * sin(z.im));
}
MPB_HD cd I_() { return cd(0.0, 1.0); }

// w(z) for Im z >= 0 by Weideman's expansion; coef[0] is the highest power:
// with r = 1 / (L - iz) and Z = (L + iz) r, w = 2 p(Z) r^2 + r / sqrt(pi).
// Re(L - iz) = L + Im z >= L, so r = conj(L - iz) / |L - iz|^2 needs one real
// division and cannot overflow or underflow for any finite z of interest.
MPB_HD cd faddeeva(cd z, const double *coef, double L) {
  const cd iz(-z.im, z.re);
  const cd Lmz = cd(L) - iz;
  const double den = 1.0 / (Lmz.re * Lmz.re + Lmz.im * Lmz.im);
  const cd r(Lmz.re * den, -Lmz.im * den);
  const cd Z = (cd(L) + iz) * r;
  cd p(coef[0]);
  for (int n = 1; n < kFaddeevaTerms; ++n) p = p * Z + coef[n];
  return (2.0 * p * r + (1.0 / sqrt(M_PI))) * r;
}

// Coefficients a_N .. a_1 (highest power first) and L = sqrt(N / sqrt 2):
// a_n = (1 / 2M) sum_m f(t_m) cos(2 pi n m / 2M), M = 2N,
// f(t) = exp(-t^2) (L^2 + t^2), t_m = L tan(theta_m / 2), theta_m = m pi / M.
inline void faddeeva_coefficients(double *coef, double *L_out) {
  const int N = kFaddeevaTerms, M = 2 * N, M2 = 2 * M;
  const double L = sqrt(N / sqrt(2.0));
  double f[4 * kFaddeevaTerms];
  for (int n = 0; n < M2; ++n) {
    const int k = n <= M ? n : n - M2;
    if (k == -M || k == M) { f[n] = 0.0; continue; }
    const double t = L * tan(0.5 * k * M_PI / M);
    f[n] = exp(-t * t) * (L * L + t * t);
  }
  for (int n = 1; n <= N; ++n) {
    double s = 0.0;
    for (int m = 0; m < M2; ++m) s += f[m] * cos(2.0 * M_PI * (double)n * m / M2);
    coef[N - n] = s / M2;
  }
  *L_out = L;
}

struct ShortPulse {
  double c, ZRl, phase, T, om0;
  const double *coef;
  double L;
  // constants of the pulse, set by short_pulse_constants: exp(2 i phase),
  // exp(-i phase), exp(-tb^2) with tb = om0 T / 2
  cd eiphi, emip;
  double g;
};

// The pulse's constants (once per source, not per point).
MPB_HD void short_pulse_constants(ShortPulse &sp) {
  const double tb = 0.5 * sp.om0 * sp.T;
  sp.eiphi = cexp_(cd(0.0, 2.0 * sp.phase));
  sp.emip = cexp_(cd(0.0, -sp.phase));
  sp.g = exp(-tb * tb);
}

// Efunc (shortpulsefunctions.cpp:28-94).
MPB_HD cd short_pulse_e(const ShortPulse &sp, double x, double y, double z, double t) {
  const cd I = I_();
  const double c = sp.c, T = sp.T, T2 = T * T, T4 = T2 * T2;
  const double tb = 0.5 * sp.om0 * T;
  const double r2 = x * x + y * y;
  const cd q(z, sp.ZRl);
  const cd rT = sp.ZRl / q;
  const cd rpiT = sqrt(M_PI) * rT;
  const cd rpT = -sp.ZRl / (q * q);
  const cd eiphi = sp.eiphi;
  const cd tpT = (t - z / c) - r2 / (2. * c * q);
  const cd tpT2 = tpT * tpT;
  const cd tpzT = (-1 / c) - r2 / (2. * c * q * q);
  cd an = -I * tb + tpT / T;
  cd ap = I * tb + tpT / T;
  const cd A = sp.emip / (rpiT * T4);
  const cd B = rT * T * (I * (1.0 + eiphi) * rpT * T2 -
                         rT * (T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) + 2.0 * I * (1.0 + eiphi) * tpT) * tpzT);
  cd C = I * eiphi * rpiT * (T * tb + I * tpT) * (rpT * T2 + 2.0 * I * rT * T * tb * tpzT - 2.0 * rT * tpT * tpzT);
  cd D = rpiT * (T * tb - I * tpT) * (I * rpT * T2 + 2.0 * rT * (T * tb - I * tpT) * tpzT);
  cd S(0.0);
  if (an.im < 0) {
    S = S + 2.0 * A * C * cexp_(2.0 * I * tpT * tb / T - tpT2 / T2);
    an = -an;
    C = -C;
  }
  if (ap.im < 0) {
    S = S + 2.0 * A * D * cexp_(-2.0 * I * tpT * tb / T - tpT2 / T2);
    ap = -ap;
    D = -D;
  }
  const cd Ef = S + A * sp.g * (B + C * faddeeva(an, sp.coef, sp.L) - D * faddeeva(ap, sp.coef, sp.L));
  return -I * Ef;
}

// Bfunc (shortpulsefunctions.cpp:96-226) with YComp = 0: bx -> i A-terms,
// by -> i (D-terms - B-terms).
MPB_HD cd short_pulse_b(const ShortPulse &sp, double x, double y, double z, double t, bool bx) {
  const cd I = I_();
  const double c = sp.c, T = sp.T, T2 = T * T, T4 = T2 * T2;
  const double tb = 0.5 * sp.om0 * T;
  const double r2 = x * x + y * y;
  const cd q(z, sp.ZRl);
  const cd rT = sp.ZRl / q;
  const cd rT2 = rT * rT;
  const cd rT4T = rT * T4;
  const cd rpiT = sqrt(M_PI) * rT;
  const cd rpT = -sp.ZRl / (q * q);
  const cd rppT = 2. * sp.ZRl / (q * q * q);
  const cd eiphi = sp.eiphi;
  const cd tpT = (t - z / c) - r2 / (2. * c * q);
  const cd tpT2 = tpT * tpT;
  const cd tpzT = (-1 / c) + r2 / (2. * c * q * q);
  const cd tpzT2 = tpzT * tpzT;
  const cd tpxT = -x / (c * q);
  const cd tpyT = -y / (c * q);
  const cd tpxxT = -1. / (c * q);
  const cd tpzzT = -r2 / (c * q * q * q);
  const cd tpxT2 = tpxT * tpxT;
  const cd aip = T * tb + I * tpT;
  const cd ain = T * tb - I * tpT;
  const cd aip2 = aip * aip;
  const cd ain2 = ain * ain;
  cd an = -I * tb + tpT / T;
  cd ap = I * tb + tpT / T;
  const cd common = T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) + 2.0 * I * (1.0 + eiphi) * tpT;
  const cd eA = sp.emip / (sqrt(M_PI) * T4);
  const double g = sp.g;
  cd e1(0.0), e2(0.0);
  const bool neg_n = an.im < 0, neg_p = ap.im < 0;
  if (neg_n) { e1 = cexp_(2.0 * I * tpT * tb / T - tpT2 / T2); an = -an; }
  if (neg_p) { e2 = cexp_(-2.0 * I * tpT * tb / T - tpT2 / T2); ap = -ap; }
  const cd wn = faddeeva(an, sp.coef, sp.L);
  const cd wp = faddeeva(ap, sp.coef, sp.L);
  if (bx) {
    const cd AB = -tpxT * tpyT * rT * T * common;
    cd AC = -tpxT * tpyT * 2.0 * eiphi * rpiT * aip2;
    cd AD = -tpxT * tpyT * 2.0 * rpiT * ain2;
    cd AS(0.0);
    if (neg_n) { AS = AS + 2.0 * eA * AC * e1; AC = -AC; }
    if (neg_p) { AS = AS + 2.0 * eA * AD * e2; AD = -AD; }
    return I * (AS + eA * g * (AB + AC * wn - AD * wp));
  }
  const cd BB = -tpxT2 * (rT * T * common) + I * T2 * tpxxT * (1.0 + eiphi) * rT * T;
  cd BC = -tpxT2 * 2.0 * eiphi * rpiT * aip2 + I * T2 * tpxxT * eiphi * rpiT * aip;
  cd BD = -tpxT2 * 2.0 * rpiT * ain2 + I * T2 * tpxxT * rpiT * (-(T * tb) + I * tpT);
  cd BS(0.0);
  const cd eD = sp.emip / (2. * sqrt(M_PI) * T4);
  const cd DB = 2.0 * T * (2.0 * I * (1.0 + eiphi) * rpT * T2 * tpzT -
                           rT * (T * (-I - 2 * tb + eiphi * (-I + 2 * tb)) * tpzT2 +
                                 I * (1.0 + eiphi) * (2.0 * tpT * tpzT2 - T2 * tpzzT)));
  cd DC = (eiphi * rpiT *
           (rppT * rT4T + 2.0 * I * rT * aip *
                              (2.0 * rpT * T2 * tpzT + rT * (2.0 * I * T * tb * tpzT2 - 2.0 * tpT * tpzT2 + T2 * tpzzT)))) /
          rT2;
  cd DD = (rpiT * (rppT * rT4T - 2.0 * rT * ain *
                                     (2.0 * I * rpT * T2 * tpzT +
                                      rT * (2.0 * T * tb * tpzT2 - 2.0 * I * tpT * tpzT2 + I * T2 * tpzzT)))) /
          rT2;
  cd DS(0.0);
  if (neg_n) { BS = BS + 2.0 * eA * BC * e1; DS = DS + 2.0 * eD * DC * e1; BC = -BC; DC = -DC; }
  if (neg_p) { BS = BS + 2.0 * eA * BD * e2; DS = DS + 2.0 * eD * DD * e2; BD = -BD; DD = -DD; }
  const cd fB = BS + eA * g * (BB + BC * wn - BD * wp);
  const cd fD = DS + eD * g * (DB + DC * wn - DD * wp);
  return I * (fD - fB);
}

}  // namespace mpb

#endif
