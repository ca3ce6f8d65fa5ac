// Test infrastructure only: direct-DFT implementation of the FFTW3 entry points
// declared in fftw3.h.  Plans remember their buffers like FFTW plans do.
#include "fftw3.h"
#include <cmath>
#include <cstdlib>
#include <vector>

struct mpb_fftw_plan_s {
  int n0, n1, sign;
  fftw_complex *in, *out;
};

void *fftw_malloc(std::size_t n) { return std::malloc(n); }
void fftw_free(void *p) { std::free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
  mpb_fftw_plan_s *p = new mpb_fftw_plan_s;
  p->n0 = 1; p->n1 = n; p->sign = sign; p->in = in; p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
  mpb_fftw_plan_s *p = new mpb_fftw_plan_s;
  p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
  return p;
}

static void dft_rows(int rows, int n, int stride, int dist, int sign,
                     const std::vector<double> &re, const std::vector<double> &im,
                     std::vector<double> &ore, std::vector<double> &oim) {
  const double tw = 2.0 * M_PI / double(n) * double(sign);
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < n; ++k) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; ++j) {
        const long long jk = (long long)j * k % n;
        const double c = std::cos(tw * double(jk)), s = std::sin(tw * double(jk));
        const int ix = r * dist + j * stride;
        sr += re[ix] * c - im[ix] * s;
        si += re[ix] * s + im[ix] * c;
      }
      ore[r * dist + k * stride] = sr;
      oim[r * dist + k * stride] = si;
    }
}

void fftw_execute(const fftw_plan p) {
  const int n = p->n0 * p->n1;
  std::vector<double> re(n), im(n), tre(n), tim(n);
  for (int i = 0; i < n; ++i) { re[i] = p->in[i][0]; im[i] = p->in[i][1]; }
  // transform along the last dimension, then along the first
  dft_rows(p->n0, p->n1, 1, p->n1, p->sign, re, im, tre, tim);
  if (p->n0 > 1) {
    dft_rows(p->n1, p->n0, p->n1, 1, p->sign, tre, tim, re, im);
  } else {
    re.swap(tre); im.swap(tim);
  }
  for (int i = 0; i < n; ++i) { p->out[i][0] = re[i]; p->out[i][1] = im[i]; }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
