// Test infrastructure only: declarations of the FFTW3 subset used by MPulse's
// gaussinject.cpp:227-327 (FFTW3 is not installed; version unpinned upstream).
// fftw_shim.cpp implements them as a direct O(n^2) DFT with FFTW's sign and
// normalisation conventions: forward uses exp(-2 pi i jk/n), backward
// exp(+2 pi i jk/n), neither is scaled.
#ifndef MPB_REFSHIM_FFTW3_H
#define MPB_REFSHIM_FFTW3_H
#include <cstddef>
typedef double fftw_complex[2];
typedef struct mpb_fftw_plan_s *fftw_plan;
enum { FFTW_FORWARD = -1, FFTW_BACKWARD = 1 };
enum { FFTW_ESTIMATE = 64 };
void *fftw_malloc(std::size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#endif
