// mp_gauss.h - gauss_inject on the device: GaussInjectSourceFunc
// (gaussinject.cpp:56-482) with its angular-spectrum precompute.
//
// The reference evaluates the beam's injection-plane fields for a block of Nt
// steps at a time (Nt = 2^round(log2(nz + 1)), gaussinject.cpp:134): for every
// transverse wave vector (kx, ky) and frequency om of a SizeX x SizeY x SizeT
// box it builds the spectrum A (fillEx / fillEy / fillBx, :329-482),
// transforms it backward over om keeping the block's Nt times (transformT,
// :257-278), then forward over ky and kx (transformY / transformX, :280-327).
// Here the spectrum is written by a kernel, the three transforms are batched
// cuFFT Z2Z plans (FP64, the same unnormalised sign conventions as FFTW) and
// the index shuffles between them are kernels; the result is kept as three
// t-major planes [Nt][ny][nx] (Bx for the E current; Ex, Ey for the H current)
// that the per-step source kernel reads.  The precompute runs once per block,
// between the step kernels of the same stream.
#ifndef MPULSE_B200_GAUSS_H
#define MPULSE_B200_GAUSS_H

#include "mpulse_b200.h"

#include <cuda_runtime.h>
#include <cufft.h>

#include <string>

namespace mpb {

struct GaussBeam {
  // setParam (gaussinject.cpp:56-111)
  int SizeT = 0, SizeX = 0, SizeY = 0, SizeTH = 0, SizeXH = 0, SizeYH = 0, Nt = 1, toff = 0;
  int nx = 0, ny = 0;
  double length = 0, width = 0, k0 = 0, Shift = 0, Time = 0, amp = 0, eps = 1;
  double DX = 0, DY = 0, DT = 0, BoxX = 0, BoxY = 0, BoxT = 0;
  long long nblocks = 0;    // blocks before the source switches off: ceil(SizeT / Nt)
  long long computed = -1;  // block held in bx / ex / ey
  // the held block, interior columns, t-major [Nt][ny][nx]
  double *bx = nullptr;  // E current (getHField): Bx
  double *ex = nullptr;  // H current (getEField): Ex
  double *ey = nullptr;  //                       Ey
  // scratch: a slab of x rows of the spectrum, then the (t, y) and (t, x) stages
  double2 *spec = nullptr;
  double2 *ybuf = nullptr;
  double2 *xbuf = nullptr;
  int slab_rows = 0;
  cufftHandle plan_t = 0, plan_t_last = 0, plan_y = 0, plan_x = 0;
  bool have_t = false, have_t_last = false, have_y = false, have_x = false;
};

// Sets up the parameters, device buffers and FFT plans.  Returns an mp_status
// and, on failure, a message in *err.
int gauss_create(GaussBeam &g, const mp_source &q, const mp_config &c, std::string *err);
void gauss_destroy(GaussBeam &g);

// State of the source at `time`: active or not and the first later time at
// which that state (or the held block) changes.  When active, the block that
// holds `time` is computed on `st` if it is not the one held; *launches counts
// the kernels of this library launched for it.
int gauss_prepare(GaussBeam &g, long long time, cudaStream_t st, bool *active, long long *block_toff,
                  long long *until, long long *launches, std::string *err);

}  // namespace mpb

#endif
