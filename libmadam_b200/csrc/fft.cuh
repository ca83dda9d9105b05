// Batched FFT convolution of baseline segments with real spectra.
//
// Replaces convolve_interval / convolve_pp (noise_routines.f90:816-913) and
// the FFTW r2c/c2r pair they call (fourier_fftw_2003.f90:101-123):
//   y = irfft_nof( rfft_nof( pad(x - mean x) ) * H ) [0:n_out],  y -= mean y
// where H is a real spectrum of nof/2+1 values (fcov or fprecond).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace madam {

struct ConvSeg;

struct FFTPlan {
  long nof = 0;     // real transform length
  long N = 0;       // complex length nof/2
  int R = 0, C = 0; // four-step split N = R * C (0 for the single-CTA path)
  int G = 0;        // columns per CTA in the column passes
  double *work = nullptr;   // nseg_max * N complex values
  double *table = nullptr;  // 2N complex twiddles exp(-2 pi i m / (2N))
  double *means = nullptr;  // nseg_max
  long nseg_max = 0;
  explicit FFTPlan(long nof_);
  ~FFTPlan();
  void reserve(long nseg);
  // segs: device table of nseg entries; spectra: [nspec][nof/2+1] (device)
  void convolve(cudaStream_t st, const ConvSeg *segs, long nseg,
                const double *spectra, const double *x, double *y);
};

}  // namespace madam
