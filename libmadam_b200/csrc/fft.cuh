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
  // Four-step tables laid out so that a row of the split reads them
  // contiguously: twrow[k1][n2] = exp(-2 pi i n2 k1 / N) (the inter-pass
  // twiddles), wrow[k1][k2] = exp(-i pi (k1 + R k2) / N) (the real split),
  // and the sub-transform twiddles exp(-2 pi i q / L) for L = R and C.  The
  // values are those of `table`.
  double *twrow = nullptr, *wrow = nullptr, *twr = nullptr, *twc = nullptr;
  // Spectra copied into the rows of the split: rows[s][k1][k2] =
  // spectra[s][k1 + R k2], one copy per spectra array, kept while the plan
  // lives (forget_spectra() drops them when an array is rewritten).
  struct RowSpectra {
    const double *src;
    long nspec;
    double *rows;
  };
  RowSpectra cache[4] = {};
  explicit FFTPlan(long nof_);
  ~FFTPlan();
  void reserve(long nseg);
  void forget_spectra();
  // segs: device table of nseg entries; spectra: [nspec][nof/2+1] (device)
  void convolve(cudaStream_t st, const ConvSeg *segs, long nseg, const double *spectra,
                long nspec, const double *x, double *y);

 private:
  void make_tables(cudaStream_t st);
  const double *row_spectra(cudaStream_t st, const double *spectra, long nspec);
};

}  // namespace madam
