// Band preconditioner of the baseline solve (sm_100a).
//
// construct_preconditioner (noise_routines.f90:920-1153) factors, for every
// trimmed segment, the band matrix Toeplitz(invcov[0:nband]) + diag(nna) with
// DPBTRF('L'); preconditioning_band (1159-1256) applies it with DPBTRS.  The
// factor is computed here with the unblocked column algorithm of DPBTF2 and
// applied with the two banded triangular solves of DPBTRS.
#include "engine.h"
#include "precond.cuh"

namespace madam {
namespace {

// One thread per segment: factor in place.  ab column j holds A(j+d, j),
// d < nband.  status[s] = 0 or the 1-based failing column.
__global__ void k_band_factor(const BandSeg *segs, int nseg, const int *spec,
                              const double *invcov, long long nof, const double *nna,
                              double *band, int *status) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const BandSeg g = segs[s];
  const int nb = g.nband, kd = nb - 1;
  const double *ic = invcov + (long long)spec[s] * nof;
  double *ab = band + g.l_off;
  for (long long j = 0; j < g.n; ++j) {
    for (int d = 0; d < nb; ++d) ab[j * nb + d] = ic[d];
    ab[j * nb] += nna[g.k0 + j];
  }
  int info = 0;
  for (long long j = 0; j < g.n; ++j) {
    double ajj = ab[j * nb];
    if (!(ajj > 0)) {
      info = (int)min(j + 1, 2147483647LL);
      break;
    }
    ajj = sqrt(ajj);
    ab[j * nb] = ajj;
    const int kn = (int)min((long long)kd, g.n - j - 1);
    if (kn > 0) {
      const double rinv = 1.0 / ajj;
      for (int i = 1; i <= kn; ++i) ab[j * nb + i] *= rinv;
      for (int c = 0; c < kn; ++c) {
        const double xc = ab[j * nb + 1 + c];
        double *col = ab + (j + 1 + c) * nb;
        for (int r = c; r < kn; ++r) col[r - c] -= ab[j * nb + 1 + r] * xc;
      }
    }
  }
  status[s] = info;
}

// One thread per segment: z = (L L^T)^-1 r on the segment.
__global__ void k_band_solve(const BandSeg *segs, int nseg, const double *band,
                             const double *r, double *z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const BandSeg g = segs[s];
  const int nb = g.nband, kd = nb - 1;
  const double *ab = band + g.l_off;
  const double *rs = r + g.k0;
  double *b = z + g.k0;
  for (long long j = 0; j < g.n; ++j) b[j] = rs[j];
  for (long long j = 0; j < g.n; ++j) {
    const double bj = b[j] / ab[j * nb];
    b[j] = bj;
    const int kn = (int)min((long long)kd, g.n - j - 1);
    for (int i = 1; i <= kn; ++i) b[j + i] -= bj * ab[j * nb + i];
  }
  for (long long j = g.n - 1; j >= 0; --j) {
    double t = b[j];
    const int kn = (int)min((long long)kd, g.n - j - 1);
    for (int i = 1; i <= kn; ++i) t -= ab[j * nb + i] * b[j + i];
    b[j] = t / ab[j * nb];
  }
}

}  // namespace

void band_factor(cudaStream_t st, const BandSeg *segs, int nseg, const int *spec,
                 const double *invcov, long long nof, const double *nna, double *band,
                 int *status) {
  if (nseg == 0) return;
  MADAM_LAUNCH(k_band_factor, (nseg + 63) / 64, 64, 0, st, segs, nseg, spec, invcov, nof, nna,
               band, status);
}

void band_solve(cudaStream_t st, const BandSeg *segs, int nseg, const double *band,
                const double *r, double *z) {
  if (nseg == 0) return;
  MADAM_LAUNCH(k_band_solve, (nseg + 63) / 64, 64, 0, st, segs, nseg, band, r, z);
}

}  // namespace madam
