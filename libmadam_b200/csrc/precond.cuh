// Launch wrappers of the band preconditioner kernels (precond.cu).
#pragma once

#include <cuda_runtime.h>

namespace madam {

struct BandSeg;

void band_factor(cudaStream_t st, const BandSeg *segs, int nseg, const int *spec,
                 const double *invcov, long long nof, const double *nna, double *band,
                 int *status);
void band_solve(cudaStream_t st, const BandSeg *segs, int nseg, const double *band,
                const double *r, double *z);

}  // namespace madam
