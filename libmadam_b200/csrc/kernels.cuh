// Types shared by the device code of the engine (engine.cu and the .inl
// files it includes) and the no-allocation entry point (noalloc.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace madam {

// Per-sample pointing record for polarised data: three weights and the
// compacted pixel number (bit pattern stored in .w).
__device__ __forceinline__ int point_pix(const float4 &p) { return __float_as_int(p.w); }

struct SampleMap {
  const long long *istart;  // first sample of each pointing period
  const int *kstart;        // first baseline of each pointing period
  int ninterval;
  long long nsamp;
  long noba_short;
  FastDiv fdn;              // division by the baseline length
};

struct MatrixRules {
  int pixmode;
  double pixlim;
  int allow_decoupling;
  int incomplete;
};

}  // namespace madam
