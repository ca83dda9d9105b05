// Shared device helpers for the sm_100a destriping kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include <cstdint>
#include <string>

#include "params.h"

namespace madam {

#define MADAM_CUDA(call)                                                      \
  do {                                                                        \
    cudaError_t err__ = (call);                                               \
    if (err__ != cudaSuccess)                                                 \
      ::madam::fail(std::string("CUDA error: ") + cudaGetErrorString(err__) + \
                    " at " + __FILE__ + ":" + std::to_string(__LINE__));      \
  } while (0)

// Every kernel launch of the library goes through this macro so the number
// of launches inside a timed region can be reported.
extern std::atomic<unsigned long long> g_kernel_launches;
#define MADAM_LAUNCH(kernel, grid, block, smem, stream, ...)                  \
  do {                                                                        \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);               \
    ++::madam::g_kernel_launches;                                             \
    MADAM_CUDA(cudaGetLastError());                                           \
  } while (0)

// Unsigned 32-bit division by a run-time invariant divisor (Granlund &
// Montgomery 1994, "Division by invariant integers using multiplication"):
// q = (t + ((n - t) >> s1)) >> s2 with t = umulhi(m, n).
struct FastDiv {
  uint32_t d = 1, m = 0, s1 = 0, s2 = 0;
  FastDiv() = default;
  explicit FastDiv(uint32_t div) : d(div) {
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < div) ++l;
    uint64_t p = (((1ull << l) - div) << 32) / div + 1;  // fits 32 bits
    m = (uint32_t)p;
    s1 = l < 1 ? l : 1;
    s2 = l > 0 ? l - 1 : 0;
  }
  __host__ __device__ inline uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
    uint32_t t = __umulhi(m, n);
#else
    uint32_t t = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
    return (t + ((n - t) >> s1)) >> s2;
  }
};

// Run of consecutive samples of one detector that stay inside one scatter
// tile (a power-of-two block of compacted pixels) and one pointing period.
struct Run {
  uint32_t s_lo;      // global sample index (det * nsamp + s), low 32 bits
  uint32_t hi_len;    // bits 0..23 run length, bits 24..31 sample index high
  int32_t kbase;      // det * noba_short + first baseline of the period
  uint32_t offiv;     // offset of the first sample inside the period
};

__device__ __forceinline__ uint64_t run_start(const Run &r) {
  return ((uint64_t)(r.hi_len >> 24) << 32) | r.s_lo;
}
__device__ __forceinline__ uint32_t run_len(const Run &r) { return r.hi_len & 0xFFFFFFu; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV doubles; result valid in thread 0.  blockDim.x must be
// a multiple of 32 and at most 1024.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) red[i][wid] = v[i];
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nw ? red[i][lane] : 0.0;
      v[i] = warp_sum(x);
    }
  }
}

}  // namespace madam
