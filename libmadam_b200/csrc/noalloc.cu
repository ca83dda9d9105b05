// Hit counts and inverse pixel matrices of a device-resident pointing,
// computed without allocating device memory
// (madam_b200_pixel_matrices_noalloc).
//
// This is the pixel-matrix part of the setup scatter of engine.cu
// (k_setup_scatter: pixel_matrix, smadam_routines.f90:111-246, and
// count_hits, smadam_routines.f90:349-422) followed by the map-level
// inversion (invert_pixelmatrix_map, map_routines.f90:218-321).  The
// destripe path accumulates into allocated, tile-bucketed buffers; here the
// accumulators are one fixed device array of this file, so a call launches
// three kernels and touches no allocator: no cudaMalloc / cudaFree, no
// CUB temporary storage, no torch.
//
// Scratch.  g_pixmat_scratch holds kNoAllocMaxPix pixels x 7 doubles (the
// six upper-triangle entries of the 3 x 3 matrix, or one entry for
// nnz = 1, and the hit count): 2.75 MB.  Its address is looked up once per
// device, with that device current, by cudaGetSymbolAddress on the first
// call made on that device, which also loads the code of all the kernels
// below (cudaFuncGetAttributes); that first call should therefore come
// before any stream capture.  Later calls load and allocate nothing.  Every call clears the npix x 7 entries it uses
// before accumulating, so nothing needs to be zero beforehand.  There is one
// scratch array per device: calls that overlap on one device (two streams,
// two threads) race on it and give wrong results.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "kernels.cuh"
#include "pixmat.cuh"

namespace madam {
namespace {

constexpr long kNoAllocMaxPix = 49152;  // 12 * 64^2: nside_map <= 64
constexpr int kScratchStride = 7;       // 6 matrix entries + hits
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_pixmat_scratch[kNoAllocMaxPix * kScratchStride];

std::atomic<double *> g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mutex;

__global__ void k_na_clear(double *s, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    s[e] = 0.0;
}

// Per sample: the weights rounded to float (the precision of the destripe
// path's device pointing) times sqrt(detector weight), as in
// k_setup_scatter; flagged samples (negative pixel), samples outside the map
// and samples of zero-weight detectors are skipped.
template <int NNZ>
__global__ void k_na_accum(const long long *pix, const double *pw, const double *detw,
                           long long nsamp, long long ntot, long long npix, double *s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntot;
       i += (long long)gridDim.x * blockDim.x) {
    const long long px = pix[i];
    if (px < 0 || px >= npix) continue;
    const double dw = detw[i / nsamp];
    if (dw == 0) continue;
    double *c = s + px * kScratchStride;
    if (NNZ == 3) {
      const double sq = sqrt(dw);
      const double w0 = (double)(float)pw[3 * i] * sq;
      const double w1 = (double)(float)pw[3 * i + 1] * sq;
      const double w2 = (double)(float)pw[3 * i + 2] * sq;
      atomicAdd(c + 0, w0 * w0);
      atomicAdd(c + 1, w0 * w1);
      atomicAdd(c + 2, w0 * w2);
      atomicAdd(c + 3, w1 * w1);
      atomicAdd(c + 4, w1 * w2);
      atomicAdd(c + 5, w2 * w2);
    } else {
      atomicAdd(c, dw);
    }
    atomicAdd(c + 6, 1.0);
  }
}

// Inversion and expansion to full nnz x nnz matrices.  Rejection as in
// invert_pixelmatrix_map with allow_decoupling = F and incomplete_matrices = F
// (the reference defaults): pixmode 0 rejects det(C) < pixlim, pixmode 1
// det(C) (3 / trace C)^3 < pixlim, pixmode 2 rcond (smallest over largest
// eigenvalue) < pixlim; a rejected or empty pixel gets a zero matrix.
// nnz = 1: 1 / sum(detw), zero for an empty pixel.
template <int NNZ>
__global__ void k_na_invert(const double *s, long long npix, int pixmode, double pixlim,
                            int *hits, double *cc) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x) {
    const double *c = s + p * kScratchStride;
    hits[p] = (int)c[6];
    if (NNZ == 1) {
      cc[p] = c[0] != 0 ? 1.0 / c[0] : 0.0;
    } else {
      double s6[6];
      for (int j = 0; j < 6; ++j) s6[j] = c[j];
      float crit = 0.0f;
      invert_map_pixel(s6, pixmode, pixlim, false, false, crit);
      double *o = cc + p * 9;
      o[0] = s6[0]; o[1] = s6[1]; o[2] = s6[2];
      o[3] = s6[1]; o[4] = s6[3]; o[5] = s6[4];
      o[6] = s6[2]; o[7] = s6[4]; o[8] = s6[5];
    }
  }
}

int set_err(char *err, long errlen, int status, const char *msg) {
  if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", msg);
  return status;
}

// True when the kernels of this call, running on device `dev`, can read `p`:
// managed memory, or device memory of `dev` itself.  Device memory of another
// GPU is refused even when peer access happens to be enabled, so a call never
// depends on a peer mapping it did not set up.
bool on_device(const void *p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// Loads the code of every kernel this file launches (lazy module loading
// would otherwise do it at the first launch of each), so that after the
// first call on a device no later call loads anything.
cudaError_t resolve_kernels() {
  cudaFuncAttributes fa;
  const void *fns[] = {(const void *)k_na_clear, (const void *)k_na_accum<1>,
                       (const void *)k_na_accum<3>, (const void *)k_na_invert<1>,
                       (const void *)k_na_invert<3>};
  for (const void *f : fns) {
    cudaError_t e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace
}  // namespace madam

extern "C" int madam_b200_pixel_matrices_noalloc(long nside, long nnz, long ndet, long nsamp,
                                                 const double *detweights, const long long *pix,
                                                 const double *pixweights, long pixmode,
                                                 double pixlim, int *hits, double *cc,
                                                 void *stream, char *err, long errlen) {
  using namespace madam;
  if (err && errlen > 0) err[0] = '\0';
  if (nside < 1 || (nside & (nside - 1)) != 0)
    return set_err(err, errlen, 1, "nside must be a power of two");
  const long long npix = 12LL * nside * nside;
  if (npix > kNoAllocMaxPix) {
    char m[160];
    std::snprintf(m, sizeof m,
                  "12*nside^2 = %lld pixels exceeds the fixed scratch of %ld pixels (nside <= 64)",
                  npix, kNoAllocMaxPix);
    return set_err(err, errlen, 1, m);
  }
  if (nnz != 1 && nnz != 3) return set_err(err, errlen, 1, "nnz must be 1 or 3");
  if (ndet < 1 || nsamp < 0) return set_err(err, errlen, 1, "ndet must be >= 1 and nsamp >= 0");
  if (pixmode < 0 || pixmode > 2) return set_err(err, errlen, 1, "pixmode must be 0, 1 or 2");
  // an error left pending by earlier work is the caller's, not this call's:
  // report it without clearing it and launch nothing
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    char m[200];
    std::snprintf(m, sizeof m, "a CUDA error was pending before the call: %s",
                  cudaGetErrorString(e));
    return set_err(err, errlen, 2, m);
  }
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(err, errlen, 2, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_err(err, errlen, 1, "device index out of range");
  const long long ntot = (long long)ndet * nsamp;
  if (!on_device(detweights, dev) || !on_device(hits, dev) || !on_device(cc, dev) ||
      (ntot > 0 && (!on_device(pix, dev) || !on_device(pixweights, dev))))
    return set_err(err, errlen, 1,
                   "all arrays must be in device memory of the current device");
  double *s = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!s) {
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    s = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!s) {
      e = cudaGetSymbolAddress((void **)&s, g_pixmat_scratch);
      if (e == cudaSuccess && s) e = resolve_kernels();
      if (e != cudaSuccess || !s) {
        cudaGetLastError();
        return set_err(err, errlen, 2, e != cudaSuccess ? cudaGetErrorString(e)
                                                        : "scratch address lookup failed");
      }
      g_scratch_ptr[dev].store(s, std::memory_order_release);
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned grid = 148 * 8;
  // each launch is checked on its own, so a status belongs to this call
  k_na_clear<<<grid, 256, 0, st>>>(s, npix * kScratchStride);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return set_err(err, errlen, 2, cudaGetErrorString(e));
  if (ntot > 0) {
    if (nnz == 3)
      k_na_accum<3><<<grid, 256, 0, st>>>(pix, pixweights, detweights, nsamp, ntot, npix, s);
    else
      k_na_accum<1><<<grid, 256, 0, st>>>(pix, pixweights, detweights, nsamp, ntot, npix, s);
    if ((e = cudaGetLastError()) != cudaSuccess)
      return set_err(err, errlen, 2, cudaGetErrorString(e));
  }
  if (nnz == 3)
    k_na_invert<3><<<grid, 128, 0, st>>>(s, npix, (int)pixmode, pixlim, hits, cc);
  else
    k_na_invert<1><<<grid, 128, 0, st>>>(s, npix, (int)pixmode, pixlim, hits, cc);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return set_err(err, errlen, 2, cudaGetErrorString(e));
  return 0;
}
