// C-ABI of libmadam.so.
//
// destripe, destripe_with_cache and clear_caches keep the reference's exact
// signatures (madam.h:1-2; smadam.F90:64-101, 593-609, 921), so a program
// or the ctypes wrapper that loads the reference library can load this one.
// Like the reference, the library keeps module state between calls
// (the Monte-Carlo caches) and is not reentrant: calls are serialised.
// Where the reference calls abort_mpi the replacement returns instead; the
// void entry points print the message on stderr and record it, the
// madam_b200_* entry points return a status and madam_b200_last_error
// gives the message.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <initializer_list>
#include <mutex>
#include <string>

#include "engine.h"
#include "comm.h"
#include "params.h"

using madam::Engine;

namespace madam {

// Where the caller's buffers live: true for device memory that the kernels of
// device `dev` (< 0: the current device) read directly (its own memory, or
// managed memory), false for host memory (pageable or page-locked), which is copied in.  Device
// memory of another GPU, or a mix of host and device buffers, is refused:
// the kernels would read a device buffer in place, and a host buffer taken
// for a device one would be read through an address the GPU cannot use.
bool inputs_on_device(int dev, std::initializer_list<const void *> ptrs) {
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    fail("no CUDA device");
  }
  int kind = -1;
  for (const void *p : ptrs) {
    if (!p) continue;
    int k = 0;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
    } else if (a.type == cudaMemoryTypeManaged) {
      k = 1;
    } else if (a.type == cudaMemoryTypeDevice) {
      if (a.device != dev)
        fail("device buffers must be memory of the CUDA device that runs the solve");
      k = 1;
    }
    if (kind >= 0 && k != kind)
      fail("timestamps, pixels, weights and signal must all be host memory or all "
           "device memory");
    kind = k;
  }
  return kind == 1;
}

}  // namespace madam

namespace {

std::mutex g_mutex;
std::unique_ptr<Engine> g_engine;
std::string g_last_error;
int g_last_status = 0;


template <typename F>
int guarded(F &&f) {
  try {
    f();
    g_last_status = 0;
    g_last_error.clear();
  } catch (const std::exception &e) {
    g_last_status = 1;
    g_last_error = e.what();
  }
  return g_last_status;
}

Engine &engine() {
  if (!g_engine) g_engine.reset(new Engine());
  return *g_engine;
}

void report(const char *who) {
  if (g_last_status != 0) std::fprintf(stderr, "%s: ERROR: %s\n", who, g_last_error.c_str());
}

}  // namespace

extern "C" {

static int destripe_impl(bool fp32, int comm, char *parstring, long ndet, char *detstring,
                         double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                         long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                         long npsdval, double *psdvals);

int madam_b200_destripe(int comm, char *parstring, long ndet, char *detstring,
                        double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                        void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                        long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                        long npsdval, double *psdvals) {
  return destripe_impl(false, comm, parstring, ndet, detstring, detweights, nsamp, nnz,
                       timestamps, pix, pixweights, signal, nperiod, periods, npsd, npsdtot,
                       psdstarts, npsdbin, psdfreqs, npsdval, psdvals);
}

int madam_b200_destripe_fp32(int comm, char *parstring, long ndet, char *detstring,
                             double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                             void *pixweights, float *signal, long nperiod, long *periods,
                             long *npsd, long npsdtot, double *psdstarts, long npsdbin,
                             double *psdfreqs, long npsdval, double *psdvals) {
  return destripe_impl(true, comm, parstring, ndet, detstring, detweights, nsamp, nnz,
                       timestamps, pix, pixweights, signal, nperiod, periods, npsd, npsdtot,
                       psdstarts, npsdbin, psdfreqs, npsdval, psdvals);
}

static int destripe_impl(bool fp32, int comm, char *parstring, long ndet, char *detstring,
                         double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                         long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                         long npsdval, double *psdvals) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    madam::Params par = madam::parse_parstring(parstring);
    if (par.mcmode && g_engine && g_engine->cached())
      madam::fail("Destripe called while caches are not empty.");
    if (par.mcmode && par.nsubchunk > 1) madam::fail("MCMode is not compatible with nsubchunk > 1.");
    if (par.temperature_only && nnz != 1)
      madam::fail("temperature_only=T but pointing weights are polarized");
    if (ndet > 10000) madam::fail("ndet > NDETMAX");
    if (ndet <= 0 || nsamp <= 0 || nnz <= 0) madam::fail("empty data");
    if (nnz != 1 && nnz != 3) madam::fail("only nnz = 1 or nnz = 3 is supported");
    auto dets = madam::read_detectors(par, detstring, ndet, detweights, npsd, npsdtot, psdstarts,
                                      npsdbin, psdfreqs, npsdval, psdvals);
    // a lone rank reads file_spectrum once before any device work, so that
    // a bad file fails fast (build_filter reads it again where the reference
    // does, noise_routines.f90:430-432; sharded ranks wait for that read,
    // which reports its error on every rank after the same collectives)
    madam::Comm *cm = madam::comm_lookup(comm);
    if (par.kfilter && !par.file_spectrum.empty() && (!cm || cm->nranks == 1))
      (void)madam::read_spectrum_file(par.file_spectrum, dets);
    const bool dev = madam::inputs_on_device(-1, {timestamps, pix, pixweights, signal});
    Engine &e = engine();
    e.clear_subchunk_results();
    // comm: a communicator of madam_b200_comm_init_* (a sharded run), else a
    // single rank (the reference's MPI handle has no meaning here)
    e.set_comm(cm);
    // subchunk passes (smadam.F90:192-196): isubchunk = 1 .. nsubchunk, then
    // 0 (the full data) last, starting from the isubchunk parameter
    const int nsub = par.nsubchunk >= 2 ? (int)par.nsubchunk : 0;
    if (nsub && (par.isubchunk < 0 || par.isubchunk > nsub))
      madam::fail("ERROR: isubchunk > nsubchunk");
    // the reference's flag_bad_baselines flags whole baselines from a
    // subchunk's sample count and those flags stay for the later passes;
    // the passes here start from the caller's pointing each time
    if (nsub && par.good_baseline_fraction != 0 && !par.kfilter)
      madam::fail("good_baseline_fraction with nsubchunk > 1 is not supported");
    for (int counter = nsub ? (int)par.isubchunk : 0; counter <= nsub; ++counter) {
      const int isub = nsub ? (counter + 1) % (nsub + 1) : 0;
      e.set_subchunk(isub, nsub);
      e.set_fp32(fp32);
      e.run(par, dets, ndet, nsamp, nnz, (double *)timestamps, (int32_t *)pix,
            (float *)pixweights, (double *)signal, nperiod, periods, dev);
      if (isub > 0) e.keep_subchunk_results(isub);
    }
    e.set_subchunk(0, 0);
  });
}

int madam_b200_destripe_with_cache(int comm, long ndet, long nsamp, long nnz, void *timestamps,
                                   void *pix, void *pixweights, void *signal, char *outpath) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    if (!g_engine || !g_engine->cached())
      madam::fail("destripe_with_cache called with empty caches.");
    // a non-empty outpath replaces path_output for this and later calls
    // (smadam.F90:644-656)
    if (outpath && outpath[0]) {
      std::string s(outpath);
      const size_t a = s.find_first_not_of(' '), b = s.find_last_not_of(' ');
      g_engine->set_output_path(a == std::string::npos ? std::string() : s.substr(a, b - a + 1));
    }
    g_engine->set_comm(madam::comm_lookup(comm));
    const bool dev = madam::inputs_on_device(-1, {timestamps, pix, pixweights, signal});
    g_engine->run_cached(ndet, nsamp, nnz, (double *)timestamps, (int32_t *)pix,
                         (float *)pixweights, (double *)signal, dev);
  });
}

int madam_b200_destripe_with_cache_batch(int comm, long ndet, long nsamp, long nnz,
                                         void *timestamps, void *pix, void *pixweights,
                                         long nrhs, void *signals) {
  (void)comm;
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    if (!g_engine || !g_engine->cached())
      madam::fail("destripe_with_cache called with empty caches.");
    const bool dev = madam::inputs_on_device(-1, {timestamps, pix, pixweights, signals});
    g_engine->run_cached_batch(ndet, nsamp, nnz, (double *)timestamps, (int32_t *)pix,
                               (float *)pixweights, nrhs, (double *)signals, dev);
  });
}

int madam_b200_destripe_with_cache_batch_fp32(int comm, long ndet, long nsamp, long nnz,
                                              void *timestamps, void *pix, void *pixweights,
                                              long nrhs, float *signals) {
  (void)comm;
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    if (!g_engine || !g_engine->cached())
      madam::fail("destripe_with_cache called with empty caches.");
    const bool dev = madam::inputs_on_device(-1, {timestamps, pix, pixweights, signals});
    g_engine->run_cached_batch(ndet, nsamp, nnz, (double *)timestamps, (int32_t *)pix,
                               (float *)pixweights, nrhs, (double *)signals, dev, true);
  });
}

int madam_b200_clear_caches(void) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    const bool had = (bool)g_engine;
    g_engine.reset();
    // the engine's buffers went back to the device's memory pool, which
    // keeps freed memory for the next call; clearing the caches hands it
    // back to the device once those frees (ordered on the legacy stream by
    // the engine's destructor) have run
    if (had) {
      int dev = 0;
      cudaMemPool_t pool;
      if (cudaStreamSynchronize(nullptr) == cudaSuccess && cudaGetDevice(&dev) == cudaSuccess &&
          cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
      cudaGetLastError();
    }
  });
}

void destripe(int comm, char *parstring, long ndet, char *detstring, double *detweights,
              long nsamp, long nnz, void *timestamps, void *pix, void *pixweights, void *signal,
              long nperiod, long *periods, long *npsd, long npsdtot, double *psdstarts,
              long npsdbin, double *psdfreqs, long npsdval, double *psdvals) {
  madam_b200_destripe(comm, parstring, ndet, detstring, detweights, nsamp, nnz, timestamps, pix,
                      pixweights, signal, nperiod, periods, npsd, npsdtot, psdstarts, npsdbin,
                      psdfreqs, npsdval, psdvals);
  report("destripe");
}

void destripe_with_cache(int comm, long ndet, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, char *outpath) {
  madam_b200_destripe_with_cache(comm, ndet, nsamp, nnz, timestamps, pix, pixweights, signal,
                                 outpath);
  report("destripe_with_cache");
}

void clear_caches(void) {
  madam_b200_clear_caches();
}

int madam_b200_last_error(char *buf, long buflen) {
  if (buf && buflen > 0) {
    std::strncpy(buf, g_last_error.c_str(), (size_t)buflen - 1);
    buf[buflen - 1] = '\0';
  }
  return g_last_status;
}

long madam_b200_result_size(const char *name) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_engine || !name) return -1;
  long n = -1;
  guarded([&] { n = g_engine->result_size(name); });
  return n;
}

int madam_b200_result_copy(const char *name, void *dst, long nbytes) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    if (!g_engine) madam::fail("no results: destripe has not run");
    g_engine->result_copy(name, dst, nbytes);
  });
}

int madam_b200_bench_iterations(int warmup, int iters, double *out, long nout) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return guarded([&] {
    if (!g_engine) madam::fail("no solve state: destripe has not run");
    std::vector<double> v;
    g_engine->bench_iterations(warmup, iters, v);
    for (long i = 0; i < nout && i < (long)v.size(); ++i) out[i] = v[i];
  });
}

unsigned long long madam_b200_kernel_launches(void) { return madam::g_kernel_launches.load(); }

// Host-side check of the invariant-divisor division used by the kernels.
int madam_b200_selftest_fastdiv(void) {
  const uint32_t divs[] = {1, 2, 3, 5, 7, 10, 49, 50, 51, 100, 1000, 65535, 65536, 1u << 20,
                           123456789u, 2147483647u, 4294967295u};
  const uint32_t nums[] = {0, 1, 2, 3, 49, 50, 99, 100, 101, 65535, 65536, 1u << 24, 2147483647u,
                           2147483648u, 4000000000u, 4294967295u};
  for (uint32_t d : divs) {
    madam::FastDiv f(d);
    for (uint32_t n : nums)
      if (f.div(n) != n / d) return 1;
    for (uint32_t k = 0; k < 100000; ++k) {
      const uint32_t n = k * 2654435761u;
      if (f.div(n) != n / d) return 1;
    }
  }
  return 0;
}

}  // extern "C"
